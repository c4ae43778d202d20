// corr_big.cuh -- the FP32 FFT correlation for transforms whose N x (N/2 + 1) half spectrum does
// not fit in one CTA's shared memory (N = 256: 264 KB): window 128 with search 64 (L = 256).
//
// The passes of fft_passes.cuh run on pieces of the spectrum, staged through a per-CTA scratch
// in global memory (it stays in L2: 148 CTAs x 397 KB = 59 MB):
//   1. row pass in chunks of 32 rows: chip rows -> shared memory -> row_forward -> the rows' half
//      spectra to the scratch (Lr x NH)
//   2. column pass in two halves of the NH columns: a half (N rows x <= 65 columns) -> shared
//      memory -> col_pass (forward, x conj(reference spectrum), inverse, rows [0, M) kept) -> the
//      scratch (M x NH)
//   3. the M rows back in shared memory -> row_inverse (normalized) -> the surface -> the
//      reference's peak epilogue
// The reference spectra are made the same way (col_pass writing them out). Persistent CTAs,
// one per SM (139 KB of shared memory), walk the (window, frame) pairs.
#pragma once

#include "corr_fft.cuh"

namespace b200 {

template <int N>
struct BigGeo {
    using G = Geo<N>;
    static constexpr int NH = G::NH, NHP = G::NHP, RP = G::RP;
    static constexpr int H0 = (NH + 1) / 2;                     // columns of the first half
    static constexpr int WS = H0 + 1;                           // their stride in shared memory
    static constexpr int CHUNK = 32;                            // rows per row-pass chunk
    static constexpr size_t work_bytes = size_t(N) * WS * sizeof(float2);
    static constexpr size_t smem_bytes = work_bytes + 2 * N * sizeof(float2);
    // the inverse row pass on M rows uses complex rows up to (M rounded up to even - 2) plus an
    // N-value exchange row pair: it must stay inside the work area
    static constexpr bool fits_M(int M) { return size_t((M + 1) / 2 * 2 - 2) * NHP + N <= size_t(N) * WS; }
    static_assert(size_t(CHUNK) * RP * sizeof(float) <= work_bytes, "row chunk");
    // per-CTA scratch, in complex values: Lr x NH row spectra, then M x NH column results
    static constexpr size_t scratch(int Lr, int M) { return size_t(Lr) * NH + size_t(M) * NH; }
};

#ifdef __CUDACC__

// the half spectra of rows [0, Lr) of a real L x L block into gs (row-major, NH per row);
// row(i, j) gives element j of row i (j < L, i < L), 0 outside
template <int N, int NT, class Row>
__device__ void big_rows(float2 *W, const float2 *TW, int Lr, int L, float2 *gs, Row &&row)
{
    using B = BigGeo<N>;
    const DevExec ex{int(threadIdx.x >> 5), NT / 32};
    float *Sr = reinterpret_cast<float *>(W);
    for (int r0 = 0; r0 < Lr; r0 += B::CHUNK) {
        const int rows = min(B::CHUNK, Lr - r0);
#pragma unroll 8
        for (int idx = threadIdx.x; idx < rows * N; idx += NT) {
            const int i = idx / N, j = idx % N;
            Sr[size_t(i) * B::RP + j] = (r0 + i < L && j < L) ? row(r0 + i, j) : 0.0f;
        }
        __syncthreads();
        row_forward<N>(ex, W, rows / 2, TW);
        __syncthreads();
#pragma unroll 4
        for (int idx = threadIdx.x; idx < rows * B::NH; idx += NT) {
            const int i = idx / B::NH, k = idx % B::NH;
            gs[size_t(r0 + i) * B::NH + k] = W[size_t(i) * B::NHP + k];
        }
        __syncthreads();
    }
}

// the column pass over both halves of the columns: CORR (spec given) keeps rows [0, M) of the
// inverse transforms in gm (M x NH); otherwise the forward spectra go to out (corr_fft.cuh order)
template <int N, int NT, bool CORR>
__device__ void big_cols(float2 *W, const float2 *TW, const float2 *TWI, int Lr, int M, const float2 *gs,
                         const float2 *spec, float2 *out, float2 *gm)
{
    using B = BigGeo<N>;
    const DevExec ex{int(threadIdx.x >> 5), NT / 32};
    for (int h = 0; h < 2; ++h) {
        const int k0 = h ? B::H0 : 0, nc = h ? B::NH - B::H0 : B::H0;
#pragma unroll 8
        for (int idx = threadIdx.x; idx < Lr * nc; idx += NT) {
            const int r = idx / nc, c = idx % nc;
            W[size_t(r) * B::WS + c] = gs[size_t(r) * B::NH + k0 + c];
        }
        __syncthreads();
        if constexpr (CORR) {
            col_pass<N, true>(ex, W, Lr, M, TW, TWI, spec + size_t(k0) * N, nullptr, nc, B::WS);
        } else {
            col_pass<N, false>(ex, W, Lr, 0, TW, TWI, nullptr, out + size_t(k0) * N, nc, B::WS);
        }
        __syncthreads();
        if constexpr (CORR) {
            for (int idx = threadIdx.x; idx < M * nc; idx += NT) {
                const int u = idx / nc, c = idx % nc;
                gm[size_t(u) * B::NH + k0 + c] = W[size_t(u) * B::WS + c];
            }
            __syncthreads();
        }
    }
}

// one reference window: its mean and norm in double (cxx/common.cpp:30-48), its spectrum
template <int N, int NT>
__device__ void big_window(const SpectraArgs &a, int k, float2 *W, const float2 *TW, const float2 *TWI, float2 *gs)
{
    using B = BigGeo<N>;
    __shared__ double red[NT / 32];
    const int Wd = a.W;
    const int y0 = a.down[k / a.nx], x0 = a.across[k % a.nx];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    auto pixel = [&](int i, int j) {
        const size_t o = size_t(y0 + i) * a.pitch + x0 + j;
        return a.framef ? double(a.framef[o]) : double(a.frame[o]);
    };
    // the window's mean and norm in double (cxx/common.cpp:30-48)
    double sum = 0.0;
    for (int idx = threadIdx.x; idx < Wd * Wd; idx += NT) sum += pixel(idx / Wd, idx % Wd);
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (lane == 0) red[warp] = sum;
    __syncthreads();
    sum = 0.0;
    for (int i = 0; i < NT / 32; ++i) sum += red[i];
    __syncthreads();
    const double mean = sum / (double(Wd) * Wd);
    double sq = 0.0;
    for (int idx = threadIdx.x; idx < Wd * Wd; idx += NT) {
        const double d = double(float(pixel(idx / Wd, idx % Wd) - mean));
        sq += d * d;
    }
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
    if (lane == 0) red[warp] = sq;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < NT / 32; ++i) t += red[i];
        a.norm[k] = float(sqrt(t));
    }
    __syncthreads();
    const int Wr = (Wd + 1) & ~1;
    big_rows<N, NT>(W, TW, Wr, Wd, gs, [&](int i, int j) { return float(pixel(i, j) - mean); });
    big_cols<N, NT, false>(W, TW, TWI, Wr, 0, gs, nullptr, a.spec + size_t(k) * B::NH * N, nullptr);
}

// the reference spectra of the big transform: persistent CTAs over the windows, scratch per CTA
template <int N, int NT>
__global__ void __launch_bounds__(NT, 1) spectra_big_kernel(SpectraArgs a, int nwin, float2 *scratch, size_t per_cta)
{
    using B = BigGeo<N>;
    extern __shared__ float4 smem_raw[];
    float2 *W = reinterpret_cast<float2 *>(smem_raw);
    float2 *TW = W + B::work_bytes / sizeof(float2), *TWI = TW + N;
    float2 *gs = scratch + size_t(blockIdx.x) * per_cta;
    for (int i = threadIdx.x; i < 2 * N; i += NT) TW[i] = a.twiddles[i];
    __syncthreads();
    for (int k = blockIdx.x; k < nwin; k += gridDim.x) big_window<N, NT>(a, k, W, TW, TWI, gs);
}

// one (window, frame) pair p of the big transform in the work area W (BigGeo<N>::smem_bytes,
// twiddles included) with this CTA's scratch gs. Every thread of the block calls it and it ends
// with a barrier (the next pair may reuse W at once).
template <int N, int NT>
__device__ void corr_big_pair(const CorrArgs &a, int p, float2 *W, float2 *gs)
{
    using B = BigGeo<N>;
    float2 *TW = W + B::work_bytes / sizeof(float2), *TWI = TW + N;
    float *Sr = reinterpret_cast<float *>(W);
    const int L = a.L, M = a.M, R = a.R;
    const int Lr = (L + 1) & ~1;
    float2 *gm = gs + size_t(Lr) * B::NH;
    const int k = p / a.nf, f = p % a.nf;
    const int64_t q = int64_t(f) * a.nwin + k;
    int gy = 0, gx = 0;
    if (a.gross_mode == 1) {
        gy = a.gross[2 * f];
        gx = a.gross[2 * f + 1];
    } else if (a.gross_mode == 2) {
        gy = a.gross[2 * q];
        gx = a.gross[2 * q + 1];
    }
    const int sy = a.down[k / a.nx] + gy - R, sx = a.across[k % a.nx] + gx - R;
    const float norm = a.norm[k];
    if (!(norm > 0) || sy < 0 || sx < 0 || sy + L > a.h || sx + L > a.w) {   // cxx/surface.h:39-45
        if (threadIdx.x == 0) invalid_outputs(q, a.offset, a.peak, a.snr, a.cov);
        if (a.surface)
            for (int i = threadIdx.x; i < M * M; i += NT) a.surface[q * M * M + i] = 0.0f;
        return;
    }
    for (int i = threadIdx.x; i < 2 * N; i += NT) TW[i] = a.twiddles[i];
    // the chip minus its mean, float(box sum) / (L L) as cxx/cpu.cpp:132
    const uint32_t *sat = a.sat + size_t(f) * a.sat_fstride;
    const size_t ss = size_t(a.w) + 1;
    const uint32_t box = sat[(sy + L) * ss + sx + L] - sat[sy * ss + sx + L] - sat[(sy + L) * ss + sx] + sat[sy * ss + sx];
    const float mean = float(box) / (float(L) * float(L));
    const uint8_t *chip = a.frames + f * a.fstride + int64_t(sy) * a.pitch + sx;
    big_rows<N, NT>(W, TW, Lr, L, gs, [&](int i, int j) { return float(__ldg(chip + int64_t(i) * a.pitch + j)) - mean; });
    big_cols<N, NT, true>(W, TW, TWI, Lr, M, gs, a.spec + size_t(k) * B::NH * N, nullptr, gm);
    // rows [0, M) of the column-inverted spectrum, whole again, then the inverse row pass
#pragma unroll 8
    for (int idx = threadIdx.x; idx < M * B::NH; idx += NT) {
        const int u = idx / B::NH, c = idx % B::NH;
        W[size_t(u) * B::NHP + c] = gm[size_t(u) * B::NH + c];
    }
    __syncthreads();
    const float inv = 1.0f / (float(N) * float(N) * norm);
    const float *dinv = a.dinv + size_t(f) * a.dinv_fstride + size_t(sy) * a.dpitch + sx;
    const int dw = a.dpitch;
    const DevExec ex{int(threadIdx.x >> 5), NT / 32};
    row_inverse<N>(ex, W, M, TWI, [&](int u, int c, float x) { return x * inv * __ldg(dinv + size_t(u) * dw + c); });
    __syncthreads();
    if (a.surface)
        for (int i = threadIdx.x; i < M * M; i += NT) a.surface[q * M * M + i] = Sr[size_t(i / M) * B::RP + i % M];
    surface_peak<NT>(Sr, B::RP, M, R, a.stat, gy, gx, a.W * a.W, q, a.offset, a.peak, a.snr, a.cov, nullptr);
    __syncthreads();
}

// the correlation of the big transform: persistent CTAs over the pairs of the group, scratch per CTA
template <int N, int NT>
__global__ void __launch_bounds__(NT, 1) corr_big_kernel(CorrArgs a, float2 *scratch, size_t per_cta)
{
    extern __shared__ float4 smem_raw[];
    float2 *W = reinterpret_cast<float2 *>(smem_raw);
    float2 *gs = scratch + size_t(blockIdx.x) * per_cta;
    const int npairs = a.nwin * a.nf;
    for (int p = blockIdx.x; p < npairs; p += gridDim.x) {
        corr_big_pair<N, NT>(a, p, W, gs);
        __syncthreads();
    }
}

#endif   // __CUDACC__

}   // namespace b200
