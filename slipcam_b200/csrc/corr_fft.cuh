// corr_fft.cuh -- the plain FP32 form: one CTA correlates one (window, frame) pair end to end in
// shared memory (gather, 2-D real FFT, product with the resident reference spectrum, inverse,
// normalization, argmax, sub-pixel peak, SNR and covariance); nothing but the outputs goes back
// to global memory. Mirrors the reference CPU backend's per-window loop (slipcam cxx/cpu.cpp:117-167)
// with its FFTW transforms replaced by our own.
#pragma once

#include <climits>

#include "fft_passes.cuh"
#include "ncc_peak.cuh"

namespace b200 {

// the outputs of a window that could not be correlated (cxx/surface.h:48-54)
B200_HD void invalid_outputs(int64_t q, float *offset, float *peak, float *snr, float *cov)
{
    offset[2 * q] = offset[2 * q + 1] = nanf("");
    peak[q] = snr[q] = 0.0f;
    cov[3 * q] = cov[3 * q + 1] = 99.0f;
    cov[3 * q + 2] = 0.0f;
}

B200_HD double parabola64(double m, double c, double p)
{
    const double den = m - 2 * c + p;
    return den < 0 ? 0.5 * (m - p) / den : 0.0;
}

// The outputs of pair q from its normalized surface around the peak (u, v) -- c points at the
// peak's value, rows `pitch` floats apart; only c's 3 x 3 neighbourhood is read, and only when
// the peak is not on the edge -- following cxx/surface.h:71-146: the 3 x 3 quadratic fit (else a parabola per axis; no
// sub-pixel at the edge), solved in FP64; the SNR from snr_sum, the sum of the squared surface
// over the stat patch clipped to the surface, and its count; the covariance from the curvature.
B200_HD void peak_outputs(const float *c, int pitch, int M, int u, int v, int R, int gy, int gx,
                          int tsize, double snr_sum, int snr_count, int64_t q, float *offset,
                          float *peak, float *snr, float *cov)
{
    const double f0 = c[0];
    const bool inside = u > 0 && u < M - 1 && v > 0 && v < M - 1;
    double du = 0.0, dv = 0.0;
    if (inside) {
        double f[3][3];
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) f[i][j] = c[(i - 1) * pitch + j - 1];
        constexpr double sixth = 1.0 / 6.0;   // the surface.h divisions by 6 and 4, as products
        const double c1 = (f[2][0] + f[2][1] + f[2][2] - f[0][0] - f[0][1] - f[0][2]) * sixth;
        const double c2 = (f[0][2] + f[1][2] + f[2][2] - f[0][0] - f[1][0] - f[2][0]) * sixth;
        const double c3 = (f[0][0] + f[0][1] + f[0][2] + f[2][0] + f[2][1] + f[2][2]
                           - 2 * (f[1][0] + f[1][1] + f[1][2])) * sixth;
        const double c5 = (f[0][0] + f[1][0] + f[2][0] + f[0][2] + f[1][2] + f[2][2]
                           - 2 * (f[0][1] + f[1][1] + f[2][1])) * sixth;
        const double c4 = (f[2][2] - f[2][0] - f[0][2] + f[0][0]) * 0.25;
        const double det = 4 * c3 * c5 - c4 * c4;
        bool fitted = false;
        if (c3 < 0 && det > 0) {
            const double rdet = 1.0 / det;
            du = (c4 * c2 - 2 * c5 * c1) * rdet;
            dv = (c4 * c1 - 2 * c3 * c2) * rdet;
            fitted = fabs(du) <= 1 && fabs(dv) <= 1;
        }
        if (!fitted) {
            du = parabola64(f[0][1], f[1][1], f[2][1]);
            dv = parabola64(f[1][0], f[1][1], f[1][2]);
        }
    }
    offset[2 * q] = float(double(gy + u - R) + du);
    offset[2 * q + 1] = float(double(gx + v - R) + dv);
    peak[q] = float(f0);
    const double mean = snr_count > 1 ? (snr_sum - f0 * f0) / (snr_count - 1) : 0.0;
    snr[q] = mean > 0 ? float(f0 * f0 / mean) : 0.0f;
    cov[3 * q] = cov[3 * q + 1] = 99.0f;
    cov[3 * q + 2] = 0.0f;
    if (inside) {
        const double T = tsize;
        const double dxx = -(c[pitch] + c[-pitch] - 2.0 * f0) * T;
        const double dyy = -(c[1] + c[-1] - 2.0 * f0) * T;
        const double dxy = (double(c[pitch + 1]) + c[-pitch - 1] - c[pitch - 1] - c[-pitch + 1]) * 0.25 * T;
        double n2 = 1.0 - f0 > 0 ? 1.0 - f0 : 0.0;
        const double n4 = n2 * n2 * 0.5 * T;
        n2 *= 2;
        const double w = dxy * dxy - dxx * dyy;
        if (fabs(w) >= 1e-2) {
            const double rw2 = 1.0 / (w * w);
            cov[3 * q] = float((-n2 * w * dyy + n4 * (dyy * dyy + dxy * dxy)) * rw2);
            cov[3 * q + 1] = float((-n2 * w * dxx + n4 * (dxx * dxx + dxy * dxy)) * rw2);
            cov[3 * q + 2] = float((n2 * w * dxy - n4 * (dxx + dyy) * dxy) * rw2);
        }
    }
}

// the rows and the columns of the stat x stat SNR patch around (u, v) inside an M x M surface
B200_HD void snr_patch(int M, int stat, int u, int v, int &i0, int &i1, int &j0, int &j1)
{
    const int n = stat < M ? stat : M;
    i0 = u - n / 2; i1 = i0 + n;
    j0 = v - n / 2; j1 = j0 + n;
    i0 = i0 < 0 ? 0 : i0; j0 = j0 < 0 ? 0 : j0;
    i1 = i1 > M ? M : i1; j1 = j1 > M ? M : j1;
}

// the better of two surface candidates: the larger, the first in raster order if equal
B200_HD void better(float &best, int &at, float b, int ib)
{
    if (b > best || (b == best && ib < at)) {
        best = b;
        at = ib;
    }
}

#ifdef __CUDACC__

// The peak of pair q's normalized M x M surface Sr (row pitch `pitch` floats) and its outputs: the
// largest value, the first in raster order if equal (cxx/cpu.cpp:148-160), invalid unless it is
// positive; then the SNR patch sum (warp 0) and peak_outputs. peak_at (optional) receives the
// peak's raster index u M + v, or -1. Every thread of the block calls it (it holds a barrier).
template <int NT>
__device__ __forceinline__ void surface_peak(const float *Sr, int pitch, int M, int R, int stat, int gy, int gx,
                                             int tsize, int64_t q, float *offset, float *peak, float *snr, float *cov,
                                             int *peak_at)
{
    __shared__ float s_best[NT / 32];
    __shared__ int s_at[NT / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float best = -2.0f;
    int at = INT_MAX;
    for (int idx = threadIdx.x; idx < M * M; idx += NT) {
        const float c = Sr[size_t(idx / M) * pitch + idx % M];
        if (c > best) {
            best = c;
            at = idx;
        }
    }
    for (int o = 16; o > 0; o >>= 1) better(best, at, __shfl_xor_sync(0xffffffffu, best, o), __shfl_xor_sync(0xffffffffu, at, o));
    if (lane == 0) {
        s_best[warp] = best;
        s_at[warp] = at;
    }
    __syncthreads();
    if (warp != 0) return;
    best = lane < NT / 32 ? s_best[lane] : -2.0f;
    at = lane < NT / 32 ? s_at[lane] : INT_MAX;
    for (int o = 16; o > 0; o >>= 1) better(best, at, __shfl_xor_sync(0xffffffffu, best, o), __shfl_xor_sync(0xffffffffu, at, o));
    if (!(best > 0)) {
        if (lane == 0) {
            invalid_outputs(q, offset, peak, snr, cov);
            if (peak_at) peak_at[q] = -1;
        }
        return;
    }
    const int u = at / M, v = at % M;
    int i0, i1, j0, j1;
    snr_patch(M, stat, u, v, i0, i1, j0, j1);
    const int pw = j1 - j0, cnt = (i1 - i0) * pw;
    double sum = 0.0;
    for (int t = lane; t < cnt; t += 32) {
        const double c = Sr[size_t(i0 + t / pw) * pitch + j0 + t % pw];
        sum += c * c;
    }
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (lane == 0) {
        peak_outputs(Sr + size_t(u) * pitch + v, pitch, M, u, v, R, gy, gx, tsize, sum, cnt, q, offset, peak, snr, cov);
        if (peak_at) peak_at[q] = at;
    }
}

// the reference spectra: one CTA per reference window. Zero-mean window (its mean in double as
// cxx/common.cpp:30-48), its norm, and its N x N forward spectrum into spec[k].
template <int N, int NT>
__global__ void __launch_bounds__(NT) spectra_kernel(SpectraArgs a)
{
    using G = Geo<N>;
    extern __shared__ float4 smem_raw[];
    float2 *S = reinterpret_cast<float2 *>(smem_raw);
    float2 *TW = S + size_t(N) * G::NHP, *TWI = TW + N;
    float *Sr = reinterpret_cast<float *>(S);
    __shared__ double red[NT / 32];
    __shared__ long long redi[NT / 32];
    const int k = blockIdx.x, W = a.W;
    const int y0 = a.down[k / a.nx], x0 = a.across[k % a.nx];
    const uint8_t *src = a.frame + size_t(y0) * a.pitch + x0;
    const float *srcf = a.framef ? a.framef + size_t(y0) * a.pitch + x0 : nullptr;
    auto pixel = [&](int i, int j) { return srcf ? double(srcf[size_t(i) * a.pitch + j]) : double(src[size_t(i) * a.pitch + j]); };
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

    for (int i = threadIdx.x; i < 2 * N; i += NT) TW[i] = a.twiddles[i];
    // the sum of the window (exact, integers; in double for a float frame)
    double mean;
    if (!srcf) {
        long long sum = 0;
        for (int idx = threadIdx.x; idx < W * W; idx += NT) sum += src[size_t(idx / W) * a.pitch + idx % W];
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        if (lane == 0) redi[warp] = sum;
        __syncthreads();
        sum = 0;
        for (int i = 0; i < NT / 32; ++i) sum += redi[i];
        mean = double(sum) / (double(W) * W);
    } else {
        double sum = 0.0;
        for (int idx = threadIdx.x; idx < W * W; idx += NT) sum += pixel(idx / W, idx % W);
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        if (lane == 0) red[warp] = sum;
        __syncthreads();
        sum = 0.0;
        for (int i = 0; i < NT / 32; ++i) sum += red[i];
        __syncthreads();
        mean = sum / (double(W) * W);
    }
    // the zero-mean window, zero-padded (rows up to the even count Wr, all N columns)
    const int Wr = (W + 1) & ~1;
    double sq = 0.0;
    for (int idx = threadIdx.x; idx < Wr * N; idx += NT) {
        const int i = idx / N, j = idx % N;
        float d = 0.0f;
        if (i < W && j < W) {
            d = float(pixel(i, j) - mean);
            sq += double(d) * d;
        }
        Sr[size_t(i) * G::RP + j] = d;
    }
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
    if (lane == 0) red[warp] = sq;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < NT / 32; ++i) t += red[i];
        a.norm[k] = float(sqrt(t));
    }
    const DevExec ex{warp, NT / 32};
    row_forward<N>(ex, S, Wr / 2, TW);
    __syncthreads();
    col_pass<N, false>(ex, S, Wr, 0, TW, TWI, nullptr, a.spec + size_t(k) * G::NH * N);
}

// one (window k, frame f) pair: the correlation, normalized, and its outputs, in the shared-memory
// tile S (Geo<N>::smem_bytes). Every thread of the block calls it; warp 0 may still be writing the
// pair's outputs when the others return, so a caller that reuses S syncs first.
template <int N, int NT>
__device__ __forceinline__ void corr_pair(const CorrArgs &a, int k, int f, float2 *S)
{
    using G = Geo<N>;
    float2 *TW = S + size_t(N) * G::NHP, *TWI = TW + N;
    float *Sr = reinterpret_cast<float *>(S);
    const int64_t q = int64_t(f) * a.nwin + k;
    const int warp = threadIdx.x >> 5;

    int gy = 0, gx = 0;
    if (a.gross_mode == 1) {
        gy = a.gross[2 * f];
        gx = a.gross[2 * f + 1];
    } else if (a.gross_mode == 2) {
        gy = a.gross[2 * q];
        gx = a.gross[2 * q + 1];
    }
    const int L = a.L, M = a.M, R = a.R;
    const int sy = a.down[k / a.nx] + gy - R, sx = a.across[k % a.nx] + gx - R;
    const float norm = a.norm[k];
    // the reference's validity (cxx/cpu.cpp:121-125 with cxx/surface.h:39-45)
    if (!(norm > 0) || sy < 0 || sx < 0 || sy + L > a.h || sx + L > a.w) {
        if (threadIdx.x == 0) invalid_outputs(q, a.offset, a.peak, a.snr, a.cov);
        if (a.ncc && threadIdx.x == 0) {
            a.ncc[3 * q] = a.ncc[3 * q + 1] = NAN;
            a.ncc[3 * q + 2] = -INFINITY;
        }
        if (a.surface)
            for (int i = threadIdx.x; i < M * M; i += NT) a.surface[q * M * M + i] = 0.0f;
        return;
    }
    for (int i = threadIdx.x; i < 2 * N; i += NT) TW[i] = a.twiddles[i];

    // the search window minus its mean, float(box sum) / (L L) as cxx/cpu.cpp:132 (the box sum
    // from the 32-bit table is exact: it is below 2^32 and the table wraps modulo 2^32)
    const uint32_t *sat = a.sat + size_t(f) * a.sat_fstride;
    const size_t ss = size_t(a.w) + 1;
    const uint32_t box = sat[(sy + L) * ss + sx + L] - sat[sy * ss + sx + L] - sat[(sy + L) * ss + sx]
        + sat[sy * ss + sx];
    const float mean = float(box) / (float(L) * float(L));
    const int Lr = (L + 1) & ~1;
    const uint8_t *frame = a.frames + f * a.fstride;
    int off = 0;
    if (((a.pitch | reinterpret_cast<uintptr_t>(frame)) & 3) == 0) {
        // 4-byte words: row i of the chip lands at float column off + j (off = sx mod 4), so every
        // word, aligned in global memory, is one aligned float4 in shared memory
        off = sx & 3;
        constexpr int NW = N / 4 + 1;   // RP = N + 4 floats = NW words per row
        const uint32_t *src = reinterpret_cast<const uint32_t *>(frame + int64_t(sy) * a.pitch + (sx - off));
        const int pw = a.pitch >> 2;
#pragma unroll 4
        for (int idx = threadIdx.x; idx < Lr * NW; idx += NT) {
            const int i = idx / NW, w = idx % NW, c0 = 4 * w - off;
            // a word with a pixel of the chip lies inside the frame row (pitch >= width rounded up to 4)
            const uint32_t word = (i < L && c0 < L) ? __ldg(src + size_t(i) * pw + w) : 0u;
            float4 v;
            v.x = (i < L && c0 >= 0 && c0 < L) ? float(word & 255u) - mean : 0.0f;
            v.y = (i < L && c0 + 1 >= 0 && c0 + 1 < L) ? float((word >> 8) & 255u) - mean : 0.0f;
            v.z = (i < L && c0 + 2 >= 0 && c0 + 2 < L) ? float((word >> 16) & 255u) - mean : 0.0f;
            v.w = (i < L && c0 + 3 < L) ? float(word >> 24) - mean : 0.0f;
            *reinterpret_cast<float4 *>(Sr + size_t(i) * G::RP + 4 * w) = v;
        }
    } else {
        const uint8_t *src = frame + int64_t(sy) * a.pitch + sx;
#pragma unroll 4
        for (int idx = threadIdx.x; idx < Lr * N; idx += NT) {
            const int i = idx / N, j = idx % N;
            Sr[size_t(i) * G::RP + j] = (i < L && j < L) ? float(__ldg(src + size_t(i) * a.pitch + j)) - mean : 0.0f;
        }
    }
    __syncthreads();

    const DevExec ex{warp, NT / 32};
    row_forward<N>(ex, S, Lr / 2, TW, off);
    __syncthreads();
    col_pass<N, true>(ex, S, Lr, M, TW, TWI, a.spec + size_t(k) * G::NH * N, nullptr);
    __syncthreads();

    // back to rows, normalized: rho = c / (N^2) / (norm sqrt(n var)), the variance term from the
    // precomputed table of the frame (0 where the search box is flat)
    const float inv = 1.0f / (float(N) * float(N) * norm);
    const float *dinv = a.dinv + size_t(f) * a.dinv_fstride + size_t(sy) * a.dpitch + sx;
    const int dw = a.dpitch;
    row_inverse<N>(ex, S, M, TWI, [&](int u, int c, float x) { return x * inv * __ldg(dinv + size_t(u) * dw + c); });
    __syncthreads();
    if (a.surface)
        for (int i = threadIdx.x; i < M * M; i += NT) a.surface[q * M * M + i] = Sr[size_t(i / M) * G::RP + i % M];
    if (a.ncc) ncc_peak_block<NT>(Sr, G::RP, M, a.ncc + 3 * q);

    surface_peak<NT>(Sr, G::RP, M, R, a.stat, gy, gx, a.W * a.W, q, a.offset, a.peak, a.snr, a.cov, nullptr);
}

// the correlation of one (window, frame) pair per CTA; blockIdx.x = window * nf + frame, so the
// CTAs of one window (one reference spectrum) run together and share it through L2
template <int N, int NT>
__global__ void __launch_bounds__(NT, (N <= 160 ? 2 : 1)) corr_kernel(CorrArgs a)
{
    extern __shared__ float4 smem_raw[];
    corr_pair<N, NT>(a, blockIdx.x / a.nf, blockIdx.x % a.nf, reinterpret_cast<float2 *>(smem_raw));
}

// one frame's pairs when their latency is what counts (a frame chain where each frame waits for the
// one before, a grid of a few dozen windows leaving most SMs idle): corr_kernel's work with NT
// threads per pair and one CTA per SM allowed the registers of the larger block
template <int N, int NT>
__global__ void __launch_bounds__(NT, 1) corr_latency_kernel(CorrArgs a)
{
    extern __shared__ float4 smem_raw[];
    corr_pair<N, NT>(a, blockIdx.x / a.nf, blockIdx.x % a.nf, reinterpret_cast<float2 *>(smem_raw));
}

#endif   // __CUDACC__

}   // namespace b200
