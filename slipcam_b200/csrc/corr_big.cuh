// corr_big.cuh -- the FP32 FFT correlation for transforms whose N x (N/2 + 1) half spectrum does
// not fit in one CTA's shared memory (N = 256: 264 KB): window 128 with search 64 (L = 256).
//
// One CTA per pair (the reference spectra, and the pairs of the multi-grid persistent launch): the
// passes of fft_passes.cuh run on pieces of the spectrum, staged through a per-CTA scratch in
// global memory (it stays in L2: 148 CTAs x 397 KB = 59 MB):
//   1. row pass in chunks of 32 rows: chip rows -> shared memory -> row_forward -> the rows' half
//      spectra to the scratch (Lr x NH)
//   2. column pass in two halves of the NH columns: a half (N rows x <= 65 columns) -> shared
//      memory -> col_pass (forward, x conj(reference spectrum), inverse, rows [0, M) kept) -> the
//      scratch (M x NH)
//   3. the M rows back in shared memory -> row_inverse (normalized) -> the surface -> the
//      reference's peak epilogue
// The reference spectra are made the same way (col_pass writing them out). Persistent CTAs,
// one per SM (139 KB of shared memory), walk the windows or pairs. A Correlator's own launches use
// the two-CTA cluster form below instead (no staging through global memory).
#pragma once

#ifdef __CUDACC__
#include <cooperative_groups.h>
#endif

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

#endif   // __CUDACC__

// The same correlation on a cluster of two CTAs (two SMs) whose shared memories hold the whole
// half spectrum between them, so nothing is staged through global memory: CTA r owns the columns
// [0, H0) (r = 0) or [H0, NH) (r = 1) as an N x WS tile, plus a staging area for row work.
//   1. each CTA transforms half of the chip's rows (chunks of 32) and scatters each row's half
//      spectrum: its own columns to its tile, the others to the partner's tile (distributed shared
//      memory stores);
//   2. each CTA runs the column pass (forward, x conj(reference spectrum), inverse) on its columns;
//   3. each CTA gathers half of the M output rows from both tiles and runs the inverse row pass
//      with the normalization;
//   4. both write their surface rows into CTA 0's tile, which runs the reference's peak epilogue.
// Cluster barriers separate the phases (five per pair). Both CTAs walk the same pairs and take the
// same validity decision, so they always meet the same barriers.
template <int N>
struct BigClusterGeo {
    using B = BigGeo<N>;
    static constexpr int MH_MAX = 66;   // surface rows of one CTA (M <= 129: fits_M)
    static constexpr size_t tile_elems = size_t(N) * B::WS;
    // the staging area: a chunk of real rows (row pass), MH_MAX gathered rows of NHP values, and
    // the inverse row pass's own reach on them (rows up to MH_MAX rounded up to even - 2, plus N)
    static constexpr size_t row_elems = size_t(B::CHUNK) * B::RP / 2;
    static constexpr size_t gather_elems = size_t(MH_MAX) * B::NHP;
    static constexpr size_t inv_elems = size_t((MH_MAX + 1) / 2 * 2 - 2) * B::NHP + N;
    static constexpr size_t stage_elems = gather_elems > inv_elems ? (gather_elems > row_elems ? gather_elems : row_elems)
                                                                   : (inv_elems > row_elems ? inv_elems : row_elems);
    static constexpr size_t smem_bytes = (tile_elems + stage_elems + 2 * size_t(N)) * sizeof(float2);
    static_assert(size_t(129) * B::RP <= 2 * tile_elems, "the assembled surface fits the tile");
};

#ifdef __CUDACC__

template <int N, int NT>
__device__ void corr_big_cluster_pair(const CorrArgs &a, int p, int rank, float2 *const *tiles, float2 *stage,
                                      const float2 *TW, const float2 *TWI, cooperative_groups::cluster_group &cluster)
{
    using B = BigGeo<N>;
    const int L = a.L, M = a.M, R = a.R;
    const int Lr = (L + 1) & ~1;
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
        if (rank == 0) {
            if (threadIdx.x == 0) invalid_outputs(q, a.offset, a.peak, a.snr, a.cov);
            if (a.surface)
                for (int i = threadIdx.x; i < M * M; i += NT) a.surface[q * M * M + i] = 0.0f;
        }
        return;   // both CTAs: no cluster barrier for this pair
    }
    const uint32_t *sat = a.sat + size_t(f) * a.sat_fstride;
    const size_t ss = size_t(a.w) + 1;
    const uint32_t box = sat[(sy + L) * ss + sx + L] - sat[sy * ss + sx + L] - sat[(sy + L) * ss + sx] + sat[sy * ss + sx];
    const float mean = float(box) / (float(L) * float(L));
    const uint8_t *chip = a.frames + f * a.fstride + int64_t(sy) * a.pitch + sx;
    const DevExec ex{int(threadIdx.x >> 5), NT / 32};
    float *Sr = reinterpret_cast<float *>(stage);

    // 1. this CTA's rows of the chip, their half spectra scattered over the two tiles
    const int rs = ((Lr / 2) + 1) & ~1;
    const int r_lo = rank ? rs : 0, r_hi = rank ? Lr : rs;
    for (int r0 = r_lo; r0 < r_hi; r0 += B::CHUNK) {
        const int rows = min(B::CHUNK, r_hi - r0);
#pragma unroll 8
        for (int idx = threadIdx.x; idx < rows * N; idx += NT) {
            const int i = idx / N, j = idx % N;
            Sr[size_t(i) * B::RP + j] = (r0 + i < L && j < L) ? float(__ldg(chip + int64_t(r0 + i) * a.pitch + j)) - mean : 0.0f;
        }
        __syncthreads();
        row_forward<N>(ex, stage, rows / 2, TW);
        __syncthreads();
#pragma unroll 4
        for (int idx = threadIdx.x; idx < rows * B::NH; idx += NT) {
            const int i = idx / B::NH, c = idx % B::NH;
            float2 *dst = c < B::H0 ? tiles[0] + size_t(r0 + i) * B::WS + c : tiles[1] + size_t(r0 + i) * B::WS + (c - B::H0);
            *dst = stage[size_t(i) * B::NHP + c];
        }
        __syncthreads();
    }
    cluster.sync();

    // 2. the column pass over this CTA's columns
    const int k0 = rank ? B::H0 : 0, nc = rank ? B::NH - B::H0 : B::H0;
    col_pass<N, true>(ex, tiles[rank], Lr, M, TW, TWI, a.spec + size_t(k) * B::NH * N + size_t(k0) * N, nullptr, nc, B::WS);
    __syncthreads();
    cluster.sync();

    // 3. this CTA's rows [u_lo, u_hi) of the surface: the rows of both tiles, the inverse row pass
    const int us = ((M + 1) / 2 + 1) & ~1;
    const int u_lo = rank ? min(us, M) : 0, u_hi = rank ? M : min(us, M), mh = u_hi - u_lo;   // mh <= MH_MAX (M <= 129)
#pragma unroll 4
    for (int idx = threadIdx.x; idx < mh * B::NH; idx += NT) {
        const int u = idx / B::NH, c = idx % B::NH;
        stage[size_t(u) * B::NHP + c] = c < B::H0 ? tiles[0][size_t(u_lo + u) * B::WS + c]
                                                  : tiles[1][size_t(u_lo + u) * B::WS + (c - B::H0)];
    }
    __syncthreads();
    const float inv = 1.0f / (float(N) * float(N) * norm);
    const float *dinv = a.dinv + size_t(f) * a.dinv_fstride + size_t(sy + u_lo) * a.dpitch + sx;
    const int dw = a.dpitch;
    if (mh > 0)
        row_inverse<N>(ex, stage, mh, TWI, [&](int u, int c, float x) { return x * inv * __ldg(dinv + size_t(u) * dw + c); },
                       M);
    __syncthreads();
    cluster.sync();   // no CTA reads a tile any more

    // 4. the surface rows into CTA 0's tile (pitch RP floats), its epilogue
    float *surf = reinterpret_cast<float *>(tiles[0]);
    for (int idx = threadIdx.x; idx < mh * M; idx += NT) {
        const int u = idx / M, v = idx % M;
        surf[size_t(u_lo + u) * B::RP + v] = Sr[size_t(u) * B::RP + v];
    }
    cluster.sync();
    if (rank == 0) {
        if (a.surface)
            for (int i = threadIdx.x; i < M * M; i += NT) a.surface[q * M * M + i] = surf[size_t(i / M) * B::RP + i % M];
        surface_peak<NT>(surf, B::RP, M, R, a.stat, gy, gx, a.W * a.W, q, a.offset, a.peak, a.snr, a.cov, nullptr);
    }
    __syncthreads();
    cluster.sync();   // CTA 0's tile is free for the next pair
}

// the correlation of the big transform on clusters of two CTAs, persistent over the pairs
template <int N, int NT>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(NT, 1) corr_big_cluster_kernel(CorrArgs a)
{
    namespace cg = cooperative_groups;
    using C = BigClusterGeo<N>;
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ float4 smem_raw[];
    float2 *tile = reinterpret_cast<float2 *>(smem_raw);
    float2 *stage = tile + C::tile_elems;
    float2 *TW = stage + C::stage_elems, *TWI = TW + N;
    const int rank = int(cluster.block_rank());
    float2 *tiles[2];
    tiles[rank] = tile;
    tiles[rank ^ 1] = cluster.map_shared_rank(tile, rank ^ 1);
    for (int i = threadIdx.x; i < 2 * N; i += NT) TW[i] = a.twiddles[i];
    __syncthreads();
    cluster.sync();   // the partner has started (its shared memory exists) before any remote access
    const int npairs = a.nwin * a.nf, ncl = int(gridDim.x) / 2, cid = int(blockIdx.x) / 2;
    for (int p = cid; p < npairs; p += ncl) corr_big_cluster_pair<N, NT>(a, p, rank, tiles, stage, TW, TWI, cluster);
    cluster.sync();   // no CTA leaves while its partner may still reach its shared memory
}

#endif   // __CUDACC__

}   // namespace b200
