// diff.cuh -- the kernels of the differentiable correlation (the math is in diff.h)
#pragma once

#include "corr_fft.cuh"
#include "diff.h"

namespace b200 {

#ifdef __CUDACC__

// the mean of a pair's L x L chip, in double, every thread of the block receives it
template <int NT>
__device__ double chip_mean(const float *x, int L)
{
    __shared__ double red[NT / 32];
    double s = 0.0;
    for (int i = threadIdx.x; i < L * L; i += NT) s += x[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    double t = 0.0;
    for (int i = 0; i < NT / 32; ++i) t += red[i];
    __syncthreads();
    return t / (double(L) * L);
}

// a frame index clamped to [0, n): the edge pixel repeats beyond the frame
__device__ __forceinline__ int clamp_index(int i, int n) { return i < 0 ? 0 : (i >= n ? n - 1 : i); }

// the chips: one CTA per pair
__global__ void __launch_bounds__(256) diff_gather_kernel(DiffArgs a)
{
    const int64_t q = blockIdx.x;
    const DiffPair p = diff_pair(a, q);
    const int L = a.L;
    float *x = a.chips + q * L * L;
    if (!p.ok) {
        for (int i = threadIdx.x; i < L * L; i += blockDim.x) x[i] = 0.0f;
        return;
    }
    float wy[kTaps], wx[kTaps], dw[kTaps];
    interp_weights(p.ay, wy, dw);
    interp_weights(p.ax, wx, dw);
    const float *F = a.frames + p.f * a.fstride;
    for (int idx = threadIdx.x; idx < L * L; idx += blockDim.x) {
        const int i = idx / L, j = idx % L;
        int cx[kTaps];
#pragma unroll
        for (int e = 0; e < kTaps; ++e) cx[e] = clamp_index(p.x0 + kTap0 + j + e, a.w);
        float v = 0.0f;
#pragma unroll
        for (int d = 0; d < kTaps; ++d) {
            const float *r = F + int64_t(clamp_index(p.y0 + kTap0 + i + d, a.h)) * a.pitch;
            float row = 0.0f;
#pragma unroll
            for (int e = 0; e < kTaps; ++e) row += wx[e] * r[cx[e]];
            v += wy[d] * row;
        }
        x[idx] = v;
    }
}

// the box statistics of each pair: (mu, 1 / s) for every (u, v), sums in FP64 over column strips
constexpr int kStatStrip = 16;
__global__ void __launch_bounds__(256) diff_stats_kernel(DiffArgs a)
{
    extern __shared__ double rs[];   // 2 x L x kStatStrip: row sums of x and x^2 over W columns
    const int64_t q = blockIdx.x;
    const DiffPair p = diff_pair(a, q);
    const int L = a.L, M = a.M, W = a.W;
    float *st = a.stats + q * M * M * 2;
    if (!p.ok) {
        for (int i = threadIdx.x; i < 2 * M * M; i += blockDim.x) st[i] = 0.0f;
        return;
    }
    const float *x = a.chips + q * L * L;
    const double n = double(W) * W;
    double *r1 = rs, *r2 = rs + L * kStatStrip;
    for (int v0 = 0; v0 < M; v0 += kStatStrip) {
        for (int idx = threadIdx.x; idx < L * kStatStrip; idx += blockDim.x) {
            const int i = idx / kStatStrip, dv = idx % kStatStrip, v = v0 + dv;
            double s1 = 0.0, s2 = 0.0;
            if (v < M)
                for (int j = v; j < v + W; ++j) {
                    const double e = x[i * L + j];
                    s1 += e;
                    s2 += e * e;
                }
            r1[idx] = s1;
            r2[idx] = s2;
        }
        __syncthreads();
        for (int idx = threadIdx.x; idx < M * kStatStrip; idx += blockDim.x) {
            const int u = idx / kStatStrip, dv = idx % kStatStrip, v = v0 + dv;
            if (v >= M) continue;
            double s1 = 0.0, s2 = 0.0;
            for (int i = u; i < u + W; ++i) {
                s1 += r1[i * kStatStrip + dv];
                s2 += r2[i * kStatStrip + dv];
            }
            const double var_n = s2 - s1 * s1 / n;   // n var
            st[2 * (u * M + v)] = float(s1 / n);
            st[2 * (u * M + v) + 1] = var_n > 0 ? float(1.0 / sqrt(var_n)) : 0.0f;
        }
        __syncthreads();
    }
}

// the normalized surfaces and the peak outputs: one CTA per pair, the FFT passes of corr_kernel
// on the float chip (minus its mean, which the zero-mean reference window does not see)
template <int N, int NT>
__global__ void __launch_bounds__(NT) diff_corr_kernel(DiffArgs a)
{
    using G = Geo<N>;
    extern __shared__ float4 smem_raw[];
    float2 *S = reinterpret_cast<float2 *>(smem_raw);
    float2 *TW = S + size_t(N) * G::NHP, *TWI = TW + N;
    float *Sr = reinterpret_cast<float *>(S);
    const int64_t q = blockIdx.x;
    const DiffPair p = diff_pair(a, q);
    const int L = a.L, M = a.M;
    if (!p.ok) {
        if (threadIdx.x == 0) {
            invalid_outputs(q, a.offset, a.peak, a.snr, a.cov);
            a.peak_at[q] = -1;
        }
        for (int i = threadIdx.x; i < M * M; i += NT) a.surface[q * M * M + i] = 0.0f;
        return;
    }
    for (int i = threadIdx.x; i < 2 * N; i += NT) TW[i] = a.twiddles[i];
    const float *x = a.chips + q * L * L;
    const float mean = float(chip_mean<NT>(x, L));
    const int Lr = (L + 1) & ~1;
    for (int idx = threadIdx.x; idx < Lr * N; idx += NT) {
        const int i = idx / N, j = idx % N;
        Sr[size_t(i) * G::RP + j] = (i < L && j < L) ? x[i * L + j] - mean : 0.0f;
    }
    __syncthreads();
    const DevExec ex{int(threadIdx.x >> 5), NT / 32};
    row_forward<N>(ex, S, Lr / 2, TW);
    __syncthreads();
    col_pass<N, true>(ex, S, Lr, M, TW, TWI, a.spec + size_t(p.k) * G::NH * N, nullptr);
    __syncthreads();
    const float inv = 1.0f / (float(N) * float(N) * a.norm[p.k]);
    const float *st = a.stats + q * M * M * 2;
    row_inverse<N>(ex, S, M, TWI, [&](int u, int c, float v) { return v * inv * st[2 * (u * M + c) + 1]; });
    __syncthreads();
    for (int i = threadIdx.x; i < M * M; i += NT) a.surface[q * M * M + i] = Sr[size_t(i / M) * G::RP + i % M];
    surface_peak<NT>(Sr, G::RP, M, a.R, a.stat, p.gy, p.gx, a.W * a.W, q, a.offset, a.peak, a.snr, a.cov, a.peak_at);
}

// the chip cotangents from the surface cotangents: one CTA per pair
template <int N, int NT>
__global__ void __launch_bounds__(NT) adjoint_kernel(DiffArgs a)
{
    using G = Geo<N>;
    extern __shared__ float4 smem_raw[];
    float2 *S = reinterpret_cast<float2 *>(smem_raw);
    float2 *TW = S + size_t(N) * G::NHP, *TWI = TW + N;
    float *Sr = reinterpret_cast<float *>(S);
    const int64_t q = blockIdx.x;
    const DiffPair p = diff_pair(a, q);
    const int L = a.L, M = a.M, W = a.W;
    float *gx = a.g_chips + q * L * L;
    if (!p.ok) {
        for (int i = threadIdx.x; i < L * L; i += NT) gx[i] = 0.0f;
        return;
    }
    for (int i = threadIdx.x; i < 2 * N; i += NT) TW[i] = a.twiddles[i];
    const float *gs = a.g_surface + q * M * M, *rho = a.surface + q * M * M, *st = a.stats + q * M * M * 2;
    const float *x = a.chips + q * L * L;
    const float rnorm = 1.0f / a.norm[p.k];
    // the reversed A = G / (norm s) at rows and columns [W - 1, L)
    const int Lr = (L + 1) & ~1;
    for (int idx = threadIdx.x; idx < Lr * N; idx += NT) {
        const int i = idx / N, j = idx % N;
        float v = 0.0f;
        if (i >= W - 1 && i < L && j >= W - 1 && j < L) {
            const int uv = (L - 1 - i) * M + (L - 1 - j);
            v = gs[uv] * st[2 * uv + 1] * rnorm;
        }
        Sr[size_t(i) * G::RP + j] = v;
    }
    __syncthreads();
    const DevExec ex{int(threadIdx.x >> 5), NT / 32};
    row_forward<N>(ex, S, Lr / 2, TW);
    __syncthreads();
    col_pass<N, true>(ex, S, Lr, L, TW, TWI, a.spec + size_t(p.k) * G::NH * N, nullptr);
    __syncthreads();
    const float inv = 1.0f / (float(N) * float(N));
    row_inverse<N>(ex, S, L, TWI, [&](int u, int c, float v) {
        gx[(L - 1 - u) * L + (L - 1 - c)] = v * inv;
        return v;
    });
    __syncthreads();

    // minus sum over the boxes holding p of B (x[p] - mu), B = G rho / s^2, as two box filters of
    // B and B mu over the M x M grid (x and mu taken about the chip mean)
    const float mean = float(chip_mean<NT>(x, L));
    float *cb = Sr;   // M x L: the column-direction box sums
    for (int pass = 0; pass < 2; ++pass) {
        for (int u = threadIdx.x; u < M; u += NT) {
            double s = 0.0;
            for (int px = 0; px < L; ++px) {
                for (int side = 0; side < 2; ++side) {
                    const int v = side ? px - W : px;
                    if (v < 0 || v >= M) continue;
                    const int uv = u * M + v;
                    const float is = st[2 * uv + 1];
                    float b = gs[uv] * rho[uv] * is * is;
                    if (pass == 1) b *= st[2 * uv] - mean;
                    s += side ? -double(b) : double(b);
                }
                cb[u * L + px] = float(s);
            }
        }
        __syncthreads();
        for (int px = threadIdx.x; px < L; px += NT) {
            double s = 0.0;
            for (int py = 0; py < L; ++py) {
                if (py < M) s += cb[py * L + px];
                if (py - W >= 0 && py - W < M) s -= cb[(py - W) * L + px];
                const int i = py * L + px;
                gx[i] = pass == 0 ? float(gx[i] - (x[i] - mean) * s) : float(gx[i] + s);
            }
        }
        __syncthreads();
    }
}

// the frame and shift cotangents from the chip cotangents (the transposed interpolation): one CTA
// per pair, frame cotangents accumulated atomically (windows overlap)
__global__ void __launch_bounds__(256) diff_scatter_kernel(DiffArgs a)
{
    __shared__ float red[2][8];
    const int64_t q = blockIdx.x;
    const DiffPair p = diff_pair(a, q);
    const int L = a.L;
    if (!p.ok) {
        if (threadIdx.x == 0 && a.g_shift) a.g_shift[2 * q] = a.g_shift[2 * q + 1] = 0.0f;
        return;
    }
    float wy[kTaps], wx[kTaps], dy[kTaps], dx[kTaps];
    interp_weights(p.ay, wy, dy);
    interp_weights(p.ax, wx, dx);
    const int64_t base = p.f * a.fstride;
    const float *F = a.frames + base;
    float *GF = a.g_frames ? a.g_frames + base : nullptr;
    const float *gx = a.g_chips + q * L * L;
    float ty = 0.0f, tx = 0.0f;
    for (int idx = threadIdx.x; idx < L * L; idx += blockDim.x) {
        const int i = idx / L, j = idx % L;
        const float g = gx[idx];
        if (g == 0.0f) continue;
        int cx[kTaps];
#pragma unroll
        for (int e = 0; e < kTaps; ++e) cx[e] = clamp_index(p.x0 + kTap0 + j + e, a.w);
        float sy = 0.0f, sx = 0.0f;
#pragma unroll
        for (int d = 0; d < kTaps; ++d) {
            const int64_t r = int64_t(clamp_index(p.y0 + kTap0 + i + d, a.h)) * a.pitch;
            float row = 0.0f, drow = 0.0f;
#pragma unroll
            for (int e = 0; e < kTaps; ++e) {
                const float fv = F[r + cx[e]];
                row += wx[e] * fv;
                drow += dx[e] * fv;
                if (GF) atomicAdd(GF + r + cx[e], g * wy[d] * wx[e]);
            }
            sy += dy[d] * row;
            sx += wy[d] * drow;
        }
        ty += g * sy;
        tx += g * sx;
    }
    if (!a.g_shift) return;
    for (int o = 16; o > 0; o >>= 1) {
        ty += __shfl_xor_sync(0xffffffffu, ty, o);
        tx += __shfl_xor_sync(0xffffffffu, tx, o);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = ty;
        red[1][threadIdx.x >> 5] = tx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        float sy = 0.0f, sx = 0.0f;
        for (int w = 0; w < int(blockDim.x >> 5); ++w) {
            sy += red[0][w];
            sx += red[1][w];
        }
        a.g_shift[2 * q] = sy;
        a.g_shift[2 * q + 1] = sx;
    }
}

#endif   // __CUDACC__

#ifdef __CUDACC__

// the surface cotangents from the offset cotangents: one thread per pair, into a zeroed g_surface
__global__ void offset_adjoint_kernel(const float *surface, const int *peak_at, const float *g_offset, float *g_surface,
                                      int M, int64_t pairs)
{
    const int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= pairs) return;
    const int at = peak_at[q];
    if (at < 0) return;
    const int u = at / M, v = at % M;
    double g[9];
    const float *s = surface + q * M * M;
    offset_adjoint(s + u * M + v, M, M, u, v, g_offset[2 * q], g_offset[2 * q + 1], g);
    if (!(u > 0 && u < M - 1 && v > 0 && v < M - 1)) return;
    float *gs = g_surface + q * M * M;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) gs[(u + i - 1) * M + v + j - 1] += float(g[3 * i + j]);
}

#endif   // __CUDACC__

}   // namespace b200
