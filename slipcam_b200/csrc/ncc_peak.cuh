// ncc_peak.cuh -- the peak of a normalized surface as stabilize.ncc_peak takes it
// (python/slipcam/stabilize.py:35-44): the largest value (the first in raster order if equal, as
// numpy.argmax), a parabola per axis through it and its two neighbours (0.5 (m - p) / (m - 2c + p),
// 0 when that denominator is below 1e-12 in magnitude or at the edge), as (dy, dx) relative to the
// surface centre, and the value. Shared by the standalone peak kernel and the correlation kernel's
// fused epilogue.
#pragma once

#include <climits>
#include <cmath>

namespace b200 {

#ifdef __CUDACC__

// the whole CTA: the peak of the M x M surface s (rows `pitch` floats apart) into out[0..2]
template <int NT>
__device__ __forceinline__ void ncc_peak_block(const float *s, int pitch, int M, double *out)
{
    __shared__ float s_best[NT / 32];
    __shared__ int s_at[NT / 32];
    float best = -INFINITY;
    int at = INT_MAX;
    for (int idx = threadIdx.x; idx < M * M; idx += NT) {
        const float c = s[size_t(idx / M) * pitch + idx % M];
        if (c > best) {   // strictly: the first of equal values in this thread's stride
            best = c;
            at = idx;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const float b = __shfl_xor_sync(0xffffffffu, best, o);
        const int ib = __shfl_xor_sync(0xffffffffu, at, o);
        if (b > best || (b == best && ib < at)) {
            best = b;
            at = ib;
        }
    }
    if ((threadIdx.x & 31) == 0) {
        s_best[threadIdx.x >> 5] = best;
        s_at[threadIdx.x >> 5] = at;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < NT / 32; ++w)
            if (s_best[w] > best || (s_best[w] == best && s_at[w] < at)) {
                best = s_best[w];
                at = s_at[w];
            }
        if (at == INT_MAX) at = 0;   // every value NaN: the first; its NaN peak fails any min_peak
        const int i = at / M, j = at % M;
        auto refine = [](double c, double m, double p) {
            const double den = m - 2 * c + p;
            return fabs(den) < 1e-12 ? 0.0 : 0.5 * (m - p) / den;
        };
        const float *pc = s + size_t(i) * pitch + j;
        const double c = *pc;
        const double di = i > 0 && i < M - 1 ? refine(c, pc[-pitch], pc[pitch]) : 0.0;
        const double dj = j > 0 && j < M - 1 ? refine(c, pc[-1], pc[1]) : 0.0;
        const double c0 = 0.5 * (M - 1);
        out[0] = i + di - c0;
        out[1] = j + dj - c0;
        out[2] = c;
    }
    __syncthreads();
}

#endif   // __CUDACC__

}   // namespace b200
