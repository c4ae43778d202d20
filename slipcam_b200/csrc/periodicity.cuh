// periodicity.cuh -- auto_slip.periodicity (python/slipcam/auto_slip.py:105-129) on the surfaces of
// the reference frame correlated with itself: per window, the largest 5 x 5 local maximum of its
// normalized surface (borders reflected as scipy.ndimage.maximum_filter does: d c b a | a b c d),
// leaving out the (2 exclude + 1)^2 box around zero shift; 1 for a flat window, 0 if no peak is
// left. One CTA per window.
#pragma once

#include "dft.cuh"

namespace b200 {

// the rows [lo, hi) of Python's slice [start:stop] over n elements (a negative start counts from
// the end; the reference slices the exclusion box this way)
B200_HD void py_slice(int start, int stop, int n, int &lo, int &hi)
{
    lo = start < 0 ? (start + n < 0 ? 0 : start + n) : (start > n ? n : start);
    hi = stop < 0 ? (stop + n < 0 ? 0 : stop + n) : (stop > n ? n : stop);
    if (hi < lo) hi = lo;
}

// scipy's 'reflect' border: index i of n mirrored about the half-sample edges
B200_HD int reflect_index(int i, int n)
{
    while (i < 0 || i >= n) i = i < 0 ? -i - 1 : 2 * n - i - 1;
    return i;
}

#ifdef __CUDACC__

template <int NT>
__global__ void __launch_bounds__(NT) periodicity_kernel(const float *__restrict__ surface, const float *__restrict__ norm,
                                                          int M, int search, int exclude, float *__restrict__ out)
{
    __shared__ float red[NT / 32];
    const int k = blockIdx.x;
    const float *s = surface + size_t(k) * M * M;
    if (!(norm[k] >= 1e-6f)) {   // a flat window (auto_slip.py:117-118)
        if (threadIdx.x == 0) out[k] = 1.0f;
        return;
    }
    int ylo, yhi, xlo, xhi;
    py_slice(search - exclude, search + exclude + 1, M, ylo, yhi);
    py_slice(search - exclude, search + exclude + 1, M, xlo, xhi);
    float best = -INFINITY;
    bool found = false;
    for (int idx = threadIdx.x; idx < M * M; idx += NT) {
        const int u = idx / M, v = idx % M;
        if (u >= ylo && u < yhi && v >= xlo && v < xhi) continue;
        const float c = s[idx];
        float m = c;
        for (int du = -2; du <= 2; ++du)
            for (int dv = -2; dv <= 2; ++dv) m = fmaxf(m, s[reflect_index(u + du, M) * M + reflect_index(v + dv, M)]);
        if (c == m) {   // a local maximum
            best = found ? fmaxf(best, c) : c;
            found = true;
        }
    }
    for (int o = 16; o > 0; o >>= 1) best = fmaxf(best, __shfl_xor_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
        float b = -INFINITY;
        for (int i = 0; i < NT / 32; ++i) b = fmaxf(b, red[i]);
        out[k] = b == -INFINITY ? 0.0f : b;
    }
}

#endif   // __CUDACC__

}   // namespace b200
