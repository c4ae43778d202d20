// scans.cuh -- the frame scans of auto_slip (python/slipcam/auto_slip.py:56-94): the mean absolute
// difference of consecutive frames, and the pieces of the burned-in text mask -- the median over
// chunks of the per-pixel temporal standard deviation, the Sobel edge magnitude of a frame (borders
// reflected as scipy.ndimage does), the threshold, the cross-shaped dilation and the filling of the
// holes (background not 4-connected to the border). All bandwidth-bound passes over uint8 frames.
#pragma once

#include <cstdint>

#include "dft.cuh"

namespace b200 {

constexpr int kScanMaxChunks = 64;   // chunks of the temporal median (nframes / chunk)

#ifdef __CUDACC__

// sum |f[k + 1] - f[k]| over the pixels, exact (64-bit), one CTA per (pair, band of rows)
__global__ void __launch_bounds__(256) frame_diff_kernel(const uint8_t *__restrict__ frames, int64_t fstride, int pitch,
                                                           int h, int w, unsigned long long *__restrict__ sums)
{
    const int k = blockIdx.y;
    const uint8_t *a = frames + k * fstride, *b = a + fstride;
    unsigned long long s = 0;
    const int rows = (h + gridDim.x - 1) / gridDim.x, r0 = blockIdx.x * rows, r1 = min(h, r0 + rows);
    for (int r = r0; r < r1; ++r) {
        const uint8_t *pa = a + int64_t(r) * pitch, *pb = b + int64_t(r) * pitch;
        if (((pitch | reinterpret_cast<uintptr_t>(a)) & 3) == 0) {
            const int wq = w / 4;
            for (int c = threadIdx.x; c < wq; c += blockDim.x) {
                const uint32_t x = reinterpret_cast<const uint32_t *>(pa)[c], y = reinterpret_cast<const uint32_t *>(pb)[c];
                s += __vabsdiffu4(x, y) & 0xFFu;
                s += (__vabsdiffu4(x, y) >> 8) & 0xFFu;
                s += (__vabsdiffu4(x, y) >> 16) & 0xFFu;
                s += __vabsdiffu4(x, y) >> 24;
            }
            for (int c = 4 * wq + threadIdx.x; c < w; c += blockDim.x) s += abs(int(pa[c]) - int(pb[c]));
        } else {
            for (int c = threadIdx.x; c < w; c += blockDim.x) s += abs(int(pa[c]) - int(pb[c]));
        }
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(sums + k, s);
}

// per pixel: the population standard deviation of each chunk of `chunk` frames (exact integer
// sums, the root in float), then their median over nchunks (the mean of the two middle values
// when nchunks is even, as numpy.median)
__global__ void __launch_bounds__(256) chunk_std_median_kernel(const uint8_t *__restrict__ frames, int64_t fstride, int pitch,
                                                                 int h, int w, int chunk, int nchunks, float *__restrict__ out)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= int64_t(h) * w) return;
    const int r = int(i / w), c = int(i % w);
    float v[kScanMaxChunks];
    for (int m = 0; m < nchunks; ++m) {
        int s1 = 0, s2 = 0;
        for (int t = 0; t < chunk; ++t) {
            const int x = frames[(int64_t(m) * chunk + t) * fstride + int64_t(r) * pitch + c];
            s1 += x;
            s2 += x * x;
        }
        const double var = (double(chunk) * s2 - double(s1) * s1) / (double(chunk) * chunk);
        v[m] = float(sqrt(var > 0 ? var : 0.0));
    }
    for (int a = 1; a < nchunks; ++a)   // insertion sort of a few values
        for (int b = a; b > 0 && v[b - 1] > v[b]; --b) {
            const float t = v[b];
            v[b] = v[b - 1];
            v[b - 1] = t;
        }
    out[i] = nchunks % 2 ? v[nchunks / 2] : 0.5f * (v[nchunks / 2 - 1] + v[nchunks / 2]);
}

__device__ __forceinline__ int scan_reflect(int i, int n) { return i < 0 ? -i - 1 : (i >= n ? 2 * n - i - 1 : i); }

// hypot(sobel along rows, sobel along columns) of a uint8 frame, float32, borders reflected
__global__ void __launch_bounds__(256) sobel_kernel(const uint8_t *__restrict__ f, int pitch, int h, int w, float *__restrict__ out)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= int64_t(h) * w) return;
    const int r = int(i / w), c = int(i % w);
    float p[3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) p[a][b] = float(f[int64_t(scan_reflect(r + a - 1, h)) * pitch + scan_reflect(c + b - 1, w)]);
    // axis 0: the difference across rows, smoothed 1 2 1 across columns; axis 1 the transpose
    const float g0 = (p[2][0] - p[0][0]) + 2.0f * (p[2][1] - p[0][1]) + (p[2][2] - p[0][2]);
    const float g1 = (p[0][2] - p[0][0]) + 2.0f * (p[1][2] - p[1][0]) + (p[2][2] - p[2][0]);
    out[i] = hypotf(g0, g1);
}

// mask = edge > thr && std < max_std
__global__ void text_seed_kernel(const float *__restrict__ edge, const float *__restrict__ sd, int64_t n, float thr, float max_std,
                                 uint8_t *__restrict__ mask)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) mask[i] = edge[i] > thr && sd[i] < max_std;
}

// one step of the binary dilation with the 3 x 3 cross (outside the image: background)
__global__ void dilate_kernel(const uint8_t *__restrict__ in, uint8_t *__restrict__ out, int h, int w)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= int64_t(h) * w) return;
    const int r = int(i / w), c = int(i % w);
    out[i] = in[i] | (r > 0 && in[i - w]) | (r + 1 < h && in[i + w]) | (c > 0 && in[i - 1]) | (c + 1 < w && in[i + 1]);
}

// the background reached from the border (4-connected): outside[i] = 1 for border background;
// each step spreads it by up to `sweeps` pixels inside a CTA's tile of rows, and flags a change
__global__ void outside_init_kernel(const uint8_t *__restrict__ mask, uint8_t *__restrict__ outside, int h, int w)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= int64_t(h) * w) return;
    const int r = int(i / w), c = int(i % w);
    outside[i] = !mask[i] && (r == 0 || c == 0 || r == h - 1 || c == w - 1);
}

__global__ void outside_step_kernel(const uint8_t *__restrict__ mask, uint8_t *__restrict__ outside, int h, int w, int *changed)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= int64_t(h) * w) return;
    if (outside[i] || mask[i]) return;
    const int r = int(i / w), c = int(i % w);
    if ((r > 0 && outside[i - w]) || (r + 1 < h && outside[i + w]) || (c > 0 && outside[i - 1]) || (c + 1 < w && outside[i + 1])) {
        outside[i] = 1;
        *changed = 1;
    }
}

// the filled mask: everything not reached from the border
__global__ void fill_kernel(const uint8_t *__restrict__ outside, uint8_t *__restrict__ out, int64_t n)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) out[i] = !outside[i];
}

#endif   // __CUDACC__

}   // namespace b200
