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

constexpr int kDiffRun = 16;   // consecutive pairs of frames per CTA of the difference scan

// sum |f[k + 1] - f[k]| over the pixels, exact (64-bit), for the pairs k0 .. k0 + kDiffRun - 1 of
// this CTA's run (blockIdx.y) over its band of rows (blockIdx.x): each thread walks a word (4
// pixels) or a pixel through the run's frames with the previous frame's value in a register, so
// every frame of the run is read once; the run's loads are independent, issued back to back
__global__ void __launch_bounds__(256) frame_diff_kernel(const uint8_t *__restrict__ frames, int64_t fstride, int pitch,
                                                           int h, int w, int npairs, unsigned long long *__restrict__ sums)
{
    const int k0 = blockIdx.y * kDiffRun, K = min(kDiffRun, npairs - k0);
    const int rows = (h + gridDim.x - 1) / gridDim.x, r0 = blockIdx.x * rows, r1 = min(h, r0 + rows);
    // a thread's own sums fit 32 bits: at most (its pieces) x 16 x 255, under 2^26 for any frame a
    // band of rows of an 8K video gives one thread; the warp and the total are 64-bit
    uint32_t acc[kDiffRun];
#pragma unroll
    for (int j = 0; j < kDiffRun; ++j) acc[j] = 0;
    if (r0 < r1) {
        const uint8_t *f0 = frames + k0 * fstride;
        const int align = pitch | int(fstride & 15) | int(reinterpret_cast<uintptr_t>(frames) & 15);
        // 16 pixels per load where rows and frames are 16-byte aligned: enough bytes in flight
        const int w16 = (align & 15) == 0 ? w / 16 : 0;
        if (w16 > 0) {
            const int64_t fv = fstride / 16, n_el = int64_t(r1 - r0) * w16;
            for (int64_t e = threadIdx.x; e < n_el; e += blockDim.x) {
                const int r = r0 + int(e / w16), c = int(e % w16);
                const uint4 *p = reinterpret_cast<const uint4 *>(f0 + int64_t(r) * pitch) + c;
                uint4 prev = __ldg(p);
#pragma unroll
                for (int j = 0; j < kDiffRun; ++j) {
                    if (j < K) {
                        const uint4 cur = __ldg(p + (j + 1) * fv);
                        acc[j] += __vsadu4(prev.x, cur.x) + __vsadu4(prev.y, cur.y) + __vsadu4(prev.z, cur.z) +
                                  __vsadu4(prev.w, cur.w);
                        prev = cur;
                    }
                }
            }
        }
        const bool words = (align & 3) == 0;
        const int wq = words ? (w - 16 * w16) / 4 : 0, cw = 16 * w16;   // words past the 16-pixel pieces
        if (wq > 0) {
            const int64_t fw = fstride / 4, n_el = int64_t(r1 - r0) * wq;
            for (int64_t e = threadIdx.x; e < n_el; e += blockDim.x) {
                const int r = r0 + int(e / wq), c = int(e % wq);
                const uint32_t *p = reinterpret_cast<const uint32_t *>(f0 + int64_t(r) * pitch + cw) + c;
                uint32_t prev = __ldg(p);
#pragma unroll
                for (int j = 0; j < kDiffRun; ++j) {
                    if (j < K) {
                        const uint32_t cur = __ldg(p + (j + 1) * fw);
                        const uint32_t d = __vabsdiffu4(prev, cur);
                        acc[j] += (d & 0xFFu) + ((d >> 8) & 0xFFu) + ((d >> 16) & 0xFFu) + (d >> 24);
                        prev = cur;
                    }
                }
            }
        }
        // the columns past the words (or every column when the frames are not word-aligned)
        const int c0 = cw + 4 * wq, tail = w - c0;
        const int64_t n_tail = int64_t(r1 - r0) * tail;
        for (int64_t e = threadIdx.x; e < n_tail; e += blockDim.x) {
            const int r = r0 + int(e / tail), c = c0 + int(e % tail);
            const uint8_t *p = f0 + int64_t(r) * pitch + c;
            int prev = p[0];
#pragma unroll
            for (int j = 0; j < kDiffRun; ++j) {
                if (j < K) {
                    const int cur = p[(j + 1) * fstride];
                    acc[j] += unsigned(abs(cur - prev));
                    prev = cur;
                }
            }
        }
    }
#pragma unroll
    for (int j = 0; j < kDiffRun; ++j) {
        unsigned long long v = acc[j];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);   // 64-bit from here
        if ((threadIdx.x & 31) == 0 && j < K && v) atomicAdd(sums + k0 + j, v);
    }
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
