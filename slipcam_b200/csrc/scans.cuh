// scans.cuh -- the frame scans of auto_slip (python/slipcam/auto_slip.py:56-94): the mean absolute
// difference of consecutive frames, and the pieces of the burned-in text mask -- the median over
// chunks of the per-pixel temporal standard deviation, the Sobel edge magnitude of a frame (borders
// reflected as scipy.ndimage does), the threshold, the cross-shaped dilation and the filling of the
// holes (background not 4-connected to the border). All bandwidth-bound passes over uint8 frames.
#pragma once

#include <cstdint>

#include <cooperative_groups.h>

#include "dft.cuh"

namespace b200 {

constexpr int kScanMaxChunks = 64;   // chunks of the temporal median (nframes / chunk)
constexpr int kSelectBins = 2048;     // bins of a pass of the percentile's radix selection (11 bits)
constexpr int kSelectScratch = 256 + 2 * kSelectBins * 4;   // its state and two histograms, bytes
constexpr int kDilateRows = 16;       // rows a CTA of the bit dilation writes
constexpr int kDilateStep = 8;        // dilation steps per launch (the tile's halo rows)
constexpr int kFloodThreads = 1024;   // threads per CTA of the hole filling
constexpr int kFloodCluster = 8;      // CTAs of the clustered hole filling, a band of rows each

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
// when nchunks is even, as numpy.median). The deviation float(sqrt(num / chunk^2)) (float64
// division and root) is non-decreasing in the exact numerator num = chunk * sum x^2 - (sum x)^2,
// so the chunks are ordered by num and only the middle one or two become deviations. A CTA takes
// kStdPixels pixels of a row (a frame whose rows are contiguous comes as one long row), 8 per
// lane in one 8-byte load where aligned; warp y sums chunks y, y + blockDim.y, ..., a batch of
// kStdBatch frames' loads in flight together. The numerators meet in shared memory (chunk m's slot t
// holds the pixel t / 32 of lane t % 32) and thread t orders slot t's column: up to kStdRegChunks
// chunks by Batcher's odd-even merge network in registers, above that by insertion in place.
// NumT: uint32_t while chunk <= 513 (num < 2^32), else uint64_t.
constexpr int kStdLanePixels = 8;
constexpr int kStdPixels = 32 * kStdLanePixels;
constexpr int kStdRegChunks = 16;
constexpr int kStdBatch = 16;   // frames of a chunk whose loads are in flight together

__device__ __forceinline__ float chunk_std(uint64_t num, int chunk)
{
    return float(sqrt(double(num) / (double(chunk) * chunk)));
}

template <typename NumT>
__global__ void __launch_bounds__(512, 2) chunk_std_median_kernel(const uint8_t *__restrict__ frames, int64_t fstride, int pitch,
                                                                    int h, int w, int chunk, int nchunks, float *__restrict__ out)
{
    extern __shared__ __align__(8) unsigned char std_smem[];
    NumT *v = reinterpret_cast<NumT *>(std_smem);   // [nchunks][kStdPixels]
    const int r = blockIdx.y, c0 = blockIdx.x * kStdPixels, lane = threadIdx.x;
    const int c = c0 + kStdLanePixels * lane;
    const uint8_t *row = frames + int64_t(r) * pitch + c;
    const bool vec = ((reinterpret_cast<uintptr_t>(row) | uintptr_t(fstride)) & 7) == 0 && c + kStdLanePixels <= w;
    for (int m = threadIdx.y; m < nchunks; m += blockDim.y) {
        uint32_t s1[kStdLanePixels], s2[kStdLanePixels];
#pragma unroll
        for (int j = 0; j < kStdLanePixels; ++j) s1[j] = s2[j] = 0;
        const uint8_t *p = row + int64_t(m) * chunk * fstride;
        if (vec) {
            for (int t0 = 0; t0 < chunk; t0 += kStdBatch, p += kStdBatch * fstride) {
                uint2 q[kStdBatch];   // the batch's loads all issue before any is used
#pragma unroll
                for (int k = 0; k < kStdBatch; ++k)
                    q[k] = t0 + k < chunk ? __ldg(reinterpret_cast<const uint2 *>(p + k * fstride)) : make_uint2(0, 0);
#pragma unroll
                for (int k = 0; k < kStdBatch; ++k)
#pragma unroll
                    for (int j = 0; j < kStdLanePixels; ++j) {
                        const uint32_t x = __byte_perm(j < 4 ? q[k].x : q[k].y, 0u, 0x4440u | unsigned(j & 3));
                        s1[j] += x;
                        s2[j] += x * x;
                    }
            }
        } else {   // unaligned rows or the row's last pixels: byte loads
            for (int t = 0; t < chunk; ++t, p += fstride)
#pragma unroll
                for (int j = 0; j < kStdLanePixels; ++j) {
                    const uint32_t x = c + j < w ? p[j] : 0u;
                    s1[j] += x;
                    s2[j] += x * x;
                }
        }
#pragma unroll
        for (int j = 0; j < kStdLanePixels; ++j)
            v[m * kStdPixels + j * 32 + lane] = NumT(uint64_t(chunk) * s2[j] - uint64_t(s1[j]) * s1[j]);
    }
    __syncthreads();
    for (int t = threadIdx.y * 32 + lane; t < kStdPixels; t += blockDim.x * blockDim.y) {
        const int col = c0 + kStdLanePixels * (t & 31) + (t >> 5);
        if (col >= w) continue;
        NumT lo = 0, hi = 0;   // the numerators of ranks (nchunks - 1) / 2 and nchunks / 2
        if (nchunks <= kStdRegChunks) {
            NumT x[kStdRegChunks];
#pragma unroll
            for (int m = 0; m < kStdRegChunks; ++m) x[m] = m < nchunks ? v[m * kStdPixels + t] : ~NumT(0);   // padding sorts last
#pragma unroll
            for (int p = 1; p < kStdRegChunks; p <<= 1)
#pragma unroll
                for (int k = p; k >= 1; k >>= 1)
#pragma unroll
                    for (int j = k % p; j + k < kStdRegChunks; j += 2 * k)
#pragma unroll
                        for (int i = 0; i < k; ++i)
                            if (i + j + k < kStdRegChunks && (i + j) / (2 * p) == (i + j + k) / (2 * p)) {
                                const NumT a = x[i + j], b = x[i + j + k];
                                x[i + j] = min(a, b);
                                x[i + j + k] = max(a, b);
                            }
#pragma unroll
            for (int m = 0; m < kStdRegChunks; ++m) {
                if (m == (nchunks - 1) / 2) lo = x[m];
                if (m == nchunks / 2) hi = x[m];
            }
        } else {
            NumT *col_v = v + t;   // this thread's column, kStdPixels apart
            for (int a = 1; a < nchunks; ++a)   // insertion sort
                for (int b = a; b > 0 && col_v[(b - 1) * kStdPixels] > col_v[b * kStdPixels]; --b) {
                    const NumT x = col_v[b * kStdPixels];
                    col_v[b * kStdPixels] = col_v[(b - 1) * kStdPixels];
                    col_v[(b - 1) * kStdPixels] = x;
                }
            lo = col_v[((nchunks - 1) / 2) * kStdPixels];
            hi = col_v[(nchunks / 2) * kStdPixels];
        }
        const float b = chunk_std(hi, chunk);
        out[int64_t(r) * w + col] = nchunks % 2 ? b : 0.5f * (chunk_std(lo, chunk) + b);
    }
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

// ---- numpy.percentile (method 'linear') of float32 values, on the device: the two order
// statistics around the virtual index by a radix selection over an order-preserving 32-bit key,
// 11 + 11 + 10 bits in three passes; the percentile itself as numpy interpolates float32 data.

// the state between the passes, at the start of the scratch; the two histograms follow it
struct SelectState {
    uint32_t prefix[2];   // the key bits resolved so far, of the lower and the upper statistic
    uint32_t rank[2];     // their ranks among the values that share the prefix
    uint32_t arrived;     // CTAs done with the current pass
};

// unsigned order of the keys == the order of the floats (negative below positive, NaN on top)
__device__ __forceinline__ uint32_t order_key(float f)
{
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__device__ __forceinline__ float key_value(uint32_t k) { return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k); }

// exclusive prefix sum over a CTA of 256 threads
__device__ __forceinline__ uint32_t cta_exclusive_sum_256(uint32_t x, uint32_t *warp_tot)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = x;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, inc, d);
        if (lane >= d) inc += y;
    }
    if (lane == 31) warp_tot[warp] = inc;
    __syncthreads();
    uint32_t before = 0;
    for (int k = 0; k < warp; ++k) before += warp_tot[k];
    __syncthreads();
    return before + inc - x;
}

// One pass of the selection of the statistics of ranks lo <= hi among x[0 .. n): pass 0 counts
// the keys' bits 31..21, pass 1 bits 20..10 of the keys that share the picked top bits, pass 2
// bits 9..0. A CTA counts in shared memory (four elements a thread per trip, their loads issued
// together; the equal bins of a warp added once, by __match_any_sync) and adds its counts to the histograms in global memory; the last CTA to finish
// (a ticket taken after a fence) picks each statistic's bin, narrows its rank, clears the
// histograms for the next pass and, after pass 2, writes the percentile to *out: numpy's lerp in
// float32, a + (b - a) * t for t < 0.5, else b - (b - a) * (1 - t), each step rounded.
__global__ void __launch_bounds__(256) select_pass_kernel(const float *__restrict__ x, int64_t n, int pass, uint32_t lo,
                                                          uint32_t hi, float t, SelectState *st, uint32_t *hist, float *out)
{
    constexpr int B = kSelectBins;
    __shared__ uint32_t cnt[2][B];
    __shared__ uint32_t warp_tot[8];
    __shared__ uint32_t pick[2][2];
    __shared__ int last;
    const int shift = pass == 0 ? 21 : (pass == 1 ? 10 : 0), bins = pass == 2 ? B / 2 : B;
    const uint32_t known = pass == 0 ? 0u : (pass == 1 ? 0xFFE00000u : 0xFFFFFC00u);
    const uint32_t p0 = pass ? st->prefix[0] : 0u, p1 = pass ? st->prefix[1] : 0u;
    const bool two = p0 != p1;   // the statistics took different bins: a histogram each
    for (int i = threadIdx.x; i < 2 * B; i += blockDim.x) (&cnt[0][0])[i] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    constexpr int U = 4;   // elements per thread per trip, their loads issued together
    const int64_t stride = int64_t(gridDim.x) * blockDim.x * U;
    for (int64_t base = int64_t(blockIdx.x) * blockDim.x * U; base < n; base += stride) {   // the same trips for a warp
        float v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int64_t i = base + int64_t(u) * blockDim.x + threadIdx.x;
            v[u] = i < n ? __ldg(x + i) : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const bool ok = base + int64_t(u) * blockDim.x + threadIdx.x < n;
            const uint32_t k = ok ? order_key(v[u]) : 0u;
            const uint32_t d = (k >> shift) & uint32_t(bins - 1);
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                if (s == 1 && !two) break;
                const bool in = ok && (k & known) == (s ? p1 : p0);
                const unsigned peers = __match_any_sync(0xffffffffu, in ? d : 0xFFFFFFFFu);
                if (in && lane == __ffs(peers) - 1) atomicAdd(&cnt[s][d], unsigned(__popc(peers)));
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < bins; i += blockDim.x) {
        if (cnt[0][i]) atomicAdd(hist + i, cnt[0][i]);
        if (two && cnt[1][i]) atomicAdd(hist + B + i, cnt[1][i]);
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(&st->arrived, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    const uint32_t r0 = pass ? st->rank[0] : lo, r1 = pass ? st->rank[1] : hi;
    const int per = bins / 256;   // bins per thread: 8, or 4 in pass 2
    for (int s = 0; s < 2; ++s) {
        const uint32_t *hs = hist + (two && s ? B : 0);
        const uint32_t r = s ? r1 : r0;
        uint32_t c8[8], tot = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            c8[j] = j < per ? __ldcg(hs + threadIdx.x * per + j) : 0u;
            tot += c8[j];
        }
        uint32_t acc = cta_exclusive_sum_256(tot, warp_tot);
        if (acc <= r && r < acc + tot)
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                if (j < per && r < acc + c8[j]) {
                    pick[s][0] = uint32_t(threadIdx.x * per + j);
                    pick[s][1] = r - acc;
                    break;
                }
                acc += c8[j];
            }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < 2 * B; i += blockDim.x) hist[i] = 0;   // for the next pass
    if (threadIdx.x == 0) {
        const uint32_t q0 = p0 | (pick[0][0] << shift), q1 = p1 | (pick[1][0] << shift);
        st->prefix[0] = q0;
        st->prefix[1] = q1;
        st->rank[0] = pick[0][1];
        st->rank[1] = pick[1][1];
        st->arrived = 0;
        if (pass == 2) {
            const float a = key_value(q0), b = key_value(q1), diff = __fsub_rn(b, a);
            *out = t < 0.5f ? __fadd_rn(a, __fmul_rn(diff, t)) : __fsub_rn(b, __fmul_rn(diff, __fsub_rn(1.0f, t)));
        }
    }
}

// ---- The text mask on bit planes: bit j of word c of a row is pixel 32 c + j; a row is wpr =
// ceil(w / 32) words, the bits past the frame's width are 0.

__device__ __forceinline__ uint32_t row_bits(int c, int w)   // the bits of word c inside the frame
{
    const int rem = w - 32 * c;
    return rem >= 32 ? 0xFFFFFFFFu : ((1u << rem) - 1u);
}

// scipy's binary_dilation with iterations < 1 repeats the dilation until nothing changes: with the
// 3 x 3 cross over a connected frame that is every pixel as soon as one is set. any_bits_kernel ORs
// every word into *flag (zeroed first); all_bits_kernel then sets every pixel if it is not zero.
__global__ void __launch_bounds__(256) any_bits_kernel(const uint32_t *__restrict__ m, int64_t words, uint32_t *flag)
{
    uint32_t v = 0;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < words; i += int64_t(gridDim.x) * blockDim.x)
        v |= m[i];
    v = __reduce_or_sync(0xffffffffu, v);
    if ((threadIdx.x & 31) == 0 && v) atomicOr(flag, 1u);
}

__global__ void __launch_bounds__(256) all_bits_kernel(uint32_t *__restrict__ m, int h, int w, int wpr,
                                                       const uint32_t *flag)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= int64_t(h) * wpr || !*flag) return;
    m[i] = row_bits(int(i % wpr), w);
}

// mask bits = edge > *thr and sd < max_std, one warp per word (a ballot of its 32 pixels)
__global__ void __launch_bounds__(256) text_seed_bits_kernel(const float *__restrict__ edge, const float *__restrict__ sd, int h,
                                                             int w, int wpr, const float *__restrict__ thr, float max_std,
                                                             uint32_t *__restrict__ bits)
{
    const int64_t word = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    if (word >= int64_t(h) * wpr) return;   // whole warps
    const int lane = threadIdx.x & 31, r = int(word / wpr), col = 32 * int(word % wpr) + lane;
    bool on = false;
    if (col < w) {
        const int64_t i = int64_t(r) * w + col;
        on = edge[i] > *thr && sd[i] < max_std;
    }
    const uint32_t v = __ballot_sync(0xffffffffu, on);
    if (lane == 0) bits[word] = v;
}

// `steps` (<= kDilateStep) steps of the binary dilation by the 3 x 3 cross (outside the frame:
// background) for kDilateRows rows per CTA: their rows and `steps` rows either side in shared
// memory, dilated there (the halo rows go wrong from the tile's edge inward, one row a step)
__global__ void __launch_bounds__(256) dilate_bits_kernel(const uint32_t *__restrict__ in, uint32_t *__restrict__ out, int h,
                                                          int w, int wpr, int steps)
{
    extern __shared__ uint32_t tile[];
    const int S = kDilateRows + 2 * steps, top = blockIdx.x * kDilateRows - steps;
    uint32_t *a = tile, *b = tile + S * wpr;
    for (int e = threadIdx.x; e < S * wpr; e += blockDim.x) {
        const int r = top + e / wpr;
        a[e] = (r >= 0 && r < h) ? in[int64_t(r) * wpr + e % wpr] : 0u;
    }
    __syncthreads();
    for (int k = 0; k < steps; ++k) {
        for (int e = threadIdx.x; e < S * wpr; e += blockDim.x) {
            const int lr = e / wpr, c = e - lr * wpr, r = top + lr;
            uint32_t v = 0;
            if (r >= 0 && r < h) {
                const uint32_t m = a[e];
                v = m | (m << 1) | (m >> 1);
                if (c > 0) v |= a[e - 1] >> 31;
                if (c + 1 < wpr) v |= a[e + 1] << 31;
                if (lr > 0) v |= a[e - wpr];
                if (lr + 1 < S) v |= a[e + wpr];
                v &= row_bits(c, w);
            }
            b[e] = v;
        }
        __syncthreads();
        uint32_t *x = a;
        a = b;
        b = x;
    }
    for (int e = steps * wpr + threadIdx.x; e < (steps + kDilateRows) * wpr; e += blockDim.x) {
        const int r = top + e / wpr;
        if (r < h) out[int64_t(r) * wpr + e % wpr] = a[e];
    }
}

// the free pixels a seed s (inside f) reaches along f's runs toward higher bits: the carry of
// f + s runs from each seed to the end of its run
__device__ __forceinline__ uint32_t fill_up(uint32_t f, uint32_t s) { return (((f + s) ^ f) & f) | s; }
__device__ __forceinline__ uint32_t fill_down(uint32_t f, uint32_t s) { return __brev(fill_up(__brev(f), __brev(s))); }
__device__ __forceinline__ uint32_t bottom_run(uint32_t f) { return f & ~(f + 1u); }   // the run of f from bit 0
__device__ __forceinline__ uint32_t top_run(uint32_t f) { return __brev(bottom_run(__brev(f))); }   // the run to bit 31

// The horizontal sweep of a row: rightward, then leftward. A lane holds K consecutive words of a
// segment of 32 K words (rows of more than 256 words come in several segments, the carry passed
// along). A word filled from its own seeds gives r; its carry out is g = the run reaching the far
// end, or the carry in when the word is all free; the carries into the lanes follow from the
// ballots of the lanes' composite carries by one addition, and a word with a carry in adds the
// run it enters by (the bottom run rightward, the top run leftward).
template <int K>
__device__ __forceinline__ bool hrow(const uint32_t *F, uint32_t *O, int64_t rb, int wpr)
{
    const int lane = threadIdx.x & 31;
    bool ch = false;
    uint32_t seg = 0;
    for (int s0 = 0; s0 < wpr; s0 += 32 * K) {   // rightward
        const int sw = min(32 * K, wpr - s0);
        uint32_t f[K], o[K], r[K], G = 0, P = 1;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int j = lane * K + k;
            f[k] = o[k] = r[k] = 0;
            if (j < sw) {
                f[k] = F[rb + s0 + j];
                o[k] = O[rb + s0 + j];
                r[k] = fill_up(f[k], o[k]);
                const uint32_t g0 = r[k] >> 31, g1 = g0 | (f[k] == 0xFFFFFFFFu ? 1u : 0u);
                G = g0 | (g1 & G);
                P = g0 | (g1 & P);
            }
        }
        const uint32_t g = __ballot_sync(0xffffffffu, G), p = __ballot_sync(0xffffffffu, P);
        const uint64_t sum = uint64_t(g) + p + seg;
        uint32_t cin = ((uint32_t(sum) ^ g ^ p) >> lane) & 1u;
        seg = uint32_t(sum >> 32);
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int j = lane * K + k;
            if (j < sw) {
                const uint32_t res = r[k] | (cin ? bottom_run(f[k]) : 0u);
                cin = res >> 31;
                if (res != o[k]) {
                    O[rb + s0 + j] = res;
                    ch = true;
                }
            }
        }
    }
    __syncwarp();
    seg = 0;
    for (int s1 = wpr; s1 > 0; s1 -= 32 * K) {   // leftward: lanes and words from the right
        const int s0 = max(0, s1 - 32 * K), sw = s1 - s0;
        uint32_t f[K], o[K], r[K], G = 0, P = 1;
#pragma unroll
        for (int k = K - 1; k >= 0; --k) {
            const int j = lane * K + k;
            f[k] = o[k] = r[k] = 0;
            if (j < sw) {
                f[k] = F[rb + s0 + j];
                o[k] = O[rb + s0 + j];
                r[k] = fill_down(f[k], o[k]);
                const uint32_t g0 = r[k] & 1u, g1 = g0 | (f[k] == 0xFFFFFFFFu ? 1u : 0u);
                G = g0 | (g1 & G);
                P = g0 | (g1 & P);
            }
        }
        const uint32_t g = __brev(__ballot_sync(0xffffffffu, G)), p = __brev(__ballot_sync(0xffffffffu, P));
        const uint64_t sum = uint64_t(g) + p + seg;
        uint32_t cin = ((uint32_t(sum) ^ g ^ p) >> (31 - lane)) & 1u;
        seg = uint32_t(sum >> 32);
#pragma unroll
        for (int k = K - 1; k >= 0; --k) {
            const int j = lane * K + k;
            if (j < sw) {
                const uint32_t res = r[k] | (cin ? top_run(f[k]) : 0u);
                cin = res & 1u;
                if (res != o[k]) {
                    O[rb + s0 + j] = res;
                    ch = true;
                }
            }
        }
    }
    return ch;
}

template <int K>
__device__ __forceinline__ bool hsweep(const uint32_t *F, uint32_t *O, int h, int wpr)
{
    bool ch = false;
    for (int r = threadIdx.x >> 5; r < h; r += blockDim.x >> 5) ch |= hrow<K>(F, O, int64_t(r) * wpr, wpr);
    return ch;
}

// one 32-row block of the vertical sweep for NC columns of words at once (their scans interleave):
// D = O | F & D_above down the block (lane order), from the carry of the block before; lane 0 of
// the block is row r0 + lane0 and rows step by dir
template <int NC>
__device__ __forceinline__ bool vblock(const uint32_t *F, uint32_t *O, int h, int wpr, const int (&col)[NC], int nc, int r,
                                       uint32_t (&carry)[NC])
{
    const int lane = threadIdx.x & 31;
    bool ch = false;
    uint32_t f[NC], o[NC], A[NC], B[NC];
#pragma unroll
    for (int q = 0; q < NC; ++q) {
        const bool in = q < nc && r < h && r >= 0;
        f[q] = in ? F[int64_t(r) * wpr + col[q]] : 0u;
        o[q] = in ? O[int64_t(r) * wpr + col[q]] : 0u;
        A[q] = in ? f[q] : 0xFFFFFFFFu;   // rows past the end pass the carry through
        B[q] = o[q];
    }
#pragma unroll
    for (int d = 1; d < 32; d <<= 1)
#pragma unroll
        for (int q = 0; q < NC; ++q) {
            const uint32_t a2 = __shfl_up_sync(0xffffffffu, A[q], d), b2 = __shfl_up_sync(0xffffffffu, B[q], d);
            if (lane >= d) {
                B[q] |= A[q] & b2;
                A[q] &= a2;
            }
        }
#pragma unroll
    for (int q = 0; q < NC; ++q) {
        const uint32_t D = B[q] | (A[q] & carry[q]);
        carry[q] = __shfl_sync(0xffffffffu, D, 31);
        if (q < nc && r < h && r >= 0 && D != o[q]) {
            O[int64_t(r) * wpr + col[q]] = D;
            ch = true;
        }
    }
    return ch;
}

// The background 4-connected to the border, by one CTA of kFloodThreads threads over the bit
// planes: in shared memory when both fit (`smem`), else in place in global memory (L1/L2). `fm`
// holds the mask on entry and the free pixels (not mask) after; `out` gets the reached pixels.
// It starts from the free pixels on the border and repeats a vertical and a horizontal sweep
// until a sweep changes nothing. Vertical: a warp per column of words (two at once) carries the
// reached bits down the column and back up, 32 rows at a time by a warp scan of
// D = O | F & D_above. Horizontal: a warp per row (hrow) fills each word's runs from its seeds
// by an addition's carry, and the runs across words by a ballot addition of the carries.
// Every sweep adds a bit or ends the loop, so it ends within h * w + 1 sweeps.
__global__ void __launch_bounds__(kFloodThreads, 1) flood_bits_kernel(uint32_t *__restrict__ fm, uint32_t *__restrict__ out, int h,
                                                                      int w, int wpr, int smem)
{
    extern __shared__ uint32_t planes[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    const int64_t words = int64_t(h) * wpr;
    uint32_t *F = smem ? planes : fm, *O = smem ? planes + words : out;
    for (int64_t i = threadIdx.x; i < words; i += blockDim.x) {
        const int r = int(i / wpr), c = int(i - int64_t(r) * wpr);
        const uint32_t f = ~fm[i] & row_bits(c, w);
        uint32_t edge = (c == 0 ? 1u : 0u) | (c == wpr - 1 ? 1u << ((w - 1) & 31) : 0u);
        if (r == 0 || r == h - 1) edge = 0xFFFFFFFFu;
        F[i] = f;
        O[i] = f & edge;
    }
    __syncthreads();
    bool go = true;
    for (int64_t sweep = 0; go && sweep <= int64_t(h) * w; ++sweep) {
        bool ch = false;
        for (int c = warp; c < wpr; c += 2 * nwarp) {
            if (c + nwarp < wpr) {   // two columns: their scans interleave
                const int col[2] = {c, c + nwarp};
                uint32_t carry[2] = {0u, 0u};
                for (int r0 = 0; r0 < h; r0 += 32) ch |= vblock<2>(F, O, h, wpr, col, 2, r0 + lane, carry);   // down
                __syncwarp();
                carry[0] = carry[1] = 0u;
                for (int r0 = ((h - 1) >> 5) << 5; r0 >= 0; r0 -= 32)   // up: lane 0 is the block's bottom row
                    ch |= vblock<2>(F, O, h, wpr, col, 2, r0 + 31 - lane, carry);
            } else {
                const int col[1] = {c};
                uint32_t carry[1] = {0u};
                for (int r0 = 0; r0 < h; r0 += 32) ch |= vblock<1>(F, O, h, wpr, col, 1, r0 + lane, carry);
                __syncwarp();
                carry[0] = 0u;
                for (int r0 = ((h - 1) >> 5) << 5; r0 >= 0; r0 -= 32) ch |= vblock<1>(F, O, h, wpr, col, 1, r0 + 31 - lane, carry);
            }
            __syncwarp();
        }
        __syncthreads();
        if (wpr <= 32)
            ch |= hsweep<1>(F, O, h, wpr);
        else if (wpr <= 64)
            ch |= hsweep<2>(F, O, h, wpr);
        else if (wpr <= 128)
            ch |= hsweep<4>(F, O, h, wpr);
        else
            ch |= hsweep<8>(F, O, h, wpr);
        go = __syncthreads_or(ch);
    }
    if (smem)
        for (int64_t i = threadIdx.x; i < words; i += blockDim.x) out[i] = O[i];
}

// the transfer of rows [0, rows) of column c of words (shared memory) in one direction: the
// reached bits at the far end are B | A & (those entering at the near end); the blocks' warp scans
// composed in order (identity: A = ~0, B = 0)
__device__ __forceinline__ void vtransfer(const uint32_t *F, const uint32_t *O, int rows, int wpr, int c, bool down,
                                          uint32_t &At, uint32_t &Bt)
{
    const int lane = threadIdx.x & 31, nb = (rows + 31) >> 5;
    At = 0xFFFFFFFFu;
    Bt = 0u;
    for (int k = 0; k < nb; ++k) {
        const int r = down ? 32 * k + lane : 32 * (nb - 1 - k) + 31 - lane;
        uint32_t A = 0xFFFFFFFFu, B = 0u;
        if (r < rows) {
            A = F[int64_t(r) * wpr + c];
            B = O[int64_t(r) * wpr + c];
        }
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t a2 = __shfl_up_sync(0xffffffffu, A, d), b2 = __shfl_up_sync(0xffffffffu, B, d);
            if (lane >= d) {
                B |= A & b2;
                A &= a2;
            }
        }
        const uint32_t a = __shfl_sync(0xffffffffu, A, 31), b = __shfl_sync(0xffffffffu, B, 31);
        Bt = b | (a & Bt);
        At &= a;
    }
}

// The hole filling by a cluster of kFloodCluster CTAs: CTA k holds rows [k hb, (k + 1) hb) of both
// planes in its shared memory (`m`: the mask in global memory; `out`: the reached pixels). A sweep:
// each CTA computes every column's transfer across its band, down and up, from its reached bits
// as they stand; after a cluster barrier each composes the transfers of the bands above (down)
// and below (up) into the carries entering its band, read from the other CTAs' shared memory, and
// sweeps its band down and up with them; then its rows horizontally (hrow). The vertical result
// equals the whole column's (a free run's pixels are reached when any pixel of the run is). The
// sweeps end when no CTA changed a bit (an OR of per-CTA flags, two sets by sweep parity so a flag
// is not rewritten before every CTA has read it); at most h * w + 1 sweeps, as the one-CTA form.
// Every CTA takes the same barriers: the flags they OR are the same.
__global__ void __cluster_dims__(kFloodCluster, 1, 1) __launch_bounds__(kFloodThreads, 1)
    flood_cluster_kernel(const uint32_t *__restrict__ m, uint32_t *__restrict__ out, int h, int w, int wpr, int hb)
{
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ uint32_t band[];
    const int rank = int(cluster.block_rank()), lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    const int r0 = rank * hb, rows = max(0, min(h, r0 + hb) - r0);
    const int64_t words = int64_t(hb) * wpr;
    uint32_t *F = band, *O = band + words, *T = band + 2 * words;   // T: down A, down B, up A, up B (wpr each)
    int *flag = reinterpret_cast<int *>(T + 4 * wpr);
    for (int64_t i = threadIdx.x; i < int64_t(rows) * wpr; i += blockDim.x) {
        const int lr = int(i / wpr), c = int(i - int64_t(lr) * wpr), r = r0 + lr;
        const uint32_t f = ~m[int64_t(r) * wpr + c] & row_bits(c, w);
        uint32_t edge = (c == 0 ? 1u : 0u) | (c == wpr - 1 ? 1u << ((w - 1) & 31) : 0u);
        if (r == 0 || r == h - 1) edge = 0xFFFFFFFFu;
        F[i] = f;
        O[i] = f & edge;
    }
    __syncthreads();
    bool go = true;
    for (int64_t sweep = 0; go && sweep <= int64_t(h) * w; ++sweep) {
        for (int c = warp; c < wpr; c += nwarp) {
            uint32_t a, b;
            vtransfer(F, O, rows, wpr, c, true, a, b);
            if (lane == 0) {
                T[c] = a;
                T[wpr + c] = b;
            }
            vtransfer(F, O, rows, wpr, c, false, a, b);
            if (lane == 0) {
                T[2 * wpr + c] = a;
                T[3 * wpr + c] = b;
            }
        }
        cluster.sync();   // every band's transfers written
        bool ch = false;
        for (int c = warp; c < wpr; c += nwarp) {
            // lane k < kFloodCluster reads band k's transfers; the carries compose them in order
            uint32_t da = 0xFFFFFFFFu, db = 0u, ua = 0xFFFFFFFFu, ub = 0u;
            if (lane < kFloodCluster && lane != rank) {
                const uint32_t *t = cluster.map_shared_rank(T, lane);
                da = t[c];
                db = t[wpr + c];
                ua = t[2 * wpr + c];
                ub = t[3 * wpr + c];
            }
            uint32_t dc = 0u, uc = 0u;
#pragma unroll
            for (int k = 0; k < kFloodCluster; ++k) {
                const uint32_t a = __shfl_sync(0xffffffffu, da, k), b = __shfl_sync(0xffffffffu, db, k);
                if (k < rank) dc = b | (a & dc);
            }
#pragma unroll
            for (int k = kFloodCluster - 1; k >= 0; --k) {
                const uint32_t a = __shfl_sync(0xffffffffu, ua, k), b = __shfl_sync(0xffffffffu, ub, k);
                if (k > rank) uc = b | (a & uc);
            }
            const int col[1] = {c};
            uint32_t carry[1] = {dc};
            for (int b0 = 0; b0 < rows; b0 += 32) ch |= vblock<1>(F, O, rows, wpr, col, 1, b0 + lane, carry);   // down
            __syncwarp();
            carry[0] = uc;
            for (int b0 = ((rows - 1) >> 5) << 5; b0 >= 0; b0 -= 32) ch |= vblock<1>(F, O, rows, wpr, col, 1, b0 + 31 - lane, carry);
            __syncwarp();
        }
        __syncthreads();
        if (wpr <= 32)
            ch |= hsweep<1>(F, O, rows, wpr);
        else if (wpr <= 64)
            ch |= hsweep<2>(F, O, rows, wpr);
        else if (wpr <= 128)
            ch |= hsweep<4>(F, O, rows, wpr);
        else
            ch |= hsweep<8>(F, O, rows, wpr);
        const int any = __syncthreads_or(ch);
        if (threadIdx.x == 0) flag[sweep & 1] = any;
        cluster.sync();   // every CTA's flag written, every band's carries read
        int all = 0;
        if (threadIdx.x < kFloodCluster) all = *cluster.map_shared_rank(flag + (sweep & 1), int(threadIdx.x));
        go = __syncthreads_or(all);
    }
    cluster.sync();   // no CTA leaves while another may still read its flags
    for (int64_t i = threadIdx.x; i < int64_t(rows) * wpr; i += blockDim.x) out[int64_t(r0) * wpr + i] = O[i];
}

// the filled mask: every pixel the border's background does not reach
__global__ void __launch_bounds__(256) fill_bits_kernel(const uint32_t *__restrict__ outside, int h, int w, int wpr,
                                                        uint8_t *__restrict__ mask)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= int64_t(h) * w) return;
    const int r = int(i / w), c = int(i % w);
    mask[i] = ((outside[int64_t(r) * wpr + (c >> 5)] >> (c & 31)) & 1u) ^ 1u;
}

#endif   // __CUDACC__

}   // namespace b200
