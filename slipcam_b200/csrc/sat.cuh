// sat.cuh -- the exact summed-area tables of the frames and the per-shift variance denominators.
//
// For each frame (h x w uint8) the tables are (h + 1) x (w + 1) with a first row and column of
// zeros, as the reference's (slipcam cxx/cpu.cpp:24-42, cxx/cuda.cu:72-110):
//   sat  = sum of x   as uint32, exact modulo 2^32 (every box sum below 2^32 -- all boxes up to
//          16.8 M pixels -- comes out exact from the 4-corner difference in wrapping arithmetic;
//          the table itself is exact outright for frames below 16.8 M pixels)
//   sat2 = sum of x^2 as int64, exact
// Two passes: a warp scans each row (16-byte stores per lane group, coalesced); then each column
// is summed in segments by a (32 x 8) block with a shared-memory carry.
//
// dinv_kernel then gives, for every W x W box of a frame, 1 / sqrt(v / n) with v = n S2 - S^2 from
// the integer box sums in int64 and the root in FP64 (0 where v <= 0, the reference's
// "not normalizable" case, cxx/surface.h:30-35).
#pragma once

#include "common.cuh"

namespace b200 {

#ifdef __CUDACC__

// one warp per row: rows y + 1 of the tables, and row 0 (zeros) by the warp of row 0
__global__ void __launch_bounds__(256) sat_rows_kernel(const uint8_t *frames, int64_t fstride, int pitch,
                                                       int h, int w, uint32_t *sat, int64_t *sat2, int64_t sfs)
{
    const int f = blockIdx.y, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int y = blockIdx.x * 8 + warp;
    if (y >= h) return;
    const size_t ss = size_t(w) + 1;
    uint32_t *s = sat + f * sfs;
    int64_t *s2 = sat2 + f * sfs;
    if (y == 0)
        for (int x = lane; x <= w; x += 32) {
            s[x] = 0;
            s2[x] = 0;
        }
    const uint8_t *row = frames + f * fstride + int64_t(y) * pitch;
    uint32_t *o = s + (y + 1) * ss;
    int64_t *o2 = s2 + (y + 1) * ss;
    if (lane == 0) {
        o[0] = 0;
        o2[0] = 0;
    }
    uint32_t carry = 0;
    int64_t carry2 = 0;
    // lane l takes pixels x0 + l, x0 + 32 + l, ...: every load and store of the warp is contiguous
    for (int x0 = 0; x0 < w; x0 += 128) {
        uint32_t v[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int x = x0 + 32 * i + lane;
            v[i] = x < w ? uint32_t(__ldg(row + x)) : 0u;
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            uint32_t sa = v[i];
            int64_t sb = int64_t(v[i] * v[i]);
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t ta = __shfl_up_sync(0xffffffffu, sa, d);
                const int64_t tb = __shfl_up_sync(0xffffffffu, sb, d);
                if (lane >= d) {
                    sa += ta;
                    sb += tb;
                }
            }
            const int x = x0 + 32 * i + lane;
            if (x < w) {
                o[1 + x] = carry + sa;
                o2[1 + x] = carry2 + sb;
            }
            carry += __shfl_sync(0xffffffffu, sa, 31);
            carry2 += __shfl_sync(0xffffffffu, sb, 31);
        }
    }
}

// the column sums of the row prefix sums; block (32, 8): 32 columns, 8 segments of rows
__global__ void __launch_bounds__(256) sat_cols_kernel(int h, int w, uint32_t *sat, int64_t *sat2, int64_t sfs)
{
    __shared__ uint32_t c32[8][32];
    __shared__ long long c64[8][32];
    const int f = blockIdx.y, tx = threadIdx.x, ty = threadIdx.y;
    const int x = blockIdx.x * 32 + tx;
    const size_t ss = size_t(w) + 1;
    uint32_t *s = sat + f * sfs;
    int64_t *s2 = sat2 + f * sfs;
    const int seg = (h + 7) / 8;
    const int r0 = 1 + ty * seg, r1 = min(h, (ty + 1) * seg) + 1;
    uint32_t a = 0;
    long long b = 0;
    if (x <= w)
        for (int r = r0; r < r1; ++r) {
            a += s[r * ss + x];
            b += s2[r * ss + x];
        }
    constexpr int B = 8;   // rows loaded together in the second pass (its stores would otherwise order them)
    c32[ty][tx] = a;
    c64[ty][tx] = b;
    __syncthreads();
    uint32_t ca = 0;
    long long cb = 0;
    for (int t = 0; t < ty; ++t) {
        ca += c32[t][tx];
        cb += c64[t][tx];
    }
    if (x <= w)
        for (int rb = r0; rb < r1; rb += B) {
            uint32_t la[B];
            long long lb[B];
#pragma unroll
            for (int j = 0; j < B; ++j)
                if (rb + j < r1) {
                    la[j] = s[(rb + j) * ss + x];
                    lb[j] = s2[(rb + j) * ss + x];
                }
#pragma unroll
            for (int j = 0; j < B; ++j)
                if (rb + j < r1) {
                    ca += la[j];
                    s[(rb + j) * ss + x] = ca;
                    cb += lb[j];
                    s2[(rb + j) * ss + x] = cb;
                }
        }
}

// dinv[y][x] (row pitch dpitch floats) for the W x W boxes at (y, x), y <= h - W, x <= w - W; and,
// when bstat is given, {the box's pixel sum, the bits of its dinv} in the same layout
__global__ void __launch_bounds__(128) dinv_kernel(const uint32_t *sat, const int64_t *sat2, int64_t sfs,
                                                   int h, int w, int W, float *dinv, int64_t dfs, int dpitch,
                                                   int2 *bstat = nullptr)
{
    const int x = blockIdx.x * 128 + threadIdx.x, y = blockIdx.y, f = blockIdx.z;
    if (x > w - W || y > h - W) return;
    const size_t ss = size_t(w) + 1;
    const uint32_t *s = sat + f * sfs;
    const int64_t *s2 = sat2 + f * sfs;
    const size_t a = y * ss + x, b = a + W, c = a + W * ss, d = c + W;
    const int64_t bs = int64_t(uint32_t(s[d] - s[b] - s[c] + s[a]));
    const int64_t bs2 = s2[d] - s2[b] - s2[c] + s2[a];
    const int64_t n = int64_t(W) * W;
    const int64_t v = n * bs2 - bs * bs;
    const float di = v > 0 ? float(1.0 / sqrt(double(v) / double(n))) : 0.0f;
    dinv[f * dfs + size_t(y) * dpitch + x] = di;
    if (bstat) bstat[f * dfs + size_t(y) * dpitch + x] = make_int2(int(bs), __float_as_int(di));
}

#endif   // __CUDACC__

}   // namespace b200
