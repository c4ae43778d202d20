// refine.cuh -- the exact refinement of the tensor-core form's peaks. The FP16 DFT-GEMMs leave an
// error of about 3e-4 in each surface value; the sub-pixel offset, the peak value and the
// covariance are read from the 3 x 3 values around the peak alone (cxx/surface.h:71-146), so this
// kernel recomputes those nine values exactly -- the integer correlation sum_ij ref(i, j) x(i + u,
// j + v) of the reference window and the frame in 32-bit integers, normalized as the exact form does
// (i8::rho) -- replaces them in the SNR patch's sum of squares, and writes the pair's outputs again.
// When an exact neighbour is larger than the peak (the FP16 argmax fell on the wrong side of a tie
// between adjacent shifts), the peak climbs to it and the SNR patch around the new peak is summed
// exactly; so is the patch of windows up to 32 px, whose small surfaces weigh the FP16 errors more
// in the SNR. One warp per pair, its reference window and chip region staged in shared memory and
// summed with dp4a; the pairs whose patch is summed exactly are queued for tc_patch_kernel, a CTA
// each.
#pragma once

#include "corr_i8.cuh"

namespace b200 {

// the bytes of a reference row held in shared memory, padded with zeros to whole words
__host__ __device__ inline int refine_rp(int W) { return (W + 3) & ~3; }
// the bytes of a staged frame-region row: whole words and one more word for the shifted reads
__host__ __device__ inline int refine_tp(int nc) { return ((nc + 3) & ~3) + 4; }

// the bytes of a staged region row on the 16-byte path: the row from its aligned 16-byte chunk
// on (up to 15 bytes before the region), and the words the sums read past it
__host__ __device__ inline int refine_rt16(int W) { return (4 * (((W + 13) >> 2) + 2) + 15) & ~15; }

// the refinement's shared memory: the CTA's reference window once, then each warp's chip region of
// its 3 x 3 (the larger of the word and 16-byte layouts)
__host__ __device__ inline size_t refine_ref_smem(int W) { return (size_t(W) * refine_rp(W) + 15) & ~size_t(15); }
__host__ __device__ inline size_t refine_tile_smem(int W)
{
    const size_t words = size_t(W + 2) * refine_tp(W + 2), b16 = size_t(W + 2) * refine_rt16(W);
    return ((words > b16 ? words : b16) + 15) & ~size_t(15);
}

// the shared memory tc_patch_kernel needs: the reference window and the chip region of the patch
__host__ __device__ inline size_t tc_patch_smem(int W, int M, int stat)
{
    const int n = stat < M ? stat : M;
    return size_t(W) * refine_rp(W) + size_t(n + W - 1) * refine_tp(n + W - 1);
}

#ifdef __CUDACC__

// the reference window (W x W bytes at ref) into dst, rows of rp bytes zero-padded
__device__ __forceinline__ void stage_ref(unsigned char *dst, const uint8_t *ref, int W, int t, int nt)
{
    const int rp = refine_rp(W);
    if ((W & 3) == 0 && (reinterpret_cast<uintptr_t>(ref) & 3) == 0) {
        const uint32_t *s = reinterpret_cast<const uint32_t *>(ref);
        uint32_t *d = reinterpret_cast<uint32_t *>(dst);
        for (int e = t; e < W * W / 4; e += nt) d[e] = __ldg(s + e);
    } else {
        for (int e = t; e < W * rp; e += nt) {
            const int i = e / rp, j = e - i * rp;
            dst[e] = j < W ? __ldg(ref + i * W + j) : 0;
        }
    }
}

// nr rows of nc bytes of the frame from src (row pitch `pitch`) into dst, rows of refine_tp(nc)
// bytes; whole words when the frame rows start on 4-byte boundaries (every aligned word read holds
// a byte of the region, so no read leaves the region's rows)
__device__ __forceinline__ void stage_region(unsigned char *dst, const uint8_t *src, int64_t pitch, bool words, int nr,
                                             int nc, int t, int nt)
{
    const int tp = refine_tp(nc), wpr = tp / 4;
    if (words) {
        uint32_t *d = reinterpret_cast<uint32_t *>(dst);
        for (int e = t; e < nr * wpr; e += nt) {
            const int r = e / wpr, w = e - r * wpr;
            uint32_t v = 0;
            if (4 * w < nc) {
                const uintptr_t base = reinterpret_cast<uintptr_t>(src + int64_t(r) * pitch) + 4 * w;
                const uint32_t *al = reinterpret_cast<const uint32_t *>(base & ~uintptr_t(3));
                const int sh = int(base & 3);
                const uint32_t lo = __ldg(al), hi = (sh != 0 && 4 * w + 4 - sh < nc) ? __ldg(al + 1) : 0u;
                v = __funnelshift_r(lo, hi, 8 * sh);
            }
            d[e] = v;
        }
    } else {
        for (int e = t; e < nr * tp; e += nt) {
            const int r = e / tp, c = e - r * tp;
            dst[e] = c < nc ? __ldg(src + int64_t(r) * pitch + c) : 0;
        }
    }
}

// 16 bytes global -> shared without the registers (cp.async, cached in L2 only); the first n of
// them read, the rest zero
__device__ __forceinline__ void cp16(unsigned char *dst, const uint8_t *src, int n)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(uint32_t(__cvta_generic_to_shared(dst))),
                 "l"(src), "r"(n)
                 : "memory");
}
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// bytes t .. t + 3 (t in 0 .. 5) of the 12 bytes x0 x1 x2 (little-endian)
__device__ __forceinline__ uint32_t bytes_at(uint32_t x0, uint32_t x1, uint32_t x2, int t)
{
    return t < 4 ? __funnelshift_r(x0, x1, 8 * t) : __funnelshift_r(x1, x2, 8 * (t - 4));
}

// the exact refinement: one warp per pair, its reference window and 3 x 3 chip region staged in
// the warp's part of the shared memory, the nine sums taken with dp4a (four uint8 products a
// step), the lanes along the words of the reference rows. When the frame rows start on 16-byte
// boundaries (and W is a multiple of 4) the staging is 16-byte cp.async copies, many in flight per
// lane: a region row is copied from its aligned chunk on, the last chunk only up to the frame's
// width, and the sums read it at the row's byte offset
// A CTA takes one window and blockDim / 32 of its frames, a warp per pair: the reference window is
// staged once for the CTA.
__global__ void __launch_bounds__(256, 4) tc_refine_kernel(CorrArgs a, const uint8_t *refwin, const int *sref,
                                                           int *queue)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int cpw = (a.nf + nw - 1) / nw;   // CTAs per window
    const int k = blockIdx.x / cpw, f = (blockIdx.x - k * cpw) * nw + warp;
    if (k >= a.nwin) return;   // the whole CTA
    const int W = a.W, M = a.M, n = W * W;
    unsigned char *sref_w = smem;
    const uint8_t *ref = refwin + size_t(k) * W * W;
    // the 16-byte path: frame rows on 16-byte boundaries, reference rows of whole words
    const bool b16 = ((reinterpret_cast<uintptr_t>(a.frames) | uintptr_t(a.pitch) | uintptr_t(a.fstride)) & 15) == 0 &&
                     (W & 3) == 0;
    if (b16) {
        for (int e = threadIdx.x; e < W * W / 16; e += blockDim.x) cp16(sref_w + 16 * e, ref + 16 * e, 16);   // W^2 = 16 (W/4)^2
        cp_wait_all();
    } else {
        stage_ref(sref_w, ref, W, threadIdx.x, blockDim.x);
    }
    __syncthreads();   // the CTA's one barrier: its warps may leave from here on
    if (f >= a.nf) return;
    const int64_t p = int64_t(f) * a.nwin + k;   // the pair (its output index)
    const PeakInfo &pi = a.peaks[p];
    const i8::Pair o = i8::pair(a, k, f);
    // only pairs the tensor-core kernel found a peak for (the search window inside the frame)
    if (!o.ok || !pi.valid || pi.u < 0 || pi.u >= M || pi.v < 0 || pi.v >= M) return;
    unsigned char *tile = smem + refine_ref_smem(W) + size_t(warp) * refine_tile_smem(W);
    const uint8_t *chip = a.frames + o.f * a.fstride + int64_t(o.sy) * a.pitch + o.sx;
    const bool words = ((a.pitch | int(a.fstride & 3) | int(reinterpret_cast<uintptr_t>(a.frames) & 3)) & 3) == 0;
    const float scale = float(1.0 / (double(n) * double(a.norm[k])));
    const int2 *bt0 = a.bstat + size_t(o.f) * a.dinv_fstride + size_t(o.sy) * a.dpitch + o.sx;
    const int sr = sref[k];
    const int wpr = refine_rp(W) / 4;
    const int rt = refine_rt16(W);
    int pu = pi.u, pv = pi.v;
    float fit[9];
    int u0 = 0, u1 = 0, v0 = 0, v1 = 0;
    bool moved = false;
    for (int step = 0; step < 8; ++step) {
        u0 = pu > 0 ? -1 : 0;   // the neighbours inside the surface
        u1 = pu < M - 1 ? 1 : 0;
        v0 = pv > 0 ? -1 : 0;
        v1 = pv < M - 1 ? 1 : 0;
        const int nr = W + u1 - u0, nc = W + v1 - v0, tp = refine_tp(nc);
        const int c0 = o.sx + pv + v0;   // the region's first frame column
        const int sh = c0 & 15;          // its byte in the aligned chunk (the same on every row)
        __syncwarp();
        if (b16) {
            // rows of nch chunks from the aligned column c0 - sh; a row's last chunk stops at the
            // frame's width (the region ends inside the frame, so every chunk starts inside the row)
            const int nch = (sh + nc + 15) >> 4;
            const uint8_t *r0 = chip + int64_t(pu + u0) * a.pitch + (pv + v0 - sh);
            for (int e = lane; e < nr * nch; e += 32) {
                const int r = e / nch, c = e - r * nch;
                const int col = c0 - sh + 16 * c;
                cp16(tile + r * rt + 16 * c, r0 + int64_t(r) * a.pitch + 16 * c, min(16, a.w - col));
            }
            cp_wait_all();
        } else {
            stage_region(tile, chip + int64_t(pu + u0) * a.pitch + pv + v0, a.pitch, words, nr, nc, lane, 32);
        }
        __syncwarp();
        uint32_t s[3][3] = {};
        if (b16 && wpr <= 32) {
            // lane (w, rg) takes word column w of the reference rows ia .. ib - 1 and slides down them
            // with the three staged region rows of the 3 x 3 in registers: per row one reference word
            // and one new region row of three words
            const int sw = sh >> 2, sb = sh & 3;   // the region's first word and byte in a staged row
            const int nrg = 32 / wpr, rpl = (W + nrg - 1) / nrg;
            const int w = lane % wpr, rg = lane / wpr;
            const int ia = rg < nrg ? rg * rpl : W, ib = min(W, ia + rpl);
            if (ia < ib) {
                const uint32_t *col = reinterpret_cast<const uint32_t *>(tile) + w + sw;
                const int rw4 = rt >> 2;   // words per staged row
                uint32_t a0 = col[ia * rw4], a1 = col[ia * rw4 + 1], a2 = col[ia * rw4 + 2];
                uint32_t b0 = col[(ia + 1) * rw4], b1 = col[(ia + 1) * rw4 + 1], b2 = col[(ia + 1) * rw4 + 2];
                for (int i = ia; i < ib; ++i) {
                    const uint32_t *cr = col + (i + 2) * rw4;   // row i + 2 (inside the W + 2 staged rows)
                    const uint32_t c0 = cr[0], c1 = cr[1], c2 = cr[2];
                    const uint32_t rw = *reinterpret_cast<const uint32_t *>(sref_w + i * W + 4 * w);
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        if (d > v1 - v0) continue;
                        s[0][d] = __dp4a(rw, bytes_at(a0, a1, a2, sb + d), s[0][d]);
                        if (u1 - u0 >= 1) s[1][d] = __dp4a(rw, bytes_at(b0, b1, b2, sb + d), s[1][d]);
                        if (u1 - u0 >= 2) s[2][d] = __dp4a(rw, bytes_at(c0, c1, c2, sb + d), s[2][d]);
                    }
                    a0 = b0;
                    a1 = b1;
                    a2 = b2;
                    b0 = c0;
                    b1 = c1;
                    b2 = c2;
                }
            }
        } else if (b16) {
            const int sw = sh >> 2, sb = sh & 3;   // the region's first word and byte in a staged row
            for (int it = lane; it < W * wpr; it += 32) {
                const int i = it / wpr, w = it - i * wpr;
                const uint32_t rw = *reinterpret_cast<const uint32_t *>(sref_w + i * W + 4 * w);
#pragma unroll
                for (int du = 0; du < 3; ++du) {
                    if (du > u1 - u0) continue;
                    const uint32_t *row = reinterpret_cast<const uint32_t *>(tile + (i + du) * rt) + w + sw;
                    const uint32_t x0 = row[0], x1 = row[1], x2 = row[2];
#pragma unroll
                    for (int d = 0; d < 3; ++d)
                        if (d <= v1 - v0) s[du][d] = __dp4a(rw, bytes_at(x0, x1, x2, sb + d), s[du][d]);
                }
            }
        } else {
            for (int it = lane; it < W * wpr; it += 32) {
                const int i = it / wpr, w = it - i * wpr;
                const uint32_t rw = *reinterpret_cast<const uint32_t *>(sref_w + i * refine_rp(W) + 4 * w);
#pragma unroll
                for (int du = 0; du < 3; ++du) {
                    if (du > u1 - u0) continue;
                    const uint32_t *row = reinterpret_cast<const uint32_t *>(tile + (i + du) * tp) + w;
                    const uint32_t lo = row[0], hi = row[1];
#pragma unroll
                    for (int d = 0; d < 3; ++d)
                        if (d <= v1 - v0) s[du][d] = __dp4a(rw, d ? __funnelshift_r(lo, hi, 8 * d) : lo, s[du][d]);
                }
            }
        }
#pragma unroll
        for (int t = 0; t < 9; ++t)
            for (int dd = 16; dd > 0; dd >>= 1) s[t / 3][t % 3] += __shfl_xor_sync(0xffffffffu, s[t / 3][t % 3], dd);
        // the exact values, and the best of the 3 x 3 (the reference's rule: the larger, the first in
        // raster order if equal); every lane computes the same
        float best = -2.0f;
        int bu = pu, bv = pv, bat = INT_MAX;
        for (int du = u0; du <= u1; ++du)
            for (int dv = v0; dv <= v1; ++dv) {
                const int t = (du + 1) * 3 + dv + 1;
                const int2 st = __ldg(bt0 + int64_t(pu + du) * a.dpitch + pv + dv);
                fit[t] = i8::rho(s[du - u0][dv - v0], st, n, sr, scale);
                const int at = (pu + du) * M + pv + dv;
                if (fit[t] > best || (fit[t] == best && at < bat)) {
                    best = fit[t];
                    bat = at;
                    bu = pu + du;
                    bv = pv + dv;
                }
            }
        if ((bu == pu && bv == pv) || step == 7) break;   // fit[] holds the values around (pu, pv)
        pu = bu;   // a neighbour is the larger: the FP16 argmax was an adjacent near-tie
        pv = bv;
        moved = true;
    }
    if (lane != 0) return;
    if (moved || W <= 32) {
        // a new patch, or a small window's (its FP16 errors weigh more in the SNR): the whole patch
        // exact, by tc_patch_kernel, a CTA per queued pair; queue[0] counts them
        PeakInfo &q = a.peaks[p];
        q.valid = 2;
        q.u = pu;
        q.v = pv;
        for (int t = 0; t < 9; ++t) q.fit[t] = fit[t];
        queue[1 + atomicAdd(queue, 1)] = int(p);
        return;
    }
    int i0, i1, j0, j1;
    snr_patch(M, a.stat, pu, pv, i0, i1, j0, j1);
    double sum = pi.sum;   // the tensor-core patch with its 3 x 3 replaced
    for (int du = u0; du <= u1; ++du)
        for (int dv = v0; dv <= v1; ++dv) {
            const int t = (du + 1) * 3 + dv + 1;
            sum += double(fit[t]) * double(fit[t]) - double(pi.fit[t]) * double(pi.fit[t]);
        }
    peak_outputs(fit + 4, 3, M, pu, pv, a.R, o.gy, o.gx, n, sum, (i1 - i0) * (j1 - j0), p, a.offset, a.peak, a.snr,
                 a.cov);
}

// the SNR patch of each queued pair summed exactly: one CTA per pair, the reference window and the
// patch's chip region in shared memory, a thread per patch position (dp4a over the reference rows'
// words), then the pair's outputs
__global__ void __launch_bounds__(256) tc_patch_kernel(CorrArgs a, const uint8_t *refwin, const int *sref,
                                                       const int *queue)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ double s_sum[8];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int W = a.W, M = a.M, n = W * W, rp = refine_rp(W), wpr = rp / 4;
    const bool words = ((a.pitch | int(a.fstride & 3) | int(reinterpret_cast<uintptr_t>(a.frames) & 3)) & 3) == 0;
    const int count = queue[0];
    unsigned char *sref_w = smem, *tile = smem + size_t(W) * rp;
    for (int t = blockIdx.x; t < count; t += gridDim.x) {
        const int p = queue[1 + t];
        const PeakInfo &pi = a.peaks[p];
        const int k = p % a.nwin, f = p / a.nwin;
        const i8::Pair o = i8::pair(a, k, f);
        const int pu = pi.u, pv = pi.v;
        int i0, i1, j0, j1;
        snr_patch(M, a.stat, pu, pv, i0, i1, j0, j1);
        const int pw = j1 - j0, np = (i1 - i0) * pw;
        const int nr = i1 - i0 + W - 1, nc = pw + W - 1, tp = refine_tp(nc);
        stage_ref(sref_w, refwin + size_t(k) * W * W, W, tid, 256);
        stage_region(tile, a.frames + o.f * a.fstride + int64_t(o.sy + i0) * a.pitch + o.sx + j0, a.pitch, words, nr, nc,
                     tid, 256);
        __syncthreads();
        const float scale = float(1.0 / (double(n) * double(a.norm[k])));
        const int2 *bt0 = a.bstat + size_t(o.f) * a.dinv_fstride + size_t(o.sy) * a.dpitch + o.sx;
        double sum = 0.0;
        for (int q = tid; q < np; q += 256) {
            const int du = q / pw, dv = q - du * pw;
            const int sh = 8 * (dv & 3);
            uint32_t acc = 0;
            for (int i = 0; i < W; ++i) {
                const uint32_t *rr = reinterpret_cast<const uint32_t *>(sref_w + i * rp);
                const uint32_t *cr = reinterpret_cast<const uint32_t *>(tile + (du + i) * tp + (dv & ~3));
                for (int w = 0; w < wpr; ++w) acc = __dp4a(rr[w], __funnelshift_r(cr[w], cr[w + 1], sh), acc);
            }
            const float x = i8::rho(acc, __ldg(bt0 + int64_t(i0 + du) * a.dpitch + j0 + dv), n, sref[k], scale);
            sum += double(x) * double(x);
        }
        for (int d = 16; d > 0; d >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, d);
        if (lane == 0) s_sum[warp] = sum;
        __syncthreads();
        if (tid == 0) {
            double tot = 0.0;
            for (int w = 0; w < 8; ++w) tot += s_sum[w];
            peak_outputs(pi.fit + 4, 3, M, pu, pv, a.R, o.gy, o.gx, n, tot, np, p, a.offset, a.peak, a.snr, a.cov);
        }
        __syncthreads();   // the shared memory is the next pair's
    }
}

#endif   // __CUDACC__

}   // namespace b200
