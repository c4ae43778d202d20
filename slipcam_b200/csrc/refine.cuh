// refine.cuh -- the exact refinement of the tensor-core form's peaks. The FP16 DFT-GEMMs leave an
// error of about 3e-4 in each surface value; the sub-pixel offset, the peak value and the
// covariance are read from the 3 x 3 values around the peak alone (cxx/surface.h:71-146), so this
// kernel recomputes those nine values exactly -- the integer correlation sum_ij ref(i, j) x(i + u,
// j + v) of the reference window and the frame in 32-bit integers, normalized as the exact form does
// (i8::rho) -- replaces them in the SNR patch's sum of squares, and writes the pair's outputs again.
// When an exact neighbour is larger than the peak (the FP16 argmax fell on the wrong side of a tie
// between adjacent shifts), the peak climbs to it and the SNR patch around the new peak is summed
// exactly; so is the patch of windows up to 32 px, whose small surfaces weigh the FP16 errors more
// in the SNR. One warp per pair, the reference rows shared between the lanes; the pairs whose patch
// is summed exactly are queued for tc_patch_kernel, a CTA each.
#pragma once

#include "corr_i8.cuh"

namespace b200 {

#ifdef __CUDACC__

__global__ void __launch_bounds__(256) tc_refine_kernel(CorrArgs a, const uint8_t *refwin, const int *sref,
                                                        int *queue)
{
    const int lane = threadIdx.x & 31;
    const int64_t p = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;   // the pair (its output index)
    if (p >= int64_t(a.nwin) * a.nf) return;
    const PeakInfo &pi = a.peaks[p];
    const int k = int(p % a.nwin), f = int(p / a.nwin);
    const i8::Pair o = i8::pair(a, k, f);
    const int W = a.W, M = a.M, n = W * W;
    // only pairs the tensor-core kernel found a peak for (the search window inside the frame)
    if (!o.ok || !pi.valid || pi.u < 0 || pi.u >= M || pi.v < 0 || pi.v >= M) return;
    const uint8_t *chip = a.frames + o.f * a.fstride + int64_t(o.sy) * a.pitch + o.sx;
    const uint8_t *ref = refwin + size_t(k) * W * W;
    const float scale = float(1.0 / (double(n) * double(a.norm[k])));
    const int2 *bt0 = a.bstat + size_t(o.f) * a.dinv_fstride + size_t(o.sy) * a.dpitch + o.sx;
    const int sr = sref[k];
    int pu = pi.u, pv = pi.v;
    float fit[9];
    int u0 = 0, u1 = 0, v0 = 0, v1 = 0;
    bool moved = false;
    for (int step = 0; step < 8; ++step) {
        u0 = pu > 0 ? -1 : 0;   // the neighbours inside the surface
        u1 = pu < M - 1 ? 1 : 0;
        v0 = pv > 0 ? -1 : 0;
        v1 = pv < M - 1 ? 1 : 0;
        // lanes along the columns j (coalesced bytes, the chip rows cached in L1), rows in turn
        int s[3][3] = {};
        for (int i = 0; i < W; ++i) {
            const uint8_t *rr = ref + size_t(i) * W;
            for (int j = lane; j < W; j += 32) {
                const uint32_t x = __ldg(rr + j);
#pragma unroll
                for (int du = -1; du <= 1; ++du) {
                    if (du < u0 || du > u1) continue;
                    // chip row pu + du + i, columns pv + v0 + j .. pv + v1 + j (inside [0, L))
                    const uint8_t *cr = chip + int64_t(pu + du + i) * a.pitch + pv + j;
                    const uint32_t bm = v0 < 0 ? __ldg(cr - 1) : 0u, b0 = __ldg(cr), bp = v1 > 0 ? __ldg(cr + 1) : 0u;
                    s[du + 1][0] += int(x * bm);
                    s[du + 1][1] += int(x * b0);
                    s[du + 1][2] += int(x * bp);
                }
            }
        }
#pragma unroll
        for (int t = 0; t < 9; ++t)
            for (int d = 16; d > 0; d >>= 1) s[t / 3][t % 3] += __shfl_xor_sync(0xffffffffu, s[t / 3][t % 3], d);
        // the exact values, and the best of the 3 x 3 (the reference's rule: the larger, the first in
        // raster order if equal); every lane computes the same
        float best = -2.0f;
        int bu = pu, bv = pv, bat = INT_MAX;
        for (int du = u0; du <= u1; ++du)
            for (int dv = v0; dv <= v1; ++dv) {
                const int t = (du + 1) * 3 + dv + 1;
                const int2 st = __ldg(bt0 + int64_t(pu + du) * a.dpitch + pv + dv);
                fit[t] = i8::rho(uint32_t(s[du + 1][dv + 1]), st, n, sr, scale);
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

// the shared memory tc_patch_kernel needs: the reference window and the chip region of the patch
inline size_t tc_patch_smem(int W, int M, int stat)
{
    const int n = stat < M ? stat : M;
    return size_t(W) * W + size_t(n + W - 1) * (n + W - 1);
}

// the SNR patch of each queued pair summed exactly (one CTA per pair: the reference window and the
// chip region in shared memory, a warp per patch position), then the pair's outputs
__global__ void __launch_bounds__(256) tc_patch_kernel(CorrArgs a, const uint8_t *refwin, const int *sref,
                                                       const int *queue)
{
    extern __shared__ unsigned char sm[];
    __shared__ double s_sum[8];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int W = a.W, M = a.M, n = W * W;
    const int count = queue[0];
    for (int t = blockIdx.x; t < count; t += gridDim.x) {
        const int p = queue[1 + t];
        const PeakInfo &pi = a.peaks[p];
        const int k = p % a.nwin, f = p / a.nwin;
        const i8::Pair o = i8::pair(a, k, f);
        const int pu = pi.u, pv = pi.v;
        int i0, i1, j0, j1;
        snr_patch(M, a.stat, pu, pv, i0, i1, j0, j1);
        const int rows = i1 - i0 + W - 1, cols = j1 - j0 + W - 1;
        unsigned char *sref_w = sm, *schip = sm + size_t(W) * W;
        const uint8_t *ref = refwin + size_t(k) * W * W;
        for (int e = tid; e < W * W; e += 256) sref_w[e] = __ldg(ref + e);
        const uint8_t *chip = a.frames + o.f * a.fstride + int64_t(o.sy + i0) * a.pitch + o.sx + j0;
        for (int e = tid; e < rows * cols; e += 256) schip[e] = __ldg(chip + int64_t(e / cols) * a.pitch + e % cols);
        __syncthreads();
        const float scale = float(1.0 / (double(n) * double(a.norm[k])));
        const int2 *bt0 = a.bstat + size_t(o.f) * a.dinv_fstride + size_t(o.sy) * a.dpitch + o.sx;
        const int pw = j1 - j0, np = (i1 - i0) * pw;
        double sum = 0.0;
        for (int idx = warp; idx < np; idx += 8) {
            const int du = idx / pw, dv = idx % pw;
            int acc = 0;
            for (int i = 0; i < W; ++i) {   // lanes along the columns: conflict-free shared memory
                const unsigned char *rr = sref_w + i * W, *cr = schip + (du + i) * cols + dv;
                for (int j = lane; j < W; j += 32) acc += int(uint32_t(rr[j]) * uint32_t(cr[j]));
            }
            for (int d = 16; d > 0; d >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, d);
            const int u = i0 + du, v = j0 + dv;
            const float x = i8::rho(uint32_t(acc), __ldg(bt0 + int64_t(u) * a.dpitch + v), n, sref[k], scale);
            sum += double(x) * double(x);
        }
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
