// corr_i8.cuh -- the exact tensor-core form: the correlation of every (window, frame) pair summed
// directly on the 5th-generation tensor cores in integers (tcgen05.mma kind::i8, uint8 x uint8
// products, int32 accumulation in TMEM), so the numerator of the normalized correlation carries no
// rounding at all; only the final normalization is floating point.
//
// The reference (slipcam cxx/cpu.cpp:117-167, cxx/cuda.cu:317-360) correlates the zero-mean
// reference window r0 = ref - mean with the search window x by FFTs in FP32. Because the sum of
// r0 is zero, the same numerator is
//     c(u, v) = sum_ij r0(i, j) x(i + u, j + v) = (n S_rx(u, v) - S_ref S_x(u, v)) / n,
//     S_rx(u, v) = sum_ij ref(i, j) x(i + u, j + v),   n = W^2,
// S_ref the window's pixel sum and S_x(u, v) the search box's pixel sum (exact, from the
// summed-area tables). S_rx is the integer GEMM below; n S_rx - S_ref S_x is exact in int64, and
// rho = c * dinv / norm follows cxx/surface.h:30-35 with the variance denominator dinv of the FP32
// form.
//
// The GEMM. For reference row i, with the chip (the L x L search window) in shared memory:
//     D[v][u] += sum_j' T_i[v][j'] X[i + u][j'],   T_i[v][j'] = ref(i, j' - v) (0 outside [0, W))
// A = T_i, a Toeplitz matrix of one reference row (128 lanes v x K = j'), is built by the producer
// warps straight into TMEM (tcgen05.st): lane v holds the row shifted right by v. B = the chip
// rows i .. i + NU - 1: the chip is stored as 16-byte column blocks whose rows are 16 bytes apart
// (the descriptor's 8-row stride is 128 bytes), so the operand for row offset i is the same
// descriptor started i * 16 bytes on -- the sliding window over the chip's rows costs nothing.
// D (lanes v, columns u) accumulates over i and the K chunks of 32 columns; lanes v >= 128 go to a
// second lane tile (searches above 63 px). Rows u >= M, lanes v >= M and chip columns >= L only
// reach outputs outside the M x M surface, which are never read.
//
// Warps: eight producers (two per TMEM lane quadrant, taking alternate stages) fill a ring of
// stages, one reference row each (every K chunk of both lane tiles, 8 TMEM columns = 128 x 32 bytes
// per chunk); four epilogue
// warps load the next group's chips into shared memory and reduce the previous group's surfaces
// (normalization, argmax with the reference's tie rule, SNR patch, 3 x 3 fit in FP64); one thread
// issues the MMAs, one wait and one commit per stage. A group is F frames of one window, so the
// Toeplitz operands serve F chips; with two accumulator buffers a group's epilogue runs under the
// next group's MMAs. Every wait is bounded (about two seconds of global time); when one gives up,
// the kernel writes status 3 and every role runs out its loop without work.
#pragma once

#include <algorithm>
#include <climits>
#include <type_traits>

#include "corr_fft.cuh"
#include "tc.cuh"

namespace b200 {

constexpr int kI8Producers = 8;   // two per TMEM lane quadrant, taking alternate ring stages
constexpr int kI8Epilogue = 4;
constexpr int kI8Threads = 32 * (kI8Producers + kI8Epilogue + 1);
constexpr int kI8Mma = 32 * (kI8Producers + kI8Epilogue);   // the thread that issues the MMAs
constexpr int kI8MaxStages = 16;
constexpr int kI8MaxWindow = 181;                 // 255^2 W^2 < 2^31: the int32 sums cannot wrap
constexpr uint32_t kI8MaxSmem = 227 * 1024 - 2048; // dynamic shared memory (the static part beside it)

// the layout of one launch, worked out on the host (i8_plan)
struct I8Geo {
    int VT;              // lane tiles of v (1, or 2 for M > 128)
    int NU;              // the MMA's N: the u extent, M rounded up to 16
    int KCOLS;           // chip columns held: L rounded up to 32 (K chunks of 32)
    int F;               // frames per group (the chips one Toeplitz operand serves)
    int NB;              // accumulator buffers (2: a group's epilogue runs under the next's MMAs)
    int NS;              // Toeplitz ring stages, one reference row each
    int CT;              // K chunks of a stage (both lane tiles), 8 TMEM columns each
    int c0[2], c1[2];    // the K chunks of each lane tile: [c0, c1)
    uint32_t lbo;        // bytes between a chip's 16-column blocks (rows * 16, rows odd)
    uint32_t chip_bytes; // one chip: KCOLS / 16 blocks
    uint32_t pw;         // bytes per padded reference row in shared memory: 128 + KCOLS
    uint32_t off_p;      // the padded reference rows, after 2 F chips
    uint32_t ring_col;   // the first TMEM column of the ring, after NB F VT NU accumulator columns
    uint32_t stage_cols; // TMEM columns of a stage: 8 CT
    uint32_t smem;       // dynamic shared memory
};

// the layout for window W and search R; false if the form does not hold the geometry
inline bool i8_plan(int W, int R, I8Geo &g)
{
    const int L = W + 2 * R, M = 2 * R + 1;
    if (W < 1 || W > kI8MaxWindow || M > 256 || L > 256) return false;
    g = I8Geo{};
    g.VT = (M + 127) / 128;
    g.NU = (M + 15) / 16 * 16;
    g.KCOLS = (L + 31) / 32 * 32;
    g.CT = 0;
    for (int vt = 0; vt < 2; ++vt) {
        const int v0 = 128 * vt;
        const int kend = std::min(L, v0 + 127 + W);   // the columns j' where T is non-zero for some lane
        g.c0[vt] = v0 / 32;
        g.c1[vt] = vt < g.VT ? (kend + 31) / 32 : g.c0[vt];
        g.CT += g.c1[vt] - g.c0[vt];
    }
    g.stage_cols = uint32_t(8 * g.CT);
    const int rows = (W - 1 + g.NU) | 1;   // odd: the blocks start on different 16-byte bank groups
    g.lbo = uint32_t(rows) * 16u;
    g.chip_bytes = uint32_t(g.KCOLS / 16) * g.lbo;
    g.pw = 128u + uint32_t(g.KCOLS);
    const int per_pair = g.VT * g.NU;
    for (int nb = 2; nb >= 1; --nb)
        for (int f = 4; f >= 1; f >>= 1) {
            const int cols = nb * f * per_pair;
            const int ns = (512 - cols) / int(g.stage_cols);
            const uint32_t off_p = (2u * uint32_t(f) * g.chip_bytes + 127u) & ~127u;
            const uint32_t smem = off_p + uint32_t(W) * g.pw + 16u;   // + the word read past the last row
            if (ns < (nb == 2 ? 3 : 2) || smem > kI8MaxSmem) continue;
            g.F = f;
            g.NB = nb;
            g.ring_col = uint32_t(cols);
            g.NS = std::min(kI8MaxStages, ns);
            g.off_p = off_p;
            g.smem = smem;
            return true;
        }
    return false;
}

// the instruction descriptor of kind::i8: int32 accumulation, unsigned 8-bit A and B, both K-major
B200_HD uint32_t i8_idesc(int M, int N)
{
    return (2u << 4) | (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

// the arguments beyond CorrArgs
struct I8Args {
    CorrArgs a;
    const int2 *bstat;       // nf x h x dpitch: {pixel sum, dinv bits} of each W x W box
    const uint8_t *refwin;   // nwin x W x W: the reference windows' pixels
    const int *sref;         // nwin: their sums
    int *status;             // 3 when a wait gave up
    I8Geo g;
};

#ifdef __CUDACC__

namespace i8 {

__device__ __forceinline__ uint64_t globaltimer()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool try_wait(uint32_t addr, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    return done != 0;
}

// wait for the phase `parity` of an mbarrier; false if *abort was raised or about two seconds
// passed (then *abort is raised here). sleep_ns > 0: a waiting role that is not on the critical
// path sleeps between polls and leaves the issue slots to the others.
__device__ __forceinline__ bool wait(uint64_t *bar, uint32_t parity, volatile int *abort, unsigned sleep_ns = 0,
                                     uint64_t limit_ns = 2000000000ull)
{
    const uint32_t addr = tc::smem_u32(bar);
    if (try_wait(addr, parity)) return true;
    if (*abort) return false;
    uint64_t t0 = 0;
    for (uint32_t it = 0;; ++it) {
        if (sleep_ns) __nanosleep(sleep_ns);
        if (try_wait(addr, parity)) return true;
        if ((it & 63) == 63) {
            if (*abort) return false;
            const uint64_t t = globaltimer();
            if (!t0) t0 = t;
            else if (t - t0 > limit_ns || it > (1u << 30)) {   // about two seconds by default
                *abort = 1;
                return false;
            }
        }
    }
}

__device__ __forceinline__ void arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc::smem_u32(bar)) : "memory");
}

// D[tmem] (+)= A[smem] * B[smem], kind::i8 (the self-test's reference path)
__device__ __forceinline__ void mma_ss(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate));
}

// D[tmem] (+)= A[tmem] * B[smem], kind::i8
__device__ __forceinline__ void mma(uint32_t d_tmem, uint32_t a_tmem, uint64_t b_desc, uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], [%1], %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "r"(a_tmem), "l"(b_desc), "r"(idesc), "r"(accumulate));
}

// 8 consecutive 32-bit TMEM columns of this thread's lane (completed by st_wait)
__device__ __forceinline__ void st8(uint32_t taddr, const uint32_t (&w)[8])
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr), "r"(w[0]),
                 "r"(w[1]), "r"(w[2]), "r"(w[3]), "r"(w[4]), "r"(w[5]), "r"(w[6]), "r"(w[7]));
}
__device__ __forceinline__ void st_wait() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// one (window, frame) pair of a group
struct Pair {
    int64_t q;           // the output index f * nwin + k
    int f, gy, gx, sy, sx;
    bool ok;             // the search window lies inside the frame and the reference window has texture
};

__device__ __forceinline__ Pair pair(const CorrArgs &a, int k, int f)
{
    Pair o{};
    o.f = f;
    o.q = int64_t(f) * a.nwin + k;
    if (a.gross_mode == 1) {
        o.gy = a.gross[2 * f];
        o.gx = a.gross[2 * f + 1];
    } else if (a.gross_mode == 2) {
        o.gy = a.gross[2 * o.q];
        o.gx = a.gross[2 * o.q + 1];
    }
    o.sy = a.down[k / a.nx] + o.gy - a.R;
    o.sx = a.across[k % a.nx] + o.gx - a.R;
    o.ok = a.norm[k] > 0 && o.sy >= 0 && o.sx >= 0 && o.sy + a.L <= a.h && o.sx + a.L <= a.w;
    return o;
}

// rho from the exact integer sum S_rx and the box's {pixel sum S_x, dinv}: (n S_rx - S_ref S_x)
// exactly in int64, rounded once to float, times dinv / (n norm)
__device__ __forceinline__ float rho(uint32_t srx, int2 st, int n, int sref, float scale)
{
    const int64_t cn = int64_t(n) * int64_t(srx) - int64_t(sref) * int64_t(st.x);
    return float(cn) * (__int_as_float(st.y) * scale);
}

}   // namespace i8

template <bool SURF>
__global__ void __launch_bounds__(kI8Threads, 1) corr_i8_kernel(I8Args args)
{
    const CorrArgs &a = args.a;
    const I8Geo &g = args.g;
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t bar_full[kI8MaxStages], bar_empty[kI8MaxStages];
    __shared__ __align__(8) uint64_t bar_cfull[2], bar_cempty[2], bar_dfull[2], bar_dempty[2], bar_final;
    __shared__ uint32_t tmem_base;
    __shared__ int s_abort;
    __shared__ float s_best[kI8Epilogue];
    __shared__ int s_at[kI8Epilogue];
    __shared__ double s_sq[kI8Epilogue];
    __shared__ float s_fit[9];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    volatile int *abort = &s_abort;

    const int W = a.W, L = a.L, M = a.M, R = a.R;
    const int VT = g.VT, NU = g.NU, F = g.F, NB = g.NB, NS = g.NS;
    const int gpw = (a.nf + F - 1) / F;          // groups per window
    const int ngroups = a.nwin * gpw;
    unsigned char *chips = smem, *P = smem + g.off_p;

    // zero the chips and the padded reference rows once: the pads are never written again
    for (uint32_t i = tid; i < g.smem / 16; i += kI8Threads) reinterpret_cast<uint4 *>(smem)[i] = make_uint4(0, 0, 0, 0);
    if (warp == 0) tc::tmem_alloc(&tmem_base, 512);
    if (tid == 0) {
        for (int s = 0; s < NS; ++s) {
            tc::mbar_init(&bar_full[s], 4);   // the four producer warps (one per quadrant) of the stage
            tc::mbar_init(&bar_empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            tc::mbar_init(&bar_cfull[b], kI8Epilogue);
            tc::mbar_init(&bar_cempty[b], 1);
            tc::mbar_init(&bar_dfull[b], 1);
            tc::mbar_init(&bar_dempty[b], kI8Epilogue);
        }
        tc::mbar_init(&bar_final, 1);
        s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc::fence_smem_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_base;

    if (warp < kI8Producers) {
        // ---- producers: the Toeplitz chunks of each reference row, one ring stage per row. No early
        // exit: the named barrier below must see all four warps, so after a failed wait a warp keeps
        // walking the groups without work (every wait returns at once once aborted).
        const int qd = warp & 3, half = warp >> 2;   // lane quadrant; the stages of this warp: parity half
        const uint32_t lane_addr = tmem + (uint32_t(32 * qd) << 16) + g.ring_col;
        int s = 0;
        uint32_t round = 0, seq = 0;   // ring position; stages filled so far by the CTA (both halves)
        int cur_k = -1;
        for (int gl = 0;; ++gl) {
            const int gi = blockIdx.x + gl * gridDim.x;
            if (gi >= ngroups) break;
            const int k = gi / gpw, f0 = (gi % gpw) * F, nfr = min(F, a.nf - f0);
            bool any = false;
            for (int fi = 0; fi < nfr; ++fi) any |= i8::pair(a, k, f0 + fi).ok;
            if (!any) continue;
            if (k != cur_k) {   // the window's rows into P (the producers are done with the previous one)
                asm volatile("bar.sync 1, %0;" ::"n"(32 * kI8Producers) : "memory");
                const uint8_t *src = args.refwin + size_t(k) * W * W;
                for (int e = tid; e < W * W; e += 32 * kI8Producers) P[(e / W) * g.pw + 128 + e % W] = src[e];
                asm volatile("bar.sync 1, %0;" ::"n"(32 * kI8Producers) : "memory");
                cur_k = k;
            }
            for (int i = 0; i < W; ++i, ++seq) {
                if ((seq & 1u) == uint32_t(half) && !*abort && (round == 0 || i8::wait(&bar_empty[s], (round - 1) & 1u, abort))) {
                    tc::fence_after_sync();
                    const uint32_t *row = reinterpret_cast<const uint32_t *>(P + i * g.pw);
                    uint32_t col = lane_addr + uint32_t(s) * g.stage_cols;
                    for (int vt = 0; vt < VT; ++vt) {
                        // bytes 128 + 32 c - v .. of the padded row: T_i[v][32 c ..] = ref(i, 32 c - v ..);
                        // chunks in batches of up to four, the batch's words loaded first
                        const int t0 = 128 + 32 * g.c0[vt] - (128 * vt + 32 * qd + lane);
                        const int sh = (t0 & 3) * 8;
                        const uint32_t *wp = row + (t0 >> 2);
                        for (int c = g.c0[vt]; c < g.c1[vt]; c += 4) {
                            const int nb = min(4, g.c1[vt] - c);
                            uint32_t p[33];
#pragma unroll
                            for (int j = 0; j < 33; ++j) p[j] = j <= 8 * nb ? wp[j] : 0u;
#pragma unroll
                            for (int q = 0; q < 4; ++q) {
                                if (q < nb) {
                                    uint32_t out[8];
#pragma unroll
                                    for (int j = 0; j < 8; ++j) out[j] = __funnelshift_r(p[8 * q + j], p[8 * q + j + 1], sh);
                                    i8::st8(col, out);
                                    col += 8u;
                                }
                            }
                            wp += 8 * nb;
                        }
                    }
                    i8::st_wait();
                    tc::fence_before_sync();
                    __syncwarp();
                    if (lane == 0) i8::arrive(&bar_full[s]);
                }
                if (++s == NS) {
                    s = 0;
                    ++round;
                }
            }
        }
    } else if (warp < kI8Producers + kI8Epilogue) {
        // ---- epilogue warps: the next group's chips into shared memory, the previous group's outputs
        const int e = tid - 32 * kI8Producers;   // 0 .. 127
        const int qd = warp - kI8Producers;      // this warp's TMEM lane quadrant
        const bool aligned = ((a.pitch | int(a.fstride & 15) | int(reinterpret_cast<uintptr_t>(a.frames) & 15)) & 15) == 0;
        const int nblk = (L + 15) / 16;
        const int n = W * W;

        // the chips of local group gl into chip buffer gl & 1; four 16-byte blocks per thread and
        // round, every load of the round first
        auto load = [&](int gl) {
            const int gi = blockIdx.x + gl * gridDim.x;
            const int k = gi / gpw, f0 = (gi % gpw) * F, nfr = min(F, a.nf - f0);
            for (int fi = 0; fi < nfr; ++fi) {
                const i8::Pair o = i8::pair(a, k, f0 + fi);
                if (!o.ok) continue;
                unsigned char *dst = chips + (uint32_t((gl & 1) * F + fi)) * g.chip_bytes;
                const uint8_t *src = a.frames + o.f * a.fstride + int64_t(o.sy) * a.pitch + o.sx;
                const int s = o.sx & 15, wq = s >> 2, wr = (s & 3) * 8;
                const int items = L * nblk;
                for (int base = e; base < items; base += 4 * 32 * kI8Epilogue) {
                    uint4 v0[4], v1[4];
#pragma unroll
                    for (int t = 0; t < 4; ++t) {
                        const int idx = base + t * 32 * kI8Epilogue;
                        v0[t] = v1[t] = make_uint4(0, 0, 0, 0);
                        if (idx < items) {
                            const int r = idx / nblk, bb = idx - r * nblk;
                            const uint8_t *gp = src + int64_t(r) * a.pitch + 16 * bb;
                            const int keep = L - 16 * bb;   // chip bytes in this block (>= 1)
                            if (aligned) {
                                const uint4 *ap = reinterpret_cast<const uint4 *>(reinterpret_cast<uintptr_t>(gp) & ~uintptr_t(15));
                                v0[t] = __ldg(ap);
                                if (s != 0 && 16 - s < keep) v1[t] = __ldg(ap + 1);
                            } else {
                                uint32_t o4[4];
#pragma unroll
                                for (int j = 0; j < 4; ++j) {
                                    uint32_t wv = 0;
#pragma unroll
                                    for (int b = 0; b < 4; ++b)
                                        if (4 * j + b < keep) wv |= uint32_t(__ldg(gp + 4 * j + b)) << (8 * b);
                                    o4[j] = wv;
                                }
                                v0[t] = make_uint4(o4[0], o4[1], o4[2], o4[3]);
                            }
                        }
                    }
#pragma unroll
                    for (int t = 0; t < 4; ++t) {
                        const int idx = base + t * 32 * kI8Epilogue;
                        if (idx >= items) continue;
                        const int r = idx / nblk, bb = idx - r * nblk;
                        const int keep = L - 16 * bb;
                        uint32_t o4[4];
                        if (aligned) {
                            const uint32_t x[8] = {v0[t].x, v0[t].y, v0[t].z, v0[t].w, v1[t].x, v1[t].y, v1[t].z, v1[t].w};
                            uint32_t y[5];
#pragma unroll
                            for (int j = 0; j < 5; ++j) {
                                const uint32_t t0 = (wq & 2) ? x[j + 2] : x[j];
                                const uint32_t t1 = (wq & 2) ? x[j + 3] : x[j + 1];
                                y[j] = (wq & 1) ? t1 : t0;
                            }
#pragma unroll
                            for (int j = 0; j < 4; ++j) o4[j] = __funnelshift_r(y[j], y[j + 1], wr);
                        } else {
                            o4[0] = v0[t].x;
                            o4[1] = v0[t].y;
                            o4[2] = v0[t].z;
                            o4[3] = v0[t].w;
                        }
                        if (keep < 16) {   // zero past the chip's last column
#pragma unroll
                            for (int j = 0; j < 4; ++j) {
                                const int kb = keep - 4 * j;   // bytes of word j to keep
                                if (kb <= 0) o4[j] = 0;
                                else if (kb < 4) o4[j] &= (1u << (8 * kb)) - 1u;
                            }
                        }
                        *reinterpret_cast<uint4 *>(dst + uint32_t(bb) * g.lbo + uint32_t(r) * 16u) = make_uint4(o4[0], o4[1], o4[2], o4[3]);
                    }
                }
            }
            tc::fence_smem_async();
            __syncwarp();
            if (lane == 0) i8::arrive(&bar_cfull[gl & 1]);
        };

        // the outputs of one pair from its accumulators at TMEM column dcol (lane tile 0)
        auto epilogue = [&](const i8::Pair &o, int k, uint32_t dcol) {
            const int sref = args.sref[k];
            const float scale = float(1.0 / (double(n) * double(a.norm[k])));
            const int2 *bt = args.bstat + size_t(o.f) * a.dinv_fstride + size_t(o.sy) * a.dpitch + o.sx;
            float *sv = SURF ? a.surface + o.q * M * M : nullptr;
            float best = -2.0f;
            int at = INT_MAX;
            for (int vt = 0; vt < VT; ++vt) {
                const int v = 128 * vt + 32 * qd + lane;
                const bool vin = v < M;
                const int2 *bv = bt + v;
                const uint32_t taddr = tmem + (uint32_t(32 * qd) << 16) + dcol + uint32_t(vt * NU);
                int2 tb[16], tn[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) tb[j] = vin && j < M ? __ldg(bv + size_t(j) * a.dpitch) : make_int2(0, 0);
                float vbest = -2.0f;
                int vat = INT_MAX;
                for (int u0 = 0; u0 < NU; u0 += 16) {
                    uint32_t r[16];
                    tc::tmem_ld16_nowait(taddr + uint32_t(u0), r);
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        const int u = u0 + 16 + j;
                        tn[j] = vin && u < M ? __ldg(bv + size_t(u) * a.dpitch) : make_int2(0, 0);
                    }
                    tc::tmem_wait();
                    if (vin) {
#pragma unroll
                        for (int j = 0; j < 16; ++j) {
                            const int u = u0 + j;
                            if (u < M) {
                                const float x = i8::rho(r[j], tb[j], n, sref, scale);
                                if (SURF) sv[u * M + v] = x;
                                if (x > vbest) {   // u ascends: ties keep the first
                                    vbest = x;
                                    vat = u * M + v;
                                }
                            }
                        }
                    }
#pragma unroll
                    for (int j = 0; j < 16; ++j) tb[j] = tn[j];
                }
                better(best, at, vbest, vat);
            }
            for (int s = 16; s > 0; s >>= 1)
                better(best, at, __shfl_xor_sync(0xffffffffu, best, s), __shfl_xor_sync(0xffffffffu, at, s));
            if (lane == 0) {
                s_best[qd] = best;
                s_at[qd] = at;
            }
            asm volatile("bar.sync 2, %0;" ::"n"(32 * kI8Epilogue) : "memory");
            best = s_best[0];
            at = s_at[0];
            for (int w = 1; w < kI8Epilogue; ++w) better(best, at, s_best[w], s_at[w]);
            const bool valid = best > 0;
            int pu = 0, pv = 0, i0 = 0, i1 = 0, j0 = 0, j1 = 0;
            double sq = 0.0;
            if (valid) {
                pu = at / M;
                pv = at % M;
                snr_patch(M, a.stat, pu, pv, i0, i1, j0, j1);
                for (int vt = 0; vt < VT; ++vt) {
                    const int vw = 128 * vt + 32 * qd;   // this warp's first lane v
                    if (vw >= j1 || vw + 32 <= j0) continue;   // warp-uniform
                    const int v = vw + lane;
                    const uint32_t taddr = tmem + (uint32_t(32 * qd) << 16) + dcol + uint32_t(vt * NU);
                    for (int cb = i0 & ~15; cb < i1; cb += 16) {
                        uint32_t r[16];
                        tc::tmem_ld16_nowait(taddr + uint32_t(cb), r);
                        tc::tmem_wait();
                        if (v >= j0 && v < j1) {
#pragma unroll
                            for (int j = 0; j < 16; ++j) {
                                const int u = cb + j;
                                if (u < i0 || u >= i1) continue;
                                const float x = i8::rho(r[j], __ldg(bt + size_t(u) * a.dpitch + v), n, sref, scale);
                                sq += double(x) * double(x);
                                const int du = u - pu, dw = v - pv;
                                if (du >= -1 && du <= 1 && dw >= -1 && dw <= 1) s_fit[(du + 1) * 3 + dw + 1] = x;
                            }
                        }
                    }
                }
            }
            for (int s = 16; s > 0; s >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, s);
            if (lane == 0) s_sq[qd] = sq;
            asm volatile("bar.sync 2, %0;" ::"n"(32 * kI8Epilogue) : "memory");
            if (e == 0) {
                if (valid) {
                    double sum = 0.0;
                    for (int w = 0; w < kI8Epilogue; ++w) sum += s_sq[w];
                    peak_outputs(s_fit + 4, 3, M, pu, pv, R, o.gy, o.gx, n, sum, (i1 - i0) * (j1 - j0), o.q, a.offset,
                                 a.peak, a.snr, a.cov);
                } else {
                    invalid_outputs(o.q, a.offset, a.peak, a.snr, a.cov);
                }
            }
            asm volatile("bar.sync 2, %0;" ::"n"(32 * kI8Epilogue) : "memory");
        };

        // no early exit either (the epilogue holds named barriers): after a failed wait the warps
        // keep walking the groups, on whatever the buffers hold, until the end
        if (int(blockIdx.x) < ngroups) load(0);
        for (int gl = 0;; ++gl) {
            const int gi = blockIdx.x + gl * gridDim.x;
            if (gi >= ngroups) break;
            // the next group's chips, once the MMAs of group gl - 1 are done with that buffer
            if (gi + int(gridDim.x) < ngroups) {
                if (gl + 1 >= 2) i8::wait(&bar_cempty[(gl + 1) & 1], uint32_t(((gl + 1) >> 1) - 1) & 1u, abort, 128);
                load(gl + 1);
            }
            const int b = NB == 2 ? gl & 1 : 0;
            i8::wait(&bar_dfull[b], uint32_t(NB == 2 ? gl >> 1 : gl) & 1u, abort, 256);
            tc::fence_after_sync();
            const int k = gi / gpw, f0 = (gi % gpw) * F, nfr = min(F, a.nf - f0);
            for (int fi = 0; fi < nfr; ++fi) {
                const i8::Pair o = i8::pair(a, k, f0 + fi);
                if (o.ok) {
                    epilogue(o, k, uint32_t((b * F + fi) * VT * NU));
                } else {
                    if (e == 0) invalid_outputs(o.q, a.offset, a.peak, a.snr, a.cov);
                    if (SURF)
                        for (int i = e; i < M * M; i += 32 * kI8Epilogue) a.surface[o.q * M * M + i] = 0.0f;
                }
            }
            tc::fence_before_sync();
            __syncwarp();
            if (lane == 0) i8::arrive(&bar_dempty[b]);
        }
    } else if (tid == kI8Mma) {
        // ---- the MMA issue: per group, per reference row, every K chunk of both lane tiles against
        // every valid chip of the group, one ring stage (one wait, one commit). Specialised on the
        // frames per group so that between two MMAs there are only descriptor increments.
        bool ok = true;
        auto issue = [&](auto FC) {
            constexpr int FF = decltype(FC)::value;
            const uint32_t idesc = i8_idesc(128, NU);
            const uint32_t blk2 = 2u * (g.lbo >> 4);   // descriptor start units between two K chunks
            int s = 0;
            uint32_t round = 0;
            auto valid_mask = [&](int gi) {
                const int k = gi / gpw, f0 = (gi % gpw) * FF, nfr = min(FF, a.nf - f0);
                unsigned m = 0;
                for (int fi = 0; fi < nfr; ++fi)
                    if (i8::pair(a, k, f0 + fi).ok) m |= 1u << fi;
                return m;
            };
            unsigned vm_next = int(blockIdx.x) < ngroups ? valid_mask(blockIdx.x) : 0u;
            for (int gl = 0; ok; ++gl) {
                const int gi = blockIdx.x + gl * gridDim.x;
                if (gi >= ngroups) break;
                const unsigned vm = vm_next;
                const int cb = gl & 1, b = NB == 2 ? gl & 1 : 0;
                if (!i8::wait(&bar_cfull[cb], uint32_t(gl >> 1) & 1u, abort) ||
                    (gl >= NB && !i8::wait(&bar_dempty[b], uint32_t((NB == 2 ? gl >> 1 : gl) - 1) & 1u, abort))) {
                    ok = false;
                    break;
                }
                tc::fence_after_sync();
                if (vm) {
                    uint32_t dcol[FF];
                    uint64_t bd[FF];
#pragma unroll
                    for (int fi = 0; fi < FF; ++fi) {
                        dcol[fi] = tmem + uint32_t(((b * FF + fi) * VT) * NU);
                        bd[fi] = tc::smem_desc(tc::smem_u32(chips) + uint32_t(cb * FF + fi) * g.chip_bytes, g.lbo, 128);
                    }
                    for (int i = 0; i < W; ++i) {
                        if (!i8::wait(&bar_full[s], round & 1u, abort)) {
                            ok = false;
                            break;
                        }
                        tc::fence_after_sync();
                        uint32_t acol = tmem + g.ring_col + uint32_t(s) * g.stage_cols;
                        for (int vt = 0; vt < VT; ++vt) {
                            const uint32_t dv = vt ? uint32_t(NU) : 0u;
                            uint64_t bb[FF];
#pragma unroll
                            for (int fi = 0; fi < FF; ++fi) bb[fi] = bd[fi] + uint64_t(blk2 * uint32_t(g.c0[vt]) + uint32_t(i));
                            for (int c = g.c0[vt]; c < g.c1[vt]; ++c) {
                                const uint32_t acc = (i | (c - g.c0[vt])) != 0 ? 1u : 0u;
#pragma unroll
                                for (int fi = 0; fi < FF; ++fi) {
                                    if (vm >> fi & 1u) i8::mma(dcol[fi] + dv, acol, bb[fi], idesc, acc);
                                    bb[fi] += blk2;
                                }
                                acol += 8u;
                            }
                        }
                        tc::mma_commit(&bar_empty[s]);
                        if (++s == NS) {
                            s = 0;
                            ++round;
                        }
                    }
                    if (!ok) break;
                }
                tc::mma_commit(&bar_dfull[b]);
                tc::mma_commit(&bar_cempty[cb]);
                if (gi + int(gridDim.x) < ngroups) vm_next = valid_mask(gi + gridDim.x);   // under this group's MMAs
            }
        };
        if (F == 4) issue(std::integral_constant<int, 4>{});
        else if (F == 2) issue(std::integral_constant<int, 2>{});
        else issue(std::integral_constant<int, 1>{});
        if (!ok) *abort = 1;
        // nothing of this CTA's may still be running on the tensor core when TMEM is released
        tc::mma_commit(&bar_final);
        volatile int never = 0;
        if (!i8::wait(&bar_final, 0, &never)) *abort = 1;
    }
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0 && s_abort && args.status) atomicExch(args.status, 3);
    if (warp == 0) tc::tmem_dealloc(tmem, 512);
}

// A check of the bounded waits the tensor-core kernels rely on, with nothing in flight on the tensor
// core: one thread waits on an mbarrier that nothing arrives at, first with the iteration bound of
// corr_tc_kernel (tc::mbar_wait, `polls` polls), then with the clock bound of corr_i8_kernel
// (i8::wait, `limit_ns`). out[0] and out[1]: 1 when the wait gave up (as it must), 0 if it returned
// as completed.
__global__ void wait_selftest_kernel(uint32_t polls, uint64_t limit_ns, int *out)
{
    __shared__ __align__(8) uint64_t bar;
    __shared__ int s_abort;
    if (threadIdx.x != 0) return;
    tc::mbar_init(&bar, 1);
    s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    out[0] = tc::mbar_wait(&bar, 0, polls) ? 0 : 1;
    out[1] = i8::wait(&bar, 0, &s_abort, 0, limit_ns) ? 0 : 1;
}

// the reference windows' pixels (nwin x W x W) and their sums, one CTA per window
__global__ void refwin_kernel(const uint8_t *frame, int pitch, int W, int nx, const int *down, const int *across,
                              uint8_t *out, int *sref)
{
    __shared__ int part[32];
    const int k = blockIdx.x;
    const int y0 = down[k / nx], x0 = across[k % nx];
    int s = 0;
    for (int e = threadIdx.x; e < W * W; e += blockDim.x) {
        const uint8_t b = frame[size_t(y0 + e / W) * pitch + x0 + e % W];
        out[size_t(k) * W * W + e] = b;
        s += b;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < int(blockDim.x >> 5); ++w) t += part[w];
        sref[k] = t;
    }
}

// A check of the exact form's tensor-core path, one CTA of 128 threads: D (128 x N, int32) =
// A (128 x K) * X[i .. i + N - 1]^T, uint8, with A written to TMEM by tcgen05.st (lane m = row m) or
// staged in shared memory (a_smem), and X (rows x K) in shared memory as the correlation kernel
// holds a chip (16-byte column blocks, rows 16 bytes apart), the operand started at row i; K in
// chunks of 32, one MMA each.
struct I8SelftestArgs {
    const uint8_t *A;   // 128 x K, row-major
    const uint8_t *X;   // rows x K, row-major
    int32_t *D;         // 128 x N, row-major
    int N, K, rows, i;
    int a_smem;         // A from shared memory (K-major core matrices) instead of TMEM
    int *status;
};

__global__ void __launch_bounds__(128) tc_i8_selftest_kernel(I8SelftestArgs a)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ uint32_t tmem_base;
    __shared__ __align__(8) uint64_t mbar;
    __shared__ int s_abort;
    const int m = threadIdx.x, warp = m >> 5, N = a.N, K = a.K;
    const int rp = a.rows | 1;
    const uint32_t lbo = uint32_t(rp) * 16u;
    const uint32_t xbytes = (uint32_t(K / 16) * lbo + 127u) & ~127u;
    unsigned char *sa = smem + xbytes;   // A, when staged in shared memory: 8-row x 16-byte core matrices
    const uint32_t a_lbo = 128u, a_sbo = uint32_t(K / 16) * 128u;
    for (int idx = m; idx < a.rows * K; idx += 128) {
        const int r = idx / K, k = idx % K;
        smem[uint32_t(k / 16) * lbo + uint32_t(r) * 16u + uint32_t(k % 16)] = a.X[idx];
    }
    if (a.a_smem)
        for (int idx = m; idx < 128 * K; idx += 128) {
            const int r = idx / K, k = idx % K;
            sa[uint32_t(r / 8) * a_sbo + uint32_t(k / 16) * a_lbo + uint32_t(r % 8) * 16u + uint32_t(k % 16)] = a.A[idx];
        }
    tc::fence_smem_async();
    if (warp == 0) tc::tmem_alloc(&tmem_base, 512);
    if (m == 0) {
        tc::mbar_init(&mbar, 1);
        s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_base, lane_base = uint32_t(32 * warp) << 16;
    if (!a.a_smem) {
        for (int c = 0; c < K / 32; ++c) {   // row m of A, 32 bytes per chunk, into TMEM columns 256 + 8 c
            uint32_t w[8];
            for (int j = 0; j < 8; ++j) {
                const uint8_t *p = a.A + size_t(m) * K + 32 * c + 4 * j;
                w[j] = uint32_t(p[0]) | uint32_t(p[1]) << 8 | uint32_t(p[2]) << 16 | uint32_t(p[3]) << 24;
            }
            i8::st8(tmem + lane_base + 256u + 8u * uint32_t(c), w);
        }
        i8::st_wait();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (m == 0) {
        const uint32_t id = i8_idesc(128, N);
        for (int c = 0; c < K / 32; ++c) {
            const uint32_t start = tc::smem_u32(smem) + uint32_t(2 * c) * lbo + uint32_t(a.i) * 16u;
            if (a.a_smem)
                i8::mma_ss(tmem, tc::smem_desc(tc::smem_u32(sa) + uint32_t(2 * c) * a_lbo, a_lbo, a_sbo),
                           tc::smem_desc(start, lbo, 128), id, c > 0);
            else
                i8::mma(tmem, tmem + 256u + 8u * uint32_t(c), tc::smem_desc(start, lbo, 128), id, c > 0);
        }
        tc::mma_commit(&mbar);
    }
    const bool ok = i8::wait(&mbar, 0, &s_abort);
    tc::fence_after_sync();
    if (!ok && a.status) atomicExch(a.status, 3);
    for (int n0 = 0; n0 < N; n0 += 16) {
        uint32_t r[16];
        tc::tmem_ld16_nowait(tmem + lane_base + uint32_t(n0), r);
        tc::tmem_wait();
        for (int j = 0; j < 16 && n0 + j < N; ++j) a.D[size_t(m) * N + n0 + j] = ok ? int32_t(r[j]) : 0;
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 512);
}

#endif   // __CUDACC__

}   // namespace b200
