// fft_passes.cuh -- the passes of the per-window 2-D FFT correlation over a shared-memory tile.
//
// The tile S holds N rows of NHP complex values (Geo<N>). A pass hands whole vectors (two per
// warp: a pair of rows or a column each) to one warp, so its exchanges need only warp barriers.
// Each pass is written once as a list of phases; an executor runs the phases of a warp with a
// barrier between them -- the real warp on the GPU (DevExec), or a loop over 32 emulated lanes
// on the host (HostExec), which lets the index arithmetic be tested on a CPU.
//
//   row_forward  rows 2p, 2p+1 (reals) -> one complex row transform -> their two half spectra
//   col_pass     each column k of the half spectrum: forward transform; then either the result
//                is stored (reference windows) or multiplied by conj(ref spectrum), transformed
//                back and rows [0, M) kept (search windows)
//   row_inverse  rows u, u+1 of the column-inverted spectrum -> one complex inverse transform ->
//                two real rows of the correlation, normalized by a functor as they are stored
#pragma once

#include "fft_steps.cuh"

namespace b200 {

#ifdef __CUDACC__
// the executor of the warp calling it
struct DevExec {
    int w, nw;
    template <class F>
    __device__ __forceinline__ void for_warps(F &&f) const { f(w); }
    __device__ __forceinline__ int nwarps() const { return nw; }
    template <class St, class... Ph>
    __device__ __forceinline__ void run(Ph &&...ph) const
    {
        const int lane = threadIdx.x & 31;
        St s;
        ((ph(lane, s), __syncwarp()), ...);
    }
};
#endif

// a host emulation of nw warps of 32 lanes, phase by phase
struct HostExec {
    int nw;
    template <class F>
    void for_warps(F &&f) const
    {
        for (int w = 0; w < nw; ++w) f(w);
    }
    int nwarps() const { return nw; }
    template <class St, class... Ph>
    void run(Ph &&...ph) const
    {
        St s[32];
        (
            [&] {
                for (int lane = 0; lane < 32; ++lane) ph(lane, s[lane]);
            }(),
            ...);
    }
};

// The row pairs a warp takes at once in the row passes: lanes 0-15 take pair_of(g, 0), lanes 16-31
// pair_of(g, 1), two pairs apart. Each half-warp then holds one pair, so its 8-byte accesses (16
// distinct slots of a row) meet no bank twice, and the two pairs' rows are 4 NHP complex values
// apart, 16 banks for NHP twice an odd number, so the warp's 4-byte reads of the two pairs do not
// overlap either. Items g < pair_items(P) cover the pairs 0 .. P - 1 (the rest idle).
B200_HD int pair_of(int g, int half) { return 4 * (g >> 1) + (g & 1) + 2 * half; }
B200_HD int pair_items(int P) { return 2 * ((P + 3) / 4); }

// rows [0, 2P) of S hold real rows (floats, pitch RP, element n of a row at float column
// off + n, off < 4); on return, their half spectra
template <int N, class Ex>
B200_HD void row_forward(const Ex &ex, float2 *S, int P, const float2 *TW, int off = 0)
{
    using G = Geo<N>;
    constexpr int N2 = G::N2, NHP = G::NHP, NU = G::NU, NH = G::NH;
    struct St {
        float2 y[16];
        float2 z[N2];
        float2 a[NU], b[NU];
    };
    ex.for_warps([&](int warp) {
        for (int g = warp; g < pair_items(P); g += ex.nwarps()) {
            ex.template run<St>(
                [&](int lane, St &s) {   // step 1 on the complex row (row 2p) + i (row 2p+1)
                    const int p = pair_of(g, lane >> 4), n2 = lane & 15;
                    if (p < P && n2 < N2) {
                        const float *xa = reinterpret_cast<const float *>(S + size_t(2 * p) * NHP) + off;
                        const float *xb = xa + G::RP;
                        fwd_step1<N>(n2, TW, s.y, [&](int n) { return make_float2(xa[n], xb[n]); });
                    }
                },
                [&](int lane, St &s) {
                    const int p = pair_of(g, lane >> 4), n2 = lane & 15;
                    if (p < P && n2 < N2) {
                        float2 *e = S + size_t(2 * p) * NHP;
#pragma unroll
                        for (int k1 = 0; k1 < 16; ++k1) e[xpos(n2, k1)] = s.y[k1];
                    }
                },
                [&](int lane, St &s) {   // step 2
                    const int p = pair_of(g, lane >> 4), k1 = lane & 15;
                    if (p < P) {
                        const float2 *e = S + size_t(2 * p) * NHP;
                        fwd_step2<N>(k1, s.z, [&](int q) { return e[q]; });
                    }
                },
                [&](int lane, St &s) {   // the row transform in natural order
                    const int p = pair_of(g, lane >> 4), k1 = lane & 15;
                    if (p < P) {
                        float2 *e = S + size_t(2 * p) * NHP;
#pragma unroll
                        for (int k2 = 0; k2 < N2; ++k2) e[k1 + 16 * k2] = s.z[k2];
                    }
                },
                [&](int lane, St &s) {   // the two half spectra
                    const int p = pair_of(g, lane >> 4), j = lane & 15;
                    if (p < P) {
                        const float2 *e = S + size_t(2 * p) * NHP;
#pragma unroll
                        for (int i = 0; i < NU; ++i) {
                            const int k = j + 16 * i;
                            if (k < NH) unpack_real_pair(e[k], e[(N - k) % N], s.a[i], s.b[i]);
                        }
                    }
                },
                [&](int lane, St &s) {
                    const int p = pair_of(g, lane >> 4), j = lane & 15;
                    if (p < P) {
                        float2 *e = S + size_t(2 * p) * NHP;
#pragma unroll
                        for (int i = 0; i < NU; ++i) {
                            const int k = j + 16 * i;
                            if (k < NH) {
                                e[k] = s.a[i];
                                e[NHP + k] = s.b[i];
                            }
                        }
                    }
                });
        }
    });
}

// The column pass over `ncols` columns of the half spectrum (rows [0, Lr) nonzero; by default all
// NH of them, `stride` complex values apart per row, NHP by default; a subset of the columns
// starting at k0 is passed as S, spec or out moved by k0 columns).
// CORR false: the forward spectra are written to out[k * N + k2 * 16 + k1] (frequency
//   k1 + 16 k2 of column k).
// CORR true: the forward spectra are multiplied by conj(spec[k * N + k2 * 16 + k1]) (the same
//   order), transformed back, and rows [0, M) of each column stored in S.
template <int N, bool CORR, class Ex>
B200_HD void col_pass(const Ex &ex, float2 *S, int Lr, int M, const float2 *TW, const float2 *TWI,
                      const float2 *spec, float2 *out, int ncols = Geo<N>::NH, int stride = Geo<N>::NHP)
{
    using G = Geo<N>;
    constexpr int N2 = G::N2;
    const int NHP = stride, NH = ncols;
    struct St {
        float2 y[16];
        float2 z[N2];
    };
    ex.for_warps([&](int warp) {
        for (int g = warp; 2 * g < NH; g += ex.nwarps()) {
            auto step1 = [&](int lane, St &s) {
                const int k = 2 * g + (lane & 1), n2 = lane >> 1;
                if (k < NH && n2 < N2)
                    fwd_step1<N>(n2, TW, s.y, [&](int r) { return r < Lr ? S[size_t(r) * NHP + k] : make_float2(0.f, 0.f); });
            };
            auto store1 = [&](int lane, St &s) {
                const int k = 2 * g + (lane & 1), n2 = lane >> 1;
                if (k < NH && n2 < N2) {
#pragma unroll
                    for (int k1 = 0; k1 < 16; ++k1) S[size_t(xpos(n2, k1)) * NHP + k] = s.y[k1];
                }
            };
            auto step2 = [&](int lane, St &s) {
                const int k = 2 * g + (lane & 1), k1 = lane >> 1;
                if (k < NH) {
                    fwd_step2<N>(k1, s.z, [&](int q) { return S[size_t(q) * NHP + k]; });
                    if constexpr (CORR) {
                        const float2 *r = spec + size_t(k) * N;
#pragma unroll
                        for (int k2 = 0; k2 < N2; ++k2) s.z[k2] = cmulc(s.z[k2], r[k2 * 16 + k1]);
                        inv_step1<N>(k1, TWI, s.z);
                    } else {
                        float2 *o = out + size_t(k) * N;
#pragma unroll
                        for (int k2 = 0; k2 < N2; ++k2) o[k2 * 16 + k1] = s.z[k2];
                    }
                }
            };
            if constexpr (CORR) {
                auto store2 = [&](int lane, St &s) {
                    const int k = 2 * g + (lane & 1), k1 = lane >> 1;
                    if (k < NH) {
#pragma unroll
                        for (int n2 = 0; n2 < N2; ++n2) S[size_t(xpos(n2, k1)) * NHP + k] = s.z[n2];
                    }
                };
                auto step3 = [&](int lane, St &s) {
                    const int k = 2 * g + (lane & 1), n2 = lane >> 1;
                    if (k < NH && n2 < N2) inv_step2<N>(n2, s.y, [&](int q) { return S[size_t(q) * NHP + k]; });
                };
                auto store3 = [&](int lane, St &s) {
                    const int k = 2 * g + (lane & 1), n2 = lane >> 1;
                    if (k < NH && n2 < N2) {
#pragma unroll
                        for (int n1 = 0; n1 < 16; ++n1) {
                            const int r = N2 * n1 + n2;
                            if (r < M) S[size_t(r) * NHP + k] = s.y[n1];
                        }
                    }
                };
                ex.template run<St>(step1, store1, step2, store2, step3, store3);
            } else {
                ex.template run<St>(step1, store1, step2);
            }
        }
    });
}

// The inverse row pass: rows [0, M) of S hold column-inverted half spectra; on return row u holds
// norm(u, c, value) for c in [0, cols) as floats (pitch RP), value the unnormalized correlation;
// cols defaults to M (a square surface; a caller with part of its rows passes the surface width).
template <int N, class Ex, class Norm>
B200_HD void row_inverse(const Ex &ex, float2 *S, int M, const float2 *TWI, Norm &&norm, int cols = -1)
{
    using G = Geo<N>;
    constexpr int N2 = G::N2, NHP = G::NHP;
    const int C = cols < 0 ? M : cols;
    struct St {
        float2 z[N2];
        float2 y[16];
    };
    const int P = (M + 1) / 2;
    float *Sr = reinterpret_cast<float *>(S);
    ex.for_warps([&](int warp) {
        for (int g = warp; g < pair_items(P); g += ex.nwarps()) {
            ex.template run<St>(
                [&](int lane, St &s) {   // step 1 on (row u1) + i (row u2), extended to full spectra
                    const int p = pair_of(g, lane >> 4), k1 = lane & 15;
                    const int u1 = 2 * p, u2 = 2 * p + 1;
                    if (p < P) {
                        const float2 *h1 = S + size_t(u1) * NHP, *h2 = S + size_t(u2) * NHP;
#pragma unroll
                        for (int k2 = 0; k2 < N2; ++k2) {
                            const int kk = k1 + 16 * k2;
                            const float2 a = hermitian<N>(h1, kk);
                            const float2 b = u2 < M ? hermitian<N>(h2, kk) : make_float2(0.f, 0.f);
                            s.z[k2] = make_float2(a.x - b.y, a.y + b.x);
                        }
                        inv_step1<N>(k1, TWI, s.z);
                    }
                },
                [&](int lane, St &s) {
                    const int p = pair_of(g, lane >> 4), k1 = lane & 15;
                    if (p < P) {
                        float2 *e = S + size_t(2 * p) * NHP;
#pragma unroll
                        for (int n2 = 0; n2 < N2; ++n2) e[xpos(n2, k1)] = s.z[n2];
                    }
                },
                [&](int lane, St &s) {   // step 2
                    const int p = pair_of(g, lane >> 4), n2 = lane & 15;
                    if (p < P && n2 < N2) {
                        const float2 *e = S + size_t(2 * p) * NHP;
                        inv_step2<N>(n2, s.y, [&](int q) { return e[q]; });
                    }
                },
                [&](int lane, St &s) {   // the two rows, normalized, as floats
                    const int p = pair_of(g, lane >> 4), n2 = lane & 15;
                    const int u1 = 2 * p, u2 = 2 * p + 1;
                    if (p < P && n2 < N2) {
#pragma unroll
                        for (int n1 = 0; n1 < 16; ++n1) {
                            const int c = N2 * n1 + n2;
                            if (c < C) {
                                Sr[size_t(u1) * G::RP + c] = norm(u1, c, s.y[n1].x);
                                if (u2 < M) Sr[size_t(u2) * G::RP + c] = norm(u2, c, s.y[n1].y);
                            }
                        }
                    }
                });
        }
    });
}

}   // namespace b200
