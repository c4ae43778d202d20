// fft_steps.cuh -- the per-thread pieces of the shared-memory 2-D FFT of one search window.
//
// A length-N transform (N = 16 * N2) is done in two register steps with one exchange through
// shared memory (the "four-step" split, n = N2 n1 + n2, k = k1 + 16 k2):
//   forward  step 1, thread n2: y[k1] = w_N^{n2 k1} * DFT16_{n1}( x[N2 n1 + n2] )  -> slot (n2, k1)
//            step 2, thread k1: X[k1 + 16 k2] = DFT_N2_{n2}( slot (n2, k1) )
//   inverse  step 1, thread k1: y[n2] = w_N^{-n2 k1} * IDFT_N2_{k2}( X[k1 + 16 k2] ) -> slot (n2, k1)
//            step 2, thread n2: x[N2 n1 + n2] = IDFT16_{k1}( slot (n2, k1) )
// A forward step 2 leaves thread k1 with exactly the frequencies an inverse step 1 needs, so the
// product with the reference spectrum sits in registers between them (no exchange).
//
// These helpers are host+device so that a whole tile can be emulated on the CPU (tests of the
// index arithmetic); the kernels in corr_fft.cuh call them with the lane mapping and barriers.
#pragma once

#include "common.cuh"

namespace b200 {

// forward step 1: load(n) gives x[n]; tw[k1 * N2 + n2] = w_N^{n2 k1}
template <int N, class Load>
B200_HD void fwd_step1(int n2, const float2 *tw, float2 (&y)[16], Load load)
{
    constexpr int N2 = N / 16;
#pragma unroll
    for (int n1 = 0; n1 < 16; ++n1) y[n1] = load(N2 * n1 + n2);
    DFT<16, false>::run(y);
#pragma unroll
    for (int k1 = 1; k1 < 16; ++k1) y[k1] = cmul(y[k1], tw[k1 * N2 + n2]);
}

// forward step 2: slot(p) reads exchange slot p; z[k2] = X[k1 + 16 k2]
template <int N, class Slot>
B200_HD void fwd_step2(int k1, float2 (&z)[N / 16], Slot slot)
{
    constexpr int N2 = N / 16;
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) z[n2] = slot(xpos(n2, k1));
    DFT<N2, false>::run(z);
}

// inverse step 1: z[k2] = X[k1 + 16 k2] in, z[n2] (twiddled) out; twi[n2 * 16 + k1] = w_N^{n2 k1}
template <int N>
B200_HD void inv_step1(int k1, const float2 *twi, float2 (&z)[N / 16])
{
    constexpr int N2 = N / 16;
    DFT<N2, true>::run(z);
#pragma unroll
    for (int n2 = 1; n2 < N2; ++n2) z[n2] = cmulc(z[n2], twi[n2 * 16 + k1]);
}

// inverse step 2: y[n1] = x[N2 n1 + n2]
template <int N, class Slot>
B200_HD void inv_step2(int n2, float2 (&y)[16], Slot slot)
{
#pragma unroll
    for (int k1 = 0; k1 < 16; ++k1) y[k1] = slot(xpos(n2, k1));
    DFT<16, true>::run(y);
}

// the spectra of two real rows a, b from the transform Z of a + i b: A[k] = (Z[k] + conj Z[N-k]) / 2,
// B[k] = (Z[k] - conj Z[N-k]) / (2i)
B200_HD void unpack_real_pair(float2 zk, float2 znk, float2 &a, float2 &b)
{
    a = make_float2(0.5f * (zk.x + znk.x), 0.5f * (zk.y - znk.y));
    b = make_float2(0.5f * (zk.y + znk.y), -0.5f * (zk.x - znk.x));
}

// element k of the full spectrum of a real row given as its half spectrum h[0..N/2]; the
// imaginary parts of h[0] and h[N/2] do not belong to a real row and are dropped
template <int N>
B200_HD float2 hermitian(const float2 *h, int k)
{
    if (k == 0 || k == N / 2) return make_float2(h[k].x, 0.0f);
    if (k < N / 2) return h[k];
    const float2 c = h[N - k];
    return make_float2(c.x, -c.y);
}

}   // namespace b200
