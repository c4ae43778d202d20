// dft.cuh -- small discrete Fourier transforms held in registers, fully unrolled.
//
// DFT<R, INV>::run(x) replaces x[0..R) by X[k] = sum_n x[n] w^{nk}, w = e^{-2 pi i / R}
// (forward) or e^{+2 pi i / R} (INV), unnormalized, natural order in and out. R = 2, 3, 4, 5 are
// written out; composite sizes split R = A * B as a Cooley-Tukey step inside the registers
// (B transforms of size A on the interleaved sub-sequences, twiddles w_R^{b k1}, A transforms of
// size B). The twiddle constants are computed at compile time from our own Taylor-series sine
// and cosine in double (cs2pi below), then rounded to float.
#pragma once

#include <cuda_runtime.h>

#define B200_HD __host__ __device__ __forceinline__
#define B200_HDC __host__ __device__ constexpr

namespace b200 {

constexpr double kPi = 3.14159265358979323846264338327950288;

// sin(x) and cos(x) for |x| <= pi/4 by their Taylor series (the terms fall below 1e-20 by k = 11)
B200_HDC double taylor_sin(double x)
{
    double term = x, sum = x;
    for (int k = 1; k < 12; ++k) {
        term *= -x * x / double((2 * k) * (2 * k + 1));
        sum += term;
    }
    return sum;
}

B200_HDC double taylor_cos(double x)
{
    double term = 1.0, sum = 1.0;
    for (int k = 1; k < 12; ++k) {
        term *= -x * x / double((2 * k - 1) * (2 * k));
        sum += term;
    }
    return sum;
}

// cos and sin of 2 pi p / q: the quadrant is taken exactly from the integers, the remaining
// angle folded into [0, pi/4]
B200_HDC void cs2pi(long p, long q, double &c, double &s)
{
    p %= q;
    if (p < 0) p += q;
    const long e = 4 * p, quad = e / q, rem = e % q;   // angle = quad * pi/2 + (rem / q) * pi/2
    double cc = 0.0, ss = 0.0;
    if (2 * rem <= q) {
        const double phi = double(rem) / double(q) * (kPi / 2);
        cc = taylor_cos(phi);
        ss = taylor_sin(phi);
    } else {
        const double psi = double(q - rem) / double(q) * (kPi / 2);
        cc = taylor_sin(psi);
        ss = taylor_cos(psi);
    }
    switch (quad) {
    case 0: c = cc; s = ss; break;
    case 1: c = -ss; s = cc; break;
    case 2: c = -cc; s = -ss; break;
    default: c = ss; s = -cc; break;
    }
}

// the table of w_R^m = e^{-2 pi i m / R}, m in [0, R), as floats
template <int R>
struct TwiddleTable {
    float c[R], s[R];
    B200_HDC TwiddleTable() : c(), s()
    {
        for (int m = 0; m < R; ++m) {
            double cc = 0.0, ss = 0.0;
            cs2pi(m, R, cc, ss);
            c[m] = float(cc);
            s[m] = float(-ss);
        }
    }
};

B200_HD float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
B200_HD float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
B200_HD float2 cmul(float2 a, float2 b)
{
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// a * conj(b)
B200_HD float2 cmulc(float2 a, float2 b)
{
    return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}
B200_HD float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// -i a, +i a
B200_HD float2 mul_mi(float2 a) { return make_float2(a.y, -a.x); }
B200_HD float2 mul_pi(float2 a) { return make_float2(-a.y, a.x); }

// a * w_R^e (forward) or a * w_R^{-e} (INV); e is a constant after unrolling, so the quarter
// turns become swaps and the other constants fold
template <int R, bool INV>
B200_HD float2 twiddle(float2 a, int e)
{
    e %= R;
    if (e == 0) return a;
    if (4 * e == R) return INV ? mul_pi(a) : mul_mi(a);
    if (2 * e == R) return make_float2(-a.x, -a.y);
    if (4 * e == 3 * R) return INV ? mul_mi(a) : mul_pi(a);
    constexpr TwiddleTable<R> t{};
    const float c = t.c[e], s = INV ? -t.s[e] : t.s[e];
    return make_float2(fmaf(a.x, c, -a.y * s), fmaf(a.x, s, a.y * c));
}

template <int R, bool INV>
struct DFT;

template <bool INV>
struct DFT<1, INV> {
    B200_HD static void run(float2 *) {}
};

template <bool INV>
struct DFT<2, INV> {
    B200_HD static void run(float2 *x)
    {
        const float2 a = x[0], b = x[1];
        x[0] = cadd(a, b);
        x[1] = csub(a, b);
    }
};

template <bool INV>
struct DFT<3, INV> {
    B200_HD static void run(float2 *x)
    {
        constexpr float h = 0.86602540378443864676f;   // sin(2 pi / 3)
        const float2 a = x[0], t = cadd(x[1], x[2]), d = csub(x[1], x[2]);
        const float2 m = make_float2(a.x - 0.5f * t.x, a.y - 0.5f * t.y);
        const float2 r = cscale(INV ? mul_pi(d) : mul_mi(d), h);   // -+ i sin(2pi/3) (b - c)
        x[0] = cadd(a, t);
        x[1] = cadd(m, r);
        x[2] = csub(m, r);
    }
};

template <bool INV>
struct DFT<4, INV> {
    B200_HD static void run(float2 *x)
    {
        const float2 a = cadd(x[0], x[2]), b = csub(x[0], x[2]);
        const float2 c = cadd(x[1], x[3]), d0 = csub(x[1], x[3]);
        const float2 d = INV ? mul_pi(d0) : mul_mi(d0);
        x[0] = cadd(a, c);
        x[1] = cadd(b, d);
        x[2] = csub(a, c);
        x[3] = csub(b, d);
    }
};

template <bool INV>
struct DFT<5, INV> {
    B200_HD static void run(float2 *x)
    {
        constexpr TwiddleTable<5> t{};
        constexpr float c1 = t.c[1], c2 = t.c[2], s1 = -t.s[1], s2 = -t.s[2];   // cos, sin of 2pi/5, 4pi/5
        const float2 a0 = x[0];
        const float2 t1 = cadd(x[1], x[4]), t2 = cadd(x[2], x[3]);
        const float2 t3 = csub(x[1], x[4]), t4 = csub(x[2], x[3]);
        const float2 m1 = make_float2(a0.x + c1 * t1.x + c2 * t2.x, a0.y + c1 * t1.y + c2 * t2.y);
        const float2 m2 = make_float2(a0.x + c2 * t1.x + c1 * t2.x, a0.y + c2 * t1.y + c1 * t2.y);
        const float2 q1 = make_float2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y);
        const float2 q2 = make_float2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y);
        const float2 r1 = INV ? mul_pi(q1) : mul_mi(q1);
        const float2 r2 = INV ? mul_pi(q2) : mul_mi(q2);
        x[0] = make_float2(a0.x + t1.x + t2.x, a0.y + t1.y + t2.y);
        x[1] = cadd(m1, r1);
        x[4] = csub(m1, r1);
        x[2] = cadd(m2, r2);
        x[3] = csub(m2, r2);
    }
};

// R = A * B: n = B a + b, k = k1 + A k2
template <int A, int B, bool INV>
struct DFTSplit {
    B200_HD static void run(float2 *x)
    {
        constexpr int R = A * B;
        float2 t[R];
#pragma unroll
        for (int b = 0; b < B; ++b) {
            float2 v[A];
#pragma unroll
            for (int a = 0; a < A; ++a) v[a] = x[B * a + b];
            DFT<A, INV>::run(v);
#pragma unroll
            for (int k1 = 0; k1 < A; ++k1) t[b * A + k1] = twiddle<R, INV>(v[k1], b * k1);
        }
#pragma unroll
        for (int k1 = 0; k1 < A; ++k1) {
            float2 v[B];
#pragma unroll
            for (int b = 0; b < B; ++b) v[b] = t[b * A + k1];
            DFT<B, INV>::run(v);
#pragma unroll
            for (int k2 = 0; k2 < B; ++k2) x[k1 + A * k2] = v[k2];
        }
    }
};

template <bool INV> struct DFT<6, INV> : DFTSplit<2, 3, INV> {};
template <bool INV> struct DFT<8, INV> : DFTSplit<2, 4, INV> {};
template <bool INV> struct DFT<9, INV> : DFTSplit<3, 3, INV> {};
template <bool INV> struct DFT<10, INV> : DFTSplit<2, 5, INV> {};
template <bool INV> struct DFT<12, INV> : DFTSplit<4, 3, INV> {};
template <bool INV> struct DFT<15, INV> : DFTSplit<3, 5, INV> {};
template <bool INV> struct DFT<16, INV> : DFTSplit<4, 4, INV> {};

}   // namespace b200
