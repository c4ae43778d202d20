/*
 * fftw_shim.cpp -- our own double-precision implementation of the single-precision FFTW calls
 * that the reference CPU backend makes (slipcam cxx/cpu.cpp). TEST INFRASTRUCTURE, oracle only.
 *
 * The 1-D transform is a recursive mixed-radix Cooley-Tukey FFT (decimation in time): a length
 * n = p * m is split into p interleaved sub-sequences of length m, each transformed recursively,
 * then combined with radix-p butterflies after multiplying by the twiddles w_n^{r k}. Radices
 * 4, 2, 3 and 5 are taken first; any other prime factor uses a direct p-point butterfly. All
 * arithmetic is in double; the 2-D transforms are row-column (rows, then columns; the inverse
 * in the opposite order) with a thread-local double buffer, so a plan can run on many threads.
 */
#include "fftw3.h"

#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

namespace {

using cd = std::complex<double>;

/// a 1-D complex transform of length n: its factors and the table w_n^k = e^{-2 pi i k / n}
struct Fft1 {
    int n = 0;
    std::vector<int> factors;
    std::vector<cd> tw;

    explicit Fft1(int len) : n(len)
    {
        int m = n;
        for (int p : {4, 2, 3, 5})
            while (m % p == 0 && !(p == 4 && m == 2)) {
                factors.push_back(p);
                m /= p;
            }
        for (int p = 7; m > 1; p += 2)
            while (m % p == 0) {
                factors.push_back(p);
                m /= p;
            }
        if (factors.empty()) factors.push_back(1);
        tw.resize(n);
        for (int k = 0; k < n; k++) {
            const double a = -2.0 * M_PI * double(k) / double(n);
            tw[k] = cd(std::cos(a), std::sin(a));
        }
    }

    /// w_n^e for the transform direction (sign -1 forward, +1 inverse)
    cd w(long e, int sign) const
    {
        const cd t = tw[size_t(e % n)];
        return sign < 0 ? t : std::conj(t);
    }

    /// out[0..len) = DFT of in[0], in[s], in[2s], ...; len = product of factors from f on
    void rec(cd *out, const cd *in, size_t s, int len, int f, int sign) const
    {
        const int p = factors[f], m = len / p;
        if (m == 1) {
            for (int r = 0; r < p; r++) out[r] = in[r * s];
        } else {
            for (int r = 0; r < p; r++) rec(out + size_t(r) * m, in + r * s, s * p, m, f + 1, sign);
        }
        if (p == 1) return;
        const long step = n / len;   // w_len = w_n^step
        cd t[64];
        std::vector<cd> big;
        cd *v = t;
        if (p > 64) {
            big.resize(p);
            v = big.data();
        }
        for (int k = 0; k < m; k++) {
            for (int r = 0; r < p; r++) v[r] = out[k + size_t(r) * m] * w(long(r) * k * step, sign);
            if (p == 2) {
                out[k] = v[0] + v[1];
                out[k + m] = v[0] - v[1];
            } else if (p == 4) {
                const cd a = v[0] + v[2], b = v[0] - v[2], c = v[1] + v[3];
                const cd d = (v[1] - v[3]) * cd(0.0, sign < 0 ? -1.0 : 1.0);
                out[k] = a + c;
                out[k + m] = b + d;
                out[k + 2 * size_t(m)] = a - c;
                out[k + 3 * size_t(m)] = b - d;
            } else {
                const long pstep = n / p;   // w_p = w_n^pstep
                for (int q = 0; q < p; q++) {
                    cd acc = 0.0;
                    for (int r = 0; r < p; r++) acc += v[r] * w(long(r) * q % p * pstep, sign);
                    out[k + size_t(q) * m] = acc;
                }
            }
        }
    }

    void run(cd *out, const cd *in, int sign) const { rec(out, in, 1, n, 0, sign); }
};

}   // namespace

struct fftwf_plan_s {
    int n0, n1, nh;
    bool forward;   // r2c if true, else c2r
    Fft1 rows, cols;
    fftwf_plan_s(int a, int b, bool fwd) : n0(a), n1(b), nh(b / 2 + 1), forward(fwd), rows(b), cols(a) {}
};

namespace {

/// per-thread work arrays, grown as needed
struct Work {
    std::vector<cd> grid, a, b;
};
thread_local Work work;

}   // namespace

extern "C" {

float *fftwf_alloc_real(size_t n)
{
    return static_cast<float *>(std::aligned_alloc(64, ((n * sizeof(float) + 63) / 64) * 64 + 64));
}

fftwf_complex *fftwf_alloc_complex(size_t n)
{
    return static_cast<fftwf_complex *>(std::aligned_alloc(64, ((n * sizeof(fftwf_complex) + 63) / 64) * 64 + 64));
}

void fftwf_free(void *p) { std::free(p); }

fftwf_plan fftwf_plan_dft_r2c_2d(int n0, int n1, float *, fftwf_complex *, unsigned)
{
    if (n0 <= 0 || n1 <= 0) return nullptr;
    return new (std::nothrow) fftwf_plan_s(n0, n1, true);
}

fftwf_plan fftwf_plan_dft_c2r_2d(int n0, int n1, fftwf_complex *, float *, unsigned)
{
    if (n0 <= 0 || n1 <= 0) return nullptr;
    return new (std::nothrow) fftwf_plan_s(n0, n1, false);
}

void fftwf_destroy_plan(fftwf_plan p) { delete p; }

void fftwf_execute_dft_r2c(const fftwf_plan p, float *in, fftwf_complex *out)
{
    const int n0 = p->n0, n1 = p->n1, nh = p->nh;
    Work &w = work;
    w.grid.resize(size_t(n0) * nh);
    w.a.resize(std::max(n0, n1));
    w.b.resize(std::max(n0, n1));
    // the rows: real to the half spectrum
    for (int i = 0; i < n0; i++) {
        for (int j = 0; j < n1; j++) w.a[j] = cd(in[size_t(i) * n1 + j], 0.0);
        p->rows.run(w.b.data(), w.a.data(), -1);
        for (int k = 0; k < nh; k++) w.grid[size_t(i) * nh + k] = w.b[k];
    }
    // the columns
    for (int k = 0; k < nh; k++) {
        for (int i = 0; i < n0; i++) w.a[i] = w.grid[size_t(i) * nh + k];
        p->cols.run(w.b.data(), w.a.data(), -1);
        for (int i = 0; i < n0; i++) {
            out[size_t(i) * nh + k][0] = float(w.b[i].real());
            out[size_t(i) * nh + k][1] = float(w.b[i].imag());
        }
    }
}

void fftwf_execute_dft_c2r(const fftwf_plan p, fftwf_complex *in, float *out)
{
    const int n0 = p->n0, n1 = p->n1, nh = p->nh;
    Work &w = work;
    w.grid.resize(size_t(n0) * nh);
    w.a.resize(std::max(n0, n1));
    w.b.resize(std::max(n0, n1));
    // the columns, inverse
    for (int k = 0; k < nh; k++) {
        for (int i = 0; i < n0; i++) w.a[i] = cd(in[size_t(i) * nh + k][0], in[size_t(i) * nh + k][1]);
        p->cols.run(w.b.data(), w.a.data(), +1);
        for (int i = 0; i < n0; i++) w.grid[size_t(i) * nh + k] = w.b[i];
    }
    // the rows: the Hermitian half to reals (the imaginary parts of the first and, for even n1,
    // the middle element do not enter a real signal's spectrum and are dropped)
    for (int i = 0; i < n0; i++) {
        const cd *h = w.grid.data() + size_t(i) * nh;
        for (int k = 0; k < n1; k++) w.a[k] = k < nh ? h[k] : std::conj(h[n1 - k]);
        w.a[0] = cd(w.a[0].real(), 0.0);
        if (n1 % 2 == 0) w.a[n1 / 2] = cd(w.a[n1 / 2].real(), 0.0);
        p->rows.run(w.b.data(), w.a.data(), +1);
        for (int j = 0; j < n1; j++) out[size_t(i) * n1 + j] = float(w.b[j].real());
    }
}

}   // extern "C"
