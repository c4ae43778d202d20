/*
 * framecor_oracle.c -- TEST INFRASTRUCTURE: a CPU restatement of slipcam framecor's
 * Correlator.correlate, used only by tests/, __graft_entry__.smoke() and bench.py's CPU leg as
 * the checker. It is never the measured or shipped path.
 *
 * It follows the reference CPU backend step by step, with the correlation itself summed
 * directly (no FFT) so that the only rounding left is the one each mode asks for:
 *
 *   orc_sat            cxx/cpu.cpp:24-42      exact int64 summed-area tables of x and x^2
 *   ref_window         cxx/common.cpp:30-48   zero-mean window, its norm
 *   searchWindow       cxx/surface.h:39-45    search window placement and validity
 *   box                cxx/surface.h:21-25    4-corner box sums
 *   normalized         cxx/surface.h:30-35    the normalized correlation of one shift
 *   the argmax         cxx/cpu.cpp:146-160    strict '>' in raster order, first index on ties
 *   invalid windows    cxx/cpu.cpp:121-124, 161-164; cxx/surface.h:48-54
 *   write_peak         cxx/surface.h:71-146   3x3 fit, per-axis parabolas, SNR, covariance
 *
 * Two modes:
 *   ORC_REF32 (0): the reference's float arithmetic. The zero-mean window and its norm are
 *     float (common.cpp), the search window minus its float mean is float (cpu.cpp:132-137),
 *     the correlation is their exact sum (double, rounded once to float, i.e. what the FFT
 *     approximates), and normalized() and writePeak() run in float as in surface.h.
 *   ORC_F64 (1): every step in double (zero-mean window, norm, correlation, normalization,
 *     argmax, fit, SNR, covariance). This is the error reference for offsets, peaks and SNR.
 *
 * Parity pinning: tests/golden holds outputs of the reference's own CPU backend (built from its
 * sources by oracle/Makefile with the FFTW-API shim in oracle/fftw_shim); tests check both modes
 * against them.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_REF32 0
#define ORC_F64 1

typedef struct orc_params {
    int height, width;     /* the frame size */
    int window, search;    /* W, R */
    int stat_size;         /* the SNR window, 21 by default */
    const int *down;       /* ny first rows of the windows */
    int ny;
    const int *across;     /* nx first columns of the windows */
    int nx;
} orc_params;

/* the exact summed-area tables of x and x^2, (h + 1) x (w + 1), first row and column zero
 * (cxx/cpu.cpp:24-42) */
void orc_sat(const uint8_t *frame, int h, int w, int64_t *sat, int64_t *sat2)
{
    const size_t stride = (size_t)w + 1;
    memset(sat, 0, stride * sizeof(int64_t));
    memset(sat2, 0, stride * sizeof(int64_t));
    for (int y = 0; y < h; y++) {
        const uint8_t *row = frame + (size_t)y * w;
        int64_t *s = sat + (size_t)(y + 1) * stride, *s2 = sat2 + (size_t)(y + 1) * stride;
        const int64_t *above = s - stride, *above2 = s2 - stride;
        int64_t a = 0, b = 0;
        s[0] = s2[0] = 0;
        for (int x = 0; x < w; x++) {
            a += row[x];
            b += (int64_t)row[x] * row[x];
            s[x + 1] = above[x + 1] + a;
            s2[x + 1] = above2[x + 1] + b;
        }
    }
}

/* the sum over the n x n box with first pixel (y, x) (cxx/surface.h:21-25) */
static inline int64_t box(const int64_t *sat, int64_t stride, int y, int x, int n)
{
    return sat[(y + n) * stride + x + n] - sat[y * stride + x + n] - sat[(y + n) * stride + x]
        + sat[y * stride + x];
}

/* the normalized correlation in float (cxx/surface.h:30-35) */
static inline float normalized32(float corr, float norm, int64_t s, int64_t s2, int n)
{
    const int64_t v = n * s2 - s * s;
    if (v <= 0 || norm <= 0) return 0.0f;
    return corr / (norm * sqrtf((float)v / (float)n));
}

/* the same in double */
static inline double normalized64(double corr, double norm, int64_t s, int64_t s2, int n)
{
    const int64_t v = (int64_t)n * s2 - s * s;
    if (v <= 0 || norm <= 0) return 0.0;
    return corr / (norm * sqrt((double)v / (double)n));
}

static void invalidate(int64_t q, float *offset, float *peak, float *snr, float *cov, double *off64)
{
    offset[2 * q] = offset[2 * q + 1] = nanf("");
    peak[q] = snr[q] = 0.0f;
    cov[3 * q] = cov[3 * q + 1] = 99.0f;
    cov[3 * q + 2] = 0.0f;
    if (off64) off64[2 * q] = off64[2 * q + 1] = nan("");
}

static inline float parabola32(float m, float c, float p)
{
    const float den = m - 2 * c + p;
    return den < 0 ? 0.5f * (m - p) / den : 0.0f;
}

static inline double parabola64(double m, double c, double p)
{
    const double den = m - 2 * c + p;
    return den < 0 ? 0.5 * (m - p) / den : 0.0;
}

/* the outputs of one pair from its surface s (M x M, row stride M), in float for the sub-pixel
 * fit as cxx/surface.h:71-146 does, or in double; SNR and covariance are in double in both */
static void write_peak(const double *s, int M, int u, int v, int R, int gy, int gx, int stat,
                       int tsize, int64_t q, int f64, float *offset, float *peak, float *snr,
                       float *cov, double *off64)
{
    const double f0 = s[u * M + v];
    const int inside = u > 0 && u < M - 1 && v > 0 && v < M - 1;
    double du = 0.0, dv = 0.0;
    if (inside) {
        if (f64) {
            double f[3][3];
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++) f[i][j] = s[(u + i - 1) * M + v + j - 1];
            const double c1 = (f[2][0] + f[2][1] + f[2][2] - f[0][0] - f[0][1] - f[0][2]) / 6;
            const double c2 = (f[0][2] + f[1][2] + f[2][2] - f[0][0] - f[1][0] - f[2][0]) / 6;
            const double c3 = (f[0][0] + f[0][1] + f[0][2] + f[2][0] + f[2][1] + f[2][2]
                               - 2 * (f[1][0] + f[1][1] + f[1][2])) / 6;
            const double c5 = (f[0][0] + f[1][0] + f[2][0] + f[0][2] + f[1][2] + f[2][2]
                               - 2 * (f[0][1] + f[1][1] + f[2][1])) / 6;
            const double c4 = (f[2][2] - f[2][0] - f[0][2] + f[0][0]) / 4;
            const double det = 4 * c3 * c5 - c4 * c4;
            int fitted = 0;
            if (c3 < 0 && det > 0) {
                du = (c4 * c2 - 2 * c5 * c1) / det;
                dv = (c4 * c1 - 2 * c3 * c2) / det;
                fitted = fabs(du) <= 1 && fabs(dv) <= 1;
            }
            if (!fitted) {
                du = parabola64(f[0][1], f[1][1], f[2][1]);
                dv = parabola64(f[1][0], f[1][1], f[1][2]);
            }
        } else {
            float f[3][3];
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++) f[i][j] = (float)s[(u + i - 1) * M + v + j - 1];
            const float c1 = (f[2][0] + f[2][1] + f[2][2] - f[0][0] - f[0][1] - f[0][2]) / 6;
            const float c2 = (f[0][2] + f[1][2] + f[2][2] - f[0][0] - f[1][0] - f[2][0]) / 6;
            const float c3 = (f[0][0] + f[0][1] + f[0][2] + f[2][0] + f[2][1] + f[2][2]
                              - 2 * (f[1][0] + f[1][1] + f[1][2])) / 6;
            const float c5 = (f[0][0] + f[1][0] + f[2][0] + f[0][2] + f[1][2] + f[2][2]
                              - 2 * (f[0][1] + f[1][1] + f[2][1])) / 6;
            const float c4 = (f[2][2] - f[2][0] - f[0][2] + f[0][0]) / 4;
            const float det = 4 * c3 * c5 - c4 * c4;
            float fu = 0.0f, fv = 0.0f;
            int fitted = 0;
            if (c3 < 0 && det > 0) {
                fu = (c4 * c2 - 2 * c5 * c1) / det;
                fv = (c4 * c1 - 2 * c3 * c2) / det;
                fitted = fabsf(fu) <= 1 && fabsf(fv) <= 1;
            }
            if (!fitted) {
                fu = parabola32(f[0][1], f[1][1], f[2][1]);
                fv = parabola32(f[1][0], f[1][1], f[1][2]);
            }
            du = fu;
            dv = fv;
        }
    }
    if (f64) {
        offset[2 * q] = (float)((double)(gy + u - R) + du);
        offset[2 * q + 1] = (float)((double)(gx + v - R) + dv);
    } else {
        offset[2 * q] = (float)(gy + u - R) + (float)du;
        offset[2 * q + 1] = (float)(gx + v - R) + (float)dv;
    }
    if (off64) {
        off64[2 * q] = (double)(gy + u - R) + du;
        off64[2 * q + 1] = (double)(gx + v - R) + dv;
    }
    peak[q] = (float)f0;

    /* the SNR over the stat x stat patch clipped to the surface, without the peak */
    const int n = stat < M ? stat : M;
    double sum = 0.0;
    int count = 0;
    for (int a = 0; a < n; a++) {
        const int i = u + a - n / 2;
        if (i < 0 || i >= M) continue;
        for (int b = 0; b < n; b++) {
            const int j = v + b - n / 2;
            if (j < 0 || j >= M) continue;
            const double c = s[i * M + j];
            sum += c * c;
            count++;
        }
    }
    const double mean = count > 1 ? (sum - f0 * f0) / (count - 1) : 0.0;
    snr[q] = mean > 0 ? (float)(f0 * f0 / mean) : 0.0f;

    /* the covariance from the curvature at the peak */
    cov[3 * q] = cov[3 * q + 1] = 99.0f;
    cov[3 * q + 2] = 0.0f;
    if (inside) {
        const double T = tsize;
        const double dxx = -(s[(u + 1) * M + v] + s[(u - 1) * M + v] - 2.0 * f0) * T;
        const double dyy = -(s[u * M + v + 1] + s[u * M + v - 1] - 2.0 * f0) * T;
        const double dxy = (s[(u + 1) * M + v + 1] + s[(u - 1) * M + v - 1] - s[(u + 1) * M + v - 1]
                            - s[(u - 1) * M + v + 1]) * 0.25 * T;
        double n2 = 1.0 - f0 > 0 ? 1.0 - f0 : 0.0;
        const double n4 = n2 * n2 * 0.5 * T;
        n2 *= 2;
        const double w = dxy * dxy - dxx * dyy;
        if (fabs(w) >= 1e-2) {
            const double w2 = w * w;
            cov[3 * q] = (float)((-n2 * w * dyy + n4 * (dyy * dyy + dxy * dxy)) / w2);
            cov[3 * q + 1] = (float)((-n2 * w * dxx + n4 * (dxx * dxx + dxy * dxy)) / w2);
            cov[3 * q + 2] = (float)((n2 * w * dxy - n4 * (dxx + dyy) * dxy) / w2);
        }
    }
}

/* the zero-mean reference window k and its norm (cxx/common.cpp:30-48), in float values and
 * norm (ref32) and in double (f64) */
static void ref_window(const orc_params *p, const uint8_t *frame, int k, float *r32, double *r64,
                       float *norm32, double *norm64)
{
    const int W = p->window;
    const int y0 = p->down[k / p->nx], x0 = p->across[k % p->nx];
    double sum = 0.0;
    for (int i = 0; i < W; i++)
        for (int j = 0; j < W; j++) sum += frame[(size_t)(y0 + i) * p->width + x0 + j];
    const double mean = sum / ((double)W * W);
    double sq = 0.0, sq64 = 0.0;
    for (int i = 0; i < W; i++)
        for (int j = 0; j < W; j++) {
            const double x = frame[(size_t)(y0 + i) * p->width + x0 + j];
            const float d = (float)(x - mean);
            r32[i * W + j] = d;
            r64[i * W + j] = x - mean;
            sq += (double)d * d;
            sq64 += (x - mean) * (x - mean);
        }
    *norm32 = (float)sqrt(sq);
    *norm64 = sqrt(sq64);
}

/*
 * Correlate n frames with the reference frame.
 *   gross: n * ny * nx * 2 int32 (down, across) per pair, or NULL
 *   mode:  ORC_REF32 or ORC_F64
 *   outputs: offset n*nwin*2, peak, snr n*nwin, cov n*nwin*3 (float, the reference layout);
 *            off64 (nullable) the offsets in double; surf (nullable) n*nwin*M*M surfaces
 *   threads: OpenMP threads, 0 for the default
 * Returns 0, or -1 if the parameters are not valid.
 */
int orc_correlate(const orc_params *p, const uint8_t *ref, const uint8_t *frames, int n,
                  const int32_t *gross, int mode, float *offset, float *peak, float *snr, float *cov,
                  double *off64, double *surf, int threads)
{
    const int W = p->window, R = p->search, L = W + 2 * R, M = 2 * R + 1;
    const int nwin = p->ny * p->nx, h = p->height, w = p->width;
    if (h <= 0 || w <= 0 || W < 3 || R < 1 || nwin <= 0 || p->stat_size < 3 || n < 0) return -1;
    const int64_t stride = w + 1;
    const int f64 = mode == ORC_F64;

    float *r32 = malloc(sizeof(float) * (size_t)nwin * W * W);
    double *r64 = malloc(sizeof(double) * (size_t)nwin * W * W);
    float *norm32 = malloc(sizeof(float) * nwin);
    double *norm64 = malloc(sizeof(double) * nwin);
    int64_t *sat = malloc(sizeof(int64_t) * (size_t)n * (h + 1) * stride);
    int64_t *sat2 = malloc(sizeof(int64_t) * (size_t)n * (h + 1) * stride);
    if (!r32 || !r64 || !norm32 || !norm64 || (n && (!sat || !sat2))) {
        free(r32); free(r64); free(norm32); free(norm64); free(sat); free(sat2);
        return -2;
    }
#ifdef _OPENMP
    const int nt = threads > 0 ? threads : omp_get_max_threads();
#else
    const int nt = 1;
    (void)threads;
#endif
    #pragma omp parallel for num_threads(nt) schedule(static)
    for (int k = 0; k < nwin; k++)
        ref_window(p, ref, k, r32 + (size_t)k * W * W, r64 + (size_t)k * W * W, norm32 + k, norm64 + k);
    #pragma omp parallel for num_threads(nt) schedule(static)
    for (int f = 0; f < n; f++)
        orc_sat(frames + (size_t)f * h * w, h, w, sat + (size_t)f * (h + 1) * stride,
                sat2 + (size_t)f * (h + 1) * stride);

    const int64_t pairs = (int64_t)n * nwin;
    #pragma omp parallel num_threads(nt)
    {
        double *chip = malloc(sizeof(double) * (size_t)L * L);
        double *s = malloc(sizeof(double) * (size_t)M * M);
        double *acc = malloc(sizeof(double) * M);
        #pragma omp for schedule(dynamic, 4)
        for (int64_t q = 0; q < pairs; q++) {
            const int f = (int)(q / nwin), k = (int)(q % nwin);
            const int gy = gross ? gross[2 * q] : 0, gx = gross ? gross[2 * q + 1] : 0;
            const int y0 = p->down[k / p->nx], x0 = p->across[k % p->nx];
            const int sy = y0 + gy - R, sx = x0 + gx - R;
            const int inframe = sy >= 0 && sx >= 0 && sy + L <= h && sx + L <= w;
            if ((f64 ? norm64[k] : (double)norm32[k]) <= 0 || !inframe) {
                invalidate(q, offset, peak, snr, cov, off64);
                if (surf) memset(surf + q * M * M, 0, sizeof(double) * (size_t)M * M);
                continue;
            }
            const uint8_t *frame = frames + (size_t)f * h * w;
            const int64_t *st = sat + (size_t)f * (h + 1) * stride, *st2 = sat2 + (size_t)f * (h + 1) * stride;
            /* the search window minus its mean (cxx/cpu.cpp:132-137) */
            const int64_t csum = box(st, stride, sy, sx, L);
            const float mean32 = (float)csum / ((float)L * L);
            const double mean64 = (double)csum / ((double)L * L);
            for (int i = 0; i < L; i++)
                for (int j = 0; j < L; j++) {
                    const uint8_t x = frame[(size_t)(sy + i) * w + sx + j];
                    chip[i * L + j] = f64 ? (double)x - mean64 : (double)((float)x - mean32);
                }
            /* the correlation at every shift, summed directly, then normalized */
            const int nn = W * W;
            const float *rw32 = r32 + (size_t)k * nn;
            const double *rw64 = r64 + (size_t)k * nn;
            for (int u = 0; u < M; u++) {
                for (int v = 0; v < M; v++) acc[v] = 0.0;
                for (int i = 0; i < W; i++) {
                    const double *xr = chip + (size_t)(u + i) * L;
                    for (int j = 0; j < W; j++) {
                        const double r = f64 ? rw64[i * W + j] : (double)rw32[i * W + j];
                        const double *xx = xr + j;
                        for (int v = 0; v < M; v++) acc[v] += r * xx[v];
                    }
                }
                for (int v = 0; v < M; v++) {
                    const int64_t bs = box(st, stride, sy + u, sx + v, W), bs2 = box(st2, stride, sy + u, sx + v, W);
                    s[u * M + v] = f64 ? normalized64(acc[v], norm64[k], bs, bs2, nn)
                                       : (double)normalized32((float)acc[v], norm32[k], bs, bs2, nn);
                }
            }
            if (surf) memcpy(surf + q * M * M, s, sizeof(double) * (size_t)M * M);
            /* the peak: the largest, the first in raster order (cxx/cpu.cpp:148-160) */
            double best = -2.0;
            int bu = 0, bv = 0;
            for (int u = 0; u < M; u++)
                for (int v = 0; v < M; v++)
                    if (s[u * M + v] > best) {
                        best = s[u * M + v];
                        bu = u;
                        bv = v;
                    }
            if (!(best > 0)) {
                invalidate(q, offset, peak, snr, cov, off64);
                continue;
            }
            write_peak(s, M, bu, bv, R, gy, gx, p->stat_size, nn, q, f64, offset, peak, snr, cov, off64);
        }
        free(chip);
        free(s);
        free(acc);
    }
    free(r32); free(r64); free(norm32); free(norm64); free(sat); free(sat2);
    return 0;
}

/* the zero-mean reference windows (W x W, float as cxx/common.cpp:30-48) and their norms */
int orc_reference_windows(const orc_params *p, const uint8_t *ref, float *windows, float *norms)
{
    const int W = p->window, nwin = p->ny * p->nx;
    double *tmp = malloc(sizeof(double) * (size_t)W * W);
    if (!tmp) return -2;
    for (int k = 0; k < nwin; k++) {
        double n64;
        ref_window(p, ref, k, windows + (size_t)k * W * W, tmp, norms + k, &n64);
    }
    free(tmp);
    return 0;
}
