// diff.h -- the differentiable correlation of float frames: the normalized surface and the
// sub-pixel offsets as functions of the frame pixels and of a continuous shift of each search
// window, and their hand-written adjoints.
//
// Forward, for pair q = f * nwin + k with shift t = (ty, tx):
//   chip    x[i][j] = sum_{d,e} w_d(ay) w_e(ax) F_f[y0 - 2 + i + d][x0 - 2 + j + e]   (i, j < L)
//           with y0 = down + gy - R + floor(ty), ay = ty - floor(ty) (same across), w Keys'
//           six-point cubic convolution weights (C1 in t; at an integer shift x is the pixels);
//           frame indices are clamped to the frame (the edge pixel repeats)
//   stats   S1, S2 = sums of x, x^2 over the W x W box at (u, v); mu = S1 / n,
//           s(u, v) = sqrt(S2 - S1^2 / n) in FP64 (the reference's sqrt((n S2 - S1^2) / n))
//   surface rho(u, v) = c(u, v) / (norm s(u, v)), c(u, v) = sum_{i,j < W} r0[i][j] x[u + i][v + j]
//           (0 where s = 0), c from the FP32 FFT passes against the resident reference spectra
//   peak    the reference's argmax, 3 x 3 fit, SNR and covariance (corr_fft.cuh)
// Backward, from a cotangent G of the surface:
//   dL/dx[p] = sum_{u,v} A(u, v) r0[p - (u, v)] - sum_{(u,v): p in box(u,v)} B(u, v) (x[p] - mu(u, v))
//   with A = G / (norm s), B = G rho / s^2. The first term is a correlation too: with the
//   reversed cotangent a[n] = A[L - 1 - n] placed at rows and columns [W - 1, L), the FFT
//   correlation against the same resident spectra gives dL/dx[p] at output L - 1 - p (no
//   spectra are kept from the forward pass). The second is a pair of box filters (running sums).
//   The chip cotangent reaches the frames through the transposed interpolation and the shift
//   through the weights' derivatives.
//
// This header holds the arguments, the per-pair geometry and the offset adjoint (host and device)
// and the launches of diff.cu, where the kernels are.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "dft.cuh"

namespace b200 {

// Keys' six-point cubic convolution (fourth order, continuous first derivative): the weights of
// the taps at -2 .. 3 for a sample at fraction t in [0, 1), and their derivatives in t. At t = 0
// the weights are (0, 0, 1, 0, 0, 0): the pixel itself.
constexpr int kTaps = 6, kTap0 = -2;
B200_HD float keys1(float x) { return (4.0f / 3.0f * x - 7.0f / 3.0f) * x * x + 1.0f; }                // |x| < 1
B200_HD float keys2(float x) { return ((-7.0f / 12.0f * x + 3.0f) * x - 59.0f / 12.0f) * x + 2.5f; }   // 1 .. 2
B200_HD float keys3(float x) { return ((1.0f / 12.0f * x - 2.0f / 3.0f) * x + 1.75f) * x - 1.5f; }     // 2 .. 3
B200_HD float dkeys1(float x) { return (4.0f * x - 14.0f / 3.0f) * x; }
B200_HD float dkeys2(float x) { return (-1.75f * x + 6.0f) * x - 59.0f / 12.0f; }
B200_HD float dkeys3(float x) { return (0.25f * x - 4.0f / 3.0f) * x + 1.75f; }
B200_HD void interp_weights(float t, float (&w)[kTaps], float (&dw)[kTaps])
{
    w[0] = keys3(t + 2.0f);
    w[1] = keys2(t + 1.0f);
    w[2] = keys1(t);
    w[3] = keys1(1.0f - t);
    w[4] = keys2(2.0f - t);
    w[5] = keys3(3.0f - t);
    dw[0] = dkeys3(t + 2.0f);
    dw[1] = dkeys2(t + 1.0f);
    dw[2] = dkeys1(t);
    dw[3] = -dkeys1(1.0f - t);
    dw[4] = -dkeys2(2.0f - t);
    dw[5] = -dkeys3(3.0f - t);
}

struct DiffArgs {
    const float *frames;       // n frames, `pitch` floats per row, `fstride` floats per frame
    int64_t fstride;
    int pitch;
    int h, w, W, R, L, M, nx, nwin, n, stat;
    const int *down, *across;
    const float *norm;         // nwin
    const float2 *spec;        // the reference spectra (corr_fft.cuh order)
    const float2 *twiddles;    // 2N
    const int32_t *gross;      // nullptr, n x 2 or n x nwin x 2
    int gross_mode;
    const float *shift;        // nullptr or n x nwin x 2: (ty, tx) of each pair
    float *chips;              // n x nwin x L x L
    float *stats;              // n x nwin x M x M x 2: (mu, 1 / s) of each box (1 / s = 0 if s = 0)
    float *surface;            // n x nwin x M x M
    int *peak_at;              // n x nwin: u M + v of the peak, or -1
    float *offset, *peak, *snr, *cov;
    const float *g_surface;    // backward: n x nwin x M x M
    float *g_chips;            // n x nwin x L x L
    float *g_frames;           // n x h x pitch (accumulated into: zero it first)
    float *g_shift;            // n x nwin x 2
};

// a pair's search window in the frame: valid as the reference's (cxx/surface.h:39-45) at the
// floored position (y0, x0); interpolation taps beyond the frame's edge take the edge pixel
struct DiffPair {
    int f, k, gy, gx, y0, x0;
    float ay, ax;
    bool ok;
};

B200_HD DiffPair diff_pair(const DiffArgs &a, int64_t q)
{
    DiffPair p{};
    p.f = int(q / a.nwin);
    p.k = int(q % a.nwin);
    if (a.gross_mode == 1) {
        p.gy = a.gross[2 * p.f];
        p.gx = a.gross[2 * p.f + 1];
    } else if (a.gross_mode == 2) {
        p.gy = a.gross[2 * q];
        p.gx = a.gross[2 * q + 1];
    }
    const float ty = a.shift ? a.shift[2 * q] : 0.0f, tx = a.shift ? a.shift[2 * q + 1] : 0.0f;
    const float fy = floorf(ty), fx = floorf(tx);
    p.y0 = a.down[p.k / a.nx] + p.gy - a.R + int(fy);
    p.x0 = a.across[p.k % a.nx] + p.gx - a.R + int(fx);
    p.ay = ty - fy;
    p.ax = tx - fx;
    p.ok = a.norm[p.k] > 0 && p.y0 >= 0 && p.x0 >= 0 && p.y0 + a.L <= a.h && p.x0 + a.L <= a.w
        && fabsf(ty) < 1e6f && fabsf(tx) < 1e6f;
    return p;
}

// The cotangent of the surface's 3 x 3 neighbourhood of the peak (u, v) from the cotangent
// (gdu, gdv) of the sub-pixel offset, for the branch peak_outputs takes (the quadratic fit, else
// a parabola per axis; no sub-pixel at the edge: zero). c points at the peak value, rows `pitch`
// apart; g receives the 9 cotangents (row-major, g[4] at the peak).
B200_HD void offset_adjoint(const float *c, int pitch, int M, int u, int v, double gdu, double gdv, double (&g)[9])
{
    for (double &e : g) e = 0.0;
    if (!(u > 0 && u < M - 1 && v > 0 && v < M - 1)) return;
    double f[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) f[i][j] = c[(i - 1) * pitch + j - 1];
    constexpr double sixth = 1.0 / 6.0;
    const double c1 = (f[2][0] + f[2][1] + f[2][2] - f[0][0] - f[0][1] - f[0][2]) * sixth;
    const double c2 = (f[0][2] + f[1][2] + f[2][2] - f[0][0] - f[1][0] - f[2][0]) * sixth;
    const double c3 = (f[0][0] + f[0][1] + f[0][2] + f[2][0] + f[2][1] + f[2][2] - 2 * (f[1][0] + f[1][1] + f[1][2])) * sixth;
    const double c5 = (f[0][0] + f[1][0] + f[2][0] + f[0][2] + f[1][2] + f[2][2] - 2 * (f[0][1] + f[1][1] + f[2][1])) * sixth;
    const double c4 = (f[2][2] - f[2][0] - f[0][2] + f[0][0]) * 0.25;
    const double det = 4 * c3 * c5 - c4 * c4;
    if (c3 < 0 && det > 0) {
        const double rdet = 1.0 / det;
        const double nu = c4 * c2 - 2 * c5 * c1, nv = c4 * c1 - 2 * c3 * c2;
        const double du = nu * rdet, dv = nv * rdet;
        if (fabs(du) <= 1 && fabs(dv) <= 1) {
            // d(du), d(dv) by c1 .. c5, then by the 9 values
            const double r2 = rdet * rdet;
            const double gc1 = gdu * (-2 * c5 * rdet) + gdv * (c4 * rdet);
            const double gc2 = gdu * (c4 * rdet) + gdv * (-2 * c3 * rdet);
            const double gc3 = gdu * (-nu * 4 * c5 * r2) + gdv * (-2 * c2 * rdet - nv * 4 * c5 * r2);
            const double gc4 = gdu * (c2 * rdet + 2 * c4 * nu * r2) + gdv * (c1 * rdet + 2 * c4 * nv * r2);
            const double gc5 = gdu * (-2 * c1 * rdet - nu * 4 * c3 * r2) + gdv * (-nv * 4 * c3 * r2);
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++) {
                    const double d1 = (i == 2) - (i == 0), d2 = (j == 2) - (j == 0);
                    const double d3 = i == 1 ? -2.0 : 1.0, d5 = j == 1 ? -2.0 : 1.0;
                    const double d4 = (i != 1 && j != 1) ? (i == j ? 1.0 : -1.0) : 0.0;
                    g[3 * i + j] = (gc1 * d1 + gc2 * d2 + gc3 * d3 + gc5 * d5) * sixth + gc4 * d4 * 0.25;
                }
            return;
        }
    }
    // per-axis parabola through (m, c, p): 0.5 (m - p) / (m - 2c + p) when the denominator is negative
    auto parabola = [](double m, double cc, double pp, double gd, double &gm, double &gc, double &gp) {
        const double den = m - 2 * cc + pp;
        if (!(den < 0)) return;
        const double r2 = 1.0 / (den * den);
        gm += gd * (pp - cc) * r2;
        gp += gd * (cc - m) * r2;
        gc += gd * (m - pp) * r2;
    };
    parabola(f[0][1], f[1][1], f[2][1], gdu, g[1], g[4], g[7]);
    parabola(f[1][0], f[1][1], f[1][2], gdv, g[3], g[4], g[5]);
}

// the launches (diff.cu); N is the FFT size of the handle's geometry
void launch_diff_forward(const DiffArgs &a, int N, cudaStream_t s);    // chips, stats, surface, peaks
void launch_diff_backward(const DiffArgs &a, int N, cudaStream_t s);   // chip, frame, shift cotangents
void launch_offset_adjoint(const float *surface, const int *peak_at, const float *g_offset, float *g_surface,
                           int M, int64_t pairs, cudaStream_t s);   // into a zeroed g_surface

}   // namespace b200
