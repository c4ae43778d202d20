// stabilize.cu -- the coarse similarity tracking of python/slipcam/stabilize.py (ncc_peak :22-44,
// apply :47-51, coarse_track :54-96, with slip_series.fit_camera :49-72) after the correlation:
// the peak of each window's normalized surface refined by a parabola per axis, then, for the whole
// frame in one CTA, the robust similarity fit in float64, the frame's transform, and the gross
// offsets of the next frame's search windows predicted from it. The frame loop therefore needs no
// host round trip: correlation -> peaks -> fit -> the next frame's correlation, stream-ordered.

#include <climits>
#include <cmath>
#include <cstdint>

#include <cuda_runtime.h>

#include "../../include/slipcam_b200.h"
#include "ncc_peak.cuh"
#include "stabilize.h"

namespace b200 {
namespace {

constexpr int kPeakThreads = 256;
constexpr int kFitThreads = 512;
constexpr int kFitWarps = kFitThreads / 32;
constexpr int kGrossLimit = 1 << 29;   // a predicted position beyond this is outside every frame

// the peak of each of a batch of M x M surfaces (ncc_peak.cuh), one CTA per surface
__global__ void __launch_bounds__(kPeakThreads) ncc_peak_kernel(const float *__restrict__ surface, int M,
                                                                double *__restrict__ out)
{
    ncc_peak_block<kPeakThreads>(surface + size_t(blockIdx.x) * M * M, M, M, out + 3 * size_t(blockIdx.x));
}

// stabilize.apply: x' = x + p - a y + s x, y' = y + q + a x + s y, evaluated left to right with
// every product and sum rounded on its own (no fused multiply-add), as numpy evaluates it
__device__ __forceinline__ void similarity(const double *m, double x, double y, double &xo, double &yo)
{
    xo = __dadd_rn(__dsub_rn(__dadd_rn(x, m[0]), __dmul_rn(m[2], y)), __dmul_rn(m[3], x));
    yo = __dadd_rn(__dadd_rn(__dadd_rn(y, m[1]), __dmul_rn(m[2], x)), __dmul_rn(m[3], y));
}

// the n finite entries of v[0, m) (the others +inf) in ascending order into srt[0, n): each entry's
// rank among them (ties broken by position) counted by up to kFitThreads / m threads, each over a
// slice of the entries, then the entries scattered to their ranks. rank: m ints of shared memory.
__device__ void sort_by_rank(const double *v, int m, double *srt, int *rank)
{
    const int S = max(1, kFitThreads / m);
    for (int i = threadIdx.x; i < m; i += kFitThreads) rank[i] = 0;
    __syncthreads();
    if (S > 1) {
        const int i = threadIdx.x % m, sl = threadIdx.x / m;
        if (threadIdx.x < S * m) {
            const double x = v[i];
            if (x < INFINITY) {
                const int j0 = sl * m / S, j1 = (sl + 1) * m / S;
                int r = 0;
#pragma unroll 8
                for (int j = j0; j < j1; ++j) {
                    const double y = v[j];
                    r += (y < x) | ((y == x) & (j < i));
                }
                atomicAdd(rank + i, r);
            }
        }
    } else {
        for (int i = threadIdx.x; i < m; i += kFitThreads) {
            const double x = v[i];
            if (!(x < INFINITY)) continue;
            int r = 0;
#pragma unroll 8
            for (int j = 0; j < m; ++j) {
                const double y = v[j];
                r += (y < x) | ((y == x) & (j < i));
            }
            rank[i] = r;
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < m; i += kFitThreads)
        if (v[i] < INFINITY) srt[rank[i]] = v[i];
    __syncthreads();
}

// numpy.median(|s - med|) of the n ascending values srt (med their median): the k + 1 values closest
// to med are consecutive in srt, so the k-th smallest deviation is the least, over the windows of
// k + 1 consecutive values, of the larger deviation at the window's two ends. The two middle ranks
// in one reduction over the windows.
__device__ double median_abs_dev(const double *srt, int n, double med, double *red2)
{
    const int k1 = (n - 1) / 2, k2 = n / 2;
    double b1 = INFINITY, b2 = INFINITY;
    for (int a0 = threadIdx.x; a0 < n; a0 += kFitThreads) {
        const double lo = fabs(srt[a0] - med);
        if (a0 + k1 < n) b1 = fmin(b1, fmax(lo, fabs(srt[a0 + k1] - med)));
        if (a0 + k2 < n) b2 = fmin(b2, fmax(lo, fabs(srt[a0 + k2] - med)));
    }
    for (int o = 16; o > 0; o >>= 1) {
        b1 = fmin(b1, __shfl_xor_sync(0xffffffffu, b1, o));
        b2 = fmin(b2, __shfl_xor_sync(0xffffffffu, b2, o));
    }
    const int warp = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        red2[2 * warp] = b1;
        red2[2 * warp + 1] = b2;
    }
    __syncthreads();
    double d1 = INFINITY, d2 = INFINITY;
    for (int w = 0; w < kFitWarps; ++w) {
        d1 = fmin(d1, red2[2 * w]);
        d2 = fmin(d2, red2[2 * w + 1]);
    }
    __syncthreads();
    return n % 2 ? d2 : (d1 + d2) / 2;
}

// sum over the CTA of kTerms doubles per thread, the same order on every run; the totals land in tot
template <int kTerms>
__device__ void block_sum(double (&x)[kTerms], double *red, double *tot)
{
    for (int t = 0; t < kTerms; ++t)
        for (int o = 16; o > 0; o >>= 1) x[t] += __shfl_xor_sync(0xffffffffu, x[t], o);
    const int warp = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0)
        for (int t = 0; t < kTerms; ++t) red[warp * kTerms + t] = x[t];
    __syncthreads();
    if (threadIdx.x < kTerms) {
        double s = 0;
        for (int w = 0; w < kFitWarps; ++w) s += red[w * kTerms + threadIdx.x];
        tot[threadIdx.x] = s;
    }
    __syncthreads();
}


// One frame of coarse_track after its peaks (stabilize.py:80-95): the offsets of the windows whose
// search window lies inside the frame and whose peak reaches min_peak, the fit of
// slip_series.fit_camera (three rounds of least squares, each dropping the windows with a residual
// of at least max(3 MAD, 0.3) pixels in either component; no fit below 4 windows), the frame's
// transform (the previous one, and 0 windows, when there is no fit), then the next frame's gross
// offsets: the rounded (half to even) position of each window under the transform, minus its
// grid position. One CTA; shared memory: 10 nwin doubles, 2 nwin ints and nwin bytes.
__global__ void __launch_bounds__(kFitThreads) coarse_fit_kernel(FitArgs a)
{
    extern __shared__ double smem[];
    const int nwin = a.ny * a.nx, half = a.window / 2;
    double *d = smem;              // 2 nwin: dx of every window, then dy
    double *r = d + 2 * nwin;      // 2 nwin: the residuals of the current fit
    double *v = r + 2 * nwin;      // 2 nwin: the entries of a median (+inf: not in use)
    double *xy = v + 2 * nwin;     // 2 nwin: each window's centre relative to the image centre (X, then Y)
    double *srt = xy + 2 * nwin;   // 2 nwin: the residuals in use, ascending
    int *rank = reinterpret_cast<int *>(srt + 2 * nwin);        // 2 nwin
    uint8_t *use = reinterpret_cast<uint8_t *>(rank + 2 * nwin);   // nwin
    __shared__ double red[kFitWarps * 14], tot[14], m[4];
    __shared__ int s_count;

    const double hw = a.width / 2.0, hh = a.height / 2.0;
    for (int k = threadIdx.x; k < nwin; k += kFitThreads) {
        const int Yg = a.yc[k / a.nx] + a.coff, Xg = a.xc[k % a.nx] + a.coff;
        const int gy = a.gross[2 * k], gx = a.gross[2 * k + 1];
        // the search window's corner, as stabilize.py:84-86
        const int y0 = Yg + gy - half - a.search, x0 = Xg + gx - half - a.search, L = a.window + 2 * a.search;
        const bool inside = y0 >= 0 && x0 >= 0 && y0 + L <= a.height && x0 + L <= a.width;
        const double oy = a.peaks[3 * k], ox = a.peaks[3 * k + 1], pk = a.peaks[3 * k + 2];
        const bool ok = a.keep[k] && inside && pk >= a.min_peak;
        use[k] = ok;
        xy[k] = Xg - hw;
        xy[nwin + k] = Yg - hh;
        // (x0 + search + half + ox) - w/2 - X0 with X0 = Xg - w/2, the reference's order
        d[k] = ok ? (double(x0 + a.search + half) + ox - hw) - (Xg - hw) : NAN;
        d[nwin + k] = ok ? (double(y0 + a.search + half) + oy - hh) - (Yg - hh) : NAN;
    }
    __syncthreads();

    bool failed = false;
    for (int it = 0; it < 3 && !failed; ++it) {
        // the least squares of dx = p - a Y + s X, dy = q + a X + s Y over the windows in use, in
        // closed form: about the means, s and a are the projections of the centred offsets on the
        // centred positions (x, y) and (-y, x); p and q restore the means. One reduction of the
        // raw moments (the grid is near the image centre: centring them after the sums loses
        // nothing that matters at these magnitudes)
        double t[8] = {};
        for (int k = threadIdx.x; k < nwin; k += kFitThreads) {
            if (!use[k]) continue;
            const double X = xy[k], Y = xy[nwin + k], dx = d[k], dy = d[nwin + k];
            t[0] += 1;
            t[1] += X;
            t[2] += Y;
            t[3] += dx;
            t[4] += dy;
            t[5] += X * X + Y * Y;
            t[6] += X * dx + Y * dy;
            t[7] += X * dy - Y * dx;
        }
        block_sum<8>(t, red, tot);
        const int nuse_it = int(tot[0]);
        if (2 * nuse_it < 8) {   // fewer than 8 rows in use
            failed = true;
            break;
        }
        if (threadIdx.x == 0) {
            const double n = nuse_it, mx = tot[1] / n, my = tot[2] / n, mdx = tot[3] / n, mdy = tot[4] / n;
            const double sxx = tot[5] - n * (mx * mx + my * my);
            const double sc = (tot[6] - n * (mx * mdx + my * mdy)) / sxx;
            const double rot = (tot[7] - n * (mx * mdy - my * mdx)) / sxx;
            m[0] = mdx + rot * my - sc * mx;
            m[1] = mdy - rot * mx - sc * my;
            m[2] = rot;
            m[3] = sc;
            s_count = nuse_it;
        }
        __syncthreads();
        // the residuals of the rows in use (NaN elsewhere); the median of the used ones
        for (int k = threadIdx.x; k < nwin; k += kFitThreads) {
            const double X = xy[k], Y = xy[nwin + k];
            const bool u = use[k];
            r[k] = u ? d[k] - (m[0] - Y * m[2] + X * m[3]) : NAN;
            r[nwin + k] = u ? d[nwin + k] - (m[1] + X * m[2] + Y * m[3]) : NAN;
        }
        __syncthreads();
        const int n = 2 * s_count;
        for (int i = threadIdx.x; i < 2 * nwin; i += kFitThreads) v[i] = use[i % nwin] ? r[i] : INFINITY;
        sort_by_rank(v, 2 * nwin, srt, rank);
        const double med = n % 2 ? srt[n / 2] : (srt[n / 2 - 1] + srt[n / 2]) / 2;   // numpy.median
        const double mad = 1.4826 * median_abs_dev(srt, n, med, red);
        const double thr = fmax(3 * mad, 0.3);
        for (int k = threadIdx.x; k < nwin; k += kFitThreads)
            use[k] = use[k] && fabs(r[k]) < thr && fabs(r[nwin + k]) < thr;
        __syncthreads();
    }

    // the frame's transform, and the next frame's prediction (stabilize.py:91-95, 80-84)
    int nuse = 0;
    for (int k = threadIdx.x; k < nwin; k += kFitThreads) nuse += use[k];
    for (int o = 16; o > 0; o >>= 1) nuse += __shfl_xor_sync(0xffffffffu, nuse, o);
    __syncthreads();
    if (threadIdx.x == 0) s_count = 0;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) atomicAdd(&s_count, nuse);
    __syncthreads();
    if (threadIdx.x == 0) {
        const bool fit = !failed && isfinite(m[0]) && isfinite(m[1]) && isfinite(m[2]) && isfinite(m[3]);
        for (int t = 0; t < 4; ++t) {
            if (fit) a.prev[t] = m[t];
            a.params[t] = a.prev[t];
            m[t] = a.prev[t];
        }
        *a.used = fit ? s_count : 0;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < nwin; k += kFitThreads) {
        const int Yg = a.yc[k / a.nx] + a.coff, Xg = a.xc[k % a.nx] + a.coff;
        double px, py;
        similarity(m, Xg - hw, Yg - hh, px, py);
        const double cx = rint(__dadd_rn(px, hw)), cy = rint(__dadd_rn(py, hh));
        const bool far = !(fabs(cx) < kGrossLimit && fabs(cy) < kGrossLimit);
        a.gross[2 * k] = far ? kGrossLimit : int(cy) - Yg;
        a.gross[2 * k + 1] = far ? kGrossLimit : int(cx) - Xg;
    }
}


}   // namespace

size_t coarse_fit_smem(int nwin) { return size_t(10) * nwin * sizeof(double) + size_t(2) * nwin * sizeof(int) + nwin; }

cudaError_t launch_ncc_peaks(const float *surface, int n, int M, double *out, cudaStream_t s)
{
    if (n > 0) ncc_peak_kernel<<<unsigned(n), kPeakThreads, 0, s>>>(surface, M, out);
    return cudaGetLastError();
}

cudaError_t launch_coarse_fit(const FitArgs &a, cudaStream_t s)
{
    static bool attr_set[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < 64 && !attr_set[dev]) {
        e = cudaFuncSetAttribute(coarse_fit_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(coarse_fit_smem(B200_COARSE_MAX_WINDOWS)));
        if (e != cudaSuccess) return e;
        attr_set[dev] = true;
    }
    coarse_fit_kernel<<<1, kFitThreads, coarse_fit_smem(a.ny * a.nx), s>>>(a);
    return cudaGetLastError();
}

}   // namespace b200

extern "C" {

int b200_ncc_peaks_device(const float *surface, int n, int M, double *out, void *stream)
{
    if (n < 0 || M < 1 || (n && (!surface || !out))) return B200_EINVAL;
    return b200::launch_ncc_peaks(surface, n, M, out, static_cast<cudaStream_t>(stream)) == cudaSuccess ? B200_OK
                                                                                                     : B200_ERUNTIME;
}

int b200_coarse_fit_device(const double *peaks, int32_t *gross, const uint8_t *keep, const int32_t *yc,
                           const int32_t *xc, int ny, int nx, int height, int width, int window, int search,
                           double min_peak, double *prev, double *params, int32_t *used, void *stream)
{
    if (ny < 1 || nx < 1 || int64_t(ny) * nx > B200_COARSE_MAX_WINDOWS || height < 1 || width < 1 || window < 2
        || search < 0 || !peaks || !gross || !keep || !yc || !xc || !prev || !params || !used)
        return B200_EINVAL;
    b200::FitArgs a{peaks, gross, keep, yc, xc, 0, ny, nx, height, width, window, search, min_peak, prev, params, used};
    return b200::launch_coarse_fit(a, static_cast<cudaStream_t>(stream)) == cudaSuccess ? B200_OK : B200_ERUNTIME;
}

}   // extern "C"
