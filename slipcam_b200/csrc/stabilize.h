// stabilize.h -- the launches of the coarse similarity tracking kernels (stabilize.cu), for the
// handle's frame loop in capi.cu.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace b200 {

struct FitArgs {
    const double *peaks;     // nwin x 3: (dy, dx, peak) of each window's surface
    int32_t *gross;          // nwin x 2 (down, across): read, then overwritten with the next frame's
    const uint8_t *keep;     // nwin: the window is used (no text, not flat)
    const int32_t *yc, *xc;  // the rows and columns of the grid; the centres are these plus coff
    int coff;
    int ny, nx, height, width, window, search;
    double min_peak;
    double *prev;            // 4: the transform the frame was predicted from; then the frame's (if fitted)
    double *params;          // 4: the frame's transform
    int32_t *used;           // 1: the windows of the fit
};

// the peak of each of n M x M surfaces, refined by a parabola per axis: n x 3 doubles (dy, dx, value)
cudaError_t launch_ncc_peaks(const float *surface, int n, int M, double *out, cudaStream_t s);

// the robust similarity fit of one frame and the next frame's gross offsets (one CTA)
cudaError_t launch_coarse_fit(const FitArgs &a, cudaStream_t s);

}   // namespace b200
