// common.cuh -- shared types of the b200 correlator kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "dft.cuh"

namespace b200 {

// The geometry of the FFT tile used for one search window: an N x N transform (N = 16 * N2 >= L,
// the search-window size W + 2R), split as N = N1 * N2 with N1 = 16 for every 1-D transform.
// The half spectrum is held in shared memory as N rows of NHP complex values (NH = N/2 + 1 used,
// one column of padding: NHP = NH + 1 is twice an odd number for N a multiple of 16, which keeps
// the strided column accesses of a warp (two columns, eight rows per half-warp) on distinct banks).
template <int N>
struct Geo {
    static constexpr int N1 = 16;
    static constexpr int N2 = N / 16;
    static constexpr int NH = N / 2 + 1;
    static constexpr int NHP = NH + 1;
    static constexpr int RP = 2 * NHP;              // a row as reals: its pitch in floats
    static constexpr int NU = (NH + 15) / 16;       // unpack steps of 16 frequencies
    static_assert(N % 16 == 0 && N2 >= 1 && N2 <= 16, "N must be 16 * N2, N2 in 1..16");
    static constexpr size_t tile_bytes = size_t(N) * NHP * sizeof(float2);
    static constexpr size_t smem_bytes = tile_bytes + 2 * N * sizeof(float2);   // + twiddles
};

// The exchange slot of element (n2, k1) between the two steps of a length-N transform: the N2
// rows of 16 are rotated by XOR so that a warp writing one k1 for many n2, or reading many k1 for
// one n2, touches distinct banks.
B200_HD int xpos(int n2, int k1) { return n2 * 16 + (k1 ^ n2); }

// the arguments of the reference-spectra kernel
struct SpectraArgs {
    const uint8_t *frame;      // the reference frame
    const float *framef;       // or a float reference frame (frame is then unused)
    int pitch;                 // elements per row
    int W, nx;
    const int *down, *across;
    float *norm;               // out: nwin norms of the zero-mean windows
    float2 *spec;              // out: nwin x NH x N spectra (see corr_fft.cuh for the order)
    const float2 *twiddles;    // 2N: the twiddle tables of the N-point transform
};

// what the tensor-core kernel leaves for the exact refinement of a pair's peak: the integer peak,
// the SNR patch's count and sum of squares, and the 3 x 3 values around the peak it used
struct PeakInfo {
    int valid, u, v, count;
    double sum;
    float fit[9];
    int pad;
};

// the arguments of the correlation kernels: one group of nf frames
struct CorrArgs {
    const uint8_t *frames;     // nf frames, `pitch` bytes per row, `fstride` bytes per frame
    int64_t fstride;
    int pitch;
    const uint32_t *sat;       // nf x (h + 1) x (w + 1): the summed-area table of the pixels
    int64_t sat_fstride;       // elements per frame
    const float *dinv;         // nf x h x dpitch: 1 / sqrt(variance * n) of each W x W box (0 if flat)
    int64_t dinv_fstride;
    int dpitch;                // floats per row of dinv: the width rounded up to 4 (16-byte rows)
    int h, w, W, R, L, M, nx, nwin, nf, stat;
    const int *down, *across;
    const float *norm;         // nwin
    const float2 *spec;        // the reference spectra
    const float4 *spec_tc;     // the same, in the order the tensor-core form reads them (or nullptr)
    const float2 *twiddles;    // 2N
    const int32_t *gross;      // nullptr, nf x 2 (per frame) or nf x nwin x 2 (per window)
    int gross_mode;            // 0 none, 1 per frame, 2 per window
    float *offset, *peak, *snr, *cov;   // nf x nwin (x 2, x 3), the pairs of this group
    float *surface;            // nullptr, or nf x nwin x M x M: the normalized surfaces
    double *ncc;               // nullptr, or nf x nwin x 3: stabilize.ncc_peak's (dy, dx, value) of each
                               // surface ((NaN, NaN, -inf) for an invalid pair)
    const int2 *bstat;         // nullptr, or nf x h x dpitch: {pixel sum, dinv bits} of each W x W box
                               // (the exact tensor-core form's table, beside dinv)
    PeakInfo *peaks;           // nullptr, or nf x nwin: the tensor-core kernel's peaks for refinement
};

}   // namespace b200
