// multi.h -- several window grids of one set of frames in one persistent launch (multi.cu): the
// arguments and the launch. Each grid keeps its own windows, reference spectra and variance
// denominators (its window size); the frames and their summed-area tables are shared.
#pragma once

#include <cstddef>

#include <cuda_runtime.h>

#include "common.cuh"

namespace b200 {

constexpr int kMaxGrids = 4;

struct MultiGrid {
    CorrArgs a;      // the grid's correlation arguments (all nf frames of the call)
    int N;           // its FFT size
    int chunk;       // (window, frame) pairs per work item, window-major: a chunk shares a spectrum
    int items;       // its work items: ceil(nwin nf / chunk)
};

struct MultiArgs {
    MultiGrid g[kMaxGrids];
    int ngrids;
    int order[kMaxGrids];     // the grids in work-list order (costliest first spreads the tail)
    int total_items;
    int *counter;             // the next work item (zero before the launch)
    float2 *big_scratch;      // per-CTA scratch of an N = 256 grid (corr_big.cuh), or nullptr
    size_t big_per_cta;
};

// the dynamic shared memory a pair of FFT size N needs in the multi-grid kernel
size_t multi_smem(int N);
// whether the multi-grid kernel holds FFT size N
bool multi_supports(int N);
// one persistent launch of `grid` CTAs of nt threads (256 or 512), smem bytes of shared memory;
// m points to the arguments in device memory (read by the kernel; the counter is zeroed first)
void launch_corr_multi(const MultiArgs *m, int nt, size_t smem, int grid, cudaStream_t s);
// the kernel attributes, outside any stream capture
void prepare_multi();
// resident CTAs per SM of the multi-grid kernel with nt threads and smem bytes of shared memory
int multi_occupancy(int nt, size_t smem);

}   // namespace b200
