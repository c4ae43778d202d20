// multi.cu -- the multi-grid persistent correlation kernel (multi.h): CTAs draw work items
// (chunks of window-major pairs of one grid) from a device counter until the list is exhausted
// and run each pair through the FP32 FFT correlation of its grid's size (corr_pair, or
// corr_big_pair for N = 256). No CTA waits on another.

#include <stdexcept>
#include <string>

#include "corr_big.cuh"
#include "multi.h"

namespace b200 {
namespace {

constexpr size_t kMultiSmem = 160 * 1024;   // the largest need: Geo<192> (154 KB)

// one pair of FFT size N, register-allocated on its own (the persistent kernel calls the size a
// work item needs; inlining every size into the kernel would make the sizes share one frame)
template <int N, int NT>
__device__ __noinline__ void multi_pair(const CorrArgs &a, int p, float2 *S, float2 *scratch)
{
    if constexpr (N == 256)
        corr_big_pair<256, NT>(a, p, S, scratch);
    else
        corr_pair<N, NT>(a, p / a.nf, p % a.nf, S);
}

// the arguments live in global memory (a grid is picked at run time: indexing the kernel's
// parameters dynamically would copy them to the stack); each work item copies its grid's
// correlation arguments to shared memory once
template <int NT>
__global__ void __launch_bounds__(NT, 1) corr_multi_kernel(const MultiArgs *__restrict__ mp)
{
    extern __shared__ float4 smem_raw[];
    float2 *S = reinterpret_cast<float2 *>(smem_raw);
    __shared__ int s_item, s_grid, s_base;
    __shared__ __align__(16) CorrArgs s_args;
    const int total = mp->total_items, ngrids = mp->ngrids;
    for (;;) {
        if (threadIdx.x == 0) {
            const int item = atomicAdd(mp->counter, 1);
            int gi = mp->order[0], base = 0;
            for (int o = 0; o < ngrids; ++o) {
                gi = mp->order[o];
                if (item < base + mp->g[gi].items) break;
                base += mp->g[gi].items;
            }
            s_item = item;
            s_grid = gi;
            s_base = base;
        }
        __syncthreads();
        const int item = s_item, gi = s_grid, base = s_base;
        if (item >= total) break;
        {
            const int *src = reinterpret_cast<const int *>(&mp->g[gi].a);
            int *dst = reinterpret_cast<int *>(&s_args);
            for (int i = threadIdx.x; i < int(sizeof(CorrArgs) / 4); i += NT) dst[i] = src[i];
        }
        __syncthreads();
        const CorrArgs &a = s_args;
        const int N = mp->g[gi].N, chunk = mp->g[gi].chunk;
        const int npairs = a.nwin * a.nf;
        const int p0 = (item - base) * chunk, p1 = min(p0 + chunk, npairs);
        for (int p = p0; p < p1; ++p) {
            switch (N) {
            case 16: multi_pair<16, NT>(a, p, S, nullptr); break;
            case 32: multi_pair<32, NT>(a, p, S, nullptr); break;
            case 48: multi_pair<48, NT>(a, p, S, nullptr); break;
            case 64: multi_pair<64, NT>(a, p, S, nullptr); break;
            case 80: multi_pair<80, NT>(a, p, S, nullptr); break;
            case 96: multi_pair<96, NT>(a, p, S, nullptr); break;
            case 128: multi_pair<128, NT>(a, p, S, nullptr); break;
            case 144: multi_pair<144, NT>(a, p, S, nullptr); break;
            case 160: multi_pair<160, NT>(a, p, S, nullptr); break;
            case 192: multi_pair<192, NT>(a, p, S, nullptr); break;
            case 256: multi_pair<256, NT>(a, p, S, mp->big_scratch + size_t(blockIdx.x) * mp->big_per_cta); break;
            default: break;
            }
            __syncthreads();
        }
    }
}

}   // namespace

bool multi_supports(int N)
{
    switch (N) {
    case 16: case 32: case 48: case 64: case 80: case 96: case 128: case 144: case 160: case 192: case 256: return true;
    default: return false;
    }
}

size_t multi_smem(int N)
{
    switch (N) {
    case 16: return Geo<16>::smem_bytes;
    case 32: return Geo<32>::smem_bytes;
    case 48: return Geo<48>::smem_bytes;
    case 64: return Geo<64>::smem_bytes;
    case 80: return Geo<80>::smem_bytes;
    case 96: return Geo<96>::smem_bytes;
    case 128: return Geo<128>::smem_bytes;
    case 144: return Geo<144>::smem_bytes;
    case 160: return Geo<160>::smem_bytes;
    case 192: return Geo<192>::smem_bytes;
    case 256: return BigGeo<256>::smem_bytes;
    default: return 0;
    }
}

static_assert(Geo<192>::smem_bytes <= kMultiSmem && BigGeo<256>::smem_bytes <= kMultiSmem, "multi-grid shared memory");

void prepare_multi()
{
    static bool done[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) throw std::runtime_error("cudaGetDevice failed");
    if (dev >= 0 && dev < 64 && done[dev]) return;
    for (cudaError_t e : {cudaFuncSetAttribute(corr_multi_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kMultiSmem)),
                          cudaFuncSetAttribute(corr_multi_kernel<512>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kMultiSmem))})
        if (e != cudaSuccess) throw std::runtime_error(std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
    if (dev >= 0 && dev < 64) done[dev] = true;
}

int multi_occupancy(int nt, size_t smem)
{
    int blocks = 0;
    const cudaError_t e = nt == 512 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, corr_multi_kernel<512>, 512, smem)
                                    : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, corr_multi_kernel<256>, 256, smem);
    if (e != cudaSuccess) throw std::runtime_error(std::string("occupancy: ") + cudaGetErrorString(e));
    return blocks > 0 ? blocks : 1;
}

void launch_corr_multi(const MultiArgs *m, int nt, size_t smem, int grid, cudaStream_t s)
{
    if (smem > kMultiSmem) throw std::invalid_argument("multi-grid shared memory");
    if (nt == 512)
        corr_multi_kernel<512><<<unsigned(grid), 512, smem, s>>>(m);
    else
        corr_multi_kernel<256><<<unsigned(grid), 256, smem, s>>>(m);
}

}   // namespace b200
