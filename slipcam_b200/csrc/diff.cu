// diff.cu -- the launches of the differentiable correlation (diff.cuh): one CTA per pair for
// every stage; the FFT stages are instantiated for the FFT sizes of the correlation kernels.

#include <stdexcept>
#include <string>

#include "diff.cuh"

namespace b200 {
namespace {

constexpr int kNT = 256;

void ck(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// the dynamic shared memory limits, once per device and kernel instance
template <int N>
void prepare()
{
    static bool done[64] = {};
    int dev = 0;
    ck(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev >= 0 && dev < 64 && done[dev]) return;
    ck(cudaFuncSetAttribute(diff_corr_kernel<N, kNT>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(Geo<N>::smem_bytes)),
       "cudaFuncSetAttribute");
    ck(cudaFuncSetAttribute(adjoint_kernel<N, kNT>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(Geo<N>::smem_bytes)),
       "cudaFuncSetAttribute");
    ck(cudaFuncSetAttribute(diff_stats_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * 256 * kStatStrip * 8),
       "cudaFuncSetAttribute");
    if (dev >= 0 && dev < 64) done[dev] = true;
}

template <int N>
void corr(const DiffArgs &a, unsigned pairs, cudaStream_t s)
{
    prepare<N>();
    diff_corr_kernel<N, kNT><<<pairs, kNT, Geo<N>::smem_bytes, s>>>(a);
}

template <int N>
void adjoint(const DiffArgs &a, unsigned pairs, cudaStream_t s)
{
    prepare<N>();
    adjoint_kernel<N, kNT><<<pairs, kNT, Geo<N>::smem_bytes, s>>>(a);
}

#define B200_DIFF_DISPATCH(N_, F, ...)                                                             \
    switch (N_) {                                                                                  \
    case 16: F<16>(__VA_ARGS__); break;                                                            \
    case 32: F<32>(__VA_ARGS__); break;                                                            \
    case 48: F<48>(__VA_ARGS__); break;                                                            \
    case 64: F<64>(__VA_ARGS__); break;                                                            \
    case 80: F<80>(__VA_ARGS__); break;                                                            \
    case 96: F<96>(__VA_ARGS__); break;                                                            \
    case 128: F<128>(__VA_ARGS__); break;                                                          \
    case 144: F<144>(__VA_ARGS__); break;                                                          \
    case 160: F<160>(__VA_ARGS__); break;                                                          \
    case 192: F<192>(__VA_ARGS__); break;                                                          \
    default: throw std::invalid_argument("no differentiable kernel for the FFT size " + std::to_string(N_)); \
    }

unsigned pair_grid(const DiffArgs &a)
{
    const int64_t pairs = int64_t(a.n) * a.nwin;
    if (pairs > int64_t(0x7fffffff)) throw std::invalid_argument("too many pairs for one launch");
    if (a.L > 256) throw std::invalid_argument("the differentiable path holds search windows up to 256 pixels");
    return unsigned(pairs);
}

}   // namespace

void launch_diff_forward(const DiffArgs &a, int N, cudaStream_t s)
{
    const unsigned pairs = pair_grid(a);
    if (!pairs) return;
    B200_DIFF_DISPATCH(N, prepare);
    diff_gather_kernel<<<pairs, 256, 0, s>>>(a);
    diff_stats_kernel<<<pairs, 256, size_t(2) * a.L * kStatStrip * sizeof(double), s>>>(a);
    B200_DIFF_DISPATCH(N, corr, a, pairs, s);
    ck(cudaGetLastError(), "the differentiable forward launches");
}

void launch_diff_backward(const DiffArgs &a, int N, cudaStream_t s)
{
    const unsigned pairs = pair_grid(a);
    if (!pairs) return;
    B200_DIFF_DISPATCH(N, adjoint, a, pairs, s);
    diff_scatter_kernel<<<pairs, 256, 0, s>>>(a);
    ck(cudaGetLastError(), "the differentiable backward launches");
}

void launch_offset_adjoint(const float *surface, const int *peak_at, const float *g_offset, float *g_surface, int M,
                           int64_t pairs, cudaStream_t s)
{
    if (pairs <= 0) return;
    offset_adjoint_kernel<<<unsigned((pairs + 127) / 128), 128, 0, s>>>(surface, peak_at, g_offset, g_surface, M, pairs);
    ck(cudaGetLastError(), "the offset adjoint launch");
}

}   // namespace b200
