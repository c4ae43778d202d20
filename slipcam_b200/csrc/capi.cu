// capi.cu -- the C ABI of include/slipcam_b200.h: the handle, parameter checks, device memory,
// the launch sequence and the host <-> device streaming.
//
// The reference's CUDA backend (slipcam cxx/cuda.cu:249-379) copies a group of frames, builds the
// tables, then runs six kernels and two cuFFT calls per batch of pairs, synchronously. Here a group
// of frames is three launches (summed-area tables in two passes, variance denominators) plus one
// fused correlation launch, and the host path double-buffers groups over two streams: while the
// device correlates group g, the copy stream brings group g + 1 in and the host stages group g + 2.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <thread>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>
#if defined(__SSE2__)
#include <emmintrin.h>
#endif

#include <cudaTypedefs.h>

#include "../../include/slipcam_b200.h"
#include "corr_fft.cuh"
#include "corr_big.cuh"
#include "corr_tc.cuh"
#include "corr_i8.cuh"
#include "refine.cuh"
#include "diff.h"
#include "multi.h"
#include "periodicity.cuh"
#include "scans.cuh"
#include "stabilize.h"
#include "sat.cuh"
#include "tc_selftest.cuh"

using namespace b200;

namespace {

constexpr int kThreads = 256;   // threads per correlation CTA
thread_local std::string g_create_error;

struct Failure {
    int code;
    std::string msg;
};

[[noreturn]] void fail(int code, const std::string &msg) { throw Failure{code, "framecor: " + msg}; }

void check(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) fail(B200_ERUNTIME, std::string(what) + ": " + cudaGetErrorString(e));
}
#define CK(call) check((call), #call)

// the FFT sizes with a compiled kernel: N = 16 N2 for the radices of dft.cuh
constexpr int kSizes[] = {16, 32, 48, 64, 80, 96, 128, 144, 160, 192, 256};
constexpr int kBigN = 256;   // the one size whose half spectrum is staged through global memory (corr_big.cuh)

int fft_size(int L)
{
    for (int n : kSizes)
        if (n >= L) return n;
    return 0;
}

// the failure injection of the tests: the n-th device or page-locked allocation from now fails as an
// out-of-memory would (0: none)
std::atomic<int> g_fail_alloc{0};

void injected_failure(const char *what)
{
    int n = g_fail_alloc.load();
    while (n > 0 && !g_fail_alloc.compare_exchange_weak(n, n - 1)) {
    }
    if (n == 1) fail(B200_ERUNTIME, std::string(what) + ": out of memory (injected)");
}

template <class T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    void alloc(size_t count)
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = count;
        injected_failure("cudaMalloc");
        CK(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)));
    }
    ~DevBuf()
    {
        if (p) cudaFree(p);
    }
};

template <class T>
struct HostBuf {
    T *p = nullptr;
    void alloc(size_t count)
    {
        if (p) cudaFreeHost(p);
        p = nullptr;
        injected_failure("cudaMallocHost");
        CK(cudaMallocHost(&p, std::max<size_t>(count, 1) * sizeof(T)));
    }
    ~HostBuf()
    {
        if (p) cudaFreeHost(p);
    }
};

// the per-group scratch of one slot
struct Slot {
    DevBuf<uint8_t> frames;
    DevBuf<uint32_t> sat;
    DevBuf<int64_t> sat2;
    DevBuf<float> dinv;
    DevBuf<int2> bstat;         // {box sum, dinv} beside dinv (the exact tensor-core form, the refinement)
    DevBuf<PeakInfo> peaks;     // the tensor-core kernel's peaks, for their exact refinement
    DevBuf<int> queue;          // the refinement's pairs whose SNR patch is summed exactly (count first)
    DevBuf<int32_t> gross;
    DevBuf<float> out;          // offset 2P | peak P | snr P | cov 3P, P = group * nwin
    HostBuf<uint8_t> hframes;
    HostBuf<int32_t> hgross;
    HostBuf<float> hout;
    cudaEvent_t in = nullptr, done = nullptr;
    ~Slot()
    {
        if (in) cudaEventDestroy(in);
        if (done) cudaEventDestroy(done);
    }
};

// A pool of host threads that split one large memcpy (pageable caller memory into the page-locked
// staging slots): one thread copies about 14 GB/s, eight about 40 GB/s. The caller takes a share
// too and returns when every share is done.
// n bytes src -> dst with streaming (non-temporal) stores where dst is 16-byte aligned: the
// page-locked staging buffer is read next by the DMA engine, not by this CPU, and streaming stores
// skip reading each destination line before writing it. Ends with a store fence, so the bytes are
// visible to the DMA once the copy is reported done.
inline void stream_copy(char *dst, const char *src, size_t n)
{
#if defined(__SSE2__)
    size_t i = 0;
    const size_t head = (16 - (reinterpret_cast<uintptr_t>(dst) & 15)) & 15;
    if (head) {
        const size_t m = std::min(head, n);
        std::memcpy(dst, src, m);
        i = m;
    }
    for (; i + 64 <= n; i += 64) {
        const __m128i a = _mm_loadu_si128(reinterpret_cast<const __m128i *>(src + i));
        const __m128i b = _mm_loadu_si128(reinterpret_cast<const __m128i *>(src + i + 16));
        const __m128i c = _mm_loadu_si128(reinterpret_cast<const __m128i *>(src + i + 32));
        const __m128i d = _mm_loadu_si128(reinterpret_cast<const __m128i *>(src + i + 48));
        _mm_stream_si128(reinterpret_cast<__m128i *>(dst + i), a);
        _mm_stream_si128(reinterpret_cast<__m128i *>(dst + i + 16), b);
        _mm_stream_si128(reinterpret_cast<__m128i *>(dst + i + 32), c);
        _mm_stream_si128(reinterpret_cast<__m128i *>(dst + i + 48), d);
    }
    if (i < n) std::memcpy(dst + i, src + i, n - i);
    _mm_sfence();
#else
    std::memcpy(dst, src, n);
#endif
}

class CopyPool {
  public:
    CopyPool()
    {
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        const int n = int(std::min(7u, hw > 1 ? hw - 1 : 0u));
        for (int i = 0; i < n; ++i) workers_.emplace_back([this, i] { run(i); });
    }
    ~CopyPool()
    {
        {
            std::lock_guard<std::mutex> lk(m_);
            stop_ = true;
        }
        cv_.notify_all();
        for (std::thread &t : workers_) t.join();
    }
    void copy(void *dst, const void *src, size_t bytes)
    {
        const int parts = int(workers_.size()) + 1;
        if (bytes < (size_t(1) << 20) || parts == 1) {
            stream_copy(static_cast<char *>(dst), static_cast<const char *>(src), bytes);
            return;
        }
        const size_t share = (bytes / parts + 4095) & ~size_t(4095);
        {
            std::lock_guard<std::mutex> lk(m_);
            dst_ = static_cast<char *>(dst);
            src_ = static_cast<const char *>(src);
            bytes_ = bytes;
            share_ = share;
            pending_ = int(workers_.size());
            ++gen_;
        }
        cv_.notify_all();
        const size_t o = size_t(parts - 1) * share;   // the caller's share: the last
        if (o < bytes) stream_copy(dst_ + o, src_ + o, bytes - o);
        std::unique_lock<std::mutex> lk(m_);
        done_.wait(lk, [this] { return pending_ == 0; });
    }

  private:
    void run(int i)
    {
        uint64_t seen = 0;
        for (;;) {
            std::unique_lock<std::mutex> lk(m_);
            cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
            if (stop_) return;
            seen = gen_;
            char *d = dst_;
            const char *sp = src_;
            const size_t o = size_t(i) * share_, n = o < bytes_ ? std::min(share_, bytes_ - o) : 0;
            lk.unlock();
            if (n) stream_copy(d + o, sp + o, n);
            lk.lock();
            if (--pending_ == 0) done_.notify_one();
        }
    }
    std::vector<std::thread> workers_;
    std::mutex m_;
    std::condition_variable cv_, done_;
    char *dst_ = nullptr;
    const char *src_ = nullptr;
    size_t bytes_ = 0, share_ = 0;
    int pending_ = 0;
    uint64_t gen_ = 0;
    bool stop_ = false;
};

// launch attributes set once per kernel instance
template <int N>
void prepare()
{
    static bool done[64] = {};
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && done[dev]) return;
    CK(cudaFuncSetAttribute(corr_kernel<N, kThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(Geo<N>::smem_bytes)));
    CK(cudaFuncSetAttribute(spectra_kernel<N, kThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(Geo<N>::smem_bytes)));
    if (dev >= 0 && dev < 64) done[dev] = true;
}

template <int N>
void launch_corr(const CorrArgs &a, cudaStream_t s)
{
    prepare<N>();
    corr_kernel<N, kThreads><<<unsigned(a.nwin) * a.nf, kThreads, Geo<N>::smem_bytes, s>>>(a);
}

// threads per pair of the latency-bound correlation (one frame of a chain at a time)
constexpr int kLatencyThreads = 512;

template <int N>
void launch_corr_latency(const CorrArgs &a, cudaStream_t s)
{
    static bool done[64] = {};
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && !done[dev]) {
        CK(cudaFuncSetAttribute(corr_latency_kernel<N, kLatencyThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                int(Geo<N>::smem_bytes)));
        done[dev] = true;
    }
    corr_latency_kernel<N, kLatencyThreads><<<unsigned(a.nwin) * a.nf, kLatencyThreads, Geo<N>::smem_bytes, s>>>(a);
}

int g_num_sms[64] = {};

int num_sms()
{
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return 148;
    if (!g_num_sms[dev]) CK(cudaDeviceGetAttribute(&g_num_sms[dev], cudaDevAttrMultiProcessorCount, dev));
    return g_num_sms[dev];
}

// the big transform: per-CTA scratch (complex values per CTA), persistent grids of one CTA per SM
size_t big_scratch_per_cta(int L, int M) { return BigGeo<kBigN>::scratch((L + 1) & ~1, M); }

void prepare_big()
{
    static bool done[64] = {};
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && done[dev]) return;
    const int smem = int(BigGeo<kBigN>::smem_bytes);
    CK(cudaFuncSetAttribute(corr_big_cluster_kernel<kBigN, kThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            int(BigClusterGeo<kBigN>::smem_bytes)));
    CK(cudaFuncSetAttribute(spectra_big_kernel<kBigN, kThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    if (dev >= 0 && dev < 64) done[dev] = true;
}

// the two-CTA clusters of the big transform that fit on the device at once (its persistent grid)
int big_clusters()
{
    static int cached[64] = {};
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && cached[dev]) return cached[dev];
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(unsigned(num_sms() / 2 * 2), 1, 1);
    cfg.blockDim = dim3(kThreads, 1, 1);
    cfg.dynamicSmemBytes = BigClusterGeo<kBigN>::smem_bytes;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, corr_big_cluster_kernel<kBigN, kThreads>, &cfg) != cudaSuccess || n < 1) {
        cudaGetLastError();
        n = num_sms() / 2;
    }
    if (dev >= 0 && dev < 64) cached[dev] = n;
    return n;
}

// the correlation of the big transform: two-CTA clusters holding the half spectrum in their
// shared memories (the per-CTA scratch serves the reference spectra only)
void launch_corr_big(const CorrArgs &a, float2 *, cudaStream_t s)
{
    prepare_big();
    const int clusters = std::min(a.nwin * a.nf, big_clusters());
    corr_big_cluster_kernel<kBigN, kThreads><<<unsigned(2 * clusters), kThreads, BigClusterGeo<kBigN>::smem_bytes, s>>>(a);
}

// cuTensorMapEncodeTiled, from the driver through the runtime (no link against libcuda)
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !p) fail(B200_ERUNTIME, "cuTensorMapEncodeTiled is not available");
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// the variance denominators of a group (nf frames of h x w floats) as a 3-D TMA tensor, box
// tc_box_width(M) x M x 1
CUtensorMap dinv_map(const float *dinv, int h, int w, int dpitch, int nf, int M)
{
    CUtensorMap m{};
    const cuuint64_t dims[3] = {cuuint64_t(w), cuuint64_t(h), cuuint64_t(nf)};
    const cuuint64_t strides[2] = {cuuint64_t(dpitch) * 4, cuuint64_t(dpitch) * h * 4};
    const cuuint32_t box[3] = {cuuint32_t(tc_box_width(M)), cuuint32_t(M), 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = tensor_map_encoder()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(dinv), dims, strides,
                                            box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) fail(B200_ERUNTIME, "cuTensorMapEncodeTiled failed (" + std::to_string(int(r)) + ")");
    return m;
}

template <int N>
void launch_corr_tc(const CorrArgs &a, const uint4 *dtab, int *status, const CUtensorMap *dmap, cudaStream_t s)
{
    static bool done[64] = {};
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && !done[dev]) {
        CK(cudaFuncSetAttribute(corr_tc_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(TcGeo<N>::smem_bytes)));
        done[dev] = true;
    }
    const int pairs = a.nwin * a.nf;
    const int grid = std::min(pairs, num_sms());
    corr_tc_kernel<N><<<unsigned(grid), kTcThreads, TcGeo<N>::smem_bytes, s>>>(a, dtab, status, dmap);
}

// the exact tensor-core form: one persistent CTA per SM over the groups of F frames of a window
void launch_corr_i8(const CorrArgs &a, const uint8_t *refwin, const int *sref, int *status, const I8Geo &g, cudaStream_t s)
{
    static bool done[64] = {};
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && !done[dev]) {
        CK(cudaFuncSetAttribute(corr_i8_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kI8MaxSmem)));
        CK(cudaFuncSetAttribute(corr_i8_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kI8MaxSmem)));
        done[dev] = true;
    }
    if (!a.bstat || !refwin || !sref) fail(B200_EINVAL, "the exact tensor-core form has no box table or reference windows");
    const int groups = a.nwin * ((a.nf + g.F - 1) / g.F);
    const int grid = std::min(groups, num_sms());
    const I8Args x{a, a.bstat, refwin, sref, status, g};
    if (a.surface)
        corr_i8_kernel<true><<<unsigned(grid), kI8Threads, g.smem, s>>>(x);
    else
        corr_i8_kernel<false><<<unsigned(grid), kI8Threads, g.smem, s>>>(x);
}

template <int N>
bool tc_fits_n(int M)
{
    // the box of variance denominators (X region), and the S5 result in the top NO TMEM columns
    // clear of every other stage's accumulators
    using G = TcGeo<N>;
    const int NO = (M + 15) / 16 * 16;
    const int used = std::max({2 * G::KP * G::T1, 2 * N, 2 * NO});
    return size_t(tc_box_width(M)) * M * 4 <= G::X_BYTES && used + NO <= int(G::TMEM_COLS);
}

// whether the tensor-core kernel holds this geometry: FFT size up to 160, up to 128 shifts per axis
bool tc_fits(int N, int M)
{
    if (M > 128) return false;
    switch (N) {
    case 16: return tc_fits_n<16>(M);
    case 32: return tc_fits_n<32>(M);
    case 48: return tc_fits_n<48>(M);
    case 64: return tc_fits_n<64>(M);
    case 80: return tc_fits_n<80>(M);
    case 96: return tc_fits_n<96>(M);
    case 128: return tc_fits_n<128>(M);
    case 144: return tc_fits_n<144>(M);
    case 160: return tc_fits_n<160>(M);
    default: return false;
    }
}

#define B200_DISPATCH_TC(N_, F, ...)                                                               \
    switch (N_) {                                                                                   \
    case 16: F<16>(__VA_ARGS__); break;                                                             \
    case 32: F<32>(__VA_ARGS__); break;                                                             \
    case 48: F<48>(__VA_ARGS__); break;                                                             \
    case 64: F<64>(__VA_ARGS__); break;                                                             \
    case 80: F<80>(__VA_ARGS__); break;                                                             \
    case 96: F<96>(__VA_ARGS__); break;                                                             \
    case 128: F<128>(__VA_ARGS__); break;                                                           \
    case 144: F<144>(__VA_ARGS__); break;                                                           \
    case 160: F<160>(__VA_ARGS__); break;                                                           \
    default: fail(B200_EINVAL, "no tensor-core kernel for the FFT size " + std::to_string(N_));    \
    }

template <int N>
void launch_spectra(const SpectraArgs &a, int nwin, cudaStream_t s)
{
    prepare<N>();
    spectra_kernel<N, kThreads><<<unsigned(nwin), kThreads, Geo<N>::smem_bytes, s>>>(a);
}

#define B200_DISPATCH(N_, F, ...)                                                                  \
    switch (N_) {                                                                                   \
    case 16: F<16>(__VA_ARGS__); break;                                                             \
    case 32: F<32>(__VA_ARGS__); break;                                                             \
    case 48: F<48>(__VA_ARGS__); break;                                                             \
    case 64: F<64>(__VA_ARGS__); break;                                                             \
    case 80: F<80>(__VA_ARGS__); break;                                                             \
    case 96: F<96>(__VA_ARGS__); break;                                                             \
    case 128: F<128>(__VA_ARGS__); break;                                                           \
    case 144: F<144>(__VA_ARGS__); break;                                                           \
    case 160: F<160>(__VA_ARGS__); break;                                                           \
    case 192: F<192>(__VA_ARGS__); break;                                                           \
    default: fail(B200_EINVAL, "no kernel for the FFT size " + std::to_string(N_));               \
    }

void launch_sat(const uint8_t *frames, int64_t fstride, int pitch, int nf, int h, int w, uint32_t *sat,
                int64_t *sat2, cudaStream_t s)
{
    const int64_t sfs = int64_t(h + 1) * (w + 1);
    sat_rows_kernel<<<dim3(unsigned((h + 7) / 8), unsigned(nf)), 256, 0, s>>>(frames, fstride, pitch, h, w, sat, sat2, sfs);
    sat_cols_kernel<<<dim3(unsigned((w + 1 + 31) / 32), unsigned(nf)), dim3(32, 8), 0, s>>>(h, w, sat, sat2, sfs);
}

}   // namespace

struct b200_handle {
    int height = 0, width = 0, W = 0, R = 0, stat = 21, batch = 4096;
    std::vector<int> down, across;
    int ny = 0, nx = 0, nwin = 0, L = 0, M = 0, N = 0;
    int device = 0;
    int group = 1;
    int form = B200_FORM_FFT32;
    bool ready = false;
    bool ref_u8 = false;         // the reference is a uint8 frame (the exact form's windows are set)
    uint64_t launches = 0;
    std::string err;
    cudaStream_t comp = nullptr, copy = nullptr;
    DevBuf<int> d_down, d_across;
    DevBuf<float> d_norm;
    DevBuf<float2> d_spec, d_tw;
    DevBuf<float4> d_spec_tc;    // the reference spectra in the tensor-core form's order
    DevBuf<float2> d_big;        // the big transform's per-CTA scratch (N = 256 only)
    DevBuf<uint8_t> d_ref;
    DevBuf<uint8_t> d_refwin;    // the exact tensor-core form: the reference windows' pixels, nwin x W x W
    DevBuf<int> d_sref;          // and their sums
    DevBuf<int2> d_bstat;        // device-path box table (beside d_dinv)
    DevBuf<PeakInfo> d_peaks;    // device-path peaks of the tensor-core form
    DevBuf<int> d_queue;         // and the refinement's queue
    DevBuf<uint32_t> d_sat;      // device-path scratch
    DevBuf<int64_t> d_sat2;
    DevBuf<float> d_dinv;
    Slot slot[2];
    bool slots_ready = false;    // the slots are allocated (ensure_slots)
    DevBuf<uint32_t> d_csat;     // coarse tracking: two sets of tables of kCoarseGroup frames
    DevBuf<int64_t> d_csat2;
    DevBuf<float> d_cdinv;
    DevBuf<uint16_t> d_dtab;     // the FP16 DFT matrices of the tensor-core form
    DevBuf<int> d_status;        // device status word (3: a tensor-core wait gave up)
    DevBuf<CUtensorMap> d_tmaps; // TMA maps of the three denominator tables: slot 0, slot 1, device path
    DevBuf<float> d_coarse;      // coarse tracking: one frame's surfaces and four outputs
    DevBuf<double> d_cpeaks;     // coarse tracking: one frame's peaks
    cudaEvent_t coarse_ev[6] = {};  // coarse tracking: tables ready (2), tables consumed (2), call start, end
    std::vector<cudaEvent_t> part_ev;   // host path: a part of a group's frames is on the device
    bool coarse_l2 = false;      // the persisting L2 carve-out for the reference spectra is set up
    cudaAccessPolicyWindow l2win{};   // the window coarse tracking puts on the handle's stream per call
    size_t l2_limit_prev = 0;    // the device's persisting L2 limit before this handle raised it
    bool l2_raised = false;
    bool tc_ok = false;          // the geometry fits the tensor-core kernel
    bool i8_ok = false;          // the geometry fits the exact tensor-core kernel
    I8Geo i8g{};                 // its layout
    int fpitch = 0;              // the pitch of the staged frames (a multiple of 16)
    bool profiling = false;      // events around the correlation launches
    std::unique_ptr<CopyPool> pool;   // host threads for staging pageable frames (made on first use)
    struct Timed {
        cudaEvent_t a, b;
        uint64_t pairs;
    };
    std::vector<Timed> timed;

    ~b200_handle()
    {
        for (Timed &t : timed) {
            cudaEventDestroy(t.a);
            cudaEventDestroy(t.b);
        }
        for (cudaEvent_t e : coarse_ev)
            if (e) cudaEventDestroy(e);
        for (cudaEvent_t e : part_ev)
            if (e) cudaEventDestroy(e);
        if (l2_raised) cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, l2_limit_prev);   // as it was
        if (comp) cudaStreamDestroy(comp);
        if (copy) cudaStreamDestroy(copy);
    }

    int64_t sat_size() const { return int64_t(height + 1) * (width + 1); }
    int64_t pixels() const { return int64_t(height) * width; }
    int dpitch() const { return (width + 3) & ~3; }                  // rows of 16-byte multiples
    int64_t dinv_size() const { return int64_t(height) * dpitch(); }

    // the host path's two slots (device and page-locked host buffers, events, the TMA maps of their
    // tables), allocated by the first host-path call: device-path callers never pay for them
    void ensure_slots()
    {
        if (slots_ready) return;
        const size_t G = size_t(group), P = G * nwin;
        for (Slot &s : slot) {
            s.frames.alloc(G * height * fpitch);
            s.sat.alloc(G * sat_size());
            s.sat2.alloc(G * sat_size());
            s.dinv.alloc(G * dinv_size());
            s.gross.alloc(2 * P);
            s.out.alloc(7 * P);
            s.hframes.alloc(G * height * fpitch);
            s.hgross.alloc(2 * P);
            s.hout.alloc(7 * P);
            if (!s.in) CK(cudaEventCreateWithFlags(&s.in, cudaEventDisableTiming));
            if (!s.done) CK(cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming));
        }
        if (tc_ok) {
            const CUtensorMap maps[2] = {dinv_map(slot[0].dinv.p, height, width, dpitch(), int(G), M),
                                         dinv_map(slot[1].dinv.p, height, width, dpitch(), int(G), M)};
            CK(cudaMemcpy(d_tmaps.p, maps, sizeof(maps), cudaMemcpyHostToDevice));
        }
        slots_ready = true;
    }

    // the device path's tables for `group` frames (and the TMA map of its denominators), allocated
    // by the first device-path call: coarse tracking and the host path never pay for them
    void ensure_tables()
    {
        if (!d_sat.p) {
            const size_t G = size_t(group);
            d_sat.alloc(G * sat_size());
            d_sat2.alloc(G * sat_size());
            d_dinv.alloc(G * dinv_size());
            if (tc_ok) {
                const CUtensorMap m = dinv_map(d_dinv.p, height, width, dpitch(), int(G), M);
                CK(cudaMemcpy(d_tmaps.p + 2, &m, sizeof(m), cudaMemcpyHostToDevice));
            }
        }
        ensure_exact(d_bstat, d_peaks, d_queue);
    }

    // the exact forms' per-launch buffers, allocated when a form that reads them first runs: the box
    // table (the exact form, and the exact refinement of the tensor-core form) and the tensor-core
    // form's peak records and refinement queue (a handle kept on the FP32 form never holds them)
    void ensure_exact(DevBuf<int2> &bstat, DevBuf<PeakInfo> &peaks, DevBuf<int> &queue)
    {
        if (form != B200_FORM_I8 && form != B200_FORM_TC) return;
        const size_t G = size_t(group), P = G * nwin;
        if (i8_ok && !bstat.p) bstat.alloc(G * dinv_size());
        if (i8_ok && tc_ok && !peaks.p) {
            peaks.alloc(P);
            CK(cudaMemset(peaks.p, 0, P * sizeof(PeakInfo)));
            queue.alloc(P + 1);
        }
    }

    // the tables and the correlation of nf frames (device memory) on stream s; bstat (the box table
    // beside dinv) serves the exact tensor-core form
    void run_group(const uint8_t *frames, int pitch, int nf, const int32_t *gross, int gross_mode,
                   uint32_t *sat, int64_t *sat2, float *dinv, int2 *bstat, PeakInfo *peaks, int *queue, float *offset,
                   float *peak, float *snr, float *cov, float *surface, cudaStream_t s, bool tables_done = false)
    {
        const int arith = group_arith(bstat);
        // the tensor-core form's peaks are refined exactly where the reference windows are at hand
        const bool refine = arith == B200_FORM_TC && peaks && queue && bstat && ref_u8;
        if (!tables_done) run_tables(frames, pitch, nf, sat, sat2, dinv, s, wants_bstat(bstat, peaks, queue) ? bstat : nullptr);
        CorrArgs a = corr_args(frames, pitch, nf, gross, gross_mode, sat, dinv, offset, peak, snr, cov, surface);
        a.bstat = bstat;
        a.peaks = refine ? peaks : nullptr;
        run_corr_tail(a, nf, dinv, arith, s);
        if (refine) {
            CK(cudaMemsetAsync(queue, 0, sizeof(int), s));
            static bool attr[64] = {};
            int dev = 0;
            CK(cudaGetDevice(&dev));
            if (dev >= 0 && dev < 64 && !attr[dev]) {
                CK(cudaFuncSetAttribute(tc_patch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
                CK(cudaFuncSetAttribute(tc_refine_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024));
                attr[dev] = true;
            }
            // one warp per pair, a CTA per window and up to 8 of its frames (the window staged once),
            // as many as 100 KB of shared memory holds (at window 64: 8 warps, 55 KB, 4 CTAs an SM)
            const size_t rsm = refine_ref_smem(W), tsm = refine_tile_smem(W);
            const int wpc = int(std::clamp<size_t>(std::min<size_t>(size_t(nf), (size_t(100 * 1024) - rsm) / tsm), 1, 8));
            const int cpw = (nf + wpc - 1) / wpc;
            tc_refine_kernel<<<unsigned(int64_t(nwin) * cpw), 32 * wpc, rsm + size_t(wpc) * tsm, s>>>(a, d_refwin.p, d_sref.p,
                                                                                                     queue);
            const size_t psm = tc_patch_smem(W, M, stat);
            tc_patch_kernel<<<unsigned(2 * num_sms()), 256, psm, s>>>(a, d_refwin.p, d_sref.p, queue);
            CK(cudaGetLastError());
            launches += 2;
        }
        launches += 3;
    }

    // the arithmetic of a launch group: the exact form needs the box table
    int group_arith(const int2 *bstat) const
    {
        return form != B200_FORM_I8 ? form : (bstat && ref_u8) ? B200_FORM_I8 : B200_FORM_FFT32;
    }
    // the box table is read by the exact form and by the exact refinement of the tensor-core form
    bool wants_bstat(const int2 *bstat, const PeakInfo *peaks, const int *queue) const
    {
        const int arith = group_arith(bstat);
        return arith == B200_FORM_I8 || (arith == B200_FORM_TC && peaks && queue && bstat && ref_u8);
    }

    // the summed-area tables and the variance denominators of nf frames (and the box table)
    void run_tables(const uint8_t *frames, int pitch, int nf, uint32_t *sat, int64_t *sat2, float *dinv, cudaStream_t s,
                    int2 *bstat = nullptr)
    {
        const int64_t fstride = int64_t(pitch) * height;
        launch_sat(frames, fstride, pitch, nf, height, width, sat, sat2, s);
        dinv_kernel<<<dim3(unsigned((width - W + 1 + 127) / 128), unsigned(height - W + 1), unsigned(nf)), 128, 0, s>>>(
            sat, sat2, sat_size(), height, width, W, dinv, dinv_size(), dpitch(), bstat);
    }

    // the correlation of nf frames with their tables at sat / dinv, in the form `arith`
    void run_corr(const uint8_t *frames, int pitch, int nf, const int32_t *gross, int gross_mode, const uint32_t *sat,
                  const float *dinv, float *offset, float *peak, float *snr, float *cov, float *surface, int arith,
                  cudaStream_t s)
    {
        const CorrArgs a = corr_args(frames, pitch, nf, gross, gross_mode, sat, dinv, offset, peak, snr, cov, surface);
        run_corr_tail(a, nf, dinv, arith, s);
    }

    // the arguments of the correlation kernels for nf frames with their tables at sat / dinv
    CorrArgs corr_args(const uint8_t *frames, int pitch, int nf, const int32_t *gross, int gross_mode,
                       const uint32_t *sat, const float *dinv, float *offset, float *peak, float *snr, float *cov,
                       float *surface) const
    {
        CorrArgs a{};
        a.frames = frames;
        a.fstride = int64_t(pitch) * height;
        a.pitch = pitch;
        a.sat = sat;
        a.sat_fstride = sat_size();
        a.dinv = dinv;
        a.dinv_fstride = dinv_size();
        a.dpitch = dpitch();
        a.h = height;
        a.w = width;
        a.W = W;
        a.R = R;
        a.L = L;
        a.M = M;
        a.nx = nx;
        a.nwin = nwin;
        a.nf = nf;
        a.stat = stat;
        a.down = d_down.p;
        a.across = d_across.p;
        a.norm = d_norm.p;
        a.spec = d_spec.p;
        a.spec_tc = d_spec_tc.p;
        a.twiddles = d_tw.p;
        a.gross = gross;
        a.gross_mode = gross_mode;
        a.offset = offset;
        a.peak = peak;
        a.snr = snr;
        a.cov = cov;
        a.surface = surface;
        return a;
    }

    // the launch of run_corr (and its profiling events)
    void run_corr_tail(const CorrArgs &a, int nf, const float *dinv, int arith, cudaStream_t s)
    {
        Timed t{};
        if (profiling) {
            CK(cudaEventCreate(&t.a));
            CK(cudaEventCreate(&t.b));
            t.pairs = uint64_t(nf) * nwin;
            CK(cudaEventRecord(t.a, s));
        }
        if (arith == B200_FORM_I8) {
            launch_corr_i8(a, d_refwin.p, d_sref.p, d_status.p, i8g, s);
        } else if (arith == B200_FORM_TC) {
            const uint4 *dt = reinterpret_cast<const uint4 *>(d_dtab.p);
            const int mi = dinv == slot[0].dinv.p ? 0 : dinv == slot[1].dinv.p ? 1 : 2;
            if (mi == 2 && dinv != d_dinv.p) fail(B200_EINVAL, "no TMA map for this denominator table");
            const CUtensorMap *dm = d_tmaps.p + mi;
            B200_DISPATCH_TC(N, launch_corr_tc, a, dt, d_status.p, dm, s);
        } else if (N == kBigN) {
            launch_corr_big(a, d_big.p, s);
        } else if (N == 192) {
            // one 154 KB tile per SM: 512 threads per pair keep 16 warps resident instead of 8
            launch_corr_latency<192>(a, s);
        } else {
            B200_DISPATCH(N, launch_corr, a, s);
        }
        CK(cudaGetLastError());
        if (profiling) {
            CK(cudaEventRecord(t.b, s));
            timed.push_back(t);
        }
        launches += 1;
    }
};

namespace {

// the twiddle tables of the N-point transform: TW[k1 * N2 + n2] = TWI[n2 * 16 + k1] = w_N^{n2 k1}
std::vector<float2> twiddles(int N)
{
    const int N2 = N / 16;
    std::vector<float2> t(2 * size_t(N));
    for (int k1 = 0; k1 < 16; ++k1)
        for (int n2 = 0; n2 < N2; ++n2) {
            double c = 0.0, s = 0.0;
            cs2pi(long(n2) * k1, N, c, s);
            const float2 w = make_float2(float(c), float(-s));
            t[k1 * N2 + n2] = w;
            t[N + n2 * 16 + k1] = w;
        }
    return t;
}

// checkParams (cxx/common.cpp:15-28), the same conditions and messages
void check_params(const b200_params *p)
{
    if (!p) fail(B200_EINVAL, "no parameters");
    if (p->height <= 0 || p->width <= 0) fail(B200_EINVAL, "the frame size must be positive");
    if (p->window < 3) fail(B200_EINVAL, "the window must be at least 3 pixels");
    if (p->search < 1) fail(B200_EINVAL, "the half search range must be at least 1 pixel");
    if (p->ny <= 0 || p->nx <= 0 || !p->down || !p->across) fail(B200_EINVAL, "no windows");
    for (int i = 0; i < p->ny; ++i)
        if (p->down[i] < 0 || p->down[i] + p->window > p->height)
            fail(B200_EINVAL, "a window is outside the frame (down " + std::to_string(p->down[i]) + ")");
    for (int i = 0; i < p->nx; ++i)
        if (p->across[i] < 0 || p->across[i] + p->window > p->width)
            fail(B200_EINVAL, "a window is outside the frame (across " + std::to_string(p->across[i]) + ")");
    if (p->stat_size < 3) fail(B200_EINVAL, "the SNR window must be at least 3 pixels");
    if (p->batch < 1) fail(B200_EINVAL, "the batch must be at least 1 window");
}

template <class F>
int guarded(b200_handle *h, F &&f)
{
    if (!h) return B200_EINVAL;
    try {
        f();
        h->err.clear();
        return B200_OK;
    } catch (const Failure &e) {
        h->err = e.msg;
        return e.code;
    } catch (const std::bad_alloc &) {
        h->err = "framecor: out of host memory";
        return B200_ERUNTIME;
    } catch (const std::invalid_argument &e) {
        h->err = std::string("framecor: ") + e.what();
        return B200_EINVAL;
    } catch (const std::exception &e) {
        h->err = std::string("framecor: ") + e.what();
        return B200_ERUNTIME;
    }
}

void upload_reference(b200_handle *h, const uint8_t *dframe, int pitch, cudaStream_t s, const float *dframef = nullptr)
{
    SpectraArgs a{};
    a.frame = dframe;
    a.framef = dframef;
    a.pitch = pitch;
    a.W = h->W;
    a.nx = h->nx;
    a.down = h->d_down.p;
    a.across = h->d_across.p;
    a.norm = h->d_norm.p;
    a.spec = h->d_spec.p;
    a.twiddles = h->d_tw.p;
    if (h->N == kBigN) {
        prepare_big();
        const int grid = std::min(h->nwin, num_sms());
        spectra_big_kernel<kBigN, kThreads><<<unsigned(grid), kThreads, BigGeo<kBigN>::smem_bytes, s>>>(
            a, h->nwin, h->d_big.p, big_scratch_per_cta(h->L, h->M));
    } else {
        B200_DISPATCH(h->N, launch_spectra, a, h->nwin, s);
    }
    CK(cudaGetLastError());
    h->launches += 1;
    if (h->tc_ok) {
        spec_tc_kernel<<<unsigned(4 * num_sms()), 256, 0, s>>>(h->d_spec.p, h->d_spec_tc.p, h->N, h->nwin);
        CK(cudaGetLastError());
        h->launches += 1;
    }
    h->ref_u8 = !dframef;
    if (h->i8_ok && !dframef) {
        refwin_kernel<<<unsigned(h->nwin), 128, 0, s>>>(dframe, pitch, h->W, h->nx, h->d_down.p, h->d_across.p,
                                                          h->d_refwin.p, h->d_sref.p);
        CK(cudaGetLastError());
        h->launches += 1;
    }
}

// the differentiable path's arguments for n frames (diff.h)
DiffArgs diff_args(b200_handle *h, const float *frames, int n, int pitch, const int32_t *gross, int gross_mode,
                   const float *shift)
{
    if (!h->ready) fail(B200_ERUNTIME, "set_reference first");
    if (n < 0) fail(B200_EINVAL, "the number of frames must not be negative");
    if (n && (!frames || pitch < h->width)) fail(B200_EINVAL, "no frames, or their pitch is below their width");
    if (gross_mode < B200_GROSS_NONE || gross_mode > B200_GROSS_WINDOW || (gross_mode && !gross))
        fail(B200_EINVAL, "gross must be frames x 2 or frames x down x across x 2");
    DiffArgs a{};
    a.frames = frames;
    a.pitch = pitch;
    a.fstride = int64_t(pitch) * h->height;
    a.h = h->height;
    a.w = h->width;
    a.W = h->W;
    a.R = h->R;
    a.L = h->L;
    a.M = h->M;
    a.nx = h->nx;
    a.nwin = h->nwin;
    a.n = n;
    a.stat = h->stat;
    a.down = h->d_down.p;
    a.across = h->d_across.p;
    a.norm = h->d_norm.p;
    a.spec = h->d_spec.p;
    a.twiddles = h->d_tw.p;
    a.gross = gross;
    a.gross_mode = gross_mode;
    a.shift = shift;
    return a;
}

}   // namespace

void b200::tc_dft_table(int N, uint16_t *out)
{
    const uint32_t sbo = uint32_t(N / 8) * 128u, bytes = uint32_t(N / 8) * sbo;
    for (int part = 0; part < 2; ++part)
        for (int r = 0; r < N; ++r)
            for (int c = 0; c < N; ++c) {
                double cc = 0.0, sn = 0.0;
                cs2pi(long(r) * c, N, cc, sn);
                const __half hv = __float2half_rn(float(part == 0 ? cc : -sn));
                const uint32_t off = part * bytes + tc::k_major_offset(r, c, sbo, 128);
                out[off / 2] = __half_as_ushort(hv);
            }
}

extern "C" {

// the library's choice: the tensor-core form (its peaks refined exactly) where it holds the geometry
// and is the faster -- windows above 32 px -- else the FP32 form
static int auto_form(const b200_handle *h)
{
    return h->tc_ok && h->i8_ok && h->W > 32 ? B200_FORM_TC : B200_FORM_FFT32;
}

int b200_create(const b200_params *p, int device, b200_handle **out)
{
    if (out) *out = nullptr;
    b200_handle *h = nullptr;
    try {
        if (!out) fail(B200_EINVAL, "no output handle");
        check_params(p);
        const int L = p->window + 2 * p->search;
        const int N = fft_size(L);
        if (!N)
            fail(B200_EINVAL, "the search window (window + 2 search = " + std::to_string(L)
                                  + ") is larger than the b200 backend's largest transform, 256");
        if (N == kBigN && !BigGeo<kBigN>::fits_M(2 * p->search + 1))
            fail(B200_EINVAL, "with a search window of " + std::to_string(L)
                                  + " pixels the b200 backend holds searches up to 64 pixels");
        h = new b200_handle;
        h->height = p->height;
        h->width = p->width;
        h->W = p->window;
        h->R = p->search;
        h->stat = p->stat_size;
        h->batch = p->batch;
        h->down.assign(p->down, p->down + p->ny);
        h->across.assign(p->across, p->across + p->nx);
        h->ny = p->ny;
        h->nx = p->nx;
        h->nwin = p->ny * p->nx;
        h->L = L;
        h->M = 2 * p->search + 1;
        h->N = N;
        h->device = device;
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || count <= device || device < 0)
            fail(B200_ERUNTIME, "no CUDA device " + std::to_string(device));
        CK(cudaSetDevice(device));
        CK(cudaStreamCreateWithFlags(&h->comp, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&h->copy, cudaStreamNonBlocking));
        // frames per launch: enough pairs to fill the GPU many times over, at most 32 frames
        h->group = std::clamp((40000 + h->nwin - 1) / h->nwin, 1, 32);
        h->fpitch = (h->width + 15) & ~15;
        h->d_down.alloc(h->ny);
        h->d_across.alloc(h->nx);
        CK(cudaMemcpy(h->d_down.p, h->down.data(), h->ny * sizeof(int), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(h->d_across.p, h->across.data(), h->nx * sizeof(int), cudaMemcpyHostToDevice));
        h->d_norm.alloc(h->nwin);
        h->d_spec.alloc(size_t(h->nwin) * (N / 2 + 1) * N);
        const std::vector<float2> tw = twiddles(N);
        h->d_tw.alloc(tw.size());
        CK(cudaMemcpy(h->d_tw.p, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice));
        h->d_ref.alloc(size_t(h->height) * h->fpitch);
        h->d_status.alloc(1);
        CK(cudaMemset(h->d_status.p, 0, sizeof(int)));
        h->tc_ok = tc_fits(N, h->M);
        if (h->tc_ok) {
            std::vector<uint16_t> dt(2 * size_t(N) * N);
            tc_dft_table(N, dt.data());
            h->d_dtab.alloc(dt.size());
            h->d_spec_tc.alloc(size_t(h->nwin) * (N / 2) * tc_kp(N));
            CK(cudaMemcpy(h->d_dtab.p, dt.data(), dt.size() * sizeof(uint16_t), cudaMemcpyHostToDevice));
        }
        if (N == kBigN) h->d_big.alloc(size_t(num_sms()) * big_scratch_per_cta(L, h->M));
        h->i8_ok = i8_plan(h->W, h->R, h->i8g);
        if (h->i8_ok) {
            h->d_refwin.alloc(size_t(h->nwin) * h->W * h->W);
            h->d_sref.alloc(h->nwin);
        }
        // the maps of the two slots and of the device path's table are written when those are allocated
        if (h->tc_ok) h->d_tmaps.alloc(3);
        h->form = auto_form(h);
        *out = h;
        g_create_error.clear();
        return B200_OK;
    } catch (const Failure &e) {
        delete h;
        g_create_error = e.msg;
        return e.code;
    } catch (const std::bad_alloc &) {
        delete h;
        g_create_error = "framecor: out of host memory";
        return B200_ERUNTIME;
    }
}

int b200_destroy(b200_handle *h)
{
    if (!h) return B200_OK;
    cudaSetDevice(h->device);
    if (h->comp) cudaStreamSynchronize(h->comp);
    if (h->copy) cudaStreamSynchronize(h->copy);
    delete h;
    return B200_OK;
}

const char *b200_last_error(const b200_handle *h) { return h ? h->err.c_str() : g_create_error.c_str(); }

int b200_set_form(b200_handle *h, int form)
{
    return guarded(h, [&] {
        if (form != B200_FORM_AUTO && form != B200_FORM_FFT32 && form != B200_FORM_TC && form != B200_FORM_I8)
            fail(B200_EINVAL, "unknown form " + std::to_string(form));
        if (form == B200_FORM_TC && !h->tc_ok)
            fail(B200_EINVAL, "the tensor-core form holds FFT sizes up to 160 and search ranges up to 63 px, not "
                                  + std::to_string(h->N) + " and " + std::to_string(h->R));
        if (form == B200_FORM_I8 && !h->i8_ok)
            fail(B200_EINVAL, "the exact tensor-core form holds windows up to " + std::to_string(kI8MaxWindow)
                                  + " px and search windows up to 256 px, not " + std::to_string(h->W) + " and "
                                  + std::to_string(h->L));
        h->form = form == B200_FORM_AUTO ? auto_form(h) : form;
    });
}

int b200_set_reference(b200_handle *h, const uint8_t *frame)
{
    return guarded(h, [&] {
        if (!frame) fail(B200_EINVAL, "no reference frame");
        CK(cudaSetDevice(h->device));
        CK(cudaMemcpy2DAsync(h->d_ref.p, h->fpitch, frame, h->width, h->width, h->height, cudaMemcpyHostToDevice, h->comp));
        upload_reference(h, h->d_ref.p, h->fpitch, h->comp);
        CK(cudaStreamSynchronize(h->comp));
        h->ready = true;
    });
}

int b200_set_reference_device(b200_handle *h, const uint8_t *frame, int pitch, void *stream)
{
    return guarded(h, [&] {
        if (!frame || pitch < h->width) fail(B200_EINVAL, "no reference frame, or its pitch is below its width");
        CK(cudaSetDevice(h->device));
        upload_reference(h, frame, pitch, static_cast<cudaStream_t>(stream));
        h->ready = true;
    });
}

int b200_correlate(b200_handle *h, const uint8_t *frames, int n, const int32_t *gross, int gross_mode,
                   float *offset, float *peak, float *snr, float *cov)
{
    return guarded(h, [&] {
        if (!h->ready) fail(B200_ERUNTIME, "set_reference first");
        if (n < 0) fail(B200_EINVAL, "the number of frames must not be negative");
        if (gross_mode < B200_GROSS_NONE || gross_mode > B200_GROSS_WINDOW || (gross_mode && !gross))
            fail(B200_EINVAL, "gross must be frames x 2 or frames x down x across x 2");
        if (n == 0) return;
        if (!frames || !offset || !peak || !snr || !cov) fail(B200_EINVAL, "null input or output");
        CK(cudaSetDevice(h->device));
        h->ensure_slots();
        for (Slot &sl : h->slot) h->ensure_exact(sl.bstat, sl.peaks, sl.queue);
        CK(cudaMemset(h->d_status.p, 0, sizeof(int)));   // a flag left by an earlier call is not this one's
        const int G = h->group, nwin = h->nwin;
        const size_t frame_bytes = size_t(h->height) * h->width;
        const int ngroups = (n + G - 1) / G;
        // frames in page-locked memory are copied to the device directly, others staged
        cudaPointerAttributes attr{};
        const bool pinned = cudaPointerGetAttributes(&attr, frames) == cudaSuccess && attr.type == cudaMemoryTypeHost;
        cudaGetLastError();
        auto drain = [&](int g) {   // the outputs of group g to the caller's arrays
            Slot &s = h->slot[g % 2];
            CK(cudaEventSynchronize(s.done));
            const int f0 = g * G, nf = std::min(G, n - f0);
            const size_t P = size_t(nf) * nwin, PG = size_t(G) * nwin, q0 = size_t(f0) * nwin;
            std::memcpy(offset + 2 * q0, s.hout.p, 2 * P * sizeof(float));
            std::memcpy(peak + q0, s.hout.p + 2 * PG, P * sizeof(float));
            std::memcpy(snr + q0, s.hout.p + 3 * PG, P * sizeof(float));
            std::memcpy(cov + 3 * q0, s.hout.p + 4 * PG, 3 * P * sizeof(float));
        };
        for (int g = 0; g < ngroups; ++g) {
            Slot &s = h->slot[g % 2];
            if (g >= 2) drain(g - 2);   // also: group g - 2 no longer needs this slot's buffers
            const int f0 = g * G, nf = std::min(G, n - f0);
            const size_t P = size_t(nf) * nwin, PG = size_t(G) * nwin;
            const uint8_t *src = frames + f0 * frame_bytes;
            const int32_t *dg = nullptr;
            size_t gbytes = 0;
            if (gross_mode == B200_GROSS_FRAME) {
                gbytes = size_t(nf) * 2 * sizeof(int32_t);
                std::memcpy(s.hgross.p, gross + 2 * size_t(f0), gbytes);
            } else if (gross_mode == B200_GROSS_WINDOW) {
                gbytes = P * 2 * sizeof(int32_t);
                std::memcpy(s.hgross.p, gross + 2 * size_t(f0) * nwin, gbytes);
            }
            // the frames in parts of four: each part's tables run on the compute stream as soon as the
            // part is on the device, under the next part's copy (and, for pageable frames, under the
            // pool's staging of the next part into the page-locked slot)
            int2 *bst = h->wants_bstat(s.bstat.p, s.peaks.p, s.queue.p) ? s.bstat.p : nullptr;
            if (!pinned && !h->pool) h->pool.reset(new CopyPool());
            for (int c0 = 0, part = 0; c0 < nf; c0 += 4, ++part) {
                const int cn = std::min(4, nf - c0);
                const uint8_t *from = src + size_t(c0) * frame_bytes;
                if (!pinned) {   // staged into the page-locked slot (the previous part's DMA runs meanwhile)
                    uint8_t *stage = s.hframes.p + size_t(c0) * frame_bytes;
                    h->pool->copy(stage, from, size_t(cn) * frame_bytes);
                    from = stage;
                }
                uint8_t *dst = s.frames.p + size_t(c0) * h->height * h->fpitch;
                CK(cudaMemcpy2DAsync(dst, h->fpitch, from, h->width, h->width, size_t(cn) * h->height,
                                     cudaMemcpyHostToDevice, h->copy));
                if (int(h->part_ev.size()) <= part) {
                    cudaEvent_t e = nullptr;
                    CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
                    h->part_ev.push_back(e);
                }
                CK(cudaEventRecord(h->part_ev[part], h->copy));
                CK(cudaStreamWaitEvent(h->comp, h->part_ev[part], 0));
                h->run_tables(dst, h->fpitch, cn, s.sat.p + size_t(c0) * h->sat_size(), s.sat2.p + size_t(c0) * h->sat_size(),
                              s.dinv.p + size_t(c0) * h->dinv_size(), h->comp,
                              bst ? bst + size_t(c0) * h->dinv_size() : nullptr);
            }
            if (gbytes) {
                CK(cudaMemcpyAsync(s.gross.p, s.hgross.p, gbytes, cudaMemcpyHostToDevice, h->copy));
                dg = s.gross.p;
            }
            CK(cudaEventRecord(s.in, h->copy));
            CK(cudaStreamWaitEvent(h->comp, s.in, 0));
            float *o = s.out.p;
            h->run_group(s.frames.p, h->fpitch, nf, dg, gross_mode, s.sat.p, s.sat2.p, s.dinv.p, s.bstat.p, s.peaks.p, s.queue.p, o, o + 2 * PG,
                         o + 3 * PG, o + 4 * PG, nullptr, h->comp, true);
            CK(cudaMemcpyAsync(s.hout.p, s.out.p, 7 * PG * sizeof(float), cudaMemcpyDeviceToHost, h->comp));
            CK(cudaEventRecord(s.done, h->comp));
        }
        for (int g = std::max(0, ngroups - 2); g < ngroups; ++g) drain(g);
        int st = 0;
        CK(cudaMemcpy(&st, h->d_status.p, sizeof(int), cudaMemcpyDeviceToHost));
        if (st) {
            CK(cudaMemset(h->d_status.p, 0, sizeof(int)));
            fail(B200_ETIMEOUT, "a tensor-core completion wait gave up; the outputs are not valid");
        }
    });
}

static int correlate_device(b200_handle *h, const uint8_t *frames, int n, int pitch, const int32_t *gross,
                            int gross_mode, float *offset, float *peak, float *snr, float *cov, float *surface,
                            void *stream)
{
    return guarded(h, [&] {
        if (!h->ready) fail(B200_ERUNTIME, "set_reference first");
        if (n < 0) fail(B200_EINVAL, "the number of frames must not be negative");
        if (gross_mode < B200_GROSS_NONE || gross_mode > B200_GROSS_WINDOW || (gross_mode && !gross))
            fail(B200_EINVAL, "gross must be frames x 2 or frames x down x across x 2");
        if (n == 0) return;
        if (!frames || pitch < h->width || !offset || !peak || !snr || !cov) fail(B200_EINVAL, "null input or output, or a pitch below the width");
        CK(cudaSetDevice(h->device));
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        h->ensure_tables();
        // groups of equal size, at most h->group frames
        const int G = (n + (n + h->group - 1) / h->group - 1) / ((n + h->group - 1) / h->group), nwin = h->nwin;
        const int64_t fstride = int64_t(pitch) * h->height;
        for (int f0 = 0; f0 < n; f0 += G) {
            const int nf = std::min(G, n - f0);
            const size_t q0 = size_t(f0) * nwin;
            const int32_t *g = gross_mode == B200_GROSS_FRAME ? gross + 2 * size_t(f0)
                             : gross_mode == B200_GROSS_WINDOW ? gross + 2 * q0 : nullptr;
            h->run_group(frames + f0 * fstride, pitch, nf, g, gross_mode, h->d_sat.p, h->d_sat2.p, h->d_dinv.p, h->d_bstat.p, h->d_peaks.p, h->d_queue.p,
                         offset + 2 * q0, peak + q0, snr + q0, cov + 3 * q0,
                         surface ? surface + q0 * size_t(h->M) * h->M : nullptr, s);
        }
    });
}

int b200_correlate_device(b200_handle *h, const uint8_t *frames, int n, int pitch, const int32_t *gross,
                          int gross_mode, float *offset, float *peak, float *snr, float *cov, void *stream)
{
    return correlate_device(h, frames, n, pitch, gross, gross_mode, offset, peak, snr, cov, nullptr, stream);
}

int b200_correlate_device_surfaces(b200_handle *h, const uint8_t *frames, int n, int pitch, const int32_t *gross,
                                   int gross_mode, float *offset, float *peak, float *snr, float *cov,
                                   float *surface, void *stream)
{
    if (!surface) {
        if (h) h->err = "framecor: no surface output";
        return B200_EINVAL;
    }
    return correlate_device(h, frames, n, pitch, gross, gross_mode, offset, peak, snr, cov, surface, stream);
}

}   // extern "C"

// ---- the correlation without allocation -------------------------------------------------------
//
// Some callers cannot allocate device memory when they correlate: a capture loop that must never
// stall on cudaMalloc's implicit device synchronization, or a host that owns all device memory
// through its own arena and forbids the library from taking more. For them,
// b200_correlate_device_noalloc keeps the per-frame tables (summed-area tables and variance
// denominators) in one static device array, reserved when the library is loaded on a device and
// held until the process exits, instead of in buffers of the handle. Nothing here calls cudaMalloc,
// cudaFree or any allocating routine.
//
// The array holds 32 MiB: the tables of one 1920 x 1080 frame (16.0 bytes per pixel). Frames are
// correlated as many per launch as their tables fit. In host code the array's name is only a
// stand-in for its device address, so the address is looked up with cudaGetSymbolAddress, once per
// device, by the first call on that device with the device current; make that first call before
// any stream capture. Every call on a device shares the array, so calls that overlap on the GPU
// (two streams, two threads) race on it; keep them ordered. No part of the array has to start at
// zero: each call writes every table entry it reads (row and column 0 of the summed-area tables
// included) before the correlation kernel reads it.
namespace {

constexpr size_t kNoAllocBytes = size_t(32) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];
void *g_noalloc_addr[64] = {};
std::mutex g_noalloc_mutex;

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

}   // namespace

extern "C" {

int b200_correlate_device_noalloc(b200_handle *h, const uint8_t *frames, int n, int pitch, const int32_t *gross,
                                  int gross_mode, float *offset, float *peak, float *snr, float *cov, void *stream)
{
    return guarded(h, [&] {
        if (!h->ready) fail(B200_ERUNTIME, "set_reference first");
        if (n < 0) fail(B200_EINVAL, "the number of frames must not be negative");
        if (gross_mode < B200_GROSS_NONE || gross_mode > B200_GROSS_WINDOW || (gross_mode && !gross))
            fail(B200_EINVAL, "gross must be frames x 2 or frames x down x across x 2");
        if (n == 0) return;
        if (!frames || pitch < h->width || !offset || !peak || !snr || !cov)
            fail(B200_EINVAL, "null input or output, or a pitch below the width");
        // the tables of one frame: 32-bit and 64-bit summed-area tables, variance denominators
        const size_t b32 = size_t(h->sat_size()) * sizeof(uint32_t), b64 = size_t(h->sat_size()) * sizeof(int64_t);
        const size_t bd = size_t(h->dinv_size()) * sizeof(float);
        const size_t per_frame = align256(b32) + align256(b64) + align256(bd);
        if (per_frame > kNoAllocBytes)
            fail(B200_EINVAL, "the frame is too large for the no-allocation entry point: its tables need "
                                  + std::to_string(per_frame) + " bytes, the static scratch holds "
                                  + std::to_string(kNoAllocBytes) + " (one 1920 x 1080 frame)");
        if (h->device < 0 || h->device >= 64) fail(B200_EINVAL, "device index out of range");
        CK(cudaSetDevice(h->device));
        void *base = nullptr;
        {
            std::lock_guard<std::mutex> lock(g_noalloc_mutex);
            if (!g_noalloc_addr[h->device]) {
                void *p = nullptr;
                CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
                g_noalloc_addr[h->device] = p;
            }
            base = g_noalloc_addr[h->device];
        }
        const int G = int(std::min<size_t>(kNoAllocBytes / per_frame, size_t(h->group)));
        unsigned char *q = static_cast<unsigned char *>(base);
        uint32_t *sat = reinterpret_cast<uint32_t *>(q);
        int64_t *sat2 = reinterpret_cast<int64_t *>(q + align256(G * b32));
        float *dinv = reinterpret_cast<float *>(q + align256(G * b32) + align256(G * b64));
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const int nwin = h->nwin;
        const int64_t fstride = int64_t(pitch) * h->height;
        for (int f0 = 0; f0 < n; f0 += G) {
            const int nf = std::min(G, n - f0);
            const size_t q0 = size_t(f0) * nwin;
            launch_sat(frames + f0 * fstride, fstride, pitch, nf, h->height, h->width, sat, sat2, s);
            dinv_kernel<<<dim3(unsigned((h->width - h->W + 1 + 127) / 128), unsigned(h->height - h->W + 1), unsigned(nf)),
                          128, 0, s>>>(sat, sat2, h->sat_size(), h->height, h->width, h->W, dinv, h->dinv_size(), h->dpitch());
            CorrArgs a{};
            a.frames = frames + f0 * fstride;
            a.fstride = fstride;
            a.pitch = pitch;
            a.sat = sat;
            a.sat_fstride = h->sat_size();
            a.dinv = dinv;
            a.dinv_fstride = h->dinv_size();
            a.dpitch = h->dpitch();
            a.h = h->height;
            a.w = h->width;
            a.W = h->W;
            a.R = h->R;
            a.L = h->L;
            a.M = h->M;
            a.nx = h->nx;
            a.nwin = nwin;
            a.nf = nf;
            a.stat = h->stat;
            a.down = h->d_down.p;
            a.across = h->d_across.p;
            a.norm = h->d_norm.p;
            a.spec = h->d_spec.p;
            a.spec_tc = h->d_spec_tc.p;
            a.twiddles = h->d_tw.p;
            a.gross = gross_mode == B200_GROSS_FRAME ? gross + 2 * size_t(f0)
                    : gross_mode == B200_GROSS_WINDOW ? gross + 2 * q0 : nullptr;
            a.gross_mode = gross_mode;
            a.offset = offset + 2 * q0;
            a.peak = peak + q0;
            a.snr = snr + q0;
            a.cov = cov + 3 * q0;
            a.surface = nullptr;
            if (h->N == kBigN)
                launch_corr_big(a, h->d_big.p, s);
            else
                B200_DISPATCH(h->N, launch_corr, a, s);
            CK(cudaGetLastError());
            h->launches += 4;
        }
    });
}

int b200_tc_selftest(const void *A, const void *B, float *D, int N, int K, int a_mn, int b_mn, int neg_b, void *stream)
{
    if (!A || !B || !D || N < 16 || N > 256 || N % 16 || K < 16 || K % 16 || K > 256) return B200_EINVAL;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int *status = nullptr;
    if (cudaMallocAsync(&status, sizeof(int), s) != cudaSuccess) return B200_ERUNTIME;
    cudaMemsetAsync(status, 0, sizeof(int), s);
    TcSelftestArgs a{static_cast<const __half *>(A), static_cast<const __half *>(B), D, N, K, a_mn, b_mn, neg_b, status};
    const size_t smem = size_t(128 + N) * K * 2;
    if (cudaFuncSetAttribute(tc_selftest_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess)
        return B200_ERUNTIME;
    tc_selftest_kernel<<<1, 128, smem, s>>>(a);
    int h = 0;
    const bool ok = cudaGetLastError() == cudaSuccess && cudaMemcpyAsync(&h, status, sizeof(int), cudaMemcpyDeviceToHost, s) == cudaSuccess
                    && cudaStreamSynchronize(s) == cudaSuccess;
    cudaFreeAsync(status, s);
    if (!ok) return B200_ERUNTIME;
    return h ? B200_ETIMEOUT : B200_OK;
}

int b200_tc_i8_selftest(const uint8_t *A, const uint8_t *X, int32_t *D, int N, int K, int rows, int i, int a_smem,
                        void *stream)
{
    if (!A || !X || !D || N < 16 || N > 256 || N % 16 || K < 32 || K % 32 || K > 256 || i < 0 || rows < i + N
        || size_t(rows | 1) * K + 128 * size_t(K) > 200 * 1024)
        return B200_EINVAL;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int *status = nullptr;
    if (cudaMallocAsync(&status, sizeof(int), s) != cudaSuccess) return B200_ERUNTIME;
    cudaMemsetAsync(status, 0, sizeof(int), s);
    const I8SelftestArgs a{A, X, D, N, K, rows, i, a_smem, status};
    const size_t smem = ((size_t(rows | 1) * K + 127) & ~size_t(127)) + 128 * size_t(K);
    if (cudaFuncSetAttribute(tc_i8_selftest_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess)
        return B200_ERUNTIME;
    tc_i8_selftest_kernel<<<1, 128, smem, s>>>(a);
    int h = 0;
    const bool ok = cudaGetLastError() == cudaSuccess && cudaMemcpyAsync(&h, status, sizeof(int), cudaMemcpyDeviceToHost, s) == cudaSuccess
                    && cudaStreamSynchronize(s) == cudaSuccess;
    cudaFreeAsync(status, s);
    if (!ok) return B200_ERUNTIME;
    return h ? B200_ETIMEOUT : B200_OK;
}

namespace {
__global__ void frame_diff_means_kernel(const unsigned long long *sums, int n, double npix, float *out)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) out[k] = float(double(sums[k]) / npix);
}
unsigned blocks_for(int64_t n, int per = 256) { return unsigned((n + per - 1) / per); }
}   // namespace

int b200_frame_diff_device(const uint8_t *frames, int n, int height, int width, int pitch, float *out, uint64_t *sums,
                           void *stream)
{
    if (n < 0 || height <= 0 || width <= 0 || pitch < width || (n > 1 && (!frames || !out || !sums))) return B200_EINVAL;
    if (n < 2) return B200_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned long long *us = reinterpret_cast<unsigned long long *>(sums);
    if (cudaMemsetAsync(us, 0, size_t(n - 1) * sizeof(uint64_t), s) != cudaSuccess) return B200_ERUNTIME;
    // runs of kDiffRun pairs, and bands of rows for two full waves of the CTAs the SMs hold at once
    int dev = 0, sms = 148, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return B200_ERUNTIME;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, frame_diff_kernel, 256, 0) != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        per_sm = 2;
    }
    const int runs = (n - 1 + kDiffRun - 1) / kDiffRun;
    const unsigned bands = unsigned(std::clamp(2 * sms * per_sm / runs, 1, height));
    frame_diff_kernel<<<dim3(bands, unsigned(runs)), 256, 0, s>>>(frames, int64_t(pitch) * height, pitch, height, width,
                                                                  n - 1, us);
    frame_diff_means_kernel<<<blocks_for(n - 1), 256, 0, s>>>(us, n - 1, double(height) * width, out);
    return cudaGetLastError() == cudaSuccess ? B200_OK : B200_ERUNTIME;
}

int b200_chunk_std_median_device(const uint8_t *frames, int nchunks, int chunk, int height, int width, int pitch,
                                 float *out, void *stream)
{
    if (nchunks < 1 || nchunks > kScanMaxChunks || chunk < 1 || chunk > 65536 || height <= 0 || width <= 0 || pitch < width ||
        !frames || !out)
        return B200_EINVAL;
    // a frame with contiguous rows is one long row: whole CTAs of pixels and 16-byte loads throughout
    const int64_t fstride = int64_t(pitch) * height;
    int rows = height, cols = width, step = pitch;
    if (pitch == width && int64_t(height) * width <= INT32_MAX) {
        cols = height * width;
        rows = 1;
        step = cols;
    }
    // the numerators fit 32 bits while chunk <= 513 (chunk^2 x 127.5^2 < 2^32)
    const bool narrow = chunk <= 513;
    const size_t smem = size_t(nchunks) * kStdPixels * (narrow ? 4 : 8);
    int dev = 0, optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
        return B200_ERUNTIME;
    if (smem > size_t(optin)) return B200_EINVAL;
    const void *kernel = narrow ? reinterpret_cast<const void *>(chunk_std_median_kernel<uint32_t>)
                                : reinterpret_cast<const void *>(chunk_std_median_kernel<uint64_t>);
    if (smem > 48 * 1024 && cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess)
        return B200_ERUNTIME;
    const dim3 grid(unsigned((cols + kStdPixels - 1) / kStdPixels), unsigned(rows));
    const dim3 block(32, unsigned(std::min(nchunks, 8)));   // 8 warps: four CTAs per SM, one's median beside another's loads
    if (narrow)
        chunk_std_median_kernel<uint32_t><<<grid, block, smem, static_cast<cudaStream_t>(stream)>>>(frames, fstride, step, rows,
                                                                                                  cols, chunk, nchunks, out);
    else
        chunk_std_median_kernel<uint64_t><<<grid, block, smem, static_cast<cudaStream_t>(stream)>>>(frames, fstride, step, rows,
                                                                                                  cols, chunk, nchunks, out);
    return cudaGetLastError() == cudaSuccess ? B200_OK : B200_ERUNTIME;
}

int b200_sobel_device(const uint8_t *frame, int height, int width, int pitch, float *out, void *stream)
{
    if (height <= 0 || width <= 0 || pitch < width || !frame || !out) return B200_EINVAL;
    sobel_kernel<<<blocks_for(int64_t(height) * width), 256, 0, static_cast<cudaStream_t>(stream)>>>(frame, pitch, height,
                                                                                                      width, out);
    return cudaGetLastError() == cudaSuccess ? B200_OK : B200_ERUNTIME;
}

namespace {

// the three selection passes of numpy.percentile(x[0 .. n), q) into *out (device), q in [0, 100]:
// the virtual index, its floor and the weight in float32, as numpy computes them for float32 data
int launch_percentile(const float *x, int64_t n, double q, float *out, void *scratch, cudaStream_t s)
{
    if (!x || !out || !scratch || n < 1 || n > int64_t(UINT32_MAX) || !(q >= 0.0 && q <= 100.0)) return B200_EINVAL;
    const float vi = float(n - 1) * (float(q) / 100.0f);
    uint32_t lo = uint32_t(n - 1), hi = lo;
    float t = 1.0f;   // past the last index: both statistics are the largest value
    if (vi < float(n - 1)) {
        lo = uint32_t(std::floor(vi));
        hi = lo + 1;
        t = vi - float(lo);
    }
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return B200_ERUNTIME;
    auto *st = static_cast<SelectState *>(scratch);
    auto *hist = reinterpret_cast<uint32_t *>(static_cast<char *>(scratch) + 256);
    if (cudaMemsetAsync(scratch, 0, kSelectScratch, s) != cudaSuccess) return B200_ERUNTIME;
    const unsigned grid = unsigned(std::clamp<int64_t>((n + 4095) / 4096, 1, 2 * sms));   // 16 elements a thread or more
    for (int pass = 0; pass < 3; ++pass) select_pass_kernel<<<grid, 256, 0, s>>>(x, n, pass, lo, hi, t, st, hist, out);
    return cudaGetLastError() == cudaSuccess ? B200_OK : B200_ERUNTIME;
}

}   // namespace

int b200_percentile_f32_device(const float *x, int64_t n, double q, float *out, void *scratch, void *stream)
{
    return launch_percentile(x, n, q, out, scratch, static_cast<cudaStream_t>(stream));
}

size_t b200_text_mask_scratch_bytes(int height, int width)
{
    if (height <= 0 || width <= 0) return 0;
    return size_t(kSelectScratch) + 2 * size_t(height) * size_t((width + 31) / 32) * 4;
}

int b200_text_mask_device(const float *edge, const float *sd, int height, int width, double edge_percentile, float max_std,
                          int dilate, uint8_t *mask, void *scratch, size_t scratch_bytes, void *stream)
{
    if (height <= 0 || width <= 0 || !edge || !sd || !mask || !scratch) return B200_EINVAL;
    const int64_t n = int64_t(height) * width;
    const int wpr = (width + 31) / 32;
    const size_t tile = size_t(2) * (kDilateRows + 2 * kDilateStep) * wpr * 4;   // the dilation's shared memory
    if (scratch_bytes < b200_text_mask_scratch_bytes(height, width) || n > int64_t(INT32_MAX) || tile > 227 * 1024)
        return B200_EINVAL;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    float *thr = reinterpret_cast<float *>(static_cast<char *>(scratch) + sizeof(SelectState));
    if (int rc = launch_percentile(edge, n, edge_percentile, thr, scratch, s); rc != B200_OK) return rc;
    uint32_t *m = reinterpret_cast<uint32_t *>(static_cast<char *>(scratch) + kSelectScratch), *o = m + int64_t(height) * wpr;
    text_seed_bits_kernel<<<unsigned((int64_t(height) * wpr * 32 + 255) / 256), 256, 0, s>>>(edge, sd, height, width, wpr,
                                                                                             thr, max_std, m);
    if (dilate < 1) {   // until nothing changes (scipy's iterations < 1): every pixel if any is set
        const int64_t words = int64_t(height) * wpr;
        if (cudaMemsetAsync(o, 0, sizeof(uint32_t), s) != cudaSuccess) return B200_ERUNTIME;
        any_bits_kernel<<<unsigned(std::min<int64_t>((words + 255) / 256, 1184)), 256, 0, s>>>(m, words, o);
        all_bits_kernel<<<unsigned((words + 255) / 256), 256, 0, s>>>(m, height, width, wpr, o);
    }
    for (int done = 0; done < dilate; done += kDilateStep) {
        const int steps = std::min(kDilateStep, dilate - done);
        const size_t bytes = size_t(2) * (kDilateRows + 2 * steps) * wpr * 4;
        if (bytes > 48 * 1024 &&
            cudaFuncSetAttribute(dilate_bits_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)) != cudaSuccess)
            return B200_ERUNTIME;
        dilate_bits_kernel<<<unsigned((height + kDilateRows - 1) / kDilateRows), 256, bytes, s>>>(m, o, height, width, wpr,
                                                                                                 steps);
        std::swap(m, o);
    }
    int dev = 0, optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
        return B200_ERUNTIME;
    // the hole filling: a cluster of CTAs holding bands of rows when a band fits a CTA's shared
    // memory (720p: 31 KB, 2160 x 3840: 273 KB, too much) and the cluster can be placed
    const int hb = ((height + kFloodCluster - 1) / kFloodCluster + 31) / 32 * 32;
    const size_t band_bytes = (2 * size_t(hb) * wpr + 4 * size_t(wpr)) * 4 + 2 * sizeof(int);
    if (band_bytes <= size_t(optin)) {
        if (band_bytes > 48 * 1024 &&
            cudaFuncSetAttribute(flood_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(band_bytes)) !=
                cudaSuccess)
            return B200_ERUNTIME;
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(kFloodCluster, 1, 1);
        cfg.blockDim = dim3(kFloodThreads, 1, 1);
        cfg.dynamicSmemBytes = band_bytes;
        int clusters = 0;
        if (cudaOccupancyMaxActiveClusters(&clusters, flood_cluster_kernel, &cfg) == cudaSuccess && clusters > 0) {
            flood_cluster_kernel<<<kFloodCluster, kFloodThreads, band_bytes, s>>>(m, o, height, width, wpr, hb);
            fill_bits_kernel<<<blocks_for(n), 256, 0, s>>>(o, height, width, wpr, mask);
            return cudaGetLastError() == cudaSuccess ? B200_OK : B200_ERUNTIME;
        }
        cudaGetLastError();
    }
    // else one CTA, the two planes in its shared memory when they fit (720p: 225 KB)
    const size_t planes = size_t(2) * height * wpr * 4;
    const bool in_smem = planes <= size_t(optin);
    if (in_smem && planes > 48 * 1024 &&
        cudaFuncSetAttribute(flood_bits_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(planes)) != cudaSuccess)
        return B200_ERUNTIME;
    flood_bits_kernel<<<1, kFloodThreads, in_smem ? planes : 0, s>>>(m, o, height, width, wpr, in_smem ? 1 : 0);
    fill_bits_kernel<<<blocks_for(n), 256, 0, s>>>(o, height, width, wpr, mask);
    return cudaGetLastError() == cudaSuccess ? B200_OK : B200_ERUNTIME;
}

// frames per group of coarse tracking's tables (two groups resident)
constexpr int kCoarseGroup = 8;

int b200_coarse_track_device(b200_handle *h, const uint8_t *frames, int n, int pitch, const uint8_t *keep,
                             double min_peak, int reset, int32_t *gross, double *prev, double *params, int32_t *used,
                             void *stream)
{
    return guarded(h, [&] {
        if (!h->ready) fail(B200_ERUNTIME, "set_reference first");
        if (n < 0) fail(B200_EINVAL, "the number of frames must not be negative");
        if (h->W % 2) fail(B200_EINVAL, "coarse tracking needs an even window");
        if (h->nwin > B200_COARSE_MAX_WINDOWS)
            fail(B200_EINVAL, "coarse tracking handles up to " + std::to_string(B200_COARSE_MAX_WINDOWS) + " windows");
        if (!keep || !gross || !prev || (n && (!frames || !params || !used || pitch < h->width)))
            fail(B200_EINVAL, "null input or output, or a pitch below the width");
        CK(cudaSetDevice(h->device));
        cudaStream_t caller = static_cast<cudaStream_t>(stream);
        const size_t nwin = size_t(h->nwin), MM = size_t(h->M) * h->M;
        if (reset) {
            CK(cudaMemsetAsync(gross, 0, 2 * nwin * sizeof(int32_t), caller));
            CK(cudaMemsetAsync(prev, 0, 4 * sizeof(double), caller));
        }
        if (n == 0) return;
        if (!h->coarse_ev[0])
            for (cudaEvent_t &e : h->coarse_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        // the frame chain runs on the handle's own stream, after the caller's work and before the
        // caller's next: there the grid's reference spectra persist in L2 (every frame reads them;
        // the next group's tables, written beside the chain, would otherwise evict them)
        cudaStream_t s = h->comp;
        if (!h->coarse_l2) {   // the carve-out once per handle (the previous limit comes back at destroy)
            cudaDeviceProp prop{};
            CK(cudaGetDeviceProperties(&prop, h->device));
            const size_t want = nwin * size_t(h->N / 2 + 1) * h->N * sizeof(float2);
            const size_t carve = std::min<size_t>(want, size_t(prop.persistingL2CacheMaxSize));
            size_t cur = 0;
            CK(cudaDeviceGetLimit(&cur, cudaLimitPersistingL2CacheSize));
            if (carve > cur) {
                CK(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, carve));
                h->l2_limit_prev = cur;
                h->l2_raised = true;
            }
            h->l2win.base_ptr = h->d_spec.p;
            h->l2win.num_bytes = std::min<size_t>(want, size_t(prop.accessPolicyMaxWindowSize));
            h->l2win.hitRatio = carve >= h->l2win.num_bytes ? 1.0f : float(double(carve) / double(h->l2win.num_bytes));
            h->l2win.hitProp = cudaAccessPropertyPersisting;
            h->l2win.missProp = cudaAccessPropertyStreaming;
            h->coarse_l2 = true;
        }
        {   // the window covers this call's chain only: the handle's stream serves other calls too
            cudaStreamAttrValue v{};
            v.accessPolicyWindow = h->l2win;
            CK(cudaStreamSetAttribute(s, cudaStreamAttributeAccessPolicyWindow, &v));
        }
        CK(cudaEventRecord(h->coarse_ev[4], caller));
        CK(cudaStreamWaitEvent(s, h->coarse_ev[4], 0));
        // the big transform has no fused peak: its surfaces go through the peak kernel
        const bool fused = h->N != kBigN;
        const size_t work = nwin * (7 + (fused ? 0 : MM));
        if (h->d_coarse.n < work) h->d_coarse.alloc(work);
        if (h->d_cpeaks.n < 3 * nwin) h->d_cpeaks.alloc(3 * nwin);
        float *o = h->d_coarse.p, *surf = fused ? nullptr : o + 7 * nwin;
        const int64_t fstride = int64_t(pitch) * h->height;
        FitArgs fa{h->d_cpeaks.p, gross, keep, h->d_down.p, h->d_across.p, h->W / 2, h->ny, h->nx, h->height,
                   h->width, h->W, h->R, min_peak, prev, nullptr, nullptr};
        // two sets of tables of up to kCoarseGroup frames: those of group g + 1 are built on the side
        // stream while the frames of group g are tracked on `stream` (the chain of one frame leaves
        // most SMs idle, and the tables of a group take a fraction of its chain)
        const int G = std::min(h->group, kCoarseGroup);
        if (!h->d_csat.p) {
            h->d_csat.alloc(2 * size_t(G) * h->sat_size());
            h->d_csat2.alloc(2 * size_t(G) * h->sat_size());
            h->d_cdinv.alloc(2 * size_t(G) * h->dinv_size());
        }
        uint32_t *sat[2] = {h->d_csat.p, h->d_csat.p + size_t(G) * h->sat_size()};
        int64_t *sat2[2] = {h->d_csat2.p, h->d_csat2.p + size_t(G) * h->sat_size()};
        float *dinv[2] = {h->d_cdinv.p, h->d_cdinv.p + size_t(G) * h->dinv_size()};
        cudaEvent_t *ready = h->coarse_ev, *consumed = h->coarse_ev + 2, start = h->coarse_ev[4];
        cudaStream_t side = h->copy;
        const int groups = (n + G - 1) / G;
        auto tables = [&](int g) {
            const int nf = std::min(G, n - g * G);
            if (g >= 2) CK(cudaStreamWaitEvent(side, consumed[g % 2], 0));
            h->run_tables(frames + int64_t(g) * G * fstride, pitch, nf, sat[g % 2], sat2[g % 2], dinv[g % 2], side);
            CK(cudaGetLastError());
            CK(cudaEventRecord(ready[g % 2], side));
            h->launches += 3;
        };
        CK(cudaStreamWaitEvent(side, start, 0));   // the frames and the state are written on the caller's stream
        // and the previous call's chain, which may still read both table sets, is done with them (a
        // caller that changes streams between calls orders nothing by itself)
        CK(cudaStreamWaitEvent(side, h->coarse_ev[5], 0));
        tables(0);
        for (int g = 0; g < groups; ++g) {
            if (g + 1 < groups) tables(g + 1);
            CK(cudaStreamWaitEvent(s, ready[g % 2], 0));
            const int nf = std::min(G, n - g * G);
            for (int j = 0; j < nf; ++j) {
                const int f = g * G + j;
                CorrArgs a = h->corr_args(frames + int64_t(f) * fstride, pitch, 1, gross, B200_GROSS_WINDOW,
                                          sat[g % 2] + j * h->sat_size(), dinv[g % 2] + j * h->dinv_size(), o,
                                          o + 2 * nwin, o + 3 * nwin, o + 4 * nwin, surf);
                if (fused) {
                    a.ncc = h->d_cpeaks.p;
                    B200_DISPATCH(h->N, launch_corr_latency, a, s);
                    CK(cudaGetLastError());
                    h->launches += 1;
                } else {
                    h->run_corr_tail(a, 1, a.dinv, B200_FORM_FFT32, s);   // counts its launch
                    CK(launch_ncc_peaks(surf, int(nwin), h->M, h->d_cpeaks.p, s));
                    h->launches += 1;
                }
                fa.params = params + 4 * size_t(f);
                fa.used = used + f;
                CK(launch_coarse_fit(fa, s));
                h->launches += 1;
            }
            CK(cudaEventRecord(consumed[g % 2], s));
        }
        CK(cudaEventRecord(h->coarse_ev[5], s));   // the caller's stream continues after the chain
        CK(cudaStreamWaitEvent(caller, h->coarse_ev[5], 0));
        cudaStreamAttrValue none{};   // later launches on the handle's stream carry no window
        none.accessPolicyWindow.num_bytes = 0;
        CK(cudaStreamSetAttribute(s, cudaStreamAttributeAccessPolicyWindow, &none));
    });
}

int b200_periodicity_device(b200_handle *h, const float *surface, int exclude, float *out, void *stream)
{
    return guarded(h, [&] {
        if (!h->ready) fail(B200_ERUNTIME, "set_reference first");
        if (!surface || !out) fail(B200_EINVAL, "null input or output");
        if (exclude < 0) fail(B200_EINVAL, "the exclusion must not be negative");
        CK(cudaSetDevice(h->device));
        periodicity_kernel<256><<<unsigned(h->nwin), 256, 0, static_cast<cudaStream_t>(stream)>>>(
            surface, h->d_norm.p, h->M, h->R, exclude, out);
        CK(cudaGetLastError());
        h->launches += 1;
    });
}

int b200_set_reference_f32_device(b200_handle *h, const float *frame, int pitch, void *stream)
{
    return guarded(h, [&] {
        if (!frame || pitch < h->width) fail(B200_EINVAL, "no reference frame, or its pitch is below its width");
        CK(cudaSetDevice(h->device));
        upload_reference(h, nullptr, pitch, static_cast<cudaStream_t>(stream), frame);
        h->ready = true;
    });
}

int b200_diff_forward(b200_handle *h, const float *frames, int n, int pitch, const int32_t *gross, int gross_mode,
                      const float *shift, float *chips, float *stats, float *surface, int *peak_at, float *offset,
                      float *peak, float *snr, float *cov, void *stream)
{
    return guarded(h, [&] {
        DiffArgs a = diff_args(h, frames, n, pitch, gross, gross_mode, shift);
        if (n == 0) return;
        if (!chips || !stats || !surface || !peak_at || !offset || !peak || !snr || !cov) fail(B200_EINVAL, "null output");
        a.chips = chips;
        a.stats = stats;
        a.surface = surface;
        a.peak_at = peak_at;
        a.offset = offset;
        a.peak = peak;
        a.snr = snr;
        a.cov = cov;
        CK(cudaSetDevice(h->device));
        launch_diff_forward(a, h->N, static_cast<cudaStream_t>(stream));
        h->launches += 3;
    });
}

int b200_diff_backward(b200_handle *h, const float *frames, int n, int pitch, const int32_t *gross, int gross_mode,
                       const float *shift, const float *chips, const float *stats, const float *surface,
                       const float *g_surface, float *g_chips, float *g_frames, float *g_shift, void *stream)
{
    return guarded(h, [&] {
        DiffArgs a = diff_args(h, frames, n, pitch, gross, gross_mode, shift);
        if (n == 0) return;
        if (!chips || !stats || !surface || !g_surface || !g_chips) fail(B200_EINVAL, "null input or output");
        a.chips = const_cast<float *>(chips);
        a.stats = const_cast<float *>(stats);
        a.surface = const_cast<float *>(surface);
        a.g_surface = g_surface;
        a.g_chips = g_chips;
        a.g_frames = g_frames;
        a.g_shift = g_shift;
        CK(cudaSetDevice(h->device));
        launch_diff_backward(a, h->N, static_cast<cudaStream_t>(stream));
        h->launches += 2;
    });
}

int b200_offset_adjoint(b200_handle *h, int n, const float *surface, const int *peak_at, const float *g_offset,
                        float *g_surface, void *stream)
{
    return guarded(h, [&] {
        if (n < 0) fail(B200_EINVAL, "the number of frames must not be negative");
        if (n == 0) return;
        if (!surface || !peak_at || !g_offset || !g_surface) fail(B200_EINVAL, "null input or output");
        CK(cudaSetDevice(h->device));
        const int64_t pairs = int64_t(n) * h->nwin;
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        CK(cudaMemsetAsync(g_surface, 0, size_t(pairs) * h->M * h->M * sizeof(float), s));
        launch_offset_adjoint(surface, peak_at, g_offset, g_surface, h->M, pairs, s);
        h->launches += 1;
    });
}

int b200_sat_device(const uint8_t *frames, int n, int height, int width, int pitch, uint32_t *sat, int64_t *sat2,
                    void *stream)
{
    if (n < 0 || height <= 0 || width <= 0 || pitch < width || (n && (!frames || !sat || !sat2))) return B200_EINVAL;
    if (n == 0) return B200_OK;
    launch_sat(frames, int64_t(pitch) * height, pitch, n, height, width, sat, sat2, static_cast<cudaStream_t>(stream));
    return cudaGetLastError() == cudaSuccess ? B200_OK : B200_ERUNTIME;
}

int b200_profile(b200_handle *h, int enable)
{
    return guarded(h, [&] { h->profiling = enable != 0; });
}

int b200_profile_read(b200_handle *h, double *kernel_ms, uint64_t *kernel_launches, uint64_t *pairs)
{
    return guarded(h, [&] {
        double ms = 0.0;
        uint64_t np = 0;
        for (auto &t : h->timed) {
            CK(cudaEventSynchronize(t.b));
            float e = 0.f;
            CK(cudaEventElapsedTime(&e, t.a, t.b));
            ms += e;
            np += t.pairs;
            cudaEventDestroy(t.a);
            cudaEventDestroy(t.b);
        }
        if (kernel_ms) *kernel_ms = ms;
        if (kernel_launches) *kernel_launches = h->timed.size();
        if (pairs) *pairs = np;
        h->timed.clear();
    });
}

int b200_status(b200_handle *h, void *stream, int *status)
{
    return guarded(h, [&] {
        if (!status) fail(B200_EINVAL, "no status output");
        CK(cudaSetDevice(h->device));
        CK(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
        CK(cudaStreamSynchronize(h->comp));
        int st = 0;
        CK(cudaMemcpy(&st, h->d_status.p, sizeof(int), cudaMemcpyDeviceToHost));
        if (st) CK(cudaMemset(h->d_status.p, 0, sizeof(int)));
        *status = st;
    });
}

int b200_inject_alloc_failure(int nth)
{
    if (nth < 0) return B200_EINVAL;
    g_fail_alloc.store(nth);
    return B200_OK;
}

int b200_host_copy(void *dst, const void *src, size_t n)
{
    if (n == 0) return B200_OK;
    if (!dst || !src) return B200_EINVAL;
    stream_copy(static_cast<char *>(dst), static_cast<const char *>(src), n);
    return B200_OK;
}

int b200_wait_selftest(unsigned polls, double limit_ms, void *stream)
{
    if (polls < 1 || !(limit_ms > 0.0) || limit_ms > 1000.0) return B200_EINVAL;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int *d = nullptr;
    if (cudaMallocAsync(&d, 2 * sizeof(int), s) != cudaSuccess) return B200_ERUNTIME;
    wait_selftest_kernel<<<1, 32, 0, s>>>(polls, uint64_t(limit_ms * 1e6), d);
    int out[2] = {0, 0};
    const bool ok = cudaGetLastError() == cudaSuccess &&
                    cudaMemcpyAsync(out, d, sizeof(out), cudaMemcpyDeviceToHost, s) == cudaSuccess &&
                    cudaStreamSynchronize(s) == cudaSuccess;
    cudaFreeAsync(d, s);
    if (!ok) return B200_ERUNTIME;
    return out[0] && out[1] ? B200_ETIMEOUT : B200_ERUNTIME;
}

int b200_info(const b200_handle *h, int *ny, int *nx, int *fft_size, uint64_t *launches)
{
    if (!h) return B200_EINVAL;
    if (ny) *ny = h->ny;
    if (nx) *nx = h->nx;
    if (fft_size) *fft_size = h->N;
    if (launches) *launches = h->launches;
    return B200_OK;
}

const char *b200_backend(const b200_handle *) { return "b200"; }

int b200_has_device(void)
{
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) return 0;
    for (int d = 0; d < count; ++d) {
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, d) == cudaSuccess && prop.major == 10) return 1;
    }
    return 0;
}

const char *b200_version(void) { return "0.1.0"; }

}   // extern "C"

// ---- groups of grids in one persistent launch (multi.h, multi.cu)

struct b200_group {
    std::vector<b200_handle *> grids;
    int height = 0, width = 0, device = 0;
    std::string err;
    cudaStream_t stream = nullptr;       // the group's own stream: graph capture and replay
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    int cap = 0;                         // frames the per-call tables hold
    DevBuf<uint32_t> sat;
    DevBuf<int64_t> sat2;
    std::vector<int> wsizes;             // the distinct window sizes, one denominator table each
    std::vector<DevBuf<float>> dinv;
    DevBuf<int> counter;
    DevBuf<MultiArgs> args;
    DevBuf<float2> big;                  // the N = 256 grid's per-CTA scratch
    size_t big_per_cta = 0;
    int nt = 256, chunk = 1;             // the launch configuration (b200_group_tune)
    bool costly_first = true, use_graph = true;
    bool per_grid = false;               // each grid's own kernel instead of the persistent launch
    MultiArgs host_args{};               // the arguments of the current step (per-grid mode)
    cudaGraphExec_t exec = nullptr;
    std::vector<uintptr_t> key;          // what the captured step was made for
    uint64_t launches = 0;

    ~b200_group()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (ev_in) cudaEventDestroy(ev_in);
        if (ev_out) cudaEventDestroy(ev_out);
        if (stream) cudaStreamDestroy(stream);
    }

    int64_t sat_size() const { return int64_t(height + 1) * (width + 1); }
    int dpitch() const { return (width + 3) & ~3; }
    int64_t dinv_size() const { return int64_t(height) * dpitch(); }

    size_t smem() const
    {
        size_t m = 0;
        for (const b200_handle *h : grids) m = std::max(m, multi_smem(h->N));
        return m;
    }

    int grid_ctas() const { return num_sms() * multi_occupancy(nt, smem()); }

    // the per-call tables for n frames and the big scratch for the current grid size
    void reserve(int n)
    {
        const size_t need_big = size_t(grid_ctas()) * big_per_cta;
        if (n <= cap && big.n >= need_big) return;
        CK(cudaStreamSynchronize(stream));   // nothing in flight may still read them
        if (n > cap) {
            sat.alloc(size_t(n) * sat_size());
            sat2.alloc(size_t(n) * sat_size());
            for (DevBuf<float> &d : dinv) d.alloc(size_t(n) * dinv_size());
            cap = n;
        }
        if (big.n < need_big) big.alloc(need_big);
        key.clear();
    }

    // the arguments of one launch over n frames
    MultiArgs make_args(const uint8_t *frames, int n, int pitch, const int32_t *const *gross, const int *mode,
                        float *const *offset, float *const *peak, float *const *snr, float *const *cov) const
    {
        MultiArgs m{};
        m.ngrids = int(grids.size());
        for (int i = 0; i < m.ngrids; ++i) {
            const b200_handle *h = grids[size_t(i)];
            CorrArgs &a = m.g[i].a;
            a.frames = frames;
            a.fstride = int64_t(pitch) * height;
            a.pitch = pitch;
            a.sat = sat.p;
            a.sat_fstride = sat_size();
            const size_t wi = size_t(std::find(wsizes.begin(), wsizes.end(), h->W) - wsizes.begin());
            a.dinv = dinv[wi].p;
            a.dinv_fstride = dinv_size();
            a.dpitch = dpitch();
            a.h = height;
            a.w = width;
            a.W = h->W;
            a.R = h->R;
            a.L = h->L;
            a.M = h->M;
            a.nx = h->nx;
            a.nwin = h->nwin;
            a.nf = n;
            a.stat = h->stat;
            a.down = h->d_down.p;
            a.across = h->d_across.p;
            a.norm = h->d_norm.p;
            a.spec = h->d_spec.p;
            a.twiddles = h->d_tw.p;
            a.gross = gross ? gross[i] : nullptr;
            a.gross_mode = gross && gross[i] ? mode[i] : 0;
            a.offset = offset[i];
            a.peak = peak[i];
            a.snr = snr[i];
            a.cov = cov[i];
            m.g[i].N = h->N;
            m.g[i].chunk = chunk;
            m.g[i].items = int((int64_t(h->nwin) * n + chunk - 1) / chunk);
            m.total_items += m.g[i].items;
            m.order[i] = i;
        }
        if (costly_first) {   // by the work of one pair, N^2 log N
            auto cost = [&](int i) { const double N = grids[size_t(i)]->N; return N * N * std::log2(N); };
            std::stable_sort(m.order, m.order + m.ngrids, [&](int x, int y) { return cost(x) > cost(y); });
        }
        m.counter = counter.p;
        m.big_scratch = big.p;
        m.big_per_cta = big_per_cta;
        return m;
    }

    // the step on the group's stream: tables, denominators, the persistent launch
    void step(const uint8_t *frames, int n, int pitch)
    {
        launch_sat(frames, int64_t(pitch) * height, pitch, n, height, width, sat.p, sat2.p, stream);
        for (size_t wi = 0; wi < wsizes.size(); ++wi) {
            const int W = wsizes[wi];
            dinv_kernel<<<dim3(unsigned((width - W + 1 + 127) / 128), unsigned(height - W + 1), unsigned(n)), 128, 0, stream>>>(
                sat.p, sat2.p, sat_size(), height, width, W, dinv[wi].p, dinv_size(), dpitch());
        }
        if (per_grid) {
            for (int i = 0; i < host_args.ngrids; ++i) {
                const MultiGrid &G = host_args.g[host_args.order[i]];
                if (G.N == kBigN)
                    launch_corr_big(G.a, big.p, stream);
                else
                    B200_DISPATCH(G.N, launch_corr, G.a, stream);
            }
        } else {
            CK(cudaMemsetAsync(counter.p, 0, sizeof(int), stream));
            launch_corr_multi(args.p, nt, smem(), grid_ctas(), stream);
        }
        CK(cudaGetLastError());
    }

    // the arguments of a step, on the device and here
    void set_args(const MultiArgs &m)
    {
        host_args = m;
        CK(cudaMemcpy(args.p, &m, sizeof(MultiArgs), cudaMemcpyHostToDevice));
    }
};

namespace {

template <class F>
int guarded_group(b200_group *g, F &&f)
{
    if (!g) return B200_EINVAL;
    try {
        f();
        g->err.clear();
        return B200_OK;
    } catch (const Failure &e) {
        g->err = e.msg;
        return e.code;
    } catch (const std::bad_alloc &) {
        g->err = "framecor: out of host memory";
        return B200_ERUNTIME;
    } catch (const std::invalid_argument &e) {
        g->err = std::string("framecor: ") + e.what();
        return B200_EINVAL;
    } catch (const std::exception &e) {
        g->err = std::string("framecor: ") + e.what();
        return B200_ERUNTIME;
    }
}

void check_group_call(const b200_group *g, const uint8_t *frames, int n, int pitch, const int32_t *const *gross,
                      const int *mode)
{
    if (n < 0) fail(B200_EINVAL, "the number of frames must not be negative");
    if (n && (!frames || pitch < g->width)) fail(B200_EINVAL, "no frames, or their pitch is below their width");
    for (size_t i = 0; i < g->grids.size(); ++i) {
        if (!g->grids[i]->ready) fail(B200_ERUNTIME, "set_reference first (grid " + std::to_string(i) + ")");
        if (gross && gross[i] && (!mode || mode[i] < B200_GROSS_FRAME || mode[i] > B200_GROSS_WINDOW))
            fail(B200_EINVAL, "gross must be frames x 2 or frames x down x across x 2");
    }
}

}   // namespace

extern "C" {

int b200_group_create(b200_handle *const *grids, int count, b200_group **out)
{
    if (out) *out = nullptr;
    b200_group *g = nullptr;
    try {
        if (!out || !grids) fail(B200_EINVAL, "no grids or no output");
        if (count < 1 || count > kMaxGrids) fail(B200_EINVAL, "a group holds 1 to 4 grids");
        g = new b200_group;
        for (int i = 0; i < count; ++i) {
            b200_handle *h = grids[i];
            if (!h) fail(B200_EINVAL, "a null grid");
            if (i && (h->height != g->height || h->width != g->width || h->device != g->device))
                fail(B200_EINVAL, "the grids of a group must share the frame size and the device");
            if (!multi_supports(h->N)) fail(B200_EINVAL, "no multi-grid kernel for the FFT size " + std::to_string(h->N));
            g->height = h->height;
            g->width = h->width;
            g->device = h->device;
            g->grids.push_back(h);
            if (std::find(g->wsizes.begin(), g->wsizes.end(), h->W) == g->wsizes.end()) g->wsizes.push_back(h->W);
            if (h->N == kBigN) g->big_per_cta = std::max(g->big_per_cta, big_scratch_per_cta(h->L, h->M));
        }
        CK(cudaSetDevice(g->device));
        CK(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&g->ev_in, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&g->ev_out, cudaEventDisableTiming));
        g->dinv.resize(g->wsizes.size());
        g->counter.alloc(1);
        g->args.alloc(1);
        prepare_multi();
        if (g->big_per_cta) prepare_big();
        *out = g;
        return B200_OK;
    } catch (const Failure &e) {
        g_create_error = e.msg;
        delete g;
        return e.code;
    } catch (const std::exception &e) {
        g_create_error = std::string("framecor: ") + e.what();
        delete g;
        return B200_ERUNTIME;
    }
}

int b200_group_destroy(b200_group *g)
{
    if (!g) return B200_EINVAL;
    cudaSetDevice(g->device);
    cudaStreamSynchronize(g->stream);
    delete g;
    return B200_OK;
}

const char *b200_group_last_error(const b200_group *g) { return g ? g->err.c_str() : g_create_error.c_str(); }

int b200_group_correlate_device(b200_group *g, const uint8_t *frames, int n, int pitch, const int32_t *const *gross,
                                const int *gross_mode, float *const *offset, float *const *peak, float *const *snr,
                                float *const *cov, void *stream)
{
    return guarded_group(g, [&] {
        check_group_call(g, frames, n, pitch, gross, gross_mode);
        if (n == 0) return;
        if (!offset || !peak || !snr || !cov) fail(B200_EINVAL, "null outputs");
        for (size_t i = 0; i < g->grids.size(); ++i)
            if (!offset[i] || !peak[i] || !snr[i] || !cov[i]) fail(B200_EINVAL, "null outputs");
        CK(cudaSetDevice(g->device));
        g->reserve(n);
        cudaStream_t user = static_cast<cudaStream_t>(stream);
        // what the step is made for: a captured graph stays valid while all of it is unchanged
        std::vector<uintptr_t> key = {uintptr_t(frames), uintptr_t(n), uintptr_t(pitch), uintptr_t(g->nt),
                                      uintptr_t(g->chunk), uintptr_t(g->costly_first), uintptr_t(g->per_grid)};
        for (size_t i = 0; i < g->grids.size(); ++i) {
            key.push_back(gross ? uintptr_t(gross[i]) : 0);
            key.push_back(gross && gross[i] ? uintptr_t(gross_mode[i]) : 0);
            for (float *const *o : {offset, peak, snr, cov}) key.push_back(uintptr_t(o[i]));
        }
        CK(cudaEventRecord(g->ev_in, user));
        CK(cudaStreamWaitEvent(g->stream, g->ev_in, 0));
        if (key != g->key) {
            CK(cudaStreamSynchronize(g->stream));   // a step in flight may still read the arguments
            g->set_args(g->make_args(frames, n, pitch, gross, gross_mode, offset, peak, snr, cov));
            if (g->use_graph) {
                cudaGraph_t graph = nullptr;
                CK(cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal));
                try {
                    g->step(frames, n, pitch);
                } catch (...) {
                    cudaStreamEndCapture(g->stream, &graph);
                    if (graph) cudaGraphDestroy(graph);
                    throw;
                }
                CK(cudaStreamEndCapture(g->stream, &graph));
                cudaGraphExecUpdateResultInfo info{};
                if (!g->exec || cudaGraphExecUpdate(g->exec, graph, &info) != cudaSuccess) {
                    cudaGetLastError();
                    if (g->exec) cudaGraphExecDestroy(g->exec);
                    g->exec = nullptr;
                    const cudaError_t e = cudaGraphInstantiate(&g->exec, graph, 0);
                    cudaGraphDestroy(graph);
                    CK(e);
                } else {
                    cudaGraphDestroy(graph);
                }
            }
            g->key = key;
        }
        if (g->use_graph)
            CK(cudaGraphLaunch(g->exec, g->stream));
        else
            g->step(frames, n, pitch);
        CK(cudaEventRecord(g->ev_out, g->stream));
        CK(cudaStreamWaitEvent(user, g->ev_out, 0));
        g->launches += 3 + g->wsizes.size();
    });
}

int b200_group_tune(b200_group *g, const uint8_t *frames, int n, int pitch, const int32_t *const *gross,
                    const int *gross_mode, void *stream, double *best_ms)
{
    return guarded_group(g, [&] {
        check_group_call(g, frames, n, pitch, gross, gross_mode);
        if (n == 0) fail(B200_EINVAL, "the autotuner needs frames");
        CK(cudaSetDevice(g->device));
        CK(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
        const size_t ng = g->grids.size();
        std::vector<DevBuf<float>> outs(ng);
        std::vector<float *> off(ng), pk(ng), sn(ng), cv(ng);
        for (size_t i = 0; i < ng; ++i) {
            const size_t P = size_t(n) * g->grids[i]->nwin;
            outs[i].alloc(7 * P);
            off[i] = outs[i].p;
            pk[i] = off[i] + 2 * P;
            sn[i] = pk[i] + P;
            cv[i] = sn[i] + P;
        }
        cudaEvent_t t0, t1;
        CK(cudaEventCreate(&t0));
        CK(cudaEventCreate(&t1));
        double best = 1e30;
        int bnt = g->nt, bchunk = g->chunk;
        bool bfirst = g->costly_first, bper = g->per_grid;
        struct Cand {
            int nt, chunk;
            bool first, per_grid;
        };
        std::vector<Cand> cands;
        for (int nt : {256, 512})
            for (int chunk : {1, 2, 4, 8})
                for (bool first : {true, false}) cands.push_back({nt, chunk, first, false});
        cands.push_back({256, 1, true, true});
        try {
            for (const Cand &c : cands) {
                g->nt = c.nt;
                g->chunk = c.chunk;
                g->costly_first = c.first;
                g->per_grid = c.per_grid;
                g->reserve(n);
                g->set_args(g->make_args(frames, n, pitch, gross, gross_mode, off.data(), pk.data(), sn.data(), cv.data()));
                g->step(frames, n, pitch);   // a warm-up
                float ms = 0.0f, total = 0.0f;
                for (int r = 0; r < 3; ++r) {   // the whole step: tables, denominators, correlation
                    CK(cudaEventRecord(t0, g->stream));
                    g->step(frames, n, pitch);
                    CK(cudaEventRecord(t1, g->stream));
                    CK(cudaEventSynchronize(t1));
                    CK(cudaEventElapsedTime(&ms, t0, t1));
                    total += ms;
                }
                if (total / 3 < best) {
                    best = total / 3;
                    bnt = c.nt;
                    bchunk = c.chunk;
                    bfirst = c.first;
                    bper = c.per_grid;
                }
            }
        } catch (...) {
            cudaEventDestroy(t0);
            cudaEventDestroy(t1);
            throw;
        }
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        CK(cudaStreamSynchronize(g->stream));
        g->nt = bnt;
        g->chunk = bchunk;
        g->costly_first = bfirst;
        g->per_grid = bper;
        g->key.clear();
        if (best_ms) *best_ms = best;
    });
}

int b200_group_config(const b200_group *g, int *threads, int *chunk, int *costly_first, int *per_grid, int *use_graph)
{
    if (!g) return B200_EINVAL;
    if (threads) *threads = g->nt;
    if (chunk) *chunk = g->chunk;
    if (costly_first) *costly_first = g->costly_first;
    if (per_grid) *per_grid = g->per_grid;
    if (use_graph) *use_graph = g->use_graph;
    return B200_OK;
}

int b200_group_set_config(b200_group *g, int threads, int chunk, int costly_first, int per_grid, int use_graph)
{
    return guarded_group(g, [&] {
        if ((threads != 256 && threads != 512) || chunk < 1 || chunk > 64)
            fail(B200_EINVAL, "threads must be 256 or 512 and chunk 1 to 64");
        g->nt = threads;
        g->chunk = chunk;
        g->costly_first = costly_first != 0;
        g->per_grid = per_grid != 0;
        g->use_graph = use_graph != 0;
        g->key.clear();
    });
}

}   // extern "C"
