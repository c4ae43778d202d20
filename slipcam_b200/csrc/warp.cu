// warp.cu -- the resampling half of python/slipcam/stabilize.py: warp (:99-106), the bilinear
// resampling of a frame onto the reference under a similarity transform, and stabilize (:109-124),
// which first blanks the burned-in text of each frame with the local mean of the pixels around it
// and also warps the text mask. The arithmetic is the reference's, step for step:
//
// * scipy.ndimage.uniform_filter(x, 31): a box mean along axis 0, rounded to float32, then along
//   axis 1, the borders reflected (half-sample). Each output is float32(window sum / size), and the
//   window sums of these values are exact in double, so summing in any order gives scipy's bits.
// * numpy's float32 mean: the pairwise sum (blocks of at most 128 values with 8 accumulators, split
//   at n / 2 rounded down to a multiple of 8) divided by n in float32. The split depends only on n;
//   the host builds the tree once; a thread sums each leaf, then a CTA per frame the tree, level by
//   level.
// * scipy.ndimage.map_coordinates(order=1, mode='constant'): a coordinate outside [0, n - 1] takes
//   cval; inside, the bilinear weights in double; the result rounded to float32.
//
// All passes are bandwidth-bound over the frames: one thread per pixel (warp, blanking) or per
// line (box sums, coalesced across neighbouring lines).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/slipcam_b200.h"

namespace {

constexpr int kLeafMax = 128;   // numpy's pairwise block size

// --------------------------------------------------------------------------------------------
// numpy's pairwise float32 sum, as a fixed tree of leaves (<= 128 values) and sums of two nodes

struct PairwisePlan {
    std::vector<int64_t> leaf_start;
    std::vector<int32_t> leaf_len;
    std::vector<int32_t> left, right;   // internal nodes in level order; children index vals[]
    std::vector<int32_t> level_off;     // internal nodes of height h: [level_off[h-1], level_off[h])
    int64_t n = 0;
};

struct NodeTmp {
    int32_t left, right, height;
};

// returns the node's index in vals[] numbering (leaves first, then internal nodes, both in the
// order they are found; internal ones renumbered by height afterwards)
int32_t plan_node(int64_t start, int64_t n, std::vector<int64_t> &ls, std::vector<int32_t> &ll,
                  std::vector<NodeTmp> &internal, std::vector<int32_t> &kind_height)
{
    if (n <= kLeafMax) {
        ls.push_back(start);
        ll.push_back(int32_t(n));
        return -int32_t(ls.size());   // leaf k as -(k + 1)
    }
    int64_t n2 = n / 2;
    n2 -= n2 % 8;
    const int32_t a = plan_node(start, n2, ls, ll, internal, kind_height);
    const int32_t b = plan_node(start + n2, n - n2, ls, ll, internal, kind_height);
    auto height = [&](int32_t id) { return id < 0 ? 0 : internal[id].height; };
    internal.push_back({a, b, 1 + std::max(height(a), height(b))});
    return int32_t(internal.size()) - 1;
}

PairwisePlan make_plan(int64_t n)
{
    PairwisePlan p;
    p.n = n;
    std::vector<NodeTmp> internal;
    std::vector<int32_t> unused;
    if (n > 0) plan_node(0, n, p.leaf_start, p.leaf_len, internal, unused);
    const int32_t L = int32_t(p.leaf_start.size());
    int H = 0;
    for (const NodeTmp &t : internal) H = std::max(H, int(t.height));
    // level order: stable by height; the root (the last node found, the only one of height H)
    // ends last
    std::vector<int32_t> order(internal.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = int32_t(i);
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return internal[a].height < internal[b].height; });
    std::vector<int32_t> pos(internal.size());
    for (size_t i = 0; i < order.size(); ++i) pos[order[i]] = int32_t(i);
    auto vid = [&](int32_t id) { return id < 0 ? -id - 1 : L + pos[id]; };
    p.left.resize(internal.size());
    p.right.resize(internal.size());
    p.level_off.assign(size_t(H) + 1, 0);
    for (size_t i = 0; i < order.size(); ++i) {
        const NodeTmp &t = internal[order[i]];
        p.left[i] = vid(t.left);
        p.right[i] = vid(t.right);
        p.level_off[t.height] = int32_t(i) + 1;
    }
    for (int h = 1; h <= H; ++h) p.level_off[h] = std::max(p.level_off[h], p.level_off[h - 1]);
    return p;
}

struct PlanDev {
    const int64_t *leaf_start;
    const int32_t *leaf_len, *left, *right, *level_off;
    int32_t leaves, internal, levels;
    int64_t n;
};

// the pairwise sum of one leaf of x (numpy's block of at most 128 values)
template <class Get>
__device__ __forceinline__ float leaf_sum(const Get &get, int64_t start, int n)
{
    if (n < 8) {
        float r = 0.0f;
        for (int i = 0; i < n; ++i) r = __fadd_rn(r, get(start + i));
        return r;
    }
    float r[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) r[j] = get(start + j);
    int i = 8;
    for (const int end = n - n % 8; i < end; i += 8)
#pragma unroll
        for (int j = 0; j < 8; ++j) r[j] = __fadd_rn(r[j], get(start + i + j));
    float res = __fadd_rn(__fadd_rn(__fadd_rn(r[0], r[1]), __fadd_rn(r[2], r[3])),
                          __fadd_rn(__fadd_rn(r[4], r[5]), __fadd_rn(r[6], r[7])));
    for (; i < n; ++i) res = __fadd_rn(res, get(start + i));
    return res;
}

constexpr int kLeafThreads = 128;
constexpr int kTreeThreads = 1024;

// numpy's pairwise sums of the leaves of frame b's values x[gather[i]] (gather may be null: x[i]),
// one thread per leaf; grid (leaves / 128, frames). vals: per frame leaves + internal floats
__global__ void __launch_bounds__(kLeafThreads) pairwise_leaves_kernel(const float *__restrict__ x, int64_t fstride,
                                                                      const int32_t *__restrict__ gather, PlanDev p,
                                                                      float *__restrict__ vals)
{
    const int l = blockIdx.x * kLeafThreads + threadIdx.x, b = blockIdx.y;
    if (l >= p.leaves) return;
    const float *xb = x + b * fstride;
    float *v = vals + size_t(b) * (p.leaves + p.internal);
    if (gather)
        v[l] = leaf_sum([&](int64_t i) { return xb[gather[i]]; }, p.leaf_start[l], p.leaf_len[l]);
    else
        v[l] = leaf_sum([&](int64_t i) { return xb[i]; }, p.leaf_start[l], p.leaf_len[l]);
}

// the tree over frame b's leaf sums, level by level, then the mean: sum / n in float32 (NaN for no
// values, as numpy). One CTA per frame.
__global__ void __launch_bounds__(kTreeThreads) pairwise_tree_kernel(PlanDev p, float *__restrict__ vals,
                                                                    float *__restrict__ mean)
{
    const int b = blockIdx.x;
    float *v = vals + size_t(b) * (p.leaves + p.internal);
    if (p.n == 0) {
        if (threadIdx.x == 0) mean[b] = NAN;
        return;
    }
    for (int h = 1; h < p.levels; ++h) {
        for (int i = p.level_off[h - 1] + threadIdx.x; i < p.level_off[h]; i += kTreeThreads)
            v[p.leaves + i] = __fadd_rn(v[p.left[i]], v[p.right[i]]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const float total = p.internal ? v[p.leaves + p.internal - 1] : v[0];
        mean[b] = __fdiv_rn(total, float(p.n));
    }
}

// numpy's float32 mean of nb frames (the leaves, then the trees) on stream st
void pairwise_mean(const float *x, int64_t fstride, const int32_t *gather, const PlanDev &p, float *vals, float *mean,
                   unsigned nb, cudaStream_t st)
{
    if (p.leaves > 0)
        pairwise_leaves_kernel<<<dim3(unsigned((p.leaves + kLeafThreads - 1) / kLeafThreads), nb), kLeafThreads, 0, st>>>(
            x, fstride, gather, p, vals);
    pairwise_tree_kernel<<<nb, kTreeThreads, 0, st>>>(p, vals, mean);
}

// --------------------------------------------------------------------------------------------
// box sums (scipy's uniform_filter, mode 'reflect', origin 0)

__device__ __forceinline__ int reflect_line(int i, int n)
{
    // half-sample symmetric extension, periodic with period 2 n (any distance from the line)
    const int period = 2 * n;
    i %= period;
    if (i < 0) i += period;
    return i < n ? i : period - 1 - i;
}

constexpr int kColSeg = 48;    // rows per thread of pass 1
constexpr int kRowTile = 32;   // pass 2: a warp's tile of 32 rows x 32 columns

// pass 1 (axis 0): the box mean over `size` rows of in(b, r, c) -> float32, where in = the frame's
// pixels where text is 0 (text null: every pixel) or, with frames null, the mask 1 - text itself.
// Integer values: the sums are exact. One thread per (column, segment of kColSeg rows, frame);
// grid (columns / 128, segments, frames), neighbouring threads on neighbouring columns.
__global__ void box_cols_kernel(const uint8_t *__restrict__ frames, int64_t fstride, int pitch,
                                const uint8_t *__restrict__ text, int h, int w, int size, float *__restrict__ out)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x, b = blockIdx.z;
    const int r0 = blockIdx.y * kColSeg, r1 = min(h, r0 + kColSeg);
    if (c >= w || r0 >= h) return;
    const uint8_t *f = frames ? frames + b * fstride : nullptr;
    auto in = [&](int r) -> int {
        const int rr = (r >= 0 && r < h) ? r : reflect_line(r, h);
        const int t = text ? text[size_t(rr) * w + c] : 0;
        return f ? (t ? 0 : int(f[int64_t(rr) * pitch + c])) : (1 - t);
    };
    const int s1 = size / 2, s2 = size - s1 - 1;
    int64_t sum = 0;
    for (int k = r0 - s1; k <= r0 + s2; ++k) sum += in(k);
    float *o = out + size_t(b) * h * w + c;
    for (int r = r0; r < r1; ++r) {
        o[size_t(r) * w] = float(double(sum) / double(size));
        sum += in(r + s2 + 1) - in(r - s1);
    }
}

// pass 2 (axis 1): the box mean over `size` columns of pass 1's float32 values (double sums,
// exact) -> float32 `local`. mode 0: out = local (the denominator table). mode 1: the blanked
// frame, out = text ? (den > 1e-3 ? local / max(den, 1e-3) : fill[b]) : the frame's pixel.
// A warp takes 32 rows x 32 columns: the rows' spans (32 + size - 1 columns, borders reflected)
// staged in shared memory by coalesced loads, each lane sliding along one row, the results
// written back a row at a time by the whole warp. Block 128 threads; grid (rows / 128,
// columns / 32, frames). Shared memory: 4 warps x 32 x (32 + size) floats + the output tiles.
__global__ void __launch_bounds__(128) box_rows_kernel(const float *__restrict__ in, int h, int w, int size, int mode,
                                                       const uint8_t *__restrict__ frames, int64_t fstride, int pitch,
                                                       const uint8_t *__restrict__ text, const float *__restrict__ den,
                                                       const float *__restrict__ fill, float *__restrict__ out)
{
    extern __shared__ float smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, b = blockIdx.z;
    const int span = kRowTile + size - 1, pitch_s = span | 1;   // odd pitch: lane i's row i is conflict-free
    float *tile = smem + warp * (kRowTile * pitch_s + kRowTile * (kRowTile + 1));
    float *res = tile + kRowTile * pitch_s;
    const int r0 = (blockIdx.x * 4 + warp) * kRowTile, c0 = blockIdx.y * kRowTile;
    if (r0 >= h) return;   // the whole warp: no barrier below is CTA-wide
    const int s1 = size / 2;
    const float *x = in + size_t(b) * h * w;
    const bool interior = c0 - s1 >= 0 && c0 - s1 + span <= w;
    for (int i = 0; i < kRowTile && r0 + i < h; ++i) {
        const float *xr = x + size_t(r0 + i) * w;
        for (int j = lane; j < span; j += 32) tile[i * pitch_s + j] = xr[interior ? c0 - s1 + j : reflect_line(c0 - s1 + j, w)];
    }
    __syncwarp();
    if (r0 + lane < h) {
        const float *row = tile + lane * pitch_s;
        double sum = 0.0;
        for (int k = 0; k < size; ++k) sum += double(row[k]);
        for (int j = 0; j < kRowTile; ++j) {
            res[lane * (kRowTile + 1) + j] = float(sum / double(size));
            if (j + 1 < kRowTile) sum += double(row[j + size]) - double(row[j]);
        }
    }
    __syncwarp();
    const int c = c0 + lane;
    if (c >= w) return;
    for (int i = 0; i < kRowTile && r0 + i < h; ++i) {
        const int r = r0 + i;
        const float local = res[i * (kRowTile + 1) + lane];
        float v;
        if (mode == 0) {
            v = local;
        } else if (text[size_t(r) * w + c]) {
            const float d = den[size_t(r) * w + c];
            v = d > 1e-3f ? __fdiv_rn(local, fmaxf(d, 1e-3f)) : fill[b];
        } else {
            v = float(frames[b * fstride + int64_t(r) * pitch + c]);
        }
        out[(size_t(b) * h + r) * w + c] = v;
    }
}

size_t box_rows_smem(int size)
{
    const int span = kRowTile + size - 1, pitch_s = span | 1;
    return size_t(4) * (kRowTile * pitch_s + kRowTile * (kRowTile + 1)) * sizeof(float);
}

// the frame as float32 (no text to blank)
__global__ void to_float_kernel(const uint8_t *__restrict__ frames, int64_t fstride, int pitch, int h, int w,
                                float *__restrict__ out)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const int b = blockIdx.y;
    if (i >= int64_t(h) * w) return;
    out[size_t(b) * h * w + i] = float(frames[b * fstride + (i / w) * pitch + i % w]);
}

// --------------------------------------------------------------------------------------------
// the warp

// stabilize.apply with every product and sum rounded on its own, as numpy evaluates it
__device__ __forceinline__ void similarity(const double *m, double x, double y, double &xo, double &yo)
{
    xo = __dadd_rn(__dsub_rn(__dadd_rn(x, m[0]), __dmul_rn(m[2], y)), __dmul_rn(m[3], x));
    yo = __dadd_rn(__dadd_rn(__dadd_rn(y, m[1]), __dmul_rn(m[2], x)), __dmul_rn(m[3], y));
}

// map_coordinates(img, [cy, cx], order=1, mode='constant', cval) at one point, float32 result
template <class Get>
__device__ __forceinline__ float bilinear(const Get &img, int h, int w, double cy, double cx, float cval)
{
    if (!(cy >= 0.0 && cy <= double(h - 1) && cx >= 0.0 && cx <= double(w - 1))) return cval;
    const double fy = floor(cy), fx = floor(cx);
    const int y0 = int(fy), x0 = int(fx), y1 = min(y0 + 1, h - 1), x1 = min(x0 + 1, w - 1);
    const double ty = __dsub_rn(cy, fy), tx = __dsub_rn(cx, fx);
    const double wy[2] = {__dsub_rn(1.0, ty), ty}, wx[2] = {__dsub_rn(1.0, tx), tx};
    double s = __dmul_rn(__dmul_rn(double(img(y0, x0)), wy[0]), wx[0]);
    s = __dadd_rn(s, __dmul_rn(__dmul_rn(double(img(y0, x1)), wy[0]), wx[1]));
    s = __dadd_rn(s, __dmul_rn(__dmul_rn(double(img(y1, x0)), wy[1]), wx[0]));
    s = __dadd_rn(s, __dmul_rn(__dmul_rn(double(img(y1, x1)), wy[1]), wx[1]));
    return __double2float_rn(s);
}

// frame b of the batch: out = uint8(clip(warp(src, params[b], fill[b]), 0, 255)) and, when text is
// given, the warped text mask above 0.5 OR-ed into the union (stores of 1 only). One thread per
// output pixel; grid (pixels / 256, frames).
__global__ void warp_kernel(const float *__restrict__ src, int h, int w, const double *__restrict__ params,
                            const float *__restrict__ fill, float fill_value, const uint8_t *__restrict__ text,
                            uint8_t *__restrict__ out, int64_t ostride, float *__restrict__ fout,
                            uint8_t *__restrict__ union_mask)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const int b = blockIdx.y;
    if (i >= int64_t(h) * w) return;
    const int r = int(i / w), c = int(i % w);
    const double hw = w / 2.0, hh = h / 2.0;
    double sx, sy;
    similarity(params + 4 * b, __dsub_rn(double(c), hw), __dsub_rn(double(r), hh), sx, sy);
    const double cy = __dadd_rn(sy, hh), cx = __dadd_rn(sx, hw);
    const float *s = src + size_t(b) * h * w;
    const float v = bilinear([&](int y, int x) { return s[size_t(y) * w + x]; }, h, w, cy, cx, fill ? fill[b] : fill_value);
    if (fout) fout[size_t(b) * h * w + i] = v;
    if (out) out[b * ostride + i] = uint8_t(fminf(fmaxf(v, 0.0f), 255.0f));
    if (text && union_mask) {
        const float t = bilinear([&](int y, int x) { return float(text[size_t(y) * w + x]); }, h, w, cy, cx, 0.0f);
        if (t > 0.5f) union_mask[i] = 1;
    }
}

}   // namespace

// --------------------------------------------------------------------------------------------
// the context

struct b200_stab {
    int h = 0, w = 0, size = 31, device = 0, batch = 8;
    bool any_text = false;
    std::string err;
    uint8_t *d_text = nullptr;     // h x w, 0 / 1
    float *d_den = nullptr;        // h x w: uniform_filter(1 - text)
    int32_t *d_keep_idx = nullptr; // the raster indices of the pixels without text
    PlanDev plan_keep{}, plan_all{};
    void *d_plans = nullptr;       // the two plans' arrays
    float *d_work = nullptr;       // batch x h x w: pass 1
    float *d_blank = nullptr;      // batch x h x w: the blanked frames
    float *d_vals = nullptr;       // batch x max(tree nodes)
    float *d_means = nullptr;      // 2 x batch: the mean without text, the blanked frame's mean
    ~b200_stab()
    {
        for (void *p : {(void *)d_text, (void *)d_den, (void *)d_keep_idx, d_plans, (void *)d_work, (void *)d_blank,
                        (void *)d_vals, (void *)d_means})
            if (p) cudaFree(p);
    }
};

namespace {

struct StabFailure {
    int code;
    std::string msg;
};

void sck(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) throw StabFailure{B200_ERUNTIME, std::string(what) + ": " + cudaGetErrorString(e)};
}

// the plans' arrays in one device allocation
size_t plan_bytes(const PairwisePlan &p)
{
    return p.leaf_start.size() * 8 + (p.leaf_len.size() + p.left.size() + p.right.size() + p.level_off.size()) * 4 + 64;
}

PlanDev upload_plan(const PairwisePlan &p, char *&dst)
{
    PlanDev d{};
    auto put = [&](const void *src, size_t bytes) {
        char *at = dst;
        if (bytes) sck(cudaMemcpy(at, src, bytes, cudaMemcpyHostToDevice), "cudaMemcpy");
        dst += (bytes + 15) & ~size_t(15);
        return at;
    };
    d.leaf_start = reinterpret_cast<const int64_t *>(put(p.leaf_start.data(), p.leaf_start.size() * 8));
    d.leaf_len = reinterpret_cast<const int32_t *>(put(p.leaf_len.data(), p.leaf_len.size() * 4));
    d.left = reinterpret_cast<const int32_t *>(put(p.left.data(), p.left.size() * 4));
    d.right = reinterpret_cast<const int32_t *>(put(p.right.data(), p.right.size() * 4));
    d.level_off = reinterpret_cast<const int32_t *>(put(p.level_off.data(), p.level_off.size() * 4));
    d.leaves = int32_t(p.leaf_start.size());
    d.internal = int32_t(p.left.size());
    d.levels = int32_t(p.level_off.size());
    d.n = p.n;
    return d;
}

}   // namespace

extern "C" {

const char *b200_stab_last_error(const b200_stab *s) { return s ? s->err.c_str() : ""; }

int b200_stab_create(int height, int width, const uint8_t *text, int size, int device, b200_stab **out)
{
    if (!out) return B200_EINVAL;
    *out = nullptr;
    if (height < 1 || width < 1 || size < 1 || !text || int64_t(height) * width > (int64_t(1) << 31) - 1)
        return B200_EINVAL;
    b200_stab *s = new (std::nothrow) b200_stab;
    if (!s) return B200_ERUNTIME;
    try {
        s->h = height;
        s->w = width;
        s->size = size;
        s->device = device;
        sck(cudaSetDevice(device), "cudaSetDevice");
        const size_t px = size_t(height) * width;
        std::vector<uint8_t> t(px);
        std::vector<int32_t> keep;
        keep.reserve(px);
        for (size_t i = 0; i < px; ++i) {
            t[i] = text[i] ? 1 : 0;
            if (!t[i]) keep.push_back(int32_t(i));
            s->any_text = s->any_text || t[i];
        }
        const PairwisePlan pk = make_plan(int64_t(keep.size())), pa = make_plan(int64_t(px));
        sck(cudaMalloc(&s->d_text, px), "cudaMalloc");
        sck(cudaMemcpy(s->d_text, t.data(), px, cudaMemcpyHostToDevice), "cudaMemcpy");
        sck(cudaMalloc(&s->d_keep_idx, std::max<size_t>(keep.size(), 1) * 4), "cudaMalloc");
        if (!keep.empty())
            sck(cudaMemcpy(s->d_keep_idx, keep.data(), keep.size() * 4, cudaMemcpyHostToDevice), "cudaMemcpy");
        sck(cudaMalloc(&s->d_plans, plan_bytes(pk) + plan_bytes(pa) + 256), "cudaMalloc");
        char *dst = static_cast<char *>(s->d_plans);
        s->plan_keep = upload_plan(pk, dst);
        s->plan_all = upload_plan(pa, dst);
        // frames per launch: about 64 MB of float32 work per buffer
        s->batch = int(std::clamp<int64_t>(int64_t(16) * 1024 * 1024 / int64_t(px), 1, 32));
        const size_t nodes = size_t(std::max(pk.leaf_start.size() + pk.left.size(), pa.leaf_start.size() + pa.left.size()));
        sck(cudaMalloc(&s->d_den, px * 4), "cudaMalloc");
        sck(cudaMalloc(&s->d_work, size_t(s->batch) * px * 4), "cudaMalloc");
        sck(cudaMalloc(&s->d_blank, size_t(s->batch) * px * 4), "cudaMalloc");
        sck(cudaMalloc(&s->d_vals, size_t(s->batch) * std::max<size_t>(nodes, 1) * 4), "cudaMalloc");
        sck(cudaMalloc(&s->d_means, size_t(2) * s->batch * 4), "cudaMalloc");
        // den = uniform_filter(1 - text, size): the mask itself through the two passes
        if (box_rows_smem(size) > size_t(200) * 1024) throw StabFailure{B200_EINVAL, "framecor: the box is too large"};
        sck(cudaFuncSetAttribute(box_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(box_rows_smem(size))),
            "cudaFuncSetAttribute");
        box_cols_kernel<<<dim3(unsigned((width + 127) / 128), unsigned((height + kColSeg - 1) / kColSeg), 1), 128>>>(
            nullptr, 0, width, s->d_text, height, width, size, s->d_work);
        box_rows_kernel<<<dim3(unsigned((height + 127) / 128), unsigned((width + kRowTile - 1) / kRowTile), 1), 128,
                          box_rows_smem(size)>>>(s->d_work, height, width, size, 0, nullptr, 0, 0, nullptr, nullptr, nullptr,
                                                 s->d_den);
        sck(cudaGetLastError(), "launch");
        sck(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
    } catch (const StabFailure &f) {
        delete s;
        return f.code;
    } catch (const std::bad_alloc &) {
        delete s;
        return B200_ERUNTIME;
    }
    *out = s;
    return B200_OK;
}

int b200_stab_destroy(b200_stab *s)
{
    delete s;
    return B200_OK;
}

int b200_stab_frames_device(b200_stab *s, const uint8_t *frames, int n, int pitch, const double *params,
                            uint8_t *out, uint8_t *union_mask, void *stream)
{
    if (!s) return B200_EINVAL;
    try {
        if (n < 0 || (n && (!frames || !params || !out || pitch < s->w)))
            throw StabFailure{B200_EINVAL, "framecor: null input or output, or a pitch below the width"};
        if (n == 0) return B200_OK;
        sck(cudaSetDevice(s->device), "cudaSetDevice");
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        const int h = s->h, w = s->w;
        const int64_t px = int64_t(h) * w, fstride = int64_t(pitch) * h;
        const unsigned pblocks = unsigned((px + 255) / 256);
        float *mean_keep = s->d_means, *mean_blank = s->d_means + s->batch;
        for (int f0 = 0; f0 < n; f0 += s->batch) {
            const unsigned nb = unsigned(std::min(s->batch, n - f0));
            const uint8_t *fr = frames + f0 * fstride;
            if (s->any_text) {
                // the text blanked with the local mean of the pixels around it (stabilize.py:118-121):
                // the mean of the pixels without text, from the float32 frame
                to_float_kernel<<<dim3(pblocks, nb), 256, 0, st>>>(fr, fstride, pitch, h, w, s->d_blank);
                pairwise_mean(s->d_blank, px, s->d_keep_idx, s->plan_keep, s->d_vals, mean_keep, nb, st);
                box_cols_kernel<<<dim3(unsigned((w + 127) / 128), unsigned((h + kColSeg - 1) / kColSeg), nb), 128, 0, st>>>(
                    fr, fstride, pitch, s->d_text, h, w, s->size, s->d_work);
                box_rows_kernel<<<dim3(unsigned((h + 127) / 128), unsigned((w + kRowTile - 1) / kRowTile), nb), 128,
                                  box_rows_smem(s->size), st>>>(s->d_work, h, w, s->size, 1, fr, fstride, pitch, s->d_text,
                                                                s->d_den, mean_keep, s->d_blank);
            } else {
                to_float_kernel<<<dim3(pblocks, nb), 256, 0, st>>>(fr, fstride, pitch, h, w, s->d_blank);
            }
            // the fill: the mean of the blanked frame (warp's default, stabilize.py:105)
            pairwise_mean(s->d_blank, px, nullptr, s->plan_all, s->d_vals, mean_blank, nb, st);
            warp_kernel<<<dim3(pblocks, nb), 256, 0, st>>>(s->d_blank, h, w, params + 4 * size_t(f0), mean_blank, 0.0f,
                                                          union_mask ? s->d_text : nullptr, out + f0 * px, px, nullptr,
                                                          union_mask);
            sck(cudaGetLastError(), "launch");
        }
    } catch (const StabFailure &f) {
        s->err = f.msg;
        return f.code;
    }
    return B200_OK;
}

int b200_warp_f32_device(const float *frame, int height, int width, const double *params, float fill, float *out,
                         void *stream)
{
    if (!frame || !params || !out || height < 1 || width < 1 || int64_t(height) * width > (int64_t(1) << 31) - 1)
        return B200_EINVAL;
    const int64_t px = int64_t(height) * width;
    warp_kernel<<<dim3(unsigned((px + 255) / 256), 1), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        frame, height, width, params, nullptr, fill, nullptr, nullptr, 0, out, nullptr);
    return cudaGetLastError() == cudaSuccess ? B200_OK : B200_ERUNTIME;
}

}   // extern "C"
