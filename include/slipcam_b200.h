/*
 * slipcam_b200.h -- the C ABI of the b200 backend of slipcam's framecor Correlator.
 *
 * The reference exposes framecor as a C++ interface (slipcam cxx/framecor.h) bound to Python by
 * pybind11 (cxx/bindings.cpp). This library is the same correlator on a B200, behind plain C:
 * plain pointers and sizes, an opaque handle, int status codes. A binding (the reference's
 * bindings.cpp, or the Python package slipcam_b200.framecor through ctypes) turns the codes into
 * the reference's exceptions:
 *
 *   B200_OK        0   success
 *   B200_EINVAL    1   std::invalid_argument -> ValueError   (cxx/common.cpp:17, bindings.cpp:44-79)
 *   B200_ERUNTIME  2   std::runtime_error    -> RuntimeError (cxx/cuda.cu:28-38, bindings.cpp:59)
 *   B200_ETIMEOUT  3   a bounded device wait gave up         -> RuntimeError
 *
 * Messages start with "framecor: " as the reference's do; b200_last_error gives the last one.
 * One handle is not re-entrant (like one reference Correlator); distinct handles are independent.
 * Host-pointer calls are synchronous: they return when the outputs are in the caller's arrays.
 *
 * Outputs, per (frame, window) pair q = frame * windows + window, windows row-major (down, then
 * across), exactly the reference layout (cxx/framecor.h:38-43):
 *   offset[2q], offset[2q+1]  (down, across) motion of the frame, NaN if not valid
 *   peak[q]                   normalized correlation at the peak
 *   snr[q]                    squared peak over the mean squared surface around it
 *   cov[3q .. 3q+2]           covariance of the offsets (down, across, cross)
 */
#ifndef SLIPCAM_B200_H
#define SLIPCAM_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define B200_API __attribute__((visibility("default")))
#else
#define B200_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define B200_OK 0
#define B200_EINVAL 1
#define B200_ERUNTIME 2
#define B200_ETIMEOUT 3

/* gross offsets: none, per frame (n x 2), per window (n x windows x 2); int32 (down, across) */
#define B200_GROSS_NONE 0
#define B200_GROSS_FRAME 1
#define B200_GROSS_WINDOW 2

/* the arithmetic of the transforms */
#define B200_FORM_AUTO 0   /* the library's choice, and the default: B200_FORM_TC for windows above 32 px
                              where it holds the geometry (FFT size up to 160, search up to 63 px),
                              else B200_FORM_FFT32 */
#define B200_FORM_FFT32 1  /* FP32 FFTs on the CUDA cores */
#define B200_FORM_TC 2     /* DFT-matrix GEMMs on the tensor cores, FP16 operands, FP32 accumulation */
#define B200_FORM_I8 3     /* direct correlation on the tensor cores in exact integers (uint8 x uint8,
                              int32 accumulation), normalized after: windows up to 181 px, search
                              windows (window + 2 search) up to 256 px */

/* The frames, the grid of reference windows and the correlation parameters.
 * Replaces framecor::Params (cxx/framecor.h:22-35); same fields, same defaults in the binding
 * (window 64, search 48, stat_size 21, batch 4096). batch is a hint here: the library picks its
 * own number of frames per launch. */
typedef struct b200_params {
    int height, width;      /* frame size, pixels */
    int window;             /* W, the size of the square reference windows */
    int search;             /* R, the half search range: shifts -R..R */
    int stat_size;          /* the size of the surface patch of the SNR */
    int batch;              /* hint (the reference's FFT batch) */
    const int32_t *down;    /* ny first rows of the windows */
    int ny;
    const int32_t *across;  /* nx first columns of the windows */
    int nx;
} b200_params;

typedef struct b200_handle b200_handle;

/* Validate the parameters (cxx/common.cpp:15-28 checkParams, the same messages), pick the device
 * and allocate everything. Replaces framecor::makeCuda (cxx/framecor.h:65, cxx/cuda.cu:389-393)
 * as chosen by bindings.cpp:38-44. On failure *out is NULL and b200_last_error(NULL) says why. */
B200_API int b200_create(const b200_params *p, int device, b200_handle **out);

/* Free the handle and its device memory (the Correlator's destructor, cxx/framecor.h:48). */
B200_API int b200_destroy(b200_handle *h);

/* The last error message of a handle, or of the calling thread's last b200_create if h is NULL. */
B200_API const char *b200_last_error(const b200_handle *h);

/* Set the reference frame, height x width uint8 in host memory, row-major: the zero-mean
 * reference windows, their norms and their spectra, kept resident on the device.
 * Replaces Correlator::setReference (cxx/framecor.h:50; bindings.cpp:47-55). */
B200_API int b200_set_reference(b200_handle *h, const uint8_t *frame);

/* Correlate n frames (n x height x width uint8, host memory) with the reference frame; gross:
 * NULL (gross_mode B200_GROSS_NONE), n x 2 (B200_GROSS_FRAME) or n x windows x 2
 * (B200_GROSS_WINDOW) int32 in host memory; outputs in host memory, n x windows (x 2, x 3).
 * n = 0 is a no-op. B200_ERUNTIME before b200_set_reference.
 * Replaces Correlator::correlate (cxx/framecor.h:53-54) with the gross handling of
 * bindings.cpp:64-80 (a per-frame gross gives results identical to the same gross per window). */
B200_API int b200_correlate(b200_handle *h, const uint8_t *frames, int n, const int32_t *gross,
                   int gross_mode, float *offset, float *peak, float *snr, float *cov);

/* The same two calls on device memory, stream-ordered on `stream` (a cudaStream_t; NULL for the
 * legacy default stream), without host synchronization. frame rows are `pitch` bytes apart,
 * frames pitch * height bytes apart. No counterpart in the reference (its CUDA backend copies
 * from host memory, cxx/cuda.cu:323-358); for inputs already in device memory. */
B200_API int b200_set_reference_device(b200_handle *h, const uint8_t *frame, int pitch, void *stream);
B200_API int b200_correlate_device(b200_handle *h, const uint8_t *frames, int n, int pitch,
                          const int32_t *gross, int gross_mode, float *offset, float *peak,
                          float *snr, float *cov, void *stream);

/* As b200_correlate_device, also writing each pair's normalized surface (2R+1) x (2R+1) float32
 * to surface[q * (2R+1)^2 ...] (zeros for invalid pairs). For tests: the surface is the
 * reference's normalized buffer of cxx/cpu.cpp:146-160. */
B200_API int b200_correlate_device_surfaces(b200_handle *h, const uint8_t *frames, int n, int pitch,
                                   const int32_t *gross, int gross_mode, float *offset, float *peak,
                                   float *snr, float *cov, float *surface, void *stream);

/* As b200_correlate_device, for callers that cannot allocate device memory when they
 * correlate: a capture loop that must never stall on cudaMalloc's implicit synchronization, or a
 * host that owns all device memory through its own arena. No counterpart in the reference.
 * The per-frame tables live in one static 32 MiB device array (enough for one 1920 x 1080 frame;
 * frames go as many per launch as fit), held by every device that loads the library until the
 * process exits; nothing is allocated. Larger frames are rejected with B200_EINVAL. The first call
 * on a device looks the array's address up (cudaGetSymbolAddress): make it before any stream
 * capture. All calls on a device share the array: calls that overlap on the GPU race.
 * It always runs the FP32 FFT form, whatever b200_set_form chose for the handle: the tensor-core
 * and exact-integer forms keep per-launch buffers (spectra, peak records, the refinement queue)
 * that this entry point has no room for. */
B200_API int b200_correlate_device_noalloc(b200_handle *h, const uint8_t *frames, int n, int pitch,
                                           const int32_t *gross, int gross_mode, float *offset,
                                           float *peak, float *snr, float *cov, void *stream);

/* ---- Several window grids of one video in one persistent launch (window sizes, search ranges
 * and grids may all differ). No counterpart in the reference, which correlates one grid per
 * Correlator (cxx/framecor.h:46-56); a group of handles created by b200_create (same frame size
 * and device, each with its reference set) is correlated together: the frames' summed-area
 * tables once, one variance-denominator table per window size, then one persistent launch of the
 * FP32 FFT correlation over every grid's (window, frame) pairs, scheduled dynamically (the
 * costliest grid first by default). The step is captured in a CUDA graph on the group's own
 * stream and replayed while the caller's pointers and sizes stay the same.
 * The handles stay owned by the caller and must outlive the group. Up to 4 grids. */
typedef struct b200_group b200_group;
B200_API int b200_group_create(b200_handle *const *grids, int count, b200_group **out);
B200_API int b200_group_destroy(b200_group *g);
B200_API const char *b200_group_last_error(const b200_group *g);

/* n frames (device memory, rows `pitch` bytes apart) through every grid: per grid i, gross[i] /
 * gross_mode[i] as for b200_correlate_device (gross may be NULL: no gross for any grid) and its
 * outputs offset[i], peak[i], snr[i], cov[i] (device memory). Stream-ordered on `stream`. */
B200_API int b200_group_correlate_device(b200_group *g, const uint8_t *frames, int n, int pitch,
                                         const int32_t *const *gross, const int *gross_mode,
                                         float *const *offset, float *const *peak, float *const *snr,
                                         float *const *cov, void *stream);

/* The autotuner: times the whole step on these frames for every candidate of the persistent
 * launch -- threads per CTA (256, 512), (window, frame) pairs per work item (1, 2, 4, 8), grid
 * order (costliest first or as given) -- and for the per-grid mode (each grid's own kernel, in
 * the same graph), keeps the fastest and returns its time (ms per step). Synchronous; allocates
 * its own temporary outputs. */
B200_API int b200_group_tune(b200_group *g, const uint8_t *frames, int n, int pitch,
                             const int32_t *const *gross, const int *gross_mode, void *stream,
                             double *best_ms);

/* The launch configuration (threads per CTA, pairs per work item, costliest grid first, per-grid
 * kernels instead of the persistent launch, CUDA graph replay), read or set. */
B200_API int b200_group_config(const b200_group *g, int *threads, int *chunk, int *costly_first, int *per_grid,
                               int *use_graph);
B200_API int b200_group_set_config(b200_group *g, int threads, int chunk, int costly_first, int per_grid,
                                   int use_graph);

/* auto_slip.periodicity (python/slipcam/auto_slip.py:105-129) for every window of the handle's
 * grid: surface holds the normalized surfaces of the reference frame correlated with itself
 * (b200_correlate_device_surfaces with the reference as the one frame), n_windows x (2R+1)^2; out
 * (n_windows floats, device memory) receives the largest 5 x 5 local maximum outside the
 * (2 exclude + 1)^2 box around zero shift, 1 for a flat window, 0 if no peak is left. */
B200_API int b200_periodicity_device(b200_handle *h, const float *surface, int exclude, float *out, void *stream);

/* ---- The coarse similarity tracking of stabilize (python/slipcam/stabilize.py:22-96), on device
 * memory, stream-ordered on `stream`. One frame is: b200_correlate_device_surfaces of the frame
 * with the handle of the grid of templates (window, search as in coarse_track; gross per window),
 * b200_ncc_peaks_device on its surfaces, then b200_coarse_fit_device, which also writes the gross
 * offsets of the next frame: the frames follow one another without a host round trip.
 *
 * b200_ncc_peaks_device: the peak of ncc_peak (stabilize.py:22-44) in each of n surfaces of M x M
 * floats: out (n x 3 doubles) receives (dy, dx) of the largest value relative to the surface
 * centre, refined by a parabola per axis, and the value. */
B200_API int b200_ncc_peaks_device(const float *surface, int n, int M, double *out, void *stream);

/* The most windows of one grid of b200_coarse_fit_device */
#define B200_COARSE_MAX_WINDOWS 2048

/* The rest of one frame of coarse_track (stabilize.py:80-95) with slip_series.fit_camera
 * (python/slipcam/slip_series.py:49-72), for the grid of ny x nx windows centred at (yc[i], xc[j])
 * in frames of height x width: peaks (ny nx x 3, from b200_ncc_peaks_device), gross (ny nx x 2
 * int32, the frame's gross offsets: the rounded predicted centres minus the grid's; overwritten
 * with the next frame's), keep (ny nx bytes: the window is used). prev (4 doubles): the transform
 * (p, q, a, s) the frame was predicted from, replaced by the frame's when it has a fit. params
 * (4 doubles) receives the frame's transform and used (1 int32) the number of windows of its fit
 * (0 when there is none: params = prev). Zero prev and gross to start a pass from the reference. */
B200_API int b200_coarse_fit_device(const double *peaks, int32_t *gross, const uint8_t *keep, const int32_t *yc,
                                    const int32_t *xc, int ny, int nx, int height, int width, int window,
                                    int search, double min_peak, double *prev, double *params, int32_t *used,
                                    void *stream);

/* coarse_track's frame loop (stabilize.py:76-95) on the handle h of the grid of templates
 * (created with the grid's first rows and columns, window and search as coarse_track places them;
 * the window even; its reference frame set): n frames (device memory, rows `pitch` bytes apart,
 * frames pitch * height bytes apart) in the order they are tracked, each searched around the
 * positions predicted by the previous one, its transform written to params (n x 4 doubles) and the
 * windows of its fit to used (n int32). keep (windows bytes): the templates in use. gross
 * (windows x 2 int32) and prev (4 doubles) carry the prediction from call to call; reset != 0 zeroes
 * them first (the start of a pass from the reference). Per group of frames the tables in one batch
 * (on a side stream, a group ahead), then per frame two launches: the FP32 correlation with the
 * peaks (whatever the handle's form) and the fit. The chain runs on the handle's own stream, ordered
 * after the work already on `stream` and before any work put there later; the reference spectra
 * stay in L2 there (an access-policy window; the first call raises the context's persisting-L2
 * limit to their size). The handle keeps one frame's peaks and outputs (allocated by the first
 * call). */
B200_API int b200_coarse_track_device(b200_handle *h, const uint8_t *frames, int n, int pitch, const uint8_t *keep,
                                      double min_peak, int reset, int32_t *gross, double *prev, double *params,
                                      int32_t *used, void *stream);

/* ---- The resampling of stabilize (python/slipcam/stabilize.py:99-124): frames warped onto the
 * reference under their similarity transforms, the burned-in text blanked first, the text mask
 * warped too. The arithmetic is the reference's: scipy.ndimage.uniform_filter's box means (axis 0
 * then axis 1, float32 between the passes, borders reflected), numpy's float32 mean (its pairwise
 * summation tree), map_coordinates' bilinear interpolation (order 1, mode 'constant', a coordinate
 * outside [0, n - 1] taking the fill).
 *
 * b200_stab_create: a context for frames of height x width with the text mask `text` (host memory,
 * height x width bytes, nonzero = text) and the blanking box of size x size pixels (31 in the
 * reference): the mask, its box mean and the summation plans on `device`. */
typedef struct b200_stab b200_stab;
B200_API int b200_stab_create(int height, int width, const uint8_t *text, int size, int device, b200_stab **out);
B200_API int b200_stab_destroy(b200_stab *s);
B200_API const char *b200_stab_last_error(const b200_stab *s);

/* stabilize's frame loop (stabilize.py:117-123) on n device frames (uint8, rows `pitch` bytes apart,
 * frames pitch * height apart) with their transforms params (device, n x 4 doubles p, q, a, s):
 * out (device, n x height x width bytes) = uint8(clip(warp(blanked frame, params[k]), 0, 255)),
 * the fill the blanked frame's mean; union_mask (device, height x width bytes; may be NULL) gets 1
 * where a frame's warped text mask exceeds 0.5 (the caller zeroes it first). Stream-ordered. */
B200_API int b200_stab_frames_device(b200_stab *s, const uint8_t *frames, int n, int pitch, const double *params,
                                     uint8_t *out, uint8_t *union_mask, void *stream);

/* stabilize.warp (stabilize.py:99-106) of one float32 frame (device, height x width) with the
 * transform params (device, 4 doubles) and the fill value: out (device, float32). */
B200_API int b200_warp_f32_device(const float *frame, int height, int width, const double *params, float fill,
                                  float *out, void *stream);

/* ---- The frame scans of auto_slip (python/slipcam/auto_slip.py:56-94), on device memory. Frames
 * are uint8, rows `pitch` bytes apart, frames pitch * height bytes apart.
 * b200_frame_diff_device: out[k] = the mean |frames[k + 1] - frames[k]| over the pixels, k < n - 1
 * (frame_differences, auto_slip.py:56-63; the sums exact); sums: n - 1 caller-owned uint64. */
B200_API int b200_frame_diff_device(const uint8_t *frames, int n, int height, int width, int pitch, float *out,
                                    uint64_t *sums, void *stream);
/* out (height x width float32): per pixel, the median over nchunks consecutive chunks of `chunk`
 * frames of the population standard deviation within a chunk (text_mask, auto_slip.py:87-90). */
B200_API int b200_chunk_std_median_device(const uint8_t *frames, int nchunks, int chunk, int height, int width,
                                          int pitch, float *out, void *stream);
/* out (height x width float32): hypot of the two Sobel derivatives of a frame, borders reflected
 * (scipy.ndimage.sobel, auto_slip.py:91). */
B200_API int b200_sobel_device(const uint8_t *frame, int height, int width, int pitch, float *out, void *stream);
/* *out (device float32) = numpy.percentile(x[0 .. n), q) of n float32 values in device memory,
 * method 'linear', computed as numpy does for float32 data (the virtual index (n - 1) * (q / 100),
 * its weight and the interpolation in float32); used for the text mask's edge threshold
 * (auto_slip.py:92). q in [0, 100], 1 <= n < 2^32; scratch: B200_PERCENTILE_SCRATCH bytes of
 * device memory. Stream-ordered, no host synchronisation. */
#define B200_PERCENTILE_SCRATCH 16640
B200_API int b200_percentile_f32_device(const float *x, int64_t n, double q, float *out, void *scratch, void *stream);
/* The text mask from the edge magnitude and the temporal deviation (auto_slip.py:92-94): edge above
 * numpy.percentile(edge, edge_percentile) and sd < max_std, `dilate` steps of the 3 x 3 cross
 * dilation, then the holes (background not 4-connected to the border) filled. mask: height x width
 * bytes (0 / 1); scratch: b200_text_mask_scratch_bytes(height, width) bytes of device memory.
 * Stream-ordered, no host synchronisation. Widths up to 28,000 pixels. */
B200_API size_t b200_text_mask_scratch_bytes(int height, int width);
B200_API int b200_text_mask_device(const float *edge, const float *sd, int height, int width, double edge_percentile,
                                   float max_std, int dilate, uint8_t *mask, void *scratch, size_t scratch_bytes,
                                   void *stream);

/* ---- The differentiable path: float frames, a continuous shift per pair, and the adjoints.
 * No counterpart in the reference (its backends take uint8 frames and give no derivatives); the
 * math follows the same correlation (cxx/cpu.cpp:115-160, cxx/surface.h:30-146) and is stated in
 * slipcam_b200/csrc/diff.h. All pointers are device memory, stream-ordered on `stream`.
 *
 * b200_set_reference_f32_device: the reference windows and spectra from a float32 frame (rows
 * `pitch` floats apart), as b200_set_reference_device does from a uint8 frame. */
B200_API int b200_set_reference_f32_device(b200_handle *h, const float *frame, int pitch, void *stream);

/* The forward pass over n float32 frames (rows `pitch` floats apart, frames pitch * height
 * floats apart). shift: NULL or n x nwin x 2 floats (ty, tx), a continuous shift of each pair's
 * search window, sampled with Keys' six-point cubic convolution (the edge pixel repeats beyond
 * the frame); a pair is invalid as in the reference, at the floored position of its shifted
 * window (cxx/surface.h:39-45). Writes chips (n x nwin x L x L),
 * stats (n x nwin x M x M x 2: the box mean and 1 / sqrt(n var)), surface (n x nwin x M x M),
 * peak_at (n x nwin: u M + v, -1 if invalid) and the reference's four outputs (the offsets
 * without the shift: the caller adds it). L = window + 2 search, M = 2 search + 1. */
B200_API int b200_diff_forward(b200_handle *h, const float *frames, int n, int pitch, const int32_t *gross,
                               int gross_mode, const float *shift, float *chips, float *stats, float *surface,
                               int *peak_at, float *offset, float *peak, float *snr, float *cov, void *stream);

/* The backward pass: from g_surface (n x nwin x M x M) and the forward's chips, stats and
 * surface, the chip cotangents g_chips (n x nwin x L x L, written), the frame cotangents g_frames
 * (n x height x pitch floats, accumulated into: zero it first; NULL to skip) and the shift
 * cotangents g_shift (n x nwin x 2, written; NULL to skip). */
B200_API int b200_diff_backward(b200_handle *h, const float *frames, int n, int pitch, const int32_t *gross,
                                int gross_mode, const float *shift, const float *chips, const float *stats,
                                const float *surface, const float *g_surface, float *g_chips, float *g_frames,
                                float *g_shift, void *stream);

/* The surface cotangent of the sub-pixel offsets: g_surface (n x nwin x M x M, zeroed here) from
 * g_offset (n x nwin x 2) through the branch of the 3 x 3 fit each pair's peak took. */
B200_API int b200_offset_adjoint(b200_handle *h, int n, const float *surface, const int *peak_at,
                                 const float *g_offset, float *g_surface, void *stream);

/* The summed-area tables of n frames on the device (cxx/cpu.cpp:24-42, cxx/cuda.cu:72-110):
 * sat (uint32, exact modulo 2^32) and sat2 (int64), each n x (height + 1) x (width + 1). */
B200_API int b200_sat_device(const uint8_t *frames, int n, int height, int width, int pitch, uint32_t *sat,
                    int64_t *sat2, void *stream);

/* A check of the tensor-core path: D (128 x N, float32) = A (128 x K) x B^T (B is N x K), both
 * float16 row-major device arrays, computed by one CTA with tcgen05.mma from operands staged in
 * shared memory K-major or MN-major (a_mn, b_mn), B negated if neg_b; N, K multiples of 16 up to
 * 256. Synchronous. B200_ETIMEOUT if the MMA completion wait gave up. No reference counterpart. */
B200_API int b200_tc_selftest(const void *A, const void *B, float *D, int N, int K, int a_mn, int b_mn,
                              int neg_b, void *stream);

/* A check of the exact form's tensor-core path: D (128 x N, int32) = A (128 x K) x X[i .. i + N - 1]^T,
 * uint8 row-major device arrays (X has `rows` rows), computed by one CTA with tcgen05.mma kind::i8:
 * A written to tensor memory (or, a_smem != 0, staged in shared memory), X staged in shared memory as
 * the exact form holds a search window (the operand started at row i). N a multiple of 16 up to 256,
 * K a multiple of 32 up to 256. Synchronous. B200_ETIMEOUT if the MMA completion wait gave up. No
 * reference counterpart. */
B200_API int b200_tc_i8_selftest(const uint8_t *A, const uint8_t *X, int32_t *D, int N, int K, int rows, int i,
                                 int a_smem, void *stream);

/* The arithmetic of the transforms, B200_FORM_*; B200_EINVAL for an unknown or unbuilt form. */
B200_API int b200_set_form(b200_handle *h, int form);

/* The device status of a handle's work: waits for `stream` (the caller's, as given to the device
 * entry points; NULL for the legacy default stream) and the handle's own stream, then *status = 0,
 * or 3 if a bounded wait inside a tensor-core kernel gave up since the last query (those outputs
 * are not valid); the flag is cleared. The host entry point b200_correlate checks it itself and
 * returns B200_ETIMEOUT; callers of the device entry points, which do not synchronize, call this
 * when they need to know. The reference has no device waits (cxx/cuda.cu:28-40 checks every CUDA
 * call's status instead). */
B200_API int b200_status(b200_handle *h, void *stream, int *status);

/* For tests of the error paths, with no GPU fault: the nth device or page-locked allocation from
 * now fails as an out-of-memory would (B200_ERUNTIME, "framecor: cudaMalloc: out of memory
 * (injected)"); 0 disables. No counterpart in the reference. */
B200_API int b200_inject_alloc_failure(int nth);

/* n bytes host memory -> host memory with streaming (non-temporal) stores where dst allows them:
 * the copy the library stages pageable frames into page-locked buffers with, for callers that stage
 * frames themselves (the scans and stabilize host paths). Touches no GPU. B200_EINVAL for a null
 * pointer with n > 0. No reference counterpart. */
B200_API int b200_host_copy(void *dst, const void *src, size_t n);

/* A check of the bounded waits of the tensor-core kernels, with nothing in flight: one thread waits
 * on an mbarrier that nothing arrives at, with an iteration bound of `polls` and then a clock bound
 * of limit_ms (at most 1000). B200_ETIMEOUT when both waits gave up, as they must; B200_ERUNTIME
 * otherwise. The context stays usable. Synchronous on `stream`. No counterpart in the reference. */
B200_API int b200_wait_selftest(unsigned polls, double limit_ms, void *stream);

/* The grid shape (Correlator.shape, bindings.cpp:139), the FFT size used for the search windows,
 * and the number of kernels this handle has launched (a running count). */
B200_API int b200_info(const b200_handle *h, int *ny, int *nx, int *fft_size, uint64_t *launches);

/* Timing of the correlation kernel: while enabled, every launch of the fused correlation kernel
 * is bracketed by CUDA events on its own stream; b200_profile_read gives the summed event time
 * (ms), the number of launches and the pairs they processed, and resets the sums. For
 * measurement; no counterpart in the reference. */
B200_API int b200_profile(b200_handle *h, int enable);
B200_API int b200_profile_read(b200_handle *h, double *kernel_ms, uint64_t *kernel_launches,
                               uint64_t *pairs);

/* "b200" (Correlator.backend, cxx/framecor.h:55). */
B200_API const char *b200_backend(const b200_handle *h);

/* Whether a CUDA device of compute capability 10.0 is present (framecor::hasCuda,
 * cxx/framecor.h:63, cxx/cuda.cu:383-387). */
B200_API int b200_has_device(void);

/* The library version (the module's __version__, bindings.cpp:114). */
B200_API const char *b200_version(void);

#ifdef __cplusplus
}
#endif

#endif /* SLIPCAM_B200_H */
