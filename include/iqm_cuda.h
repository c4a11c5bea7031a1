/*
 * iqm_cuda.h -- C ABI of the B200 (sm_100a) image-quality-metric library (libiqm_cuda.so).
 *
 * This is the drop-in boundary for cadik/IQM's metric-evaluation path.  The reference exposes one
 * C++ class per metric, each with
 *     XResult computeMetric(const VulkanRuntime&, const InputImage&, const InputImage&[, args])
 * (src/gpu/ssim/ssim.h:25-35, src/gpu/fsim/fsim.h:33-36, src/gpu/flip/flip.h:27-30,
 *  src/gpu/svd/svd.h:25-28), taking RGBA8 host images (src/input_image.h: tightly packed
 * width*height*4 bytes, src/main.cpp:37-57) and returning scores and maps by value.
 * Each entry point below replaces one of those calls; the C++ wrappers in iqm_b200/host keep the
 * reference's class and result shapes on top of it.
 *
 * Conventions
 *   - Plain C types only; no exceptions cross this boundary.  Every call returns IQM_OK (0) or a
 *     negative IQM_E* code, and iqm_last_error() describes the last failure on that context.
 *   - Images are RGBA8, row-major, `row_bytes` apart (>= 4*w); the alpha byte is ignored, as in
 *     the reference's shaders.  Sides up to 65536 and fewer than 2^31 pixels per image.  "input" is the distorted image, "ref" the reference image
 *     (the CLI's --input / --ref, src/args.cpp:38-43).
 *   - Host entry points (iqm_ssim, iqm_fsim, iqm_flip, iqm_msvd and the *_batch forms) take host
 *     pointers (pageable or pinned), copy to the device, compute, copy results back and return
 *     when results are in host memory.
 *   - *_dev entry points take DEVICE pointers, enqueue on the context's stream and return
 *     immediately; scores are written to device memory.  They never synchronise the host.
 *   - A context is not thread-safe (neither is the reference's VulkanRuntime, whose single
 *     command buffer all metric objects share, src/gpu/base/vulkan_runtime.h:54-61).
 */
#ifndef IQM_CUDA_H
#define IQM_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------------------- */
#define IQM_OK 0
#define IQM_EINVAL (-1)       /* bad argument: null pointer, size, mismatch, parameter range  */
#define IQM_ECUDA (-2)        /* a CUDA runtime call failed (text in iqm_last_error)            */
#define IQM_ENOMEM (-3)       /* device or host allocation failed                               */
#define IQM_EUNSUPPORTED (-4) /* valid request this build does not implement                    */

typedef struct iqm_ctx iqm_ctx;

typedef enum {
    IQM_FP32 = 0,       /* plain FP32 arithmetic, FP64 pooling sums                              */
    IQM_MIXED = 1,      /* FSIM: inverse transforms on the tensor cores as FP16 tiles with
                           split-precision (hi + lo) products and FP32 accumulation, FP16
                           intermediate planes; FP64 noise threshold and pooling as in IQM_FP32.
                           Plane sizes without tensor-core engines (all but 480x270, the plane of
                           1080p and 4K pairs) run the FP32 transforms.
                           SSIM: the Gaussian window sums on the tensor cores, moments staged as
                           FP16 hi + lo pairs, split-precision products, FP32 accumulation.
                           Scores within 1e-4 of the FP64 oracle.  FLIP and M-SVD compute in FP32
                           whatever is asked.                                                      */
    IQM_MIXED_FAST = 2  /* as IQM_MIXED with single FP16 operands and products (hi parts only)  */
} iqm_precision;

/* ---- context --------------------------------------------------------------------------- */
/* Replaces VulkanRuntime() (src/gpu/base/vulkan_runtime.cpp:22-67): binds `device`, creates a
 * stream and a grow-only device arena reused across calls. */
int iqm_create(int device, iqm_ctx **out);
int iqm_destroy(iqm_ctx *ctx);
/* Text of the last error on `ctx` (or of the last iqm_create failure when ctx is NULL). */
const char *iqm_last_error(const iqm_ctx *ctx);
/* Run subsequent work on a caller-owned cudaStream_t (NULL restores the context's own stream). */
int iqm_set_stream(iqm_ctx *ctx, void *cuda_stream);
int iqm_synchronize(iqm_ctx *ctx);
/* Device name as the reference prints it with -v ("Selected device: ...", src/main.cpp:80). */
int iqm_device_name(iqm_ctx *ctx, char *buf, size_t len);

/* ---- SSIM (src/gpu/ssim/ssim.h:25-35, src/gpu/ssim/ssim.cpp:71-243,386-401) ------------- */
typedef struct {
    int kernel_size; /* Gaussian window side; radius (kernel_size-1)/2 in [1, 7]; default 11   */
    float k1;        /* default 0.01 */
    float k2;        /* default 0.03 */
    float sigma;     /* default 1.5  */
    int precision;   /* iqm_precision; default IQM_FP32 (a zeroed struct asks for FP32)         */
} iqm_ssim_params;
void iqm_ssim_default_params(iqm_ssim_params *p);

/* MSSIM of one pair; `map_out` (nullable, w*h floats) receives the SSIM map
 * (SSIMResult::imageData, src/gpu/ssim/ssim.h:17-23).  `mssim` must not be NULL. */
int iqm_ssim(iqm_ctx *ctx, const uint8_t *rgba_in, const uint8_t *rgba_ref, int w, int h,
             size_t row_bytes, const iqm_ssim_params *params, float *map_out, double *mssim);

/* Allocation-free SSIM.  This entry point has no counterpart in the reference.  It is for callers
 * that cannot let a library allocate device memory -- a host application that reserves the whole
 * GPU for its own allocator, or a plugin host that accounts for every byte it hands out.  It calls
 * no cudaMalloc/cudaFree and creates no context: the caller passes DEVICE pointers for the two
 * images (`d_in`, `d_ref`), the score (`d_mssim`, one double) and optionally the map (`d_map`,
 * w*h floats), plus the stream to run on (NULL = the default stream); the call returns without
 * synchronising.  The kernel's scratch is a fixed array inside the library (about 33 KB) that every
 * GPU which loads the library holds until the process exits, so the image may span at most
 * IQM_SSIM_NOALLOC_MAX_TILES tiles of 128 columns x 122 rows (11-tap window; e.g. 7680x4320 uses
 * 2160); larger images return IQM_EINVAL.  The first call on a device looks up that array's device
 * address with the device current, so make it before any stream capture.  The address is kept for
 * the device's primary context (the one the CUDA runtime uses): callers in other driver-API
 * contexts, or after cudaDeviceReset, are not supported.  All calls share the one array: calls
 * that overlap on the GPU (other streams, other threads) race -- serialise them.  `d_in`, `d_ref`,
 * `row_bytes` and `d_map` must be multiples of 4 and `d_mssim` of 8 (else IQM_EINVAL, before any
 * launch).  Only IQM_FP32 is served here: another `params->precision` returns IQM_EINVAL.
 * Returns IQM_OK, IQM_EINVAL (null or misaligned pointer, size or parameter out of range) or IQM_ECUDA (a launch of this call failed; errors pending from the caller's earlier work
 * are left pending, not reported or cleared). */
#define IQM_SSIM_NOALLOC_MAX_TILES 4096
int iqm_ssim_noalloc(const uint8_t *d_in, const uint8_t *d_ref, int w, int h, size_t row_bytes,
                     const iqm_ssim_params *params, float *d_map, double *d_mssim, void *cuda_stream);

/* ---- M-SVD (src/gpu/svd/svd.h:25-28, src/gpu/svd/svd.cpp:39-164) ----------------------- */
/* `block_map` (nullable, (w/8)*(h/8) floats) receives D/max(D) (SVDResult::imageData). */
int iqm_msvd(iqm_ctx *ctx, const uint8_t *rgba_in, const uint8_t *rgba_ref, int w, int h,
             size_t row_bytes, float *block_map, double *msvd);

/* ---- FLIP (src/gpu/flip/flip.h:21-30, src/gpu/flip/flip.cpp:121-172) -------------------- */
typedef struct {
    float monitor_resolution_x; /* default 2560 (FLIP_RES)      */
    float monitor_distance;     /* default 0.7  (FLIP_DISTANCE) */
    float monitor_width;        /* default 0.6  (FLIP_WIDTH)    */
} iqm_flip_params;
void iqm_flip_default_params(iqm_flip_params *p);
/* pixels per degree exactly as src/gpu/flip/flip.cpp:125 computes it */
double iqm_flip_ppd(const iqm_flip_params *p);
/* Mean of the per-pixel FLIP value (shaders/flip/combine_error_maps.glsl:28).  The reference
 * computes that map but never pools it (FLIPResult::mean_flip is never set); `err_map`
 * (nullable, w*h floats) receives the map itself. */
int iqm_flip(iqm_ctx *ctx, const uint8_t *rgba_in, const uint8_t *rgba_ref, int w, int h,
             size_t row_bytes, const iqm_flip_params *params, float *err_map, double *mean_flip);

/* ---- FSIM / FSIMc (src/gpu/fsim/fsim.h:27-36, src/gpu/fsim/fsim.cpp:80-163) ------------- */
/* energy_mode selects how the noise-energy estimates are pooled:
 *   0 = as the reference (only the first ceil(N/2) pixels contribute, the rest read as 0);
 *   1 = over all N pixels. */
int iqm_fsim(iqm_ctx *ctx, const uint8_t *rgba_in, const uint8_t *rgba_ref, int w, int h,
             size_t row_bytes, iqm_precision precision, int energy_mode, double *fsim,
             double *fsimc);

/* Size-only FSIM constants of a W'xH' plane, as used by the noise model: EM_n(o) (the filter
 * energy of fsim_filter_combinations.cpp:76-134) and the estimated noise-energy sums EstSumAn2(o),
 * EstSumAiAj(o) (shaders/fsim/fsim_mult_filters.glsl) pooled per energy_mode; 4 values each. */
int iqm_fsim_plan_constants(iqm_ctx *ctx, int w2, int h2, int energy_mode, double *em, double *an2,
                            double *aiaj);

/* ---- batches: many pairs (uneven sizes allowed) in one launch sequence -------------------- */
typedef struct {
    const uint8_t *input; /* RGBA8 distorted image */
    const uint8_t *ref;   /* RGBA8 reference image */
    int w, h;
    size_t row_bytes;
} iqm_pair;

/* Device-resident forms: `pairs` is a HOST array of n descriptors whose pointers are DEVICE
 * pointers; scores go to DEVICE memory (`d_scores`, n doubles; FSIM writes 2n: fsim then fsimc
 * per pair).  Enqueued on the context stream; no host synchronisation.  The images are read in
 * place, so each image pointer and row_bytes must be a multiple of 4 (IQM_EINVAL otherwise). */
int iqm_ssim_dev(iqm_ctx *ctx, const iqm_pair *pairs, int n, const iqm_ssim_params *params,
                 double *d_scores);
int iqm_msvd_dev(iqm_ctx *ctx, const iqm_pair *pairs, int n, double *d_scores);
int iqm_flip_dev(iqm_ctx *ctx, const iqm_pair *pairs, int n, const iqm_flip_params *params,
                 double *d_scores);
int iqm_fsim_dev(iqm_ctx *ctx, const iqm_pair *pairs, int n, iqm_precision precision,
                 int energy_mode, double *d_scores);

/* Host forms of the same: HOST image pointers and HOST score arrays; synchronous. */
int iqm_ssim_batch(iqm_ctx *ctx, const iqm_pair *pairs, int n, const iqm_ssim_params *params,
                   double *scores);
int iqm_msvd_batch(iqm_ctx *ctx, const iqm_pair *pairs, int n, double *scores);
int iqm_flip_batch(iqm_ctx *ctx, const iqm_pair *pairs, int n, const iqm_flip_params *params,
                   double *scores);
int iqm_fsim_batch(iqm_ctx *ctx, const iqm_pair *pairs, int n, iqm_precision precision,
                   int energy_mode, double *scores);

/* Number of kernel launches the last *_dev / host call enqueued on this context (for the
 * benchmark's launch accounting). */
int iqm_last_launch_count(const iqm_ctx *ctx);

/* Per-kernel device timing, the device-side counterpart of the reference's Timestamps
 * (src/timestamps.h:11-40, printed by `-v`).  With enable != 0 the context records a CUDA event on
 * its stream after every kernel launch and after every copy or memset it enqueues, and charges each
 * kernel the interval since the event before it; enabling or disabling clears the totals.  The
 * events add a little work between launches, so time throughput with timing off. */
int iqm_set_kernel_timing(iqm_ctx *ctx, int enable);

/* Waits for the context stream and writes one line per kernel name, "name launches total_ms\n",
 * into buf (NUL-terminated); IQM_EINVAL if cap is too small. */
int iqm_kernel_times(iqm_ctx *ctx, char *buf, size_t cap);

/* Page-locked host memory for staging images (the reference keeps images in pageable vectors,
 * src/input_image.h): copies from it run at full host-link speed and overlap with other work. */
int iqm_host_alloc(size_t bytes, void **out);
int iqm_host_free(void *p);

/* ---- batches over several metrics ------------------------------------------------------------
 * The reference evaluates one pair with one metric per invocation (src/main.cpp:271-286, the method
 * chosen by IQM::Method, src/methods.h:13-19); these run many pairs through several metrics at once.
 * Scores are laid out metric by metric, in the order below, for the metrics in the mask:
 * SSIM n doubles, FSIM 2n (FSIM, FSIMc per pair), FLIP n, M-SVD n. */
#define IQM_METRIC_SSIM 1
#define IQM_METRIC_FSIM 2
#define IQM_METRIC_FLIP 4
#define IQM_METRIC_MSVD 8

/* Host pairs (sizes may differ): upload, evaluate every metric of the mask, copy the scores to the
 * host and return.  ssim/flip may be NULL for the defaults.  `precision` is FSIM's; SSIM takes its
 * own from ssim->precision (the defaults: IQM_FP32). */
int iqm_batch(iqm_ctx *ctx, int metric_mask, const iqm_pair *pairs, int n, const iqm_ssim_params *ssim,
              const iqm_flip_params *flip, iqm_precision precision, int energy_mode, double *scores);

/* A reusable plan for one fixed batch of device-resident pairs: creation validates the arguments,
 * runs the batch once (building per-size tables and sizing the plan's own device buffers), with
 * autotune != 0 times FSIM's launch-shape candidates and keeps the fastest, and captures the whole
 * launch sequence of every metric into a CUDA graph.  iqm_batch_plan_run replays it on the context
 * stream (asynchronous; scores land in d_scores).  The pairs' device memory, d_scores and the context
 * must outlive the plan; a plan's runs must not overlap one another on the GPU. */
typedef struct iqm_batch_plan iqm_batch_plan;
int iqm_batch_plan_create(iqm_ctx *ctx, int metric_mask, const iqm_pair *dev_pairs, int n,
                          const iqm_ssim_params *ssim, const iqm_flip_params *flip, iqm_precision precision,
                          int energy_mode, int autotune, double *d_scores, iqm_batch_plan **out);
int iqm_batch_plan_run(iqm_batch_plan *plan);
/* Text describing the chosen launch shapes, and the kernel launches one run replays. */
int iqm_batch_plan_info(const iqm_batch_plan *plan, char *buf, size_t cap, int *launches);
int iqm_batch_plan_destroy(iqm_batch_plan *plan);

#ifdef __cplusplus
}
#endif
#endif /* IQM_CUDA_H */
