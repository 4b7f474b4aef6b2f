/*
 * astrotransit_b200.h -- C ABI of the B200-native Box Least Squares engine.
 *
 * Plain C types only: device buffers are passed as raw pointers, the CUDA
 * stream as `void*` (a cudaStream_t), and every call returns an int status.
 * No exception crosses this boundary; the message of the last failure on a
 * handle is available from atb_last_error().
 *
 * Reference interfaces replaced (ubunbun18/Astro_Transit_GPU, paths within
 * the reference project):
 *   - search/gpu_bls.py:42-144 run_gpu_bls  +  search/kernels/bls.cu:12-172
 *       (the CuPy RawKernel launch at gpu_bls.py:122-128)
 *       -> atb_run_gpu_bls(), or the batched plan API with ATB_GEOM_FIXED
 *   - search/v42_parity.py:27-107 run_vbls_exact_parity  +
 *     search/kernels/vbls_v42_parity.cu:12-181
 *       (the CuPy RawModule launch at v42_parity.py:79-87)
 *       -> atb_run_vbls_exact_parity(), or the plan API with ATB_GEOM_BINNED
 *   - search/api.py:27-140 BoxLeastSquaresGPU.power dispatches to the two
 *     above; its Python counterpart is astro_transit_gpu_b200.api.
 * The reference has no native FFI of its own (CuPy JIT-compiles the kernels
 * at run time, gpu_bls.py:18-40, v42_parity.py:7-25); these entry points are
 * what a maintainer binds instead, with ctypes (the single-call entry points
 * take the same arrays the CuPy launches take).
 */
#ifndef ASTROTRANSIT_B200_H
#define ASTROTRANSIT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define ATB_OK 0
#define ATB_EINVAL 1    /* invalid argument (reference: ValueError, api.py:54-70) */
#define ATB_ENOMEM 2    /* device allocation failed (reference: MemoryError, gpu_bls.py:113-114) */
#define ATB_ECUDA 3     /* CUDA runtime error */
#define ATB_EINTERNAL 4 /* internal consistency error */
#define ATB_EDATA 5     /* a kernel flagged invalid input data (non-finite value, weight <= 0) */

/* geometry (the `method` argument of BoxLeastSquaresGPU.power) */
#define ATB_GEOM_FIXED 0  /* method="fast":   fixed n_bins phase bins, bls.cu */
#define ATB_GEOM_BINNED 1 /* method="parity": bin = min(duration)/oversample, V42 */

/* objective */
#define ATB_OBJ_FAST 0       /* two-sided score sqrt(s^2/(r(1-r))) of bls.cu:128-131,165 */
#define ATB_OBJ_SNR 1        /* depth/depth_err, dip-only, vbls_v42_parity.cu:116-119 */
#define ATB_OBJ_LIKELIHOOD 2 /* 0.5*depth^2*W_in*W_out/(W_in+W_out), dip-only */

typedef struct atb_handle atb_handle;
typedef struct atb_plan atb_plan;

typedef struct {
    int32_t geometry;   /* ATB_GEOM_* */
    int32_t objective;  /* ATB_OBJ_*; FIXED requires FAST, BINNED requires SNR or LIKELIHOOD */
    int32_t n_bins;     /* FIXED: phase bins per period (reference default 200, api.py:37) */
    int32_t oversample; /* BINNED: bins per minimum duration (reference default 10, api.py:76) */
    int32_t max_bins;   /* BINNED: 0 = no cap; >0 reproduces the reference's bin cap
                           n_bins = min(n_bins, max_bins-1), vbls_v42_parity.cu:46-47 */
    int32_t tile_periods; /* periods per work-queue tile, 1..64; 0 = chosen from the batch
                             size (no reference counterpart; results do not depend on it) */
    /* Fold strategy (no reference counterpart; results do not depend on it): a
     * period whose bins hold at least merge_run time-ordered points on average
     * (bin width x the curve's mean point density) adds the points a thread
     * holds once when they provably share a slot.  0 = the default (8),
     * < 0 = never. */
    int32_t merge_run;
    /* Threads per search CTA (no reference counterpart; results do not depend
     * on it): 512 (two CTAs per SM) or 256 (four per SM); 0 = the geometry's
     * default, 256 for ATB_GEOM_FIXED and 512 for ATB_GEOM_BINNED. */
    int32_t cta_threads;
} atb_params;

/*
 * A batch of light curves.  Index arrays are HOST memory; data arrays are
 * DEVICE memory on the handle's device.  Curve c has
 *   points   [point_offset[c], point_offset[c+1]) of y and w,
 *   times    [time_offset[c], time_offset[c]+n_c) of t (time_offset NULL:
 *            same as point_offset; all-zero offsets = one time axis shared by
 *            every curve, the flux_matrix layout of v42_parity.py:27),
 *   periods  [period_begin[c], period_begin[c]+period_count[c]) of periods,
 *   durations[dur_begin[c], dur_begin[c]+dur_count[c]) of durations,
 *   outputs  [out_begin[c], out_begin[c]+period_count[c]) of every output.
 * Grids may be shared between curves (equal begin values).
 */
typedef struct {
    int32_t n_curves;
    int32_t y_is_f64;             /* 0: y is float32, 1: y is float64 */
    const int64_t* point_offset;  /* [n_curves+1] */
    const int64_t* time_offset;   /* [n_curves] or NULL */
    const int64_t* period_begin;  /* [n_curves] */
    const int64_t* period_count;  /* [n_curves] */
    const int64_t* dur_begin;     /* [n_curves] */
    const int32_t* dur_count;     /* [n_curves], each in [1, 32] */
    const int64_t* out_begin;     /* [n_curves] */
    const double* t;              /* device, float64 times */
    const void* y;                /* device, float32 or float64 flux */
    const float* w;               /* device, float32 weights 1/dy^2, or NULL for unit weights */
    const double* periods;        /* device, float64, > 0 */
    const double* durations;      /* device, float64, > 0 */
} atb_batch;

/* Device output arrays indexed by output slot; any may be NULL except power. */
typedef struct {
    float* power;          /* objective value of the best window per period */
    float* depth;          /* mean(out) - mean(in) of that window */
    float* depth_err;      /* sqrt(1/W_in + 1/W_out) */
    double* t0;            /* transit time (BINNED: mid-transit mod period; FIXED: box start) */
    float* duration;       /* BINNED: dur_bins*bin_duration; FIXED: the duration grid value */
    int32_t* window;       /* start_bin * n_durations + duration_index, -1 when no valid window */
    int32_t* best_period;  /* [n_curves]: index of the maximum power within the curve's grid */
    /* Winner-take-all screening (search/vbls.py:62-188 keeps only a best record
     * per target): [n_curves] packed (power bits << 32 | ~period index),
     * raised with atomicMax, zeroed by the caller before the execution.  With
     * it, every per-period array above may be NULL (nothing per period is
     * written) and best_period is decoded from it (first maximum; -1 when no
     * period has a valid window). */
    uint64_t* best_key;
} atb_outputs;

/* Handle: one per device (and per host thread using it concurrently). */
int atb_create(int device, atb_handle** out);
void atb_destroy(atb_handle* h);
/* Copies the message of the last failure on h (empty if none); returns its length. */
int atb_last_error(const atb_handle* h, char* buf, size_t len);
/* Library version string, e.g. "astrotransit-b200 0.1.0 sm_100a". */
const char* atb_version(void);

/*
 * Plans.  atb_plan_create validates the batch, allocates the plan's device
 * scratch (staged points, per-curve constants, the work-queue counter) and may
 * synchronise the handle's device once.  atb_plan_execute only enqueues
 * kernels on `stream` (no allocation, no synchronisation), so it can be called
 * repeatedly and captured into a CUDA graph.  Device pointers are bound at
 * creation; their contents may change between executions, their sizes not.
 */
int atb_plan_create(atb_handle* h, const atb_params* params, const atb_batch* batch,
                    const atb_outputs* outputs, atb_plan** out);
/*
 * The same plan, set up without waiting for other streams' work (no reference
 * counterpart; for servers that overlap batches): its scratch comes from the
 * stream-ordered allocator on `stream`, its set-up copies and status reads run
 * on `stream`, and atb_plan_destroy releases it in `stream` order.  The batch's
 * device inputs must be ready in `stream` order, and the plan must be executed
 * on `stream`.
 */
int atb_plan_create_async(atb_handle* h, const atb_params* params, const atb_batch* batch,
                          const atb_outputs* outputs, void* stream, atb_plan** out);
int atb_plan_execute(atb_plan* p, void* stream);
/* Synchronises `stream`-independent plan state: returns ATB_EDATA if the last
   execution met invalid input data, ATB_OK otherwise. */
int atb_plan_check(atb_plan* p);
/* Number of kernels one atb_plan_execute enqueues (for launch accounting). */
int atb_plan_kernel_count(const atb_plan* p);
/* Bytes of device scratch the plan holds. */
int64_t atb_plan_scratch_bytes(const atb_plan* p);
void atb_plan_destroy(atb_plan* p);

/*
 * Top-k peaks of each curve's power spectrum after an execution, on the device
 * (replaces the host scipy.signal.find_peaks(power, distance) + sort of
 * search/gpu_bls.py:146-174 for batches): out_idx [n_curves * k] int32 receives
 * per curve the period indices of the k largest peaks at least `distance`
 * samples apart, largest first (equal powers: higher index first), -1 where
 * there are fewer; with no peak at all, the k largest powers.  1 <= k <= 32.
 * Enqueued on `stream`.
 */
int atb_plan_top_k(atb_plan* p, int32_t k, int32_t distance, int32_t* out_idx, void* stream);

/*
 * Diagnostics (no reference counterpart): after an atb_plan_execute has
 * completed, the histogram word layout each curve used and the bit length of
 * its bin-occupancy bound (64: no bound).  Layouts: ATB_LAYOUT_SPLIT (weights
 * not uniform), ATB_LAYOUT_COUNT (uniform weights), ATB_LAYOUT_TIGHT (uniform
 * weights and fewer than 2^12 points can share a bin: two 32-bit reductions
 * per point instead of three), ATB_LAYOUT_TIGHT_CHECKED (uniform weights, no
 * proven bound but few points per bin on average: the two-word layout, with
 * each period's point count checked and a period whose bin overflowed folded
 * again in the count layout).  The layout never changes the results.
 * Synchronous; both arrays hold one entry per curve.
 */
#define ATB_LAYOUT_SPLIT 0
#define ATB_LAYOUT_COUNT 1
#define ATB_LAYOUT_TIGHT 2
#define ATB_LAYOUT_TIGHT_CHECKED 3
int atb_plan_curve_layout(atb_plan* p, int32_t* layout, int32_t* occupancy_bits);

/* One-shot: create, execute on `stream`, synchronise, check, destroy. */
int atb_search(atb_handle* h, const atb_params* params, const atb_batch* batch,
               const atb_outputs* outputs, void* stream);

/*
 * Profiling: executes the plan once with CUDA events between its kernels and
 * synchronises; writes the milliseconds of the staging, search and best-peak
 * kernels (any pointer may be NULL).
 */
int atb_plan_profile(atb_plan* p, void* stream, float* ms_stage, float* ms_search,
                     float* ms_best);

/*
 * Microbenchmarks that measure the roofline denominators of the search kernel
 * on the handle's device (each synchronises; a few milliseconds):
 *   atb_bench_smem_red_u64  64-bit shared-memory reductions per second
 *                           (pattern 0: conflict-free, 1: pseudo-random bins)
 *   atb_bench_smem_red_u32  the same for 32-bit reductions, the width the
 *                           search kernel's histogram words use
 *   atb_bench_dfma          FP64 fused multiply-adds per second
 */
int atb_bench_smem_red_u64(atb_handle* h, int pattern, double* reductions_per_s);
int atb_bench_smem_red_u32(atb_handle* h, int pattern, double* reductions_per_s);
int atb_bench_dfma(atb_handle* h, double* fma_per_s);

/*
 * Single-curve fast path, the counterpart of run_gpu_bls (gpu_bls.py:42) and
 * its bls_kernel launch (gpu_bls.py:122-128).  All arrays are device memory;
 * w may be NULL (unit weights, gpu_bls.py:63-64).  Outputs have n_periods
 * entries (any may be NULL except power); *best_index receives the argmax
 * (gpu_bls.py:131) when best_index is not NULL (HOST pointer; synchronises).
 */
int atb_run_gpu_bls(atb_handle* h, const double* t, const float* y, const float* w, int64_t n,
                    const double* periods, int64_t n_periods, const double* durations,
                    int32_t n_durations, int32_t n_bins, float* power, double* t0,
                    float* duration, float* depth, int32_t* best_index, void* stream);

/*
 * Multi-target parity path, the counterpart of run_vbls_exact_parity
 * (v42_parity.py:27) and its vbls_v42_parity_kernel launch
 * (v42_parity.py:79-87): n_targets curves of n_data points on one shared
 * time axis; flux and weights are [n_targets, n_data] row-major (weights NULL
 * = unit).  Outputs are [n_targets, n_periods]; best_index is a DEVICE array
 * of n_targets (or NULL).  max_bins = 0 disables the reference's cap.
 */
int atb_run_vbls_exact_parity(atb_handle* h, const double* time, const float* flux,
                              const float* weights, int64_t n_targets, int64_t n_data,
                              const double* periods, int64_t n_periods, const double* durations,
                              int32_t n_durations, int32_t oversample, int32_t max_bins,
                              int32_t objective, float* power, double* t0, float* duration,
                              float* depth, int32_t* best_index, void* stream);

/*
 * Debug/verification: per-point histogram slots of one curve for a list of
 * periods (slot = V42 bin index for BINNED; bin+1, or n_bins+1 when dropped,
 * for FIXED).  out_slots is a device array [n_periods, n] row-major.  Runs
 * the same staging and fold code as the search.
 */
int atb_debug_fold(atb_handle* h, const atb_params* params, const double* t, const float* y,
                   const float* w, int64_t n, const double* periods, int64_t n_periods,
                   const double* durations, int32_t n_durations, int32_t* out_slots,
                   void* stream);

/*
 * Single-curve search that allocates nothing.  No counterpart in the
 * reference: it exists for callers that cannot allocate device memory while
 * they run -- a host application that has already reserved (nearly) all of the
 * GPU's memory for its own pool, or a latency-critical loop where cudaMalloc
 * and cudaFree (which may synchronise the whole device) are not allowed.
 *
 * The caller passes device inputs and outputs as for atb_run_gpu_bls /
 * atb_run_vbls_exact_parity (y is float32, or float64 when y_is_f64; w may be
 * NULL; any output except power may be NULL; best_index is a DEVICE int32 or
 * NULL).  All other working memory is one array built into the library,
 * ATB_STATIC_SCRATCH_BYTES large, that every GPU which loads the library holds
 * until the process exits.  Limits: at most ATB_STATIC_MAX_POINTS points, at
 * most 32 durations, and a period whose bins do not fit one shared-memory
 * histogram is accepted only where the search takes it in bin-range passes
 * through shared memory (astropy-binned geometry, oversample <= 16, the
 * longest window at least 64 bins shorter than a pass); others -- fixed bins
 * beyond the histogram, finer or longer-windowed astropy bins -- would need a
 * global histogram and are rejected (use the plan API).  The
 * search runs 512-thread CTAs: params->cta_threads must be 0 or 512.
 * Errors are written to err (err_len bytes, may be NULL); no exception.  The
 * call itself allocates nothing on host or device: it calls no cudaMalloc,
 * cudaFree or allocating library routine.
 *
 * The call is synchronous on `stream`.  Each call looks up the array's device
 * address and sets the kernels' shared-memory limit (neither allocates).  With
 * CUDA's lazy module loading, the first call on a device is the one that makes
 * the runtime load this library's kernels and map the array on that device,
 * which may allocate and synchronise inside the driver: make that first call
 * at start-up (a call with n = 1 is enough) and before any stream capture;
 * from the second call on nothing is loaded or mapped.  Every call uses the same array
 * (the previous call's contents remain; the call resets what must start at
 * zero), so calls on the same device must not overlap on the GPU: concurrent
 * calls from several streams or threads race and corrupt each other's results.
 */
#define ATB_STATIC_MAX_POINTS 65536
#define ATB_STATIC_SCRATCH_BYTES (16 * ATB_STATIC_MAX_POINTS + 4096)
int atb_search_curve_static(const atb_params* params, const double* t, const void* y,
                            int32_t y_is_f64, const float* w, int64_t n, const double* periods,
                            int64_t n_periods, const double* durations, int32_t n_durations,
                            float* power, float* depth, float* depth_err, double* t0,
                            float* duration, int32_t* window, int32_t* best_index, void* stream,
                            char* err, size_t err_len);

#ifdef __cplusplus
}
#endif

#endif /* ASTROTRANSIT_B200_H */
