/*
 * stpgpu.h -- C ABI of the B200 snapshot imager and source finder.
 *
 * Drop-in boundary for the hot path of the Slow Transients Pipeline (STP):
 *   stp::image_visibilities / stp::ImageVisibilities  (src/stp/imager/imager.h:233-411)
 *   stp::convolve_to_grid                             (src/stp/gridder/gridder.h:240-997)
 *   stp::SourceFindImage                              (src/stp/sourcefind/sourcefind.h:143-216)
 * Plain pointers and sizes only.  All matrices are column-major (Armadillo
 * layout): element (r, c) of an R x C matrix is at c*R + r.
 *
 * Every entry point returns an stpgpu_status (0 = success).  On failure
 * stpgpu_last_error(ctx) returns a message.  A context is bound to one CUDA
 * device and owns one stream; calls on one context must be serialised by the
 * caller, different contexts are independent.
 */
#ifndef STPGPU_H
#define STPGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define STPGPU_ABI_VERSION 2

#if defined(__GNUC__)
#define STPGPU_API __attribute__((visibility("default")))
#else
#define STPGPU_API
#endif

typedef enum {
    STPGPU_OK = 0,
    STPGPU_ERR_INVALID_ARG = 1, /* bad sizes / parameters (the reference asserts) */
    STPGPU_ERR_UNSUPPORTED = 2, /* option outside the GPU path (A-projection, Hankel, Ceres fit) */
    STPGPU_ERR_CUDA = 3,        /* CUDA runtime error */
    STPGPU_ERR_CUFFT = 4,       /* cuFFT plan / exec failure (reference: std::runtime_error, fft.cpp:100-103) */
    STPGPU_ERR_OOM = 5,         /* device allocation failed or admission budget exceeded */
    STPGPU_ERR_CAPACITY = 6,    /* caller buffer too small; required size returned */
    STPGPU_ERR_DEVICE = 7,      /* a kernel reported an internal error (bounded loop gave up) */
    STPGPU_ERR_TIMEOUT = 8,     /* a bounded wait expired */
    STPGPU_ERR_NO_DEVICE = 9    /* no CUDA device / driver */
} stpgpu_status;

/* Enum values are those of src/stp/types.h:32-89. */
typedef enum { STPGPU_TOPHAT = 0, STPGPU_TRIANGLE, STPGPU_SINC, STPGPU_GAUSSIAN, STPGPU_GAUSSIANSINC, STPGPU_PSWF } stpgpu_kernel_function;
typedef enum { STPGPU_ZEROMEDIAN = 0, STPGPU_BINMEDIAN, STPGPU_BINAPPROX, STPGPU_NTHELEMENT } stpgpu_median_method;

/* Arithmetic of the imager.  FP64 is the plain form matched to the
 * reference's double build; FP32 uses single-precision visibilities, kernel
 * weights, grid and FFT; FP32C adds two-sum compensated accumulation of the
 * grid cells, and stores the grid in double with a double-precision c2r
 * when the grid correction amplifies the FFT's rounding by more than 4096
 * (1/gcf_min^2 over the output field; e.g. PSWF kernels).  uvw -> pixel
 * scaling, W-kernel generation and the final normalisation stay FP64 in all
 * modes. */
typedef enum { STPGPU_FP64 = 0, STPGPU_FP32 = 1, STPGPU_FP32C = 2 } stpgpu_precision;

typedef enum { STPGPU_C128 = 0, STPGPU_C64 = 1 } stpgpu_vis_dtype;
typedef enum { STPGPU_F64 = 0, STPGPU_F32 = 1 } stpgpu_real_dtype;

/* stp::ImagerPars, src/stp/types.h:93-177.  padded_image_size = 0 means
 * image_size * padding_factor (types.h:157).  r_fft is accepted and ignored
 * (cuFFT replaces the FFTW planner modes, fft.cpp:53-76). */
typedef struct {
    int32_t image_size;
    int32_t padded_image_size;
    double cell_size; /* arcsec */
    double padding_factor;
    int32_t kernel_function; /* stpgpu_kernel_function */
    int32_t kernel_support;
    int32_t kernel_exact;
    int32_t oversampling;
    int32_t generate_beam;
    int32_t gridding_correction;
    int32_t analytic_gcf;
    int32_t r_fft;
} stpgpu_imager_pars;

/* stp::W_ProjectionPars, src/stp/types.h:182-250.  With hankel_opt the
 * W-kernels come from the Hankel transform of the radial profile
 * (hankel_proj_slice = 0) or from the 1-D transform of the kernel's
 * projection (hankel_proj_slice = 1), interpolated with interp_type
 * (stp::InterpType: 0 LINEAR, 1 CUBIC, 2 COSINE = linear), as in
 * generate_convolution_kernel_wproj, src/stp/gridder/aw_projection.cpp:211-287. */
typedef struct {
    int32_t num_wplanes;
    int32_t max_wpconv_support;
    int32_t undersampling_opt;
    double kernel_trunc_perc;
    int32_t hankel_opt;
    int32_t hankel_proj_slice;
    int32_t interp_type;
    int32_t wplanes_median;
} stpgpu_wproj_pars;

/* stp::A_ProjectionPars, src/stp/types.h:255-316 (the reference's
 * experimental ENABLE_APROJECTION build).  num_timesteps > 0 enables it
 * (needs W-projection, no Hankel option): lha holds each visibility's local
 * hour angle in hours (n_vis values; a device pointer when the call takes
 * device pointers), pbeam_coefs the 2*degree+1 spherical-harmonic
 * coefficients of the primary beam (host memory).  aproj_mask_perc is
 * accepted and unused, as in the reference. */
typedef struct {
    int32_t num_timesteps;
    double obs_dec;           /* degrees */
    double obs_ra;            /* degrees */
    int32_t aproj_opt;        /* rotate the convolution kernel instead of the beam */
    double aproj_mask_perc;
    const double* lha;
    const double* pbeam_coefs;
    int32_t n_pbeam_coefs;
    int32_t reserved;
} stpgpu_aproj_pars;

/* Per-call imaging report. */
typedef struct {
    double sample_grid_total;   /* 2 * sum of good weights (gridder.h:417-423) */
    int64_t n_good_vis;         /* visibilities that passed the bounds check */
    int64_t n_grid_items;       /* gridded items incl. mirrored duplicates */
    int32_t padded_image_size;
    int32_t image_size;
    int32_t num_wplanes;
    int32_t max_plane_support; /* largest truncated W-kernel support */
    double device_ms;           /* device time of the call (CUDA events) */
    /* With stpgpu_set_timing(ctx, 1): device time of the phases the
     * reference reports (reduce/common_functions.cpp:164-228), ms:
     * [0] grid init (prepass, W-planes and W-kernels, binning),
     * [1] grid loop (the tile gridder kernel), [2] FFT, [3] normalise. */
    double phase_ms[4];
    int32_t n_launches; /* kernels of this library the call ran, graph replays included (cuFFT's excluded) */
    /* bit 0: the compensated-FP32 call kept its grid in double and ran the
     * c2r in double precision, because the grid correction amplifies the
     * single-precision transform's rounding by 1/gcf_min^2 > 4096 over the
     * output field */
    int32_t flags;
} stpgpu_imager_info;

/* One island, stp::IslandParams (src/stp/sourcefind/sourcefind.h:63-133).
 * moments = Gaussian2dParams from estimate_moments_fit:
 * {amplitude, x_centre, y_centre, semimajor, semiminor, theta}. */
typedef struct {
    int32_t label_idx;
    int32_t sign;
    double extremum_val;
    int32_t extremum_y_idx;
    int32_t extremum_x_idx;
    int32_t num_samples;
    int32_t bbox_top, bbox_bottom, bbox_left, bbox_right;
    double moments_fit[6];
    double leastsq_fit[6]; /* with gaussian_fitting: least-squares 2-D Gaussian, else zeros */
    int32_t fit_iterations; /* Levenberg-Marquardt iterations of the fit (0: not fitted) */
    int32_t reserved;
} stpgpu_island;

/* SourceFindImage ctor arguments, src/stp/sourcefind/sourcefind.h:188-201.
 * ccl_slice_cols: width of the reference's TBB column slices, which decides
 * one 8-connectivity link (src/stp/common/ccl.h:207 vs :386); 0 = the
 * decomposition of an 8-thread host, max(2, cols/8). */
typedef struct {
    double detection_n_sigma;
    double analysis_n_sigma;
    double rms_est;
    int32_t find_negative_sources;
    int32_t sigma_clip_iters;
    int32_t median_method; /* stpgpu_median_method */
    int32_t gaussian_fitting; /* least-squares 2-D Gaussian per island (Levenberg-Marquardt in place of Ceres) */
    int32_t ccl_4connectivity;
    int32_t generate_labelmap;
    int32_t source_min_area;
    int32_t ccl_slice_cols;
} stpgpu_sf_pars;

typedef struct {
    double bg_level;
    double rms_est;
    double mean;
    double sigma;
    int32_t n_labels_pos; /* CCL labels before the detection filter */
    int32_t n_labels_neg;
    int32_t n_valid_labels;
    int32_t n_islands;
    double device_ms;
} stpgpu_sf_info;

typedef struct stpgpu_context stpgpu_context;

STPGPU_API int stpgpu_abi_version(void);

/* Create a context on `device` (its own CUDA stream). */
STPGPU_API stpgpu_status stpgpu_create(int device, stpgpu_context** ctx);
STPGPU_API stpgpu_status stpgpu_destroy(stpgpu_context* ctx);
STPGPU_API const char* stpgpu_last_error(const stpgpu_context* ctx);
/* The context's stream (cudaStream_t), for callers that order work around it. */
STPGPU_API void* stpgpu_stream(stpgpu_context* ctx);
/* Record per-phase CUDA events in subsequent imaging calls (info->phase_ms). */
STPGPU_API stpgpu_status stpgpu_set_timing(stpgpu_context* ctx, int enable);
/* Release cached device buffers, cuFFT plans and W-kernel caches. */
STPGPU_API stpgpu_status stpgpu_trim(stpgpu_context* ctx);

/* stp::image_visibilities through stp_python.image_visibilities_wrapper
 * (src/stp-python/stp_python.cpp:17-140), FP64, host buffers:
 *   vis      n_vis complex128 (interleaved re, im)
 *   weights  n_vis float64
 *   uvw      n_vis x 3 float64, column-major (u[], v[], w[])
 *   image    image_size^2 float64 out, column-major, unshifted (DC at [0,0])
 *   beam     nullable; image_size^2 float64 when generate_beam
 * Sizes are used as given (stp::ImagerPars semantics); the Python binding
 * rounds them up to multiples of 4 first as stp_python does
 * (stp_python.cpp:60-67).  When the sampling total is zero the reference
 * returns empty matrices (imager.h:355); then info->image_size is 0 and
 * nothing is written. */
STPGPU_API stpgpu_status stpgpu_image_visibilities(stpgpu_context* ctx, const double* vis, const double* weights, const double* uvw,
    int64_t n_vis, const stpgpu_imager_pars* pars, const stpgpu_wproj_pars* wproj, const stpgpu_aproj_pars* aproj,
    double* image, double* beam, stpgpu_imager_info* info);

/* Same computation with explicit precision and memory location.
 * vis_dtype: STPGPU_C128 or STPGPU_C64; out_dtype: STPGPU_F64 or STPGPU_F32.
 * device_ptrs != 0: all pointers are device pointers on the context's
 * device and the call is asynchronous on the context's stream except for
 * the small scalar read-backs it needs; info->device_ms is then 0. */
STPGPU_API stpgpu_status stpgpu_image_visibilities_ex(stpgpu_context* ctx, const void* vis, int vis_dtype, const double* weights,
    const double* uvw, int64_t n_vis, const stpgpu_imager_pars* pars, const stpgpu_wproj_pars* wproj,
    const stpgpu_aproj_pars* aproj, int precision, void* image, void* beam, int out_dtype, int device_ptrs,
    stpgpu_imager_info* info);

/* stp::convolve_to_grid (src/stp/gridder/gridder.h:240-997), FP64, host
 * buffers.  uv: n_vis x 2 column-major in pixels; w: nullable (W-projection
 * only).  kernel_trunc is the functor's own parameter (truncation radius or
 * half_base_width).  Grids: rows x image_size complex128 column-major with
 * rows = image_size/2+1 when halfplane else image_size. */
STPGPU_API stpgpu_status stpgpu_convolve_to_grid(stpgpu_context* ctx, int kernel_function, double kernel_trunc, int support,
    int image_size, const double* uv, const double* vis, const double* weights, int64_t n_vis, int kernel_exact,
    int oversampling, int shift_uv, int halfplane, int generate_beam, const stpgpu_wproj_pars* wproj, const double* w,
    double cell_size, int analytic_gcf, double* vis_grid, double* sampling_grid, double* sample_grid_total);

/* stp::SourceFindImage (src/stp/sourcefind/sourcefind.cpp:156-292), host
 * buffers.  image: rows x cols float64 column-major, as produced by the
 * imager (unshifted).  label_map: nullable rows x cols int32 out.  islands:
 * capacity entries; *n_islands receives the count (STPGPU_ERR_CAPACITY when
 * it exceeds capacity, nothing else written). */
STPGPU_API stpgpu_status stpgpu_source_find(stpgpu_context* ctx, const double* image, int32_t rows, int32_t cols,
    const stpgpu_sf_pars* pars, int32_t* label_map, stpgpu_island* islands, int32_t capacity, int32_t* n_islands,
    stpgpu_sf_info* info);

/* Same with image_dtype (STPGPU_F64 / STPGPU_F32) and device pointers for
 * image and label_map when device_ptrs != 0 (islands stay host memory). */
STPGPU_API stpgpu_status stpgpu_source_find_ex(stpgpu_context* ctx, const void* image, int image_dtype, int32_t rows, int32_t cols,
    const stpgpu_sf_pars* pars, int32_t* label_map, int device_ptrs, stpgpu_island* islands, int32_t capacity,
    int32_t* n_islands, stpgpu_sf_info* info);

/* stp::generate_visibilities_from_local_skymodel (src/stp/visibility/visibility.cpp:30-40,
 * visibilities_for_point_source :15-28): model visibilities of a point-source
 * sky model, FP64.  skymodel: n_src x 3 column-major (l[], m[], flux[]);
 * uvw: n_vis x 3 column-major (lambda); vis_out: n_vis complex128
 * (interleaved).  vis_in non-null: vis_out = vis_in - model (the residual
 * visibilities of reduce.cpp:113-122; vis_in may equal vis_out).  Device
 * pointers when device_ptrs != 0. */
STPGPU_API stpgpu_status stpgpu_model_visibilities(stpgpu_context* ctx, const double* skymodel, int32_t n_src,
    const double* uvw, int64_t n_vis, const double* vis_in, double* vis_out, int device_ptrs);

/* One snapshot of a batch (stpgpu_image_batch).  Pointers are device
 * pointers when the batch call's device_ptrs != 0, else host pointers.
 * vis_dtype: STPGPU_C128 / STPGPU_C64; uvw n_vis x 3 column-major; image:
 * image_size^2 out, column-major, of the batch's out_dtype.  generate_beam
 * must be 0 (the batch path images the visibilities only). */
typedef struct {
    const void* vis;
    int32_t vis_dtype;
    int32_t reserved;
    const double* weights;
    const double* uvw;
    int64_t n_vis;
    stpgpu_imager_pars pars;
    stpgpu_wproj_pars wproj;
    void* image;
} stpgpu_snapshot;

typedef struct {
    double device_ms;        /* device time of the whole batch (CUDA events) */
    int32_t graph;           /* 1: ran as a replay of a captured CUDA graph */
    int32_t gridder_launches; /* persistent gridder launches (one per kernel variant) */
    int32_t tuned_classes;   /* size classes the tile autotuner measured in this call */
    int32_t n_launches;      /* kernels of this library the call ran, graph replays included (cuFFT's excluded) */
} stpgpu_batch_info;

/* Many snapshots of uneven sizes in one call: per-snapshot preparation on
 * parallel streams, ONE persistent gridder launch per kernel variant over a
 * (snapshot, tile) work queue, then the c2r transforms and normalisation of
 * every snapshot.  Results equal stpgpu_image_visibilities_ex on each
 * snapshot alone.  The tile width (32 or 16 grid columns) of each size class
 * (padded size, kernel mode, precision, support) is chosen by an autotuner
 * that times both shapes on the first batch containing that class.  With
 * device pointers, the second and later calls with the same snapshots
 * (sizes, parameters and pointers) replay a CUDA graph captured from the
 * previous one.  infos: nullable, n_snapshots entries. No counterpart in the
 * reference (it images one snapshot per call, imager.h:233-376). */
STPGPU_API stpgpu_status stpgpu_image_batch(stpgpu_context* ctx, const stpgpu_snapshot* snapshots, int32_t n_snapshots,
    int precision, int out_dtype, int device_ptrs, stpgpu_imager_info* infos, stpgpu_batch_info* batch_info);

/* ------------------------------------------------------------ serving
 * A request loop over one GPU: imaging (+ optional source finding) requests
 * are queued, admitted first-in first-out as soon as a slot is free and the
 * request's estimated device working set fits in the HBM budget next to the
 * requests in flight (continuous admission: a request that arrives while
 * others run starts as soon as they release enough), and run concurrently,
 * each slot on its own context and stream, so their kernels overlap on the
 * device.  Slot contexts keep their buffers, cuFFT plans and W-kernel tables
 * resident between requests.  A request's result does not depend on what
 * else is in flight (up to floating-point summation order in the gridder).
 * No counterpart in the reference (it is a library called once per snapshot). */
typedef struct stpgpu_server stpgpu_server;

typedef struct {
    int32_t device;
    int32_t slots;            /* requests in flight at most (>= 1) */
    int64_t hbm_budget_bytes; /* admission budget for the working sets in flight */
    int32_t precision;        /* stpgpu_precision of every request */
    int32_t reserved;
} stpgpu_server_pars;

/* Host buffers, owned by the caller until the request completes (page-locked
 * buffers make the copies asynchronous and several times faster). */
typedef struct {
    const void* vis;
    int32_t vis_dtype;
    int32_t out_dtype;        /* image dtype: STPGPU_F64 / STPGPU_F32 */
    const double* weights;
    const double* uvw;        /* n_vis x 3 column-major */
    int64_t n_vis;
    stpgpu_imager_pars pars;
    stpgpu_wproj_pars wproj;
    void* image;              /* image_size^2 out; nullable when find_sources (islands only) */
    int32_t find_sources;     /* run the source finder on the image */
    int32_t island_capacity;
    stpgpu_sf_pars sf;
    int32_t* label_map;       /* nullable, image_size^2 out */
    stpgpu_island* islands;   /* island_capacity entries out */
} stpgpu_request;

typedef struct {
    int32_t status;           /* stpgpu_status of the request */
    int32_t n_islands;        /* may exceed island_capacity (then STPGPU_ERR_CAPACITY) */
    int64_t est_bytes;        /* working-set estimate used for admission */
    double submit_ms, admit_ms, done_ms; /* host clock, ms since the server started */
    stpgpu_imager_info imager;
    stpgpu_sf_info sf;
    char error[160];
} stpgpu_result;

typedef struct {
    int64_t submitted, completed, failed, in_flight, queued;
    int64_t peak_in_flight;
    int64_t peak_admitted_bytes; /* largest sum of working-set estimates in flight */
    double p50_ms, p99_ms, mean_ms; /* submit -> done latency of completed requests */
    double throughput_rps;          /* completed / (last done - first submit) */
} stpgpu_server_stats;

STPGPU_API stpgpu_status stpgpu_server_create(const stpgpu_server_pars* pars, stpgpu_server** server);
/* Waits for every queued and running request, then releases the slots. */
STPGPU_API stpgpu_status stpgpu_server_destroy(stpgpu_server* server);
/* Queue a request; *ticket identifies it.  STPGPU_ERR_OOM when its working
 * set alone exceeds the budget; STPGPU_ERR_INVALID_ARG for bad parameters. */
STPGPU_API stpgpu_status stpgpu_server_submit(stpgpu_server* server, const stpgpu_request* request, int64_t* ticket);
/* Run a request once on every slot, in the calling thread, while admission
 * is held (queued requests wait; the requests in flight finish first).  Each
 * slot then holds the buffers, cuFFT plans and tuned gridder layout of the
 * request's size class, so requests of that class admitted later pay no
 * allocation, plan creation or tuning (which can stall every slot on the
 * device for up to a second).  Outputs go to the request's buffers; *result
 * (nullable) holds the last slot's outcome.  Not counted in the statistics. */
STPGPU_API stpgpu_status stpgpu_server_prepare(stpgpu_server* server, const stpgpu_request* request,
    stpgpu_result* result);
/* Wait up to timeout_s (< 0: forever) for a ticket; STPGPU_ERR_TIMEOUT if it
 * is not done by then (the ticket stays valid).  On success *result holds
 * the request's outcome and the ticket is released. */
STPGPU_API stpgpu_status stpgpu_server_wait(stpgpu_server* server, int64_t ticket, double timeout_s, stpgpu_result* result);
STPGPU_API stpgpu_status stpgpu_server_stats_get(stpgpu_server* server, stpgpu_server_stats* stats);

/* Allocation-free connected-component labelling.  No counterpart in the
 * reference: it is the labelling step of stpgpu_source_find (the reference's
 * labeling_8con / labeling_4con, src/stp/common/ccl.h:107-504) for callers
 * that cannot allocate device memory (a detection stage between the launches
 * of a stream-ordered imaging pipeline, where cudaMalloc/cudaFree would
 * synchronise the device; a process whose HBM is already reserved by another
 * allocator).  It needs no context, allocates nothing, and keeps its working
 * arrays in one static device array of 9 bytes per pixel plus the per-chunk
 * counts; images above STPGPU_NOALLOC_MAX_PIXELS pixels are rejected with
 * STPGPU_ERR_INVALID_ARG.  image (rows x cols, column-major, image_dtype
 * STPGPU_F64 / STPGPU_F32) and label_map (rows x cols int32) are device
 * pointers on `device`; stream is a cudaStream_t (NULL: the legacy default
 * stream).  Pixels > analysis_thresh_pos are positive, < analysis_thresh_neg
 * negative (when find_negative_sources); labels are numbered as
 * stpgpu_source_find numbers them before its detection filter, and
 * ccl_slice_cols <= 0 selects max(2, cols / 8).  The call returns after the
 * labels are written.  The scratch array is shared by all calls on a device
 * and keeps the previous call's contents (each call clears what must start at
 * zero): calls whose work overlaps on the GPU race on it.  The array
 * (about 9 MiB) is committed on a device when this library's device code is
 * loaded there: with CUDA's lazy loading that is the first launch of any of
 * the library's kernels on that device, otherwise the first CUDA call of the
 * process.  A caller that hands the rest of HBM to another allocator should
 * make one small call first, so the array is in place.  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress) with
 * that device current and keeps it for the life of the process; make that
 * first call before any stream capture.  A cudaDeviceReset (or a reset of
 * the primary context) unloads the module and leaves the kept address
 * stale: a process that resets a device must not call this entry point on
 * it afterwards.  err_msg (nullable) receives a message on failure. */
#define STPGPU_NOALLOC_MAX_PIXELS (1024 * 1024)
STPGPU_API stpgpu_status stpgpu_label_noalloc(int device, void* stream, const void* image, int image_dtype, int32_t rows,
    int32_t cols, double analysis_thresh_pos, double analysis_thresh_neg, int find_negative_sources, int ccl_4connectivity,
    int ccl_slice_cols, int32_t* label_map, int32_t* n_labels_pos, int32_t* n_labels_neg, char* err_msg, size_t err_msg_len);

#ifdef __cplusplus
}
#endif

#endif /* STPGPU_H */
