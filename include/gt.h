/*
 * gt.h -- C ABI of libgt, the B200 (sm_100a) locate-and-link library.
 *
 * Drop-in boundary for gpu_tracking's hot path.  Each entry point names the
 * reference interface it replaces (paths relative to the reference repo
 * amfaber/tracking_optimizations):
 *
 *   gt_batch           gpu-tracking/src/lib.rs:46-121 `batch_rust`
 *                      -> execute_gpu.rs:496-508 `execute_ndarray`
 *                      -> execute_gpu.rs:372-494 `execute_gpu`
 *   gt_batch_device    same computation on device-resident frames; the
 *                      result table stays on the device
 *   gt_link            gpu-tracking/src/lib.rs:202-212 `link_rust`
 *                      -> linking.rs:570-580 `linker_all` over
 *                      linking.rs:12-61 `FrameSubsetter`
 *   gt_column_names    execute_gpu.rs:197-226 `column_names`
 *   gt_batch_file      gpu-tracking/src/lib.rs:124-200 `batch_file_rust`
 *                      -> execute_gpu.rs:510-542 `execute_file`
 *   gt_ets_channels, gt_file_info, gt_file_read
 *                      lib.rs:215-232 `parse_ets` over decoderiter.rs
 *
 * Entry points with no reference counterpart (the adjoint of the locate
 * path at fixed peaks; see the declarations below):
 *   gt_batch_device_walk, gt_adjoint_forward, gt_adjoint_backward,
 *   gt_adjoint_uncertainty
 *
 * Conventions: plain pointers and sizes, no C++ or torch types.  Every call
 * returns a gt_status; on failure gt_last_error() describes it.  A context
 * is bound to one device, owns one CUDA stream and is not thread-safe.
 * Input pointers are borrowed for the duration of the call.
 */
#ifndef GT_H
#define GT_H
#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define GT_API __attribute__((visibility("default")))
#else
#define GT_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum gt_status {
    GT_OK = 0,
    GT_ERR_ARG = 1,             /* invalid argument (shape, dtype, range) */
    GT_ERR_CUDA = 2,            /* CUDA runtime error */
    GT_ERR_OOM = 3,             /* device allocation failed */
    GT_ERR_SUBNET_BUDGET = 4,   /* a linking subnetwork exceeded the search budget */
    GT_ERR_DEVICE_TIMEOUT = 5,  /* a bounded device wait expired */
    GT_ERR_UNSUPPORTED = 6,     /* parameter the reference rejects (lib.rs:73-74) */
    GT_ERR_CAPACITY = 7         /* a per-frame capacity was exceeded after retries */
} gt_status;

typedef enum gt_dtype { GT_U16 = 0, GT_F32 = 1 } gt_dtype;

/* The 21 keyword arguments of gpu_tracking.batch (gpu_tracking/lib.py:6-28),
 * each Option<> carried as a has_* flag (0 = None).  Defaults are applied as
 * lib.rs:77-91 does. */
typedef struct gt_params {
    uint32_t diameter;
    int32_t has_minmass;        float minmass;
    int32_t has_maxsize;        float maxsize;
    int32_t has_separation;     uint32_t separation;
    int32_t has_noise_size;     float noise_size;
    int32_t has_smoothing_size; uint32_t smoothing_size;
    int32_t has_threshold;      float threshold;
    int32_t has_invert;         int32_t invert;
    int32_t has_percentile;     float percentile;
    int32_t has_topn;           uint32_t topn;
    int32_t has_preprocess;     int32_t preprocess;
    int32_t has_max_iterations; uint32_t max_iterations;
    int32_t has_characterize;   int32_t characterize;
    int32_t has_filter_close;   int32_t filter_close;
    int32_t has_search_range;   float search_range;
    int32_t has_memory;         uint32_t memory;
    int32_t has_cpu_processed;  int32_t cpu_processed;
    int32_t has_sig_radius;     float sig_radius;
    int32_t has_bg_radius;      float bg_radius;
    int32_t has_gap_radius;     float gap_radius;
} gt_params;

#define GT_MAX_COLS 16

/* Result of gt_batch: nrows x ncols row-major f32 (the reference returns the
 * same matrix plus its column list, lib.rs:119-120).  `data` is owned by the
 * library (page-locked host memory where the driver grants it, reused by
 * later calls once released); release it with gt_table_free. */
typedef struct gt_table {
    float* data;
    int64_t nrows;
    int32_t ncols;
    char names[GT_MAX_COLS][24];
    char types[GT_MAX_COLS][8];
} gt_table;

typedef struct gt_ctx gt_ctx;

/* Library version string. */
GT_API const char* gt_version(void);

/* Create a context on CUDA device `device`. */
GT_API int gt_ctx_create(int device, gt_ctx** out);

/* Destroy a context and free its device memory. */
GT_API void gt_ctx_destroy(gt_ctx* ctx);

/* Description of the last failure on this context ("" if none); with a NULL
 * context, the last failure of a context-free call on this thread. */
GT_API const char* gt_last_error(const gt_ctx* ctx);

/* Column names/types for a parameter set: "frame:int,mass:float,...".
 * Returns the number of columns, or a negative gt_status. */
GT_API int gt_column_names(const gt_params* params, char* buf, size_t buflen);

/* Locate (and link when has_search_range) T frames of H x W pixels held in
 * HOST memory (u16 or f32, C-contiguous).  Host->device and device->host
 * copies happen inside the call.  Replaces batch_rust / execute_ndarray. */
GT_API int gt_batch(gt_ctx* ctx, const void* frames, int dtype, int T, int H, int W,
             const gt_params* params, gt_table* out);

/* Same on DEVICE-resident frames.  The table is written to the device
 * buffer `d_out` (capacity out_rows x ncols floats); *nrows receives the row
 * count (rows beyond out_rows are not written, *nrows still reports them).
 * `stream` is a cudaStream_t (NULL = the context's stream); the call
 * returns after the work on it has finished. */
GT_API int gt_batch_device(gt_ctx* ctx, const void* d_frames, int dtype, int T, int H, int W,
                    const gt_params* params, float* d_out, int64_t out_rows,
                    int64_t* nrows, void* stream);

/* One movie of a batched call (gt_batch_many_device): device-resident
 * frames with their own shape, dtype and parameters, and the device buffer
 * that receives the movie's gt_batch_device table. */
typedef struct gt_movie {
    const void* frames;   /* T x H x W, u16 or f32, device */
    int32_t dtype;        /* gt_dtype */
    int32_t T, H, W;
    gt_params params;
    float* out;           /* out_rows x ncols f32, device (rows beyond are dropped) */
    int64_t out_rows;
    int64_t nrows;        /* written: rows of the movie's table */
} gt_movie;

/* Locate (and link) n movies of uneven sizes and parameters in one CUDA
 * graph launch on `stream`: the movies' locate / ordering / output kernels
 * run as parallel graph branches and all linking runs in one cooperative
 * kernel over every movie.  The graph is built on the first call and
 * replayed while the movies' pointers, shapes and parameters stay the same.
 * Tile rows of the specialised locate kernel are chosen per (frame size,
 * diameter) by timing both variants once per context.  A movie whose
 * per-frame capacities overflow is rerun through the gt_batch_device path.
 * Each movie's table equals what gt_batch_device returns for it.  No
 * reference counterpart (the reference processes one movie per call). */
GT_API int gt_batch_many_device(gt_ctx* ctx, gt_movie* movies, int n, void* stream);

/* gt_batch_device that also writes, for each output row r < out_rows, the
 * walk record d_walk[5r .. 5r+4] = {frame, last-read row, last-read column,
 * final row, final column} (int32, device).  The refined position is
 * (final + centroid at the last-read pixel), so these records are the fixed
 * peaks of the gt_adjoint_* calls.  No reference counterpart. */
GT_API int gt_batch_device_walk(gt_ctx* ctx, const void* d_frames, int dtype, int T, int H, int W,
                         const gt_params* params, float* d_out, int64_t out_rows,
                         int64_t* nrows, int32_t* d_walk, void* stream);

/* Bandpass + centroid refinement at fixed peaks (no reference counterpart;
 * the forward arithmetic is that of centers.wgsl:23-109 and
 * walk_cols.wgsl:38-74 over preprocess_rows/cols.wgsl).  d_frames: T x H x W
 * f32 on the device; d_walk: n walk records (gt_batch_device_walk).
 * Writes d_yxm (n x 3: y, x, mass), equal bit for bit to the located rows
 * for the frames and parameters that produced the walk records.  Params
 * follow gt_batch (diameter <= 31, max_iterations >= 1).  A walk record
 * outside the frames returns GT_ERR_ARG. */
GT_API int gt_adjoint_forward(gt_ctx* ctx, const float* d_frames, int T, int H, int W,
                       const gt_params* params, const int32_t* d_walk, int64_t n,
                       float* d_yxm, void* stream);

/* Adjoint of gt_adjoint_forward: given dL/d(y, x, mass) (d_grad_yxm, n x 3),
 * overwrites d_grad_frames (T x H x W f32, device) with dL/dframes and
 * d_grad_params (2 doubles, device) with dL/dnoise_size and
 * dL/dsmoothing_size.  The clip of the bandpass at 0 takes subgradient 0;
 * smoothing_size is differentiated through the box normalisation 1/k^2
 * treated as continuous in k (window and Gaussian taps held fixed).
 * d_grad_params is reduced in a fixed order (per-block partials, then one
 * ordered pass) and is the same on every run; d_grad_frames is summed with
 * atomic additions where particle circles overlap, so those pixels may
 * differ in the last bits from run to run. */
GT_API int gt_adjoint_backward(gt_ctx* ctx, const float* d_frames, int T, int H, int W,
                        const gt_params* params, const int32_t* d_walk, int64_t n,
                        const float* d_grad_yxm, float* d_grad_frames,
                        double* d_grad_params, void* stream);

/* Localisation uncertainty by linear propagation through the same Jacobian:
 * pixel variance gain * max(I, 0) + read_noise^2 (Poisson counts scaled by
 * the gain, plus read noise), independent pixels.  Writes the standard
 * deviations of (y, x, mass) to d_sd (n x 3, device). */
GT_API int gt_adjoint_uncertainty(gt_ctx* ctx, const float* d_frames, int T, int H, int W,
                           const gt_params* params, const int32_t* d_walk, int64_t n,
                           float gain, float read_noise, float* d_sd, void* stream);

/* Locate (and link) the frames of a movie FILE (execute_gpu.rs:510-542):
 * ".tif"/".tiff" -- every page a frame, 8- or 16-bit unsigned single-sample
 * pages (else GT_ERR_UNSUPPORTED "Wrong bit depth"), compression none, LZW,
 * Deflate or PackBits; ".ets" -- frames of `channel` (0 when has_channel is
 * 0), u16 only.  Frames are decoded by host threads into pinned memory and
 * uploaded in chunks that overlap the locate kernels.  Output as gt_batch. */
GT_API int gt_batch_file(gt_ctx* ctx, const char* path, int has_channel, uint32_t channel,
                  const gt_params* params, gt_table* out);

/* Frame count and size of a movie file as gt_batch_file reads it (for ETS,
 * H = dims[0] and W = dims[1], the order execute_gpu.rs:527 passes them). */
GT_API int gt_file_info(const char* path, int has_channel, uint32_t channel, int32_t* T, int32_t* H,
                 int32_t* W);

/* The frames themselves (T * H * W u16, host), e.g. for parse_ets. */
GT_API int gt_file_read(const char* path, int has_channel, uint32_t channel, uint16_t* out,
                 int64_t max_values);

/* Channels of an ETS file and their frame counts (up to max_channels), and
 * its two dimensions (decoderiter.rs:133-183). */
GT_API int gt_ets_channels(const char* path, int32_t* channels, int32_t* frames, int32_t max_channels,
                    int32_t* nchannels, int32_t* dim0, int32_t* dim1);

/* Link an (n x ncols) host f32 table whose columns 0, 2, 3 are frame, y, x
 * (link_rust's FrameSubsetter layout).  Writes n trajectory IDs. */
GT_API int gt_link(gt_ctx* ctx, const float* rows, int64_t n, int ncols, float search_range,
            int has_memory, uint32_t memory, uint64_t* ids);

/* Trajectory post-processing of a linked table, the lab pipeline's steps
 * after linking (all_cleaned_up/hatzakis_lab_tracking.py:216-230).  Host
 * arrays of n rows in table order; `ids` is the particle column as
 * integers.  Particles are taken in pandas' groupby order: ascending id,
 * the rows of a particle in table order. */

/* trackpy.filter_stubs(tracks, threshold) (hatzakis_lab_tracking.py:217):
 * keep[i] = 1 when ids[i] occurs in at least `threshold` rows, else 0;
 * *nkept = number of kept rows.  count (may be NULL) receives the number of
 * rows of each row's particle -- the duration column of line 223 for the
 * kept rows. */
GT_API int gt_filter_stubs(gt_ctx* ctx, const int64_t* ids, int64_t n, int64_t threshold, uint8_t* keep,
                           int64_t* count, int64_t* nkept);

/* step_tracker (hatzakis_lab_tracking.py:53-83): xs, ys = x * mpp, y * mpp
 * (float32, table order); then per particle the step from its previous row
 * (0 for its first row) and the step length sqrt(y_step^2 + x_step^2) in
 * float64 (the lab code turns the float32 values into Python floats with
 * tolist()).  x_step, y_step and steplength are in groupby order -- the
 * sequence step_tracker assigns to the table by position -- and order[j] is
 * the table row of entry j. */
GT_API int gt_steps(gt_ctx* ctx, const int64_t* ids, const float* x, const float* y, int64_t n, double mpp,
                    float* xs, float* ys, double* x_step, double* y_step, double* steplength, int64_t* order);

/* Per-particle mean squared displacement, trackpy.msd(traj, mpp, fps,
 * max_lagtime) of every particle concatenated and stacked as mp_imsd and
 * tracker() do (hatzakis_lab_tracking.py:199-214, 230-232): positions
 * xy * mpp (float32) on the frame axis from a particle's first to its last
 * frame; for lag L = 1 .. min(max_lagtime, span - 1) the mean over pairs
 * with both frames present of the squared x and y differences, summed.
 * *out is an (m x 3) table (lag, particle, msd), ordered by lag then
 * particle, without lags that have no pair; particle ids must lie in
 * [0, 2^24).  A particle with two rows in one frame is GT_ERR_ARG (trackpy
 * refuses it: one trajectory per particle).  Release with gt_table_free. */
GT_API int gt_imsd(gt_ctx* ctx, const int64_t* ids, const int64_t* frames, const float* x, const float* y,
                   int64_t n, double mpp, int64_t max_lagtime, gt_table* out);

/* Locate (no linking) ONE device-resident frame while allocating nothing,
 * for callers that cannot call cudaMalloc: processes whose device memory
 * belongs to another framework's pool (an allocation beside it can fail or
 * fragment it) and acquisition loops that forbid allocation once running.
 * No counterpart in the reference.  Frames up to 2^20 pixels (H, W <= 8192)
 * and 32768 features before the separation filter (more is
 * GT_ERR_CAPACITY); sig_radius/bg_radius <= 31; search_range must be unset.
 * Writes min(*nrows, out_rows) rows of the gt_batch_device columns to d_out
 * (device) and the row count to *nrows, on `stream` (a cudaStream_t, NULL =
 * default stream), returning after the work has finished: the call waits on
 * the stream and reads its row count back to the host.  Scratch
 * lives in one 16 MiB __device__ array per GPU, held until the process
 * exits and shared by every call, which clears what must start at zero:
 * calls that overlap on one GPU (other streams, other host threads) race on
 * it and must be serialised by the caller.  The first call on a device looks
 * up that array's address and sets up the device (under a lock, so threads
 * may call concurrently for different GPUs); make that first call before any
 * stream capture.  Errors: gt_last_error(NULL) of the calling thread. */
GT_API int gt_locate_frame_static(const void* d_frame, int dtype, int H, int W, const gt_params* params,
                                  float* d_out, int64_t out_rows, int64_t* nrows, void* stream);

/* Free a table returned by gt_batch. */
GT_API void gt_table_free(gt_table* table);

/* Options of a context (no reference counterpart):
 *   "locate_tile_rows"  output tile height of the specialised locate kernel, 32 or 64
 *   "force_generic"     1 = always use the generic locate kernel
 *   "locate_tiles_per_cta"
 *                       output tiles located one after another by a CTA of
 *                       the specialised kernel, 1-64 (0 = the default: up to
 *                       16, as long as a launch keeps about four waves of CTAs)
 *   "autotune"          0 = gt_batch_many_device keeps the configured tile rows
 *   "normalized_taps"   1 = Gaussian taps divided by their sum on the host and
 *                       no division in the passes (kernels.rs:86-97 gauss_1d,
 *                       the form of the reference's own mass-plane dump);
 *                       0 (default) = the live shaders' in-pass normalisation
 *   "subnet_budget"     option trials per linking subnetwork before
 *                       GT_ERR_SUBNET_BUDGET (0 = the default, 2^26)
 *   "test_withhold_tile_copy"
 *                       1 = the specialised locate kernel issues no TMA copy of
 *                       its tiles, so its bounded wait runs out after a short
 *                       limit and the call returns GT_ERR_DEVICE_TIMEOUT (a
 *                       test of the timeout path; no fault, nothing in flight)
 * Returns GT_ERR_ARG for an unknown key or value. */
GT_API int gt_ctx_set_option(gt_ctx* ctx, const char* key, int value);

/* Statistics of the last call on this context: fixed-point iterations of the
 * memory linker, fallback walks, candidates and particles. */
typedef struct gt_stats {
    int32_t link_iterations;   /* fixed-point passes of the memory linker */
    int32_t fallback_walks;    /* walks that left a tile's halo */
    int64_t candidates;        /* located features before the separation filter */
    int64_t particles;         /* rows of the output table */
    int32_t retries;           /* capacity retries */
    int32_t launches;          /* kernels launched by the call */
    float ms_locate;           /* device time of the locate kernel(s) */
    float ms_finalize;         /* fallback walks + ordering + separation filter */
    float ms_link;             /* linking incl. fixed-point passes and ids */
    float ms_assemble;         /* output table */
    float ms_total;            /* first to last kernel of the call */
    int32_t locate_kernel;     /* 0 generic, 1 specialised, 2 specialised with TMA staging */
    float link_phase_ms[4];    /* linker: first pass, roots, memory entries, relinking */
    int32_t link_dirty[8];     /* frames relinked by fixed-point passes 1..8 */
    float ms_adjoint_particles; /* gt_adjoint_*: per-particle kernel */
    float ms_adjoint_dense;     /* gt_adjoint_backward: zeroing + transposed bandpass */
    int32_t batch_graph;        /* gt_batch_many_device: 2 graph replayed, 1 graph built, 0 no graph */
    int32_t batch_fallbacks;    /* gt_batch_many_device: movies rerun through gt_batch_device */
    float ms_msd;               /* gt_imsd: device time of the per-particle MSD kernel */
} gt_stats;

GT_API int gt_last_stats(const gt_ctx* ctx, gt_stats* out);

#ifdef __cplusplus
}
#endif
#endif /* GT_H */
