/*
 * gt_oracle.h -- CPU restatement of gpu_tracking's locate-and-link path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * product path: only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg (and its `--impl reference` arm) load it.  The product
 * library never links or calls it.
 *
 * Parity status: PINNED against the reference's own output for the
 * bandpass and centroid-mass stages.  The reference ships a dump of the
 * masses plane of its GPU path (gpu-tracking/masses.bin, centers.wgsl over
 * the 524 x 800 image gpu-tracking/inp, diameter 9, smoothing_size 9,
 * noise_size 1, taps normalised on the host as kernels.rs:86-97 does), and
 * this restatement reproduces it bit for bit on all 419,200 pixels
 * (tests/test_reference_dump.py).  That dump fixes the reference GPU's
 * arithmetic conventions, which the restatement follows everywhere:
 *   - `acc += a * b` is a fused multiply-add (the compiler contracts it);
 *   - a division `a / b` is a multiplication by the reciprocal of b (taken
 *     correctly rounded), and `a - b / c` contracts into
 *     fma(-b, 1/c, a).
 * The rest of the path (walk, separation filter, linking) is integer/index
 * work or host Rust code with IEEE arithmetic, restated line by line; the
 * reference binary itself cannot run here (Rust host, WGSL through wgpu).
 *
 * Documented choices where the reference itself is not reproducible:
 *   - the live shaders compute the Gaussian taps with the GPU's exp(); the
 *     restatement takes the C library's expf (the dump, made with taps
 *     from Rust's f32::exp on the host, does not pin the GPU's exp);
 *   - the third-party kd-tree 0.4.2 iteration order (separation-filter output
 *     order, link neighbour order, new-ID order) is replaced by canonical
 *     raster order of each feature's originating pixel, and neighbour lists in
 *     ascending index order.
 */
#ifndef GT_ORACLE_H
#define GT_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_params {
    int32_t diameter;
    float minmass;
    int32_t separation;
    float noise_size;
    int32_t smoothing_size;
    int32_t max_iterations;
    int32_t characterize;
    int32_t cpu_processed;
    int32_t has_search_range;
    float search_range;
    int32_t memory;
    int32_t has_sig_radius;
    float sig_radius;
    int32_t has_bg_radius;
    float bg_radius;
    float gap_radius;
    int32_t normalized_taps;  /* 1: taps divided by their sum on the host
                                 (kernels.rs:86-97), no division in the passes */
} or_params;

/* Full locate (+ link when has_search_range) over T frames of f32 pixels.
 * fp64 != 0 runs the locate arithmetic in double (accuracy reference).
 * *out is malloc'd (nrows x ncols, row-major f32); free with or_free.
 * Returns 0 on success, 4 when a subnet exceeded the node budget. */
int or_batch(const float* frames, int T, int H, int W, const or_params* p,
             int nthreads, int fp64, float** out, int64_t* nrows, int* ncols);

/* or_batch (FP32) that also returns, per output row, the walk record
 * {frame, last-read row, last-read column, final row, final column}
 * (malloc'd n x 5 int32; free with or_free). */
int or_batch_walk(const float* frames, int T, int H, int W, const or_params* p, int nthreads,
                  float** out, int64_t* nrows, int* ncols, int32_t** walk);

/* Same as or_batch on uint16 pixels (converted exactly to f32). */
int or_batch_u16(const uint16_t* frames, int T, int H, int W, const or_params* p,
                 int nthreads, int fp64, float** out, int64_t* nrows, int* ncols);

/* Standalone linking of a (frame, mass, y, x, ...) f32 table: ids[n]. */
int or_link(const float* rows, int64_t n, int ncols, float search_range,
            int memory, uint64_t* ids);

/* Bandpass of one frame (FP32 restatement); processed is H*W. */
void or_bandpass(const float* frame, int H, int W, int smoothing_size,
                 float noise_size, int normalized_taps, float* processed);

/* Dense centers (c0, c1) and masses planes of centers.wgsl at every pixel
 * (H*W floats each; zeros in the border band). */
void or_centers(const float* frame, int H, int W, const or_params* p, float* c0, float* c1,
                float* mass);

/* Raw results planes of the locate shaders for one frame: mass, y, x at the
 * originating pixel (3*H*W floats, zero where nothing was emitted). */
void or_locate_planes(const float* frame, int H, int W, const or_params* p,
                      float* planes);

/* Derived dilation size and its window offset. */
void or_dilation(int separation, int* size, int* offset);

void or_free(void* ptr);

#ifdef __cplusplus
}
#endif
#endif
