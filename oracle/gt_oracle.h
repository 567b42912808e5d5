/*
 * gt_oracle.h -- CPU restatement of gpu_tracking's locate-and-link path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * product path: only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg (and its `--impl reference` arm) load it.  The product
 * library never links or calls it.
 *
 * Parity status: UNPINNED against the reference binary.  The reference's
 * GPU path is WGSL through wgpu (needs Vulkan/DX12/Metal; none exists here or
 * on the GPU hosts) and its host code is Rust (no cargo/rustc here), and the
 * reference ships no tests or golden vectors for this path.  The restatement
 * is pinned instead by hand-derived known-answer tests (tests/test_oracle_kat.py)
 * written from the reference source, and every function below cites the
 * reference lines it restates.
 *
 * Two documented choices where the reference itself is not reproducible:
 *   - `acc += a * b` in the WGSL shaders is evaluated as a fused multiply-add
 *     (SPIR-V permits contraction; NVIDIA's Vulkan compiler contracts).
 *   - The third-party kd-tree 0.4.2 iteration order (separation-filter output
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
                 float noise_size, float* processed);

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
