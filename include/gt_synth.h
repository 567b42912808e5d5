/* gt_synth.h -- synthetic movie renderer of libgt (workload generator; no
 * reference counterpart).
 *
 * Renders T frames of H x W u16 pixels on the device with the spot model of
 * tracking_optimizations_b200/synth.py: background Poisson(background) plus
 * N(0, read_noise^2), plus Gaussian spots A exp(-r^2 / (2 sigma^2)) sampled
 * at pixel centres within ceil(4 sigma) of the rounded centre; rounded and
 * clipped to [0, 65535].  Spots: d_spots[(t * N + s) * 3 + {0, 1, 2}] =
 * (y, x, A) on the device, A = 0 for a spot that is off in frame t.
 * Random numbers: Philox4x32-10 keyed by `seed`.  d_scratch holds
 * chunk_frames * H * W floats.  Returns 0, 1 for an invalid argument, 2 for
 * a CUDA launch error.  Asynchronous on `stream`.
 */
#ifndef GT_SYNTH_H
#define GT_SYNTH_H
#include <stdint.h>

#if defined(__GNUC__)
#ifndef GT_API
#define GT_API __attribute__((visibility("default")))
#endif
#else
#ifndef GT_API
#define GT_API
#endif
#endif

#ifdef __cplusplus
extern "C" {
#endif

GT_API int gt_synth_render(const float* d_spots, int N, int T, int H, int W, float sigma, float background,
                           float read_noise, uint64_t seed, uint16_t* d_frames, float* d_scratch,
                           int chunk_frames, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* GT_SYNTH_H */
