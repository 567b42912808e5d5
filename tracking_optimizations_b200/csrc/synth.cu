// synth.cu -- synthetic movies rendered on the device, for workloads too
// large to generate on the host (tens of GB of u16 frames).
//
// Same model as the host generator (tracking_optimizations_b200/synth.py):
// background Poisson(lambda) plus N(0, read_noise^2) per pixel, plus spots
// A * exp(-r^2 / (2 sigma^2)) sampled at pixel centres within ceil(4 sigma)
// of the rounded spot centre, rounded to the nearest integer and clipped to
// [0, 65535].  Spot positions and amplitudes (with blinking as amplitude 0)
// come from the caller, one (y, x, A) triple per spot and frame.
//
// Random numbers: Philox4x32-10 (J. Salmon, M. Moraes, R. Dror, D. Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC 2011), keyed by the
// seed and counted by (pixel, frame, draw), so the frames do not depend on
// the chunking.  Poisson variates by Knuth's multiplication method on
// sub-rates of at most 25 (a sum of independent Poisson variates is Poisson
// with the summed rate); normal variates by the Box-Muller transform.
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>
#include <algorithm>

#include "gt_synth.h"

namespace {

struct U4 {
    uint32_t x, y, z, w;
};

__device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
        const uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
        c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
        k0 += W0;
        k1 += W1;
    }
    return c;
}

// uniform in (0, 1]
__device__ __forceinline__ float unit(uint32_t v) { return ((float)(v >> 8) + 1.0f) * (1.0f / 16777216.0f); }

struct Stream {
    U4 ctr;
    uint32_t k0, k1;
    U4 buf;
    int left;
    __device__ float next() {
        if (left == 0) {
            buf = philox4x32_10(ctr, k0, k1);
            ctr.z += 1;
            left = 4;
        }
        const uint32_t v = left == 4 ? buf.x : left == 3 ? buf.y : left == 2 ? buf.z : buf.w;
        --left;
        return unit(v);
    }
};

__global__ void background_kernel(float* S, int nf, int H, int W, int frame0, float lam, float read_noise,
                                  uint32_t k0, uint32_t k1) {
    const size_t n = (size_t)nf * H * W;
    const int parts = (int)ceilf(lam / 25.0f);
    const float sub = parts > 0 ? lam / (float)parts : 0.f;
    const float lim = expf(-sub);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const size_t f = i / ((size_t)H * W), px = i - f * (size_t)H * W;
        Stream s{U4{(uint32_t)px, (uint32_t)(frame0 + f), 0u, 0x5eedu}, k0, k1, U4{0, 0, 0, 0}, 0};
        int k = 0;
        for (int q = 0; q < parts; ++q) {
            // Knuth: smallest j with u_1 ... u_j <= exp(-sub), minus one;
            // bounded at 64 * sub + 64 draws (tail probability < 1e-30)
            float p = 1.0f;
            int j = 0;
            const int cap = (int)(64.0f * sub) + 64;
            do {
                p *= s.next();
                ++j;
            } while (p > lim && j < cap);
            k += j - 1;
        }
        float v = (float)k;
        if (read_noise > 0.f) {
            const float u1 = s.next(), u2 = s.next();
            v += read_noise * sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);
        }
        S[i] = v;
    }
}

__global__ void spots_kernel(float* S, const float* spots, int N, int nf, int H, int W, int frame0, float sigma,
                             int R) {
    const int side = 2 * R + 1;
    const size_t per_frame = (size_t)N * side * side;
    const size_t n = (size_t)nf * per_frame;
    const float inv2s2 = 1.0f / (2.0f * sigma * sigma);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const size_t f = i / per_frame;
        const size_t rem = i - f * per_frame;
        const int sp = (int)(rem / (side * side));
        const int q = (int)(rem - (size_t)sp * side * side);
        const float* t = spots + ((size_t)(frame0 + f) * N + sp) * 3;
        const float a = t[2];
        if (a == 0.f) continue;
        const float y = t[0], x = t[1];
        const int r = (int)rintf(y) + q / side - R, c = (int)rintf(x) + q % side - R;
        if (r < 0 || r >= H || c < 0 || c >= W) continue;
        const float dy = (float)r - y, dx = (float)c - x;
        atomicAdd(S + f * (size_t)H * W + (size_t)r * W + c, a * expf(-(dy * dy + dx * dx) * inv2s2));
    }
}

__global__ void quantize_kernel(const float* S, uint16_t* out, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float v = rintf(S[i]);
        out[i] = (uint16_t)fminf(fmaxf(v, 0.f), 65535.f);
    }
}

}  // namespace

extern "C" GT_API int gt_synth_render(const float* d_spots, int N, int T, int H, int W, float sigma, float background,
                               float read_noise, uint64_t seed, uint16_t* d_frames, float* d_scratch,
                               int chunk_frames, void* stream) {
    if (!d_frames || !d_scratch || (N > 0 && !d_spots) || T < 1 || H < 1 || W < 1 || N < 0 || chunk_frames < 1 ||
        !(sigma > 0.f) || !(background >= 0.f) || !(read_noise >= 0.f))
        return 1;
    cudaStream_t st = (cudaStream_t)stream;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int R = (int)ceilf(4.0f * sigma);
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    for (int f0 = 0; f0 < T; f0 += chunk_frames) {
        const int nf = std::min(chunk_frames, T - f0);
        const size_t n = (size_t)nf * H * W;
        background_kernel<<<sms * 8, 256, 0, st>>>(d_scratch, nf, H, W, f0, background, read_noise, k0, k1);
        if (N > 0) spots_kernel<<<sms * 8, 256, 0, st>>>(d_scratch, d_spots, N, nf, H, W, f0, sigma, R);
        quantize_kernel<<<sms * 8, 256, 0, st>>>(d_scratch, d_frames + (size_t)f0 * H * W, n);
    }
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}
