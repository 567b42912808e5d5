// adjoint.cu -- bandpass + centroid refinement at fixed peaks, its adjoint
// and the per-particle localisation uncertainty.
//
// At a fixed walk (last-read pixel (ul, vl), final position (up, vp)) a
// located feature is a smooth function of the frame away from the clip:
//
//   R(p) = G(p) - B(p)             bandpass before the clip, G the Gaussian
//                                  pass (zero padded, normalised by the full
//                                  tap sum), B the boxcar mean (reflect
//                                  padded, divided by k*k)
//   P(p) = max(R(p), 0)
//   m    = sum_c P(ul + i_c, vl + j_c)          over the centroid circle
//   y    = up + sum_c i_c P(..) / m,  x = vp + sum_c j_c P(..) / m
//
// (walk_cols.wgsl:38-74, centers.wgsl:23-109, preprocess_rows.wgsl:14-53,
// preprocess_cols.wgsl:14-61).  The forward kernel re-evaluates the bandpass
// at the circle pixels with the locate kernels' exact operation order, so
// its (y, x, mass) equal the located rows bit for bit.  The backward pass
// recomputes the same bandpass values (nothing from the forward is stored),
// scatters dL/dR onto a zeroed plane and applies the transposed bandpass as
// one dense stencil pass.  The clip has subgradient 0 at R == 0.
//
// Parameter derivatives: noise_size is the Gaussian variance s, and
// dG/ds = (da (x) a + a (x) da) * I with a_i = w_i / sum(w).  smoothing_size
// k is an integer window; its derivative is taken through the box
// normalisation 1/k^2 treated as continuous (window and Gaussian tap count
// held fixed): dR/dk = 2 B / k.
#include <cuda_runtime.h>
#include <algorithm>
#include "gt_internal.cuh"

namespace gt {

namespace {

constexpr int ADJ_NT = 128;
constexpr int TR_TH = 32, TR_TW = 64, TR_NT = 256;

struct BpTerms {
    float r;      // bandpass before the clip
    float bmean;  // boxcar mean B
    float dg;     // dG/ds
};

// The bandpass at (u, v) in the operation order of the locate kernels
// (row pass: fmaf over taps, times the reciprocal of the tap sum; column
// pass likewise, boxcar subtracted as fma(-box, 1/k^2, gauss); box sums in
// tap order), plus B and dG/ds in real-valued arithmetic.
__device__ __forceinline__ BpTerms bandpass_terms(const AdjParams& p, const float* fr, int u, int v) {
    const int kr = p.krad, H = p.H, W = p.W;
    float gs = 0.f, cs = 0.f, dg = 0.f;
    for (int i = -kr; i <= kr; ++i) {
        int pu = u + i;
        bool in_r = true;
        if (pu < 0) { pu = -pu - 1; in_r = false; }
        else if (pu >= H) { pu = 2 * H - pu - 1; in_r = false; }
        float rg = 0.f, rb = 0.f, ra = 0.f, rda = 0.f;
        const float* row = fr + (size_t)pu * W;
        for (int j = -kr; j <= kr; ++j) {
            int pv = v + j;
            bool in_c = true;
            if (pv < 0) { pv = -pv - 1; in_c = false; }
            else if (pv >= W) { pv = 2 * W - pv - 1; in_c = false; }
            const float val = __ldg(row + pv);
            if (in_c) {
                rg = fmaf(p.w[j + kr], val, rg);
                ra = fmaf(p.a[j + kr], val, ra);
                rda = fmaf(p.da[j + kr], val, rda);
            }
            rb = rb + val;
        }
        const float tg = rg * p.rn;
        if (in_r) {
            gs = fmaf(p.w[i + kr], tg, gs);
            dg = fmaf(p.da[i + kr], ra, dg);
            dg = fmaf(p.a[i + kr], rda, dg);
        }
        cs = cs + rb;
    }
    BpTerms t;
    t.r = fmaf(-cs, p.rkk, gs * p.rn);
    t.bmean = cs * p.rkk;
    t.dg = dg;
    return t;
}

// Number of taps of the reflect-padded box at p (window +-kr, one
// reflection) that land on q, along one axis of length n.
__device__ __forceinline__ int box_count(int pp, int q, int n, int kr) {
    return (abs(q - pp) <= kr) + (abs(-q - 1 - pp) <= kr) + (abs(2 * n - q - 1 - pp) <= kr);
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;  // every lane
}

}  // namespace

enum AdjMode { ADJ_FORWARD = 0, ADJ_BACKWARD = 1, ADJ_UNCERTAINTY = 2 };

// One warp per particle (grid-stride over warps), ADJ_NT / 32 warps per
// CTA sharing the circle table.  walk rows: {frame, ul, vl, up, vp}.
// FORWARD writes yxm (n x 3).  BACKWARD reads grad (n x 3), adds dL/dR into
// the zeroed plane gR (T x H x W) and dL/d{noise_size, smoothing_size} into
// gpar.  UNCERTAINTY writes the standard deviations of (y, x, mass) under
// var(I) = gain * max(I, 0) + read_var by linear propagation (n x 3).
template <int MODE>
__global__ void __launch_bounds__(ADJ_NT) adjoint_particle_kernel(AdjParams p, const float* __restrict__ frames,
                                                                  const int* __restrict__ walk, long long n,
                                                                  const int* __restrict__ circ,
                                                                  const float* __restrict__ grad, float* yxm,
                                                                  float* gR, double* gpar, int* err) {
    extern __shared__ __align__(16) float asm_[];
    constexpr int NW = ADJ_NT / 32;
    const int K = p.K;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int* sci = (int*)asm_;                      // 2K circle offsets {i, j}, shared
    float* sR = asm_ + 2 * K + wid * 6 * K;     // this warp's R at the circle pixels
    float* sB = sR + K;                         // B
    float* sD = sB + K;                         // dG/ds
    float* sJ = sD + K;                         // 3K: dy/dR, dx/dR, dm/dR (uncertainty)
    for (int q = threadIdx.x; q < 2 * K; q += ADJ_NT) sci[q] = circ[q];
    __syncthreads();
    const int H = p.H, W = p.W, kr = p.krad, b = p.border;
    const long long wstride = (long long)gridDim.x * NW;
    double acc_ds = 0.0, acc_dk = 0.0;  // this warp's parameter gradients (BACKWARD)
    for (long long k = (long long)blockIdx.x * NW + wid; k < n; k += wstride) {
        const int* wr = walk + 5 * k;
        const int t = __ldg(wr), ul = __ldg(wr + 1), vl = __ldg(wr + 2), up = __ldg(wr + 3), vp = __ldg(wr + 4);
        const bool valid = t >= 0 && t < p.T && ul >= 0 && ul < H && vl >= 0 && vl < W && up >= 0 && up < H &&
                           vp >= 0 && vp < W;
        if (!valid) {
            if (lane == 0) atomicOr(err, 1);
            continue;
        }
        const bool interior = !(ul - b < 0 || ul + b >= H || vl - b < 0 || vl + b >= W);
        if (!interior) {
            // centers.wgsl border band: offset (0, 0), mass 0, no dependence
            // on the frame
            if (lane == 0) {
                if (MODE == ADJ_FORWARD) {
                    yxm[3 * k] = (float)up; yxm[3 * k + 1] = (float)vp; yxm[3 * k + 2] = 0.f;
                } else if (MODE == ADJ_UNCERTAINTY) {
                    yxm[3 * k] = 0.f; yxm[3 * k + 1] = 0.f; yxm[3 * k + 2] = 0.f;
                }
            }
            continue;
        }
        const float* fr = frames + (size_t)t * H * W;
        __syncwarp();  // the previous particle's reads of this warp's arrays are done
        for (int c = lane; c < K; c += 32) {
            const BpTerms bt = bandpass_terms(p, fr, ul + sci[2 * c], vl + sci[2 * c + 1]);
            sR[c] = bt.r;
            sB[c] = bt.bmean;
            sD[c] = bt.dg;
        }
        __syncwarp();
        float c0 = 0.f, c1 = 0.f, m = 0.f;
        if (lane == 0) {
            // centers.wgsl:23-109 accumulation order (i outer, j inner)
            float a0 = 0.f, a1 = 0.f, mm = 0.f;
            for (int c = 0; c < K; ++c) {
                const float data = sR[c] < 0.f ? 0.f : sR[c];
                a0 = fmaf(data, (float)sci[2 * c], a0);
                a1 = fmaf(data, (float)sci[2 * c + 1], a1);
                mm = mm + data;
            }
            c0 = __fmul_rn(a0, __frcp_rn(mm));  // centers.wgsl:82-83, a shader division
            c1 = __fmul_rn(a1, __frcp_rn(mm));
            m = mm;
        }
        c0 = __shfl_sync(0xffffffffu, c0, 0);
        c1 = __shfl_sync(0xffffffffu, c1, 0);
        m = __shfl_sync(0xffffffffu, m, 0);
        if constexpr (MODE == ADJ_FORWARD) {
            if (lane == 0) {
                yxm[3 * k] = (float)up + c0;
                yxm[3 * k + 1] = (float)vp + c1;
                yxm[3 * k + 2] = m;
            }
            continue;
        }
        if (!(m > 0.f) || !isfinite(m)) {
            // zero mass: the centroid is undefined and the row is never
            // emitted (mass > minmass and mass != 0)
            if (MODE == ADJ_UNCERTAINTY && lane == 0) {
                yxm[3 * k] = 0.f; yxm[3 * k + 1] = 0.f; yxm[3 * k + 2] = 0.f;
            }
            continue;
        }
        const float inv_m = 1.f / m;
        if constexpr (MODE == ADJ_BACKWARD) {
            const float gy = __ldg(grad + 3 * k), gx = __ldg(grad + 3 * k + 1), gm = __ldg(grad + 3 * k + 2);
            float ds = 0.f, dk = 0.f;
            float* plane = gR + (size_t)t * H * W;
            for (int c = lane; c < K; c += 32) {
                if (!(sR[c] > 0.f)) continue;
                const float ic = (float)sci[2 * c], jc = (float)sci[2 * c + 1];
                const float g = gm + (gy * (ic - c0) + gx * (jc - c1)) * inv_m;
                atomicAdd(plane + (size_t)(ul + sci[2 * c]) * W + (vl + sci[2 * c + 1]), g);
                ds = fmaf(g, sD[c], ds);
                dk = fmaf(g, 2.f * sB[c] / p.k, dk);
            }
            acc_ds += (double)warp_sum(ds);
            acc_dk += (double)warp_sum(dk);
            continue;
        }
        if constexpr (MODE == ADJ_UNCERTAINTY) {
            // Jacobian rows over the window that the circle's bandpass
            // reads, J(q) = sum_c dR_c/dI(q) * dOut/dR_c
            for (int c = lane; c < K; c += 32) {
                const bool on = sR[c] > 0.f;
                sJ[c] = on ? ((float)sci[2 * c] - c0) * inv_m : 0.f;
                sJ[K + c] = on ? ((float)sci[2 * c + 1] - c1) * inv_m : 0.f;
                sJ[2 * K + c] = on ? 1.f : 0.f;
            }
            __syncwarp();
            const int WR = p.rc + kr, WS = 2 * WR + 1;
            float vy = 0.f, vx = 0.f, vm = 0.f;
            for (int q = lane; q < WS * WS; q += 32) {
                const int qu = ul - WR + q / WS, qv = vl - WR + q % WS;
                if (qu < 0 || qu >= H || qv < 0 || qv >= W) continue;
                float jy = 0.f, jx = 0.f, jm = 0.f;
                for (int c = 0; c < K; ++c) {
                    const int pu = ul + sci[2 * c], pv = vl + sci[2 * c + 1];
                    const int du = qu - pu, dv = qv - pv;
                    float wgt = 0.f;
                    if (abs(du) <= kr && abs(dv) <= kr) wgt = p.a[du + kr] * p.a[dv + kr];
                    const int nb = box_count(pu, qu, H, kr) * box_count(pv, qv, W, kr);
                    if (nb) wgt -= (float)nb / p.kk;
                    jy = fmaf(sJ[c], wgt, jy);
                    jx = fmaf(sJ[K + c], wgt, jx);
                    jm = fmaf(sJ[2 * K + c], wgt, jm);
                }
                const float iq = __ldg(fr + (size_t)qu * W + qv);
                const float var = fmaf(p.gain, fmaxf(iq, 0.f), p.read_var);
                vy = fmaf(jy * jy, var, vy);
                vx = fmaf(jx * jx, var, vx);
                vm = fmaf(jm * jm, var, vm);
            }
            const float ty = warp_sum(vy), tx = warp_sum(vx), tm = warp_sum(vm);
            if (lane == 0) {
                yxm[3 * k] = sqrtf(ty);
                yxm[3 * k + 1] = sqrtf(tx);
                yxm[3 * k + 2] = sqrtf(tm);
            }
        }
    }
    if constexpr (MODE == ADJ_BACKWARD) {
        // this block's partial sums, in warp order; adjoint_param_reduce_kernel
        // adds the blocks' partials in block order, so the parameter
        // gradient is the same on every run (particles map to warps and
        // blocks by a fixed grid stride)
        __shared__ double red[2 * NW];
        if (lane == 0) { red[2 * wid] = acc_ds; red[2 * wid + 1] = acc_dk; }
        __syncthreads();
        if (threadIdx.x == 0) {
            double a = 0.0, c = 0.0;
            for (int w = 0; w < NW; ++w) { a += red[2 * w]; c += red[2 * w + 1]; }
            gpar[2 * blockIdx.x] = a;
            gpar[2 * blockIdx.x + 1] = c;
        }
    }
}

// out[0..1] = the sums of part[2b], part[2b + 1] over blocks b in a fixed
// order: thread i takes blocks i, i + 256, ... in order, then a fixed tree.
__global__ void __launch_bounds__(256) adjoint_param_reduce_kernel(const double* part, int nblocks, double* out) {
    __shared__ double sa[256], sc[256];
    double a = 0.0, c = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += 256) {
        a += part[2 * b];
        c += part[2 * b + 1];
    }
    sa[threadIdx.x] = a;
    sc[threadIdx.x] = c;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            sa[threadIdx.x] += sa[threadIdx.x + h];
            sc[threadIdx.x] += sc[threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = sa[0];
        out[1] = sc[0];
    }
}

// Transposed bandpass of dL/dR:  dL/dI = G^T gR - B^T gR.  G is separable,
// symmetric and zero padded, so G^T is the same Gaussian pass; B^T weights
// each tap by the number of reflect-padded window positions that land on it
// (box_count), all of which lie within +-kr of the output pixel.  One CTA per
// 32 x 64 output tile, gR staged with a kr halo (zero outside the frame).
template <int KRT>  // smoothing half window; 0 = taken from p.krad at run time
__global__ void __launch_bounds__(TR_NT) adjoint_transpose_kernel(AdjParams p, const float* __restrict__ gR,
                                                                  float* __restrict__ gI) {
    extern __shared__ __align__(16) float tsm[];
    const int kr = KRT > 0 ? KRT : p.krad;
    const int H = p.H, W = p.W;
    const int SH = TR_TH + 2 * kr, SW = TR_TW + 2 * kr;
    constexpr int RS = TR_TW + 1;  // row stride of the row-pass planes (odd: conflict-free column reads)
    float* S = tsm;               // SH x SW
    float* RG = S + SH * SW;      // SH x RS, Gaussian row pass
    float* RB = RG + SH * RS;     // SH x RS, box row pass
    const int ntx = (W + TR_TW - 1) / TR_TW;
    const int u0 = (blockIdx.x / ntx) * TR_TH, v0 = (blockIdx.x % ntx) * TR_TW;
    const int t = blockIdx.y;
    const float* src = gR + (size_t)t * H * W;
    for (int q = threadIdx.x; q < SH * SW; q += TR_NT) {
        const int r = q / SW, c = q - r * SW;
        const int gu = u0 - kr + r, gv = v0 - kr + c;
        S[q] = (gu >= 0 && gu < H && gv >= 0 && gv < W) ? __ldg(src + (size_t)gu * W + gv) : 0.f;
    }
    __syncthreads();
    // away from the frame edges every box tap counts once
    const bool cols_inner = v0 >= kr && v0 + TR_TW <= W - kr;
    const bool rows_inner = u0 >= kr && u0 + TR_TH <= H - kr;
    if (KRT > 0 && cols_inner) {
        // 8 outputs of one row per item (taps loaded once), rows fastest
        // across the lanes
        constexpr int TP = 2 * KRT + 1, RF = 8, NCH = TR_TW / RF;
        float a[TP];
#pragma unroll
        for (int j = 0; j < TP; ++j) a[j] = p.a[j];
        for (int it = threadIdx.x; it < SH * NCH; it += TR_NT) {
            const int ch = it / SH, r = it - ch * SH;
            const int c0 = ch * RF;
            const float* srow = S + r * SW + c0;
            float v[RF + TP - 1];
#pragma unroll
            for (int i = 0; i < RF + TP - 1; ++i) v[i] = srow[i];
            float* rg = RG + r * RS + c0;
            float* rb = RB + r * RS + c0;
#pragma unroll
            for (int m = 0; m < RF; ++m) {
                float g = 0.f;
#pragma unroll
                for (int j = 0; j < TP; ++j) g = fmaf(a[j], v[m + j], g);
                rg[m] = g;
            }
            // direct sums, not a running difference: a window of zeros
            // must give exactly zero (no gradient outside the particles)
#pragma unroll
            for (int m = 0; m < RF; ++m) {
                float bs = 0.f;
#pragma unroll
                for (int j = 0; j < TP; ++j) bs = bs + v[m + j];
                rb[m] = bs;
            }
        }
    } else {
        for (int q = threadIdx.x; q < SH * TR_TW; q += TR_NT) {
            const int r = q / TR_TW, c = q % TR_TW;
            const int qv = v0 + c;
            float g = 0.f, bx = 0.f;
            const float* srow = S + r * SW + c + kr;
            if (qv < W) {
                for (int j = -kr; j <= kr; ++j) {
                    const float v = srow[j];
                    g = fmaf(p.a[j + kr], v, g);
                    const int pv = qv + j;
                    if (pv >= 0 && pv < W) bx = fmaf((float)box_count(pv, qv, W, kr), v, bx);
                }
            }
            RG[r * RS + c] = g;
            RB[r * RS + c] = bx;
        }
    }
    __syncthreads();
    float* dst = gI + (size_t)t * H * W;
    const float ikk = 1.f / p.kk;
    if (KRT > 0 && rows_inner && v0 + TR_TW <= W) {
        // 8 outputs of one column per item, columns fastest across the lanes
        constexpr int TP = 2 * KRT + 1, CF = 8;
        float a[TP];
#pragma unroll
        for (int j = 0; j < TP; ++j) a[j] = p.a[j];
        for (int it = threadIdx.x; it < TR_TW * (TR_TH / CF); it += TR_NT) {
            const int c = it % TR_TW, r0 = (it / TR_TW) * CF;
            float g[CF + TP - 1], b[CF + TP - 1];
#pragma unroll
            for (int i = 0; i < CF + TP - 1; ++i) {
                g[i] = RG[(r0 + i) * RS + c];
                b[i] = RB[(r0 + i) * RS + c];
            }
#pragma unroll
            for (int m = 0; m < CF; ++m) {
                float bs = 0.f;
#pragma unroll
                for (int i = 0; i < TP; ++i) bs = bs + b[m + i];
                float gs = 0.f;
#pragma unroll
                for (int i = 0; i < TP; ++i) gs = fmaf(a[i], g[m + i], gs);
                dst[(size_t)(u0 + r0 + m) * W + (v0 + c)] = fmaf(-bs, ikk, gs);
            }
        }
    } else {
        for (int q = threadIdx.x; q < TR_TH * TR_TW; q += TR_NT) {
            const int r = q / TR_TW, c = q % TR_TW;
            const int qu = u0 + r, qv = v0 + c;
            if (qu >= H || qv >= W) continue;
            float g = 0.f, bx = 0.f;
            for (int i = -kr; i <= kr; ++i) {
                const int rr = (r + kr + i) * RS + c;
                g = fmaf(p.a[i + kr], RG[rr], g);
                const int pu = qu + i;
                if (pu >= 0 && pu < H) bx = fmaf((float)box_count(pu, qu, H, kr), RB[rr], bx);
            }
            dst[(size_t)qu * W + qv] = fmaf(-bx, ikk, g);
        }
    }
}

size_t adjoint_particle_smem(int K) { return sizeof(float) * (size_t)(2 * K + (ADJ_NT / 32) * 6 * K); }

size_t adjoint_transpose_smem(int kr) {
    const int SH = TR_TH + 2 * kr, SW = TR_TW + 2 * kr;
    return sizeof(float) * (size_t)(SH * SW + 2 * SH * (TR_TW + 1));
}

// Upper bound of the particle kernel's grid (partial sums of the backward
// pass: two doubles per block).
int adjoint_particle_blocks_max(int num_sms) { return num_sms * 16; }

cudaError_t launch_adjoint_particles(int mode, const AdjParams& p, const float* frames, const int* walk, long long n,
                                     const int* circ, const float* grad, float* yxm, float* gR, double* gpar,
                                     double* gpart, int* err, int num_sms, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const size_t smem = adjoint_particle_smem(p.K);
    const int grid = (int)std::min<long long>((n + ADJ_NT / 32 - 1) / (ADJ_NT / 32), (long long)num_sms * 16);
    cudaError_t e = cudaSuccess;
    switch (mode) {
        case ADJ_FORWARD:
            e = cudaFuncSetAttribute(adjoint_particle_kernel<ADJ_FORWARD>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e) return e;
            adjoint_particle_kernel<ADJ_FORWARD><<<grid, ADJ_NT, smem, st>>>(p, frames, walk, n, circ, grad, yxm,
                                                                             gR, gpar, err);
            break;
        case ADJ_BACKWARD:
            e = cudaFuncSetAttribute(adjoint_particle_kernel<ADJ_BACKWARD>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e) return e;
            adjoint_particle_kernel<ADJ_BACKWARD><<<grid, ADJ_NT, smem, st>>>(p, frames, walk, n, circ, grad, yxm,
                                                                              gR, gpart, err);
            e = cudaGetLastError();
            if (e) return e;
            adjoint_param_reduce_kernel<<<1, 256, 0, st>>>(gpart, grid, gpar);
            break;
        default:
            e = cudaFuncSetAttribute(adjoint_particle_kernel<ADJ_UNCERTAINTY>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e) return e;
            adjoint_particle_kernel<ADJ_UNCERTAINTY><<<grid, ADJ_NT, smem, st>>>(p, frames, walk, n, circ, grad,
                                                                                 yxm, gR, gpar, err);
            break;
    }
    return cudaGetLastError();
}

template <int KRT>
cudaError_t transpose_launch(const AdjParams& p, const float* gR, float* gI, size_t smem, cudaStream_t st) {
    cudaError_t e = cudaFuncSetAttribute(adjoint_transpose_kernel<KRT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e) return e;
    const int ntx = (p.W + TR_TW - 1) / TR_TW, nty = (p.H + TR_TH - 1) / TR_TH;
    for (int f0 = 0; f0 < p.T; f0 += 65535) {
        const int nf = std::min(65535, p.T - f0);
        dim3 grid(ntx * nty, nf);
        adjoint_transpose_kernel<KRT><<<grid, TR_NT, smem, st>>>(p, gR + (size_t)f0 * p.H * p.W,
                                                                 gI + (size_t)f0 * p.H * p.W);
    }
    return cudaGetLastError();
}

cudaError_t launch_adjoint_transpose(const AdjParams& p, const float* gR, float* gI, cudaStream_t st) {
    const size_t smem = adjoint_transpose_smem(p.krad);
    switch (p.krad) {
        case 1: return transpose_launch<1>(p, gR, gI, smem, st);
        case 2: return transpose_launch<2>(p, gR, gI, smem, st);
        case 3: return transpose_launch<3>(p, gR, gI, smem, st);
        case 4: return transpose_launch<4>(p, gR, gI, smem, st);
        case 5: return transpose_launch<5>(p, gR, gI, smem, st);
        case 6: return transpose_launch<6>(p, gR, gI, smem, st);
        case 7: return transpose_launch<7>(p, gR, gI, smem, st);
        default: return transpose_launch<0>(p, gR, gI, smem, st);
    }
}

}  // namespace gt
