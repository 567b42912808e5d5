// gt_device.cuh -- device helpers shared by the locate kernels: exact
// restatements of the per-pixel arithmetic of the WGSL shaders
// (gpu-tracking/src/shaders/*.wgsl) in the same operation order, so that
// every kernel variant produces identical bits.
//
// Compiled with --fmad=false: the only fused multiply-adds are the explicit
// fmaf() calls, which stand for the shaders' `acc += a * b` statements and
// for `a - b / c`, which the reference's GPU contracts into fma(-b, 1/c, a).
//
// Division convention of the reference's GPU: a WGSL `a / b` is evaluated as
// a multiplication by the reciprocal of b.  Both conventions are pinned by
// the reference's own dump of its mass plane (gpu-tracking/masses.bin),
// which the oracle reproduces bit for bit; the reciprocal is taken
// correctly rounded.
#pragma once
#include <cuda_runtime.h>
#include <math_constants.h>
#include "gt_internal.cuh"

namespace gt {

__device__ __forceinline__ int reflect_once(int x, int n) {
    // preprocess_rows.wgsl:34-41 / preprocess_cols.wgsl:36-43
    if (x < 0) return -x - 1;
    if (x >= n) return 2 * n - x - 1;
    return x;
}

__device__ __forceinline__ int clampi(int x, int lo, int hi) { return x < lo ? lo : (x > hi ? hi : x); }

// A shader division a / b: a times the correctly rounded reciprocal of b.
__device__ __forceinline__ float gpu_div(float a, float b) { return __fmul_rn(a, __frcp_rn(b)); }

__device__ __forceinline__ float load_px(const void* frames, int dtype, size_t idx) {
    if (dtype == 0) return (float)__ldg((const unsigned short*)frames + idx);
    return __ldg((const float*)frames + idx);
}

// Centroid at pixel (u, v) of the processed plane (centers.wgsl:23-109),
// read through an accessor `P(u, v)` in frame coordinates.  Returns false
// when the accessor cannot serve the whole circle (the caller falls back).
// Border-band pixels yield (0, 0) and mass 0 without reading anything.
template <class Acc>
__device__ __forceinline__ bool centroid_at(const LocParams& p, const Acc& P, int u, int v,
                                            float& c0, float& c1, float& m) {
    const int b = p.border;
    if (u - b < 0 || u + b >= p.H || v - b < 0 || v + b >= p.W) {
        c0 = 0.f; c1 = 0.f; m = 0.f;
        return true;
    }
    const int rint = p.rint_c;
    if (!P.covers(u - rint, v - rint) || !P.covers(u + rint, v + rint)) return false;
    const float r = (float)rint;
    const float r2 = r * r;
    float a0 = 0.f, a1 = 0.f, mm = 0.f;
    for (int i = -rint; i <= rint; ++i) {
        const float x = (float)i;
        const float x2 = x * x;
        for (int j = -rint; j <= rint; ++j) {
            const float y = (float)j;
            const float y2 = y * y;
            const float mask = x2 + y2;
            if (mask > r2) continue;
            const float data = P(u + i, v + j);
            a0 = fmaf(data, x, a0);
            a1 = fmaf(data, y, a1);
            mm = mm + data;
        }
    }
    c0 = gpu_div(a0, mm);  // centers.wgsl:82-83
    c1 = gpu_div(a1, mm);
    m = mm;
    return true;
}

struct WalkOut {
    float y, x, mass;
    int ok;      // 0 when the accessor could not serve a step
    int ul, vl;  // pixel of the last centroid read
    int up, vp;  // final position
};

// walk_cols.wgsl:38-74.  WGSL zero-initialises `center` and `idx`; with
// max_iterations == 0 the mass is read at pixel 0 (handled by the caller).
template <class Acc>
__device__ __forceinline__ WalkOut walk_from(const LocParams& p, const Acc& P, int u, int v) {
    WalkOut o;
    float c0 = 0.f, c1 = 0.f, m = 0.f;
    const float thr = p.thr;
    o.ul = 0; o.vl = 0;  // WGSL zero-initialised idx
    for (int it = 0; it < p.max_iter; ++it) {
        if (!centroid_at(p, P, u, v, c0, c1, m)) { o.ok = 0; o.y = o.x = o.mass = 0.f; return o; }
        o.ul = u; o.vl = v;
        bool changed = false;
        if (c0 > thr && u < p.H - 1) { u += 1; changed = true; }
        else if (c0 < -thr && u > 0) { u -= 1; changed = true; }
        if (c1 > thr && v < p.W - 1) { v += 1; changed = true; }
        else if (c1 < -thr && v > 0) { v -= 1; changed = true; }
        if (!changed) break;
    }
    o.y = (float)u + c0;
    o.x = (float)v + c1;
    o.mass = m;
    o.ok = 1;
    o.up = u; o.vp = v;
    return o;
}

// ndarray 0.15.6 unrolled_fold over K products computed by `prod(q)`
// (execute_gpu.rs:289-291 sum_axis on a contiguous lane).
template <class Prod>
__device__ __forceinline__ float unrolled_sum(int K, const Prod& prod) {
    float p0 = 0.f, p1 = 0.f, p2 = 0.f, p3 = 0.f, p4 = 0.f, p5 = 0.f, p6 = 0.f, p7 = 0.f;
    int i = 0;
    for (; K - i >= 8; i += 8) {
        p0 = p0 + prod(i + 0); p1 = p1 + prod(i + 1); p2 = p2 + prod(i + 2); p3 = p3 + prod(i + 3);
        p4 = p4 + prod(i + 4); p5 = p5 + prod(i + 5); p6 = p6 + prod(i + 6); p7 = p7 + prod(i + 7);
    }
    float acc = 0.f;
    acc = acc + (p0 + p4);
    acc = acc + (p1 + p5);
    acc = acc + (p2 + p6);
    acc = acc + (p3 + p7);
    for (; i < K; ++i) acc = acc + prod(i);
    return acc;
}

// cpu_processed features at the originating pixel (execute_gpu.rs:165-172,
// 286-299): sums of processed * {r2, sin2, cos2} over circle_inds(d/2).
template <class Acc>
__device__ __forceinline__ void cpu_features(const LocParams& p, const MovieBufs& b, const Acc& P,
                                             int u0, int v0, Cand& c) {
    const int K = p.n_char;
    const float* tab = b.char_tab;
    const int* off = b.char_off;
    auto nb = [&](int q) { return P(u0 + __ldg(off + 2 * q), v0 + __ldg(off + 2 * q + 1)); };
    const float rg = unrolled_sum(K, [&](int q) { return nb(q) * __ldg(tab + 3 * q); });
    const float s = unrolled_sum(K, [&](int q) { return nb(q) * __ldg(tab + 3 * q + 1); });
    const float co = unrolled_sum(K, [&](int q) { return nb(q) * __ldg(tab + 3 * q + 2); });
    float sig = nb(0);
    for (int q = 1; q < K; ++q) sig = fmaxf(sig, nb(q));
    c.rg_sum = rg;
    c.eccn = sqrtf(s * s + co * co);
    c.mid = P(u0, v0);
    c.signal = sig;
}

// characterize=True columns at the originating pixel (centers.wgsl:64-80).
template <class Acc, class RawAcc>
__device__ __forceinline__ void gpu_features(const LocParams& p, const MovieBufs& b, const Acc& P,
                                             const RawAcc& Rw, int u, int v, Cand& c) {
    const int rint = p.rint_c;
    const float r = (float)rint;
    const float r2 = r * r;
    float Rg = 0.f, rm = 0.f, s = 0.f, es = 0.f, ec = 0.f, m = 0.f;
    int t = 0;
    for (int i = -rint; i <= rint; ++i) {
        const float x = (float)i;
        const float x2 = x * x;
        for (int j = -rint; j <= rint; ++j) {
            const float y = (float)j;
            const float y2 = y * y;
            const float mask = x2 + y2;
            if (mask > r2) continue;
            const float data = P(u + i, v + j);
            m = m + data;
            Rg = fmaf(data, mask, Rg);
            rm = rm + Rw(u + i, v + j);
            s = fmaxf(s, data);
            es = fmaf(data, __ldg(b.gchar_tab + 2 * t), es);
            ec = fmaf(data, __ldg(b.gchar_tab + 2 * t + 1), ec);
            ++t;
        }
    }
    es = es * es;
    ec = ec * ec;
    c.g_ecc = gpu_div(sqrtf(es + ec), m - P(u, v));
    c.g_rg = sqrtf(gpu_div(Rg, m));
    c.g_raw = rm;
    c.g_sig = s;
}

// Block-wide exclusive scan of one int per thread (NT threads).
template <int NT>
__device__ __forceinline__ int block_excl_scan(int v, int* warp_tot, int* total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += y;
    }
    if (lane == 31) warp_tot[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int t = lane < NT / 32 ? warp_tot[lane] : 0;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, t, d);
            if (lane >= d) t += y;
        }
        if (lane < NT / 32) warp_tot[lane] = t;
        if (lane == NT / 32 - 1) *total = t;
    }
    __syncthreads();
    int base = wid > 0 ? warp_tot[wid - 1] : 0;
    int r = base + x - v;
    __syncthreads();
    return r;
}

}  // namespace gt
