// gt_oracle.cpp -- CPU restatement of gpu_tracking's locate-and-link path.
//
// TEST INFRASTRUCTURE ONLY (see gt_oracle.h).  Parity against the reference
// binary is UNPINNED: the reference cannot be built or run here (Rust host
// code, WGSL through wgpu), and it ships no golden vectors.  Every function
// cites the reference file:line it restates; paths are relative to the
// reference repository root.
//
// Built with -ffp-contract=off: every fused multiply-add below is explicit.

#include "gt_oracle.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <functional>
#include <type_traits>
#include <limits>
#include <string>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

namespace {

// ---------------------------------------------------------------------------
// Parameter derivation: gpu-tracking/src/gpu_setup.rs:45-60 and the WGSL
// window arithmetic in shaders/max_rows.wgsl:17, walk_cols.wgsl:21.
// ---------------------------------------------------------------------------
void derive_dilation(int separation, int* size, int* offset) {
    // gpu_setup.rs:48: (2. * sep as f32 / (2 as f32).sqrt()) as u32
    float v = (2.0f * (float)separation) / std::sqrt(2.0f);
    unsigned d = v <= 0.0f ? 0u : (unsigned)v;
    // max_rows.wgsl:17: i32(f32(kernel_cols) / 2. - 0.5), truncation toward 0
    float half = (float)(int)d / 2.0f - 0.5f;
    *size = (int)d;
    *offset = (int)half;
}

template <typename F>
struct Weights {
    std::vector<F> w;  // taps i = -rint..rint
    F norm = 0;
    F rn = 1;          // reciprocal of norm, by which the passes multiply
    int rint = 0;
};

// The reference's GPU evaluates a WGSL division `a / b` as a multiplication
// by the reciprocal of b, and contracts `a - b * c` into one fused
// multiply-add.  Both are pinned by the reference's own dump of the mass
// plane (gpu-tracking/masses.bin over gpu-tracking/inp, d = 9,
// smoothing_size = 9, noise_size = 1), which this restatement reproduces on
// all 419,200 pixels (tests/test_reference_dump.py): the boxcar term
// `constant_sum / f32(k*k)` of preprocess_cols.wgsl:54 is
// fma(-constant_sum, RN(1/k^2), gauss).  The reciprocal is taken as the
// correctly rounded one (the dump pins it for k^2 = 81).  The FP64 twin
// divides exactly: it is the accuracy reference.
template <typename F>
inline F gpu_div(F a, F b) {
    if constexpr (std::is_same<F, float>::value) return a * (1.0f / b);
    else return a / b;
}

// preprocess_rows.wgsl:30-45: gauss = exp(-x*x / (2*sigma2)), sigma2 is the
// `noise_size` parameter itself (gpu_setup.rs:52), gauss_norm accumulates
// every tap in order -rint..rint.  With `normalized` the taps are instead
// divided by their sum on the host and the passes do not divide
// (kernels.rs:86-97 `gauss_1d`, the form of the shaders' commented-out
// `gauss1d` binding, preprocess_rows.wgsl:7-8, preprocess_cols.wgsl:4-5,49):
// the form in which the reference produced its dump of the mass plane.
template <typename F>
Weights<F> gauss_weights(int smoothing_size, float noise_size, int normalized) {
    Weights<F> W;
    W.rint = smoothing_size / 2;
    F sigma2 = (F)noise_size;
    for (int i = -W.rint; i <= W.rint; ++i) {
        F x = (F)i;
        F g = std::exp(-x * x / ((F)2 * sigma2));
        W.w.push_back(g);
        W.norm = W.norm + g;
    }
    if (normalized) {
        for (auto& g : W.w) g = g / W.norm;  // kernels.rs:19-22 normalize
        W.rn = 1;
    } else {
        W.rn = std::is_same<F, float>::value ? (F)1 / W.norm : (F)1;
    }
    return W;
}

// preprocess_rows.wgsl:14-53 then preprocess_cols.wgsl:14-61.
// Gaussian taps are zero-padded (skipped) but normalised by the full window
// sum; the boxcar is reflect-padded and divided by f32(k*k).
template <typename F>
void bandpass(const float* pic, int H, int W, int k, float noise_size, int normalized, F* out) {
    Weights<F> G = gauss_weights<F>(k, noise_size, normalized);
    const bool f32 = std::is_same<F, float>::value;
    const int rint = G.rint;
    std::vector<F> tg((size_t)H * W), tb((size_t)H * W);
    for (int u = 0; u < H; ++u) {
        for (int v = 0; v < W; ++v) {
            F gs = 0, cs = 0;
            for (int i = -rint; i <= rint; ++i) {
                int pv = v + i;
                bool dg = true;
                if (pv < 0) { pv = -pv - 1; dg = false; }
                else if (pv >= W) { pv = 2 * W - pv - 1; dg = false; }
                F val = (F)pic[(size_t)u * W + pv];
                if (dg) gs = std::fma(G.w[i + rint], val, gs);
                cs = cs + val;
            }
            // preprocess_rows.wgsl:52 gauss_sum / gauss_norm
            tg[(size_t)u * W + v] = f32 ? gs * G.rn : (normalized ? gs : gs / G.norm);
            tb[(size_t)u * W + v] = cs;
        }
    }
    const F kk = (F)(k * k);
    const F rkk = (F)1 / kk;
    for (int u = 0; u < H; ++u) {
        for (int v = 0; v < W; ++v) {
            F gs = 0, cs = 0;
            for (int i = -rint; i <= rint; ++i) {
                int pu = u + i;
                bool dg = true;
                if (pu < 0) { pu = -pu - 1; dg = false; }
                else if (pu >= H) { pu = 2 * H - pu - 1; dg = false; }
                size_t idx = (size_t)pu * W + v;
                if (dg) gs = std::fma(G.w[i + rint], tg[idx], gs);
                cs = cs + tb[idx];
            }
            // preprocess_cols.wgsl:54 gauss_sum/gauss_norm - constant_sum/f32(k*k)
            F res = f32 ? std::fma(-cs, rkk, gs * G.rn) : (normalized ? gs : gs / G.norm) - cs / kk;
            out[(size_t)u * W + v] = res < (F)0 ? (F)0 : res;
        }
    }
}

// Per-pixel centroid (centers.wgsl:23-109), evaluated lazily: the value at a
// pixel is a pure function of the processed plane, so computing it on demand
// gives the same bits as the full-plane shader.
template <typename F>
struct Centers {
    const F* P;
    const float* raw;
    int H, W, d;
    std::vector<unsigned char> done;
    std::vector<F> c0, c1, mass;
    // characterize=True extras (centers.wgsl:64-80), at the same pixel
    bool want_char;
    std::vector<F> rg, rawm, sig, ecc;
    const std::vector<float>* sin2;
    const std::vector<float>* cos2;

    void init(const F* P_, const float* raw_, int H_, int W_, int d_, bool ch,
              const std::vector<float>* s2, const std::vector<float>* c2) {
        P = P_; raw = raw_; H = H_; W = W_; d = d_; want_char = ch; sin2 = s2; cos2 = c2;
        size_t n = (size_t)H * W;
        done.assign(n, 0); c0.assign(n, 0); c1.assign(n, 0); mass.assign(n, 0);
        if (ch) { rg.assign(n, 0); rawm.assign(n, 0); sig.assign(n, 0); ecc.assign(n, 0); }
    }

    void eval(int u, int v) {
        size_t idx = (size_t)u * W + v;
        if (done[idx]) return;
        done[idx] = 1;
        // centers.wgsl:99-103: border band of width d/2 gets zeros
        int kr = d, kc = d;
        if (u - kr / 2 < 0 || u + kr / 2 >= H || v - kc / 2 < 0 || v + kc / 2 >= W) {
            c0[idx] = 0; c1[idx] = 0; mass[idx] = 0;
            return;
        }
        const int rint = (kr - 1) / 2;
        const F r = (F)rint;
        const F r2 = r * r;
        F a0 = 0, a1 = 0, m = 0;
        F Rg = 0, rm = 0, s = 0, es = 0, ec = 0;
        int t = 0;  // index into the circle tables (same i-outer/j-inner order)
        for (int i = -rint; i <= rint; ++i) {
            F x = (F)i;
            F x2 = x * x;
            for (int j = -rint; j <= rint; ++j) {
                F y = (F)j;
                F y2 = y * y;
                F mask = x2 + y2;
                if (mask > r2) continue;
                int pu = u + i, pv = v + j;
                if (pu < 0 || pu >= H || pv < 0 || pv >= W) { ++t; continue; }
                size_t pidx = (size_t)pu * W + pv;
                F data = P[pidx];
                a0 = std::fma(data, x, a0);
                a1 = std::fma(data, y, a1);
                m = m + data;
                if (want_char) {
                    Rg = std::fma(data, mask, Rg);
                    rm = rm + (F)raw[pidx];
                    s = std::max(s, data);
                    es = std::fma(data, (F)(*sin2)[t], es);
                    ec = std::fma(data, (F)(*cos2)[t], ec);
                }
                ++t;
            }
        }
        if (want_char) {
            es = es * es;
            ec = ec * ec;
            ecc[idx] = gpu_div<F>(std::sqrt(es + ec), m - P[idx]);
            rg[idx] = std::sqrt(gpu_div<F>(Rg, m));
            rawm[idx] = rm;
            sig[idx] = s;
        }
        // centers.wgsl:82-83 centers /= mass
        c0[idx] = gpu_div<F>(a0, m);
        c1[idx] = gpu_div<F>(a1, m);
        mass[idx] = m;
    }
};

// Circle stencil tables: kernels.rs:134-150 (circle_inds), 169-206
// (r2_in_circle, sin_in_circle, cos_in_circle).  Integer radius R: i outer
// (row offset), j inner (column offset), i^2 + j^2 <= R^2.
struct Circle {
    std::vector<int> di, dj;
    std::vector<float> r2, sin2, cos2;
    int middle = -1;
};

Circle circle_table(int R) {
    Circle c;
    for (int i = -R; i <= R; ++i)
        for (int j = -R; j <= R; ++j)
            if (i * i + j * j <= R * R) {
                if (i == 0 && j == 0) c.middle = (int)c.di.size();
                c.di.push_back(i);
                c.dj.push_back(j);
                c.r2.push_back((float)(i * i + j * j));
                float th = std::atan2((float)j, (float)i);
                c.sin2.push_back(std::sin(2.0f * th));
                c.cos2.push_back(std::cos(2.0f * th));
            }
    return c;
}

// circle_inds with a float radius (kernels.rs:134-150) and annulus_inds
// (kernels.rs:152-167), for the raw sig/bg columns.
void circle_inds_f(float radius, std::vector<int>& di, std::vector<int>& dj) {
    int rb = (int)std::ceil(radius);
    float r2 = radius * radius;
    for (int i = -rb; i <= rb; ++i)
        for (int j = -rb; j <= rb; ++j)
            if ((float)(i * i + j * j) <= r2) { di.push_back(i); dj.push_back(j); }
}

void annulus_inds_f(float outer, float inner, std::vector<int>& di, std::vector<int>& dj) {
    int b = (int)std::ceil(outer);
    float or2 = outer * outer, ir2 = inner * inner;
    for (int i = -b; i <= b; ++i)
        for (int j = -b; j <= b; ++j) {
            float r2 = (float)(i * i + j * j);
            if (r2 <= or2 && r2 >= ir2) { di.push_back(i); dj.push_back(j); }
        }
}

// ndarray 0.15.6 `sum()` on a contiguous lane (numeric_util::unrolled_fold):
// eight interleaved accumulators, combined (p0+p4),(p1+p5),(p2+p6),(p3+p7),
// then the < 8 leftover elements in order.  Used by sum_axis in
// execute_gpu.rs:289-291.
float unrolled_sum(const float* xs, int n) {
    float acc = 0.0f;
    float p[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int i = 0;
    while (n - i >= 8) {
        for (int l = 0; l < 8; ++l) p[l] = p[l] + xs[i + l];
        i += 8;
    }
    acc = acc + (p[0] + p[4]);
    acc = acc + (p[1] + p[5]);
    acc = acc + (p[2] + p[6]);
    acc = acc + (p[3] + p[7]);
    for (; i < n; ++i) acc = acc + xs[i];
    return acc;
}

struct Feature {
    int origin;        // raster index of the originating pixel
    float y, x, mass;  // walk result (walk_cols.wgsl:69-73)
    int ul, vl;        // pixel of the last centroid read (`idx`)
    int up, vp;        // final position of the walk
    // cpu_processed (execute_gpu.rs:286-299, 346-352)
    float Rg, ecc, signal;
    // characterize=True (centers.wgsl:64-80 read at the originating pixel)
    float g_rg, g_raw, g_sig, g_ecc;
    // raw sig/bg (execute_gpu.rs:301-333)
    float raw_mass, bg_median, corrected;
};

// kd-tree 0.4.2 `within_radius`, restated from its call-site twin
// linking.rs:73-105: box pre-filter per axis, then squared distance
// (item - query), accumulated from zero, strictly below radius^2.
inline bool within(float qy, float qx, float iy, float ix, float radius, float* dist) {
    if (iy < qy - radius || iy > qy + radius) return false;
    if (ix < qx - radius || ix > qx + radius) return false;
    float dy = iy - qy, dx = ix - qx;
    float dd = 0.0f;
    dd = dd + dy * dy;
    dd = dd + dx * dx;
    if (dist) *dist = dd;
    return dd < radius * radius;
}

template <typename F>
std::vector<Feature> locate_frame(const float* pic, int H, int W, const or_params& p,
                                  const Circle& cc, const Circle& gc, bool filter = true) {
    const size_t n = (size_t)H * W;
    std::vector<F> P(n);
    bandpass<F>(pic, H, W, p.smoothing_size, p.noise_size, p.normalized_taps, P.data());

    int D, o;
    derive_dilation(p.separation, &D, &o);
    // max_rows.wgsl:10-28
    std::vector<F> rowmax(n);
    for (int u = 0; u < H; ++u)
        for (int v = 0; v < W; ++v) {
            F m = P[(size_t)u * W + v];
            int pv = v - o;
            for (int j = 0; j < D; ++j, ++pv)
                if (pv >= 0 && pv < W) m = std::max(m, P[(size_t)u * W + pv]);
            rowmax[(size_t)u * W + v] = m;
        }

    Centers<F> C;
    C.init(P.data(), pic, H, W, p.diameter, p.characterize != 0, &gc.sin2, &gc.cos2);
    const F thr = (F)0.6f;  // gpu_setup.rs:57 shift_threshold
    const F minmass = (F)p.minmass;

    std::vector<Feature> feats;
    for (int u0 = 0; u0 < H; ++u0) {
        for (int v0 = 0; v0 < W; ++v0) {
            // walk_cols.wgsl:19-36 is_max (non-strict)
            F center = P[(size_t)u0 * W + v0];
            bool ismax = true;
            int pu = u0 - o;
            for (int i = 0; i < D; ++i, ++pu)
                if (pu >= 0 && pu < H && rowmax[(size_t)pu * W + v0] > center) { ismax = false; break; }
            if (!ismax) continue;
            // walk_cols.wgsl:38-74 walk; WGSL zero-initialises `center`/`idx`
            int u = u0, v = v0;
            F cy = 0, cx = 0;
            size_t idx = 0;
            for (int it = 0; it < p.max_iterations; ++it) {
                idx = (size_t)u * W + v;
                C.eval(u, v);
                cy = C.c0[idx];
                cx = C.c1[idx];
                bool changed = false;
                if (cy > thr && u < H - 1) { u += 1; changed = true; }
                else if (cy < -thr && u > 0) { u -= 1; changed = true; }
                if (cx > thr && v < W - 1) { v += 1; changed = true; }
                else if (cx < -thr && v > 0) { v -= 1; changed = true; }
                if (!changed) break;
            }
            C.eval((int)(idx / W), (int)(idx % W));
            F fy = (F)u + cy;
            F fx = (F)v + cx;
            F fm = C.mass[idx];
            // walk_cols.wgsl:86 `mass > minmass`, then the raster scan keeps
            // mass != 0 (execute_gpu.rs:159-160)
            if (!(fm > minmass) || fm == (F)0) continue;
            Feature f{};
            f.origin = u0 * W + v0;
            f.y = (float)fy; f.x = (float)fx; f.mass = (float)fm;
            f.ul = (int)(idx / W); f.vl = (int)(idx % W);
            f.up = u; f.vp = v;
            if (p.cpu_processed) {
                // execute_gpu.rs:165-172 gather at the originating pixel, then
                // 286-299 and 346-352.  Emitted origins are interior, so the
                // radius-d/2 circle is always inside the frame (no NaN).
                const int K = (int)cc.di.size();
                std::vector<float> nb(K), t(K);
                for (int q = 0; q < K; ++q)
                    nb[q] = (float)P[(size_t)(u0 + cc.di[q]) * W + (v0 + cc.dj[q])];
                for (int q = 0; q < K; ++q) t[q] = nb[q] * cc.r2[q];
                float rg = unrolled_sum(t.data(), K);
                for (int q = 0; q < K; ++q) t[q] = nb[q] * cc.sin2[q];
                float s = unrolled_sum(t.data(), K);
                for (int q = 0; q < K; ++q) t[q] = nb[q] * cc.cos2[q];
                float c = unrolled_sum(t.data(), K);
                float eccn = std::sqrt(s * s + c * c);
                float mid = nb[cc.middle];
                float sig = nb[0];
                for (int q = 1; q < K; ++q) sig = std::max(sig, nb[q]);
                f.Rg = std::sqrt(rg / f.mass);
                f.ecc = eccn / (f.mass - mid);
                f.signal = sig;
            }
            if (p.characterize) {
                size_t oidx = (size_t)u0 * W + v0;
                C.eval(u0, v0);
                f.g_rg = (float)C.rg[oidx];
                f.g_raw = (float)C.rawm[oidx];
                f.g_sig = (float)C.sig[oidx];
                f.g_ecc = (float)C.ecc[oidx];
            }
            feats.push_back(f);
        }
    }

    if (!filter) return feats;
    // execute_gpu.rs:258-284: single-pass separation filter.  `idx` is the
    // position in the raster scan; canonical (raster) order is kept.
    const float sep = (float)p.separation;
    std::vector<Feature> kept;
    const int N = (int)feats.size();
    for (int a = 0; a < N; ++a) {
        bool keep = true;
        for (int b = 0; b < N && keep; ++b) {
            if (b == a) continue;
            if (!within(feats[a].y, feats[a].x, feats[b].y, feats[b].x, sep, nullptr)) continue;
            if (feats[a].mass < feats[b].mass) keep = false;
            else if (feats[a].mass == feats[b].mass && a > b) keep = false;
        }
        if (keep) kept.push_back(feats[a]);
    }

    // execute_gpu.rs:301-333: raw signal and annulus median around the
    // rounded refined position; out-of-frame pixels are NaN and skipped.
    if (p.has_sig_radius) {
        std::vector<int> si, sj, bi, bj;
        circle_inds_f(p.sig_radius, si, sj);
        if (p.has_bg_radius) annulus_inds_f(p.bg_radius, p.sig_radius + p.gap_radius, bi, bj);
        auto get = [&](int r, int c) -> float {
            if (r < 0 || r >= H || c < 0 || c >= W) return std::numeric_limits<float>::quiet_NaN();
            return pic[(size_t)r * W + c];
        };
        for (auto& f : kept) {
            int mr = (int)std::round(f.y), mc = (int)std::round(f.x);
            float acc = 0.0f;
            for (size_t q = 0; q < si.size(); ++q) {
                float val = get(mr + si[q], mc + sj[q]);
                if (!std::isnan(val)) acc = acc + val;
            }
            f.raw_mass = acc;
            if (p.has_bg_radius) {
                std::vector<float> vals;
                for (size_t q = 0; q < bi.size(); ++q) {
                    float val = get(mr + bi[q], mc + bj[q]);
                    if (!std::isnan(val)) vals.push_back(val);
                }
                float med;
                if (vals.empty()) {
                    med = std::numeric_limits<float>::quiet_NaN();
                } else {
                    // ndarray-stats 0.5.1 quantile_axis_skipnan_mut, q = 0.5,
                    // Linear interpolation between floor/ceil order statistics
                    std::sort(vals.begin(), vals.end());
                    double fi = 0.5 * (double)(vals.size() - 1);
                    size_t lo = (size_t)std::floor(fi), hi = (size_t)std::ceil(fi);
                    double frac = fi - std::floor(fi);
                    float a = vals[lo], b = vals[hi];
                    med = a + (float)(frac * ((double)b - (double)a));
                }
                f.bg_median = med;
                f.corrected = f.raw_mass - med * (float)si.size();
            }
        }
    }
    return kept;
}

// ---------------------------------------------------------------------------
// Linker: linking.rs:197-492 (Linker::new/advance, link, recurse, recurse2).
// ---------------------------------------------------------------------------
struct Src {
    float y, x;
    uint64_t id;
};

struct Linker {
    float radius;
    int memory;
    std::vector<Src> prev;
    size_t prev_N = 0;
    std::deque<std::vector<Src>> memvec;
    uint64_t part_idx = 0;
    int status = 0;
    uint64_t budget = (uint64_t)1 << 40;  // effectively uncapped, as the reference

    Linker(float r, int mem) : radius(r), memory(mem) {
        for (int i = 0; i < mem; ++i) memvec.emplace_back();
    }

    // linking.rs:234-281
    std::vector<uint64_t> advance(const std::vector<std::array<float, 2>>& frame) {
        const size_t N = frame.size();
        bool has_mem = memory > 0;
        if (has_mem) {
            std::unordered_set<uint64_t> seen;
            for (auto& s : prev) seen.insert(s.id);
            for (auto& lst : memvec)
                for (auto& e : lst)
                    if (!seen.count(e.id)) { prev.push_back(e); seen.insert(e.id); }
        }
        std::vector<Src> unused;
        std::vector<uint64_t> result = link(frame, has_mem, unused);
        std::vector<Src> np;
        np.reserve(N);
        for (size_t i = 0; i < N; ++i) np.push_back({frame[i][0], frame[i][1], result[i]});
        prev.swap(np);
        if (has_mem) { memvec.push_back(unused); memvec.pop_front(); }
        prev_N = N;
        return result;
    }

    // recurse2, linking.rs:390-452
    void recurse2(size_t progress, const std::vector<size_t>& dests, float& score, float& best,
                  std::unordered_map<uint64_t, size_t>& used, std::unordered_set<size_t>& nulls,
                  std::vector<int64_t>& output,
                  const std::vector<std::vector<std::pair<size_t, float>>>& d2s, float null_cost,
                  uint64_t& nodes) {
        size_t cur = dests[progress];
        const auto& opts = d2s[cur];
        for (size_t oi = 0; oi <= opts.size(); ++oi) {
            if (++nodes > budget) { status = 4; return; }
            bool is_null = oi == opts.size();
            float cost = is_null ? null_cost : opts[oi].second;
            uint64_t sid = is_null ? 0 : prev[opts[oi].first].id;
            if (score > best) return;
            score += cost;
            if (!is_null) {
                if (used.count(sid)) { score -= cost; continue; }
                used[sid] = cur;
            } else {
                nulls.insert(cur);
            }
            if (progress == dests.size() - 1) {
                if (score < best) {
                    best = score;
                    for (auto& kv : used) output[kv.second] = (int64_t)kv.first;
                    for (auto v : nulls) output[v] = -1;
                }
            } else {
                recurse2(progress + 1, dests, score, best, used, nulls, output, d2s, null_cost, nodes);
            }
            if (!is_null) used.erase(sid);
            else nulls.erase(cur);
            score -= cost;
        }
    }

    // link, linking.rs:286-492.  Neighbour order of src_to_dest is ascending
    // destination index (kd-tree order is unpinned); dest_to_src is ascending
    // source index, as the reference builds it.
    std::vector<uint64_t> link(const std::vector<std::array<float, 2>>& dest, bool has_mem,
                               std::vector<Src>& unused) {
        const size_t NS = prev.size(), ND = dest.size();
        std::vector<std::vector<size_t>> s2d(NS);
        std::vector<std::vector<std::pair<size_t, float>>> d2s(ND);
        // candidate pairs through a uniform grid of cell size `radius` over
        // the destinations (+-2 cells, so that no pair passing `within` is
        // missed to rounding); each source's list is then put in ascending
        // destination order, exactly the order of an all-pairs scan
        std::unordered_map<long long, std::vector<size_t>> grid;
        auto cell = [&](float v) { return (long long)std::floor(v / radius); };
        auto key = [](long long a, long long b) { return a * 1000003LL + b; };
        for (size_t d = 0; d < ND; ++d) grid[key(cell(dest[d][0]), cell(dest[d][1]))].push_back(d);
        for (size_t s = 0; s < NS; ++s) {
            const long long cy = cell(prev[s].y), cx = cell(prev[s].x);
            for (long long a = cy - 2; a <= cy + 2; ++a)
                for (long long b = cx - 2; b <= cx + 2; ++b) {
                    auto it = grid.find(key(a, b));
                    if (it == grid.end()) continue;
                    for (size_t d : it->second) {
                        float dd;
                        if (within(prev[s].y, prev[s].x, dest[d][0], dest[d][1], radius, &dd)) s2d[s].push_back(d);
                    }
                }
            std::sort(s2d[s].begin(), s2d[s].end());
            for (size_t d : s2d[s]) {
                float dd = 0.0f;
                within(prev[s].y, prev[s].x, dest[d][0], dest[d][1], radius, &dd);
                d2s[d].push_back({s, dd});
            }
        }
        std::vector<char> vis_s(NS, 0), vis_d(ND, 0);
        std::vector<int64_t> output(ND, -2);  // -2 = None (unassigned)
        std::vector<std::pair<std::vector<size_t>, std::vector<size_t>>> paths;
        // recurse, linking.rs:316-342 (recursive preorder DFS)
        std::vector<size_t> ps, pd;
        std::function<void(size_t, int)> dfs = [&](size_t node, int side) {
            if (side == 0) {
                if (vis_s[node]) return;
                vis_s[node] = 1;
                ps.push_back(node);
                for (size_t d : s2d[node]) dfs(d, 1);
            } else {
                if (vis_d[node]) return;
                vis_d[node] = 1;
                pd.push_back(node);
                for (auto& e : d2s[node]) dfs(e.first, 0);
            }
        };
        for (size_t i = 0; i < ND; ++i) {
            ps.clear(); pd.clear();
            dfs(i, 1);
            if (pd.size() == 1) {
                if (ps.size() == 0) {
                } else if (ps.size() == 1) {
                    output[i] = (int64_t)prev[ps[0]].id;
                } else {
                    paths.push_back({ps, pd});
                }
            } else if (pd.size() > 0) {
                paths.push_back({ps, pd});
            }
        }
        const float null_cost = radius * radius;
        for (auto& path : paths) {
            std::unordered_map<uint64_t, size_t> used;
            std::unordered_set<size_t> nulls;
            float score = 0.0f, best = std::numeric_limits<float>::infinity();
            uint64_t nodes = 0;
            recurse2(0, path.second, score, best, used, nulls, output, d2s, null_cost, nodes);
        }
        std::vector<uint64_t> res(ND);
        for (size_t i = 0; i < ND; ++i) {
            if (output[i] >= 0) res[i] = (uint64_t)output[i];
            else res[i] = part_idx++;
        }
        if (has_mem) {
            std::unordered_set<uint64_t> usedids(res.begin(), res.end());
            for (size_t s = 0; s < prev_N && s < NS; ++s)
                if (!usedids.count(prev[s].id)) unused.push_back(prev[s]);
        }
        return res;
    }
};

// execute_gpu.rs:197-226 column_names
std::vector<std::string> column_names(const or_params& p) {
    std::vector<std::string> c = {"frame", "mass", "y", "x"};
    if (p.has_search_range) c.push_back("particle");
    if (p.cpu_processed) { c.push_back("Rg"); c.push_back("ecc"); c.push_back("signal"); }
    if (p.has_sig_radius) c.push_back("raw_mass");
    if (p.has_bg_radius) { c.push_back("raw_bg_median"); c.push_back("raw_mass_corrected"); }
    if (p.characterize) {
        c.push_back("Rg_gpu"); c.push_back("raw_mass_gpu"); c.push_back("signal_gpu"); c.push_back("ecc_gpu");
    }
    return c;
}

int run_batch(const float* frames, int T, int H, int W, const or_params* pp, int nthreads,
              int fp64, float** out, int64_t* nrows, int* ncols, int32_t** walk = nullptr) {
    const or_params p = *pp;
    if (p.has_bg_radius && !p.has_sig_radius) return 1;
    Circle cc = circle_table(p.diameter / 2);
    Circle gc = circle_table((p.diameter - 1) / 2);
    std::vector<std::vector<Feature>> per(T);
    if (nthreads < 1) nthreads = 1;
    std::vector<std::thread> th;
    for (int w = 0; w < nthreads; ++w)
        th.emplace_back([&, w]() {
            for (int t = w; t < T; t += nthreads) {
                const float* pic = frames + (size_t)t * H * W;
                per[t] = fp64 ? locate_frame<double>(pic, H, W, p, cc, gc)
                              : locate_frame<float>(pic, H, W, p, cc, gc);
            }
        });
    for (auto& x : th) x.join();

    int status = 0;
    std::vector<std::vector<uint64_t>> ids(T);
    if (p.has_search_range) {
        Linker L(p.search_range, p.memory);
        for (int t = 0; t < T; ++t) {
            std::vector<std::array<float, 2>> fr;
            for (auto& f : per[t]) fr.push_back({f.y, f.x});
            ids[t] = L.advance(fr);
            if (L.status) status = L.status;
        }
    }
    std::vector<std::string> names = column_names(p);
    const int nc = (int)names.size();
    int64_t nr = 0;
    for (int t = 0; t < T; ++t) nr += (int64_t)per[t].size();
    float* o = (float*)std::malloc(sizeof(float) * (size_t)std::max<int64_t>(nr, 1) * nc);
    int64_t r = 0;
    for (int t = 0; t < T; ++t)
        for (size_t i = 0; i < per[t].size(); ++i, ++r) {
            const Feature& f = per[t][i];
            float* row = o + (size_t)r * nc;
            int c = 0;
            row[c++] = (float)t;
            row[c++] = f.mass;
            row[c++] = f.y;
            row[c++] = f.x;
            if (p.has_search_range) row[c++] = (float)ids[t][i];
            if (p.cpu_processed) { row[c++] = f.Rg; row[c++] = f.ecc; row[c++] = f.signal; }
            if (p.has_sig_radius) row[c++] = f.raw_mass;
            if (p.has_bg_radius) { row[c++] = f.bg_median; row[c++] = f.corrected; }
            if (p.characterize) { row[c++] = f.g_rg; row[c++] = f.g_raw; row[c++] = f.g_sig; row[c++] = f.g_ecc; }
        }
    if (walk) {
        int32_t* wk = (int32_t*)std::malloc(sizeof(int32_t) * 5 * (size_t)std::max<int64_t>(nr, 1));
        int64_t q = 0;
        for (int t = 0; t < T; ++t)
            for (const Feature& f : per[t]) {
                int32_t* w5 = wk + 5 * q++;
                w5[0] = t; w5[1] = f.ul; w5[2] = f.vl; w5[3] = f.up; w5[4] = f.vp;
            }
        *walk = wk;
    }
    *out = o;
    *nrows = nr;
    *ncols = nc;
    return status;
}

}  // namespace

extern "C" {

int or_batch(const float* frames, int T, int H, int W, const or_params* p, int nthreads,
             int fp64, float** out, int64_t* nrows, int* ncols) {
    return run_batch(frames, T, H, W, p, nthreads, fp64, out, nrows, ncols);
}

int or_batch_walk(const float* frames, int T, int H, int W, const or_params* p, int nthreads,
                  float** out, int64_t* nrows, int* ncols, int32_t** walk) {
    return run_batch(frames, T, H, W, p, nthreads, 0, out, nrows, ncols, walk);
}

int or_batch_u16(const uint16_t* frames, int T, int H, int W, const or_params* p, int nthreads,
                 int fp64, float** out, int64_t* nrows, int* ncols) {
    std::vector<float> f((size_t)T * H * W);
    for (size_t i = 0; i < f.size(); ++i) f[i] = (float)frames[i];
    return run_batch(f.data(), T, H, W, p, nthreads, fp64, out, nrows, ncols);
}

// lib.rs:202-212 link_rust -> FrameSubsetter (linking.rs:12-61) -> linker_all
// (linking.rs:570-580).  Positions are columns 2 and 3; a group is a run of
// consecutive rows with equal column 0, and the iterator's first group is
// empty when the first frame value is not 0.
int or_link(const float* rows, int64_t n, int ncols, float search_range, int memory,
            uint64_t* ids) {
    Linker L(search_range, memory);
    int64_t idx = 0;
    float cur = 0.0f;
    int64_t w = 0;
    while (true) {
        std::vector<std::array<float, 2>> grp;
        bool end = false;
        while (true) {
            if (idx >= n) { end = true; break; }
            float fr = rows[idx * ncols + 0];
            if (fr != cur) { cur = fr; break; }
            grp.push_back({rows[idx * ncols + 2], rows[idx * ncols + 3]});
            ++idx;
        }
        if (end && grp.empty()) break;
        std::vector<uint64_t> r = L.advance(grp);
        for (auto v : r) ids[w++] = v;
        if (end) break;
    }
    return L.status;
}

void or_bandpass(const float* frame, int H, int W, int smoothing_size, float noise_size,
                 int normalized_taps, float* processed) {
    bandpass<float>(frame, H, W, smoothing_size, noise_size, normalized_taps, processed);
}

void or_centers(const float* frame, int H, int W, const or_params* p, float* c0, float* c1, float* mass) {
    // The centers/masses planes of centers.wgsl:88-109 at every pixel.
    std::vector<float> P((size_t)H * W);
    bandpass<float>(frame, H, W, p->smoothing_size, p->noise_size, p->normalized_taps, P.data());
    Centers<float> C;
    C.init(P.data(), frame, H, W, p->diameter, false, nullptr, nullptr);
    for (int u = 0; u < H; ++u)
        for (int v = 0; v < W; ++v) {
            C.eval(u, v);
            const size_t i = (size_t)u * W + v;
            c0[i] = C.c0[i];
            c1[i] = C.c1[i];
            mass[i] = C.mass[i];
        }
}

void or_locate_planes(const float* frame, int H, int W, const or_params* pp, float* planes) {
    // Results planes as walk_cols.wgsl:86-91 writes them: before the
    // separation filter, keyed by the originating pixel.
    or_params p = *pp;
    p.cpu_processed = 0;
    p.characterize = 0;
    p.has_sig_radius = 0;
    p.has_bg_radius = 0;
    Circle cc = circle_table(p.diameter / 2);
    Circle gc = circle_table((p.diameter - 1) / 2);
    std::memset(planes, 0, sizeof(float) * 3 * (size_t)H * W);
    std::vector<Feature> all = locate_frame<float>(frame, H, W, p, cc, gc, false);
    for (auto& f : all) {
        size_t o2 = (size_t)f.origin;
        planes[o2] = f.mass;
        planes[(size_t)H * W + o2] = f.y;
        planes[2 * (size_t)H * W + o2] = f.x;
    }
}

void or_dilation(int separation, int* size, int* offset) { derive_dilation(separation, size, offset); }

void or_free(void* ptr) { std::free(ptr); }

}  // extern "C"
