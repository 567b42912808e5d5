// locate_fast.cu -- specialised locate kernel for sm_100a.
//
// Same results, bit for bit, as locate_tiles_kernel (and the oracle): the
// per-pixel arithmetic chains are unchanged, only packed two per FP32x2
// instruction, and the boxcar of uint16 frames uses running sums, which are
// exact because every partial sum is an integer below 2^24.
//
// Specialised on (smoothing radius KR, dilation size DD, tile height TH0,
// centroid radius RC with diameter 2*RC + 1), so the whole tile geometry is
// known at compile time: every shared-memory offset is an immediate and
// every loop has a constant trip count.  A CTA (256 or 512 threads) takes a
// run of consecutive TH0 x 64 output tiles; per tile:
//   0. the uint16 tile plus halo is staged by one TMA load (zero fill
//      outside the frame) into U[RH][US] (US >= RW: rows padded so that
//      16-byte loads of consecutive row pairs spread over the banks); the
//      next tile's load is issued once the row pass is done with U;
//   1. (no separate conversion) the row pass reads row pairs of U with
//      16-byte loads, turns each u16 into an exact float (2^23 + u, minus
//      2^23) and filters 8 columns per thread (FFMA2 chains in tap order),
//      Gaussian and boxcar -> Gp, Bp (row pairs); tiles at a frame edge
//      then repair the boxcar's reflect padding (the Gaussian pads with 0);
//   2. column pass: a thread filters one column over 8 rows (4 row pairs),
//      scales by the reciprocal of the Gaussian norm, subtracts the boxcar
//      as fma(-box, 1/k^2, gauss) and clips at 0 -> P2 (row pairs); tiles at
//      a frame edge then write -inf outside the frame;
//   3. row max over the dilation window (register sliding max) -> RM2;
//   4. column max of RM2 compared with the centre: the local maxima of a
//      warp's rows are listed at once by per-row ballots into the CTA list;
//   5. the list is walked one candidate per lane by the walker warps, which
//      compute the features and emit the records (ranks from per-row bit
//      masks, one slot atomic per warp) while the other warps run the next
//      tile's phases 0-3.
// Row strides of the pair arrays are odd (in 8-byte units), so every
// lane-per-row access is bank-conflict free.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstring>

#include "gt_device.cuh"
#include "gt_simd.cuh"

namespace gt {

namespace {
constexpr int FT = 64;    // output tile width
constexpr int FNT = 256;  // threads of a 32-row tile

// 8 warps per 32 output rows: 64-row tiles (less halo recomputed per
// output row) keep 16 warps per SM slot at 2 CTAs per SM
__host__ __device__ constexpr int fast_threads(int th) { return th == 32 ? FNT : 2 * FNT; }
constexpr int FM = 8;     // outputs per thread item
// Walker warps of a run of tiles (64-row tiles: 2 of 16 warps, 32-row
// tiles: 2 of 8): they walk a tile of at most 32 NWO candidates while the
// other warps start the next one.
#ifndef GT_WALKERS64
#define GT_WALKERS64 2
#endif
__host__ __device__ constexpr int walker_warps(int th) { return th == 32 ? 2 : GT_WALKERS64; }

__host__ __device__ constexpr int cmax(int a, int b) { return a > b ? a : b; }
__host__ __device__ constexpr int round8(int x) { return (x + 7) / 8 * 8; }
__host__ __device__ constexpr int align128(int x) { return (x + 127) / 128 * 128; }
__host__ __device__ constexpr int fast_offset(int DD) { return (int)((float)DD / 2.0f - 0.5f); }
__host__ __device__ constexpr int circle_size(int RC) {
    int k = 0;
    for (int i = -RC; i <= RC; ++i)
        for (int j = -RC; j <= RC; ++j) k += (i * i + j * j <= RC * RC);
    return k;
}

// CTAs of the specialised kernel per SM with `smem` bytes of dynamic shared
// memory: 228 KB per SM, 1 KB reserved per CTA and about 1 KB of static
// arrays; the registers allow 2 CTAs of 512 threads or 4 of 256.
__host__ __device__ constexpr int fast_ctas(int th, int smem) {
    return cmax(0, (th == 32 ? 4 : 2) < 233472 / (smem + 2048) ? (th == 32 ? 4 : 2) : 233472 / (smem + 2048));
}

// Compile-time tile geometry.
template <int KR, int DD, int TH0, int RC>
struct Geo {
    static constexpr int O = fast_offset(DD);
    static constexpr int HP0 = cmax(cmax(O, DD - 1 - O), cmax(RC + 2, 1));  // d/2 == RC for odd d
    static constexpr int HP = HP0 + ((HP0 - O) & 1);  // hp - O even: row pairs align
    static constexpr int L = round8(HP + KR);        // raw columns left of the tile
    static constexpr int HX = L - KR;                // processed columns left of the tile
    static constexpr int RW = round8(L + FT + HP + KR);
    static constexpr int RH = TH0 + 2 * HP + 2 * KR;
    static constexpr int RP = RH / 2;
    static constexpr int PH = TH0 + 2 * HP;
    static constexpr int PP = PH / 2;
    static constexpr int PW = RW - 2 * KR;
    static constexpr int NPW = (PW + FM - 1) / FM;
    static constexpr int PWC = FM * NPW;
    static constexpr int NRQ = (PH + FM - 1) / FM;  // column-pass items per column
    static constexpr int GPS = PWC | 1;
    static constexpr int P2S = PW | 1;
    static constexpr int RMS = FT | 1;
    static constexpr int NV = (FM + 2 * KR + 7) / 8;  // 16-byte loads per raw row of a row-pass item
    // raw tile row stride: a row pair spans an odd number of 16-byte units
    // (quarter-warp 16-byte loads of consecutive row pairs hit 2 banks at most)
    static constexpr int US = ((RW / 8) % 2 == 0) ? RW + 8 : RW;
    static constexpr int NTK = fast_threads(TH0);
    static constexpr int SZ_P2 = align128(PP * P2S * 8);
    static constexpr int SZ_U = align128(RH * US * 2 + 16 * NV);  // + the last item's overrun
    static constexpr int SZ_GP = align128(cmax(RP * GPS * 8, (PP + 1) * RMS * 8));
    // boxcar rows, then the candidate list (u16) and the walkers' emission staging
    static constexpr int SZ_BP = align128(cmax(RP * GPS * 8, TH0 * FT * 2 + (NTK / 32) * 32 * 20));
    static constexpr int K = circle_size(RC);
    static constexpr int SZ_TAB = align128(K * 20);  // (sin2, cos2), P2 offsets by parity, r2
    static constexpr int NWO = walker_warps(TH0);
    static constexpr int SZ_STG = align128(NWO * 32 * 20);  // emission staging of the overlapping walkers
    static constexpr int SMEM1 = SZ_P2 + SZ_GP + SZ_BP + SZ_U + SZ_TAB + SZ_STG;
    // Two processed planes (the walkers read the previous tile's while the
    // stencil warps write the next one) where that keeps the CTAs per SM.
    static constexpr bool WS =
        fast_ctas(TH0, SMEM1 + SZ_P2) >= fast_ctas(TH0, SMEM1) && SMEM1 + SZ_P2 <= 227 * 1024;
    static constexpr int NP2 = WS ? 2 : 1;
    static constexpr int OFF_GP = NP2 * SZ_P2;
    static constexpr int OFF_BP = OFF_GP + SZ_GP;
    static constexpr int OFF_U = OFF_BP + SZ_BP;
    static constexpr int OFF_TAB = OFF_U + SZ_U;
    static constexpr int OFF_STG = OFF_TAB + SZ_TAB;
    static constexpr int SMEM = OFF_STG + SZ_STG;
    // index invariants of the phases below
    static_assert(((HP - O) & 1) == 0, "row pairs of the local-max pass must align");
    static_assert(HX >= HP && HX - O >= 0, "row max window starts inside the processed region");
    static_assert(FT - 1 + HX + (DD - 1 - O) <= PW - 1, "row max window ends inside the computed columns");
    static_assert(((TH0 - FM + HP - O) >> 1) + (FM + DD) / 2 - 1 <= PP, "column max rows allocated");
    static_assert(TH0 - 1 + HP + (DD - 1 - O) <= PH - 1, "column max window inside the processed rows");
    static_assert(FT + HX <= PW, "centre columns computed");
    // a column-pass item covers row pairs p0 .. p0 + FM/2 - 1, p0 <= PP - FM/2,
    // and reads row pairs up to p0 + FM/2 + KR - 1
    static_assert(PP >= FM / 2 && PP + KR <= RP, "column pass reads computed row pairs");
    static_assert(PWC <= GPS && PW <= P2S && FT <= RMS, "row strides");
    static_assert(US <= 256 && RH <= 256 && (US * 2) % 16 == 0, "TMA box");
    static_assert((NPW - 1) * FM < US && (FM * 2) % 16 == 0, "16-byte raw loads start inside a U row");
    static_assert(SMEM <= 227 * 1024, "shared memory");
    static_assert(RC + 2 <= HP && RC <= HX, "walk and feature circles inside the processed region");
    static_assert(NTK / 32 > 2 * NWO, "stencil warps besides the walkers");
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y,
                                            int z) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
        "l"(map), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// max(a, b, c) in one instruction (sm_100 three-input max.f32)
__device__ __forceinline__ float fmax3(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// max over v[m .. m+DD-1] for m = 0..M-1, sharing the common core
template <int DD, int M>
__device__ __forceinline__ void slide_max(const float (&v)[M + DD - 1], float (&out)[M]) {
    if constexpr (DD < M) {
#pragma unroll
        for (int m = 0; m < M; ++m) {
            float x = v[m];
            int j = 1;
#pragma unroll
            for (; j + 1 < DD; j += 2) x = fmax3(x, v[m + j], v[m + j + 1]);
            if (j < DD) x = fmaxf(x, v[m + j]);
            out[m] = x;
        }
    } else {
        // core = max(v[M-1 .. DD-1])
        float core = v[M - 1];
        int j = M;
#pragma unroll
        for (; j + 1 < DD; j += 2) core = fmax3(core, v[j], v[j + 1]);
        if (j < DD) core = fmaxf(core, v[j]);
        float suf[M];  // suf[m] = max(v[m .. M-2]), m <= M-2
        suf[M - 1] = -CUDART_INF_F;
#pragma unroll
        for (int m = M - 2; m >= 0; --m) suf[m] = fmaxf(v[m], suf[m + 1]);
        float pre = -CUDART_INF_F;  // max(v[DD .. DD+m-1])
#pragma unroll
        for (int m = 0; m < M; ++m) {
            if (m > 0) pre = fmaxf(pre, v[DD + m - 1]);
            out[m] = fmax3(suf[m], core, pre);
        }
    }
}

// processed plane as row pairs, frame coordinates, compile-time geometry
template <class G>
struct P2Acc {
    const float* P;
    int py0, px0;
    __device__ bool covers(int u, int v) const {
        const int r = u - py0, c = v - px0;
        return r >= 0 && r < G::PH && c >= 0 && c < G::PW;
    }
    __device__ float operator()(int u, int v) const {
        const int r = u - py0, c = v - px0;
        return P[(((r >> 1) * G::P2S + c) << 1) + (r & 1)];
    }
};

struct GRawAcc {  // raw pixels straight from the frame (characterize only)
    const unsigned short* F;
    int W;
    __device__ float operator()(int u, int v) const { return (float)__ldg(F + (size_t)u * W + v); }
};

// Centroid sums at a centre whose processed row has parity E, fully unrolled
// (centers.wgsl:39-85 order: i outer, j inner, mask x^2 + y^2 <= r^2).
template <int RC, int E, int S>
__device__ __forceinline__ void circle_centroid(const float* P, int base, float& a0, float& a1, float& mm) {
#pragma unroll
    for (int i = -RC; i <= RC; ++i) {
#pragma unroll
        for (int j = -RC; j <= RC; ++j) {
            if (i * i + j * j > RC * RC) continue;
            const float data = P[base + ((((E + i) >> 1) * S + j) << 1) + ((E + i) & 1)];
            a0 = fmaf(data, (float)i, a0);
            a1 = fmaf(data, (float)j, a1);
            mm = mm + data;
        }
    }
}

// cpu_processed sums of processed * {r2, sin2, cos2} over the d/2 circle
// (equal to the centroid circle for odd d), folded as ndarray's sum_axis
// does (execute_gpu.rs:289-291: eight interleaved accumulators, combined
// (p0+p4), (p1+p5), (p2+p6), (p3+p7) into 0 in that order, then the
// leftover elements in order), and the maximum (signal), computed by the 8
// lanes of a lane group (l = lane & 7,
// groups of 8 consecutive lanes share one record): lane l accumulates the
// products of circle elements l, l + 8, l + 16, ... (accumulator l), the
// group folds them, and group lane 0 adds the leftover elements.  offs
// holds each element's P2 offset for a centre row of parity 0 (.x) and 1
// (.y).  Every lane of the warp must call it; results on group lane 0.
template <int RC>
__device__ __forceinline__ void circle_features_group(const float* P, int base, int E, const int2* offs,
                                                      const float* r2, const float2* sc, int l, float& rg,
                                                      float& sn, float& cs, float& sig) {
    constexpr int K = circle_size(RC);
    constexpr int K8 = K & ~7;
    const unsigned full = 0xffffffffu;
    float pr = 0.f, ps = 0.f, pc = 0.f, mx = -CUDART_INF_F;
#pragma unroll
    for (int q0 = 0; q0 < K8; q0 += 8) {
        const int q = q0 + l;
        const int2 o = offs[q];
        const float nb = P[base + (E ? o.y : o.x)];
        const float2 t = sc[q];
        pr = pr + nb * r2[q];
        ps = ps + nb * t.x;
        pc = pc + nb * t.y;
        mx = fmaxf(mx, nb);
    }
    // (p_l + p_{l+4}) on lanes l < 4 of the group
    const float qr = pr + __shfl_down_sync(full, pr, 4);
    const float qs = ps + __shfl_down_sync(full, ps, 4);
    const float qc = pc + __shfl_down_sync(full, pc, 4);
    float ar = 0.f, as = 0.f, ac = 0.f;
    ar = ar + qr; as = as + qs; ac = ac + qc;
#pragma unroll
    for (int k = 1; k < 4; ++k) {
        ar = ar + __shfl_down_sync(full, qr, k);
        as = as + __shfl_down_sync(full, qs, k);
        ac = ac + __shfl_down_sync(full, qc, k);
    }
    mx = fmaxf(mx, __shfl_xor_sync(full, mx, 1));
    mx = fmaxf(mx, __shfl_xor_sync(full, mx, 2));
    mx = fmaxf(mx, __shfl_xor_sync(full, mx, 4));
#pragma unroll
    for (int q = K8; q < K; ++q) {  // leftover elements, in order
        const int2 o = offs[q];
        const float nb = P[base + (E ? o.y : o.x)];
        const float2 t = sc[q];
        ar = ar + nb * r2[q];
        as = as + nb * t.x;
        ac = ac + nb * t.y;
        mx = fmaxf(mx, nb);
    }
    rg = ar;
    sn = as;
    cs = ac;
    sig = mx;
}

template <class G, int RC>
__device__ __forceinline__ bool centroid_fixed(const LocParams& p, const P2Acc<G>& P, int u, int v, float& c0,
                                               float& c1, float& m) {
    const int bd = p.border;
    if (u - bd < 0 || u + bd >= p.H || v - bd < 0 || v + bd >= p.W) {
        c0 = 0.f; c1 = 0.f; m = 0.f;
        return true;
    }
    if (!P.covers(u - RC, v - RC) || !P.covers(u + RC, v + RC)) return false;
    const int r0 = u - P.py0, cc = v - P.px0;
    const int base = (((r0 >> 1) * G::P2S + cc) << 1);
    float a0 = 0.f, a1 = 0.f, mm = 0.f;
    if (r0 & 1) circle_centroid<RC, 1, G::P2S>(P.P, base, a0, a1, mm);
    else circle_centroid<RC, 0, G::P2S>(P.P, base, a0, a1, mm);
    c0 = gpu_div(a0, mm);  // centers.wgsl:82-83
    c1 = gpu_div(a1, mm);
    m = mm;
    return true;
}

}  // namespace

namespace {
// Output tile g of a launch: tiles are numbered frame by frame, frame0 first.
struct FTile {
    int t, tj, ty0, tx0, TH;
};

template <int TH0>
__device__ __forceinline__ FTile tile_of(const LocParams& p, int frame0, int ntiles, int g) {
    FTile f;
    const int fr = g / ntiles, tile = g - fr * ntiles;
    const int ti = tile / p.ntx;
    f.t = frame0 + fr;
    f.tj = tile - ti * p.ntx;
    f.ty0 = ti * TH0;
    f.tx0 = f.tj * FT;
    f.TH = min(TH0, p.H - f.ty0);
    return f;
}

// The tile after f in launch order, without divisions.
template <int TH0>
__device__ __forceinline__ FTile next_tile(const LocParams& p, FTile f) {
    f.tj += 1;
    f.tx0 += FT;
    if (f.tj == p.ntx) {
        f.tj = 0;
        f.tx0 = 0;
        f.ty0 += TH0;
        if (f.ty0 >= p.H) {
            f.ty0 = 0;
            f.t += 1;
        }
    }
    f.TH = min(TH0, p.H - f.ty0);
    return f;
}

__device__ __forceinline__ void bar_sync(int id, int n) { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory"); }
__device__ __forceinline__ void bar_arrive(int id, int n) {
    asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(n) : "memory");
}

// ---- 5. walks and emission of tile f, by the walker warps ----
// The list is walked one candidate per lane, so the walks, the costliest
// code per candidate, run with full warps.  Lane index c holds list entry q
// when `have` (read by the caller); list entries c + wstride, c + 2 wstride,
// ... (candidates beyond one per walker thread) are read from the list here
// and emitted as pending without a walk (fallback_walk_kernel walks them).
// Records are ranked within their (row, tile) segment from a per-row bit
// mask of the columns that emit, which is what finalize_kernel needs; slots
// come from one atomic per warp.  Named barrier 1 syncs the nwt walker
// threads.
template <class G, int RC>
__device__ __forceinline__ void walk_emit(const LocParams& p, const MovieBufs& b, const FTile& f, const float* P2f,
                                          const unsigned short* clist, unsigned long long* rowmask, int* stage,
                                          float4* sfeat, const int2* offs, const float* r2s, const float2* sc,
                                          int ncand, int c, bool have, int q, int wstride, int nwt) {
    const int H = p.H, W = p.W;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const int t = f.t, ty0 = f.ty0, tx0 = f.tx0;
    const int py0 = ty0 - G::HP, px0 = tx0 - G::HX;
    P2Acc<G> acc{P2f, py0, px0};
    const int tr = q / FT, tc = q - tr * FT;
    const int u0 = ty0 + tr, v0 = tx0 + tc;
    int st = CAND_REJECT;
    float y = 0.f, x = 0.f, m = 0.f;
    unsigned int lp = 0, fp = 0;
    if (have) {
        if (p.max_iter <= 0) {
            st = CAND_PENDING;
        } else {
            // walk_cols.wgsl:38-74
            int u = u0, v = v0;
            float w0 = 0.f, w1 = 0.f;
            bool ok = true;
            for (int iter = 0; iter < p.max_iter; ++iter) {
                if (!centroid_fixed<G, RC>(p, acc, u, v, w0, w1, m)) { ok = false; break; }
                lp = ((unsigned)u << 16) | (unsigned)v;
                bool changed = false;
                if (w0 > p.thr && u < H - 1) { u += 1; changed = true; }
                else if (w0 < -p.thr && u > 0) { u -= 1; changed = true; }
                if (w1 > p.thr && v < W - 1) { v += 1; changed = true; }
                else if (w1 < -p.thr && v > 0) { v -= 1; changed = true; }
                if (!changed) break;
            }
            if (!ok) {
                st = CAND_PENDING;
                m = 0.f;
            } else {
                y = (float)u + w0;
                x = (float)v + w1;
                st = (m > p.minmass && m != 0.f) ? CAND_EMIT : CAND_REJECT;
                fp = ((unsigned)u << 16) | (unsigned)v;
            }
        }
    }
    if (st != CAND_REJECT) atomicOr(&rowmask[tr], 1ull << tc);
    int nrec = __popc(__ballot_sync(0xffffffffu, st != CAND_REJECT));
    for (int c0 = wstride; c0 < ncand; c0 += wstride) {
        const bool more = c0 + c < ncand;
        if (more) {
            const int q2 = clist[c0 + c];
            atomicOr(&rowmask[q2 / FT], 1ull << (q2 % FT));
        }
        nrec += __popc(__ballot_sync(0xffffffffu, more));
    }
    // this warp's slots; the result is first needed at the stores, so the
    // atomic's latency overlaps the barrier and the sums below
    int gbase = 0;
    if (lane == 0 && nrec) gbase = atomicAdd(b.fcount + t, nrec);
    if (nwt > 32) bar_sync(1, nwt);
    else __syncwarp();
    if (warp == 0)
        for (int r = lane; r < f.TH; r += 32)
            b.rowcnt[((size_t)t * H + ty0 + r) * p.ntx + f.tj] = __popcll(rowmask[r]);

    // emission: the first stride of the list from the walks above, later
    // strides as pending records.  The cpu_processed sums of a stride's
    // records are computed by lane groups of 8, four records at a time
    // (circle_features_group); the slot atomic issued above completes
    // meanwhile.
    const unsigned short* frame = (const unsigned short*)b.frames + (size_t)t * H * W;
    GRawAcc racc{frame, W};
    int roff = 0;
    for (int c0 = 0; c0 < ncand; c0 += wstride) {
        int rq = q, rtr = tr, rtc = tc, rst = st;
        float ry = y, rx = x, rm = m;
        unsigned int rlp = lp, rfp = fp;
        if (c0 > 0) {
            const bool more = c0 + c < ncand;
            rq = more ? clist[c0 + c] : 0;
            rtr = rq / FT;
            rtc = rq - rtr * FT;
            rst = more ? CAND_PENDING : CAND_REJECT;
            ry = rx = rm = 0.f;
            rlp = rfp = 0;
        }
        const bool em = rst != CAND_REJECT;
        const unsigned eb = __ballot_sync(0xffffffffu, em);
        const int ne = __popc(eb), e = __popc(eb & lt);
        const int ru = ty0 + rtr, rv = tx0 + rtc;
        float4 feat = make_float4(0.f, 0.f, 0.f, 0.f);
        if (p.cpu_processed && ne) {
            // execute_gpu.rs:165-172, 286-299 at the originating pixel
            if (em) stage[e] = ((ru - py0) << 16) | (rv - px0);
            __syncwarp();
            for (int g = 0; g < ne; g += 4) {
                const int er = min(g + (lane >> 3), ne - 1);
                const int code = stage[er];
                const int rr = code >> 16, cc = code & 0xffff;
                float a0, a1, a2, a3;
                circle_features_group<RC>(P2f, ((rr >> 1) * G::P2S + cc) * 2, rr & 1, offs, r2s, sc, lane & 7,
                                          a0, a1, a2, a3);
                if ((lane & 7) == 0 && g + (lane >> 3) < ne) sfeat[g + (lane >> 3)] = make_float4(a0, a1, a2, a3);
            }
            __syncwarp();
            if (em) feat = sfeat[e];
            __syncwarp();  // stage and sfeat are reused by the next stride
        }
        // the slot base of lane 0's atomic, read only now: its latency
        // overlapped the sums above
        int gb = __shfl_sync(0xffffffffu, gbase, 0);
        if (gb + nrec > b.cap_c) {
            if (lane == 0 && c0 == 0) atomicOr(b.err, ERR_CAND_OVERFLOW);
            gb = -1;
        }
        if (em) {
            Cand rec;
            rec.u = ru; rec.v = rv;
            rec.y = ry; rec.x = rx; rec.mass = rm;
            rec.rowrank = __popcll(rowmask[rtr] & ((1ull << rtc) - 1ull));
            rec.state = rst;
            rec.rg_sum = rec.eccn = rec.mid = rec.signal = 0.f;
            rec.g_rg = rec.g_raw = rec.g_sig = rec.g_ecc = 0.f;
            rec.ul = (int)(rlp >> 16); rec.vl = (int)(rlp & 0xffffu);
            rec.up = (int)(rfp >> 16); rec.vp = (int)(rfp & 0xffffu);
            rec.pad = 0;
            if (p.cpu_processed) {
                rec.rg_sum = feat.x;
                rec.eccn = sqrtf(feat.y * feat.y + feat.z * feat.z);
                rec.mid = acc(ru, rv);
                rec.signal = feat.w;
            }
            if (p.characterize) gpu_features(p, b, acc, racc, ru, rv, rec);
            if (gb >= 0) {
                const int slot = gb + roff + e;
                b.cand[(size_t)t * b.cap_c + slot] = rec;
                if (rec.state == CAND_PENDING) {
                    const int k = atomicAdd(b.npend, 1);
                    b.pend[k] = t * b.cap_c + slot;
                }
            }
        }
        roff += ne;
    }
}
}  // namespace

// A CTA locates a run of consecutive tiles [g0, g0 + ntl) of the launch.
// The walker warps [0, NWO) walk tile k - 1's candidates and emit its
// records (when it has at most 32 NWO) while the stencil warps run tile k's
// row pass, and, with two
// processed planes (G::WS), its column pass and row max too: the warps meet
// only for the column max and the list.  With one plane the walkers hold the
// plane until the column pass.  A tile with more candidates is walked by as
// many warps as it needs before the next tile starts.  The next raw tile is
// copied in as soon as a row pass is done with the current one.  Named
// barriers: 1 the walker warps, 2 "tile k - 1's list is read" (walkers
// arrive, the stencil warps wait), 3 all warps before the column max (two
// planes) or the column pass (one plane), 4 the stencil warps once the raw
// tile is in (one thread's wait for its copy, or their own staging without
// TMA), 5 the stencil warps between their phases.  A tile
// copy that does not land within the bounded wait sets ERR_DEVICE_TIMEOUT;
// the CTA then issues no further copies, lists no candidates and finishes its
// run (every barrier is still reached; the host discards the results).
template <int KR, int DD, int TH0, int RC>
__global__ void __launch_bounds__(fast_threads(TH0), (TH0 == 32 ? 4 : 2))
    locate_fast_kernel(const LocParams p, const MovieBufs b, const __grid_constant__ CUtensorMap tmap, int use_tma,
                       int frame0, int ntiles, int total, int per_cta) {
    using G = Geo<KR, DD, TH0, RC>;
    constexpr int NTK = fast_threads(TH0);
    constexpr int NW = NTK / 32;
    constexpr int TAPS = 2 * KR + 1;
    constexpr int O = G::O;
    constexpr int HP = G::HP, HX = G::HX;
    constexpr int NWO = G::NWO;
    constexpr int NWT = NWO * 32;       // walker threads while tiles overlap
    constexpr int NS = NTK - NWT;       // stencil threads
    constexpr int PROD = NTK - 32;      // issues the tile copies: a stencil thread
    // column pass and row max: the stencil warps (two planes) or all warps
    constexpr int CB = G::WS ? NWT : 0, CN = NTK - CB;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ int s_fail, s_nc;
    __shared__ unsigned long long rowmask[TH0];  // columns of the tile row that emit a record

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int g0 = blockIdx.x * per_cta;
    const int ntl = min(per_cta, total - g0);
    const int H = p.H, W = p.W;

    float2* Gp = (float2*)(smem + G::OFF_GP);
    float2* Bp = (float2*)(smem + G::OFF_BP);
    unsigned short* U = (unsigned short*)(smem + G::OFF_U);  // raw tile, row stride US
    float2* RM2 = Gp;                                         // after the column pass
    unsigned short* clist = (unsigned short*)Bp;  // candidate list: the boxcar is dead after the column pass
    float2* sc = (float2*)(smem + G::OFF_TAB);    // (sin2, cos2) of the d/2 circle
    int2* offs = (int2*)(smem + G::OFF_TAB + G::K * 8);  // P2 offsets of the d/2 circle by centre parity
    float* r2s = (float*)(smem + G::OFF_TAB + G::K * 16);
    // emission staging of the walker warps: their own region while the
    // next tile's row pass fills the boxcar rows, else after the list
    int* stage_ov = (int*)(smem + G::OFF_STG);
    float4* sfeat_ov = (float4*)(smem + G::OFF_STG + NWO * 32 * 4);
    int* stage_bp = (int*)((unsigned char*)Bp + TH0 * FT * 2);
    float4* sfeat_bp = (float4*)((unsigned char*)Bp + TH0 * FT * 2 + NW * 32 * 4);

    // ---- set-up: the first tile's copy, tables ----
    if (tid == 0) { s_fail = 0; s_nc = 0; }
    if (tid < TH0) rowmask[tid] = 0ull;
    if (use_tma && tid == PROD) {
        mbar_init(&bar, 1);
        const FTile f = tile_of<TH0>(p, frame0, ntiles, g0);
        mbar_expect_tx(&bar, (uint32_t)(G::RH * G::US * 2));
        // tma_withhold (a test of the timeout path) issues no copy: the
        // barrier then never completes and the bounded wait runs out
        if (!p.tma_withhold) tma_load_3d(U, &tmap, &bar, f.tx0 - G::L, f.ty0 - HP - KR, f.t);
    }
    if (p.cpu_processed)
        for (int k = tid; k < G::K; k += NTK) {
            sc[k] = make_float2(__ldg(b.char_tab + 3 * k + 1), __ldg(b.char_tab + 3 * k + 2));
            r2s[k] = __ldg(b.char_tab + 3 * k);
            const int di = __ldg(b.char_off + 2 * k), dj = __ldg(b.char_off + 2 * k + 1);
            offs[k] = make_int2(((di >> 1) * G::P2S + dj) * 2 + (di & 1),
                                (((1 + di) >> 1) * G::P2S + dj) * 2 + ((1 + di) & 1));
        }
    __syncthreads();

    float2 W2[TAPS];
#pragma unroll
    for (int j = 0; j < TAPS; ++j) W2[j] = make_float2(p.w[j], p.w[j]);
    const float2 RN2 = make_float2(p.rn, p.rn), NRKK2 = make_float2(-p.rkk, -p.rkk);
    const float NEG = -CUDART_INF_F;

    FTile prev{};  // tile k - 1, walked at the top of iteration k
    FTile f = tile_of<TH0>(p, frame0, ntiles, g0);  // tile k
    int last = 0;  // the last tile whose copy was issued (copy-issuing thread)
    for (int k = 0; k <= ntl; ++k) {
        if (k > 0) {
            const int ncand = s_nc;
            const bool more = k < ntl;
            const float* P2w = (const float*)(smem + (G::WS ? ((k - 1) & 1) * G::SZ_P2 : 0));
            // at most 32 NWO candidates: the walker warps take equal shares
            // of the list, and the stencil warps go on once every walker has
            // read its entry; a crowded tile is walked by warps [0, nwalk),
            // one candidate per thread, before the next tile starts
            const bool ov = ncand <= NWT;
            const int nwt = ov ? NWT : min(NW, (ncand + 31) >> 5) * 32;
            if (tid < nwt) {
                const int h = (ncand + NWO - 1) / NWO;
                const int c = ov ? warp * h + lane : tid;
                const bool have = ov ? lane < h && c < ncand : c < ncand;
                const int q = have ? clist[c] : 0;
                if (ov && more) bar_arrive(2, NTK);  // the list (and s_nc) may be overwritten
                walk_emit<G, RC>(p, b, prev, P2w, clist, rowmask, (ov ? stage_ov : stage_bp) + warp * 32,
                                 (ov ? sfeat_ov : sfeat_bp) + warp * 32, offs, r2s, sc, ncand, c, have, q, nwt, nwt);
                if (!more) break;
                if (nwt > 32) bar_sync(1, nwt);  // every walker reads rowmask until its last record
                else __syncwarp();
                for (int r = tid; r < TH0; r += nwt) rowmask[r] = 0ull;
                if (!ov) bar_sync(2, NTK);
            } else {
                if (!more) break;
                bar_sync(2, NTK);
            }
            if (tid == PROD) s_nc = 0;  // every thread has read it (barrier 2)
        }
        const int ry0 = f.ty0 - HP - KR, rx0 = f.tx0 - G::L;
        const int py0 = f.ty0 - HP, px0 = f.tx0 - HX;
        float2* P2 = (float2*)(smem + (G::WS ? (k & 1) * G::SZ_P2 : 0));
        if (warp >= NWO) {
            const int stid = tid - NWT;
            // ---- 0. the raw tile ----
            if (use_tma) {
                // one thread waits for the copy, the stencil warps meet it
                if (tid == PROD) {
                    bool done = false;
                    for (int it = 0; it < p.tma_spin && !done && !s_fail; ++it) done = mbar_try_wait(&bar, k & 1);
                    if (!done && !s_fail) {
                        atomicOr(b.err, ERR_DEVICE_TIMEOUT);
                        s_fail = 1;
                    }
                }
                bar_sync(4, NS);
            } else {
                const unsigned short* fr = (const unsigned short*)b.frames + (size_t)f.t * H * W;
                for (int i = stid; i < G::RH * G::US; i += NS) {
                    const int r = i / G::US, c = i - r * G::US;
                    const int gy = ry0 + r, gx = rx0 + c;
                    unsigned short v = 0;
                    if (gy >= 0 && gy < H && gx >= 0 && gx < W) v = __ldg(fr + (size_t)gy * W + gx);
                    U[i] = v;
                }
                bar_sync(4, NS);
            }

            // ---- 1. row pass (preprocess_rows.wgsl) on row pairs ----
            for (int it = stid; it < G::RP * G::NPW; it += NS) {
                const int q = it / G::RP, pr = it - q * G::RP;
                const int pc0 = q * FM;
                // raw rows 2 pr and 2 pr + 1 as exact floats: 0x4B000000 | u is 2^23 + u
                const uint4* r0 = (const uint4*)(U + (2 * pr) * G::US + pc0);
                const uint4* r1 = (const uint4*)(U + (2 * pr + 1) * G::US + pc0);
                float2 v[8 * G::NV];
#pragma unroll
                for (int l = 0; l < G::NV; ++l) {
                    const uint4 a4 = r0[l], c4 = r1[l];
                    const unsigned int wa[4] = {a4.x, a4.y, a4.z, a4.w}, wc[4] = {c4.x, c4.y, c4.z, c4.w};
#pragma unroll
                    for (int h = 0; h < 4; ++h) {
                        const float2 lo = make_float2(__uint_as_float(__byte_perm(wa[h], 0x4B00u, 0x5410)),
                                                      __uint_as_float(__byte_perm(wc[h], 0x4B00u, 0x5410)));
                        const float2 hi = make_float2(__uint_as_float(__byte_perm(wa[h], 0x4B00u, 0x5432)),
                                                      __uint_as_float(__byte_perm(wc[h], 0x4B00u, 0x5432)));
                        v[8 * l + 2 * h] = add2(lo, make_float2(-8388608.f, -8388608.f));
                        v[8 * l + 2 * h + 1] = add2(hi, make_float2(-8388608.f, -8388608.f));
                    }
                }
                float2* gd = Gp + pr * G::GPS + pc0;
                float2* bd = Bp + pr * G::GPS + pc0;
#pragma unroll
                for (int m = 0; m < FM; ++m) {
                    float2 acc = make_float2(0.f, 0.f);
#pragma unroll
                    for (int j = 0; j < TAPS; ++j) acc = fma2(W2[j], v[m + j], acc);
                    gd[m] = mul2(acc, RN2);  // preprocess_rows.wgsl:52
                }
                // boxcar over the zero-filled raw tile; the columns whose
                // reflect-padded window differs are redone below
                float2 s = v[0];
#pragma unroll
                for (int j = 1; j < TAPS; ++j) s = add2(s, v[j]);
                bd[0] = s;
#pragma unroll
                for (int m = 1; m < FM; ++m) {
                    s = sub2(add2(s, v[m + 2 * KR]), v[m - 1]);
                    bd[m] = s;
                }
            }
            // ---- 1b. reflect-padded boxcar at the frame edges (preprocess_rows.wgsl:34-41,
            //          preprocess_cols.wgsl:36-43), edge tiles only.  Boxcar column c is
            //          centred on frame column rx0 + KR + c and raw row r is frame row
            //          ry0 + r.  (h) the in-frame columns within KR of the left or right
            //          edge add their window's taps outside the frame, reflected into
            //          it, to the row pass's zero-padded sums; (v) then each raw row
            //          within KR outside the top or bottom edge takes the boxcar row of
            //          its reflected row, so that the column pass's running sums give the
            //          reflect-padded vertical sums.  All sums are integers below 2^24,
            //          exact in any order. ----
            // (only tiles whose raw rows or boxcar columns reach a frame edge)
            if (rx0 < 0 || rx0 + KR + G::PWC > W - KR || ry0 < 0 || ry0 + G::RH > H) {
                float* Bf = (float*)Bp;
                const int cl0 = max(0, rx0 + KR), cl1 = min(KR, rx0 + KR + G::PWC);
                const int cr0 = max(max(W - KR, cl1), rx0 + KR), cr1 = min(W, rx0 + KR + G::PWC);
                const int nl = max(0, cl1 - cl0), nh = nl + max(0, cr1 - cr0);
                const int rt0 = max(0, -KR - ry0), rt1 = max(rt0, min(G::RH, -ry0));
                const int rb0 = max(0, H - ry0), rb1 = max(rb0, min(G::RH, H + KR - ry0));
                const int nt = rt1 - rt0, nv = nt + (rb1 - rb0);
                if (nh + nv > 0) bar_sync(5, NS);  // the row pass is done
                if (nh > 0) {
                    for (int i = stid; i < nh * G::RH; i += NS) {
                        const int j = i / G::RH, r = i - j * G::RH;
                        const int fc = j < nl ? cl0 + j : cr0 + (j - nl);
                        // the row pass summed the window over zeros outside the
                        // frame; add the taps x < 0 and x >= W reflected to
                        // frame columns -x - 1 and 2W - x - 1
                        const unsigned short* Ur = U + r * G::US - rx0;  // frame column y at Ur[y]
                        float corr = 0.f;
#pragma unroll
                        for (int t = 0; t < KR; ++t) {
                            if (t < KR - fc) corr = corr + (float)Ur[t];
                            if (t < fc + KR - W + 1) corr = corr + (float)Ur[W - 1 - t];
                        }
                        float* d = Bf + ((((r >> 1) * G::GPS + (fc - rx0 - KR)) << 1) + (r & 1));
                        *d = *d + corr;
                    }
                    if (nv > 0) bar_sync(5, NS);
                }
                if (nv > 0) {
                    for (int i = stid; i < nv * G::PWC; i += NS) {
                        const int k2 = i / G::PWC, c = i - k2 * G::PWC;
                        const int r = k2 < nt ? rt0 + k2 : rb0 + (k2 - nt);
                        const int rs = clampi(reflect_once(ry0 + r, H) - ry0, 0, G::RH - 1);  // an in-frame row
                        Bf[(((r >> 1) * G::GPS + c) << 1) + (r & 1)] = Bf[(((rs >> 1) * G::GPS + c) << 1) + (rs & 1)];
                    }
                }
            }
        }
        if (G::WS) {
            if (warp >= NWO) bar_sync(5, NS);
        } else {
            bar_sync(3, NTK);  // the walkers of tile k - 1 arrive after their records
        }
        // the raw tile is read: the next tile's copy lands during this one
        if (use_tma && tid == PROD && k + 1 < ntl && !s_fail) {
            const FTile n = next_tile<TH0>(p, f);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_expect_tx(&bar, (uint32_t)(G::RH * G::US * 2));
            if (!p.tma_withhold) tma_load_3d(U, &tmap, &bar, n.tx0 - G::L, n.ty0 - HP - KR, n.t);
            last = k + 1;
        }

        if (tid >= CB) {
            const int ctid = tid - CB;
            // ---- 2. column pass (preprocess_cols.wgsl) -> P2 ----
            // item rq of a column covers row pairs p0 .. p0 + FM/2 - 1; the
            // last one is moved up to end at the last processed row pair
            // (the rows it shares with the item before come out the same)
            for (int it = ctid; it < G::PW * G::NRQ; it += CN) {
                const int rq = it / G::PW, c = it - rq * G::PW;
                const int p0 = min(rq * (FM / 2), G::PP - FM / 2);
                float2 L[FM / 2 + KR], ML[FM / 2 + KR - 1];
#pragma unroll
                for (int k2 = 0; k2 < FM / 2 + KR; ++k2) L[k2] = Gp[(p0 + k2) * G::GPS + c];
#pragma unroll
                for (int k2 = 0; k2 < FM / 2 + KR - 1; ++k2) ML[k2] = make_float2(L[k2].y, L[k2 + 1].x);
                float2 gq[FM / 2];
#pragma unroll
                for (int m = 0; m < FM / 2; ++m) {
                    float2 acc = make_float2(0.f, 0.f);
#pragma unroll
                    for (int j = 0; j < TAPS; ++j)
                        acc = fma2(W2[j], (j & 1) ? ML[m + (j >> 1)] : L[m + (j >> 1)], acc);
                    gq[m] = mul2(acc, RN2);
                }
                // the rows' box sums in scalar: the first window summed in tap
                // order, each next row's window slid by one row; every partial
                // sum is an integer below 2^24 (u16 frames), so all orders give
                // the same bits
                float2 cs[FM / 2];
                {
#pragma unroll
                    for (int k2 = 0; k2 < FM / 2 + KR; ++k2) L[k2] = Bp[(p0 + k2) * G::GPS + c];
                    float bsum[FM + 2 * KR];
#pragma unroll
                    for (int k2 = 0; k2 < FM / 2 + KR; ++k2) { bsum[2 * k2] = L[k2].x; bsum[2 * k2 + 1] = L[k2].y; }
                    float sb[FM];
                    float s0 = bsum[0];
#pragma unroll
                    for (int j = 1; j < TAPS; ++j) s0 = s0 + bsum[j];
                    sb[0] = s0;
#pragma unroll
                    for (int m = 1; m < FM; ++m) {
                        s0 = s0 + bsum[m + 2 * KR];
                        s0 = s0 - bsum[m - 1];
                        sb[m] = s0;
                    }
#pragma unroll
                    for (int m = 0; m < FM / 2; ++m) cs[m] = make_float2(sb[2 * m], sb[2 * m + 1]);
                }
#pragma unroll
                for (int m = 0; m < FM / 2; ++m) {
                    // preprocess_cols.wgsl:54 contracted: fma(-cs, 1/k^2, gauss);
                    // cs * -rkk is exactly -(cs * rkk)
                    const float2 res = fma2(cs[m], NRKK2, gq[m]);
                    // preprocess_cols.wgsl:55-60 clip at 0; res is never NaN or -0
                    // here (u16 frames, non-negative sums), where max equals the
                    // shader's select; positions outside the frame take -inf below
                    float2 o;
                    o.x = fmaxf(res.x, 0.f);
                    o.y = fmaxf(res.y, 0.f);
                    P2[(p0 + m) * G::P2S + c] = o;
                }
            }
            if (G::WS) bar_sync(5, NS);
            else __syncthreads();
            // ---- 2b. processed positions outside the frame take -inf (edge
            //          tiles only): rows above and below the frame, then
            //          columns left and right of it ----
            if (py0 < 0 || px0 < 0 || py0 + G::PH > H || px0 + G::PW > W) {
                float* Pf = (float*)P2;
                const int ra = min(G::PH, max(0, -py0)), rb = max(ra, min(G::PH, H - py0));
                const int ca = min(G::PW, max(0, -px0)), cb = max(ca, min(G::PW, W - px0));
                const int nrow = ra + (G::PH - rb), ncol = ca + (G::PW - cb);
                for (int i = ctid; i < nrow * G::PW; i += CN) {
                    const int k2 = i / G::PW, c = i - k2 * G::PW;
                    const int r = k2 < ra ? k2 : rb + (k2 - ra);
                    Pf[(((r >> 1) * G::P2S + c) << 1) + (r & 1)] = NEG;
                }
                for (int i = ctid; i < ncol * G::PH; i += CN) {
                    const int k2 = i / G::PH, r = i - k2 * G::PH;
                    const int c = k2 < ca ? k2 : cb + (k2 - ca);
                    Pf[(((r >> 1) * G::P2S + c) << 1) + (r & 1)] = NEG;
                }
                if (G::WS) bar_sync(5, NS);
                else __syncthreads();
            }

            // ---- 3. row max over the dilation window (max_rows.wgsl) ----
            for (int it = ctid; it < G::PP * (FT / FM); it += CN) {
                const int q = it / G::PP, pr = it - q * G::PP;
                const int tc0 = q * FM;
                const float2* src = P2 + pr * G::P2S + tc0 + HX - O;
                float vx[FM + DD - 1], vy[FM + DD - 1];
#pragma unroll
                for (int i = 0; i < FM + DD - 1; ++i) {
                    const float2 z = src[i];
                    vx[i] = z.x;
                    vy[i] = z.y;
                }
                float ox[FM], oy[FM];
                slide_max<DD, FM>(vx, ox);
                slide_max<DD, FM>(vy, oy);
#pragma unroll
                for (int m = 0; m < FM; ++m) RM2[pr * G::RMS + tc0 + m] = make_float2(ox[m], oy[m]);
            }
        }
        if (G::WS) bar_sync(3, NTK);  // the walkers of tile k - 1 arrive after their records
        else __syncthreads();

        // ---- 4. column max vs centre: non-strict local max (walk_cols.wgsl:19-36),
        //         listed at once: warp w owns tile rows 8 (w / 2) .. + 7 of
        //         column half w % 2, ballots each row and appends its flagged
        //         pixels to the CTA list (one shared atomic per warp; the order
        //         of the list does not matter: records carry their rank) ----
        static_assert(FT * (TH0 / FM) == NTK && FT == 64, "one column of 8 rows per thread");
        {
            const int tc = tid % FT, rq = tid / FT;
            const int tr0 = rq * FM;
            const int k0 = (tr0 + HP - O) >> 1;  // HP - O is even
            constexpr int NPR = (FM + DD - 1 + 1) / 2;
            float vv[2 * NPR];
#pragma unroll
            for (int k2 = 0; k2 < NPR; ++k2) {
                const float2 z = RM2[(k0 + k2) * G::RMS + tc];
                vv[2 * k2] = z.x;
                vv[2 * k2 + 1] = z.y;
            }
            float v[FM + DD - 1];
#pragma unroll
            for (int i = 0; i < FM + DD - 1; ++i) v[i] = vv[i];
            float cm[FM];
            slide_max<DD, FM>(v, cm);
            // a tile whose copy ran out of its wait lists nothing
            const bool col_in = f.tx0 + tc < W && !*(volatile int*)&s_fail;
            unsigned bal[FM];
            int nc = 0;
            const int nin = col_in ? f.TH - tr0 : 0;  // rows m < nin are in the frame
            // the centres: processed rows tr0 + HP .. tr0 + HP + FM - 1, read
            // as row pairs
            constexpr int CPO = HP & 1, NCP = (CPO + FM + 1) / 2;
            float cen[2 * NCP];
            {
                const int b0 = (tr0 + HP) >> 1;
#pragma unroll
                for (int k2 = 0; k2 < NCP; ++k2) {
                    const float2 z = P2[(b0 + k2) * G::P2S + tc + HX];
                    cen[2 * k2] = z.x;
                    cen[2 * k2 + 1] = z.y;
                }
            }
            // in-frame centres are >= 0: with zero_skip a centre must be > 0
            const float zthr = p.zero_skip ? 0.f : -1.f;
#pragma unroll
            for (int m = 0; m < FM; ++m) {
                const float center = cen[CPO + m];
                const bool fl = m < nin && cm[m] <= center && center > zthr;
                bal[m] = __ballot_sync(0xffffffffu, fl);
                nc += __popc(bal[m]);
            }
            const unsigned lt = (1u << lane) - 1u;
            int wbase = 0;
            if (lane == 0 && nc) wbase = atomicAdd(&s_nc, nc);
            wbase = __shfl_sync(0xffffffffu, wbase, 0);
#pragma unroll
            for (int m = 0; m < FM; ++m) {
                if (bal[m] != 0u) {  // warp-uniform: most rows list nothing
                    if ((bal[m] >> lane) & 1u)
                        clist[wbase + __popc(bal[m] & lt)] = (unsigned short)((tr0 + m) * FT + tc);
                    wbase += __popc(bal[m]);
                }
            }
        }
        __syncthreads();
        prev = f;
        f = next_tile<TH0>(p, f);
    }
    // a copy that ran out of the bounded wait gets a second one to land in
    // this CTA's shared memory before the CTA exits (no copy is issued after
    // a timeout, so only the last one can be in flight)
    if (use_tma && tid == PROD && s_fail) {
        bool done = false;
        for (int it = 0; it < p.tma_spin && !done; ++it) done = mbar_try_wait(&bar, last & 1);
    }
}

namespace {
// TMA descriptor over the movie (u16, dims W x H x T) with a box of the raw
// tile.  Needs a 16-byte aligned base and a row pitch multiple of 16 bytes.
bool make_tensor_map(CUtensorMap* map, const void* frames, int T, int H, int W, int box_w, int box_h) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return false;
        encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
    if (((uintptr_t)frames & 15) || (W * 2) % 16) return false;
    cuuint64_t dims[3] = {(cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)T};
    cuuint64_t strides[2] = {(cuuint64_t)W * 2, (cuuint64_t)W * H * 2};
    cuuint32_t box[3] = {(cuuint32_t)box_w, (cuuint32_t)box_h, 1};
    cuuint32_t es[3] = {1, 1, 1};
    CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_UINT16, 3, const_cast<void*>(frames), dims, strides, box, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}
}  // namespace

// (smoothing radius, dilation size, centroid radius) triples with a
// specialised kernel: diameters 5, 7, 9, 11 (odd, centroid radius
// (d - 1) / 2) with the default smoothing (= diameter) and separation
// (= diameter + 1), plus neighbouring separations.  Everything else uses
// locate_tiles_kernel.
#define GT_FAST_LIST(X) X(2, 8, 2) X(3, 11, 3) X(4, 14, 4) X(5, 16, 5) X(3, 8, 3) X(4, 11, 4) X(2, 7, 2) X(3, 12, 3)

bool fast_supported(int kr, int dd, int rc, int diameter) {
    if (diameter != 2 * rc + 1) return false;
#define GT_FAST_CASE(KR, DD, RC) if (kr == KR && dd == DD && rc == RC) return true;
    GT_FAST_LIST(GT_FAST_CASE)
#undef GT_FAST_CASE
    return false;
}

// Tiles per CTA of a launch of `total` tiles: runs of up to 16 consecutive
// tiles (within a run each tile's walks overlap the next tile's stencil
// phases and the next raw tile is copied in behind the current one), as
// long as the launch keeps about four waves of CTAs; p.tiles_per_cta > 0
// sets it.
int fast_tiles_per_cta(const LocParams& p, int total, int th) {
    if (p.tiles_per_cta > 0) return p.tiles_per_cta;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int slots = sms * (th == 32 ? 4 : 2);
    return std::max(1, std::min(16, total / (4 * slots)));
}

// Launches the specialised kernel over frames [frame0, frame0 + grid.y),
// grid.x tiles per frame.  *used_tma reports whether the raw tiles were
// staged by TMA.
cudaError_t launch_locate_fast(int kr, int dd, int rc, int th, dim3 grid, cudaStream_t st, const LocParams& p,
                               const MovieBufs& b, int T, int frame0, int* used_tma) {
    const long long total = (long long)grid.x * grid.y;
    if (total <= 0 || total > (1LL << 30)) return cudaErrorInvalidValue;
    const int per = fast_tiles_per_cta(p, (int)total, th);
    const unsigned nblk = (unsigned)((total + per - 1) / per);
#define GT_FAST_LAUNCH(KR, DD, RC, TH)                                                                  \
    {                                                                                                   \
        using G = Geo<KR, DD, TH, RC>;                                                                  \
        CUtensorMap map;                                                                                \
        std::memset(&map, 0, sizeof(map));                                                              \
        const int tma = make_tensor_map(&map, b.frames, T, p.H, p.W, G::US, G::RH) ? 1 : 0;            \
        *used_tma = tma;                                                                                \
        cudaError_t e = cudaFuncSetAttribute(locate_fast_kernel<KR, DD, TH, RC>,                         \
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM);      \
        if (e != cudaSuccess) return e;                                                                 \
        locate_fast_kernel<KR, DD, TH, RC><<<nblk, fast_threads(TH), G::SMEM, st>>>(p, b, map, tma, frame0, \
                                                                                   (int)grid.x, (int)total, per); \
        return cudaGetLastError();                                                                      \
    }
#define GT_FAST_CASE(KR, DD, RC)                                                                        \
    if (kr == KR && dd == DD && rc == RC) {                                                             \
        if (th == 32) GT_FAST_LAUNCH(KR, DD, RC, 32)                                                    \
        else GT_FAST_LAUNCH(KR, DD, RC, 64)                                                             \
    }
    GT_FAST_LIST(GT_FAST_CASE)
#undef GT_FAST_CASE
#undef GT_FAST_LAUNCH
    return cudaErrorInvalidValue;
}

}  // namespace gt
