// locate_fast.cu -- instruction-lean locate kernel for sm_100a.
//
// Same results, bit for bit, as locate_tiles_kernel (and the oracle): the
// per-pixel arithmetic chains are unchanged, only packed two per f32x2
// instruction, and the boxcar of uint16 frames uses running sums, which are
// exact because every partial sum is an integer below 2^24.
//
// One CTA per (frame, 64 x 64 output tile), 256 threads, 2 CTAs per SM:
//   0. the uint16 tile plus halo is staged by one TMA load (zero fill
//      outside the frame) into U[RH][RW];
//   1. U -> Rp: f32, rows interleaved in pairs (float2 = rows 2p, 2p+1);
//   2. row pass: a thread filters one row pair over 8 columns (f32x2 FMA
//      chains in tap order), Gaussian and boxcar -> Gp, Bp (row pairs);
//   3. column pass: a thread filters one column over 8 rows (4 row pairs),
//      divides by the Gaussian norm and k^2, clips at 0 -> P2 (row pairs);
//   4. row max over the dilation window (register sliding max) -> RM2;
//   5. column max of RM2 compared with the centre -> local-max flags;
//   6. flagged pixels are compacted in raster order, walked and emitted as
//      in locate_tiles_kernel.
// Row strides of the pair arrays are odd (in 8-byte units), so every
// lane-per-row access is bank-conflict free.
#include <cuda.h>

#include "gt_device.cuh"
#include "gt_simd.cuh"

namespace gt {

namespace {
constexpr int FT = 64;    // output tile width
constexpr int FNT = 256;  // threads
constexpr int FM = 8;     // outputs per thread item
constexpr int FCMAX = 512;

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

// max over v[m .. m+DD-1] for m = 0..M-1, sharing the common core
template <int DD, int M>
__device__ __forceinline__ void slide_max(const float (&v)[M + DD - 1], float (&out)[M]) {
    if constexpr (DD <= 0) {
#pragma unroll
        for (int m = 0; m < M; ++m) out[m] = -CUDART_INF_F;
    } else if constexpr (DD < M) {
#pragma unroll
        for (int m = 0; m < M; ++m) {
            float x = v[m];
#pragma unroll
            for (int j = 1; j < DD; ++j) x = fmaxf(x, v[m + j]);
            out[m] = x;
        }
    } else {
        float core = v[M - 1];
#pragma unroll
        for (int j = M; j < DD; ++j) core = fmaxf(core, v[j]);
        float suf[M];  // suf[m] = max(v[m .. M-2]), m <= M-2
        suf[M - 1] = -CUDART_INF_F;
#pragma unroll
        for (int m = M - 2; m >= 0; --m) suf[m] = fmaxf(v[m], suf[m + 1]);
        float pre = -CUDART_INF_F;  // max(v[DD .. DD+m-1])
#pragma unroll
        for (int m = 0; m < M; ++m) {
            if (m > 0) pre = fmaxf(pre, v[DD + m - 1]);
            out[m] = fmaxf(fmaxf(suf[m], core), pre);
        }
    }
}

struct P2Acc {  // processed plane held as row pairs, frame coordinates
    const float* P;  // float view of the float2 array
    int py0, px0, PH, PW, S;  // S = row-pair stride in float2
    __device__ bool covers(int u, int v) const {
        const int r = u - py0, c = v - px0;
        return r >= 0 && r < PH && c >= 0 && c < PW;
    }
    __device__ float operator()(int u, int v) const {
        const int r = u - py0, c = v - px0;
        return P[(((r >> 1) * S + c) << 1) + (r & 1)];
    }
};

struct GRawAcc {  // raw pixels straight from the frame (characterize only)
    const unsigned short* F;
    int W;
    __device__ float operator()(int u, int v) const { return (float)__ldg(F + (size_t)u * W + v); }
};

// floor(n / d) for n, d < 2^16 by one multiply-high (m = ceil(2^32 / d))
__device__ __forceinline__ int fdiv16(int n, unsigned int m) { return (int)__umulhi((unsigned int)n, m); }

// Centroid at (u, v) from the shared-memory tables (same order and
// arithmetic as centroid_at).
__device__ __forceinline__ bool centroid_tab(const LocParams& p, const P2Acc& P, const int* toff,
                                             const float2* tij, int K, int u, int v, float& c0, float& c1,
                                             float& m) {
    const int bd = p.border;
    if (u - bd < 0 || u + bd >= p.H || v - bd < 0 || v + bd >= p.W) {
        c0 = 0.f; c1 = 0.f; m = 0.f;
        return true;
    }
    const int rint = p.rint_c;
    if (!P.covers(u - rint, v - rint) || !P.covers(u + rint, v + rint)) return false;
    const int r0 = u - P.py0, cc = v - P.px0;
    const int base = (((r0 >> 1) * P.S + cc) << 1);
    const int* T = toff + (r0 & 1) * K;
    float a0 = 0.f, a1 = 0.f, mm = 0.f;
#pragma unroll 4
    for (int k = 0; k < K; ++k) {
        const float data = P.P[base + T[k]];
        const float2 ij = tij[k];
        a0 = fmaf(data, ij.x, a0);
        a1 = fmaf(data, ij.y, a1);
        mm = mm + data;
    }
    c0 = a0 / mm;
    c1 = a1 / mm;
    m = mm;
    return true;
}

__host__ __device__ constexpr int fast_offset(int DD) { return (int)((float)DD / 2.0f - 0.5f); }

}  // namespace

template <int KR, int DD, int TH0>
__global__ void __launch_bounds__(FNT, (TH0 == 32 ? 4 : 2))
    locate_fast_kernel(const LocParams p, const MovieBufs b, const FastGeo g,
                       const __grid_constant__ CUtensorMap tmap, int frame0) {
    constexpr int TAPS = 2 * KR + 1;
    constexpr int O = fast_offset(DD);
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ int warp_tot[FNT / 32];
    __shared__ int s_total, s_base, s_fail;
    __shared__ int rowcount[TH0];
    __shared__ int rowstart[TH0];

    const int tid = threadIdx.x;
    const int tile = blockIdx.x;
    const int t = frame0 + blockIdx.y;
    const int ti = tile / p.ntx, tj = tile - ti * p.ntx;
    const int ty0 = ti * TH0, tx0 = tj * FT;
    const int H = p.H, W = p.W;
    const int hp = g.hp, hx = g.hx;
    const int RH = g.RH, RW = g.RW, PH = g.PH, PW = g.PW;
    const int ry0 = ty0 - hp - KR, rx0 = tx0 - g.L;
    const int py0 = ty0 - hp, px0 = tx0 - hx;
    const int TH = min(TH0, H - ty0);

    float2* Rp = (float2*)(smem + g.off_rp);
    float2* P2 = Rp;  // P2 replaces Rp once the row pass is done
    float2* Gp = (float2*)(smem + g.off_gp);
    float2* Bp = (float2*)(smem + g.off_bp);
    unsigned short* U = (unsigned short*)Bp;   // raw tile until converted
    float2* RM2 = Gp;                          // after the column pass
    int* clist = (int*)Gp;                     // after the local-max pass
    unsigned char* flags = (unsigned char*)Bp;  // after the column pass
    float* wy = (float*)(smem + g.off_bp + TH0 * FT);
    float* wx = wy + FCMAX;
    float* wm = wx + FCMAX;
    int* wst = (int*)(wm + FCMAX);
    // circle tables (persist through the tile)
    int* ctoff = (int*)(smem + g.off_tab);            // 2 x K1: centroid offsets (even/odd base row)
    float2* ctij = (float2*)(ctoff + 2 * g.K1);       // K1: (i, j)
    int* xtoff = (int*)(ctij + g.K1);                 // 2 x K2: d/2 circle offsets
    float4* xtab = (float4*)(smem + g.off_tab2);      // K2: (r2, sin2, cos2, 0)

    // ---- 0. stage the raw tile ----
    if (g.use_tma) {
        if (tid == 0) {
            mbar_init(&bar, 1);
            s_fail = 0;
        }
        __syncthreads();
        if (tid == 0) {
            mbar_expect_tx(&bar, (uint32_t)(RH * RW * 2));
            tma_load_3d(U, &tmap, &bar, rx0, ry0, t);
            bool done = false;
            for (int it = 0; it < (1 << 22) && !done; ++it) done = mbar_try_wait(&bar, 0);
            if (!done) {
                atomicOr(b.err, ERR_DEVICE_TIMEOUT);
                s_fail = 1;
            }
        }
        __syncthreads();
        if (s_fail) return;
    } else {
        const unsigned short* fr = (const unsigned short*)b.frames + (size_t)t * H * W;
        for (int i = tid; i < RH * RW; i += FNT) {
            const int r = fdiv16(i, g.mRW), c = i - r * RW;
            const int gy = ry0 + r, gx = rx0 + c;
            unsigned short v = 0;
            if (gy >= 0 && gy < H && gx >= 0 && gx < W) v = __ldg(fr + (size_t)gy * W + gx);
            U[i] = v;
        }
        __syncthreads();
    }
    if (tid < TH0) {
        rowstart[tid] = 0x7fffffff;
        rowcount[tid] = 0;
    }
    // offsets of the centroid circle (radius (d-1)/2, centers.wgsl order) and
    // of the cpu_processed circle (radius d/2, kernels.rs order) in the row-pair
    // layout, for an even (first half) and an odd (second half) base row
    if (tid == 0) {
        int k = 0;
        const int rc = p.rint_c;
        for (int i = -rc; i <= rc; ++i)
            for (int j = -rc; j <= rc; ++j) {
                const float x = (float)i, y = (float)j;
                if (x * x + y * y > (float)rc * (float)rc) continue;
                for (int e = 0; e < 2; ++e)
                    ctoff[e * g.K1 + k] = ((((e + i) >> 1) * g.P2S + j) << 1) + ((e + i) & 1);
                ctij[k] = make_float2(x, y);
                ++k;
            }
    }
    for (int k = tid; k < g.K2; k += FNT) {
        const int i = __ldg(b.char_off + 2 * k), j = __ldg(b.char_off + 2 * k + 1);
        for (int e = 0; e < 2; ++e) xtoff[e * g.K2 + k] = ((((e + i) >> 1) * g.P2S + j) << 1) + ((e + i) & 1);
        xtab[k] = make_float4(__ldg(b.char_tab + 3 * k), __ldg(b.char_tab + 3 * k + 1),
                              __ldg(b.char_tab + 3 * k + 2), 0.f);
    }

    // ---- 1. u16 -> f32 row pairs ----
    const int RP = RH >> 1;
    for (int i = tid; i < RP * RW; i += FNT) {
        const int pr = fdiv16(i, g.mRW), c = i - pr * RW;
        Rp[pr * g.RPS + c] = make_float2((float)U[(2 * pr) * RW + c], (float)U[(2 * pr + 1) * RW + c]);
    }
    __syncthreads();

    float2 W2[TAPS];
#pragma unroll
    for (int j = 0; j < TAPS; ++j) W2[j] = make_float2(p.w[j], p.w[j]);
    constexpr bool fd = true;  // the host verified the fixed-divisor division

    // ---- 2. row pass (preprocess_rows.wgsl) on row pairs ----
    for (int it = tid; it < RP * g.NPW; it += FNT) {
        const int q = fdiv16(it, g.mRP), pr = it - q * RP;
        const int pc0 = q * FM;
        const float2* src = Rp + pr * g.RPS + pc0;
        float2 v[FM + 2 * KR];
#pragma unroll
        for (int i = 0; i < FM + 2 * KR; ++i) v[i] = src[i];
        float2* gd = Gp + pr * g.GPS + pc0;
        float2* bd = Bp + pr * g.GPS + pc0;
#pragma unroll
        for (int m = 0; m < FM; ++m) {
            float2 acc = make_float2(0.f, 0.f);
#pragma unroll
            for (int j = 0; j < TAPS; ++j) acc = fma2(W2[j], v[m + j], acc);
            gd[m] = fd ? div2(acc, g.dnorm) : make_float2(acc.x / p.norm, acc.y / p.norm);
        }
        const int fc0 = rx0 + pc0;  // frame column of v[0]
        if (fc0 >= 0 && fc0 + FM + 2 * KR - 1 < W) {
            float2 s = v[0];
#pragma unroll
            for (int j = 1; j < TAPS; ++j) s = add2(s, v[j]);
            bd[0] = s;
#pragma unroll
            for (int m = 1; m < FM; ++m) {
                s = sub2(add2(s, v[m + 2 * KR]), v[m - 1]);
                bd[m] = s;
            }
        } else {
            // reflect-padded boxcar at the left/right frame edges
#pragma unroll
            for (int m = 0; m < FM; ++m) {
                const int fc = fc0 + m + KR;
                float2 s = make_float2(0.f, 0.f);
#pragma unroll
                for (int j = 0; j < TAPS; ++j) {
                    const int cc = clampi(reflect_once(fc - KR + j, W) - rx0, 0, RW - 1);
                    s = add2(s, Rp[pr * g.RPS + cc]);
                }
                bd[m] = s;
            }
        }
    }
    __syncthreads();

    // ---- 3. column pass (preprocess_cols.wgsl) -> P2 ----
    const float NEG = -CUDART_INF_F;
    for (int it = tid; it < g.PWC * g.NRQ; it += FNT) {
        const int rq = fdiv16(it, g.mPWC), c = it - rq * g.PWC;
        const int p0 = rq * (FM / 2);
        float2 L[FM / 2 + KR], ML[FM / 2 + KR - 1];
#pragma unroll
        for (int k = 0; k < FM / 2 + KR; ++k) L[k] = Gp[(p0 + k) * g.GPS + c];
#pragma unroll
        for (int k = 0; k < FM / 2 + KR - 1; ++k) ML[k] = make_float2(L[k].y, L[k + 1].x);
        float2 gq[FM / 2];
#pragma unroll
        for (int m = 0; m < FM / 2; ++m) {
            float2 acc = make_float2(0.f, 0.f);
#pragma unroll
            for (int j = 0; j < TAPS; ++j) acc = fma2(W2[j], (j & 1) ? ML[m + (j >> 1)] : L[m + (j >> 1)], acc);
            gq[m] = fd ? div2(acc, g.dnorm) : make_float2(acc.x / p.norm, acc.y / p.norm);
        }
        float2 cs[FM / 2];
        const int fr0 = ry0 + 2 * p0;  // frame row of raw row 2*p0
        if (fr0 >= 0 && fr0 + FM + 2 * KR - 1 < H) {
#pragma unroll
            for (int k = 0; k < FM / 2 + KR; ++k) L[k] = Bp[(p0 + k) * g.GPS + c];
#pragma unroll
            for (int k = 0; k < FM / 2 + KR - 1; ++k) ML[k] = make_float2(L[k].y, L[k + 1].x);
#pragma unroll
            for (int m = 0; m < FM / 2; ++m) {
                float2 s = L[m];
#pragma unroll
                for (int j = 1; j < TAPS; ++j) s = add2(s, (j & 1) ? ML[m + (j >> 1)] : L[m + (j >> 1)]);
                cs[m] = s;
            }
        } else {
            // reflect-padded boxcar at the top/bottom frame edges
            const float* Bf = (const float*)Bp;
#pragma unroll
            for (int m = 0; m < FM / 2; ++m) {
                float sx = 0.f, sy = 0.f;
                const int fa = fr0 + 2 * m + KR;  // frame row of the output pair's first row
#pragma unroll
                for (int j = 0; j < TAPS; ++j) {
                    const int ra = clampi(reflect_once(fa - KR + j, H) - ry0, 0, RH - 1);
                    const int rb = clampi(reflect_once(fa + 1 - KR + j, H) - ry0, 0, RH - 1);
                    sx = sx + Bf[(((ra >> 1) * g.GPS + c) << 1) + (ra & 1)];
                    sy = sy + Bf[(((rb >> 1) * g.GPS + c) << 1) + (rb & 1)];
                }
                cs[m] = make_float2(sx, sy);
            }
        }
        const int fc = px0 + c;
        const bool cin = fc >= 0 && fc < W && c < PW;
#pragma unroll
        for (int m = 0; m < FM / 2; ++m) {
            const float2 bq = fd ? div2(cs[m], g.dkk) : make_float2(cs[m].x / p.kk, cs[m].y / p.kk);
            const float2 res = sub2(gq[m], bq);
            const int fa = py0 + 2 * (p0 + m);
            float2 o;
            o.x = (cin && fa >= 0 && fa < H) ? (res.x < 0.f ? 0.f : res.x) : NEG;
            o.y = (cin && fa + 1 >= 0 && fa + 1 < H) ? (res.y < 0.f ? 0.f : res.y) : NEG;
            P2[(p0 + m) * g.P2S + c] = o;
        }
    }
    __syncthreads();

    // ---- 4. row max over the dilation window (max_rows.wgsl) ----
    const int PP = PH >> 1;
    for (int it = tid; it < PP * (FT / FM); it += FNT) {
        const int q = fdiv16(it, g.mPP), pr = it - q * PP;
        const int tc0 = q * FM;
        const float2* src = P2 + pr * g.P2S + tc0 + hx - O;
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
        for (int m = 0; m < FM; ++m) RM2[pr * g.RMS + tc0 + m] = make_float2(ox[m], oy[m]);
    }
    __syncthreads();

    // ---- 5. column max vs centre: non-strict local max (walk_cols.wgsl:19-36) ----
    for (int it = tid; it < FT * (TH0 / FM); it += FNT) {
        const int tc = it % FT, rq = it / FT;
        const int tr0 = rq * FM;
        const int k0 = (tr0 + hp - O) >> 1;  // hp - O is even
        constexpr int NPR = (FM + DD - 1 + 1) / 2;
        float v[2 * NPR];
#pragma unroll
        for (int k = 0; k < NPR; ++k) {
            const float2 z = RM2[(k0 + k) * g.RMS + tc];
            v[2 * k] = z.x;
            v[2 * k + 1] = z.y;
        }
        float vv[FM + DD - 1];
#pragma unroll
        for (int i = 0; i < FM + DD - 1; ++i) vv[i] = v[i];
        float cm[FM];
        slide_max<DD, FM>(vv, cm);
        const float* Pf = (const float*)P2;
#pragma unroll
        for (int m = 0; m < FM; ++m) {
            const int r = tr0 + m + hp;  // processed row of the centre
            const float center = Pf[(((r >> 1) * g.P2S + tc + hx) << 1) + (r & 1)];
            const bool in = tr0 + m < TH && tx0 + tc < W;
            const bool f = in && cm[m] <= center && !(p.zero_skip && center == 0.f);
            flags[(tr0 + m) * FT + tc] = f ? 1 : 0;
        }
    }
    __syncthreads();

    // ---- 6. raster-order compaction, walks, emission ----
    const int npx = TH0 * FT;
    const int chunk = npx / FNT;  // 8 or 16 flags per thread
    const int q0 = tid * chunk;
    int mine = 0;
    for (int i = 0; i < chunk; ++i) mine += flags[q0 + i];
    int pos = block_excl_scan<FNT>(mine, warp_tot, &s_total);
    const int ncand = s_total;
    for (int q = q0; q < q0 + chunk; ++q)
        if (flags[q]) clist[pos++] = q;
    __syncthreads();

    P2Acc acc{(const float*)P2, py0, px0, PH, PW, g.P2S};
    const unsigned short* frame = (const unsigned short*)b.frames + (size_t)t * H * W;
    GRawAcc racc{frame, W};
    // thread k serves candidate (k % 32) * 8 + k / 32: one lane per warp first
    const int cidx = (tid & 31) * (FNT / 32) + (tid >> 5);
    int emitted = 0;
    for (int r0 = 0; r0 < ncand; r0 += FCMAX) {
        const int nr = min(FCMAX, ncand - r0);
        for (int c = cidx; c < nr; c += FNT) {
            const int q = clist[r0 + c];
            const int u0 = ty0 + q / FT, v0 = tx0 + q % FT;
            int st;
            float y = 0.f, x = 0.f, m = 0.f;
            if (p.max_iter <= 0) {
                st = CAND_PENDING;
            } else {
                // walk_cols.wgsl:38-74
                int u = u0, v = v0;
                float c0 = 0.f, c1 = 0.f;
                bool ok = true;
                for (int iter = 0; iter < p.max_iter; ++iter) {
                    if (!centroid_tab(p, acc, ctoff, ctij, g.K1, u, v, c0, c1, m)) { ok = false; break; }
                    bool changed = false;
                    if (c0 > p.thr && u < H - 1) { u += 1; changed = true; }
                    else if (c0 < -p.thr && u > 0) { u -= 1; changed = true; }
                    if (c1 > p.thr && v < W - 1) { v += 1; changed = true; }
                    else if (c1 < -p.thr && v > 0) { v -= 1; changed = true; }
                    if (!changed) break;
                }
                if (!ok) {
                    st = CAND_PENDING;
                    m = 0.f;
                } else {
                    y = (float)u + c0;
                    x = (float)v + c1;
                    st = (m > p.minmass && m != 0.f) ? CAND_EMIT : CAND_REJECT;
                }
            }
            wy[c] = y; wx[c] = x; wm[c] = m; wst[c] = st;
        }
        __syncthreads();
        const int cchunk = (nr + FNT - 1) / FNT;
        const int c0 = tid * cchunk, c1 = min(c0 + cchunk, nr);
        int ne = 0;
        for (int c = c0; c < c1; ++c) ne += (wst[c] != CAND_REJECT);
        int epos = block_excl_scan<FNT>(ne, warp_tot, &s_total);
        const int nemit = s_total;
        if (tid == 0) {
            int base = 0;
            if (nemit > 0) base = atomicAdd(b.fcount + t, nemit);
            if (base + nemit > b.cap_c) { atomicOr(b.err, ERR_CAND_OVERFLOW); base = -1; }
            s_base = base;
        }
        {
            int e = emitted + epos;
            for (int c = c0; c < c1; ++c) {
                if (wst[c] == CAND_REJECT) continue;
                const int tr = clist[r0 + c] / FT;
                atomicMin(&rowstart[tr], e);
                atomicAdd(&rowcount[tr], 1);
                ++e;
            }
        }
        __syncthreads();
        const int base = s_base;
        for (int c = c0; c < c1; ++c) {
            if (wst[c] == CAND_REJECT) continue;
            const int q = clist[r0 + c];
            const int tr = q / FT;
            const int u0 = ty0 + tr, v0 = tx0 + (q - tr * FT);
            Cand rec;
            rec.u = u0; rec.v = v0;
            rec.y = wy[c]; rec.x = wx[c]; rec.mass = wm[c];
            rec.rowrank = emitted + epos - rowstart[tr];
            rec.state = wst[c];
            rec.rg_sum = rec.eccn = rec.mid = rec.signal = 0.f;
            rec.g_rg = rec.g_raw = rec.g_sig = rec.g_ecc = 0.f;
            rec.pad = 0.f;
            if (p.cpu_processed) {
                // execute_gpu.rs:286-299: products summed per ndarray's
                // eight-accumulator fold, all three sums in one pass
                const int rr = u0 - py0, cc = v0 - px0;
                const int base2 = (((rr >> 1) * g.P2S + cc) << 1);
                const int* T = xtoff + (rr & 1) * g.K2;
                const float* Pf = (const float*)P2;
                float ar[8], as[8], ac[8];
#pragma unroll
                for (int l = 0; l < 8; ++l) { ar[l] = 0.f; as[l] = 0.f; ac[l] = 0.f; }
                const int K = g.K2, K8 = K & ~7;
                float sig = Pf[base2 + T[0]];
                for (int k0 = 0; k0 < K8; k0 += 8) {
#pragma unroll
                    for (int l = 0; l < 8; ++l) {
                        const float nb = Pf[base2 + T[k0 + l]];
                        const float4 tb = xtab[k0 + l];
                        ar[l] = ar[l] + nb * tb.x;
                        as[l] = as[l] + nb * tb.y;
                        ac[l] = ac[l] + nb * tb.z;
                        sig = fmaxf(sig, nb);
                    }
                }
                float rg = 0.f, sn = 0.f, cs = 0.f;
                rg = rg + (ar[0] + ar[4]); rg = rg + (ar[1] + ar[5]); rg = rg + (ar[2] + ar[6]); rg = rg + (ar[3] + ar[7]);
                sn = sn + (as[0] + as[4]); sn = sn + (as[1] + as[5]); sn = sn + (as[2] + as[6]); sn = sn + (as[3] + as[7]);
                cs = cs + (ac[0] + ac[4]); cs = cs + (ac[1] + ac[5]); cs = cs + (ac[2] + ac[6]); cs = cs + (ac[3] + ac[7]);
                for (int k = K8; k < K; ++k) {
                    const float nb = Pf[base2 + T[k]];
                    const float4 tb = xtab[k];
                    rg = rg + nb * tb.x;
                    sn = sn + nb * tb.y;
                    cs = cs + nb * tb.z;
                    sig = fmaxf(sig, nb);
                }
                rec.rg_sum = rg;
                rec.eccn = sqrtf(sn * sn + cs * cs);
                rec.mid = acc(u0, v0);
                rec.signal = sig;
            }
            if (p.characterize) gpu_features(p, b, acc, racc, u0, v0, rec);
            if (base >= 0) {
                const int slot = base + epos;
                b.cand[(size_t)t * b.cap_c + slot] = rec;
                if (rec.state == CAND_PENDING) {
                    const int k = atomicAdd(b.npend, 1);
                    b.pend[k] = t * b.cap_c + slot;
                }
            }
            ++epos;
        }
        emitted += nemit;
        __syncthreads();
    }
    for (int r = tid; r < TH; r += FNT) b.rowcnt[((size_t)t * H + ty0 + r) * p.ntx + tj] = rowcount[r];
}

// Checks div1() against IEEE division for 0 and every binary32 dividend in
// [2^-100, FLT_MAX].  Dividends of the fast kernel lie there: boxcar sums are
// integers, and with every Gaussian weight >= 2^-40 (checked on the host) a
// nonzero weighted sum of integer pixels is >= 2^-86.
__global__ void verify_division_kernel(float divisor, FixedDiv f, unsigned int* mismatches) {
    const unsigned int stride = gridDim.x * blockDim.x;
    unsigned int bad = 0;
    const unsigned int lo = 0x0d800000u;  // 2^-100
    const unsigned int tid0 = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid0 == 0) bad += (__float_as_uint(div1(0.f, f)) != __float_as_uint(__fdiv_rn(0.f, divisor)));
    for (unsigned int bits = lo + tid0; bits < 0x7f800000u; bits += stride) {
        const float a = __uint_as_float(bits);
        const float want = __fdiv_rn(a, divisor);
        const float got = div1(a, f);
        bad += (__float_as_uint(want) != __float_as_uint(got));
    }
    if (bad) atomicAdd(mismatches, bad);
}

// (smoothing radius, dilation size) pairs with a specialised kernel; other
// parameter sets use locate_tiles_kernel.  Covers diameters 5-11 with the
// default separation (diameter + 1) and smoothing (diameter).
#define GT_FAST_LIST(X) X(2, 8) X(3, 11) X(4, 14) X(5, 16) X(2, 11) X(3, 8) X(4, 11) X(3, 14)

bool fast_supported(int kr, int dd) {
#define GT_FAST_CASE(KR, DD) if (kr == KR && dd == DD) return true;
    GT_FAST_LIST(GT_FAST_CASE)
#undef GT_FAST_CASE
    return false;
}

cudaError_t launch_locate_fast(int kr, int dd, int th, dim3 grid, cudaStream_t st, const LocParams& p,
                               const MovieBufs& b, const FastGeo& g, const CUtensorMap& map, int frame0) {
#define GT_FAST_CASE(KR, DD)                                                                          \
    if (kr == KR && dd == DD) {                                                                       \
        if (th == 32) {                                                                               \
            cudaError_t e = cudaFuncSetAttribute(locate_fast_kernel<KR, DD, 32>,                       \
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, g.smem); \
            if (e != cudaSuccess) return e;                                                           \
            locate_fast_kernel<KR, DD, 32><<<grid, FNT, g.smem, st>>>(p, b, g, map, frame0);           \
        } else {                                                                                      \
            cudaError_t e = cudaFuncSetAttribute(locate_fast_kernel<KR, DD, 64>,                       \
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, g.smem); \
            if (e != cudaSuccess) return e;                                                           \
            locate_fast_kernel<KR, DD, 64><<<grid, FNT, g.smem, st>>>(p, b, g, map, frame0);           \
        }                                                                                             \
        return cudaGetLastError();                                                                    \
    }
    GT_FAST_LIST(GT_FAST_CASE)
#undef GT_FAST_CASE
    return cudaErrorInvalidValue;
}

cudaError_t launch_verify_division(float divisor, FixedDiv f, unsigned int* d_count, int num_sms,
                                   cudaStream_t st) {
    verify_division_kernel<<<num_sms * 16, 256, 0, st>>>(divisor, f, d_count);
    return cudaGetLastError();
}

}  // namespace gt
