// locate.cu -- fused bandpass -> grey-dilation local max -> centroid walk
// kernel, one CTA per (frame, TH x TW tile).
//
// Replaces the five WGSL dispatches of the reference
// (shaders/preprocess_rows.wgsl, preprocess_cols.wgsl, centers.wgsl,
// max_rows.wgsl, walk_cols.wgsl, dispatched by execute_gpu.rs:82-88) and the
// host-side dense raster scan (execute_gpu.rs:157-183): the processed plane
// never leaves shared memory, the centroid is evaluated only where a walk
// reads it, and features are emitted as compact records with per-(row, tile
// column) counts from which the finalize kernel restores raster order.
//
// Shared-memory layout of one tile (floats):
//   R   raw pixels, (PH + 2k) x (PW + 2k), zero outside the frame
//   Gr  row-pass Gaussian, (PH + 2k) x PW
//   Br  row-pass boxcar,   (PH + 2k) x PW
//   P   processed,          PH x PW, -inf outside the frame
// with PH = TH + 2*hp, PW = TW + 2*hp, k = smoothing radius.
#include "gt_device.cuh"

namespace gt {

namespace {

struct TileAcc {  // processed plane in shared memory, frame coordinates
    const float* P;
    int py0, px0, PH, PW;
    __device__ bool covers(int u, int v) const {
        return u >= py0 && u < py0 + PH && v >= px0 && v < px0 + PW;
    }
    __device__ float operator()(int u, int v) const { return P[(u - py0) * PW + (v - px0)]; }
};

struct RawAcc {
    const float* R;
    int ry0, rx0, RW;
    __device__ float operator()(int u, int v) const { return R[(u - ry0) * RW + (v - rx0)]; }
};

constexpr int NT = 256;
constexpr int CMAX = 512;  // walk results held in shared memory per round

}  // namespace

__global__ void __launch_bounds__(NT) locate_tiles_kernel(const LocParams p, const MovieBufs b,
                                                          int frame0) {
    extern __shared__ __align__(16) float sm[];
    __shared__ int warp_tot[NT / 32];
    __shared__ int s_total, s_base;
    __shared__ int rowcount[128];
    __shared__ int rowstart[128];

    const int tile = blockIdx.x;
    const int t = frame0 + blockIdx.y;
    const int ti = tile / p.ntx, tj = tile - ti * p.ntx;
    const int ty0 = ti * p.TH, tx0 = tj * p.TW;
    const int TH = min(p.TH, p.H - ty0), TW = p.TW;  // TW fixed for layout
    const int hp = p.hp, kr = p.krad, taps = p.taps;
    const int PH = p.TH + 2 * hp, PW = TW + 2 * hp;
    const int RH = PH + 2 * kr, RW = PW + 2 * kr;
    const int py0 = ty0 - hp, px0 = tx0 - hp;
    const int ry0 = py0 - kr, rx0 = px0 - kr;
    const int H = p.H, W = p.W;
    const bool border = ry0 < 0 || rx0 < 0 || ry0 + RH > H || rx0 + RW > W;

    float* R = sm;
    float* Gr = R + RH * RW;
    float* Br = Gr + RH * PW;
    float* P = Br + RH * PW;
    int* clist = (int*)(P + PH * PW);                 // TH*TW candidate pixels
    float* wy = (float*)(clist + p.TH * TW);           // CMAX walk results
    float* wx = wy + CMAX;
    float* wm = wx + CMAX;
    int* wst = (int*)(wm + CMAX);
    unsigned int* wlp = (unsigned int*)(wst + CMAX);  // last-read pixel (u << 16 | v)
    unsigned int* wfp = wlp + CMAX;                   // final position (u << 16 | v)
    unsigned char* flags = (unsigned char*)(wfp + CMAX);

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const size_t fbase = (size_t)t * H * W;

    // ---- A: raw tile (zero outside the frame) ----
    for (int r = warp; r < RH; r += NT / 32) {
        const int fr = ry0 + r;
        for (int c = lane; c < RW; c += 32) {
            const int fc = rx0 + c;
            float val = 0.f;
            if (fr >= 0 && fr < H && fc >= 0 && fc < W) val = load_px(b.frames, p.dtype, fbase + (size_t)fr * W + fc);
            R[r * RW + c] = val;
        }
    }
    if (threadIdx.x < 128) { rowstart[threadIdx.x] = 0x7fffffff; rowcount[threadIdx.x] = 0; }
    __syncthreads();

    // ---- B: row pass (preprocess_rows.wgsl:30-52) ----
    for (int r = warp; r < RH; r += NT / 32) {
        const float* Rr = R + r * RW;
        for (int pc = lane; pc < PW; pc += 32) {
            float gs = 0.f, cs = 0.f;
            if (!border) {
                for (int j = 0; j < taps; ++j) {
                    const float val = Rr[pc + j];
                    gs = fmaf(p.w[j], val, gs);
                    cs = cs + val;
                }
            } else {
                const int fc = px0 + pc;
                for (int j = 0; j < taps; ++j) {
                    gs = fmaf(p.w[j], Rr[pc + j], gs);  // zero outside: exact skip
                    const int cc = clampi(reflect_once(fc + j - kr, W) - rx0, 0, RW - 1);
                    cs = cs + Rr[cc];
                }
            }
            Gr[r * PW + pc] = gs * p.rn;  // preprocess_rows.wgsl:52 gauss_sum / gauss_norm
            Br[r * PW + pc] = cs;
        }
    }
    __syncthreads();

    // ---- C: column pass + clip (preprocess_cols.wgsl:32-60) ----
    for (int pr = warp; pr < PH; pr += NT / 32) {
        const int fr = py0 + pr;
        for (int pc = lane; pc < PW; pc += 32) {
            const int fc = px0 + pc;
            float out = -CUDART_INF_F;
            if (fr >= 0 && fr < H && fc >= 0 && fc < W) {
                float gs = 0.f, cs = 0.f;
                if (!border) {
                    for (int j = 0; j < taps; ++j) {
                        gs = fmaf(p.w[j], Gr[(pr + j) * PW + pc], gs);
                        cs = cs + Br[(pr + j) * PW + pc];
                    }
                } else {
                    for (int j = 0; j < taps; ++j) {
                        gs = fmaf(p.w[j], Gr[(pr + j) * PW + pc], gs);  // zero rows outside
                        const int rr = clampi(reflect_once(fr + j - kr, H) - ry0, 0, RH - 1);
                        cs = cs + Br[rr * PW + pc];
                    }
                }
                // preprocess_cols.wgsl:54, contracted: fma(-cs, 1/k^2, gs / norm)
                const float res = fmaf(-cs, p.rkk, gs * p.rn);
                out = res < 0.f ? 0.f : res;
            }
            P[pr * PW + pc] = out;
        }
    }
    __syncthreads();

    // ---- D: row max over the dilation window (max_rows.wgsl:10-28) ----
    float* RM = Gr;  // PH x TW
    for (int pr = warp; pr < PH; pr += NT / 32) {
        for (int tc = lane; tc < TW; tc += 32) {
            const float* Pr = P + pr * PW + tc + hp;
            float m = Pr[0];
            for (int j = 0; j < p.D; ++j) m = fmaxf(m, Pr[j - p.o]);
            RM[pr * TW + tc] = m;
        }
    }
    __syncthreads();

    // ---- E: non-strict local max (walk_cols.wgsl:19-36) ----
    const int npx = p.TH * TW;
    for (int q = threadIdx.x; q < npx; q += NT) {
        const int tr = q / TW, tc = q - tr * TW;
        unsigned char f = 0;
        if (tr < TH && tx0 + tc < W) {
            const float center = P[(tr + hp) * PW + tc + hp];
            bool ismax = true;
            for (int i = 0; i < p.D; ++i)
                if (RM[(tr + hp - p.o + i) * TW + tc] > center) { ismax = false; break; }
            if (ismax && !(p.zero_skip && center == 0.f)) f = 1;
        }
        flags[q] = f;
    }
    __syncthreads();
    // compaction in raster order: thread owns a contiguous chunk
    const int chunk = (npx + NT - 1) / NT;
    const int q0 = threadIdx.x * chunk;
    int mine = 0;
    for (int q = q0; q < min(q0 + chunk, npx); ++q) mine += flags[q];
    int pos = block_excl_scan<NT>(mine, warp_tot, &s_total);
    const int ncand = s_total;
    for (int q = q0; q < min(q0 + chunk, npx); ++q)
        if (flags[q]) clist[pos++] = q;
    __syncthreads();

    // ---- F/G: walks and emission, in raster-ordered rounds of CMAX ----
    TileAcc acc{P, py0, px0, PH, PW};
    RawAcc racc{R, ry0, rx0, RW};
    int emitted = 0;  // emitted records of this tile before the round
    for (int r0 = 0; r0 < ncand; r0 += CMAX) {
        const int nr = min(CMAX, ncand - r0);
        for (int c = threadIdx.x; c < nr; c += NT) {
            const int q = clist[r0 + c];
            const int u0 = ty0 + q / TW, v0 = tx0 + q % TW;
            int st;
            float y = 0.f, x = 0.f, m = 0.f;
            unsigned int lp = 0, fp = 0;
            if (p.max_iter <= 0) {
                st = CAND_PENDING;  // mass read at pixel 0: resolved by the fallback kernel
            } else {
                WalkOut wo = walk_from(p, acc, u0, v0);
                if (!wo.ok) {
                    st = CAND_PENDING;
                } else {
                    y = wo.y; x = wo.x; m = wo.mass;
                    st = (m > p.minmass && m != 0.f) ? CAND_EMIT : CAND_REJECT;
                    lp = ((unsigned)wo.ul << 16) | (unsigned)wo.vl;
                    fp = ((unsigned)wo.up << 16) | (unsigned)wo.vp;
                }
            }
            wy[c] = y; wx[c] = x; wm[c] = m; wst[c] = st; wlp[c] = lp; wfp[c] = fp;
        }
        __syncthreads();
        const int cchunk = (nr + NT - 1) / NT;
        const int c0 = threadIdx.x * cchunk, c1 = min(c0 + cchunk, nr);
        int ne = 0;
        for (int c = c0; c < c1; ++c) ne += (wst[c] != CAND_REJECT);
        int epos = block_excl_scan<NT>(ne, warp_tot, &s_total);
        const int nemit = s_total;
        if (threadIdx.x == 0) {
            int base = 0;
            if (nemit > 0) base = atomicAdd(b.fcount + t, nemit);
            if (base + nemit > b.cap_c) { atomicOr(b.err, ERR_CAND_OVERFLOW); base = -1; }
            s_base = base;
        }
        {
            int e = emitted + epos;
            for (int c = c0; c < c1; ++c) {
                if (wst[c] == CAND_REJECT) continue;
                const int tr = clist[r0 + c] / TW;
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
            const int tr = q / TW;
            const int u0 = ty0 + tr, v0 = tx0 + (q - tr * TW);
            Cand rec;
            rec.u = u0; rec.v = v0;
            rec.y = wy[c]; rec.x = wx[c]; rec.mass = wm[c];
            rec.rowrank = emitted + epos - rowstart[tr];
            rec.state = wst[c];
            rec.rg_sum = rec.eccn = rec.mid = rec.signal = 0.f;
            rec.g_rg = rec.g_raw = rec.g_sig = rec.g_ecc = 0.f;
            rec.ul = (int)(wlp[c] >> 16); rec.vl = (int)(wlp[c] & 0xffffu);
            rec.up = (int)(wfp[c] >> 16); rec.vp = (int)(wfp[c] & 0xffffu);
            rec.pad = 0;
            if (p.cpu_processed) cpu_features(p, b, acc, u0, v0, rec);
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
    // per-(row, tile column) record counts
    for (int r = threadIdx.x; r < TH; r += NT)
        b.rowcnt[((size_t)t * H + ty0 + r) * p.ntx + tj] = rowcount[r];
}

// Fallback walk for features whose walk left the tile halo (and for
// max_iterations == 0): recompute the processed values it needs straight
// from the frame, with the same arithmetic, into a shared-memory window.
namespace {
struct WinAcc {
    const float* P;
    int y0, x0, n;
    __device__ bool covers(int u, int v) const { return u >= y0 && u < y0 + n && v >= x0 && v < x0 + n; }
    __device__ float operator()(int u, int v) const { return P[(u - y0) * n + (v - x0)]; }
};
}  // namespace

// processed value at one pixel, straight from the frame (row pass then column
// pass in shader order); used to fill the fallback window.
__device__ float processed_at(const LocParams& p, const void* frames, size_t fbase, int u, int v) {
    const int kr = p.krad, H = p.H, W = p.W;
    float gs = 0.f, cs = 0.f;
    for (int i = -kr; i <= kr; ++i) {
        int pu = u + i;
        bool dg = true;
        if (pu < 0) { pu = -pu - 1; dg = false; }
        else if (pu >= H) { pu = 2 * H - pu - 1; dg = false; }
        // row pass at (pu, v)
        float rg = 0.f, rb = 0.f;
        for (int j = -kr; j <= kr; ++j) {
            int pv = v + j;
            bool dgv = true;
            if (pv < 0) { pv = -pv - 1; dgv = false; }
            else if (pv >= W) { pv = 2 * W - pv - 1; dgv = false; }
            const float val = load_px(frames, p.dtype, fbase + (size_t)pu * W + pv);
            if (dgv) rg = fmaf(p.w[j + kr], val, rg);
            rb = rb + val;
        }
        const float tg = rg * p.rn;
        if (dg) gs = fmaf(p.w[i + kr], tg, gs);
        cs = cs + rb;
    }
    const float res = fmaf(-cs, p.rkk, gs * p.rn);
    return res < 0.f ? 0.f : res;
}

__global__ void __launch_bounds__(128) fallback_walk_kernel(const LocParams p, const MovieBufs b, int win,
                                                            const int* pbeg) {
    extern __shared__ __align__(16) float wsm[];
    const int npend = *b.npend;
    const int n = 2 * win + 1;
    // entries from *pbeg on: those of the frames located since (chunked calls)
    for (int k = (pbeg ? *pbeg : 0) + blockIdx.x; k < npend; k += gridDim.x) {
        const int code = b.pend[k];
        const int t = code / b.cap_c;
        Cand* rec = b.cand + code;
        const int u0 = rec->u, v0 = rec->v;
        const size_t fbase = (size_t)t * p.H * p.W;
        const int y0 = u0 - win, x0 = v0 - win;
        __syncthreads();
        for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
            const int u = y0 + q / n, v = x0 + q % n;
            float val = 0.f;
            if (u >= 0 && u < p.H && v >= 0 && v < p.W) val = processed_at(p, b.frames, fbase, u, v);
            wsm[q] = val;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            WinAcc acc{wsm, y0, x0, n};
            float y, x, m;
            bool ok = true;
            int ul = 0, vl = 0, up = u0, vp = v0;
            if (p.max_iter <= 0) {
                // walk_cols.wgsl:69-73 with no iteration: offset (0, 0) and the
                // mass of pixel 0, which is interior only when d/2 == 0 (its
                // circle is then the pixel itself)
                y = (float)u0; x = (float)v0;
                m = (p.border == 0) ? processed_at(p, b.frames, fbase, 0, 0) : 0.f;
            } else {
                WalkOut wo = walk_from(p, acc, u0, v0);
                ok = wo.ok != 0;
                y = wo.y; x = wo.x; m = wo.mass;
                ul = wo.ul; vl = wo.vl; up = wo.up; vp = wo.vp;
            }
            if (!ok) {  // window too small for this walk: report, never guess
                atomicOr(b.err, ERR_SCRATCH_OVERFLOW);
                rec->state = CAND_REJECT;
            } else {
                rec->y = y; rec->x = x; rec->mass = m;
                rec->ul = ul; rec->vl = vl; rec->up = up; rec->vp = vp;
                rec->state = (m > p.minmass && m != 0.f) ? CAND_EMIT : CAND_REJECT;
            }
        }
    }
}

}  // namespace gt
