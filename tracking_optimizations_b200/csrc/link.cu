// link.cu -- frame-to-frame linking on the device.
//
// Restates the reference linker (gpu-tracking/src/linking.rs:197-492):
// candidate pairs closer than search_range (strict, squared distance),
// connected components of the bipartite source/destination graph discovered
// from each destination in index order, 1-1 components linked directly, and
// every other component resolved by the reference's exhaustive
// branch-and-bound (recurse2, linking.rs:390-452) with the same f32 score
// arithmetic, option order (sources ascending, null last) and tie rule.
//
// Parallel structure.  Frame t's assignment depends only on the positions of
// frames t-1 and t and on the memory entries M(t) (unlinked particles of the
// previous `memory` frames, deduplicated by trajectory).  All frames are
// linked at once for a guessed M; M is then recomputed from the result, and
// only frames whose M changed are linked again, until M is a fixed point.
// M(t) depends on frames < t only, so iteration k settles frame k at the
// latest and the fixed point is the sequential result.
#include <cooperative_groups.h>

#include "gt_device.cuh"

namespace cg = cooperative_groups;

namespace gt {



namespace {
constexpr int NTL = 256;   // threads of a linker block for small frames
constexpr int NTL_BIG = 1024;  // for large frames: one block per SM, 32 warps per frame

__device__ __forceinline__ bool within_r(float qy, float qx, float iy, float ix, float r, float* dist) {
    // kd-tree box pre-filter + linking.rs:91-100 distance (dest - source)
    if (iy < qy - r || iy > qy + r) return false;
    if (ix < qx - r || ix > qx + r) return false;
    const float dy = iy - qy, dx = ix - qx;
    float dd = 0.f;
    dd = dd + dy * dy;
    dd = dd + dx * dx;
    *dist = dd;
    return dd < r * r;
}

__device__ __forceinline__ int cell_of(float y, float x, float G, int ncy, int ncx) {
    int cy = (int)floorf(y / G), cx = (int)floorf(x / G);
    cy = clampi(cy, 0, ncy - 1);
    cx = clampi(cx, 0, ncx - 1);
    return cy * ncx + cx;
}

__device__ int uf_find(int* uf, int x) {
    while (true) {
        int p = uf[x];
        if (p == x) return x;
        int gp = uf[p];
        if (gp != p) atomicCAS(&uf[x], p, gp);  // path halving
        x = p;
    }
}

__device__ void uf_union(int* uf, int a, int b) {
    while (true) {
        a = uf_find(uf, a);
        b = uf_find(uf, b);
        if (a == b) return;
        if (a < b) { int t = a; a = b; b = t; }
        if (atomicCAS(&uf[a], a, b) == a) return;
    }
}

template <int NT>
__device__ int block_scan_inplace_l(int* data, int n, int* warp_tot, int* s_total) {
    const int chunk = (n + NT - 1) / NT;
    const int q0 = threadIdx.x * chunk, q1 = min(q0 + chunk, n);
    int mine = 0;
    for (int q = q0; q < q1; ++q) mine += data[q];
    int pos = block_excl_scan<NT>(mine, warp_tot, s_total);
    for (int q = q0; q < q1; ++q) { int v = data[q]; data[q] = pos; pos += v; }
    __syncthreads();
    return *s_total;
}

// Exhaustive search of one subnet (linking.rs:390-452) by one thread.
// dests: destination indices in DFS order; sources are chosen through the
// per-destination lists d_src/d_w (ascending source index); null costs r^2.
// Returns false when the option-trial budget is exhausted.
__device__ bool solve_subnet(const LinkBufs& L, const int* dests, int nd, const int* d_off,
                             const int* d_src, const float* d_w, unsigned char* used, int* oi,
                             int* cur, int* best_choice, float null_cost) {
    float score = 0.f, best = CUDART_INF_F;
    long long trials = 0;
    int l = 0;
    oi[0] = 0;
    bool after_child = false;
    while (true) {
        const int d = dests[l];
        const int nopt = d_off[d + 1] - d_off[d] + 1;
        if (after_child) {
            // child returned: undo this level's option and advance
            const int o = oi[l];
            const float c = (o == nopt - 1) ? null_cost : d_w[d_off[d] + o];
            if (o != nopt - 1) used[d_src[d_off[d] + o]] = 0;
            score -= c;
            oi[l] = o + 1;
            after_child = false;
            continue;
        }
        const int o = oi[l];
        if (o >= nopt || score > best) {  // loop exhausted, or early return
            if (l == 0) break;
            --l;
            after_child = true;
            continue;
        }
        if (++trials > L.budget) {
            // give back the sources the open levels hold
            for (int q = 0; q < l; ++q)
                if (cur[q] >= 0) used[cur[q]] = 0;
            return false;
        }
        const bool is_null = (o == nopt - 1);
        const float c = is_null ? null_cost : d_w[d_off[d] + o];
        score += c;
        if (!is_null) {
            const int s = d_src[d_off[d] + o];
            if (used[s]) { score -= c; oi[l] = o + 1; continue; }
            used[s] = 1;
            cur[l] = s;
        } else {
            cur[l] = -1;
        }
        if (l == nd - 1) {
            if (score < best) {
                best = score;
                for (int q = 0; q < nd; ++q) best_choice[q] = cur[q];
            }
            if (!is_null) used[cur[l]] = 0;
            score -= c;
            oi[l] = o + 1;
        } else {
            ++l;
            oi[l] = 0;
        }
    }
    return true;
}
}  // namespace

// One CTA per frame (grid-stride); frame t >= 1 links P(t-1) + M(t) to P(t).
template <int NT>
// only_dirty: 0 = every frame, else the dirty bit of the pass (frames whose
// memory entries that pass changed).
__device__ void link_frames_body(const LinkBufs& L, int only_dirty, int t0, int tstride) {
    __shared__ int warp_tot[NT / 32];
    __shared__ int s_total;
    __shared__ int s_bump;
    extern __shared__ __align__(16) int lsm[];  // per-frame scratch pool
    const int slot = blockIdx.x;
    const int cap_p = L.cap_p;
    const float r = L.r;
    const float G = (float)L.G;
    const int ncell = L.ncx * L.ncy;
    const int pool = L.lsm_bytes / 4;

    for (int t = L.tb + t0; t < L.te; t += tstride) {
        if (only_dirty && !(__ldcg(L.dirty + t) & only_dirty)) continue;
        const int nd = L.npart[t];
        int* pred = L.pred + L.off[t];
        if (t == 0) {
            for (int i = threadIdx.x; i < nd; i += NT) pred[i] = -1;
            __syncthreads();
        } else {
            const int n1 = L.npart[t - 1];
            const int nm = __ldcg(L.mcount + t);
            const int ns = n1 + nm;
            const int nnode = ns + nd;
            // the frame's particles, grid and scratch live in shared memory
            // when they fit (latency), else in this block's global slot
            // the cell index is staged too when it fits beside the rest
            const int need_rest = 3 * nd + 4 * ns + 1 + nd + 1 + 8 * nnode + (nnode + 3) / 4;
            const bool sm = need_rest <= pool;
            const bool grid_sm = sm && need_rest + ncell + 1 <= pool;
            const int need = need_rest + (grid_sm ? ncell + 1 : 0);
            int* o = lsm;
            auto take = [&](int n) { int* q = o; o += n; return q; };
            const float* dy;
            const float* dx;
            const int* gs;
            const int* gi;
            float *sy, *sx;
            int *sh, *sdeg, *dcnt, *uf, *cnd, *cns, *cmin, *work;
            unsigned char* vis;
            if (sm) {
                float* ddy = (float*)take(nd);
                float* ddx = (float*)take(nd);
                int* ggi = take(nd);
                const float* py_t = L.py + (size_t)t * cap_p;
                const float* px_t = L.px + (size_t)t * cap_p;
                const int* gs_t = L.gstart + (size_t)t * (ncell + 1);
                const int* gi_t = L.gidx + (size_t)t * cap_p;
                for (int i = threadIdx.x; i < nd; i += NT) { ddy[i] = py_t[i]; ddx[i] = px_t[i]; ggi[i] = gi_t[i]; }
                if (grid_sm) {
                    int* ggs = take(ncell + 1);
                    for (int i = threadIdx.x; i <= ncell; i += NT) ggs[i] = gs_t[i];
                    gs = ggs;
                } else {
                    gs = gs_t;
                }
                dy = ddy; dx = ddx; gi = ggi;
                sy = (float*)take(ns); sx = (float*)take(ns); sh = take(ns); sdeg = take(ns + 1);
                dcnt = take(nd + 1);
                uf = take(nnode); cnd = take(nnode); cns = take(nnode); cmin = take(nnode);
                work = take(4 * nnode);
                vis = (unsigned char*)take((nnode + 3) / 4);
            } else {
                dy = L.py + (size_t)t * cap_p;
                dx = L.px + (size_t)t * cap_p;
                gs = L.gstart + (size_t)t * (ncell + 1);
                gi = L.gidx + (size_t)t * cap_p;
                sy = L.s_y + (size_t)slot * L.st_s;
                sx = L.s_x + (size_t)slot * L.st_s;
                sh = L.s_h + (size_t)slot * L.st_s;
                sdeg = L.s_deg + (size_t)slot * L.st_s1;
                dcnt = L.d_cnt + (size_t)slot * L.st_p1;
                uf = L.uf + (size_t)slot * L.st_n;
                cnd = L.c_nd + (size_t)slot * L.st_n;
                cns = L.c_ns + (size_t)slot * L.st_n;
                cmin = L.c_min + (size_t)slot * L.st_n;
                vis = L.vis + (size_t)slot * L.st_n;
                work = L.work + (size_t)slot * 4 * L.st_n;
            }
            int* bump = &s_bump;
            if (threadIdx.x == 0) *bump = 0;
            // sources: P(t-1) then M(t) (linking.rs:244-259 order)
            for (int s = threadIdx.x; s < ns; s += NT) {
                int h;
                if (s < n1) h = (t - 1) * cap_p + s;
                else h = __ldcg(L.mlist + (size_t)t * L.cap_m + (s - n1));
                sh[s] = h;
                sy[s] = L.py[h];
                sx[s] = L.px[h];
            }
            for (int s = threadIdx.x; s < n1; s += NT) L.lnext[(size_t)(t - 1) * cap_p + s] = 0;
            __syncthreads();
            // candidate pairs: degree pass
            for (int s = threadIdx.x; s < ns; s += NT) {
                const float qy = sy[s], qx = sx[s];
                const int c = cell_of(qy, qx, G, L.ncy, L.ncx);
                const int cy0 = c / L.ncx, cx0 = c - cy0 * L.ncx;
                int deg = 0;
                for (int ddy = -1; ddy <= 1; ++ddy) {
                    const int yy = cy0 + ddy;
                    if (yy < 0 || yy >= L.ncy) continue;
                    for (int ddx = -1; ddx <= 1; ++ddx) {
                        const int xx = cx0 + ddx;
                        if (xx < 0 || xx >= L.ncx) continue;
                        const int cc = yy * L.ncx + xx;
                        for (int k = gs[cc]; k < gs[cc + 1]; ++k) {
                            const int d = gi[k];
                            float dist;
                            if (within_r(qy, qx, dy[d], dx[d], r, &dist)) ++deg;
                        }
                    }
                }
                sdeg[s] = deg;
            }
            __syncthreads();
            const int ne = block_scan_inplace_l<NT>(sdeg, ns, warp_tot, &s_total);
            if (threadIdx.x == 0) sdeg[ns] = ne;
            int *edst, *dsrc;
            float *ew, *dw;
            if (sm && need + 4 * ne <= pool) {
                edst = take(ne); ew = (float*)take(ne); dsrc = take(ne); dw = (float*)take(ne);
            } else {
                edst = L.e_dst + (size_t)slot * L.st_e;
                ew = L.e_w + (size_t)slot * L.st_e;
                dsrc = L.d_src + (size_t)slot * L.st_e;
                dw = L.d_w + (size_t)slot * L.st_e;
            }
            if (ne > L.cap_e) {
                if (threadIdx.x == 0) atomicOr(L.err, ERR_EDGE_OVERFLOW);
                for (int i = threadIdx.x; i < nd; i += NT) pred[i] = -1;
                __syncthreads();
                continue;
            }
            for (int i = threadIdx.x; i <= nd; i += NT) dcnt[i] = 0;
            __syncthreads();
            // fill, then order each source's list by destination index
            for (int s = threadIdx.x; s < ns; s += NT) {
                const float qy = sy[s], qx = sx[s];
                const int c = cell_of(qy, qx, G, L.ncy, L.ncx);
                const int cy0 = c / L.ncx, cx0 = c - cy0 * L.ncx;
                int w = sdeg[s];
                const int w0 = w;
                for (int ddy = -1; ddy <= 1; ++ddy) {
                    const int yy = cy0 + ddy;
                    if (yy < 0 || yy >= L.ncy) continue;
                    for (int ddx = -1; ddx <= 1; ++ddx) {
                        const int xx = cx0 + ddx;
                        if (xx < 0 || xx >= L.ncx) continue;
                        const int cc = yy * L.ncx + xx;
                        for (int k = gs[cc]; k < gs[cc + 1]; ++k) {
                            const int d = gi[k];
                            float dist;
                            if (within_r(qy, qx, dy[d], dx[d], r, &dist)) {
                                int q = w++;
                                while (q > w0 && edst[q - 1] > d) { edst[q] = edst[q - 1]; ew[q] = ew[q - 1]; --q; }
                                edst[q] = d; ew[q] = dist;
                            }
                        }
                    }
                }
            }
            __syncthreads();
            // per-destination counts in a pass of their own: atomics inside
            // the neighbour search above stall it several-fold
            for (int q = threadIdx.x; q < ne; q += NT) atomicAdd(&dcnt[edst[q]], 1);
            __syncthreads();
            block_scan_inplace_l<NT>(dcnt, nd + 1, warp_tot, &s_total);
            // destination lists, ascending source index (linking.rs:310-315)
            int* dcur = cmin;  // reuse: cursors per destination
            for (int d = threadIdx.x; d < nd; d += NT) dcur[d] = dcnt[d];
            __syncthreads();
            for (int s = threadIdx.x; s < ns; s += NT) {
                for (int q = sdeg[s]; q < sdeg[s + 1]; ++q) {
                    const int d = edst[q];
                    const int k = atomicAdd(&dcur[d], 1);
                    dsrc[k] = s;
                    dw[k] = ew[q];
                }
            }
            __syncthreads();
            for (int d = threadIdx.x; d < nd; d += NT) {
                const int a = dcnt[d], e = dcnt[d + 1];
                for (int q = a + 1; q < e; ++q) {
                    const int ks = dsrc[q];
                    const float kw = dw[q];
                    int z = q;
                    while (z > a && dsrc[z - 1] > ks) { dsrc[z] = dsrc[z - 1]; dw[z] = dw[z - 1]; --z; }
                    dsrc[z] = ks; dw[z] = kw;
                }
            }
            // union-find over sources [0, ns) and destinations [ns, ns + nd)
            for (int i = threadIdx.x; i < nnode; i += NT) {
                uf[i] = i; cnd[i] = 0; cns[i] = 0; vis[i] = 0;
            }
            __syncthreads();
            for (int s = threadIdx.x; s < ns; s += NT)
                for (int q = sdeg[s]; q < sdeg[s + 1]; ++q) uf_union(uf, s, ns + edst[q]);
            __syncthreads();
            for (int i = threadIdx.x; i < nnode; i += NT) uf[i] = uf_find(uf, i);
            __syncthreads();
            for (int i = threadIdx.x; i < nnode; i += NT) cmin[i] = 0x7fffffff;
            __syncthreads();
            for (int s = threadIdx.x; s < ns; s += NT)
                if (sdeg[s + 1] > sdeg[s]) atomicAdd(&cns[uf[s]], 1);
            for (int d = threadIdx.x; d < nd; d += NT) {
                const int rt = uf[ns + d];
                atomicAdd(&cnd[rt], 1);
                atomicMin(&cmin[rt], d);
            }
            __syncthreads();
            // components, each resolved by the thread of its first destination
            const float null_cost = r * r;
            for (int d = threadIdx.x; d < nd; d += NT) {
                const int rt = uf[ns + d];
                if (cmin[rt] != d) continue;
                const int cd = cnd[rt], cs = cns[rt];
                if (cd == 1 && cs == 0) { pred[d] = -1; continue; }
                if (cd == 1 && cs == 1) {
                    const int s = dsrc[dcnt[d]];
                    const int h = sh[s];
                    pred[d] = L.off[h / cap_p] + (h % cap_p);
                    if (s < n1) L.lnext[(size_t)(t - 1) * cap_p + s] = 1;
                    continue;
                }
                // subnet: DFS preorder from d (linking.rs:316-342)
                const int sz = cd + cs;
                const int base = atomicAdd(bump, 4 * sz);
                int* stk_n = work + base;          // node ids (dest: ns + d)
                int* stk_p = stk_n + sz;           // next neighbour position
                int* path = stk_p + sz;            // destinations in DFS order
                int* choice = path + sz;           // per level: cur | best
                int top = 0, npath = 0;
                stk_n[0] = ns + d; stk_p[0] = 0; vis[ns + d] = 1; path[npath++] = d;
                top = 1;
                while (top > 0) {
                    const int node = stk_n[top - 1];
                    int pos = stk_p[top - 1];
                    int next = -1;
                    if (node >= ns) {
                        const int dd2 = node - ns;
                        if (dcnt[dd2] + pos < dcnt[dd2 + 1]) next = dsrc[dcnt[dd2] + pos];
                    } else {
                        if (sdeg[node] + pos < sdeg[node + 1]) next = ns + edst[sdeg[node] + pos];
                    }
                    if (next < 0) { --top; continue; }
                    stk_p[top - 1] = pos + 1;
                    if (vis[next]) continue;
                    vis[next] = 1;
                    if (next >= ns) path[npath++] = next - ns;
                    stk_n[top] = next; stk_p[top] = 0; ++top;
                }
                // branch and bound; `vis` bytes of sources double as `used`
                // flags: reset them first (all sources of the subnet were
                // visited above)
                for (int q = 0; q < npath; ++q) {
                    const int dd2 = path[q];
                    for (int z = dcnt[dd2]; z < dcnt[dd2 + 1]; ++z) vis[dsrc[z]] = 0;
                }
                int* oi = stk_n;                     // reuse the DFS stack
                int* cur = stk_p;
                int* bestc = choice;
                for (int q = 0; q < npath; ++q) bestc[q] = -1;
                const bool ok = solve_subnet(L, path, npath, dcnt, dsrc, dw, vis, oi, cur, bestc, null_cost);
                if (!ok) atomicOr(L.err, ERR_SUBNET_BUDGET);
                for (int q = 0; q < npath; ++q) {
                    const int s = bestc[q];
                    if (s < 0) { pred[path[q]] = -1; continue; }
                    const int h = sh[s];
                    pred[path[q]] = L.off[h / cap_p] + (h % cap_p);
                    if (s < n1) L.lnext[(size_t)(t - 1) * cap_p + s] = 1;
                }
            }
            __syncthreads();
        }
        // rank of each new particle within the frame (linking.rs:470)
        int* nr = L.newrank + L.off[t];
        const int chunk = (nd + NT - 1) / NT;
        const int q0 = threadIdx.x * chunk, q1 = min(q0 + chunk, nd);
        int mine = 0;
        for (int q = q0; q < q1; ++q) mine += (pred[q] < 0);
        int pos = block_excl_scan<NT>(mine, warp_tot, &s_total);
        for (int q = q0; q < q1; ++q) nr[q] = pred[q] < 0 ? pos++ : -1;
        if (threadIdx.x == 0) L.newcount[t] = s_total;
        __syncthreads();
    }
}

// Memory entries M(t) (linking.rs:244-259): particles of frames
// [t-1-memory, t-2] that the next frame did not link (the `unused` lists of
// linking.rs:479-485, oldest list first, index order within a list),
// skipping trajectories present in frame t-1 and keeping the first entry of
// each trajectory.  Marks frames whose M changed.
template <int NT>
__device__ void memory_body(const LinkBufs& L, int memory, int* ndirty, int wbit, int t0, int tstride) {
    __shared__ int warp_tot[NT / 32];
    __shared__ int s_total;
    __shared__ int s_diff;
    __shared__ int s_red;
    extern __shared__ __align__(16) int lsm[];
    const int slot = blockIdx.x;
    const int cap_p = L.cap_p;
    const int nn = L.cap_s + cap_p;
    const int pool = L.lsm_bytes / 4;
    for (int t = L.tb + t0; t < L.te; t += tstride) {
        const int fbeg = max(0, t - 1 - memory), fend = t - 2;
        if (fend < fbeg) continue;
        // number of candidates, to place the scratch
        if (threadIdx.x == 0) s_red = 0;
        __syncthreads();
        {
            int cnt = 0;
            for (int f = fbeg; f <= fend; ++f) {
                const int n = L.npart[f];
                const unsigned char* ln = L.lnext + (size_t)f * cap_p;
                for (int i = threadIdx.x; i < n; i += NT) cnt += __ldcg(ln + i) ? 0 : 1;
            }
            atomicAdd(&s_red, cnt);
        }
        __syncthreads();
        const int ncnt = s_red;
        const int n1 = L.npart[t - 1];
        int hs1 = 64;
        while (hs1 < 2 * n1) hs1 <<= 1;
        int hs2 = 64;
        while (hs2 < 2 * ncnt) hs2 <<= 1;
        int nmax = 0;
        for (int f = fbeg; f <= fend; ++f) nmax = max(nmax, L.npart[f]);
        const int cn = max(ncnt, nmax) + 1;
        const bool sm = 3 * cn + 2 * (hs1 + hs2) <= pool;
        int *ch, *cr, *cpos, *hk, *hv;
        int lim;
        if (sm) {
            ch = lsm; cr = ch + cn; cpos = cr + cn; hk = cpos + cn; hv = hk + hs1 + hs2;
            lim = cn;
        } else {
            ch = L.work + (size_t)slot * 4 * L.st_n;
            cr = ch + nn;
            cpos = cr + nn;
            hk = L.hkey + (size_t)slot * L.st_h;
            hv = L.hval + (size_t)slot * L.st_h;
            lim = nn;
        }
        // candidates in (frame, index) order
        int nc = 0;
        for (int f = fbeg; f <= fend; ++f) {
            const int n = L.npart[f];
            const unsigned char* ln = L.lnext + (size_t)f * cap_p;
            for (int i = threadIdx.x; i < n; i += NT) cpos[i] = __ldcg(ln + i) ? 0 : 1;
            __syncthreads();
            const int k = block_scan_inplace_l<NT>(cpos, n, warp_tot, &s_total);
            for (int i = threadIdx.x; i < n; i += NT) {
                if (__ldcg(ln + i)) continue;
                const int j = nc + cpos[i];
                if (j < lim) {
                    ch[j] = f * cap_p + i;
                    cr[j] = __ldcg(L.root + L.off[f] + i);
                }
            }
            nc += k;
            __syncthreads();
        }
        if (nc > lim) { if (threadIdx.x == 0) atomicOr(L.err, ERR_MEM_OVERFLOW); nc = lim; }
        if (!sm && hs1 + hs2 > L.hsize) { if (threadIdx.x == 0) atomicOr(L.err, ERR_SCRATCH_OVERFLOW); continue; }
        int* k1 = hk;
        int* k2 = hk + hs1;
        int* v2 = hv + hs1;
        for (int i = threadIdx.x; i < hs1 + hs2; i += NT) { hk[i] = -1; hv[i] = 0x7fffffff; }
        __syncthreads();
        // trajectories present in frame t-1
        for (int i = threadIdx.x; i < n1; i += NT) {
            const int key = __ldcg(L.root + L.off[t - 1] + i);
            unsigned hsh = ((unsigned)key * 2654435761u) & (hs1 - 1);
            while (true) {
                const int prev = atomicCAS(&k1[hsh], -1, key);
                if (prev == -1 || prev == key) break;
                hsh = (hsh + 1) & (hs1 - 1);
            }
        }
        // first candidate of each trajectory
        for (int j = threadIdx.x; j < nc; j += NT) {
            const int key = cr[j];
            unsigned hsh = ((unsigned)key * 2654435761u) & (hs2 - 1);
            while (true) {
                const int prev = atomicCAS(&k2[hsh], -1, key);
                if (prev == -1 || prev == key) break;
                hsh = (hsh + 1) & (hs2 - 1);
            }
            atomicMin(&v2[hsh], j);
        }
        __syncthreads();
        for (int j = threadIdx.x; j < nc; j += NT) {
            const int key = cr[j];
            bool keep = true;
            unsigned hsh = ((unsigned)key * 2654435761u) & (hs1 - 1);
            while (true) {
                const int kk = k1[hsh];
                if (kk == -1) break;
                if (kk == key) { keep = false; break; }
                hsh = (hsh + 1) & (hs1 - 1);
            }
            if (keep) {
                hsh = ((unsigned)key * 2654435761u) & (hs2 - 1);
                while (k2[hsh] != key) hsh = (hsh + 1) & (hs2 - 1);
                keep = v2[hsh] == j;
            }
            cpos[j] = keep ? 1 : 0;
        }
        if (threadIdx.x == 0) s_diff = 0;
        __syncthreads();
        const int nk = block_scan_inplace_l<NT>(cpos, nc, warp_tot, &s_total);
        int* ml = L.mlist + (size_t)t * L.cap_m;
        const int old = __ldcg(L.mcount + t);
        if (nk > L.cap_m) { if (threadIdx.x == 0) atomicOr(L.err, ERR_MEM_OVERFLOW); continue; }
        if (old != nk && threadIdx.x == 0) s_diff = 1;
        __syncthreads();
        for (int j = threadIdx.x; j < nc; j += NT) {
            const int a = cpos[j];
            const int nxt = (j + 1 < nc) ? cpos[j + 1] : nk;
            if (nxt > a && __ldcg(ml + a) != ch[j]) s_diff = 1;
        }
        __syncthreads();
        if (s_diff) {
            for (int j = threadIdx.x; j < nc; j += NT) {
                const int a = cpos[j];
                const int nxt = (j + 1 < nc) ? cpos[j + 1] : nk;
                if (nxt > a) ml[a] = ch[j];
            }
            if (threadIdx.x == 0) {
                L.mcount[t] = nk;
                atomicOr(L.dirty + t, wbit);
                atomicAdd(ndirty, 1);
            }
        } else if (threadIdx.x == 0) {
            atomicAnd(L.dirty + t, ~wbit);
        }
        __syncthreads();
    }
}

// Memory entries M(t) for memory 1 or 2, without trajectory roots.
//
// With at most two memory lists no trajectory branches: a particle left
// unused by the next frame is a memory candidate for the next two frames
// only, and once it is linked as a memory entry its trajectory id is
// present in the following frame, which excludes it there.  So, with ids
// unique within a frame (every source links at most one destination):
//   - a frame t-2 particle unused by frame t-1 never shares its id with a
//     frame t-1 particle (memory links into t-1 come from frames t-4 and
//     t-3) nor with a frame t-3 candidate (neither descends from the
//     other, and a common ancestor would be a branch);
//   - a frame t-3 particle unused by frame t-2 shares its id with a frame
//     t-1 particle exactly when that particle's pred is it (it was linked
//     into t-1 as a memory entry): it has no descendant in t-2.
// linking.rs:244-259 (unused lists oldest first, index order within a
// list, dedupe by id against prev and among the entries) thus gives:
// M(t) = the frame t-3 particles unused by t-2 and not the pred of a
// frame t-1 particle, then the frame t-2 particles unused by t-1 (memory 1:
// the latter only).  Marks frames whose M changed.
// M(t) reads lnext of frames t-3 and t-2 and pred of frame t-1, which only
// relinking frames t-2 and t-1 writes (lnext of a frame is written by the
// link into the next frame), so from the second pass on (k > 1) a frame
// whose frames t-1 and t-2 (memory 1: t-1) the previous pass did not relink
// keeps its M.  Pass k marks with wbit = 1 << (k & 1) and reads the previous
// pass's bit, so that concurrent marks never touch the bit being read.
template <int NT>
__device__ void memory_body_short(const LinkBufs& L, int memory, int* ndirty, int k, int t0, int tstride) {
    __shared__ int warp_tot[NT / 32];
    __shared__ int s_total;
    __shared__ int s_diff;
    extern __shared__ __align__(16) int lsm[];
    const int slot = blockIdx.x;
    const int cap_p = L.cap_p;
    const int pool = L.lsm_bytes / 4;
    const int wbit = 1 << (k & 1), pbit = 1 << ((k - 1) & 1);
    for (int t = L.tb + t0; t < L.te; t += tstride) {
        const int fbeg = max(0, t - 1 - memory), fend = t - 2;
        if (fend < fbeg) continue;
        if (k > 1 && !(__ldcg(L.dirty + t - 1) & pbit) && !(memory == 2 && (__ldcg(L.dirty + t - 2) & pbit))) {
            if (threadIdx.x == 0) atomicAnd(L.dirty + t, ~wbit);
            continue;
        }
        const int fo = (fend > fbeg) ? fbeg : -1;  // frame t-3 (memory 2)
        const int no = fo >= 0 ? L.npart[fo] : 0;
        const int nb = L.npart[fbeg], ne = L.npart[fend];
        const int nmax = max(nb, ne);
        const int ccap = nb + (fo >= 0 ? ne : 0);
        int *taken, *cpos, *ch;
        if (no + nmax + ccap + 1 <= pool) {
            taken = lsm; cpos = taken + no; ch = cpos + nmax;
        } else {
            int* w = L.work + (size_t)slot * 4 * L.st_n;
            taken = w; cpos = w + L.st_n; ch = w + 2 * L.st_n;
        }
        for (int i = threadIdx.x; i < no; i += NT) taken[i] = 0;
        if (threadIdx.x == 0) s_diff = 0;
        __syncthreads();
        if (fo >= 0) {
            const int o0 = L.off[fo], n1 = L.npart[t - 1];
            const int* pr = L.pred + L.off[t - 1];
            for (int x = threadIdx.x; x < n1; x += NT) {
                const int p = __ldcg(pr + x);
                if (p >= o0 && p < o0 + no) taken[p - o0] = 1;
            }
        }
        __syncthreads();
        int nc = 0;
        for (int f = fbeg; f <= fend; ++f) {
            const int n = L.npart[f];
            const unsigned char* ln = L.lnext + (size_t)f * cap_p;
            const bool old = f == fo;
            for (int i = threadIdx.x; i < n; i += NT) cpos[i] = (__ldcg(ln + i) || (old && taken[i])) ? 0 : 1;
            __syncthreads();
            const int k = block_scan_inplace_l<NT>(cpos, n, warp_tot, &s_total);
            for (int i = threadIdx.x; i < n; i += NT)
                if (!(__ldcg(ln + i) || (old && taken[i]))) ch[nc + cpos[i]] = f * cap_p + i;
            nc += k;
            __syncthreads();
        }
        int* ml = L.mlist + (size_t)t * L.cap_m;
        const int oldn = __ldcg(L.mcount + t);
        if (nc > L.cap_m) { if (threadIdx.x == 0) atomicOr(L.err, ERR_MEM_OVERFLOW); continue; }
        if (oldn != nc && threadIdx.x == 0) s_diff = 1;
        for (int j = threadIdx.x; j < nc; j += NT)
            if (__ldcg(ml + j) != ch[j]) s_diff = 1;
        __syncthreads();
        if (s_diff) {
            for (int j = threadIdx.x; j < nc; j += NT) ml[j] = ch[j];
            if (threadIdx.x == 0) {
                L.mcount[t] = nc;
                atomicOr(L.dirty + t, wbit);
                atomicAdd(ndirty, 1);
            }
        } else if (threadIdx.x == 0) {
            atomicAnd(L.dirty + t, ~wbit);
        }
        __syncthreads();
    }
}

// Trajectory roots (the first particle of each trajectory, compact index),
// in two levels.  Compact indices run in frame order and a pred always
// points to an earlier particle, so a chain only ever steps to smaller
// indices.  The window's particles are cut into about sqrt(frames) chunks
// of consecutive indices:
//   roots_local:  every particle walks its pred chain while it stays inside
//                 its own chunk (at most the chunk's frame count of hops)
//                 and records where the chain enters the chunk (lroot);
//                 root[] is cleared meanwhile;
//   roots_global: every particle steps from chunk to chunk through
//                 lroot(pred(entry)) until a trajectory start, a particle of
//                 an earlier (final) window, or a root another thread has
//                 written -- at most the chunk count of hops.
// root[] only ever receives final values, so no barrier is needed between
// hops; a chain costs O(sqrt(frames)) dependent loads instead of O(frames).
__device__ __forceinline__ int root_chunk(const LinkBufs& L) {
    const int n = L.off[L.te] - L.off[L.tb];
    int nc = 1;
    while (nc * nc < L.te - L.tb) ++nc;
    return max(1, (n + nc - 1) / nc);
}

__device__ void roots_local(const LinkBufs& L) {
    const int g0 = L.off[L.tb], n = L.off[L.te];
    const int cs = root_chunk(L);
    const int stride = gridDim.x * blockDim.x;
    for (int g = g0 + blockIdx.x * blockDim.x + threadIdx.x; g < n; g += stride) {
        const int cbeg = g0 + (g - g0) / cs * cs;
        int r = g;
        while (true) {
            const int p = __ldcg(L.pred + r);
            if (p < cbeg) break;
            r = p;
        }
        L.lroot[g] = r;
        L.root[g] = -1;
    }
}

__device__ void roots_global(const LinkBufs& L) {
    const int g0 = L.off[L.tb], n = L.off[L.te];
    const int stride = gridDim.x * blockDim.x;
    volatile int* root = L.root;
    for (int g = g0 + blockIdx.x * blockDim.x + threadIdx.x; g < n; g += stride) {
        int r = __ldcg(L.lroot + g);
        while (true) {
            const int known = root[r];
            if (known >= 0) { r = known; break; }
            const int p = __ldcg(L.pred + r);
            if (p < 0) break;
            if (p < g0) { r = root[p]; break; }  // earlier window: final
            r = __ldcg(L.lroot + p);
        }
        root[g] = r;
    }
}

__device__ void roots_body(const LinkBufs& L, cg::grid_group& grid) {
    roots_local(L);
    grid.sync();
    roots_global(L);
}

// The whole linker in one cooperative launch: link every frame with M = {},
// then alternate {trajectory roots, memory entries M(t), relink frames whose
// M changed} until no M changes (at most T + 1 passes).  ndirty[k] counts
// the frames changed by pass k (zeroed by the host).
namespace {
__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}
}  // namespace

// phase_ns: [0] first linking, [1] roots, [2] memory entries, [3] relinking
// (nanoseconds summed over passes, stamped by block 0 after each barrier).
// The memory entries of every frame are computed from one consistent state
// (a grid barrier before and after): a frame read while another block
// relinks its neighbour could see that neighbour's links half rewritten,
// which inflates the entries and the subnetworks they form.
template <int NT>
__global__ void __launch_bounds__(NT, NT == NTL ? 4 : 1) link_fixpoint_kernel(LinkBufs L, int memory, int max_passes, int rounds,
                                                               int* ndirty, int* passes,
                                                               unsigned long long* phase_ns) {
    cg::grid_group grid = cg::this_grid();
    const bool stamp = blockIdx.x == 0 && threadIdx.x == 0;
    unsigned long long t0 = stamp ? gtimer() : 0, acc[4] = {0, 0, 0, 0};
    link_frames_body<NT>(L, 0, blockIdx.x, gridDim.x);
    int k = 0;
    if (memory > 0 && L.te > 2) {
        // memory 1 or 2: the entries need no trajectory roots
        // (memory_body_short), so the roots are computed once, at the end
        const bool short_mem = memory <= 2;
        for (k = 1; k <= max_passes; ++k) {
            grid.sync();
            if (stamp) { const unsigned long long t = gtimer(); acc[k == 1 ? 0 : 3] += t - t0; t0 = t; }
            if (!short_mem) {
                roots_body(L, grid);
                grid.sync();
            }
            if (stamp) { const unsigned long long t = gtimer(); acc[1] += t - t0; t0 = t; }
            if (short_mem) memory_body_short<NT>(L, memory, ndirty + k, k, blockIdx.x, gridDim.x);
            else memory_body<NT>(L, memory, ndirty + k, 1 << (k & 1), blockIdx.x, gridDim.x);
            grid.sync();
            if (stamp) { const unsigned long long t = gtimer(); acc[2] += t - t0; t0 = t; }
            if (*(volatile int*)(ndirty + k) == 0) break;
            link_frames_body<NT>(L, 1 << (k & 1), blockIdx.x, gridDim.x);
        }
    }
    grid.sync();
    if (stamp) { const unsigned long long t = gtimer(); acc[k <= 1 ? 0 : 3] += t - t0; t0 = t; }
    roots_body(L, grid);
    grid.sync();  // so that the last stamp covers every block's walk
    if (stamp) {
        acc[1] += gtimer() - t0;
        *passes = max(*passes, k);  // several launches (frame windows) add up
        for (int i = 0; i < 4; ++i) phase_ns[i] += acc[i];
    }
    (void)rounds;
}

template __global__ void link_fixpoint_kernel<NTL>(LinkBufs, int, int, int, int*, int*, unsigned long long*);
template __global__ void link_fixpoint_kernel<NTL_BIG>(LinkBufs, int, int, int, int*, int*, unsigned long long*);

// Host side: the kernel for `nt` threads per block (256 or 1024), its
// resident blocks per SM, and a cooperative launch of it.
static const void* link_fixpoint_fn(int nt) {
    return nt == NTL_BIG ? (const void*)link_fixpoint_kernel<NTL_BIG> : (const void*)link_fixpoint_kernel<NTL>;
}

cudaError_t link_fixpoint_occupancy(int nt, int smem, int* per_sm) {
    cudaError_t e = cudaFuncSetAttribute(link_fixpoint_fn(nt), cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, link_fixpoint_fn(nt), nt, smem);
}

cudaError_t launch_link_fixpoint(int nt, int grid, void** args, int smem, cudaStream_t st) {
    return cudaLaunchCooperativeKernel(link_fixpoint_fn(nt), dim3(grid), dim3(nt), args, smem, st);
}

// Several movies in one cooperative launch (the batched path): every phase
// of link_fixpoint_kernel runs over the frames of all movies, movie m's
// frame t on block (fstart[m] + t) mod gridDim.x so that short movies spread
// over the grid; one grid barrier per phase serves all movies, and the
// fixed point ends when no movie's memory entries change.  Ls[m] share one
// per-block scratch pool (slot strides st_*), since a block links one frame
// at a time.
__global__ void __launch_bounds__(NTL, 4) link_fixpoint_multi_kernel(const LinkBufs* Ls, const int* memory,
                                                                     const int* fstart, int nm, int max_passes,
                                                                     int* ndirty, int* passes) {
    cg::grid_group grid = cg::this_grid();
    const int G = gridDim.x;
    auto t0_of = [&](int m) { const int s = fstart[m] % G; return ((int)blockIdx.x - s + G) % G; };
    bool any_mem = false;
    for (int m = 0; m < nm; ++m) {
        link_frames_body<NTL>(Ls[m], 0, t0_of(m), G);
        any_mem |= memory[m] > 0 && Ls[m].T > 2;
    }
    // ndirty[k * nm + m]: frames of movie m changed by pass k.  A movie
    // whose memory entries did not change in a pass is at its fixed point
    // (movies are independent): later passes skip it.
    auto active = [&](int m, int k) {
        return memory[m] > 0 && Ls[m].T > 2 && (k == 1 || *(volatile int*)(ndirty + (k - 1) * nm + m) > 0);
    };
    int k = 0;
    if (any_mem) {
        for (k = 1; k <= max_passes; ++k) {
            grid.sync();
            for (int m = 0; m < nm; ++m)
                if (active(m, k) && memory[m] > 2) roots_local(Ls[m]);
            grid.sync();
            for (int m = 0; m < nm; ++m)
                if (active(m, k) && memory[m] > 2) roots_global(Ls[m]);
            grid.sync();
            for (int m = 0; m < nm; ++m) {
                if (!active(m, k)) continue;
                if (memory[m] <= 2) memory_body_short<NTL>(Ls[m], memory[m], ndirty + k * nm + m, k, t0_of(m), G);
                else memory_body<NTL>(Ls[m], memory[m], ndirty + k * nm + m, 1 << (k & 1), t0_of(m), G);
            }
            grid.sync();
            int total = 0;
            for (int m = 0; m < nm; ++m) total += *(volatile int*)(ndirty + k * nm + m);
            if (total == 0) break;
            for (int m = 0; m < nm; ++m)
                if (*(volatile int*)(ndirty + k * nm + m) > 0) link_frames_body<NTL>(Ls[m], 1 << (k & 1), t0_of(m), G);
        }
    }
    grid.sync();
    for (int m = 0; m < nm; ++m) roots_local(Ls[m]);
    grid.sync();
    for (int m = 0; m < nm; ++m) roots_global(Ls[m]);
    if (blockIdx.x == 0 && threadIdx.x == 0) *passes = k;
}

}  // namespace gt
