// finalize.cu -- per-frame ordering, separation filter and particle tables.
//
// Replaces the host-side raster scan (execute_gpu.rs:157-183) and the
// kd-tree separation filter (execute_gpu.rs:258-284).  One CTA per frame:
//   1. exclusive scan of the per-(row, tile column) record counts gives every
//      record its raster position (the reference's pre-filter `idx`);
//   2. records waiting on nothing (state EMIT) are compacted in raster order;
//   3. a uniform grid (cell >= separation + 1) bins them, and a point is
//      dropped if a neighbour closer than `separation` has a larger mass, or
//      an equal mass and a smaller raster index (single pass, as the
//      reference);
//   4. survivors form the frame's particle table in raster order, and a
//      second grid over them serves the linker's candidate search.
#include "gt_device.cuh"

namespace gt {

namespace {
constexpr int NTF = 512;

// In-place exclusive scan of n ints (any memory space), thread-chunked.
__device__ int block_scan_inplace(int* data, int n, int* warp_tot, int* s_total) {
    const int chunk = (n + NTF - 1) / NTF;
    const int q0 = threadIdx.x * chunk, q1 = min(q0 + chunk, n);
    int mine = 0;
    for (int q = q0; q < q1; ++q) mine += data[q];
    int pos = block_excl_scan<NTF>(mine, warp_tot, s_total);
    for (int q = q0; q < q1; ++q) { int v = data[q]; data[q] = pos; pos += v; }
    __syncthreads();
    return *s_total;
}

__device__ __forceinline__ int cell_of(float y, float x, float G, int ncy, int ncx) {
    int cy = (int)floorf(y / G), cx = (int)floorf(x / G);
    cy = clampi(cy, 0, ncy - 1);
    cx = clampi(cx, 0, ncx - 1);
    return cy * ncx + cx;
}

// Counting sort of n points into cells: start[ncell+1], idx[n].
__device__ void build_grid(const float* ys, const float* xs, const int* sel, int n, float G,
                           int ncy, int ncx, int* cnt_s, int* start, int* idx, int* warp_tot,
                           int* s_total) {
    const int ncell = ncy * ncx;
    for (int c = threadIdx.x; c < ncell; c += NTF) cnt_s[c] = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += NTF) {
        const int j = sel ? sel[i] : i;
        atomicAdd(&cnt_s[cell_of(ys[j], xs[j], G, ncy, ncx)], 1);
    }
    __syncthreads();
    block_scan_inplace(cnt_s, ncell, warp_tot, s_total);
    for (int c = threadIdx.x; c < ncell; c += NTF) start[c] = cnt_s[c];
    if (threadIdx.x == 0) start[ncell] = n;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += NTF) {
        const int j = sel ? sel[i] : i;
        const int k = atomicAdd(&cnt_s[cell_of(ys[j], xs[j], G, ncy, ncx)], 1);
        idx[k] = i;
    }
    __syncthreads();
}

// kd-tree 0.4.2 within_radius restated from its twin in linking.rs:73-105:
// per-axis box test, then (item - query)^2 summed from zero, strictly < r^2.
__device__ __forceinline__ bool within_r(float qy, float qx, float iy, float ix, float r, float* dist) {
    if (iy < qy - r || iy > qy + r) return false;
    if (ix < qx - r || ix > qx + r) return false;
    const float dy = iy - qy, dx = ix - qx;
    float dd = 0.f;
    dd = dd + dy * dy;
    dd = dd + dx * dx;
    *dist = dd;
    return dd < r * r;
}
}  // namespace

__global__ void __launch_bounds__(NTF) finalize_kernel(const LocParams p, MovieBufs b, float sep,
                                                       int link_grid, int frame0) {
    __shared__ int warp_tot[NTF / 32];
    __shared__ int s_total;
    extern __shared__ int cnt_s[];  // ncell ints (<= MAX_CELLS)
    const int t = frame0 + blockIdx.x;
    const int cap_c = b.cap_c;
    const int nrc = p.H * p.ntx;
    int* rc = b.rowcnt + (size_t)t * nrc;
    const Cand* cand = b.cand + (size_t)t * cap_c;
    int* perm = b.cperm + (size_t)t * cap_c;
    float* cy = b.cy + (size_t)t * cap_c;
    float* cx = b.cx + (size_t)t * cap_c;
    float* cm = b.cm + (size_t)t * cap_c;
    int* crec = b.crec + (size_t)t * cap_c;
    int* keep = b.ccell + (size_t)t * cap_c;

    const int nrec = b.fcount[t];
    if (nrec > cap_c) {
        // the locate kernel flagged the overflow and left slots unwritten;
        // the host retries with larger slabs
        if (threadIdx.x == 0) b.npart[t] = 0;
        if (link_grid) {  // empty particle grid keeps the linker in bounds
            const int ncell = b.ncx * b.ncy;
            int* gs = b.gstart + (size_t)t * (ncell + 1);
            for (int c = threadIdx.x; c <= ncell; c += NTF) gs[c] = 0;
        }
        return;
    }

    // 1. raster positions
    block_scan_inplace(rc, nrc, warp_tot, &s_total);
    for (int k = threadIdx.x; k < nrec; k += NTF) perm[k] = k;
    __syncthreads();
    for (int k = threadIdx.x; k < nrec; k += NTF) {
        const Cand& c = cand[k];
        if (c.u < 0 || c.u >= p.H || c.v < 0 || c.v >= p.W) continue;
        const int dest = rc[c.u * p.ntx + c.v / p.TW] + c.rowrank;
        if (dest >= 0 && dest < nrec) perm[dest] = k;
    }
    __syncthreads();

    // 2. compact emitted records in raster order
    for (int i = threadIdx.x; i < nrec; i += NTF) keep[i] = cand[perm[i]].state == CAND_EMIT ? 1 : 0;
    __syncthreads();
    const int ne = block_scan_inplace(keep, nrec, warp_tot, &s_total);
    for (int i = threadIdx.x; i < nrec; i += NTF) {
        const int k = perm[i];
        const Cand& c = cand[k];
        if (c.state != CAND_EMIT) continue;
        const int e = keep[i];
        cy[e] = c.y; cx[e] = c.x; cm[e] = c.mass; crec[e] = k;
    }
    __syncthreads();

    // 3. separation filter on a uniform grid
    const float G = (float)b.G;
    const int ncell = b.ncx * b.ncy;
    int* cstart = b.cstart + (size_t)t * (ncell + 1);
    int* cidx = b.cidx + (size_t)t * cap_c;
    build_grid(cy, cx, nullptr, ne, G, b.ncy, b.ncx, cnt_s, cstart, cidx, warp_tot, &s_total);
    for (int i = threadIdx.x; i < ne; i += NTF) {
        const float qy = cy[i], qx = cx[i], qm = cm[i];
        const int c = cell_of(qy, qx, G, b.ncy, b.ncx);
        const int gy = c / b.ncx, gx = c - gy * b.ncx;
        bool k = true;
        for (int dy = -1; dy <= 1 && k; ++dy) {
            const int yy = gy + dy;
            if (yy < 0 || yy >= b.ncy) continue;
            for (int dx = -1; dx <= 1 && k; ++dx) {
                const int xx = gx + dx;
                if (xx < 0 || xx >= b.ncx) continue;
                const int cc = yy * b.ncx + xx;
                for (int s = cstart[cc]; s < cstart[cc + 1]; ++s) {
                    const int j = cidx[s];
                    if (j == i) continue;
                    float dd;
                    if (!within_r(qy, qx, cy[j], cx[j], sep, &dd)) continue;
                    const float nm = cm[j];
                    if (qm < nm || (qm == nm && i > j)) { k = false; break; }
                }
            }
        }
        keep[i] = k ? 1 : 0;
    }
    __syncthreads();

    // 4. survivors in raster order
    const int np = block_scan_inplace(keep, ne, warp_tot, &s_total);
    const bool over = np > b.cap_p;
    if (over && threadIdx.x == 0) atomicOr(b.err, ERR_PART_OVERFLOW);
    float* py = b.py + (size_t)t * b.cap_p;
    float* px = b.px + (size_t)t * b.cap_p;
    float* pm = b.pm + (size_t)t * b.cap_p;
    int* prec = b.prec + (size_t)t * b.cap_p;
    // keep[i] now holds the survivor index; recompute survivorship from the
    // scan (a survivor is where the next prefix value increases)
    for (int i = threadIdx.x; i < ne; i += NTF) {
        const int a = keep[i];
        const int nxt = (i + 1 < ne) ? keep[i + 1] : np;
        if (nxt > a && a < b.cap_p) {
            py[a] = cy[i]; px[a] = cx[i]; pm[a] = cm[i]; prec[a] = crec[i];
        }
    }
    if (threadIdx.x == 0) b.npart[t] = over ? b.cap_p : np;
    __syncthreads();

    // 5. grid over the particles for the linker
    if (link_grid) {
        const int n = over ? b.cap_p : np;
        build_grid(py, px, nullptr, n, G, b.ncy, b.ncx, cnt_s, b.gstart + (size_t)t * (ncell + 1),
                   b.gidx + (size_t)t * b.cap_p, warp_tot, &s_total);
    }
}

// Grid over externally supplied particle tables (standalone linking).
__global__ void __launch_bounds__(NTF) grid_kernel(const float* py, const float* px, const int* npart,
                                                   int cap_p, int G, int ncy, int ncx, int* gstart,
                                                   int* gidx) {
    __shared__ int warp_tot[NTF / 32];
    __shared__ int s_total;
    extern __shared__ int cnt_s[];
    const int t = blockIdx.x;
    const int ncell = ncx * ncy;
    build_grid(py + (size_t)t * cap_p, px + (size_t)t * cap_p, nullptr, npart[t], (float)G, ncy, ncx, cnt_s,
               gstart + (size_t)t * (ncell + 1), gidx + (size_t)t * cap_p, warp_tot, &s_total);
}

}  // namespace gt
