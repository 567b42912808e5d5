// traj.cu -- trajectory post-processing of a linked table on the device:
// the lab pipeline's steps after linking (all_cleaned_up/
// hatzakis_lab_tracking.py:216-230): trackpy.filter_stubs, step_tracker
// (hatzakis_lab_tracking.py:53-83) and the per-particle mean squared
// displacement of trackpy.msd, concatenated as mp_imsd does
// (hatzakis_lab_tracking.py:199-214).
//
// Rows are grouped by particle with a stable order: keys (particle - min id)
// << 32 | row are radix-sorted, which gives exactly pandas' groupby order
// (ascending particle, rows of a particle in table order).
//
// MSD of one particle (trackpy.msd's definition): positions p = xy * mpp in
// float32, placed on the frame axis from the particle's first to its last
// frame (missing frames are gaps); for lag L = 1 .. min(max_lagtime,
// span - 1), <x^2>(L) is the mean of (x[f+L] - x[f])^2 over the pairs with
// both frames present (float32 differences and squares, summed in float64),
// likewise <y^2>, and msd = <x^2> + <y^2>.  A lag without a valid pair has
// no entry.
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include <algorithm>
#include <string>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "gt.h"

namespace gt {

namespace {

__global__ void id_range_kernel(const int64_t* ids, int64_t n, unsigned long long* lohi) {
    long long lo = LLONG_MAX, hi = LLONG_MIN;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const long long v = (long long)ids[i];
        lo = min(lo, v);
        hi = max(hi, v);
    }
    for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin((long long*)&lohi[0], lo);
        atomicMax((long long*)&lohi[1], hi);
    }
}

__global__ void group_keys_kernel(const int64_t* ids, int64_t n, long long idmin, unsigned long long* keys) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        keys[i] = ((unsigned long long)(ids[i] - idmin) << 32) | (unsigned long long)i;
}

__device__ __forceinline__ unsigned int gkey(unsigned long long k) { return (unsigned int)(k >> 32); }

// 1 where a sorted position starts a particle's group
__global__ void heads_kernel(const unsigned long long* keys, int64_t n, int64_t* heads) {
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x)
        heads[j] = (j == 0 || gkey(keys[j - 1]) != gkey(keys[j])) ? 1 : 0;
}

// gstart[g] = first sorted position of group g (groups in particle order)
__global__ void gstart_kernel(const unsigned long long* keys, int64_t n, const int64_t* gid, int64_t* gstart) {
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x)
        if (j == 0 || gkey(keys[j - 1]) != gkey(keys[j])) gstart[gid[j]] = j;
}

// keep[row] for every row of groups with at least `threshold` rows;
// count[row] = rows of the row's group
__global__ void stubs_kernel(const unsigned long long* keys, int64_t n, const int64_t* gstart, int64_t G,
                             int64_t threshold, uint8_t* keep, int64_t* count, unsigned long long* nkept) {
    unsigned long long mine = 0;
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < G; g += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = gstart[g], e = g + 1 < G ? gstart[g + 1] : n;
        const uint8_t k = (e - j) >= threshold ? 1 : 0;
        for (int64_t q = j; q < e; ++q) {
            keep[keys[q] & 0xffffffffu] = k;
            count[keys[q] & 0xffffffffu] = e - j;
        }
        if (k) mine += (unsigned long long)(e - j);
    }
    if (mine) atomicAdd(nkept, mine);
}
// step_tracker: scaled positions per row (float32), steps in group order
// (float64: the lab code takes the float32 values as Python floats)
__global__ void steps_kernel(const unsigned long long* keys, int64_t n, const float* x, const float* y, float mppf,
                             float* xs, float* ys, double* x_step, double* y_step, double* steplength,
                             int64_t* order) {
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = (int64_t)(keys[j] & 0xffffffffu);
        const float xr = __fmul_rn(x[r], mppf), yr = __fmul_rn(y[r], mppf);
        xs[r] = xr;
        ys[r] = yr;
        double dx = 0.0, dy = 0.0;
        if (j > 0 && gkey(keys[j - 1]) == gkey(keys[j])) {
            const int64_t rp = (int64_t)(keys[j - 1] & 0xffffffffu);
            dx = __dsub_rn((double)xr, (double)__fmul_rn(x[rp], mppf));
            dy = __dsub_rn((double)yr, (double)__fmul_rn(y[rp], mppf));
        }
        x_step[j] = dx;
        y_step[j] = dy;
        // np.sqrt(y**2 + x**2) (hatzakis_lab_tracking.py:76)
        steplength[j] = __dsqrt_rn(__dadd_rn(__dmul_rn(dy, dy), __dmul_rn(dx, dx)));
        order[j] = r;
    }
}

// per group: first frame, span and number of lags
__global__ void msd_groups_kernel(const unsigned long long* keys, int64_t n, const int64_t* frames,
                                  const int64_t* gstart, int64_t G, int64_t max_lagtime, int64_t* gfirst,
                                  int64_t* gspan, int64_t* glags, int* err) {
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < G; g += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = gstart[g], e = g + 1 < G ? gstart[g + 1] : n;
        int64_t fmin = LLONG_MAX, fmax = LLONG_MIN;
        for (int64_t q = j; q < e; ++q) {
            const int64_t f = frames[keys[q] & 0xffffffffu];
            fmin = min(fmin, f);
            fmax = max(fmax, f);
        }
        int64_t span = fmax - fmin + 1;
        if (span > ((int64_t)1 << 31) || span < 1) {
            atomicOr(err, 2);
            span = 1;
        }
        gfirst[g] = fmin;
        gspan[g] = span;
        glags[g] = min(max_lagtime, span - 1);
    }
}

// positions of the groups on their frame axes (NaN = gap); a frame taken
// twice by one particle is an error (trackpy: "more than one trajectory
// per particle")
__global__ void msd_scatter_kernel(const unsigned long long* keys, int64_t n, const int64_t* frames, const float* x,
                                   const float* y, float mppf, const int64_t* gstart, const int64_t* gfirst,
                                   const int64_t* gbase, int64_t ngroups, float2* pos, int* taken, int* err) {
    for (int64_t g = blockIdx.x; g < ngroups; g += gridDim.x) {
        const int64_t e = g + 1 < ngroups ? gstart[g + 1] : n;
        for (int64_t q = gstart[g] + threadIdx.x; q < e; q += blockDim.x) {
            const int64_t r = (int64_t)(keys[q] & 0xffffffffu);
            const int64_t s = gbase[g] + (frames[r] - gfirst[g]);
            if (atomicExch(taken + s, 1) != 0) atomicOr(err, 1);
            pos[s] = make_float2(__fmul_rn(x[r], mppf), __fmul_rn(y[r], mppf));
        }
    }
}

// one block per (group, chunk of MSD_LAGS lags), threads over the lags:
// the lags of a long-lived particle spread over several blocks
constexpr int MSD_LAGS = 128;
__global__ void msd_chunks_kernel(const int64_t* glags, int64_t ngroups, int64_t* gchunks) {
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < ngroups; g += (int64_t)gridDim.x * blockDim.x)
        gchunks[g] = (glags[g] + MSD_LAGS - 1) / MSD_LAGS;
}

__global__ void msd_kernel(const float2* pos, const int* taken, const int64_t* gbase, const int64_t* gspan,
                           const int64_t* glags, const int64_t* gout, const int64_t* cstart, int64_t ngroups,
                           int64_t nchunks, float* msd) {
    for (int64_t it = blockIdx.x; it < nchunks; it += gridDim.x) {
        // the group whose chunk range [cstart[g], cstart[g + 1]) holds it
        int64_t lo = 0, hi = ngroups - 1;
        while (lo < hi) {
            const int64_t mid = (lo + hi + 1) / 2;
            if (cstart[mid] <= it) lo = mid;
            else hi = mid - 1;
        }
        const int64_t g = lo;
        const float2* p = pos + gbase[g];
        const int* tk = taken + gbase[g];
        const int64_t span = gspan[g], nl = glags[g];
        const int64_t L0 = 1 + (it - cstart[g]) * MSD_LAGS;
        const int64_t L1 = min(nl, L0 + MSD_LAGS - 1);
        for (int64_t L = L0 + threadIdx.x; L <= L1; L += blockDim.x) {
            double sx = 0.0, sy = 0.0;
            int64_t cnt = 0;
            for (int64_t i = 0; i + L < span; ++i) {
                if (!tk[i] || !tk[i + L]) continue;
                const float2 a = p[i], b = p[i + L];
                const float dx = __fsub_rn(b.x, a.x), dy = __fsub_rn(b.y, a.y);
                sx += (double)__fmul_rn(dx, dx);
                sy += (double)__fmul_rn(dy, dy);
                ++cnt;
            }
            float v = CUDART_NAN_F;
            if (cnt > 0) v = __fadd_rn((float)(sx / (double)cnt), (float)(sy / (double)cnt));
            msd[gout[g] + L - 1] = v;
        }
    }
}

// (lag, particle) sort keys of the entries; entries without a pair last
__global__ void msd_keys_kernel(const float* msd, const int64_t* gout, const int64_t* glags,
                                const unsigned long long* keys, const int64_t* gstart, int64_t ngroups,
                                unsigned long long* ekeys, int64_t* eidx) {
    for (int64_t g = blockIdx.x; g < ngroups; g += gridDim.x) {
        const unsigned int pid = gkey(keys[gstart[g]]);
        for (int64_t L = 1 + threadIdx.x; L <= glags[g]; L += blockDim.x) {
            const int64_t e = gout[g] + L - 1;
            ekeys[e] = isnan(msd[e]) ? ~0ull : (((unsigned long long)L << 32) | pid);
            eidx[e] = e;
        }
    }
}

__global__ void msd_table_kernel(const unsigned long long* ekeys, const int64_t* eidx, const float* msd,
                                 int64_t nvalid, long long idmin, float* out) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nvalid; e += (int64_t)gridDim.x * blockDim.x) {
        const unsigned long long k = ekeys[e];
        out[3 * e + 0] = (float)(k >> 32);
        out[3 * e + 1] = (float)((long long)(k & 0xffffffffu) + idmin);
        out[3 * e + 2] = msd[eidx[e]];
    }
}

__global__ void count_valid_kernel(const unsigned long long* ekeys, int64_t ne, unsigned long long* nvalid) {
    unsigned long long mine = 0;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += (int64_t)gridDim.x * blockDim.x)
        mine += ekeys[e] != ~0ull;
    for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd(nvalid, mine);
}

int bits_for(unsigned long long v) {
    int b = 0;
    while (b < 64 && (v >> b)) ++b;
    return b;
}

// Stream-ordered device buffers, freed when the object goes out of scope.
struct DevBuf {
    cudaStream_t st;
    std::vector<void*> ptrs;
    explicit DevBuf(cudaStream_t s) : st(s) {}
    template <class X>
    X* get(size_t n) {
        void* p = nullptr;
        if (cudaMallocAsync(&p, sizeof(X) * (n ? n : 1), st) != cudaSuccess) return nullptr;
        ptrs.push_back(p);
        return (X*)p;
    }
    ~DevBuf() {
        for (void* p : ptrs) cudaFreeAsync(p, st);
    }
};

#define TK(x)                              \
    do {                                   \
        cudaError_t e_ = (x);              \
        if (e_ != cudaSuccess) {           \
            *msg = cudaGetErrorString(e_); \
            return GT_ERR_CUDA;            \
        }                                  \
    } while (0)
#define TA(p)                                  \
    do {                                       \
        if (!(p)) {                            \
            *msg = "device allocation failed"; \
            return GT_ERR_OOM;                 \
        }                                      \
    } while (0)

// Grouping of the rows by particle: the keys sorted in pandas' groupby
// order and the first sorted position of every group.
struct Groups {
    unsigned long long* keys = nullptr;
    int64_t* gstart = nullptr;
    int64_t G = 0;
    long long idmin = 0;
    unsigned long long range = 0;
};

int make_groups(const int64_t* h_ids, int64_t n, DevBuf& B, cudaStream_t st, int grid, Groups* out,
                std::string* msg) {
    int64_t* ids = B.get<int64_t>(n);
    unsigned long long* lohi = B.get<unsigned long long>(2);
    unsigned long long* k0 = B.get<unsigned long long>(n);
    unsigned long long* k1 = B.get<unsigned long long>(n);
    int64_t* heads = B.get<int64_t>(n);
    int64_t* gid = B.get<int64_t>(n);
    TA(ids && lohi && k0 && k1 && heads && gid);
    TK(cudaMemcpyAsync(ids, h_ids, sizeof(int64_t) * n, cudaMemcpyHostToDevice, st));
    const unsigned long long init[2] = {(unsigned long long)LLONG_MAX, (unsigned long long)LLONG_MIN};
    TK(cudaMemcpyAsync(lohi, init, sizeof(init), cudaMemcpyHostToDevice, st));
    id_range_kernel<<<grid, 256, 0, st>>>(ids, n, lohi);
    TK(cudaGetLastError());
    unsigned long long h[2];
    TK(cudaMemcpyAsync(h, lohi, sizeof(h), cudaMemcpyDeviceToHost, st));
    TK(cudaStreamSynchronize(st));
    out->idmin = (long long)h[0];
    const long long idmax = (long long)h[1];
    if (idmax - out->idmin >= (1LL << 31) || idmax < out->idmin) {
        *msg = "particle ids span more than 2^31 values";
        return GT_ERR_ARG;
    }
    out->range = (unsigned long long)(idmax - out->idmin);
    group_keys_kernel<<<grid, 256, 0, st>>>(ids, n, out->idmin, k0);
    TK(cudaGetLastError());
    const int end_bit = 32 + bits_for(out->range);
    cub::DoubleBuffer<unsigned long long> db(k0, k1);
    size_t tmp = 0, tmp2 = 0;
    TK(cub::DeviceRadixSort::SortKeys(nullptr, tmp, db, (int)n, 0, end_bit, st));
    TK(cub::DeviceScan::ExclusiveSum(nullptr, tmp2, heads, gid, (int)n, st));
    void* t = B.get<char>(std::max(tmp, tmp2));
    TA(t);
    TK(cub::DeviceRadixSort::SortKeys(t, tmp, db, (int)n, 0, end_bit, st));
    out->keys = db.Current();
    heads_kernel<<<grid, 256, 0, st>>>(out->keys, n, heads);
    TK(cudaGetLastError());
    TK(cub::DeviceScan::ExclusiveSum(t, tmp2, heads, gid, (int)n, st));
    int64_t last[2];
    TK(cudaMemcpyAsync(&last[0], gid + n - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    TK(cudaMemcpyAsync(&last[1], heads + n - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    TK(cudaStreamSynchronize(st));
    out->G = last[0] + last[1];
    out->gstart = B.get<int64_t>(out->G);
    TA(out->gstart);
    gstart_kernel<<<grid, 256, 0, st>>>(out->keys, n, gid, out->gstart);
    TK(cudaGetLastError());
    return GT_OK;
}

// exclusive prefix sum of v[0..G) into o, total returned in *tot
int exclusive_sum(const int64_t* v, int64_t* o, int64_t G, DevBuf& B, cudaStream_t st, int64_t* tot,
                  std::string* msg) {
    size_t tmp = 0;
    TK(cub::DeviceScan::ExclusiveSum(nullptr, tmp, v, o, (int)G, st));
    void* t = B.get<char>(tmp);
    TA(t);
    TK(cub::DeviceScan::ExclusiveSum(t, tmp, v, o, (int)G, st));
    int64_t a = 0, b = 0;
    TK(cudaMemcpyAsync(&a, o + G - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    TK(cudaMemcpyAsync(&b, v + G - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    TK(cudaStreamSynchronize(st));
    *tot = a + b;
    return GT_OK;
}

}  // namespace

int traj_filter_stubs(const int64_t* h_ids, int64_t n, int64_t threshold, uint8_t* h_keep, int64_t* h_count,
                      int64_t* nkept, cudaStream_t st, int num_sms, std::string* msg) {
    DevBuf B(st);
    const int grid = num_sms * 8;
    Groups Gr;
    int rc = make_groups(h_ids, n, B, st, grid, &Gr, msg);
    if (rc) return rc;
    uint8_t* keep = B.get<uint8_t>(n);
    int64_t* count = B.get<int64_t>(n);
    unsigned long long* cnt = B.get<unsigned long long>(1);
    TA(keep && count && cnt);
    TK(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), st));
    stubs_kernel<<<grid, 256, 0, st>>>(Gr.keys, n, Gr.gstart, Gr.G, threshold, keep, count, cnt);
    TK(cudaGetLastError());
    unsigned long long hk = 0;
    TK(cudaMemcpyAsync(h_keep, keep, n, cudaMemcpyDeviceToHost, st));
    if (h_count) TK(cudaMemcpyAsync(h_count, count, sizeof(int64_t) * n, cudaMemcpyDeviceToHost, st));
    TK(cudaMemcpyAsync(&hk, cnt, sizeof(hk), cudaMemcpyDeviceToHost, st));
    TK(cudaStreamSynchronize(st));
    *nkept = (int64_t)hk;
    return GT_OK;
}

int traj_steps(const int64_t* h_ids, const float* h_x, const float* h_y, int64_t n, float mppf, float* h_xs,
               float* h_ys, double* h_xstep, double* h_ystep, double* h_len, int64_t* h_order, cudaStream_t st,
               int num_sms, std::string* msg) {
    DevBuf B(st);
    const int grid = num_sms * 8;
    Groups Gr;
    int rc = make_groups(h_ids, n, B, st, grid, &Gr, msg);
    if (rc) return rc;
    float* x = B.get<float>(n);
    float* y = B.get<float>(n);
    float* sxy = B.get<float>(2 * (size_t)n);
    double* st3 = B.get<double>(3 * (size_t)n);
    int64_t* order = B.get<int64_t>(n);
    TA(x && y && sxy && st3 && order);
    TK(cudaMemcpyAsync(x, h_x, sizeof(float) * n, cudaMemcpyHostToDevice, st));
    TK(cudaMemcpyAsync(y, h_y, sizeof(float) * n, cudaMemcpyHostToDevice, st));
    steps_kernel<<<grid, 256, 0, st>>>(Gr.keys, n, x, y, mppf, sxy, sxy + n, st3, st3 + n, st3 + 2 * n, order);
    TK(cudaGetLastError());
    TK(cudaMemcpyAsync(h_xs, sxy, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
    TK(cudaMemcpyAsync(h_ys, sxy + n, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
    double* dst[3] = {h_xstep, h_ystep, h_len};
    for (int i = 0; i < 3; ++i)
        TK(cudaMemcpyAsync(dst[i], st3 + (size_t)i * n, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    TK(cudaMemcpyAsync(h_order, order, sizeof(int64_t) * n, cudaMemcpyDeviceToHost, st));
    TK(cudaStreamSynchronize(st));
    return GT_OK;
}

// Entries (lag, particle, msd) ordered by lag then particle, without the
// lags that have no valid pair; *out (3 floats per entry) comes from
// alloc(bytes).  *ms_msd: device time of the MSD kernel.
int traj_imsd(const int64_t* h_ids, const int64_t* h_frames, const float* h_x, const float* h_y, int64_t n,
              float mppf, int64_t max_lagtime, float* (*alloc)(size_t), float** out, int64_t* nout, float* ms_msd,
              cudaStream_t st, int num_sms, std::string* msg) {
    DevBuf B(st);
    const int grid = num_sms * 8;
    Groups Gr;
    int rc = make_groups(h_ids, n, B, st, grid, &Gr, msg);
    if (rc) return rc;
    if (Gr.idmin < 0 || Gr.idmin + (long long)Gr.range >= (1LL << 24)) {
        *msg = "particle ids must lie in [0, 2^24) for the float32 result table";
        return GT_ERR_ARG;
    }
    const int64_t G = Gr.G;
    int64_t* frames = B.get<int64_t>(n);
    float* x = B.get<float>(n);
    float* y = B.get<float>(n);
    int64_t* g5 = B.get<int64_t>(5 * (size_t)G);  // first, span, lags, base, out offset per group
    int* err = B.get<int>(1);
    TA(frames && x && y && g5 && err);
    int64_t *gfirst = g5, *gspan = g5 + G, *glags = g5 + 2 * G, *gbase = g5 + 3 * G, *gout = g5 + 4 * G;
    TK(cudaMemcpyAsync(frames, h_frames, sizeof(int64_t) * n, cudaMemcpyHostToDevice, st));
    TK(cudaMemcpyAsync(x, h_x, sizeof(float) * n, cudaMemcpyHostToDevice, st));
    TK(cudaMemcpyAsync(y, h_y, sizeof(float) * n, cudaMemcpyHostToDevice, st));
    TK(cudaMemsetAsync(err, 0, sizeof(int), st));
    if (max_lagtime < 0) max_lagtime = 0;
    msd_groups_kernel<<<grid, 256, 0, st>>>(Gr.keys, n, frames, Gr.gstart, G, max_lagtime, gfirst, gspan, glags, err);
    TK(cudaGetLastError());
    int64_t tot_span = 0, tot_out = 0;
    rc = exclusive_sum(gspan, gbase, G, B, st, &tot_span, msg);
    if (rc) return rc;
    rc = exclusive_sum(glags, gout, G, B, st, &tot_out, msg);
    if (rc) return rc;
    int h_err = 0;
    TK(cudaMemcpyAsync(&h_err, err, sizeof(h_err), cudaMemcpyDeviceToHost, st));
    TK(cudaStreamSynchronize(st));
    if (h_err) {
        *msg = "a particle spans more than 2^31 frames";
        return GT_ERR_ARG;
    }
    if (tot_span > ((int64_t)1 << 32) || tot_out >= ((int64_t)1 << 31)) {
        *msg = "trajectories span too many frames in total";
        return GT_ERR_ARG;
    }
    float2* pos = B.get<float2>(tot_span);
    int* taken = B.get<int>(tot_span);
    TA(pos && taken);
    TK(cudaMemsetAsync(taken, 0, sizeof(int) * tot_span, st));
    const int gg = (int)std::min<int64_t>(std::max<int64_t>(G, 1), (int64_t)num_sms * 64);
    msd_scatter_kernel<<<gg, 128, 0, st>>>(Gr.keys, n, frames, x, y, mppf, Gr.gstart, gfirst, gbase, G, pos, taken,
                                           err);
    TK(cudaGetLastError());
    TK(cudaMemcpyAsync(&h_err, err, sizeof(h_err), cudaMemcpyDeviceToHost, st));
    TK(cudaStreamSynchronize(st));
    if (h_err) {
        *msg = "more than one position for a particle in one frame (one trajectory per particle expected)";
        return GT_ERR_ARG;
    }
    int64_t nvalid = 0;
    *ms_msd = 0.f;
    float* tab = nullptr;
    if (tot_out > 0) {
        float* msd = B.get<float>(tot_out);
        unsigned long long* ekeys = B.get<unsigned long long>(tot_out);
        unsigned long long* ekeys2 = B.get<unsigned long long>(tot_out);
        int64_t* eidx = B.get<int64_t>(tot_out);
        int64_t* eidx2 = B.get<int64_t>(tot_out);
        unsigned long long* nv = B.get<unsigned long long>(1);
        TA(msd && ekeys && ekeys2 && eidx && eidx2 && nv);
        int64_t* gch = B.get<int64_t>(2 * (size_t)G);
        TA(gch);
        msd_chunks_kernel<<<grid, 256, 0, st>>>(glags, G, gch);
        TK(cudaGetLastError());
        int64_t nchunks = 0;
        rc = exclusive_sum(gch, gch + G, G, B, st, &nchunks, msg);
        if (rc) return rc;
        const int gc = (int)std::min<int64_t>(std::max<int64_t>(nchunks, 1), (int64_t)num_sms * 64);
        cudaEvent_t e0, e1;
        TK(cudaEventCreate(&e0));
        TK(cudaEventCreate(&e1));
        TK(cudaEventRecord(e0, st));
        msd_kernel<<<gc, MSD_LAGS, 0, st>>>(pos, taken, gbase, gspan, glags, gout, gch + G, G, nchunks, msd);
        TK(cudaEventRecord(e1, st));
        TK(cudaGetLastError());
        msd_keys_kernel<<<gg, 128, 0, st>>>(msd, gout, glags, Gr.keys, Gr.gstart, G, ekeys, eidx);
        TK(cudaGetLastError());
        cub::DoubleBuffer<unsigned long long> dk(ekeys, ekeys2);
        cub::DoubleBuffer<int64_t> dv(eidx, eidx2);
        size_t tmp = 0;
        TK(cub::DeviceRadixSort::SortPairs(nullptr, tmp, dk, dv, (int)tot_out, 0, 64, st));
        void* t = B.get<char>(tmp);
        TA(t);
        TK(cub::DeviceRadixSort::SortPairs(t, tmp, dk, dv, (int)tot_out, 0, 64, st));
        TK(cudaMemsetAsync(nv, 0, sizeof(unsigned long long), st));
        count_valid_kernel<<<grid, 256, 0, st>>>(dk.Current(), tot_out, nv);
        TK(cudaGetLastError());
        unsigned long long hv = 0;
        TK(cudaMemcpyAsync(&hv, nv, sizeof(hv), cudaMemcpyDeviceToHost, st));
        TK(cudaStreamSynchronize(st));
        cudaEventElapsedTime(ms_msd, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        nvalid = (int64_t)hv;
        tab = B.get<float>(3 * (size_t)std::max<int64_t>(nvalid, 1));
        TA(tab);
        if (nvalid > 0) {
            msd_table_kernel<<<grid, 256, 0, st>>>(dk.Current(), dv.Current(), msd, nvalid, Gr.idmin, tab);
            TK(cudaGetLastError());
        }
    }
    *out = alloc(sizeof(float) * 3 * (size_t)std::max<int64_t>(nvalid, 1));
    if (!*out) {
        *msg = "host allocation failed";
        return GT_ERR_OOM;
    }
    if (nvalid > 0) TK(cudaMemcpyAsync(*out, tab, sizeof(float) * 3 * (size_t)nvalid, cudaMemcpyDeviceToHost, st));
    TK(cudaStreamSynchronize(st));
    *nout = nvalid;
    return GT_OK;
}

}  // namespace gt
