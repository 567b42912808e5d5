// gt_api.cu -- host side of libgt: parameter derivation, workspace, launch
// sequence and the extern "C" entry points declared in include/gt.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <array>
#include <atomic>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <climits>
#include <cstring>
#include <string>
#include <vector>

#include <cuda.h>
#include <cudaTypedefs.h>

#include <map>

#include "gt.h"
#include "gt_internal.cuh"
#include "ingest.h"

namespace gt {
__global__ void locate_tiles_kernel(const LocParams p, const MovieBufs b, int frame0);
__global__ void fallback_walk_kernel(const LocParams p, const MovieBufs b, int win, const int* pbeg);
__global__ void finalize_kernel(const LocParams p, MovieBufs b, float sep, int link_grid, int frame0);
cudaError_t link_fixpoint_occupancy(int nt, int smem, int* per_sm);
cudaError_t launch_link_fixpoint(int nt, int grid, void** args, int smem, cudaStream_t st);
__global__ void scan_frames_kernel(const int* in, int* out, int n);
__global__ void scan_frames_from_kernel(const int* in, int* out, int f0, int n);
__global__ void newid_kernel(const int* newrank, const int* newbase, const int* off, const int* npart,
                             int* newid, int T);
__global__ void assemble_kernel(AsmArgs a);
__global__ void grid_kernel(const float* py, const float* px, const int* npart, int cap_p, int G,
                            int ncy, int ncx, int* gstart, int* gidx);
bool fast_supported(int kr, int dd, int rc, int diameter);
cudaError_t launch_locate_fast(int kr, int dd, int rc, int th, dim3 grid, cudaStream_t st, const LocParams& p,
                               const MovieBufs& b, int T, int frame0, int* used_tma);
void gauss_taps(int smoothing_size, float noise_size, int normalized, float* w, float* norm, float* rn);
cudaError_t launch_adjoint_particles(int mode, const AdjParams& p, const float* frames, const int* walk, long long n,
                                     const int* circ, const float* grad, float* yxm, float* gR, double* gpar,
                                     double* gpart, int* err, int num_sms, cudaStream_t st);
int adjoint_particle_blocks_max(int num_sms);
cudaError_t launch_adjoint_transpose(const AdjParams& p, const float* gR, float* gI, cudaStream_t st);
__global__ void link_fixpoint_multi_kernel(const LinkBufs* Ls, const int* memory, const int* fstart, int nm,
                                           int max_passes, int* ndirty, int* passes);
int traj_filter_stubs(const int64_t* h_ids, int64_t n, int64_t threshold, uint8_t* h_keep, int64_t* h_count,
                      int64_t* nkept, cudaStream_t st, int num_sms, std::string* msg);
int traj_steps(const int64_t* h_ids, const float* h_x, const float* h_y, int64_t n, float mppf, float* h_xs,
               float* h_ys, double* h_xstep, double* h_ystep, double* h_len, int64_t* h_order, cudaStream_t st,
               int num_sms, std::string* msg);
int traj_imsd(const int64_t* h_ids, const int64_t* h_frames, const float* h_x, const float* h_y, int64_t n,
              float mppf, int64_t max_lagtime, float* (*alloc)(size_t), float** out, int64_t* nout, float* ms_msd,
              cudaStream_t st, int num_sms, std::string* msg);

// preprocess_rows.wgsl:44-45: taps exp(-i^2 / (2 * noise_size)) for
// i = -k/2..k/2 and their running sum; the passes multiply by the
// reciprocal of that sum (a shader division).  With `normalized` the taps
// are divided by their sum on the host instead and the passes multiply by 1
// (kernels.rs:86-97 `gauss_1d` and `normalize`, the form in which the
// reference dumped its mass plane).
void gauss_taps(int smoothing_size, float noise_size, int normalized, float* w, float* norm, float* rn) {
    const int kr = smoothing_size / 2;
    float s = 0.0f;
    for (int i = -kr; i <= kr; ++i) {
        const float x = (float)i;
        const float g = std::exp(-x * x / (2.0f * noise_size));
        w[i + kr] = g;
        s = s + g;
    }
    *norm = s;
    if (normalized) {
        for (int i = 0; i < 2 * kr + 1; ++i) w[i] = w[i] / s;
        *rn = 1.0f;
    } else {
        *rn = 1.0f / s;
    }
}
}  // namespace gt

using namespace gt;

struct gt_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    char* arena = nullptr;
    size_t arena_size = 0;
    gt_stats stats{};
    int num_sms = 148;
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    int normalized_taps = 0;          // Gaussian taps divided by their sum on the host
    long long subnet_budget = 1LL << 26;  // option trials per linking subnetwork
    int withhold_tma = 0;             // test switch of the bounded tile-copy wait
    int force_generic = 0;            // always use locate_tiles_kernel
    int fast_tile_rows = 64;          // output tile height of the fast kernel (32 or 64)
    int tiles_per_cta = 0;            // fast kernel: tiles per CTA (0 = chosen per launch)
    // batched path (gt_batch_many_device)
    std::map<std::array<int, 6>, int> tile_rows;  // autotuned tile rows per (H, W, krad, D, rc, dtype)
    std::string batch_key;            // inputs of the cached graph
    cudaGraphExec_t batch_exec = nullptr;
    cudaStream_t side[8] = {};
    cudaEvent_t bev[20] = {};         // fork/join events
    int* h_status = nullptr;          // pinned: 8 ints per movie
    int* h_stage = nullptr;           // pinned: one call's statistics, read back in one go
    int link_per_sm = 0;              // resident link_fixpoint_kernel<256> blocks per SM (queried once)
    int link_per_sm_big = 0;          // the same for link_fixpoint_kernel<1024>
    size_t h_stage_n = 0;
    uint16_t* h_frames = nullptr;     // pinned: decoded file frames
    size_t h_frames_n = 0;
    size_t h_status_n = 0;
    int tune_disabled = 0;
    int batch_cap_div = 64;           // first candidate capacity of batched movies: H*W / this
    cudaStream_t copy_stream = nullptr;  // host->device frame chunks
    cudaEvent_t cev[9] = {};
};

namespace {

constexpr int LOC_TH = 32;
constexpr int LOC_TW = 64;
constexpr int LOC_CMAX = 512;
constexpr int FB_WIN_MAX = 100;
constexpr long long SUBNET_BUDGET = 1LL << 26;  // option trials per subnet
// shared-memory pool of a linker block: 4 blocks of 256 threads per SM, so
// that one round of blocks covers ~600 frames; frames whose data does not
// fit use the block's global scratch slot
constexpr int LINK_POOL_BYTES = 48 * 1024;
// frames of at least this many pixels are linked by 1024-thread blocks (one
// per SM, a larger shared-memory pool): their linking is latency-bound on
// global scratch, and 32 warps per frame hide four times more of it
constexpr long long LINK_BIG_PIXELS = 1LL << 20;
constexpr int LINK_POOL_BYTES_BIG = 160 * 1024;
constexpr int LINK_WINDOWS = 16;  // upload chunks of the host-frames path, at most

struct Resolved {
    // lib.rs:77-91 defaults
    uint32_t diameter;
    float minmass;
    uint32_t separation;
    float noise_size;
    uint32_t smoothing_size;
    uint32_t max_iterations;
    int characterize;
    int cpu_processed;
    int has_search_range;
    float search_range;
    uint32_t memory;
    int has_sig, has_bg;
    float sig_radius, bg_radius, gap_radius;
    int normalized_taps;  // context option, not a reference parameter
};

int resolve(const gt_params* p, Resolved* r, std::string* msg) {
    // lib.rs:73-74 not_implemented!(maxsize, threshold, invert, percentile, topn, preprocess)
    const char* ni = nullptr;
    if (p->has_maxsize) ni = "maxsize";
    else if (p->has_threshold) ni = "threshold";
    else if (p->has_invert) ni = "invert";
    else if (p->has_percentile) ni = "percentile";
    else if (p->has_topn) ni = "topn";
    else if (p->has_preprocess) ni = "preprocess";
    if (ni) { *msg = std::string(ni) + " is not implemented"; return GT_ERR_UNSUPPORTED; }
    r->diameter = p->diameter;
    r->minmass = p->has_minmass ? p->minmass : 0.0f;
    r->separation = p->has_separation ? p->separation : p->diameter + 1;
    r->noise_size = p->has_noise_size ? p->noise_size : 1.0f;
    r->smoothing_size = p->has_smoothing_size ? p->smoothing_size : p->diameter;
    r->max_iterations = p->has_max_iterations ? p->max_iterations : 10;
    r->characterize = p->has_characterize ? (p->characterize != 0) : 0;
    r->cpu_processed = p->has_cpu_processed ? (p->cpu_processed != 0) : 0;
    r->has_search_range = p->has_search_range;
    r->search_range = p->search_range;
    r->memory = p->has_memory ? p->memory : 0;  // Linker::new(range, memory.unwrap_or(0))
    r->has_sig = p->has_sig_radius;
    r->sig_radius = p->sig_radius;
    r->has_bg = p->has_bg_radius;
    r->bg_radius = p->bg_radius;
    r->gap_radius = p->has_gap_radius ? p->gap_radius : 0.0f;  // lib.rs:91
    r->normalized_taps = 0;
    if (r->has_bg && !r->has_sig) {
        // execute_gpu.rs:301-333 only gathers raw pixels when sig_radius is
        // set; the reference then fails reshaping its output.
        *msg = "bg_radius requires sig_radius";
        return GT_ERR_ARG;
    }
    if (r->smoothing_size < 1 || r->smoothing_size / 2 * 2 + 1 > GT_MAX_TAPS) {
        *msg = "smoothing_size must be in [1, 63]";
        return GT_ERR_ARG;
    }
    if (r->diameter > 63) { *msg = "diameter must be <= 63"; return GT_ERR_ARG; }
    if (r->separation > 4096) { *msg = "separation must be <= 4096"; return GT_ERR_ARG; }
    if (r->has_search_range && !(r->search_range > 0.0f && r->search_range < 4096.0f)) {
        *msg = "search_range must be in (0, 4096)";
        return GT_ERR_ARG;
    }
    if (r->memory > 1000) { *msg = "memory must be <= 1000"; return GT_ERR_ARG; }
    return GT_OK;
}

void column_list(const Resolved& r, std::vector<std::string>& names, std::vector<std::string>& types) {
    // execute_gpu.rs:197-226
    names = {"frame", "mass", "y", "x"};
    types = {"int", "float", "float", "float"};
    if (r.has_search_range) { names.push_back("particle"); types.push_back("int"); }
    if (r.cpu_processed) for (auto n : {"Rg", "ecc", "signal"}) { names.push_back(n); types.push_back("float"); }
    if (r.has_sig) { names.push_back("raw_mass"); types.push_back("float"); }
    if (r.has_bg) for (auto n : {"raw_bg_median", "raw_mass_corrected"}) { names.push_back(n); types.push_back("float"); }
    if (r.characterize)
        for (auto n : {"Rg_gpu", "raw_mass_gpu", "signal_gpu", "ecc_gpu"}) { names.push_back(n); types.push_back("float"); }
}

// gpu_setup.rs:48 dilation and max_rows.wgsl:17 offset
void dilation(uint32_t sep, int* D, int* o) {
    float v = (2.0f * (float)sep) / std::sqrt(2.0f);
    unsigned d = v <= 0.0f ? 0u : (unsigned)v;
    float half = (float)(int)d / 2.0f - 0.5f;
    *D = (int)d;
    *o = (int)half;
}

int next_pow2(long long x) {
    int p = 1;
    while (p < x) p <<= 1;
    return p;
}

struct Plan {
    int T = 0, H = 0, W = 0, dtype = 0;
    Resolved r{};
    LocParams lp{};
    float sep = 0.f;
    int link = 0;
    int cap_c = 0, cap_p = 0, cap_m = 0, cap_s = 0, cap_e = 0;
    int G = 8, ncx = 1, ncy = 1;
    int nslot = 1, hsize = 64;
    size_t smem_loc = 0, smem_fb = 0, smem_fin = 0;
    int fb_win = 0;
    int fast = 0;
    int fast_th = 32;
    std::vector<float> char_tab, gchar_tab;
    std::vector<int> char_off, sig_off, bg_off;
    std::vector<std::string> names, types;
};

void circle_tables(int R, std::vector<float>& tab, std::vector<int>* off, int stride3) {
    // kernels.rs:134-150, 169-206: i outer (row), j inner (column)
    for (int i = -R; i <= R; ++i)
        for (int j = -R; j <= R; ++j)
            if (i * i + j * j <= R * R) {
                float th = std::atan2((float)j, (float)i);
                if (stride3) tab.push_back((float)(i * i + j * j));
                tab.push_back(std::sin(2.0f * th));
                tab.push_back(std::cos(2.0f * th));
                if (off) { off->push_back(i); off->push_back(j); }
            }
}

void circle_inds_f(float radius, std::vector<int>& off) {
    // kernels.rs:134-150 with a float radius
    int rb = (int)std::ceil(radius);
    float r2 = radius * radius;
    for (int i = -rb; i <= rb; ++i)
        for (int j = -rb; j <= rb; ++j)
            if ((float)(i * i + j * j) <= r2) { off.push_back(i); off.push_back(j); }
}

void annulus_inds_f(float outer, float inner, std::vector<int>& off) {
    // kernels.rs:152-167
    int b = (int)std::ceil(outer);
    float or2 = outer * outer, ir2 = inner * inner;
    for (int i = -b; i <= b; ++i)
        for (int j = -b; j <= b; ++j) {
            float r2 = (float)(i * i + j * j);
            if (r2 <= or2 && r2 >= ir2) { off.push_back(i); off.push_back(j); }
        }
}

int make_plan(const Resolved& r, int T, int H, int W, int dtype, int scale, int num_sms, Plan* pl,
              std::string* msg, int force_generic_flag = 0, int fast_tile_rows = 32, int cap_div = 64) {
    Plan& P = *pl;
    P.T = T; P.H = H; P.W = W; P.dtype = dtype; P.r = r;
    LocParams& lp = P.lp;
    std::memset(&lp, 0, sizeof(lp));
    lp.H = H; lp.W = W;
    const int k = (int)r.smoothing_size;
    lp.krad = k / 2;
    lp.taps = 2 * lp.krad + 1;
    if (H <= lp.krad || W <= lp.krad) { *msg = "frame smaller than the smoothing window"; return GT_ERR_ARG; }
    gauss_taps(k, r.noise_size, r.normalized_taps, lp.w, &lp.norm, &lp.rn);
    lp.kk = (float)(k * k);
    lp.rkk = 1.0f / lp.kk;
    dilation(r.separation, &lp.D, &lp.o);
    lp.d = (int)r.diameter;
    lp.rint_c = ((int)r.diameter - 1) / 2;
    lp.border = (int)r.diameter / 2;
    lp.char_r = (int)r.diameter / 2;
    lp.max_iter = (int)r.max_iterations;
    lp.thr = 0.6f;  // gpu_setup.rs:57
    lp.minmass = r.minmass;
    lp.hp = std::max({lp.o, lp.D - 1 - lp.o, lp.char_r, lp.rint_c + 2, 1});
    lp.TH = LOC_TH; lp.TW = LOC_TW;
    lp.ntx = (W + lp.TW - 1) / lp.TW;
    lp.nty = (H + lp.TH - 1) / lp.TH;
    lp.dtype = dtype;
    lp.cpu_processed = r.cpu_processed;
    lp.characterize = r.characterize;
    lp.zero_skip = lp.max_iter >= 1 && lp.rint_c <= lp.o && lp.rint_c <= lp.D - 1 - lp.o;
    lp.tma_spin = 1 << 22;
    lp.tma_withhold = 0;
    P.fast = 0;
    const bool want_fast = dtype == GT_U16 && fast_supported(lp.krad, lp.D, lp.rint_c, lp.d) && !force_generic_flag;
    P.char_tab.clear(); P.char_off.clear(); P.gchar_tab.clear();
    circle_tables(lp.char_r, P.char_tab, &P.char_off, 1);
    circle_tables(lp.rint_c, P.gchar_tab, nullptr, 0);
    lp.n_char = (int)P.char_off.size() / 2;
    lp.n_gchar = (int)P.gchar_tab.size() / 2;
    if (want_fast) {
        P.fast = 1;
        P.fast_th = fast_tile_rows;
        lp.TH = fast_tile_rows;
        lp.TW = 64;
        lp.ntx = (W + lp.TW - 1) / lp.TW;
        lp.nty = (H + lp.TH - 1) / lp.TH;
    }
    P.sig_off.clear(); P.bg_off.clear();
    if (r.has_sig) circle_inds_f(r.sig_radius, P.sig_off);
    if (r.has_bg) annulus_inds_f(r.bg_radius, r.sig_radius + r.gap_radius, P.bg_off);
    P.sep = (float)r.separation;
    P.link = r.has_search_range;

    const int PH = LOC_TH + 2 * lp.hp, PW = LOC_TW + 2 * lp.hp;  // generic kernel plan
    const int RH = PH + 2 * lp.krad, RW = PW + 2 * lp.krad;
    P.smem_loc = sizeof(float) * ((size_t)RH * RW + 2 * (size_t)RH * PW + (size_t)PH * PW) +
                 sizeof(int) * (size_t)LOC_TH * LOC_TW + 6 * sizeof(float) * LOC_CMAX + (size_t)LOC_TH * LOC_TW;
    P.smem_loc = (P.smem_loc + 15) / 16 * 16;
    if (P.smem_loc > 227 * 1024) { *msg = "diameter/separation too large for the tile plan"; return GT_ERR_ARG; }
    P.fb_win = std::min(FB_WIN_MAX, std::max(lp.rint_c + 1, lp.max_iter - 1 + lp.rint_c + 1));
    P.smem_fb = sizeof(float) * (size_t)(2 * P.fb_win + 1) * (2 * P.fb_win + 1);

    // capacities (bounds; overflow is detected on the device and retried)
    const long long HW = (long long)H * W;
    long long cc = std::max<long long>(4096, HW / cap_div) * scale;
    P.cap_c = (int)std::min<long long>(cc, std::max<long long>(HW, 1));
    const double s = std::max(1.0f, P.sep);
    const double ext_h = H + 2.0 * lp.rint_c + s, ext_w = W + 2.0 * lp.rint_c + s;
    long long pack = (long long)(ext_h * ext_w / (0.785 * s * s)) + 16;
    P.cap_p = (int)std::min<long long>(P.cap_c, pack * scale);
    P.cap_m = (int)std::max<long long>(1, (long long)r.memory * P.cap_p);
    P.cap_s = P.cap_p + P.cap_m;
    const double sr = P.link ? r.search_range : 1.0;
    long long deg = (long long)((2 * sr + s) * (2 * sr + s) / (0.785 * s * s)) + 2;
    P.cap_e = (int)std::min<long long>((long long)P.cap_s * std::min<long long>(deg * scale, P.cap_p),
                                       (long long)1 << 30);
    P.G = std::max({(int)std::ceil(P.sep) + 1, P.link ? (int)std::ceil(r.search_range) + 1 : 0, 8,
                    (int)std::ceil(std::sqrt((double)HW / 16384.0))});
    P.ncy = (H + P.G - 1) / P.G;
    P.ncx = (W + P.G - 1) / P.G;
    P.smem_fin = sizeof(int) * (size_t)P.ncx * P.ncy;
    if (P.smem_fin > 200 * 1024) { *msg = "grid too fine"; return GT_ERR_ARG; }
    P.hsize = 2 * next_pow2(2LL * std::max({P.cap_p, P.cap_m, 32}));
    // link slots: bounded scratch
    const size_t nn = (size_t)P.cap_s + P.cap_p;
    const size_t per_slot = 4 * (3 * (size_t)P.cap_s + 1) + 8 * (size_t)P.cap_e * 2 + 4 * ((size_t)P.cap_p + 1) +
                            4 * 4 * nn + nn + 16 * nn + 4 + 8 * (size_t)P.hsize;
    const size_t budget = (size_t)6 << 30;
    P.nslot = (int)std::max<size_t>(1, std::min<size_t>({(size_t)T, (size_t)num_sms * 4, budget / per_slot}));
    column_list(r, P.names, P.types);
    return GT_OK;
}

// Device workspace carved from one arena.
struct Work {
    void* frames;
    Cand* cand;
    int *fcount, *rowcnt, *pend, *npend;
    float *py, *px, *pm;
    int *prec, *npart, *gstart, *gidx;
    int *cperm, *crec, *ccell, *cstart, *cidx;
    float *cy, *cx, *cm;
    float *char_tab, *gchar_tab;
    int *char_off, *sig_off, *bg_off;
    int* err;
    int *off, *pred, *mlist, *mcount, *dirty, *ndirty, *newrank, *newcount, *newbase, *root, *lroot, *newid;
    int* pbeg;  // fallback list position at the start of each chunk's locate
    unsigned long long* phase_ns;
    unsigned char* lnext;
    float *s_y, *s_x, *e_w, *d_w;
    int *s_h, *s_deg, *e_dst, *d_cnt, *d_src, *uf, *c_nd, *c_ns, *c_min, *work, *bump, *hkey, *hval;
    unsigned char* vis;
    float* out;
};

struct Carver {
    char* base;
    size_t off = 0;
    template <class X>
    X* take(size_t n) {
        off = (off + 255) / 256 * 256;
        X* p = (X*)(base ? base + off : nullptr);
        off += sizeof(X) * std::max<size_t>(n, 1);
        return p;
    }
};

size_t carve(const Plan& P, char* base, Work* w, size_t frame_bytes, bool need_locate, bool own_out = true) {
    Carver c{base};
    const size_t T = P.T;
    const size_t ncell = (size_t)P.ncx * P.ncy;
    w->frames = c.take<char>(frame_bytes);
    const size_t cc = need_locate ? T * P.cap_c : 1;
    w->cand = c.take<Cand>(cc);
    w->fcount = c.take<int>(T);
    w->rowcnt = c.take<int>(need_locate ? T * P.H * P.lp.ntx : 1);
    w->pend = c.take<int>(cc);
    w->npend = c.take<int>(1);
    w->py = c.take<float>(T * P.cap_p);
    w->px = c.take<float>(T * P.cap_p);
    w->pm = c.take<float>(T * P.cap_p);
    w->prec = c.take<int>(T * P.cap_p);
    w->npart = c.take<int>(T);
    w->gstart = c.take<int>(T * (ncell + 1));
    w->gidx = c.take<int>(T * P.cap_p);
    w->cperm = c.take<int>(cc);
    w->crec = c.take<int>(cc);
    w->ccell = c.take<int>(cc);
    w->cstart = c.take<int>(need_locate ? T * (ncell + 1) : 1);
    w->cidx = c.take<int>(cc);
    w->cy = c.take<float>(cc);
    w->cx = c.take<float>(cc);
    w->cm = c.take<float>(cc);
    w->char_tab = c.take<float>(P.char_tab.size());
    w->gchar_tab = c.take<float>(P.gchar_tab.size());
    w->char_off = c.take<int>(P.char_off.size());
    w->sig_off = c.take<int>(P.sig_off.size());
    w->bg_off = c.take<int>(P.bg_off.size());
    w->err = c.take<int>(4);
    w->off = c.take<int>(T + 1);
    const size_t np = P.link ? T * P.cap_p : 1;
    w->pred = c.take<int>(np);
    w->lnext = c.take<unsigned char>(np);
    w->mlist = c.take<int>(P.link ? T * P.cap_m : 1);
    w->mcount = c.take<int>(T);
    w->dirty = c.take<int>(T);
    w->ndirty = c.take<int>((T + 2) * LINK_WINDOWS);  // per linker launch (frame window)
    w->pbeg = c.take<int>(LINK_WINDOWS);
    w->phase_ns = c.take<unsigned long long>(4);
    w->newrank = c.take<int>(np);
    w->newcount = c.take<int>(T);
    w->newbase = c.take<int>(T + 1);
    w->root = c.take<int>(np);
    w->lroot = c.take<int>(P.link ? np : 1);
    w->newid = c.take<int>(np);
    const size_t S = P.link ? P.nslot : 0;
    const size_t nn = (size_t)P.cap_s + P.cap_p;
    w->s_y = c.take<float>(S * P.cap_s);
    w->s_x = c.take<float>(S * P.cap_s);
    w->s_h = c.take<int>(S * P.cap_s);
    w->s_deg = c.take<int>(S * (P.cap_s + 1));
    w->e_dst = c.take<int>(S * P.cap_e);
    w->e_w = c.take<float>(S * P.cap_e);
    w->d_cnt = c.take<int>(S * (P.cap_p + 1));
    w->d_src = c.take<int>(S * P.cap_e);
    w->d_w = c.take<float>(S * P.cap_e);
    w->uf = c.take<int>(S * nn);
    w->c_nd = c.take<int>(S * nn);
    w->c_ns = c.take<int>(S * nn);
    w->c_min = c.take<int>(S * nn);
    w->vis = c.take<unsigned char>(S * nn);
    w->work = c.take<int>(S * 4 * nn);
    w->bump = c.take<int>(S);
    w->hkey = c.take<int>(S * P.hsize);
    w->hval = c.take<int>(S * P.hsize);
    w->out = c.take<float>(need_locate && own_out ? T * P.cap_p * P.names.size() : 1);
    return c.off + 256;
}

#define CK(x)                                                                              \
    do {                                                                                   \
        cudaError_t e_ = (x);                                                              \
        if (e_ != cudaSuccess) {                                                           \
            ctx->err = std::string(#x) + ": " + cudaGetErrorString(e_);                    \
            return e_ == cudaErrorMemoryAllocation ? GT_ERR_OOM : GT_ERR_CUDA;             \
        }                                                                                  \
    } while (0)

int ensure_arena(gt_ctx* ctx, size_t bytes) {
    if (ctx->arena_size >= bytes) return GT_OK;
    if (ctx->arena) { cudaFree(ctx->arena); ctx->arena = nullptr; ctx->arena_size = 0; }
    size_t want = bytes + bytes / 8;
    CK(cudaMalloc((void**)&ctx->arena, want));
    ctx->arena_size = want;
    return GT_OK;
}

LinkBufs link_bufs(const Plan& P, const Work& w, long long budget) {
    LinkBufs L{};
    L.tb = 0;
    L.te = P.T;
    L.T = P.T; L.cap_p = P.cap_p; L.cap_m = P.cap_m; L.cap_e = P.cap_e; L.cap_s = P.cap_s;
    L.r = P.r.search_range;
    L.G = P.G; L.ncx = P.ncx; L.ncy = P.ncy;
    L.py = w.py; L.px = w.px; L.npart = w.npart; L.off = w.off; L.gstart = w.gstart; L.gidx = w.gidx;
    L.pred = w.pred; L.lnext = w.lnext; L.mlist = w.mlist; L.mcount = w.mcount; L.dirty = w.dirty;
    L.ndirty = w.ndirty; L.newrank = w.newrank; L.newcount = w.newcount; L.root = w.root; L.lroot = w.lroot; L.err = w.err;
    L.budget = budget;
    L.nslot = P.nslot;
    L.s_y = w.s_y; L.s_x = w.s_x; L.s_h = w.s_h; L.s_deg = w.s_deg; L.e_dst = w.e_dst; L.e_w = w.e_w;
    L.d_cnt = w.d_cnt; L.d_src = w.d_src; L.d_w = w.d_w; L.uf = w.uf; L.c_nd = w.c_nd; L.c_ns = w.c_ns;
    L.c_min = w.c_min; L.vis = w.vis; L.work = w.work; L.bump = w.bump; L.hkey = w.hkey; L.hval = w.hval;
    L.hsize = P.hsize;
    L.st_s = P.cap_s; L.st_s1 = (long long)P.cap_s + 1; L.st_p1 = (long long)P.cap_p + 1;
    L.st_n = (long long)P.cap_s + P.cap_p; L.st_e = P.cap_e; L.st_h = P.hsize;
    return L;
}

// Linking over the particle tables already in the workspace (npart, py, px,
// gstart/gidx, off): cooperative launches of link_fixpoint_kernel run the
// fixed point, then new trajectory ids are numbered.  Leaves the trajectory
// id of particle g in newid[root[g]].
//
// The linker in frame windows.  link_window links frames [tb, te) to their
// fixed point, given final links for the frames before tb: the memory
// entries of a frame depend only on earlier frames, so windows taken in
// order give the sequential result (the host-frames path links each
// uploaded chunk while the next one is copied).  link_prepare runs once
// before the first window, link_finish once after the last.
int link_prepare(gt_ctx* ctx, const Plan& P, const Work& w, cudaStream_t st) {
    const int T = P.T;
    CK(cudaMemsetAsync(w.mcount, 0, sizeof(int) * T, st));
    CK(cudaMemsetAsync(w.dirty, 0, sizeof(int) * T, st));
    CK(cudaMemsetAsync(w.ndirty, 0, sizeof(int) * (T + 2) * LINK_WINDOWS, st));
    CK(cudaMemsetAsync(w.phase_ns, 0, sizeof(unsigned long long) * 4, st));
    return GT_OK;
}

// Threads per linker block for frames of H x W pixels, its resident blocks
// per SM (queried once per context) and its shared-memory pool.
int link_shape(gt_ctx* ctx, long long px, int* nt, int* per_sm, int* pool) {
    const bool big = px >= LINK_BIG_PIXELS;
    *nt = big ? 1024 : 256;
    *pool = big ? LINK_POOL_BYTES_BIG : LINK_POOL_BYTES;
    int& cached = big ? ctx->link_per_sm_big : ctx->link_per_sm;
    if (!cached) {
        int q = 0;
        CK(link_fixpoint_occupancy(*nt, *pool, &q));
        cached = std::max(1, q);
    }
    *per_sm = cached;
    return GT_OK;
}

int link_window(gt_ctx* ctx, const Plan& P, const Work& w, cudaStream_t st, int tb, int te, int wi) {
    LinkBufs L = link_bufs(P, w, ctx->subnet_budget);
    L.tb = tb;
    L.te = te;
    const int T = P.T;
    int rounds = 0;
    int nt = 256, per_sm = 1, pool = LINK_POOL_BYTES;
    int rc = link_shape(ctx, (long long)P.H * P.W, &nt, &per_sm, &pool);
    if (rc) return rc;
    L.lsm_bytes = pool;
    const int grid = std::max(1, std::min(P.nslot, per_sm * ctx->num_sms));
    int memory = (int)P.r.memory;
    int max_passes = te - tb + 1;
    int* ndirty = w.ndirty + (size_t)wi * (T + 2);
    int* passes = w.err + 1;
    unsigned long long* phase_ns = w.phase_ns;
    void* args[] = {&L, &memory, &max_passes, &rounds, &ndirty, &passes, &phase_ns};
    CK(launch_link_fixpoint(nt, grid, args, pool, st));
    ctx->stats.launches += 1;
    return GT_OK;
}

int link_finish(gt_ctx* ctx, const Plan& P, const Work& w, cudaStream_t st) {
    const int T = P.T;
    scan_frames_kernel<<<1, 1024, 0, st>>>(w.newcount, w.newbase, T);
    newid_kernel<<<T, 256, 0, st>>>(w.newrank, w.newbase, w.off, w.npart, w.newid, T);
    CK(cudaGetLastError());
    ctx->stats.launches += 2;
    return GT_OK;
}

int run_link(gt_ctx* ctx, const Plan& P, const Work& w, cudaStream_t st) {
    int rc = link_prepare(ctx, P, w, st);
    if (!rc) rc = link_window(ctx, P, w, st, 0, P.T, 0);
    if (!rc) rc = link_finish(ctx, P, w, st);
    return rc;
}

int upload_tables(gt_ctx* ctx, const Plan& P, const Work& w, cudaStream_t st) {
    auto up = [&](void* dst, const void* src, size_t bytes) -> int {
        if (bytes) CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
        return GT_OK;
    };
    int rc;
    if ((rc = up(w.char_tab, P.char_tab.data(), sizeof(float) * P.char_tab.size()))) return rc;
    if ((rc = up(w.gchar_tab, P.gchar_tab.data(), sizeof(float) * P.gchar_tab.size()))) return rc;
    if ((rc = up(w.char_off, P.char_off.data(), sizeof(int) * P.char_off.size()))) return rc;
    if ((rc = up(w.sig_off, P.sig_off.data(), sizeof(int) * P.sig_off.size()))) return rc;
    if ((rc = up(w.bg_off, P.bg_off.data(), sizeof(int) * P.bg_off.size()))) return rc;
    return GT_OK;
}

MovieBufs movie_bufs(const Plan& P, const Work& w, const void* frames) {
    MovieBufs b{};
    b.frames = frames;
    b.T = P.T;
    b.cap_c = P.cap_c; b.cap_p = P.cap_p; b.cap_m = P.cap_m; b.cap_e = P.cap_e;
    b.cand = w.cand; b.fcount = w.fcount; b.rowcnt = w.rowcnt; b.pend = w.pend; b.npend = w.npend;
    b.py = w.py; b.px = w.px; b.pm = w.pm; b.prec = w.prec; b.npart = w.npart;
    b.G = P.G; b.ncx = P.ncx; b.ncy = P.ncy; b.gstart = w.gstart; b.gidx = w.gidx;
    b.cperm = w.cperm; b.cy = w.cy; b.cx = w.cx; b.cm = w.cm; b.crec = w.crec; b.ccell = w.ccell;
    b.cstart = w.cstart; b.cidx = w.cidx;
    b.char_tab = w.char_tab; b.char_off = w.char_off; b.gchar_tab = w.gchar_tab;
    b.err = w.err;
    return b;
}

// The whole locate(+link) pipeline on device frames; table left in w.out.
// With h_frames set, d_frames is the workspace copy of host frames: the
// copy runs in chunks of frames on the context's copy stream and each
// chunk's locate launch waits only for its own chunk, so host->device
// transfer and locate overlap.
int run_pipeline(gt_ctx* ctx, const Plan& P, const Work& w, const void* d_frames, cudaStream_t st,
                 int* err_bits, int64_t* nrows, int* d_walk = nullptr, int64_t walk_rows = 0,
                 const void* h_frames = nullptr, size_t elem = 0,
                 const std::function<int(int, int)>* ready = nullptr, float* d_out = nullptr,
                 int64_t out_rows = 0) {
    const int T = P.T;
    MovieBufs b = movie_bufs(P, w, d_frames);
    int rc = upload_tables(ctx, P, w, st);
    if (rc) return rc;
    CK(cudaMemsetAsync(w.fcount, 0, sizeof(int) * T, st));
    CK(cudaMemsetAsync(w.npend, 0, sizeof(int), st));
    CK(cudaMemsetAsync(w.err, 0, sizeof(int) * 4, st));
    CK(cudaFuncSetAttribute(locate_tiles_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P.smem_loc));
    for (int i = 0; i < 5; ++i)
        if (!ctx->ev[i]) CK(cudaEventCreate(&ctx->ev[i]));
    const int ntiles = P.lp.ntx * P.lp.nty;
    const bool fast = P.fast != 0;
    ctx->stats.locate_kernel = fast ? 1 : 0;
    // frame chunks: up to 16 for host frames (copy/locate overlap; the
    // locate of the last chunk is what remains after the copy), else as
    // large as the grid allows
    const int chunk = h_frames ? std::min(65535, std::max(16, (T + 15) / 16)) : 65535;
    const size_t fbytes = (size_t)P.H * P.W * elem;
    int ci = 0;
    auto stage = [&](int f0, int nf) -> int {
        if (!h_frames) return GT_OK;
        if (!ctx->copy_stream) CK(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
        for (auto& e : ctx->cev)
            if (!e) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        if (ci == 0) {
            CK(cudaEventRecord(ctx->cev[8], st));
            CK(cudaStreamWaitEvent(ctx->copy_stream, ctx->cev[8], 0));
        }
        if (ready) {
            // host frames still being produced (file decode): wait for these
            const int rr = (*ready)(f0, nf);
            if (rr) return rr;
        }
        CK(cudaMemcpyAsync((char*)d_frames + (size_t)f0 * fbytes, (const char*)h_frames + (size_t)f0 * fbytes,
                           (size_t)nf * fbytes, cudaMemcpyHostToDevice, ctx->copy_stream));
        CK(cudaEventRecord(ctx->cev[ci & 7], ctx->copy_stream));
        CK(cudaStreamWaitEvent(st, ctx->cev[ci & 7], 0));
        ++ci;
        return GT_OK;
    };
    // With host frames and linking, each uploaded chunk is also finalized
    // (pending walks, ordering, separation filter, offsets) and linked
    // behind its copy, so only the last chunk's work follows the upload.
    const int nchunks = (T + chunk - 1) / chunk;
    const bool chunked = h_frames && P.link && nchunks > 1 && nchunks <= LINK_WINDOWS;
    if (P.link) {
        rc = link_prepare(ctx, P, w, st);
        if (rc) return rc;
    }
    CK(cudaMemsetAsync(w.pbeg, 0, sizeof(int) * LINK_WINDOWS, st));
    CK(cudaFuncSetAttribute(fallback_walk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P.smem_fb));
    CK(cudaFuncSetAttribute(finalize_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P.smem_fin));
    int wi = 0;
    auto post = [&](int f0, int nf) -> int {
        fallback_walk_kernel<<<ctx->num_sms * 4, 128, P.smem_fb, st>>>(P.lp, b, P.fb_win, w.pbeg + wi);
        finalize_kernel<<<nf, 512, P.smem_fin, st>>>(P.lp, b, P.sep, P.link, f0);
        scan_frames_from_kernel<<<1, 1024, 0, st>>>(w.npart, w.off, f0, nf);
        CK(cudaGetLastError());
        ctx->stats.launches += 3;
        if (P.link) {
            const int r2 = link_window(ctx, P, w, st, f0, f0 + nf, wi);
            if (r2) return r2;
        }
        ++wi;
        return GT_OK;
    };
    // the fallback list position where chunk wi's entries begin
    auto mark = [&]() -> int {
        if (chunked && wi > 0) CK(cudaMemcpyAsync(w.pbeg + wi, w.npend, sizeof(int), cudaMemcpyDeviceToDevice, st));
        return GT_OK;
    };
    if (fast) {
        CK(cudaEventRecord(ctx->ev[0], st));
        for (int f0 = 0; f0 < T; f0 += chunk) {
            const int nf = std::min(chunk, T - f0);
            rc = stage(f0, nf);
            if (!rc) rc = mark();
            if (rc) return rc;
            dim3 grid(ntiles, nf);
            int used_tma = 0;
            CK(launch_locate_fast(P.lp.krad, P.lp.D, P.lp.rint_c, P.fast_th, grid, st, P.lp, b, T, f0, &used_tma));
            ctx->stats.launches += 1;
            ctx->stats.locate_kernel = used_tma ? 2 : 1;
            if (chunked && (rc = post(f0, nf))) return rc;
        }
    } else {
        LocParams lg = P.lp;  // generic tile plan (its own tile height)
        lg.TH = LOC_TH;
        lg.TW = LOC_TW;
        lg.ntx = (P.W + LOC_TW - 1) / LOC_TW;
        lg.nty = (P.H + LOC_TH - 1) / LOC_TH;
        CK(cudaEventRecord(ctx->ev[0], st));
        for (int f0 = 0; f0 < T; f0 += chunk) {
            const int nf = std::min(chunk, T - f0);
            rc = stage(f0, nf);
            if (!rc) rc = mark();
            if (rc) return rc;
            dim3 grid(lg.ntx * lg.nty, nf);
            locate_tiles_kernel<<<grid, 256, P.smem_loc, st>>>(lg, b, f0);
            ctx->stats.launches += 1;
            if (chunked && (rc = post(f0, nf))) return rc;
        }
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->ev[1], st));
    if (!chunked) {
        // the whole movie as one window: finalize, then link
        fallback_walk_kernel<<<ctx->num_sms * 4, 128, P.smem_fb, st>>>(P.lp, b, P.fb_win, w.pbeg);
        finalize_kernel<<<T, 512, P.smem_fin, st>>>(P.lp, b, P.sep, P.link, 0);
        scan_frames_from_kernel<<<1, 1024, 0, st>>>(w.npart, w.off, 0, T);
        CK(cudaGetLastError());
        ctx->stats.launches += 3;
    }
    CK(cudaEventRecord(ctx->ev[2], st));
    if (P.link) {
        if (!chunked) rc = link_window(ctx, P, w, st, 0, T, 0);
        if (!rc) rc = link_finish(ctx, P, w, st);
        if (rc) return rc;
    }
    CK(cudaEventRecord(ctx->ev[3], st));
    AsmArgs a{};
    a.T = T; a.H = P.H; a.W = P.W; a.cap_p = P.cap_p; a.cap_c = P.cap_c; a.ncols = (int)P.names.size();
    a.has_link = P.link; a.cpu_processed = P.r.cpu_processed; a.characterize = P.r.characterize;
    a.sig = P.r.has_sig; a.bg = P.r.has_bg;
    a.frames = d_frames; a.dtype = P.dtype;
    a.py = w.py; a.px = w.px; a.pm = w.pm; a.prec = w.prec; a.npart = w.npart; a.off = w.off;
    a.cand = w.cand; a.root = w.root; a.newid = w.newid;
    a.sig_off = w.sig_off; a.n_sig = (int)P.sig_off.size() / 2;
    a.bg_off = w.bg_off; a.n_bg = (int)P.bg_off.size() / 2;
    // a caller's device buffer takes the rows directly (those beyond its
    // capacity are not written; the caller learns the count)
    a.out = d_out ? d_out : w.out;
    a.out_rows = d_out ? out_rows : LLONG_MAX;
    a.walk = d_walk;
    a.walk_rows = walk_rows;
    assemble_kernel<<<T, 256, 0, st>>>(a);
    CK(cudaGetLastError());
    ctx->stats.launches += 1;
    CK(cudaEventRecord(ctx->ev[4], st));
    // every statistic of the call in one readback: error words, row count,
    // pending walks, per-frame record counts, linker phases and dirty counts
    const int nwin = std::max(wi, 1);
    const size_t n_nd = P.link ? (size_t)(T + 2) * nwin : 0;
    const size_t ph_off = (6 + (size_t)T + 1) & ~(size_t)1;  // 8-byte aligned for the phase times
    const size_t need_ints = ph_off + 8 + n_nd;
    if (ctx->h_stage_n < need_ints) {
        if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
        ctx->h_stage = nullptr;
        ctx->h_stage_n = 0;
        CK(cudaHostAlloc((void**)&ctx->h_stage, sizeof(int) * need_ints, cudaHostAllocDefault));
        ctx->h_stage_n = need_ints;
    }
    int* hs = ctx->h_stage;
    CK(cudaMemcpyAsync(hs, w.err, sizeof(int) * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(hs + 4, w.off + T, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(hs + 5, w.npend, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(hs + 6, w.fcount, sizeof(int) * T, cudaMemcpyDeviceToHost, st));
    unsigned long long* hph = (unsigned long long*)(hs + ph_off);  // 4 u64
    if (P.link) {
        CK(cudaMemcpyAsync(hph, w.phase_ns, sizeof(unsigned long long) * 4, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(hs + ph_off + 8, w.ndirty, sizeof(int) * n_nd, cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
    int hb[5] = {hs[0], hs[1], hs[2], hs[3], hs[4]};
    const int np = hs[5];
    long long nc_total = 0;
    for (int t = 0; t < T; ++t) nc_total += hs[6 + t];
    *err_bits = hb[0];
    *nrows = hb[4];
    ctx->stats.link_iterations = P.link ? hb[1] : 0;
    if (P.link) {
        for (int i = 0; i < 4; ++i) ctx->stats.link_phase_ms[i] = (float)(hph[i] * 1e-6);
        const int* nd = hs + ph_off + 8;
        for (int i = 0; i < 8; ++i) {
            int v = 0;
            for (int c = 0; c < nwin; ++c) v += i + 1 < T + 2 ? nd[(size_t)c * (T + 2) + i + 1] : 0;
            ctx->stats.link_dirty[i] = v;
        }
    }
    ctx->stats.fallback_walks = np;
    ctx->stats.particles = hb[4];
    ctx->stats.candidates = nc_total;
    cudaEventElapsedTime(&ctx->stats.ms_locate, ctx->ev[0], ctx->ev[1]);
    cudaEventElapsedTime(&ctx->stats.ms_finalize, ctx->ev[1], ctx->ev[2]);
    cudaEventElapsedTime(&ctx->stats.ms_link, ctx->ev[2], ctx->ev[3]);
    cudaEventElapsedTime(&ctx->stats.ms_assemble, ctx->ev[3], ctx->ev[4]);
    cudaEventElapsedTime(&ctx->stats.ms_total, ctx->ev[0], ctx->ev[4]);
    return GT_OK;
}

int err_status(gt_ctx* ctx, int bits, bool* retry) {
    *retry = false;
    if (bits & ERR_DEVICE_TIMEOUT) {
        ctx->err = "a bounded device wait expired (TMA tile load)";
        return GT_ERR_DEVICE_TIMEOUT;
    }
    if (bits & ERR_SUBNET_BUDGET) {
        ctx->err = "a linking subnetwork exceeded the search budget";
        return GT_ERR_SUBNET_BUDGET;
    }
    if (bits & (ERR_CAND_OVERFLOW | ERR_PART_OVERFLOW | ERR_EDGE_OVERFLOW | ERR_MEM_OVERFLOW |
                ERR_SCRATCH_OVERFLOW)) {
        *retry = true;
        ctx->err = "per-frame capacity exceeded (bits " + std::to_string(bits) + ")";
        return GT_ERR_CAPACITY;
    }
    return GT_OK;
}

size_t elem_size(int dtype) { return dtype == GT_U16 ? 2 : 4; }

// Host tables (gt_table.data) live in page-locked memory, so the
// device->host copy of a table runs at full PCIe speed and touches no fresh
// pages.  Released tables go back to a small process-wide pool (gt_table_free
// has no context) and are reused by later calls of a similar size; memory
// that cannot be page-locked falls back to malloc.
struct TablePool {
    std::mutex m;
    std::vector<std::pair<void*, size_t>> idle;  // page-locked blocks not in use
    std::map<void*, size_t> locked;               // every page-locked block handed out or idle
    size_t idle_bytes = 0;
};
TablePool& table_pool() {
    static TablePool* pool = new TablePool();  // never destroyed: tables may be freed at exit
    return *pool;
}
constexpr size_t TABLE_IDLE_MAX_BLOCKS = 4;
constexpr size_t TABLE_IDLE_MAX_BYTES = (size_t)1 << 30;

float* table_alloc(size_t bytes) {
    TablePool& tp = table_pool();
    {
        std::lock_guard<std::mutex> g(tp.m);
        int best = -1;
        for (int i = 0; i < (int)tp.idle.size(); ++i) {
            const size_t sz = tp.idle[i].second;
            if (sz >= bytes && sz <= 2 * bytes + ((size_t)2 << 20) && (best < 0 || sz < tp.idle[best].second))
                best = i;
        }
        if (best >= 0) {
            void* q = tp.idle[best].first;
            tp.idle_bytes -= tp.idle[best].second;
            tp.idle.erase(tp.idle.begin() + best);
            return (float*)q;
        }
    }
    const size_t sz = (bytes + ((size_t)2 << 20) - 1) / ((size_t)2 << 20) * ((size_t)2 << 20);
    void* q = nullptr;
    if (cudaHostAlloc(&q, sz, cudaHostAllocPortable) == cudaSuccess && q) {
        std::lock_guard<std::mutex> g(tp.m);
        tp.locked[q] = sz;
        return (float*)q;
    }
    cudaGetLastError();
    return (float*)std::malloc(bytes);
}

void table_release(void* q) {
    if (!q) return;
    TablePool& tp = table_pool();
    std::lock_guard<std::mutex> g(tp.m);
    auto it = tp.locked.find(q);
    if (it == tp.locked.end()) {
        std::free(q);
        return;
    }
    if (tp.idle.size() < TABLE_IDLE_MAX_BLOCKS && tp.idle_bytes + it->second <= TABLE_IDLE_MAX_BYTES) {
        tp.idle.push_back({q, it->second});
        tp.idle_bytes += it->second;
        return;
    }
    tp.locked.erase(it);
    cudaFreeHost(q);  // an error here (runtime already unloading at exit) is harmless
}

int batch_common(gt_ctx* ctx, const void* frames, bool host, int dtype, int T, int H, int W,
                 const gt_params* params, gt_table* out_tab, float* d_out, int64_t out_rows,
                 int64_t* nrows_out, cudaStream_t st, int* d_walk = nullptr,
                 const std::function<int(int, int)>* ready = nullptr) {
    if (!ctx) return GT_ERR_ARG;
    ctx->err.clear();
    ctx->stats = gt_stats{};
    if (!frames || !params || T < 1 || H < 1 || W < 1 || (dtype != GT_U16 && dtype != GT_F32)) {
        ctx->err = "invalid frames/shape/dtype";
        return GT_ERR_ARG;
    }
    if ((long long)H * W > (1LL << 28) || H > 65535 || W > 65535) { ctx->err = "frame too large"; return GT_ERR_ARG; }
    Resolved r;
    int rc = resolve(params, &r, &ctx->err);
    if (rc) return rc;
    r.normalized_taps = ctx->normalized_taps;
    CK(cudaSetDevice(ctx->device));
    for (int scale = 1; scale <= 64; scale *= 4) {
        Plan P;
        rc = make_plan(r, T, H, W, dtype, scale, ctx->num_sms, &P, &ctx->err, ctx->force_generic,
                       ctx->fast_tile_rows);
        if (rc) return rc;
        if (ctx->withhold_tma) {
            P.lp.tma_withhold = 1;
            P.lp.tma_spin = 1 << 10;
        }
        P.lp.tiles_per_cta = ctx->tiles_per_cta;
        const size_t fbytes = host ? (size_t)T * H * W * elem_size(dtype) : 0;
        Work w{};
        // a caller's device buffer receives the rows directly: no table slab
        const size_t need = carve(P, nullptr, &w, fbytes, true, d_out == nullptr);
        rc = ensure_arena(ctx, need);
        if (rc) return rc;
        carve(P, ctx->arena, &w, fbytes, true, d_out == nullptr);
        const void* dfr = host ? w.frames : frames;
        int bits = 0;
        int64_t nrows = 0;
        rc = run_pipeline(ctx, P, w, dfr, st, &bits, &nrows, d_walk, d_walk ? out_rows : 0, host ? frames : nullptr,
                          elem_size(dtype), ready, d_out, out_rows);
        if (rc) return rc;
        bool retry;
        rc = err_status(ctx, bits, &retry);
        ctx->stats.retries = scale > 1 ? (int)std::log2((double)scale) / 2 : 0;
        if (rc && retry && scale < 64) continue;
        if (rc) return rc;
        const int ncols = (int)P.names.size();
        if (out_tab) {
            out_tab->nrows = nrows;
            out_tab->ncols = ncols;
            std::memset(out_tab->names, 0, sizeof(out_tab->names));
            std::memset(out_tab->types, 0, sizeof(out_tab->types));
            for (int i = 0; i < ncols && i < GT_MAX_COLS; ++i) {
                std::snprintf(out_tab->names[i], sizeof(out_tab->names[i]), "%s", P.names[i].c_str());
                std::snprintf(out_tab->types[i], sizeof(out_tab->types[i]), "%s", P.types[i].c_str());
            }
            out_tab->data = table_alloc(sizeof(float) * (size_t)std::max<int64_t>(1, nrows) * ncols);
            if (!out_tab->data) { ctx->err = "host allocation failed"; return GT_ERR_OOM; }
            if (nrows > 0) {
                CK(cudaMemcpyAsync(out_tab->data, w.out, sizeof(float) * (size_t)nrows * ncols,
                                   cudaMemcpyDeviceToHost, st));
                CK(cudaStreamSynchronize(st));
            }
        }
        // with d_out the rows were written there directly (run_pipeline
        // returns after the stream is synchronised)
        if (nrows_out) *nrows_out = nrows;
        return GT_OK;
    }
    return GT_ERR_CAPACITY;
}


// ---------------------------------------------------------------------------
// Batched uneven movies (gt_batch_many_device).
//
// Every movie gets its own plan and workspace in one arena.  The locate,
// fallback, ordering/separation and output kernels of the movies are
// enqueued on side streams (parallel graph branches), the linking of all
// movies runs in one cooperative kernel (link_fixpoint_multi_kernel) whose
// blocks share one scratch pool, and the sequence is captured once into a
// CUDA graph that is replayed while the inputs stay the same.
// ---------------------------------------------------------------------------

struct BatchMovie {
    Plan P;
    Work w;
    size_t off = 0;
    bool fast = false;
    int link_slot = -1;  // index among the movies of the shared linker launch
    bool solo = false;   // linked by its own cooperative launch (large movie)
    LinkBufs solo_L{};
    int solo_grid = 0;
    int solo_nt = 256;   // threads per block of its own linker launch
    int solo_pool = 0;   // and that launch's shared-memory pool
};

struct BatchShared {
    LinkBufs* d_L = nullptr;
    int* d_mem = nullptr;
    int* d_fstart = nullptr;
    int* d_ndirty = nullptr;
    int* d_passes = nullptr;
    int* d_status = nullptr;  // 8 ints per movie: err[0..3], nrows
    int nlink = 0, max_passes = 0, link_grid = 0;
    int nsolo = 0, solo_grid = 0;
    int launches = 0;
};

// Tile rows of the specialised locate kernel for one (frame size, diameter)
// class: both variants timed on up to 32 frames of the movie, the faster
// kept for the context's lifetime.
int tune_tile_rows(gt_ctx* ctx, BatchMovie& bm, const void* frames, cudaStream_t st) {
    Plan& P = bm.P;
    const std::array<int, 6> key{P.H, P.W, P.lp.krad, P.lp.D, P.lp.rint_c, P.dtype};
    auto it = ctx->tile_rows.find(key);
    int best = P.fast_th;
    if (it != ctx->tile_rows.end()) {
        best = it->second;
    } else if (!ctx->tune_disabled) {
        for (int i = 0; i < 2; ++i)
            if (!ctx->ev[i]) CK(cudaEventCreate(&ctx->ev[i]));
        const int nf = std::min(P.T, 32);
        float ms[2] = {0.f, 0.f};
        const int ths[2] = {32, 64};
        for (int v = 0; v < 2; ++v) {
            Plan Q;
            std::string msg;
            if (make_plan(P.r, P.T, P.H, P.W, P.dtype, 1, ctx->num_sms, &Q, &msg, 0, ths[v])) return GT_ERR_ARG;
            MovieBufs b = movie_bufs(Q, bm.w, frames);
            const int ntiles = Q.lp.ntx * Q.lp.nty;
            for (int rep = 0; rep < 2; ++rep) {
                CK(cudaMemsetAsync(bm.w.fcount, 0, sizeof(int) * P.T, st));
                CK(cudaMemsetAsync(bm.w.npend, 0, sizeof(int), st));
                CK(cudaMemsetAsync(bm.w.err, 0, sizeof(int) * 4, st));
                CK(cudaEventRecord(ctx->ev[0], st));
                int used_tma = 0;
                CK(launch_locate_fast(Q.lp.krad, Q.lp.D, Q.lp.rint_c, ths[v], dim3(ntiles, nf), st, Q.lp, b, P.T, 0,
                                      &used_tma));
                CK(cudaEventRecord(ctx->ev[1], st));
                CK(cudaEventSynchronize(ctx->ev[1]));
                CK(cudaEventElapsedTime(&ms[v], ctx->ev[0], ctx->ev[1]));
            }
        }
        best = ms[1] < ms[0] ? 64 : 32;
        ctx->tile_rows[key] = best;
    }
    if (best != P.fast_th) {
        Plan Q;
        std::string msg;
        if (make_plan(P.r, P.T, P.H, P.W, P.dtype, 1, ctx->num_sms, &Q, &msg, 0, best)) return GT_ERR_ARG;
        Work w2{};
        Plan Qc = Q, Pc = P;
        Qc.nslot = 0;
        Pc.nslot = 0;
        if (carve(Qc, nullptr, &w2, 0, true, false) == carve(Pc, nullptr, &w2, 0, true, false)) P = Q;
    }
    return GT_OK;
}

// Locate, fallback walks, ordering + separation filter and frame offsets of
// one movie (the front half of run_pipeline, without host synchronisation).
int enqueue_front(gt_ctx* ctx, BatchMovie& bm, const void* frames, cudaStream_t s, int* launches) {
    const Plan& P = bm.P;
    const Work& w = bm.w;
    const int T = P.T;
    MovieBufs b = movie_bufs(P, w, frames);
    CK(cudaMemsetAsync(w.fcount, 0, sizeof(int) * T, s));
    CK(cudaMemsetAsync(w.npend, 0, sizeof(int), s));
    CK(cudaMemsetAsync(w.err, 0, sizeof(int) * 4, s));
    const int ntiles = P.lp.ntx * P.lp.nty;
    if (bm.fast) {
        for (int f0 = 0; f0 < T; f0 += 65535) {
            int used_tma = 0;
            CK(launch_locate_fast(P.lp.krad, P.lp.D, P.lp.rint_c, P.fast_th, dim3(ntiles, std::min(65535, T - f0)), s,
                                  P.lp, b, T, f0, &used_tma));
            ++*launches;
        }
    } else {
        LocParams lg = P.lp;
        lg.TH = LOC_TH;
        lg.TW = LOC_TW;
        lg.ntx = (P.W + LOC_TW - 1) / LOC_TW;
        lg.nty = (P.H + LOC_TH - 1) / LOC_TH;
        for (int f0 = 0; f0 < T; f0 += 65535) {
            dim3 grid(lg.ntx * lg.nty, std::min(65535, T - f0));
            locate_tiles_kernel<<<grid, 256, P.smem_loc, s>>>(lg, b, f0);
            ++*launches;
        }
    }
    CK(cudaGetLastError());
    fallback_walk_kernel<<<ctx->num_sms, 128, P.smem_fb, s>>>(P.lp, b, P.fb_win, nullptr);
    finalize_kernel<<<T, 512, P.smem_fin, s>>>(P.lp, b, P.sep, P.link, 0);
    scan_frames_kernel<<<1, 1024, 0, s>>>(w.npart, w.off, T);
    CK(cudaGetLastError());
    *launches += 3;
    if (P.link) {
        CK(cudaMemsetAsync(w.mcount, 0, sizeof(int) * T, s));
        CK(cudaMemsetAsync(w.dirty, 0, sizeof(int) * T, s));
    }
    return GT_OK;
}

// Trajectory ids and the output table of one movie, then its status words.
int enqueue_back(gt_ctx* ctx, BatchMovie& bm, const gt_movie& mv, int* d_status, cudaStream_t s, int* launches) {
    const Plan& P = bm.P;
    const Work& w = bm.w;
    const int T = P.T;
    if (P.link) {
        scan_frames_kernel<<<1, 1024, 0, s>>>(w.newcount, w.newbase, T);
        newid_kernel<<<T, 256, 0, s>>>(w.newrank, w.newbase, w.off, w.npart, w.newid, T);
        *launches += 2;
    }
    AsmArgs a{};
    a.T = T; a.H = P.H; a.W = P.W; a.cap_p = P.cap_p; a.cap_c = P.cap_c; a.ncols = (int)P.names.size();
    a.has_link = P.link; a.cpu_processed = P.r.cpu_processed; a.characterize = P.r.characterize;
    a.sig = P.r.has_sig; a.bg = P.r.has_bg;
    a.frames = mv.frames; a.dtype = P.dtype;
    a.py = w.py; a.px = w.px; a.pm = w.pm; a.prec = w.prec; a.npart = w.npart; a.off = w.off;
    a.cand = w.cand; a.root = w.root; a.newid = w.newid;
    a.sig_off = w.sig_off; a.n_sig = (int)P.sig_off.size() / 2;
    a.bg_off = w.bg_off; a.n_bg = (int)P.bg_off.size() / 2;
    a.out = mv.out;
    a.out_rows = mv.out ? mv.out_rows : 0;
    assemble_kernel<<<T, 256, 0, s>>>(a);
    CK(cudaGetLastError());
    *launches += 1;
    CK(cudaMemcpyAsync(d_status, w.err, sizeof(int) * 4, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(d_status + 4, w.off + T, sizeof(int), cudaMemcpyDeviceToDevice, s));
    return GT_OK;
}

// The whole batch on `st`, fanned out over the context's side streams.
int enqueue_batch(gt_ctx* ctx, std::vector<BatchMovie>& B, gt_movie* mv, int n, BatchShared& S, cudaStream_t st) {
    const int K = 8;
    S.launches = 0;
    CK(cudaEventRecord(ctx->bev[0], st));
    for (int k = 0; k < K; ++k) CK(cudaStreamWaitEvent(ctx->side[k], ctx->bev[0], 0));
    for (int i = 0; i < n; ++i) {
        int rc = enqueue_front(ctx, B[i], mv[i].frames, ctx->side[i % K], &S.launches);
        if (rc) return rc;
    }
    for (int k = 0; k < K; ++k) {
        CK(cudaEventRecord(ctx->bev[1 + k], ctx->side[k]));
        CK(cudaStreamWaitEvent(st, ctx->bev[1 + k], 0));
    }
    if (S.nlink > 0) {
        CK(cudaMemsetAsync(S.d_ndirty, 0, sizeof(int) * (size_t)(S.max_passes + 2) * S.nlink, st));
        const LinkBufs* Ls = S.d_L;
        const int* mem = S.d_mem;
        const int* fst = S.d_fstart;
        int nm = S.nlink, mp = S.max_passes;
        int* nd = S.d_ndirty;
        int* ps = S.d_passes;
        void* args[] = {(void*)&Ls, (void*)&mem, (void*)&fst, &nm, &mp, &nd, &ps};
        CK(cudaLaunchCooperativeKernel((const void*)link_fixpoint_multi_kernel, dim3(S.link_grid), dim3(256), args,
                                       LINK_POOL_BYTES, st));
        S.launches += 1;
    }
    for (int i = 0; i < n; ++i) {
        if (!B[i].solo) continue;
        BatchMovie& bm = B[i];
        CK(cudaMemsetAsync(bm.w.ndirty, 0, sizeof(int) * (bm.P.T + 2), st));
        CK(cudaMemsetAsync(bm.w.phase_ns, 0, sizeof(unsigned long long) * 4, st));
        LinkBufs L = bm.solo_L;
        int memory = (int)bm.P.r.memory, max_passes = bm.P.T + 1, rounds = 0;
        int* nd = bm.w.ndirty;
        int* ps = bm.w.err + 1;
        unsigned long long* ph = bm.w.phase_ns;
        void* args[] = {&L, &memory, &max_passes, &rounds, &nd, &ps, &ph};
        CK(launch_link_fixpoint(bm.solo_nt, bm.solo_grid, args, bm.solo_pool, st));
        S.launches += 1;
    }
    CK(cudaEventRecord(ctx->bev[9], st));
    for (int k = 0; k < K; ++k) CK(cudaStreamWaitEvent(ctx->side[k], ctx->bev[9], 0));
    for (int i = 0; i < n; ++i) {
        int rc = enqueue_back(ctx, B[i], mv[i], S.d_status + 8 * i, ctx->side[i % K], &S.launches);
        if (rc) return rc;
    }
    for (int k = 0; k < K; ++k) {
        CK(cudaEventRecord(ctx->bev[10 + k], ctx->side[k]));
        CK(cudaStreamWaitEvent(st, ctx->bev[10 + k], 0));
    }
    CK(cudaMemcpyAsync(ctx->h_status, S.d_status, sizeof(int) * 8 * (size_t)n, cudaMemcpyDeviceToHost, st));
    return GT_OK;
}

int batch_many(gt_ctx* ctx, gt_movie* mv, int n, cudaStream_t st) {
    if (!ctx) return GT_ERR_ARG;
    ctx->err.clear();
    ctx->stats = gt_stats{};
    if (n < 0 || (n > 0 && !mv)) { ctx->err = "invalid movie list"; return GT_ERR_ARG; }
    if (n == 0) return GT_OK;
    CK(cudaSetDevice(ctx->device));
    std::vector<BatchMovie> B(n);
    std::string key;
    for (int i = 0; i < n; ++i) {
        const gt_movie& m = mv[i];
        const std::string who = "movie " + std::to_string(i) + ": ";
        if (!m.frames || m.T < 1 || m.H < 1 || m.W < 1 || (m.dtype != GT_U16 && m.dtype != GT_F32) ||
            (m.out_rows > 0 && !m.out) || m.out_rows < 0) {
            ctx->err = who + "invalid frames/shape/dtype/output";
            return GT_ERR_ARG;
        }
        if ((long long)m.H * m.W > (1LL << 28) || m.H > 65535 || m.W > 65535) {
            ctx->err = who + "frame too large";
            return GT_ERR_ARG;
        }
        Resolved r;
        std::string msg;
        int rc = resolve(&m.params, &r, &msg);
        if (rc) { ctx->err = who + msg; return rc; }
        r.normalized_taps = ctx->normalized_taps;
        rc = make_plan(r, m.T, m.H, m.W, m.dtype, 1, ctx->num_sms, &B[i].P, &msg, ctx->force_generic, ctx->fast_tile_rows,
                       ctx->batch_cap_div);
        if (rc) { ctx->err = who + msg; return rc; }
        B[i].P.lp.tiles_per_cta = ctx->tiles_per_cta;
        char buf[128];
        std::snprintf(buf, sizeof(buf), "%p|%d|%d|%d|%d|%p|%lld|", m.frames, m.dtype, m.T, m.H, m.W, (void*)m.out,
                      (long long)m.out_rows);
        key += buf;
        key.append((const char*)&m.params, sizeof(gt_params));
    }
    // pinned status words, side streams, events
    if (ctx->h_status_n < (size_t)8 * n) {
        if (ctx->h_status) cudaFreeHost(ctx->h_status);
        ctx->h_status = nullptr;
        ctx->h_status_n = 0;
        CK(cudaHostAlloc((void**)&ctx->h_status, sizeof(int) * 8 * (size_t)n, cudaHostAllocDefault));
        ctx->h_status_n = (size_t)8 * n;
    }
    for (auto& sd : ctx->side)
        if (!sd) CK(cudaStreamCreateWithFlags(&sd, cudaStreamNonBlocking));
    for (auto& e : ctx->bev)
        if (!e) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (int i = 0; i < 5; ++i)
        if (!ctx->ev[i]) CK(cudaEventCreate(&ctx->ev[i]));
    // kernel choice
    for (int i = 0; i < n; ++i) B[i].fast = B[i].P.fast != 0;
    // linked movies: a movie whose per-block scratch would cap the linker
    // grid below full residency is linked by its own launch (as in the
    // one-movie path); the others share one launch whose blocks share one
    // scratch pool (slot strides of the largest of them)
    BatchShared S;
    const size_t budget = (size_t)6 << 30;
    auto slot_bytes = [](long long s_, long long s1, long long p1, long long n_, long long e_, long long h_) {
        return (size_t)(4 * (3 * s_ + s1) + 8 * e_ * 2 + 4 * p1 + 4 * 4 * n_ + n_ + 16 * n_ + 4 + 8 * h_);
    };
    int per_sm_multi = 0, per_sm_solo = 0;
    CK(cudaFuncSetAttribute(link_fixpoint_multi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, LINK_POOL_BYTES));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_multi, link_fixpoint_multi_kernel, 256, LINK_POOL_BYTES));
    CK(link_fixpoint_occupancy(256, LINK_POOL_BYTES, &per_sm_solo));
    const size_t full_grid = (size_t)std::max(1, per_sm_multi) * ctx->num_sms;
    long long st_s = 1, st_s1 = 1, st_p1 = 1, st_n = 1, st_e = 1, st_h = 64;        // shared launch
    long long bt_s = 1, bt_s1 = 1, bt_p1 = 1, bt_n = 1, bt_e = 1, bt_h = 64;        // solo launches
    for (int i = 0; i < n; ++i) {
        const Plan& P = B[i].P;
        if (!P.link) continue;
        const size_t own = slot_bytes(P.cap_s, (long long)P.cap_s + 1, (long long)P.cap_p + 1,
                                      (long long)P.cap_s + P.cap_p, P.cap_e, P.hsize);
        if (budget / own < full_grid) {
            B[i].solo = true;
            ++S.nsolo;
            bt_s = std::max<long long>(bt_s, P.cap_s);
            bt_s1 = std::max<long long>(bt_s1, (long long)P.cap_s + 1);
            bt_p1 = std::max<long long>(bt_p1, (long long)P.cap_p + 1);
            bt_n = std::max<long long>(bt_n, (long long)P.cap_s + P.cap_p);
            bt_e = std::max<long long>(bt_e, P.cap_e);
            bt_h = std::max<long long>(bt_h, P.hsize);
            continue;
        }
        B[i].link_slot = S.nlink++;
        st_s = std::max<long long>(st_s, P.cap_s);
        st_s1 = std::max<long long>(st_s1, (long long)P.cap_s + 1);
        st_p1 = std::max<long long>(st_p1, (long long)P.cap_p + 1);
        st_n = std::max<long long>(st_n, (long long)P.cap_s + P.cap_p);
        st_e = std::max<long long>(st_e, P.cap_e);
        st_h = std::max<long long>(st_h, P.hsize);
        S.max_passes = std::max(S.max_passes, P.T + 1);
    }
    if (S.nlink > 0)
        S.link_grid = (int)std::max<size_t>(1, std::min<size_t>(full_grid,
                                                                budget / slot_bytes(st_s, st_s1, st_p1, st_n, st_e, st_h)));
    if (S.nsolo > 0)
        S.solo_grid = (int)std::max<size_t>(1, std::min<size_t>((size_t)std::max(1, per_sm_solo) * ctx->num_sms,
                                                                budget / slot_bytes(bt_s, bt_s1, bt_p1, bt_n, bt_e, bt_h)));
    // arena layout: movies, link pool, shared arrays
    size_t total = 0;
    for (int i = 0; i < n; ++i) {
        Plan Pc = B[i].P;
        Pc.nslot = 0;
        Work w{};
        B[i].off = total;
        total += carve(Pc, nullptr, &w, 0, true, false);
        total = (total + 255) / 256 * 256;
    }
    const size_t G = S.link_grid, GB = S.solo_grid;
    Carver pc{nullptr};
    auto slots = [](Carver& c, Work& pw, size_t g, long long s_, long long s1, long long p1, long long n_,
                    long long e_, long long h_) {
        pw.s_y = c.take<float>(g * s_); pw.s_x = c.take<float>(g * s_); pw.s_h = c.take<int>(g * s_);
        pw.s_deg = c.take<int>(g * s1); pw.e_dst = c.take<int>(g * e_); pw.e_w = c.take<float>(g * e_);
        pw.d_cnt = c.take<int>(g * p1); pw.d_src = c.take<int>(g * e_); pw.d_w = c.take<float>(g * e_);
        pw.uf = c.take<int>(g * n_); pw.c_nd = c.take<int>(g * n_); pw.c_ns = c.take<int>(g * n_);
        pw.c_min = c.take<int>(g * n_); pw.vis = c.take<unsigned char>(g * n_);
        pw.work = c.take<int>(g * 4 * n_); pw.bump = c.take<int>(g); pw.hkey = c.take<int>(g * h_);
        pw.hval = c.take<int>(g * h_);
    };
    // solo launches run one after another: each lays out its own grid of
    // slots with its own strides at the start of one shared region
    size_t big_bytes = 0;
    for (int i = 0; i < n; ++i) {
        if (!B[i].solo) continue;
        const Plan& P = B[i].P;
        const size_t own = slot_bytes(P.cap_s, (long long)P.cap_s + 1, (long long)P.cap_p + 1,
                                      (long long)P.cap_s + P.cap_p, P.cap_e, P.hsize);
        int per_sm_own = 1;
        int rc_s = link_shape(ctx, (long long)P.H * P.W, &B[i].solo_nt, &per_sm_own, &B[i].solo_pool);
        if (rc_s) return rc_s;
        B[i].solo_grid = (int)std::max<size_t>(1, std::min<size_t>({(size_t)P.T,
                                                                   (size_t)per_sm_own * ctx->num_sms,
                                                                   budget / own}));
        Carver dry{nullptr};
        Work wd{};
        slots(dry, wd, B[i].solo_grid, P.cap_s, (long long)P.cap_s + 1, (long long)P.cap_p + 1,
              (long long)P.cap_s + P.cap_p, P.cap_e, P.hsize);
        big_bytes = std::max(big_bytes, dry.off);
    }
    char* big_base = nullptr;
    (void)GB;
    auto pool_layout = [&](Carver& c, Work& pw) {
        slots(c, pw, G, st_s, st_s1, st_p1, st_n, st_e, st_h);
        big_base = c.take<char>(big_bytes);
        S.d_L = c.take<LinkBufs>(std::max(1, S.nlink));
        S.d_mem = c.take<int>(std::max(1, S.nlink));
        S.d_fstart = c.take<int>(std::max(1, S.nlink));
        S.d_ndirty = c.take<int>((size_t)(S.max_passes + 2) * std::max(1, S.nlink));
        S.d_passes = c.take<int>(1);
        S.d_status = c.take<int>(8 * (size_t)n);
    };
    Work pool{};
    pool_layout(pc, pool);
    const size_t pool_bytes = pc.off + 256;
    const size_t need = total + pool_bytes;
    {
        // the batch must fit beside the caller's data: tighter first
        // candidate capacities (overflowing movies are rerun alone)
        size_t free_b = 0, total_b = 0;
        CK(cudaMemGetInfo(&free_b, &total_b));
        const size_t avail = free_b + (ctx->arena ? ctx->arena_size : 0);
        if (need > avail - avail / 8) {
            if (ctx->batch_cap_div < 1024) {
                ctx->batch_cap_div *= 4;
                const int rc2 = batch_many(ctx, mv, n, st);
                ctx->batch_cap_div = 64;
                return rc2;
            }
            ctx->err = "the batch does not fit in device memory; split it";
            return GT_ERR_OOM;
        }
    }
    int rc = ensure_arena(ctx, need);
    if (rc) return rc;
    {
        char buf[96];
        std::snprintf(buf, sizeof(buf), "arena %p %p %d %d %d", (void*)ctx->arena, (void*)st, ctx->force_generic,
                      ctx->tune_disabled, ctx->batch_cap_div);
        key += buf;
    }
    for (int i = 0; i < n; ++i) {
        Plan Pc = B[i].P;
        Pc.nslot = 0;
        carve(Pc, ctx->arena + B[i].off, &B[i].w, 0, true, false);
    }
    Carver c2{ctx->arena + total};
    pool_layout(c2, pool);
    const bool replay = ctx->batch_exec && key == ctx->batch_key;
    // constant tables and linker descriptors (other calls may have reused
    // the arena since the graph was built)
    for (int i = 0; i < n; ++i) {
        rc = upload_tables(ctx, B[i].P, B[i].w, st);
        if (rc) return rc;
    }
    std::vector<LinkBufs> hL(std::max(1, S.nlink));
    std::vector<int> hm(std::max(1, S.nlink)), hf(std::max(1, S.nlink));
    if (S.nlink > 0) {
        int fs = 0;
        for (int i = 0; i < n; ++i) {
            if (B[i].link_slot < 0) continue;
            LinkBufs L = link_bufs(B[i].P, B[i].w, ctx->subnet_budget);
            L.nslot = (int)G;
            L.s_y = pool.s_y; L.s_x = pool.s_x; L.s_h = pool.s_h; L.s_deg = pool.s_deg;
            L.e_dst = pool.e_dst; L.e_w = pool.e_w; L.d_cnt = pool.d_cnt; L.d_src = pool.d_src; L.d_w = pool.d_w;
            L.uf = pool.uf; L.c_nd = pool.c_nd; L.c_ns = pool.c_ns; L.c_min = pool.c_min; L.vis = pool.vis;
            L.work = pool.work; L.bump = pool.bump; L.hkey = pool.hkey; L.hval = pool.hval;
            L.st_s = st_s; L.st_s1 = st_s1; L.st_p1 = st_p1; L.st_n = st_n; L.st_e = st_e; L.st_h = st_h;
            L.lsm_bytes = LINK_POOL_BYTES;
            hL[B[i].link_slot] = L;
            hm[B[i].link_slot] = (int)B[i].P.r.memory;
            hf[B[i].link_slot] = fs;
            fs += B[i].P.T;
        }
        CK(cudaMemcpyAsync(S.d_L, hL.data(), sizeof(LinkBufs) * S.nlink, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(S.d_mem, hm.data(), sizeof(int) * S.nlink, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(S.d_fstart, hf.data(), sizeof(int) * S.nlink, cudaMemcpyHostToDevice, st));
    }
    for (int i = 0; i < n; ++i) {
        if (!B[i].solo) continue;
        const Plan& P = B[i].P;
        Work pool_big{};
        Carver cb{big_base};
        slots(cb, pool_big, B[i].solo_grid, P.cap_s, (long long)P.cap_s + 1, (long long)P.cap_p + 1,
              (long long)P.cap_s + P.cap_p, P.cap_e, P.hsize);
        LinkBufs L = link_bufs(B[i].P, B[i].w, ctx->subnet_budget);
        L.nslot = B[i].solo_grid;
        L.s_y = pool_big.s_y; L.s_x = pool_big.s_x; L.s_h = pool_big.s_h; L.s_deg = pool_big.s_deg;
        L.e_dst = pool_big.e_dst; L.e_w = pool_big.e_w; L.d_cnt = pool_big.d_cnt; L.d_src = pool_big.d_src;
        L.d_w = pool_big.d_w; L.uf = pool_big.uf; L.c_nd = pool_big.c_nd; L.c_ns = pool_big.c_ns;
        L.c_min = pool_big.c_min; L.vis = pool_big.vis; L.work = pool_big.work; L.bump = pool_big.bump;
        L.hkey = pool_big.hkey; L.hval = pool_big.hval;
        L.lsm_bytes = B[i].solo_pool;  // slot strides: the movie's own (link_bufs)
        B[i].solo_L = L;
    }
    if (!replay) {
        if (ctx->batch_exec) { cudaGraphExecDestroy(ctx->batch_exec); ctx->batch_exec = nullptr; }
        ctx->batch_key.clear();
        // autotuned tile rows (timed on this movie's frames and workspace)
        for (int i = 0; i < n; ++i)
            if (B[i].fast) {
                rc = tune_tile_rows(ctx, B[i], mv[i].frames, st);
                if (rc) return rc;
            }
        size_t sl = 0, sf = 0, sn = 0;
        for (int i = 0; i < n; ++i) {
            sl = std::max(sl, B[i].P.smem_loc);
            sf = std::max(sf, B[i].P.smem_fb);
            sn = std::max(sn, B[i].P.smem_fin);
        }
        CK(cudaFuncSetAttribute(locate_tiles_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sl));
        CK(cudaFuncSetAttribute(fallback_walk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sf));
        CK(cudaFuncSetAttribute(finalize_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sn));
        CK(cudaStreamSynchronize(st));
        // capture; where capture is refused, run the same sequence directly
        cudaGraph_t graph = nullptr;
        bool captured = false;
        if (cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed) == cudaSuccess) {
            const int erc = enqueue_batch(ctx, B, mv, n, S, st);
            const cudaError_t ee = cudaStreamEndCapture(st, &graph);
            if (erc == GT_OK && ee == cudaSuccess && graph) {
                cudaGraphExec_t ex = nullptr;
                if (cudaGraphInstantiate(&ex, graph, 0) == cudaSuccess) {
                    ctx->batch_exec = ex;
                    ctx->batch_key = key;
                    captured = true;
                }
            }
            if (graph) cudaGraphDestroy(graph);
            if (!captured) {
                cudaGetLastError();
                ctx->err.clear();
            }
        } else {
            cudaGetLastError();
        }
        CK(cudaEventRecord(ctx->ev[0], st));
        if (captured) {
            CK(cudaGraphLaunch(ctx->batch_exec, st));
            ctx->stats.batch_graph = 1;
        } else {
            rc = enqueue_batch(ctx, B, mv, n, S, st);
            if (rc) return rc;
        }
    } else {
        CK(cudaStreamSynchronize(st));
        CK(cudaEventRecord(ctx->ev[0], st));
        CK(cudaGraphLaunch(ctx->batch_exec, st));
        ctx->stats.batch_graph = 2;
        // launches of the captured sequence
        int cnt = 0;
        for (int i = 0; i < n; ++i) {
            const Plan& P = B[i].P;
            cnt += (P.T + 65534) / 65535 + 3 + (P.link ? 2 : 0) + 1;
        }
        S.launches = cnt + (S.nlink > 0 ? 1 : 0) + S.nsolo;
    }
    CK(cudaEventRecord(ctx->ev[1], st));
    CK(cudaStreamSynchronize(st));
    cudaEventElapsedTime(&ctx->stats.ms_total, ctx->ev[0], ctx->ev[1]);
    ctx->stats.launches = S.launches;
    if (S.nlink > 0) {
        int passes = 0;
        CK(cudaMemcpy(&passes, S.d_passes, sizeof(int), cudaMemcpyDeviceToHost));
        ctx->stats.link_iterations = passes;
    }
    for (int i = 0; i < n; ++i)
        if (B[i].solo) ctx->stats.link_iterations = std::max(ctx->stats.link_iterations, ctx->h_status[8 * i + 1]);
    // per-movie status; capacity overflows are rerun through the plain path
    std::vector<int> status(ctx->h_status, ctx->h_status + 8 * (size_t)n);
    gt_stats keep = ctx->stats;
    int fallbacks = 0;
    int64_t rows_total = 0;
    for (int i = 0; i < n; ++i) {
        const int bits = status[8 * i];
        bool retry = false;
        rc = err_status(ctx, bits, &retry);
        if (rc && !retry) { ctx->err = "movie " + std::to_string(i) + ": " + ctx->err; return rc; }
        if (rc && retry) {
            ++fallbacks;
            int64_t nr = 0;
            rc = batch_common(ctx, mv[i].frames, false, mv[i].dtype, mv[i].T, mv[i].H, mv[i].W, &mv[i].params,
                              nullptr, mv[i].out, mv[i].out_rows, &nr, st);
            if (rc) { ctx->err = "movie " + std::to_string(i) + ": " + ctx->err; return rc; }
            mv[i].nrows = nr;
        } else {
            mv[i].nrows = status[8 * i + 4];
        }
        rows_total += mv[i].nrows;
    }
    ctx->err.clear();
    ctx->stats = keep;
    ctx->stats.batch_fallbacks = fallbacks;
    ctx->stats.particles = rows_total;
    return GT_OK;
}

// Parameters of the gt_adjoint_* calls: the forward weights exactly as
// make_plan derives them, the normalised taps a_i = w_i / sum(w) and
// da_i / ds in double precision, and the centroid circle in the order of
// the centroid loop (i outer, j inner, float mask <= r^2).
int adjoint_setup(gt_ctx* ctx, const float* d_frames, int T, int H, int W, const gt_params* params,
                  const int32_t* d_walk, int64_t n, AdjParams* ap, std::vector<int>* circ) {
    if (!ctx) return GT_ERR_ARG;
    ctx->err.clear();
    ctx->stats = gt_stats{};
    if (!d_frames || !params || T < 1 || H < 1 || W < 1 || n < 0 || (n > 0 && !d_walk)) {
        ctx->err = "invalid frames/shape/walk";
        return GT_ERR_ARG;
    }
    if ((long long)H * W > (1LL << 28) || H > 65535 || W > 65535) { ctx->err = "frame too large"; return GT_ERR_ARG; }
    Resolved r;
    int rc = resolve(params, &r, &ctx->err);
    if (rc) return rc;
    if (r.max_iterations < 1) {
        ctx->err = "the adjoint needs max_iterations >= 1";
        return GT_ERR_UNSUPPORTED;
    }
    if (r.diameter > 31) {
        ctx->err = "the adjoint supports diameter <= 31";
        return GT_ERR_UNSUPPORTED;
    }
    std::memset(ap, 0, sizeof(*ap));
    ap->T = T; ap->H = H; ap->W = W;
    const int k = (int)r.smoothing_size;
    ap->krad = k / 2;
    if (H <= ap->krad || W <= ap->krad) { ctx->err = "frame smaller than the smoothing window"; return GT_ERR_ARG; }
    const float sigma2 = r.noise_size;
    if (!(sigma2 > 0.0f)) { ctx->err = "noise_size must be > 0"; return GT_ERR_ARG; }
    gauss_taps(k, sigma2, ctx->normalized_taps, ap->w, &ap->norm, &ap->rn);
    double sw = 0.0, swi = 0.0;
    for (int i = -ap->krad; i <= ap->krad; ++i) {
        const double gd = std::exp(-(double)i * i / (2.0 * sigma2));
        sw += gd;
        swi += gd * i * i;
    }
    ap->kk = (float)(k * k);
    ap->rkk = 1.0f / ap->kk;
    const double s2 = (double)sigma2 * sigma2;
    for (int i = -ap->krad; i <= ap->krad; ++i) {
        const double ai = std::exp(-(double)i * i / (2.0 * sigma2)) / sw;
        ap->a[i + ap->krad] = (float)ai;
        // d/ds [exp(-i^2 / 2s) / sum_j exp(-j^2 / 2s)] = a_i (i^2 - <j^2>) / (2 s^2)
        ap->da[i + ap->krad] = (float)(ai * ((double)i * i - swi / sw) / (2.0 * s2));
    }
    ap->k = (float)k;
    ap->rc = ((int)r.diameter - 1) / 2;
    ap->border = (int)r.diameter / 2;
    circ->clear();
    const float rr = (float)ap->rc;
    const float r2 = rr * rr;
    for (int i = -ap->rc; i <= ap->rc; ++i)
        for (int j = -ap->rc; j <= ap->rc; ++j) {
            const float x = (float)i, y = (float)j;
            if (x * x + y * y > r2) continue;
            circ->push_back(i);
            circ->push_back(j);
        }
    ap->K = (int)circ->size() / 2;
    ap->gain = 1.0f;
    ap->read_var = 0.0f;
    CK(cudaSetDevice(ctx->device));
    return GT_OK;
}

// Scratch of the gt_adjoint_* calls in the context arena: the error word,
// the circle table and (backward only) the dL/dR plane.
struct AdjWork {
    int* err;
    int* circ;
    float* plane;
    double* gpart;  // per-block partial parameter gradients (backward only)
};

int adjoint_work(gt_ctx* ctx, const AdjParams& ap, const std::vector<int>& circ, bool plane, AdjWork* aw,
                 cudaStream_t st) {
    const size_t off_circ = 256;
    const size_t off_part = off_circ + ((sizeof(int) * circ.size() + 255) / 256) * 256;
    const size_t n_part = 2 * (size_t)adjoint_particle_blocks_max(ctx->num_sms);
    const size_t off_plane = off_part + ((sizeof(double) * n_part + 255) / 256) * 256;
    const size_t need = off_plane + (plane ? sizeof(float) * (size_t)ap.T * ap.H * ap.W : 0);
    int rc = ensure_arena(ctx, need);
    if (rc) return rc;
    aw->err = (int*)ctx->arena;
    aw->circ = (int*)(ctx->arena + off_circ);
    aw->gpart = (double*)(ctx->arena + off_part);
    aw->plane = plane ? (float*)(ctx->arena + off_plane) : nullptr;
    CK(cudaMemsetAsync(aw->err, 0, sizeof(int), st));
    CK(cudaMemcpyAsync(aw->circ, circ.data(), sizeof(int) * circ.size(), cudaMemcpyHostToDevice, st));
    for (int i = 0; i < 3; ++i)
        if (!ctx->ev[i]) CK(cudaEventCreate(&ctx->ev[i]));
    return GT_OK;
}

int adjoint_finish(gt_ctx* ctx, const AdjWork& aw, cudaStream_t st) {
    int herr = 0;
    CK(cudaMemcpyAsync(&herr, aw.err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (herr) {
        ctx->err = "a walk record lies outside the frames";
        return GT_ERR_ARG;
    }
    return GT_OK;
}
}  // namespace

namespace {
thread_local std::string g_noctx_err;  // errors of calls made without a context
}

namespace gt {
void set_noctx_error(const char* msg) { g_noctx_err = msg; }
}  // namespace gt

extern "C" {

const char* gt_version(void) { return "gt-b200 0.1.0 (sm_100a)"; }

int gt_ctx_create(int device, gt_ctx** out) {
    if (!out) return GT_ERR_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) return GT_ERR_CUDA;
    gt_ctx* c = new gt_ctx();
    c->device = device;
    if (cudaSetDevice(device) != cudaSuccess) { delete c; return GT_ERR_CUDA; }
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) { delete c; return GT_ERR_CUDA; }
    cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
    *out = c;
    return GT_OK;
}

void gt_ctx_destroy(gt_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->arena) cudaFree(ctx->arena);
    if (ctx->batch_exec) cudaGraphExecDestroy(ctx->batch_exec);
    if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
    for (auto& e : ctx->cev)
        if (e) cudaEventDestroy(e);
    if (ctx->h_status) cudaFreeHost(ctx->h_status);
    if (ctx->h_frames) cudaFreeHost(ctx->h_frames);
    if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
    for (auto& sd : ctx->side)
        if (sd) cudaStreamDestroy(sd);
    for (auto& e : ctx->bev)
        if (e) cudaEventDestroy(e);
    for (auto& e : ctx->ev)
        if (e) cudaEventDestroy(e);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char* gt_last_error(const gt_ctx* ctx) {
    if (ctx) return ctx->err.c_str();
    return g_noctx_err.c_str();
}

int gt_column_names(const gt_params* params, char* buf, size_t buflen) {
    if (!params || !buf) return -GT_ERR_ARG;
    g_noctx_err.clear();
    Resolved r;
    int rc = resolve(params, &r, &g_noctx_err);
    if (rc) return -rc;
    std::vector<std::string> names, types;
    column_list(r, names, types);
    std::string s;
    for (size_t i = 0; i < names.size(); ++i) {
        if (i) s += ",";
        s += names[i] + ":" + types[i];
    }
    if (s.size() + 1 > buflen) return -GT_ERR_ARG;
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return (int)names.size();
}

int gt_batch(gt_ctx* ctx, const void* frames, int dtype, int T, int H, int W, const gt_params* params,
             gt_table* out) {
    if (!out) return GT_ERR_ARG;
    out->data = nullptr;
    out->nrows = 0;
    out->ncols = 0;
    return batch_common(ctx, frames, true, dtype, T, H, W, params, out, nullptr, 0, nullptr,
                        ctx ? ctx->stream : nullptr);
}

int gt_file_info(const char* path, int has_channel, uint32_t channel, int32_t* T, int32_t* H, int32_t* W) {
    g_noctx_err.clear();
    if (!T || !H || !W) { g_noctx_err = "null output"; return GT_ERR_ARG; }
    gt::MovieFile mf;
    std::string msg;
    const int rc = mf.open(path, has_channel != 0, channel, &msg);
    if (rc) { g_noctx_err = msg; return rc == 2 ? GT_ERR_UNSUPPORTED : GT_ERR_ARG; }
    *T = mf.T; *H = mf.H; *W = mf.W;
    return GT_OK;
}

int gt_file_read(const char* path, int has_channel, uint32_t channel, uint16_t* out, int64_t max_values) {
    g_noctx_err.clear();
    gt::MovieFile mf;
    std::string msg;
    const int rc = mf.open(path, has_channel != 0, channel, &msg);
    if (rc) { g_noctx_err = msg; return rc == 2 ? GT_ERR_UNSUPPORTED : GT_ERR_ARG; }
    const int64_t fpx = (int64_t)mf.H * mf.W;
    if (!out || max_values < fpx * mf.T) { g_noctx_err = "output buffer too small"; return GT_ERR_ARG; }
    for (int t = 0; t < mf.T; ++t)
        if (mf.read_frame(t, out + fpx * t, &msg)) { g_noctx_err = msg; return GT_ERR_ARG; }
    return GT_OK;
}

int gt_ets_channels(const char* path, int32_t* channels, int32_t* frames, int32_t max_channels, int32_t* nchannels,
                    int32_t* dim0, int32_t* dim1) {
    g_noctx_err.clear();
    if (!nchannels || !dim0 || !dim1 || (max_channels > 0 && (!channels || !frames))) {
        g_noctx_err = "null output";
        return GT_ERR_ARG;
    }
    std::vector<std::pair<uint32_t, int>> ch;
    uint32_t dims[2];
    std::string msg;
    if (gt::ets_channels(path, &ch, dims, &msg)) { g_noctx_err = msg; return GT_ERR_ARG; }
    *nchannels = (int32_t)ch.size();
    *dim0 = (int32_t)dims[0];
    *dim1 = (int32_t)dims[1];
    for (int i = 0; i < (int)ch.size() && i < max_channels; ++i) {
        channels[i] = (int32_t)ch[i].first;
        frames[i] = ch[i].second;
    }
    return GT_OK;
}

int gt_batch_file(gt_ctx* ctx, const char* path, int has_channel, uint32_t channel, const gt_params* params,
                  gt_table* out) {
    if (!ctx) return GT_ERR_ARG;
    ctx->err.clear();
    if (!params || !out) { ctx->err = "null params/output"; return GT_ERR_ARG; }
    gt::MovieFile mf;
    std::string msg;
    int rc = mf.open(path, has_channel != 0, channel, &msg);
    if (rc) { ctx->err = msg; return rc == 2 ? GT_ERR_UNSUPPORTED : GT_ERR_ARG; }
    const size_t fpx = (size_t)mf.H * mf.W, npx = fpx * mf.T;
    CK(cudaSetDevice(ctx->device));
    if (ctx->h_frames_n < npx) {
        if (ctx->h_frames) cudaFreeHost(ctx->h_frames);
        ctx->h_frames = nullptr;
        ctx->h_frames_n = 0;
        CK(cudaHostAlloc((void**)&ctx->h_frames, sizeof(uint16_t) * npx, cudaHostAllocDefault));
        ctx->h_frames_n = npx;
    }
    // frames are decoded by a pool of host threads into pinned memory; each
    // chunk's upload (and its locate launch) waits for its own frames only
    const int T = mf.T;
    std::vector<std::atomic<unsigned char>> done(T);
    for (auto& d : done) d.store(0);
    std::atomic<int> next{0}, failed{0};
    std::mutex mu;
    std::condition_variable cv;
    std::string err;
    uint16_t* dst = ctx->h_frames;
    auto worker = [&]() {
        std::string m;
        for (int t = next.fetch_add(1); t < T && !failed.load(); t = next.fetch_add(1)) {
            if (mf.read_frame(t, dst + fpx * t, &m)) {
                std::lock_guard<std::mutex> lk(mu);
                if (!failed.exchange(1)) err = m;
                cv.notify_all();
                return;
            }
            done[t].store(1);
            std::lock_guard<std::mutex> lk(mu);
            cv.notify_all();
        }
    };
    const int nthr = (int)std::max(1u, std::min<unsigned>({std::thread::hardware_concurrency(), 16u, (unsigned)T}));
    std::vector<std::thread> pool;
    for (int i = 0; i < nthr; ++i) pool.emplace_back(worker);
    const std::function<int(int, int)> ready = [&](int f0, int nf) -> int {
        std::unique_lock<std::mutex> lk(mu);
        for (int t = f0; t < f0 + nf; ++t) {
            cv.wait(lk, [&] { return done[t].load() || failed.load(); });
            if (failed.load()) return GT_ERR_ARG;
        }
        return GT_OK;
    };
    rc = batch_common(ctx, dst, true, GT_U16, T, mf.H, mf.W, params, out, nullptr, 0, nullptr, ctx->stream, nullptr,
                      &ready);
    failed.store(failed.load() | (rc ? 2 : 0));
    for (auto& th : pool) th.join();
    if (rc == GT_ERR_ARG && !err.empty()) ctx->err = err;
    return rc;
}

int gt_batch_device(gt_ctx* ctx, const void* d_frames, int dtype, int T, int H, int W,
                    const gt_params* params, float* d_out, int64_t out_rows, int64_t* nrows, void* stream) {
    cudaStream_t st = stream ? (cudaStream_t)stream : (ctx ? ctx->stream : nullptr);
    return batch_common(ctx, d_frames, false, dtype, T, H, W, params, nullptr, d_out, out_rows, nrows, st);
}

int gt_batch_device_walk(gt_ctx* ctx, const void* d_frames, int dtype, int T, int H, int W,
                         const gt_params* params, float* d_out, int64_t out_rows, int64_t* nrows, int32_t* d_walk,
                         void* stream) {
    if (ctx && !d_walk && out_rows > 0) {
        ctx->err = "null walk buffer";
        return GT_ERR_ARG;
    }
    cudaStream_t st = stream ? (cudaStream_t)stream : (ctx ? ctx->stream : nullptr);
    return batch_common(ctx, d_frames, false, dtype, T, H, W, params, nullptr, d_out, out_rows, nrows, st,
                        (int*)d_walk);
}

int gt_adjoint_forward(gt_ctx* ctx, const float* d_frames, int T, int H, int W, const gt_params* params,
                       const int32_t* d_walk, int64_t n, float* d_yxm, void* stream) {
    AdjParams ap;
    std::vector<int> circ;
    int rc = adjoint_setup(ctx, d_frames, T, H, W, params, d_walk, n, &ap, &circ);
    if (rc) return rc;
    if (n > 0 && !d_yxm) { ctx->err = "null output"; return GT_ERR_ARG; }
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    AdjWork aw;
    rc = adjoint_work(ctx, ap, circ, false, &aw, st);
    if (rc) return rc;
    CK(cudaEventRecord(ctx->ev[0], st));
    CK(launch_adjoint_particles(0, ap, d_frames, d_walk, n, aw.circ, nullptr, d_yxm, nullptr, nullptr, nullptr, aw.err,
                                ctx->num_sms, st));
    CK(cudaEventRecord(ctx->ev[1], st));
    ctx->stats.launches = n > 0 ? 1 : 0;
    rc = adjoint_finish(ctx, aw, st);
    cudaEventElapsedTime(&ctx->stats.ms_adjoint_particles, ctx->ev[0], ctx->ev[1]);
    ctx->stats.ms_total = ctx->stats.ms_adjoint_particles;
    return rc;
}

int gt_adjoint_backward(gt_ctx* ctx, const float* d_frames, int T, int H, int W, const gt_params* params,
                        const int32_t* d_walk, int64_t n, const float* d_grad_yxm, float* d_grad_frames,
                        double* d_grad_params, void* stream) {
    AdjParams ap;
    std::vector<int> circ;
    int rc = adjoint_setup(ctx, d_frames, T, H, W, params, d_walk, n, &ap, &circ);
    if (rc) return rc;
    if (!d_grad_frames || !d_grad_params || (n > 0 && !d_grad_yxm)) { ctx->err = "null output"; return GT_ERR_ARG; }
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    AdjWork aw;
    rc = adjoint_work(ctx, ap, circ, true, &aw, st);
    if (rc) return rc;
    if (n == 0) CK(cudaMemsetAsync(d_grad_params, 0, 2 * sizeof(double), st));
    CK(cudaEventRecord(ctx->ev[0], st));
    CK(cudaMemsetAsync(aw.plane, 0, sizeof(float) * (size_t)T * H * W, st));
    CK(cudaEventRecord(ctx->ev[1], st));
    CK(launch_adjoint_particles(1, ap, d_frames, d_walk, n, aw.circ, d_grad_yxm, nullptr, aw.plane, d_grad_params,
                                aw.gpart, aw.err, ctx->num_sms, st));
    CK(cudaEventRecord(ctx->ev[2], st));
    CK(launch_adjoint_transpose(ap, aw.plane, d_grad_frames, st));
    ctx->stats.launches = (n > 0 ? 2 : 0) + (T + 65534) / 65535;
    // the dense part is the zeroing plus the transposed bandpass
    if (!ctx->ev[3]) CK(cudaEventCreate(&ctx->ev[3]));
    CK(cudaEventRecord(ctx->ev[3], st));
    rc = adjoint_finish(ctx, aw, st);
    cudaEventElapsedTime(&ctx->stats.ms_adjoint_particles, ctx->ev[1], ctx->ev[2]);
    float tz = 0.f, tt = 0.f;
    cudaEventElapsedTime(&tz, ctx->ev[0], ctx->ev[1]);
    cudaEventElapsedTime(&tt, ctx->ev[2], ctx->ev[3]);
    ctx->stats.ms_adjoint_dense = tz + tt;
    cudaEventElapsedTime(&ctx->stats.ms_total, ctx->ev[0], ctx->ev[3]);
    return rc;
}

int gt_adjoint_uncertainty(gt_ctx* ctx, const float* d_frames, int T, int H, int W, const gt_params* params,
                           const int32_t* d_walk, int64_t n, float gain, float read_noise, float* d_sd,
                           void* stream) {
    AdjParams ap;
    std::vector<int> circ;
    int rc = adjoint_setup(ctx, d_frames, T, H, W, params, d_walk, n, &ap, &circ);
    if (rc) return rc;
    if (n > 0 && !d_sd) { ctx->err = "null output"; return GT_ERR_ARG; }
    if (!(gain >= 0.0f) || !(read_noise >= 0.0f) || !std::isfinite(gain) || !std::isfinite(read_noise)) {
        ctx->err = "gain and read_noise must be finite and >= 0";
        return GT_ERR_ARG;
    }
    ap.gain = gain;
    ap.read_var = read_noise * read_noise;
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    AdjWork aw;
    rc = adjoint_work(ctx, ap, circ, false, &aw, st);
    if (rc) return rc;
    CK(cudaEventRecord(ctx->ev[0], st));
    CK(launch_adjoint_particles(2, ap, d_frames, d_walk, n, aw.circ, nullptr, d_sd, nullptr, nullptr, nullptr, aw.err,
                                ctx->num_sms, st));
    CK(cudaEventRecord(ctx->ev[1], st));
    ctx->stats.launches = n > 0 ? 1 : 0;
    rc = adjoint_finish(ctx, aw, st);
    cudaEventElapsedTime(&ctx->stats.ms_adjoint_particles, ctx->ev[0], ctx->ev[1]);
    ctx->stats.ms_total = ctx->stats.ms_adjoint_particles;
    return rc;
}

int gt_batch_many_device(gt_ctx* ctx, gt_movie* movies, int n, void* stream) {
    cudaStream_t st = stream ? (cudaStream_t)stream : (ctx ? ctx->stream : nullptr);
    return batch_many(ctx, movies, n, st);
}

int gt_ctx_set_option(gt_ctx* ctx, const char* key, int value) {
    if (!ctx || !key) return GT_ERR_ARG;
    const std::string k(key);
    if (k == "locate_tile_rows" && (value == 32 || value == 64)) { ctx->fast_tile_rows = value; return GT_OK; }
    if (k == "force_generic" && (value == 0 || value == 1)) { ctx->force_generic = value; return GT_OK; }
    if (k == "autotune" && (value == 0 || value == 1)) { ctx->tune_disabled = !value; return GT_OK; }
    if (k == "subnet_budget" && value > 0) { ctx->subnet_budget = value; return GT_OK; }
    if (k == "subnet_budget" && value == 0) { ctx->subnet_budget = SUBNET_BUDGET; return GT_OK; }
    if (k == "test_withhold_tile_copy" && (value == 0 || value == 1)) { ctx->withhold_tma = value; return GT_OK; }
    if (k == "locate_tiles_per_cta" && value >= 0 && value <= 64) {
        ctx->tiles_per_cta = value;
        if (ctx->batch_exec) {  // the cached batch graph holds the old launch shape
            cudaGraphExecDestroy(ctx->batch_exec);
            ctx->batch_exec = nullptr;
            ctx->batch_key.clear();
        }
        return GT_OK;
    }
    if (k == "normalized_taps" && (value == 0 || value == 1)) {
        ctx->normalized_taps = value;
        if (ctx->batch_exec) {  // the cached batch graph holds the old taps
            cudaGraphExecDestroy(ctx->batch_exec);
            ctx->batch_exec = nullptr;
            ctx->batch_key.clear();
        }
        return GT_OK;
    }
    ctx->err = "unknown option or value: " + k;
    return GT_ERR_ARG;
}

void gt_table_free(gt_table* table) {
    if (table && table->data) { table_release(table->data); table->data = nullptr; }
}

namespace {
// trajectory entry points share the argument checks
int traj_begin(gt_ctx* ctx, int64_t n, bool ok_ptrs) {
    if (!ctx) return GT_ERR_ARG;
    ctx->err.clear();
    ctx->stats = gt_stats{};
    if (n < 0 || (n > 0 && !ok_ptrs)) {
        ctx->err = "invalid arrays";
        return GT_ERR_ARG;
    }
    if (n >= ((int64_t)1 << 31)) {
        ctx->err = "table too large";
        return GT_ERR_ARG;
    }
    if (cudaSetDevice(ctx->device) != cudaSuccess) {
        ctx->err = "cudaSetDevice failed";
        return GT_ERR_CUDA;
    }
    return GT_OK;
}
}  // namespace

int gt_filter_stubs(gt_ctx* ctx, const int64_t* ids, int64_t n, int64_t threshold, uint8_t* keep, int64_t* count,
                    int64_t* nkept) {
    int rc = traj_begin(ctx, n, ids && keep && nkept);
    if (rc || !nkept) return rc ? rc : GT_ERR_ARG;
    *nkept = 0;
    if (n == 0) return GT_OK;
    return traj_filter_stubs(ids, n, threshold, keep, count, nkept, ctx->stream, ctx->num_sms, &ctx->err);
}

int gt_steps(gt_ctx* ctx, const int64_t* ids, const float* x, const float* y, int64_t n, double mpp, float* xs,
             float* ys, double* x_step, double* y_step, double* steplength, int64_t* order) {
    int rc = traj_begin(ctx, n, ids && x && y && xs && ys && x_step && y_step && steplength && order);
    if (rc) return rc;
    if (n == 0) return GT_OK;
    return traj_steps(ids, x, y, n, (float)mpp, xs, ys, x_step, y_step, steplength, order, ctx->stream,
                      ctx->num_sms, &ctx->err);
}

int gt_imsd(gt_ctx* ctx, const int64_t* ids, const int64_t* frames, const float* x, const float* y, int64_t n,
            double mpp, int64_t max_lagtime, gt_table* out) {
    if (!out) return GT_ERR_ARG;
    out->data = nullptr;
    out->nrows = 0;
    out->ncols = 0;
    int rc = traj_begin(ctx, n, ids && frames && x && y);
    if (rc) return rc;
    float* data = nullptr;
    int64_t m = 0;
    float ms = 0.f;
    if (n > 0) {
        rc = traj_imsd(ids, frames, x, y, n, (float)mpp, max_lagtime, table_alloc, &data, &m, &ms, ctx->stream,
                       ctx->num_sms, &ctx->err);
        if (rc) {
            if (data) table_release(data);
            return rc;
        }
    } else {
        data = table_alloc(sizeof(float) * 3);
        if (!data) { ctx->err = "host allocation failed"; return GT_ERR_OOM; }
    }
    ctx->stats.ms_msd = ms;
    out->data = data;
    out->nrows = m;
    out->ncols = 3;
    std::memset(out->names, 0, sizeof(out->names));
    std::memset(out->types, 0, sizeof(out->types));
    const char* names[3] = {"lag", "particle", "msd"};
    for (int i = 0; i < 3; ++i) {
        std::snprintf(out->names[i], sizeof(out->names[i]), "%s", names[i]);
        std::snprintf(out->types[i], sizeof(out->types[i]), "%s", i < 2 ? "int" : "float");
    }
    return GT_OK;
}

int gt_last_stats(const gt_ctx* ctx, gt_stats* out) {
    if (!ctx || !out) return GT_ERR_ARG;
    *out = ctx->stats;
    return GT_OK;
}

int gt_link(gt_ctx* ctx, const float* rows, int64_t n, int ncols, float search_range, int has_memory,
            uint32_t memory, uint64_t* ids) {
    if (!ctx) return GT_ERR_ARG;
    ctx->err.clear();
    ctx->stats = gt_stats{};
    if ((!rows && n > 0) || ncols < 4 || n < 0 || (n > 0 && !ids)) { ctx->err = "invalid table"; return GT_ERR_ARG; }
    if (!(search_range > 0.0f && search_range < 4096.0f)) { ctx->err = "search_range must be in (0, 4096)"; return GT_ERR_ARG; }
    if (n == 0) return GT_OK;
    if (n > (1LL << 30)) { ctx->err = "table too large"; return GT_ERR_ARG; }
    const uint32_t mem = has_memory ? memory : 0;
    // FrameSubsetter (linking.rs:33-61): runs of equal column-0 values; the
    // iterator starts with cur_frame = 0, so a first value != 0 yields a
    // leading empty group.
    std::vector<int64_t> gstart;
    std::vector<int> gsize;
    {
        int64_t idx = 0;
        float cur = 0.0f;
        while (true) {
            int64_t s = idx;
            bool end = false;
            while (true) {
                if (idx >= n) { end = true; break; }
                const float fr = rows[idx * ncols];
                if (fr != cur) { cur = fr; break; }
                ++idx;
            }
            if (end && idx == s) break;
            gstart.push_back(s);
            gsize.push_back((int)(idx - s));
            if (end) break;
        }
    }
    const int T = (int)gstart.size();
    int maxg = 1;
    float ymin = 0.f, ymax = 1.f, xmin = 0.f, xmax = 1.f;
    bool first = true;
    for (int64_t i = 0; i < n; ++i) {
        const float y = rows[i * ncols + 2], x = rows[i * ncols + 3];
        if (!std::isfinite(y) || !std::isfinite(x)) { ctx->err = "non-finite position"; return GT_ERR_ARG; }
        if (first) { ymin = ymax = y; xmin = xmax = x; first = false; }
        ymin = std::min(ymin, y); ymax = std::max(ymax, y);
        xmin = std::min(xmin, x); xmax = std::max(xmax, x);
    }
    for (int g : gsize) maxg = std::max(maxg, g);
    CK(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    for (int scale = 1; scale <= 64; scale *= 4) {
        Plan P;
        P.T = T;
        P.link = 1;
        P.r = Resolved{};
        P.r.has_search_range = 1;
        P.r.search_range = search_range;
        P.r.memory = mem;
        P.cap_p = maxg;
        P.cap_m = (int)std::max<long long>(1, (long long)mem * P.cap_p);
        P.cap_s = P.cap_p + P.cap_m;
        P.cap_e = (int)std::min<long long>((long long)P.cap_s * std::min(16 * scale, P.cap_p), 1LL << 30);
        // grid over the positions' bounding box, shifted to start at 0
        // cells of absolute positions; negative coordinates clamp into the
        // first cell (clamping is monotone, so neighbours stay adjacent)
        const double ext = std::max({(double)ymax, (double)xmax, 0.0}) + 1.0;
        P.G = std::max({(int)std::ceil(search_range) + 1, 8, (int)std::ceil(ext / 128.0)});
        P.ncy = (int)(std::max(ymax, 0.0f) / P.G) + 1;
        P.ncx = (int)(std::max(xmax, 0.0f) / P.G) + 1;
        (void)ymin; (void)xmin;
        P.hsize = 2 * next_pow2(2LL * std::max({P.cap_p, P.cap_m, 32}));
        const size_t nn = (size_t)P.cap_s + P.cap_p;
        const size_t per_slot = 4 * (3 * (size_t)P.cap_s + 1) + 8 * (size_t)P.cap_e * 2 +
                                4 * ((size_t)P.cap_p + 1) + 4 * 4 * nn + nn + 16 * nn + 4 + 8 * (size_t)P.hsize;
        P.nslot = (int)std::max<size_t>(1, std::min<size_t>({(size_t)T, (size_t)ctx->num_sms * 4,
                                                             ((size_t)6 << 30) / per_slot}));
        P.cap_c = 1;
        Work w{};
        const size_t need = carve(P, nullptr, &w, 0, false);
        int rc = ensure_arena(ctx, need);
        if (rc) return rc;
        carve(P, ctx->arena, &w, 0, false);
        // particle slabs, positions shifted so the grid starts at the origin
        std::vector<float> hy((size_t)T * P.cap_p, 0.f), hx((size_t)T * P.cap_p, 0.f);
        for (int t = 0; t < T; ++t)
            for (int i = 0; i < gsize[t]; ++i) {
                const int64_t rr = gstart[t] + i;
                hy[(size_t)t * P.cap_p + i] = rows[rr * ncols + 2];
                hx[(size_t)t * P.cap_p + i] = rows[rr * ncols + 3];
            }
        CK(cudaMemcpyAsync(w.py, hy.data(), sizeof(float) * hy.size(), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(w.px, hx.data(), sizeof(float) * hx.size(), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(w.npart, gsize.data(), sizeof(int) * T, cudaMemcpyHostToDevice, st));
        CK(cudaMemsetAsync(w.err, 0, sizeof(int) * 4, st));
        CK(cudaFuncSetAttribute(grid_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(sizeof(int) * (size_t)P.ncx * P.ncy)));
        grid_kernel<<<T, 512, sizeof(int) * (size_t)P.ncx * P.ncy, st>>>(w.py, w.px, w.npart, P.cap_p, P.G,
                                                                        P.ncy, P.ncx, w.gstart, w.gidx);
        CK(cudaGetLastError());
        scan_frames_kernel<<<1, 1024, 0, st>>>(w.npart, w.off, T);
        rc = run_link(ctx, P, w, st);
        if (rc) return rc;
        // ids in row order: compact index g == row index
        std::vector<int> root(n), newid(n);
        CK(cudaMemcpyAsync(root.data(), w.root, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(newid.data(), w.newid, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
        int bits = 0;
        CK(cudaMemcpyAsync(&bits, w.err, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        bool retry;
        rc = err_status(ctx, bits, &retry);
        if (rc && retry && scale < 64) continue;
        if (rc) return rc;
        for (int64_t i = 0; i < n; ++i) ids[i] = (uint64_t)newid[root[i]];
        ctx->stats.particles = n;
        return GT_OK;
    }
    return GT_ERR_CAPACITY;
}

}  // extern "C"
