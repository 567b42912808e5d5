// noalloc.cu -- gt_locate_frame_static: locate one device-resident frame
// without allocating any memory.
//
// For callers that must not allocate device memory: hosts whose device
// memory is fully owned by another framework's pool (a cudaMalloc beside it
// can fail or fragment it), and real-time acquisition loops that forbid
// allocation after start-up (an allocation can stall on the driver).  The
// caller passes the frame and the output buffer; every other byte the call
// needs lives in one file-scope __device__ array of kScratchBytes, which
// each GPU that loads the library keeps until the process exits.  The call
// waits for its own work on the caller's stream and reads its row count
// back to the host.
//
// The kernels are the ones gt_batch_device launches for the same frame
// (locate, fallback walk, ordering and separation filter, output rows);
// linking needs several frames and is not offered here.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <climits>
#include <cstring>
#include <mutex>

#include "gt.h"
#include "gt_internal.cuh"

namespace gt {
__global__ void locate_tiles_kernel(const LocParams p, const MovieBufs b, int frame0);
__global__ void fallback_walk_kernel(const LocParams p, const MovieBufs b, int win, const int* pbeg);
__global__ void finalize_kernel(const LocParams p, MovieBufs b, float sep, int link_grid, int frame0);
__global__ void scan_frames_kernel(const int* in, int* out, int n);
__global__ void assemble_kernel(AsmArgs a);
bool fast_supported(int kr, int dd, int rc, int diameter);
cudaError_t launch_locate_fast(int kr, int dd, int rc, int th, dim3 grid, cudaStream_t st, const LocParams& p,
                               const MovieBufs& b, int T, int frame0, int* used_tma);
void gauss_taps(int smoothing_size, float noise_size, int normalized, float* w, float* norm, float* rn);
void set_noctx_error(const char* msg);
}  // namespace gt

using namespace gt;

namespace {

constexpr size_t kScratchBytes = (size_t)16 << 20;  // 16 MiB per device
constexpr int kMaxPixels = 1 << 20;                 // frames up to 2^20 pixels
constexpr int kMaxSide = 8192;
constexpr int kMaxCand = 32768;                     // features per frame before filtering
constexpr int kMaxCircle = 3200;                    // stencil entries (radius <= 31)
constexpr int kMaxDevices = 64;

// The shared scratch of every call on this device.  Host code must not take
// its address directly (that is a host-side stand-in); the device address
// comes from cudaGetSymbolAddress at set-up.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

struct DeviceState {
    bool ready = false;
    unsigned char* scratch = nullptr;  // device address of g_scratch
    int num_sms = 0;
};

DeviceState g_dev[kMaxDevices];
std::mutex g_dev_mutex;  // guards the one-time set-up of each device

// Messages go to the calling thread's context-free error (gt_last_error(NULL)).
int fail(int status, const char* msg) {
    set_noctx_error(msg);
    return status;
}

#define SCK(x)                                                                    \
    do {                                                                          \
        cudaError_t e_ = (x);                                                     \
        if (e_ != cudaSuccess) {                                                  \
            char m_[256];                                                         \
            std::snprintf(m_, sizeof(m_), "%s: %s", #x, cudaGetErrorString(e_));  \
            set_noctx_error(m_);                                                  \
            return GT_ERR_CUDA;                                                   \
        }                                                                         \
    } while (0)

// Stencil tables as in the batch path (kernels.rs:134-206), into fixed arrays.
int circle_tab(int R, float* tab3, int* off, float* tab2) {
    int k = 0;
    for (int i = -R; i <= R; ++i)
        for (int j = -R; j <= R; ++j)
            if (i * i + j * j <= R * R) {
                const float th = std::atan2((float)j, (float)i);
                if (tab3) {
                    tab3[3 * k] = (float)(i * i + j * j);
                    tab3[3 * k + 1] = std::sin(2.0f * th);
                    tab3[3 * k + 2] = std::cos(2.0f * th);
                }
                if (tab2) {
                    tab2[2 * k] = std::sin(2.0f * th);
                    tab2[2 * k + 1] = std::cos(2.0f * th);
                }
                if (off) { off[2 * k] = i; off[2 * k + 1] = j; }
                ++k;
            }
    return k;
}

int circle_f(float radius, int* off) {
    const int rb = (int)std::ceil(radius);
    const float r2 = radius * radius;
    int k = 0;
    for (int i = -rb; i <= rb; ++i)
        for (int j = -rb; j <= rb; ++j)
            if ((float)(i * i + j * j) <= r2) { off[2 * k] = i; off[2 * k + 1] = j; ++k; }
    return k;
}

int annulus_f(float outer, float inner, int* off) {
    const int b = (int)std::ceil(outer);
    const float or2 = outer * outer, ir2 = inner * inner;
    int k = 0;
    for (int i = -b; i <= b; ++i)
        for (int j = -b; j <= b; ++j) {
            const float r2 = (float)(i * i + j * j);
            if (r2 <= or2 && r2 >= ir2) { off[2 * k] = i; off[2 * k + 1] = j; ++k; }
        }
    return k;
}

struct Carve {
    unsigned char* base;
    size_t off = 0;
    template <class X>
    X* take(size_t n) {
        off = (off + 255) / 256 * 256;
        X* p = (X*)(base + off);
        off += sizeof(X) * (n ? n : 1);
        return p;
    }
};

}  // namespace

extern "C" int gt_locate_frame_static(const void* d_frame, int dtype, int H, int W, const gt_params* pr,
                                      float* d_out, int64_t out_rows, int64_t* nrows, void* stream) {
    set_noctx_error("");
    if (!d_frame || !pr || !nrows || (out_rows > 0 && !d_out)) return fail(GT_ERR_ARG, "null argument");
    if (dtype != GT_U16 && dtype != GT_F32) return fail(GT_ERR_ARG, "dtype must be GT_U16 or GT_F32");
    if (H < 1 || W < 1 || H > kMaxSide || W > kMaxSide || (long long)H * W > kMaxPixels)
        return fail(GT_ERR_ARG, "frame larger than the static scratch allows (H*W <= 1048576, H, W <= 8192)");
    // gpu_tracking defaults (lib.rs:77-91) and the options the reference rejects
    if (pr->has_maxsize || pr->has_threshold || pr->has_invert || pr->has_percentile || pr->has_topn ||
        pr->has_preprocess)
        return fail(GT_ERR_UNSUPPORTED, "maxsize/threshold/invert/percentile/topn/preprocess are not implemented");
    if (pr->has_search_range) return fail(GT_ERR_ARG, "linking needs several frames: use gt_batch_device");
    const int d = (int)pr->diameter;
    const int k = pr->has_smoothing_size ? (int)pr->smoothing_size : d;
    const unsigned sep = pr->has_separation ? pr->separation : pr->diameter + 1;
    const float noise = pr->has_noise_size ? pr->noise_size : 1.0f;
    const int max_iter = pr->has_max_iterations ? (int)pr->max_iterations : 10;
    const int cpu_processed = pr->has_cpu_processed ? (pr->cpu_processed != 0) : 0;
    const int characterize = pr->has_characterize ? (pr->characterize != 0) : 0;
    const int sig = pr->has_sig_radius, bg = pr->has_bg_radius;
    const float gap = pr->has_gap_radius ? pr->gap_radius : 0.0f;
    if (bg && !sig) return fail(GT_ERR_ARG, "bg_radius requires sig_radius");
    if (d > 63 || k < 1 || k / 2 * 2 + 1 > GT_MAX_TAPS || sep > 4096)
        return fail(GT_ERR_ARG, "diameter <= 63, smoothing_size in [1, 63], separation <= 4096");
    if ((sig && !(pr->sig_radius >= 0.f && pr->sig_radius <= 31.f)) ||
        (bg && !(pr->bg_radius >= 0.f && pr->bg_radius <= 31.f)))
        return fail(GT_ERR_ARG, "sig_radius and bg_radius must be in [0, 31]");

    int dev = 0;
    SCK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(GT_ERR_ARG, "device index out of range");
    DeviceState ds;
    {
        std::lock_guard<std::mutex> lock(g_dev_mutex);
        DeviceState& gd = g_dev[dev];
        if (!gd.ready) {
            // once per device, with it current: the device address of the scratch
            void* ptr = nullptr;
            SCK(cudaGetSymbolAddress(&ptr, g_scratch));
            SCK(cudaDeviceGetAttribute(&gd.num_sms, cudaDevAttrMultiProcessorCount, dev));
            gd.scratch = (unsigned char*)ptr;
            gd.ready = true;
        }
        ds = gd;
    }
    cudaStream_t st = (cudaStream_t)stream;

    // parameters (gpu_setup.rs:45-60), as the batch path derives them
    LocParams lp;
    std::memset(&lp, 0, sizeof(lp));
    lp.H = H; lp.W = W;
    lp.krad = k / 2;
    lp.taps = 2 * lp.krad + 1;
    if (H <= lp.krad || W <= lp.krad) return fail(GT_ERR_ARG, "frame smaller than the smoothing window");
    gauss_taps(k, noise, 0, lp.w, &lp.norm, &lp.rn);
    lp.kk = (float)(k * k);
    lp.rkk = 1.0f / lp.kk;
    {
        const float v = (2.0f * (float)sep) / std::sqrt(2.0f);
        const unsigned dd = v <= 0.0f ? 0u : (unsigned)v;
        lp.D = (int)dd;
        lp.o = (int)((float)(int)dd / 2.0f - 0.5f);
    }
    lp.d = d;
    lp.rint_c = (d - 1) / 2;
    lp.border = d / 2;
    lp.char_r = d / 2;
    lp.max_iter = max_iter;
    lp.thr = 0.6f;
    lp.minmass = pr->has_minmass ? pr->minmass : 0.0f;
    lp.hp = std::max({lp.o, lp.D - 1 - lp.o, lp.char_r, lp.rint_c + 2, 1});
    lp.dtype = dtype;
    lp.cpu_processed = cpu_processed;
    lp.characterize = characterize;
    lp.zero_skip = lp.max_iter >= 1 && lp.rint_c <= lp.o && lp.rint_c <= lp.D - 1 - lp.o;
    lp.tma_spin = 1 << 22;

    // host staging of the stencil tables, one set per calling thread
    thread_local float char_tab[3 * kMaxCircle], gchar_tab[2 * kMaxCircle];
    thread_local int char_off[2 * kMaxCircle], sig_off[2 * kMaxCircle], bg_off[2 * kMaxCircle];
    lp.n_char = circle_tab(lp.char_r, char_tab, char_off, nullptr);
    lp.n_gchar = circle_tab(lp.rint_c, nullptr, nullptr, gchar_tab);
    const int n_sig = sig ? circle_f(pr->sig_radius, sig_off) : 0;
    const int n_bg = bg ? annulus_f(pr->bg_radius, pr->sig_radius + gap, bg_off) : 0;

    const bool fast = dtype == GT_U16 && fast_supported(lp.krad, lp.D, lp.rint_c, lp.d);
    const int th = fast ? 64 : 32;
    lp.TH = th;
    lp.TW = 64;
    lp.ntx = (W + 63) / 64;
    lp.nty = (H + th - 1) / th;
    const int ncols = 4 + (cpu_processed ? 3 : 0) + (sig ? 1 : 0) + (bg ? 2 : 0) + (characterize ? 4 : 0);
    const int cap_c = std::min(H * W, kMaxCand);
    const int G = std::max({(int)sep + 1, 8, (int)std::ceil(std::sqrt((double)H * W / 16384.0))});
    const int ncy = (H + G - 1) / G, ncx = (W + G - 1) / G;
    const int ncell = ncx * ncy;

    // carve the scratch
    Carve c{ds.scratch};
    MovieBufs b;
    std::memset(&b, 0, sizeof(b));
    b.frames = d_frame;
    b.T = 1;
    b.cap_c = cap_c; b.cap_p = cap_c; b.cap_m = 1; b.cap_e = 1;
    b.cand = c.take<Cand>(cap_c);
    b.fcount = c.take<int>(1);
    b.rowcnt = c.take<int>((size_t)H * lp.ntx);
    b.pend = c.take<int>(cap_c);
    b.npend = c.take<int>(1);
    b.py = c.take<float>(cap_c);
    b.px = c.take<float>(cap_c);
    b.pm = c.take<float>(cap_c);
    b.prec = c.take<int>(cap_c);
    b.npart = c.take<int>(1);
    b.G = G; b.ncx = ncx; b.ncy = ncy;
    b.gstart = c.take<int>(ncell + 1);
    b.gidx = c.take<int>(cap_c);
    b.cperm = c.take<int>(cap_c);
    b.cy = c.take<float>(cap_c);
    b.cx = c.take<float>(cap_c);
    b.cm = c.take<float>(cap_c);
    b.crec = c.take<int>(cap_c);
    b.ccell = c.take<int>(cap_c);
    b.cstart = c.take<int>(ncell + 1);
    b.cidx = c.take<int>(cap_c);
    float* d_char_tab = c.take<float>(3 * lp.n_char);
    int* d_char_off = c.take<int>(2 * lp.n_char);
    float* d_gchar_tab = c.take<float>(2 * lp.n_gchar);
    int* d_sig_off = c.take<int>(2 * n_sig);
    int* d_bg_off = c.take<int>(2 * n_bg);
    b.char_tab = d_char_tab;
    b.char_off = d_char_off;
    b.gchar_tab = d_gchar_tab;
    b.err = c.take<int>(4);
    int* off = c.take<int>(2);
    float* stage = c.take<float>((size_t)cap_c * ncols);
    if (c.off > kScratchBytes) return fail(GT_ERR_ARG, "parameters need more than the 16 MiB static scratch");

    // every call starts from cleared counters (the scratch keeps the last
    // call's contents)
    SCK(cudaMemsetAsync(b.fcount, 0, sizeof(int), st));
    SCK(cudaMemsetAsync(b.npend, 0, sizeof(int), st));
    SCK(cudaMemsetAsync(b.err, 0, 4 * sizeof(int), st));
    SCK(cudaMemcpyAsync(d_char_tab, char_tab, sizeof(float) * 3 * lp.n_char, cudaMemcpyHostToDevice, st));
    SCK(cudaMemcpyAsync(d_char_off, char_off, sizeof(int) * 2 * lp.n_char, cudaMemcpyHostToDevice, st));
    SCK(cudaMemcpyAsync(d_gchar_tab, gchar_tab, sizeof(float) * 2 * lp.n_gchar, cudaMemcpyHostToDevice, st));
    if (n_sig) SCK(cudaMemcpyAsync(d_sig_off, sig_off, sizeof(int) * 2 * n_sig, cudaMemcpyHostToDevice, st));
    if (n_bg) SCK(cudaMemcpyAsync(d_bg_off, bg_off, sizeof(int) * 2 * n_bg, cudaMemcpyHostToDevice, st));

    if (fast) {
        int used_tma = 0;
        SCK(launch_locate_fast(lp.krad, lp.D, lp.rint_c, 64, dim3(lp.ntx * lp.nty, 1), st, lp, b, 1, 0, &used_tma));
    } else {
        const int PH = 32 + 2 * lp.hp, PW = 64 + 2 * lp.hp;
        const int RH = PH + 2 * lp.krad, RW = PW + 2 * lp.krad;
        size_t smem = sizeof(float) * ((size_t)RH * RW + 2 * (size_t)RH * PW + (size_t)PH * PW) +
                      sizeof(int) * 32 * 64 + 6 * sizeof(float) * 512 + 32 * 64;
        smem = (smem + 15) / 16 * 16;
        if (smem > 227 * 1024) return fail(GT_ERR_ARG, "diameter/separation too large for the tile plan");
        SCK(cudaFuncSetAttribute(locate_tiles_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        locate_tiles_kernel<<<dim3(lp.ntx * lp.nty, 1), 256, smem, st>>>(lp, b, 0);
        SCK(cudaGetLastError());
    }
    const int fb_win = std::min(100, std::max(lp.rint_c + 1, lp.max_iter - 1 + lp.rint_c + 1));
    const size_t smem_fb = sizeof(float) * (size_t)(2 * fb_win + 1) * (2 * fb_win + 1);
    SCK(cudaFuncSetAttribute(fallback_walk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_fb));
    fallback_walk_kernel<<<ds.num_sms * 4, 128, smem_fb, st>>>(lp, b, fb_win, nullptr);
    SCK(cudaGetLastError());
    SCK(cudaFuncSetAttribute(finalize_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(4 * ncell)));
    finalize_kernel<<<1, 512, 4 * ncell, st>>>(lp, b, (float)sep, 0, 0);
    scan_frames_kernel<<<1, 1024, 0, st>>>(b.npart, off, 1);
    AsmArgs a;
    std::memset(&a, 0, sizeof(a));
    a.T = 1; a.H = H; a.W = W; a.cap_p = cap_c; a.cap_c = cap_c; a.ncols = ncols;
    a.has_link = 0; a.cpu_processed = cpu_processed; a.characterize = characterize; a.sig = sig; a.bg = bg;
    a.frames = d_frame; a.dtype = dtype;
    a.py = b.py; a.px = b.px; a.pm = b.pm; a.prec = b.prec; a.npart = b.npart; a.off = off; a.cand = b.cand;
    a.root = b.npart; a.newid = b.npart;  // unused without linking
    a.sig_off = d_sig_off; a.n_sig = n_sig; a.bg_off = d_bg_off; a.n_bg = n_bg;
    a.out = stage;
    a.out_rows = LLONG_MAX;
    assemble_kernel<<<1, 256, 0, st>>>(a);
    SCK(cudaGetLastError());
    int hb[2] = {0, 0};
    SCK(cudaMemcpyAsync(&hb[0], b.err, sizeof(int), cudaMemcpyDeviceToHost, st));
    SCK(cudaMemcpyAsync(&hb[1], off + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    SCK(cudaStreamSynchronize(st));
    if (hb[0] & ERR_DEVICE_TIMEOUT) return fail(GT_ERR_DEVICE_TIMEOUT, "a bounded device wait expired");
    if (hb[0]) return fail(GT_ERR_CAPACITY, "more features than the static scratch holds (32768 per frame)");
    *nrows = hb[1];
    const int64_t n = std::min<int64_t>(hb[1], out_rows);
    if (n > 0) {
        SCK(cudaMemcpyAsync(d_out, stage, sizeof(float) * (size_t)n * ncols, cudaMemcpyDeviceToDevice, st));
        SCK(cudaStreamSynchronize(st));
    }
    return GT_OK;
}
