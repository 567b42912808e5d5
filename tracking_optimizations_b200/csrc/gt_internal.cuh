// gt_internal.cuh -- device-side types shared by the locate, finalize and link
// kernels of the B200 gpu_tracking path.
//
// Data layout in HBM (one movie = T frames of H x W pixels, row-major):
//   frames     u16 or f32, T*H*W                    (input, read once)
//   cand       Cand records, T*cap_c                (per-frame slab, unordered)
//   fcount     int, T                               (records per frame)
//   rowcnt     int, T*H*ntx                         (records per (row, tile column))
//   part_*     y, x, mass, rec: T*cap_p             (survivors, raster order)
//   npart      int, T
//   grid_*     cell starts (T*(ncell+1)) and indices (T*cap_p) for linking
//   pred       int, T*cap_p  (global index of the linked source, -1 = new)
#pragma once
#include <cstdint>

#define GT_MAX_TAPS 64
#define GT_MAX_CIRCLE 1024

namespace gt {

// Derived per-movie parameters (gpu_setup.rs:45-60 plus the tile plan).
struct LocParams {
    int H, W;
    int taps, krad;             // smoothing window: taps = 2*krad + 1
    float w[GT_MAX_TAPS];       // exp(-i^2 / (2 * noise_size)), i = -krad..krad
                                // (divided by norm when the taps are normalised on the host)
    float norm;                 // sum of the exp() taps in order
    float kk;                   // f32(smoothing_size^2), the boxcar divisor
    float rn;                   // RN(1 / norm), or 1 with host-normalised taps
    float rkk;                  // RN(1 / kk)
    int D, o;                   // dilation size and window offset
    int d, rint_c, border;      // diameter, centroid radius (d-1)/2, border d/2
    int char_r;                 // cpu_processed circle radius d/2
    int max_iter;
    float thr, minmass;
    int hp;                     // processed halo of a tile
    int TH, TW, ntx, nty;       // tile shape and tile counts
    int dtype;                  // 0 = u16, 1 = f32
    int cpu_processed, characterize;
    int zero_skip;              // zero-valued maxima provably have zero mass
    int n_char;                 // entries of the d/2 circle table
    int n_gchar;                // entries of the (d-1)/2 circle table
    int tma_spin;               // iteration limit of the bounded wait for a staged tile
    int tma_withhold;           // test switch: issue no tile copy, so the wait runs out
    int tiles_per_cta;          // specialised kernel: tiles per CTA (0 = chosen per launch)
};

// One located feature, keyed by its originating pixel (walk_cols.wgsl:87-91).
struct __align__(16) Cand {
    int u, v;             // originating pixel
    float y, x, mass;     // walk result
    int rowrank;          // rank within its (row, tile column) segment
    int state;            // 0 emitted, 1 waiting for the fallback walk, 2 rejected
    float rg_sum;         // cpu_processed pieces at the originating pixel
    float eccn;           // sqrt(sin_sum^2 + cos_sum^2)
    float mid;            // processed value at the originating pixel
    float signal;
    float g_rg, g_raw, g_sig, g_ecc;   // characterize=True columns
    int ul, vl;           // pixel of the walk's last centroid read
    int up, vp;           // walk's final position (differs when the walk ran out)
    int pad;
};

enum CandState { CAND_EMIT = 0, CAND_PENDING = 1, CAND_REJECT = 2 };

// Error word bits written by kernels (never a trap).
enum ErrBits {
    ERR_CAND_OVERFLOW = 1,
    ERR_PART_OVERFLOW = 2,
    ERR_EDGE_OVERFLOW = 4,
    ERR_SUBNET_BUDGET = 8,
    ERR_MEM_OVERFLOW = 16,
    ERR_SCRATCH_OVERFLOW = 32,
    ERR_DEVICE_TIMEOUT = 64,
};

// Per-movie device buffers and capacities.
struct MovieBufs {
    const void* frames;
    int T;
    int cap_c, cap_p, cap_m, cap_e;
    Cand* cand;
    int* fcount;
    int* rowcnt;
    int* pend;            // fallback list: frame*cap_c + slot
    int* npend;
    float* py;
    float* px;
    float* pm;
    int* prec;
    int* npart;
    int G, ncx, ncy;      // link/separation grid: cell size and counts
    int* gstart;          // T*(ncx*ncy+1)
    int* gidx;            // T*cap_p
    int* cperm;           // T*cap_c finalize scratch (raster permutation)
    float* cy;            // T*cap_c emitted candidates in raster order
    float* cx;
    float* cm;
    int* crec;
    int* ccell;           // T*cap_c
    int* cstart;          // T*(ncx*ncy+1) separation grid starts
    int* cidx;            // T*cap_c
    const float* char_tab;   // n_char x {r2, sin2, cos2}, d/2 circle
    const int* char_off;     // n_char x {di, dj}
    const float* gchar_tab;  // n_gchar x {sin2, cos2}, (d-1)/2 circle
    int* err;
};

struct LinkBufs {
    int T, cap_p, cap_m, cap_e, cap_s;
    int tb, te;           // frames linked by this launch; earlier frames are final
    float r;              // search range
    int G, ncx, ncy;
    const float* py;
    const float* px;
    const int* npart;
    const int* off;       // exclusive prefix of npart (compact particle index)
    const int* gstart;
    const int* gidx;
    int* pred;            // compact index of the linked source, -1 = new
    unsigned char* lnext; // slab: particle linked by the next frame
    int* mlist;           // T*cap_m slab handles
    int* mcount;          // T
    int* dirty;           // T
    int* ndirty;
    int* newrank;         // compact: rank among new particles of its frame
    int* newcount;        // T
    int* root;            // compact
    int* lroot;           // compact: where the pred chain enters the particle's chunk
    int* err;
    long long budget;     // branch-and-bound option trials per subnet
    // per-CTA scratch, `nslot` slots of these sizes
    int nslot;
    float* s_y;           // cap_s
    float* s_x;
    int* s_h;             // slab handle of each source
    int* s_deg;           // cap_s + 1
    int* e_dst;           // cap_e
    float* e_w;
    int* d_cnt;           // cap_p + 1
    int* d_src;           // cap_e
    float* d_w;
    int* uf;              // cap_s + cap_p
    int* c_nd;            // cap_s + cap_p
    int* c_ns;
    int* c_min;
    unsigned char* vis;   // cap_s + cap_p
    int* work;            // 4 * (cap_s + cap_p): stacks, paths, choices
    int* bump;            // 1 per slot
    int* hkey;            // hash tables, hsize per slot
    int* hval;
    int hsize;
    int lsm_bytes;        // dynamic shared memory pool of the linker blocks
    // slot strides of the scratch arrays (>= the capacities above; equal to
    // the largest movie's when several movies share one pool)
    long long st_s, st_s1, st_p1, st_n, st_e, st_h;
};

// Adjoint of bandpass + refine at fixed peaks.  The forward arithmetic uses
// the same weights as LocParams; a / da are the real-valued normalised
// Gaussian taps w_i / sum(w) and their derivative with respect to
// noise_size (the Gaussian variance).
struct AdjParams {
    int T, H, W;
    int krad;                // smoothing half window
    int rc;                  // centroid circle radius, (diameter - 1) / 2
    int border;              // diameter / 2: centroids inside this band are zero
    int K;                   // circle pixel count
    float w[GT_MAX_TAPS];    // forward weights, as LocParams::w
    float norm, kk;          // forward normaliser and f32(k * k)
    float rn, rkk;           // their reciprocals, as LocParams
    float a[GT_MAX_TAPS];    // w_i / sum(w)
    float da[GT_MAX_TAPS];   // d a_i / d noise_size
    float k;                 // smoothing_size as a real number
    float gain, read_var;    // noise model of the uncertainty kernel
};

struct AsmArgs {
    int T, H, W, cap_p, cap_c, ncols;
    int has_link, cpu_processed, characterize, sig, bg;
    const void* frames;
    int dtype;
    const float* py;
    const float* px;
    const float* pm;
    const int* prec;
    const int* npart;
    const int* off;
    const Cand* cand;
    const int* root;
    const int* newid;
    const int* sig_off;   // n_sig x {di, dj}, circle_inds(sig_radius)
    int n_sig;
    const int* bg_off;    // n_bg x {di, dj}, annulus_inds
    int n_bg;
    float* out;
    long long out_rows;   // rows of `out` (rows beyond are not written)
    int* walk;            // optional n x 5 {frame, last-read row, col, final row, col}
    long long walk_rows;  // rows of `walk` (rows beyond are not written)
};

}  // namespace gt
