// assemble.cu -- frame offsets, trajectory IDs and the output table.
//
// The output table has the reference's column layout (execute_gpu.rs:197-226,
// rows written at 337-368): frame, mass, y, x, [particle], [Rg, ecc, signal],
// [raw_mass], [raw_bg_median, raw_mass_corrected], [Rg_gpu, raw_mass_gpu,
// signal_gpu, ecc_gpu], all f32, frames ascending, particles of a frame in
// raster order of their originating pixel.
#include <math_constants.h>
#include "gt_device.cuh"

namespace gt {



// Exclusive scan of n ints into out[0..n] by one CTA of 1024 threads.
__global__ void __launch_bounds__(1024) scan_frames_kernel(const int* in, int* out, int n) {
    __shared__ int warp_tot[32];
    __shared__ int s_total;
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int b0 = 0; b0 < n; b0 += 1024) {
        const int i = b0 + threadIdx.x;
        const int v = i < n ? in[i] : 0;
        const int e = block_excl_scan<1024>(v, warp_tot, &s_total);
        if (i < n) out[i] = carry + e;
        __syncthreads();
        if (threadIdx.x == 0) carry += s_total;
        __syncthreads();
    }
    if (threadIdx.x == 0) out[n] = carry;
}

// Continues the exclusive scan of in[] into out[] over [f0, f0 + n): out[f0]
// holds the prefix of the earlier frames (0 when f0 = 0); writes
// out[f0 + 1 .. f0 + n].
__global__ void __launch_bounds__(1024) scan_frames_from_kernel(const int* in, int* out, int f0, int n) {
    __shared__ int warp_tot[32];
    __shared__ int s_total;
    __shared__ int carry;
    if (threadIdx.x == 0) carry = f0 > 0 ? out[f0] : 0;
    __syncthreads();
    for (int b0 = 0; b0 < n; b0 += 1024) {
        const int i = b0 + threadIdx.x;
        const int v = i < n ? in[f0 + i] : 0;
        const int e = block_excl_scan<1024>(v, warp_tot, &s_total);
        if (i < n) out[f0 + i] = carry + e;
        __syncthreads();
        if (threadIdx.x == 0) carry += s_total;
        __syncthreads();
    }
    if (threadIdx.x == 0) out[f0 + n] = carry;
}

// newid[g] for particles that start a trajectory: running counter in
// (frame, index) order (linking.rs:470).
__global__ void newid_kernel(const int* newrank, const int* newbase, const int* off, const int* npart,
                             int* newid, int T) {
    const int t = blockIdx.x;
    if (t >= T) return;
    const int n = npart[t];
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int g = off[t] + i;
        const int r = newrank[g];
        newid[g] = r >= 0 ? newbase[t] + r : -1;
    }
}

namespace {
__device__ __forceinline__ float raw_at(const AsmArgs& a, size_t fbase, int r, int c) {
    if (r < 0 || r >= a.H || c < 0 || c >= a.W) return CUDART_NAN_F;
    return load_px(a.frames, a.dtype, fbase + (size_t)r * a.W + c);
}
}  // namespace

__global__ void assemble_kernel(AsmArgs a) {
    const int t = blockIdx.x;
    if (t >= a.T) return;
    const int n = a.npart[t];
    const size_t fbase = (size_t)t * a.H * a.W;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int g = a.off[t] + i;
        if (g >= a.out_rows) break;  // rows in index order: the rest are beyond too
        const size_t s = (size_t)t * a.cap_p + i;
        float* row = a.out + (size_t)g * a.ncols;
        const float mass = a.pm[s];
        const float y = a.py[s], x = a.px[s];
        int c = 0;
        row[c++] = (float)t;
        row[c++] = mass;
        row[c++] = y;
        row[c++] = x;
        if (a.has_link) row[c++] = (float)a.newid[a.root[g]];
        const Cand& rec = a.cand[(size_t)t * a.cap_c + a.prec[s]];
        if (a.walk && g < a.walk_rows) {
            int* wr = a.walk + (size_t)g * 5;
            wr[0] = t; wr[1] = rec.ul; wr[2] = rec.vl; wr[3] = rec.up; wr[4] = rec.vp;
        }
        if (a.cpu_processed) {
            // execute_gpu.rs:349-351
            row[c++] = sqrtf(rec.rg_sum / mass);
            row[c++] = rec.eccn / (mass - rec.mid);
            row[c++] = rec.signal;
        }
        if (a.sig) {
            // execute_gpu.rs:311-331: rounded refined position, NaN outside
            const int mr = (int)roundf(y), mc = (int)roundf(x);
            float acc = 0.f;
            for (int q = 0; q < a.n_sig; ++q) {
                const float v = raw_at(a, fbase, mr + a.sig_off[2 * q], mc + a.sig_off[2 * q + 1]);
                if (!isnan(v)) acc = acc + v;
            }
            row[c++] = acc;
            if (a.bg) {
                // median with linear interpolation (ndarray-stats Linear, q=0.5):
                // order statistics by counting, NaN skipped
                int nv = 0;
                for (int q = 0; q < a.n_bg; ++q)
                    nv += !isnan(raw_at(a, fbase, mr + a.bg_off[2 * q], mc + a.bg_off[2 * q + 1]));
                float med = CUDART_NAN_F;
                if (nv > 0) {
                    const int lo = (nv - 1) / 2, hi = nv / 2;
                    float vlo = 0.f, vhi = 0.f;
                    for (int q = 0; q < a.n_bg; ++q) {
                        const float v = raw_at(a, fbase, mr + a.bg_off[2 * q], mc + a.bg_off[2 * q + 1]);
                        if (isnan(v)) continue;
                        int less = 0, leq = 0;
                        for (int z = 0; z < a.n_bg; ++z) {
                            const float w = raw_at(a, fbase, mr + a.bg_off[2 * z], mc + a.bg_off[2 * z + 1]);
                            if (isnan(w)) continue;
                            less += (w < v);
                            leq += (w <= v);
                        }
                        // v occupies sorted positions [less, leq)
                        if (lo >= less && lo < leq) vlo = v;
                        if (hi >= less && hi < leq) vhi = v;
                    }
                    const double frac = (hi == lo) ? 0.0 : 0.5;
                    med = vlo + (float)(frac * ((double)vhi - (double)vlo));
                }
                row[c++] = med;
                row[c++] = acc - med * (float)a.n_sig;
            }
        }
        if (a.characterize) {
            row[c++] = rec.g_rg;
            row[c++] = rec.g_raw;
            row[c++] = rec.g_sig;
            row[c++] = rec.g_ecc;
        }
    }
}

}  // namespace gt
