// Shared definitions for the pyfourier_b200 CUDA library (sm_100a).
//
// Axis convention inside the library: axis 0 is x (fastest in memory), then y,
// then z.  A grid plane of extent (nx, ny, nz) is stored as ((z*ny)+y)*nx+x.
// The public C-ABI takes per-axis parameters in the reference's (z, y, x)
// order and coordinates per sample in (x, y, z) order, as the reference does
// (src/pyfourier/_nufft/_plan.py:89-93).
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>
#include <stdint.h>

#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/pfb200.h"

namespace pfb {

constexpr int kMaxDim = 3;
constexpr int kMaxWidth = 8;

// Status plumbing: every C entry point returns a PFB_* code and records a
// human-readable message retrievable with pfb_last_error().
void set_error(const std::string &msg);
int fail(int code, const std::string &msg);

#define PFB_CUDA_TRY(expr)                                                                  \
    do {                                                                                    \
        cudaError_t _e = (expr);                                                            \
        if (_e != cudaSuccess)                                                              \
            return ::pfb::fail(PFB_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
    } while (0)

#define PFB_CUFFT_TRY(expr)                                                                 \
    do {                                                                                    \
        cufftResult _r = (expr);                                                            \
        if (_r != CUFFT_SUCCESS)                                                            \
            return ::pfb::fail(PFB_ERR_CUFFT, std::string(#expr) + ": cufft status " + std::to_string((int)_r)); \
    } while (0)

#define PFB_CHECK_LAUNCH() PFB_CUDA_TRY(cudaGetLastError())

// Raise a kernel's dynamic shared-memory limit to at least `bytes` on the current
// device.  The attribute stays with the context, so each (kernel, device) pays the
// driver call once; later launches only look it up.
int raise_smem_limit(const void *kernel, size_t bytes);
#define PFB_RAISE_SMEM(kernel, bytes) PFB_TRY_ST_RAISE(::pfb::raise_smem_limit((const void *)(kernel), (size_t)(bytes)))
#define PFB_TRY_ST_RAISE(expr)        \
    do {                               \
        int _st = (expr);              \
        if (_st) return _st;           \
    } while (0)

// Per-axis geometry, x-first.
struct Geom {
    int ndim;
    int n[kMaxDim];      // image extent N
    int nos[kMaxDim];    // oversampled grid extent ceil(osf * N)
    int w[kMaxDim];      // kernel width (1 on Cartesian axes)
    int cart[kMaxDim];   // 1 if the axis is Cartesian (integer positions, width 1)
    float beta[kMaxDim]; // Kaiser-Bessel beta
    int tile[kMaxDim];   // bin / tile extent for the spread
    int toff[kMaxDim];   // tile offset: tile t covers [t * tile - toff, (t + 1) * tile - toff) clipped to the grid
    int nbins[kMaxDim];  // ceil((nos + toff) / tile)
    int sh[kMaxDim];     // index shift folding fftshift into the grid layout (nos / 2)
    int64_t gvol;        // prod(nos)
    int64_t nvol;        // prod(n)
};

// First grid index and extent of tile tc along axis a.  Tiles start at
// tc * tile - toff, so when toff > 0 the first tile is toff points narrower and
// the remainder of the grid extent goes to the last tile.
__host__ __device__ __forceinline__ int tile_org(const Geom &g, int a, int tc) {
    const int o = tc * g.tile[a] - g.toff[a];
    return o > 0 ? o : 0;
}
__host__ __device__ __forceinline__ int tile_extent(const Geom &g, int a, int tc) {
    const int e = (tc + 1) * g.tile[a] - g.toff[a];
    return (e < g.nos[a] ? e : g.nos[a]) - tile_org(g, a, tc);
}

// Work item of the spread: a contiguous run of bin-sorted samples that all
// start (x0) inside one tile.  frame < 0 means samples of several frames.
struct SpreadItem {
    int begin, end, bin, frame;
};

// Work item of the owner-computes spread: output tile `tile` (of frame
// `frame`, or all frames when < 0) gathers the samples of its 2^d lower
// neighbour bins, virtual positions of their concatenation (item_stride /
// item_visits below).  atomic = the number of items when the tile is split
// over several (combined with float2 atomics after the tile was zeroed), else 0.
struct OwnerItem {
    int tile, frame, v0, v1, atomic;
};

// The visits of an owner item: v0, v0 + s, v0 + 2 s, ... below v1 with stride
// s = atomic when the tile is split over atomic > 1 items (item r of a split tile
// has v0 = r and v1 = the tile's visit count, so every item mixes all neighbour
// ranges and all blocks of the tile get work), else s = 1.
__host__ __device__ __forceinline__ int item_stride(const OwnerItem &it) { return it.atomic > 1 ? it.atomic : 1; }
__host__ __device__ __forceinline__ int item_visits(const OwnerItem &it) {
    const int s = item_stride(it);
    return it.v1 > it.v0 ? (it.v1 - it.v0 + s - 1) / s : 0;
}

// Arguments describing the "channels" of an apply: coils (B), subspace
// coefficients / frames (C), B0 segments (L).
struct ApplyDesc {
    int64_t batch;          // B
    int ncoeff;             // C: K with a basis, else number of frames F
    const float2 *basis;    // (F, K) complex64 or nullptr
    const float *weight;    // per-sample float32 (Mtot) or nullptr
    int nseg;               // L (>= 1)
    const float2 *b0_time;  // (L, readout) complex64 or nullptr
    const float2 *b0_space; // (L, prod(N)) complex64 or nullptr
    int norm;               // 0: none, 1: ortho
};

// One axis of the fused FFT: a mixed-radix Stockham factorisation of n and
// the offsets of each stage's twiddles exp(-2 pi i j q / (ns * radix)),
// j < ns, 1 <= q < radix, in a device table.
constexpr int kFftMaxStages = 16;
struct FftAxis {
    int n = 0, nst = 0;
    int radix[kFftMaxStages] = {};
    int ns[kFftMaxStages] = {};
    int twoff[kFftMaxStages] = {};
    unsigned magic[kFftMaxStages] = {};  // floor(i / ns) = umulhi(i, magic) for i < 2^16 (ns > 1)
    const float2 *tw = nullptr;
};

// Channels of an apply on the oversampled grids: nch channels per group
// (segment l, batch b, coefficient k with k fastest), ngrp groups (frames, or
// one group with a basis).
struct Chan {
    int nch;       // channels per group
    int ngrp;      // groups
    int B, L, K;   // batch, segments, coefficients (K = 0 without basis)
    int F;
};

}  // namespace pfb

// Opaque plan handle (declared in pfb200.h).
struct pfb_plan {
    int device = 0;
    pfb::Geom g{};
    int nframes = 1;
    int64_t mtot = 0;
    int readout = 1;
    double scale = 1.0;          // sum of node-centred kernel samples
    std::vector<int64_t> frame_off;   // host copy, F + 1
    int64_t *d_frame_off = nullptr;   // device copy
    float *d_cos[pfb::kMaxDim] = {nullptr, nullptr, nullptr};  // bin-sorted oversampled coords
    int *d_perm = nullptr;       // sorted position -> global sample index
    int *d_iperm = nullptr;      // global sample index -> sorted position
    float *d_wtap = nullptr;     // per sorted sample a record: D x WM kernel weights (WM = 4 for W <= 4,
                                 // else 8), the D first taps x0 mod n_os, padded to 16 bytes
    int *d_xtap = nullptr;       // d_wtap + D * WM (first taps inside the records, not a separate buffer)
    int *d_sframe = nullptr;     // sorted position -> frame
    int *d_bin_start = nullptr;  // (nbins_total * ncode * F + 1) offsets into the sorted order
    int nbins_total = 0;
    int ncode = 1;               // 2^ndim edge codes per tile (which next tiles a footprint reaches)
    std::vector<int> bin_start;  // host copy
    pfb::SpreadItem *d_items_frame = nullptr;  // per (bin, frame) runs
    int n_items_frame = 0;
    pfb::SpreadItem *d_items_all = nullptr;    // per bin runs over all frames
    int n_items_all = 0;
    int chunk = 0;               // max samples per work item
    int max_bin = 0;             // most samples starting in one (tile, frame)
    float *d_apod[pfb::kMaxDim] = {nullptr, nullptr, nullptr};  // deapodisation per axis (length n)
    std::mutex fft_mu;
    std::map<int64_t, cufftHandle> fft_plans;  // keyed by number of planes
    std::map<int64_t, size_t> fft_work;
    int spread_threads = 256;
    int interp_threads = 256;
    int spread_channels = 0;     // channels per CTA (0 = automatic)
    // channel-interleaved pipeline
    pfb::OwnerItem *d_own_frame = nullptr, *d_zero_frame = nullptr;
    int n_own_frame = 0, n_zero_frame = 0;
    pfb::OwnerItem *d_own_all = nullptr, *d_zero_all = nullptr;
    int n_own_all = 0, n_zero_all = 0;
    int own_chunk = 0;
    // fused pruned FFT of the channel-interleaved pipeline (tables made on first use)
    int fft_fused = -1;          // -1 not decided, 0 not applicable, 1 ready
    pfb::FftAxis fft_ax[pfb::kMaxDim];
    float2 *d_fft_tw = nullptr;  // twiddles of all axes and stages
    int *d_fft_err = nullptr;    // set by a fused-FFT kernel whose bounded wait gave up
    int fft_nsm = 0;             // SMs of the plan's device (persistent grids)
};

namespace pfb {

// ------------------------------------------------------------------------------------
// Kaiser-Bessel kernel, the reference's form (src/pyfourier/_subroutines/_grid/_plan.py:157-189):
// KB(u) = I0(beta * sqrt(1 - u^2)) for |u| <= 1, else 0, with I0 from the
// Abramowitz-Stegun 9.8.1 (a < 3.75) / 9.8.2 (a >= 3.75) polynomial forms.
// Evaluated here in float32 with Horner's rule.
// ------------------------------------------------------------------------------------
__device__ __forceinline__ float kb_small(float t2) {
    return 1.0f + t2 * (3.5156229f + t2 * (3.0899424f + t2 * (1.2067492f +
           t2 * (0.2659732f + t2 * (0.0360768f + t2 * 0.0045813f)))));
}

__device__ __forceinline__ float kb_large_poly(float ti) {
    return 0.39894228f + ti * (0.01328592f + ti * (0.00225319f + ti * (-0.00157565f +
           ti * (0.00916281f + ti * (-0.02057706f + ti * (0.02635537f +
           ti * (-0.01647633f + ti * 0.00392377f)))))));
}

__device__ __forceinline__ float kb_eval(float u, float beta) {
    if (fabsf(u) > 1.0f) return 0.0f;
    float a = beta * sqrtf(fmaf(-u, u, 1.0f));
    if (a < 3.75f) {
        float t = a * (1.0f / 3.75f);
        return kb_small(t * t);
    }
    float ti = 3.75f / a;
    return rsqrtf(a) * expf(a) * kb_large_poly(ti);
}

// Value and derivative d/du of the same polynomial form.
__device__ __forceinline__ float kb_eval_deriv(float u, float beta, float *dval) {
    if (fabsf(u) > 1.0f) { *dval = 0.0f; return 0.0f; }
    float s = fmaf(-u, u, 1.0f);
    float a = beta * sqrtf(s);
    // da/du = -beta^2 u / a  (finite form used below where a -> 0)
    if (a < 3.75f) {
        const float c = 1.0f / 3.75f;
        float t = a * c;
        float t2 = t * t;
        // dP/da = (dP/dt2)(2 t c);  dP/du = dP/da * da/du = dP/dt2 * 2 c^2 * (-beta^2 u)
        float dp_dt2 = 3.5156229f + t2 * (2.0f * 3.0899424f + t2 * (3.0f * 1.2067492f +
                       t2 * (4.0f * 0.2659732f + t2 * (5.0f * 0.0360768f + t2 * 6.0f * 0.0045813f))));
        *dval = dp_dt2 * 2.0f * c * c * (-beta * beta * u);
        return kb_small(t2);
    }
    float ti = 3.75f / a;
    float p = kb_large_poly(ti);
    // d/dti of the polynomial
    float dp_dti = 0.01328592f + ti * (2.0f * 0.00225319f + ti * (3.0f * -0.00157565f +
                   ti * (4.0f * 0.00916281f + ti * (5.0f * -0.02057706f + ti * (6.0f * 0.02635537f +
                   ti * (7.0f * -0.01647633f + ti * 8.0f * 0.00392377f))))));
    float ea = rsqrtf(a) * expf(a);               // a^-1/2 e^a
    float val = ea * p;
    // d/da [a^-1/2 e^a p(3.75/a)] = ea * ((1 - 0.5/a) p - dp_dti * 3.75 / a^2)
    float dda = ea * ((1.0f - 0.5f / a) * p - dp_dti * ti / a);
    float dadu = -beta * beta * u / a;
    *dval = dda * dadu;
    return val;
}

// Asynchronous global -> shared copies (cp.async, completed by cp_async_wait_all)
__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
// 8-byte copy; valid = false writes zeros (nothing is read)
__device__ __forceinline__ void cp_async8(void *dst, const void *src, bool valid) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 8 : 0) : "memory");
}
// 16-byte copy bypassing L1 (both addresses 16-byte aligned); valid = false writes zeros
__device__ __forceinline__ void cp_async16(void *dst, const void *src, bool valid) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 16 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// a mod n in [0, n); the common cases (|a| within one period) avoid the 64-bit division
__host__ __device__ __forceinline__ int pmod(long long a, int n) {
    if (a >= 0 && a < n) return (int)a;
    if (a < 0 && a >= -(long long)n) return (int)(a + n);
    if (a >= n && a < 2LL * n) return (int)(a - n);
    long long r = a % n;
    return (int)(r < 0 ? r + n : r);
}

// x0 = ceil(c - W/2) evaluated in float64 exactly like the reference table build
// (src/pyfourier/_subroutines/_grid/_plan.py:201); Cartesian axes use the
// nearest integer position.
__device__ __forceinline__ long long start_index(float c, int w, int cart) {
    if (cart) return (long long)rint((double)c);
    return (long long)ceil((double)c - 0.5 * (double)w);
}

// Per-axis kernel weights for one sample.  Returns x0 (unwrapped).
__device__ __forceinline__ long long axis_weights(float c, int w, int cart, float beta, float *wv) {
    long long x0 = start_index(c, w, cart);
    if (cart) {
        wv[0] = 1.0f;
#pragma unroll
        for (int i = 1; i < kMaxWidth; ++i) wv[i] = 0.0f;
        return x0;
    }
    const float halfw = 0.5f * (float)w;
#pragma unroll
    for (int i = 0; i < kMaxWidth; ++i) {
        float u = ((float)(x0 + i) - c) / halfw;
        wv[i] = (i < w) ? kb_eval(u, beta) : 0.0f;
    }
    return x0;
}

__device__ __forceinline__ long long axis_weights_deriv(float c, int w, int cart, float beta,
                                                        float *wv, float *dv) {
    long long x0 = start_index(c, w, cart);
    if (cart) {
#pragma unroll
        for (int i = 0; i < kMaxWidth; ++i) { wv[i] = (i == 0) ? 1.0f : 0.0f; dv[i] = 0.0f; }
        return x0;
    }
    const float halfw = 0.5f * (float)w;
#pragma unroll
    for (int i = 0; i < kMaxWidth; ++i) {
        float u = ((float)(x0 + i) - c) / halfw;
        float d = 0.0f;
        wv[i] = (i < w) ? kb_eval_deriv(u, beta, &d) : 0.0f;
        // d/dc of KB(((x0+i) - c) / halfw) = -KB'(u) / halfw
        dv[i] = (i < w) ? -d / halfw : 0.0f;
    }
    return x0;
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {  // a * conj(b)
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ float2 cfma(float w, float2 v, float2 acc) {
    return make_float2(fmaf(w, v.x, acc.x), fmaf(w, v.y, acc.y));
}

// Host-side launchers (implemented in the .cu files).
int launch_spread(const pfb_plan *p, const ApplyDesc &d, const float2 *y, float2 *grid,
                  bool fft_layout, cudaStream_t s);
int launch_interp(const pfb_plan *p, const ApplyDesc &d, const float2 *grid, float2 *y,
                  bool fft_layout, cudaStream_t s, bool accumulate);
int launch_traj_grad(const pfb_plan *p, const ApplyDesc &d, const float2 *grid, const float2 *v,
                     float *grad, bool fft_layout, cudaStream_t s, bool accumulate);
int launch_deapod_pad(const pfb_plan *p, const ApplyDesc &d, const float2 *img, float2 *grid,
                      float factor, cudaStream_t s);
int launch_crop_deapod(const pfb_plan *p, const ApplyDesc &d, const float2 *grid, float2 *img,
                       float factor, cudaStream_t s, bool accumulate);

// Gram helpers
int launch_embed(int ndim, const int *n, const int *nos, const float2 *img, float2 *grid,
                 int64_t nplanes, const float2 *Cl, int L, cudaStream_t s);
int launch_extract(int ndim, const int *n, const int *nos, const float2 *grid, float2 *img,
                   int64_t nplanes, float factor, const float2 *Cl, int L, cudaStream_t s);
int launch_mix(int64_t gvol, int K, int lowrank, int64_t batch, const float2 *T, float2 *grid,
               cudaStream_t s, float scale = 1.f);

// plan.cu
int plan_create(const float *coord, int ndim, int nframes, const int64_t *frame_offsets,
                int readout_len, const int *shape, const int *os_shape, const int *width,
                const float *beta, const int *is_cart, const int *tile, int device,
                cudaStream_t stream, pfb_plan **out);
int plan_tables(const pfb_plan *p, int axis_zyx, int32_t *index, float *value, cudaStream_t s);
void plan_free(pfb_plan *p);
int rebuild_items(pfb_plan *p, int chunk);

// capi.cu: planar batched cuFFT plans (cached per plane count) and execution
int get_fft_plan(std::mutex &mu, std::map<int64_t, cufftHandle> &plans, std::map<int64_t, size_t> &work,
                 int ndim, const int *nos_xyz, int64_t nplanes, cufftHandle *out, size_t *wbytes);
// Both hold `mu` (the owner's fft_mu) from cufftSetStream to the end of the exec:
// the handle, its stream and its work area are shared by all applies of a plan.
int run_fft(std::mutex &mu, cufftHandle h, size_t wbytes, float2 *data, int direction, void *work,
            size_t work_avail, cudaStream_t s);
// Out-of-place C2C transform src -> dst (src is read only; dst may equal src).
int run_fft_to(std::mutex &mu, cufftHandle h, size_t wbytes, const float2 *src, float2 *dst, int direction,
               void *work, size_t work_avail, cudaStream_t s);
// Apply options -> ApplyDesc with every argument check of the C entry points.
int to_desc(const pfb_plan *p, const pfb_apply_t *o, ApplyDesc &d);

// fast.cu (channel-interleaved pipeline)
int fast_supported(const pfb_plan *p, const ApplyDesc &d, std::string *why);
int fast_workspace(pfb_plan *p, const ApplyDesc &d, size_t *bytes);
int fast_fwd(pfb_plan *p, const ApplyDesc &d, const float2 *img, float2 *ksp, void *ws, size_t wsb, float factor,
             bool accumulate, cudaStream_t s);
int fast_adj(pfb_plan *p, const ApplyDesc &d, const float2 *ksp, float2 *img, void *ws, size_t wsb, float factor,
             bool accumulate, cudaStream_t s);
int fast_traj_grad(pfb_plan *p, const ApplyDesc &d, const float2 *img, const float2 *vals, float *grad, void *ws,
                   size_t wsb, float factor, bool accumulate, cudaStream_t s);
int fast_stage(pfb_plan *p, const ApplyDesc &d, int stage, const void *src, void *dst, void *ws, size_t wsb,
               float factor, bool accumulate, cudaStream_t s);
int build_owner_items(pfb_plan *p, int chunk);
// per-sample kernel weights and first taps of the sorted samples (plan time)
int build_plan_taps(pfb_plan *p, cudaStream_t s);
void free_owner_items(pfb_plan *p);

// sort.cu: stable LSD counting sort of (int key, int value) pairs over the low
// end_bit bits of the keys, keys in [0, 2^31); temp of counting_sort_temp_bytes(n)
size_t counting_sort_temp_bytes(int64_t n);

// Plan memory (pfb_pool.cu): blocks from a library-owned pool per device that keeps
// what destroyed plans give back.  pool_alloc's block is usable on every stream when
// it returns; pool_free is ordered on stream s (the caller orders s after the last
// use, or synchronises the device first).
int pool_alloc(void **p, size_t bytes);
void pool_free(void *p, cudaStream_t s);
int counting_sort_pairs(const int *keys, const int *vals, int *keys_out, int *vals_out, int64_t n, int end_bit,
                        void *temp, size_t temp_bytes, cudaStream_t s);

// fused pruned FFT (pfb_fft.cu): 1 when it applies to the plan (tables ready)
int fft_fused_ready(pfb_plan *p);
void fft_fused_free(pfb_plan *p);
// forward passes: 0 image -> first intermediate, 1 middle (3D only), 2 -> interleaved grid
int fft_fused_fwd(pfb_plan *p, int pass, const Chan &c, int C, const float2 *img, const float *const *apod,
                  const float2 *Cl, float factor, float2 *gridp, float2 *gridi, cudaStream_t s);
// adjoint passes: 0 planar grid -> intermediate(s), 1 -> image (crop, deapodisation, sum over segments)
int fft_fused_adj(pfb_plan *p, int pass, const Chan &c, int C, float2 *img, const float *const *apod,
                  const float2 *Cl, float factor, bool accumulate, float2 *gridp, float2 *gridi, cudaStream_t s);

}  // namespace pfb
