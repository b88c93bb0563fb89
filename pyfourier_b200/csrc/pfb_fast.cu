// Channel-interleaved NUFFT pipeline (the path behind pfb_nufft_fwd / pfb_nufft_adj).
//
// Two grid layouts share the workspace:
//   planar       [group][channel][point]  -- what the spread writes, the z / y passes read
//   interleaved  [group][point][channel]  -- what the interp gathers from
//   without a basis: group = frame f, channel = l * B + b        (B0 segment l, batch b)
//   with a basis:    group = 0,       channel = (l * B + b) * K + k
// point is the FFT-layout position ((centred index - n_os//2) mod n_os, x fastest).
// In the interleaved layout a tap of a sample is one contiguous run of channels,
// so a warp whose lanes are channels gathers it with one coalesced access.  In
// 2D / 3D the transforms are the fused pruned FFT passes of pfb_fft.cu (pad and
// deapodise in the first pass, the last forward pass writes the interleaved
// grid; the adjoint's passes start from the spread's planar grid and crop in the
// last pass); the planar kernels below serve 1D and the layouts those passes do
// not take.
//
// Kernels:
//   pad_pl       image (B, C, *N) -> planar grid, deapodised, zero-padded, times C_l (B0)
//   transpose    planar grid -> interleaved grid
//   interp_il    interleaved grid -> res[j][channel] (one warp per sample, lanes =
//                channels x tap groups; x rows of the kernel box at 32 channels)
//   out_il       res -> k-space (B, M): sum over segments / coefficients with
//                B_l(t) basis[f, k], density weight
//   vals_il      k-space (B, M) -> vals[j][channel] in bin-sorted order, with the
//                density weight and conj(B_l(t)) conj(basis[f, k]) factors
//   spread_reg3 / spread_reg2 / spread_il
//                vals -> planar grid, owner-computes: one CTA per output tile (and
//                channel group) accumulates the contributions of the samples whose
//                first tap lies in the tile or in its 2^d - 1 lower neighbours, in
//                registers (3D, and 2D above 16 channels) or in shared memory, then
//                stores the tile (plain stores; tiles too crowded for one CTA are
//                split and combined with float2 atomics after a zeroing pass)
//   crop_pl      planar grid -> image, cropped, deapodised, sum_l conj(C_l) (B0)
//   traj_il      d/dk of sum_b Re(conj(A x)_b v_b) (analytic Kaiser-Bessel derivative)
#include <cmath>

#include <type_traits>

#include "pfb_common.cuh"

namespace pfb {

namespace {

constexpr int kTileWarps = 8;        // warps per CTA of the sample kernels
constexpr int kOutRows = 32;         // samples per CTA in the transposing kernels
constexpr int kSpreadWarps = 16;     // warps per CTA of the spread

Chan make_chan(const pfb_plan *p, const ApplyDesc &d) {
    Chan c;
    c.B = (int)d.batch;
    c.L = d.nseg;
    c.K = d.basis ? d.ncoeff : 0;
    c.F = p->nframes;
    c.nch = c.L * c.B * (c.K ? c.K : 1);
    c.ngrp = c.K ? 1 : p->nframes;
    return c;
}

__device__ __forceinline__ int log2i(int v) { return 31 - __clz(v); }

// ------------------------------------------------------------------------------------
// pad / crop on the planar grid
// ------------------------------------------------------------------------------------
struct PadPL {
    Geom g;
    const float2 *src;      // pad: image (B, C, nvol);     crop: planar grid
    float2 *dst;            // pad: planar grid;            crop: image (B, C, nvol)
    const float *apod0, *apod1, *apod2;
    const float2 *Cl;       // (L, nvol) or null
    Chan ch;
    int C;                  // image planes per batch item (F or K)
    float factor;
    int accumulate;
};

// Both kernels walk rows of the grid / image: a warp takes a segment of up to
// kRowSeg points of one row (no per-element divisions), lanes take consecutive
// points, so loads and stores are coalesced along x.
constexpr int kRowSeg = 256;

// grid plane (grp, ch), FFT-layout position p -> image pixel r = (p + N//2) mod n_os, valid if r < N
__global__ void __launch_bounds__(256) pad_pl_kernel(const PadPL P) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nx = P.g.nos[0], nseg = (nx + kRowSeg - 1) / kRowSeg;
    const int nrows = P.g.nos[1] * P.g.nos[2];
    const int64_t units = (int64_t)nrows * nseg;
    const int64_t u = (int64_t)blockIdx.x * 8 + warp;
    if (u >= units) return;
    const int row = (int)(u / nseg), seg = (int)(u - (int64_t)row * nseg);
    const int p1 = row % P.g.nos[1], p2 = row / P.g.nos[1];
    int r1 = p1 + P.g.n[1] / 2; r1 = r1 >= P.g.nos[1] ? r1 - P.g.nos[1] : r1;
    int r2 = p2 + P.g.n[2] / 2; r2 = r2 >= P.g.nos[2] ? r2 - P.g.nos[2] : r2;
    const bool inside = r1 < P.g.n[1] && r2 < P.g.n[2];
    float arow = P.factor;
    if (inside) {
        if (P.apod1) arow *= P.apod1[r1];
        if (P.apod2) arow *= P.apod2[r2];
    }
    const int x0 = seg * kRowSeg, x1 = min(nx, x0 + kRowSeg);
    const int Kc = P.ch.K ? P.ch.K : 1, B = P.ch.B;
    const int64_t rbase = ((int64_t)r2 * P.g.n[1] + r1) * P.g.n[0];
    const int nplanes = P.ch.ngrp * P.ch.nch;
    for (int plane = blockIdx.y; plane < nplanes; plane += gridDim.y) {
        const int grp = plane / P.ch.nch, ch = plane - grp * P.ch.nch;
        const int k = ch % Kc, lb = ch / Kc, b = lb % B, l = lb / B;
        const int c = P.ch.K ? k : grp;
        const float2 *src = P.src + ((int64_t)b * P.C + c) * P.g.nvol + rbase;
        const float2 *cl = P.Cl ? P.Cl + (int64_t)l * P.g.nvol + rbase : nullptr;
        float2 *dst = P.dst + (int64_t)plane * P.g.gvol + (int64_t)row * nx;
        for (int p0 = x0 + lane; p0 < x1; p0 += 32) {
            int r0 = p0 + P.g.n[0] / 2;
            r0 = r0 >= nx ? r0 - nx : r0;
            float2 out = make_float2(0.f, 0.f);
            if (inside && r0 < P.g.n[0]) {
                float2 v = src[r0];
                if (cl) v = cmul(v, cl[r0]);
                const float a = P.apod0 ? arow * P.apod0[r0] : arow;
                out = make_float2(v.x * a, v.y * a);
            }
            dst[p0] = out;
        }
    }
}

// image (b, c, r) = factor * apod(r) * sum_l conj(C_l(r)) * grid[plane(l, b, c)][(r - N//2) mod n_os]
__global__ void __launch_bounds__(256) crop_pl_kernel(const PadPL P) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n0 = P.g.n[0], nseg = (n0 + kRowSeg - 1) / kRowSeg;
    const int nrows = P.g.n[1] * P.g.n[2];
    const int64_t units = (int64_t)nrows * nseg;
    const int64_t u = (int64_t)blockIdx.x * 8 + warp;
    if (u >= units) return;
    const int row = (int)(u / nseg), seg = (int)(u - (int64_t)row * nseg);
    const int r1 = row % P.g.n[1], r2 = row / P.g.n[1];
    int p1 = r1 - P.g.n[1] / 2; p1 = p1 < 0 ? p1 + P.g.nos[1] : p1;
    int p2 = r2 - P.g.n[2] / 2; p2 = p2 < 0 ? p2 + P.g.nos[2] : p2;
    float arow = P.factor;
    if (P.apod1) arow *= P.apod1[r1];
    if (P.apod2) arow *= P.apod2[r2];
    const int x0 = seg * kRowSeg, x1 = min(n0, x0 + kRowSeg);
    const int B = P.ch.B, L = P.ch.L, Kc = P.ch.K ? P.ch.K : 1;
    const int64_t gbase = ((int64_t)p2 * P.g.nos[1] + p1) * P.g.nos[0];
    const int64_t rbase = (int64_t)row * n0;
    const int nbc = B * P.C;
    for (int bc = blockIdx.y; bc < nbc; bc += gridDim.y) {
        const int b = bc / P.C, c = bc - b * P.C;
        const int grp = P.ch.K ? 0 : c;
        float2 *dst = P.dst + (int64_t)bc * P.g.nvol + rbase;
        for (int r0 = x0 + lane; r0 < x1; r0 += 32) {
            int p0 = r0 - n0 / 2;
            p0 = p0 < 0 ? p0 + P.g.nos[0] : p0;
            float2 acc = make_float2(0.f, 0.f);
            for (int l = 0; l < L; ++l) {
                const int ch = P.ch.K ? (l * B + b) * Kc + c : l * B + b;
                float2 v = P.src[((int64_t)grp * P.ch.nch + ch) * P.g.gvol + gbase + p0];
                if (P.Cl) v = cmulc(v, P.Cl[(int64_t)l * P.g.nvol + rbase + r0]);
                acc.x += v.x;
                acc.y += v.y;
            }
            const float a = P.apod0 ? arow * P.apod0[r0] : arow;
            acc.x *= a;
            acc.y *= a;
            if (P.accumulate) {
                const float2 o = dst[r0];
                acc.x += o.x;
                acc.y += o.y;
            }
            dst[r0] = acc;
        }
    }
}

// planar [grp][ch][point] -> interleaved [grp][point][ch], through a shared tile of
// tc channels x tp points (tc * tp = 1024); loads coalesced along points, stores along channels.
__global__ void __launch_bounds__(256) transpose_kernel(const float2 *__restrict__ src, float2 *__restrict__ dst,
                                                        int64_t gvol, int nch, int tc) {
    __shared__ float2 sm[1024 + 32];
    const int tp = 1024 / tc;
    const int grp = blockIdx.z;
    const int64_t p0 = (int64_t)blockIdx.x * tp;
    const int c0 = blockIdx.y * tc;
    const float2 *S = src + (int64_t)grp * nch * gvol;
    float2 *Dd = dst + (int64_t)grp * nch * gvol;
    for (int e = threadIdx.x; e < 1024; e += blockDim.x) {
        int cl = e / tp, pl = e - cl * tp;
        int c = c0 + cl;
        int64_t p = p0 + pl;
        if (c < nch && p < gvol) sm[cl * (tp + 1) + pl] = S[(int64_t)c * gvol + p];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < 1024; e += blockDim.x) {
        int pl = e / tc, cl = e - pl * tc;
        int c = c0 + cl;
        int64_t p = p0 + pl;
        if (c < nch && p < gvol) Dd[p * nch + c] = sm[cl * (tp + 1) + pl];
    }
}

// Wide form for 32-channel chunks: a tile of 64 points x 32 channels; a warp
// reads 64 consecutive points of one channel (512 B, as float4 when the planes
// are 16-byte aligned) and writes the 32 channels of one point (256 B).
__global__ void __launch_bounds__(256) transpose32_kernel(const float2 *__restrict__ src, float2 *__restrict__ dst,
                                                          int64_t gvol, int nch, int vec) {
    __shared__ float2 sm[32][64 + 1];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grp = blockIdx.z;
    const int64_t p0 = (int64_t)blockIdx.x * 64;
    const int c0 = blockIdx.y * 32;
    const float2 *S = src + (int64_t)grp * nch * gvol;
    float2 *Dd = dst + (int64_t)grp * nch * gvol;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int cl = warp + 8 * q, c = c0 + cl;
        if (c >= nch) continue;
        const int64_t p = p0 + 2 * lane;
        const float2 *row = S + (int64_t)c * gvol;
        float2 a = make_float2(0.f, 0.f), b = a;
        if (vec && p + 1 < gvol) {
            const float4 v = __ldg(reinterpret_cast<const float4 *>(row + p));
            a = make_float2(v.x, v.y);
            b = make_float2(v.z, v.w);
        } else {
            if (p < gvol) a = row[p];
            if (p + 1 < gvol) b = row[p + 1];
        }
        sm[cl][2 * lane] = a;
        sm[cl][2 * lane + 1] = b;
    }
    __syncthreads();
    const int c = c0 + lane;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int pl = warp + 8 * q;
        const int64_t p = p0 + pl;
        if (c < nch && p < gvol) Dd[p * nch + c] = sm[lane][pl];
    }
}

// ------------------------------------------------------------------------------------
// sample-side transposes
// ------------------------------------------------------------------------------------
struct SampIL {
    const int *iperm, *sframe;
    const int64_t *frame_off;
    int64_t mtot;
    int readout;
    const float *weight;
    const float2 *basis;
    const float2 *tB;
    Chan ch;
    const float2 *src;  // vals_il: k-space (B, M);  out_il: res [M][nch]
    float2 *dst;        // vals_il: vals [M][nch];   out_il: k-space (B, M)
    int factors;        // vals_il: apply conj(tB) conj(basis) (1) or only the weight (0)
    int accumulate;
    int rows;           // samples per CTA (kOutRows .. kMaxOutRows, a power of two)
    int lrows;          // log2(rows)
    unsigned m_nch, m_kc, m_b;  // reciprocals for fdiv by nch, K (or 1) and B
};

// floor(e / d) for 0 <= e < 2^32 / d as a multiply-high by M = ceil(2^32 / d)
// (magic_of(d); M = 0 stands for d = 1): the index splits of the transposes need no
// integer division
__device__ __forceinline__ int fdiv(int e, unsigned M) { return M ? (int)__umulhi((unsigned)e, M) : e; }
inline unsigned magic_of(int d) { return d <= 1 ? 0u : (unsigned)((0x100000000ull + (unsigned)d - 1) / (unsigned)d); }

constexpr int kMaxOutRows = 128;

// samples per CTA of a transpose whose wider side has `width` float2 per sample:
// as many as fit about 32 KB of shared memory, between kOutRows and kMaxOutRows
inline int out_rows(int width) {
    int r = kOutRows;
    while (r < kMaxOutRows && (size_t)(2 * r) * width * sizeof(float2) <= 32 * 1024) r *= 2;
    return r;
}

// the rows and reciprocals of a transpose of `width` float2 per sample (O.ch set)
inline void set_samp_rows(SampIL &O, int width) {
    O.rows = out_rows(width);
    O.lrows = 0;
    while ((1 << O.lrows) < O.rows) ++O.lrows;
    O.m_nch = magic_of(O.ch.nch);
    O.m_kc = magic_of(O.ch.K ? O.ch.K : 1);
    O.m_b = magic_of(O.ch.B);
}

// Both transposes walk the samples in their original order, P.rows per CTA, so
// the k-space side is read / written coalesced and the sorted side moves whole
// rows of nch channels (iperm: original -> sorted position, staged once per CTA).

// vals[iperm[g]][ch] = y[b][g] * w[g] * conj(B_l(t)) * conj(basis[f, k])
__global__ void __launch_bounds__(256) vals_il_kernel(const SampIL P) {
    extern __shared__ float2 sm[];  // [rows][B | 1]
    __shared__ int s_j[kMaxOutRows];
    const int R = P.rows;
    const int64_t g0 = (int64_t)blockIdx.x * R;
    const int B = P.ch.B, SP = B | 1;  // odd row pitch: a warp's column accesses hit distinct banks
    for (int gg = threadIdx.x; gg < R; gg += blockDim.x) s_j[gg] = g0 + gg < P.mtot ? P.iperm[g0 + gg] : 0;
    // four loads in flight per thread before their shared-memory stores
    constexpr int U = 4;
    for (int e0 = threadIdx.x; e0 < R * B; e0 += U * blockDim.x) {
        float2 v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int e = e0 + u * blockDim.x;
            const int b = e >> P.lrows, gg = e & (R - 1);
            const int64_t g = g0 + gg;
            v[u] = make_float2(0.f, 0.f);
            if (e < R * B && g < P.mtot) {
                v[u] = P.src[(int64_t)b * P.mtot + g];
                if (P.weight) {
                    const float w = P.weight[g];
                    v[u].x *= w;
                    v[u].y *= w;
                }
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int e = e0 + u * blockDim.x;
            if (e < R * B) sm[(e & (R - 1)) * SP + (e >> P.lrows)] = v[u];
        }
    }
    __syncthreads();
    const int nch = P.ch.nch, Kc = P.ch.K ? P.ch.K : 1;
    for (int e = threadIdx.x; e < R * nch; e += blockDim.x) {
        const int gg = fdiv(e, P.m_nch), c = e - gg * nch;
        const int64_t g = g0 + gg;
        if (g >= P.mtot) continue;
        const int64_t j = s_j[gg];
        const int lb = fdiv(c, P.m_kc), k = c - lb * Kc, l = fdiv(lb, P.m_b), b = lb - l * B;
        float2 v = sm[gg * SP + b];
        if (P.factors && (P.tB || P.ch.K)) {
            const int f = P.sframe[j];
            if (P.tB) {
                const int t = (int)((g - P.frame_off[f]) % P.readout);
                v = cmulc(v, P.tB[(int64_t)l * P.readout + t]);
            }
            if (P.ch.K) v = cmulc(v, P.basis[(int64_t)f * P.ch.K + k]);
        }
        P.dst[j * nch + c] = v;
    }
}

// y[b][g] (+)= w[g] * sum_{l,k} B_l(t) basis[f, k] res[iperm[g]][(l, b, k)]
__global__ void __launch_bounds__(256) out_il_kernel(const SampIL P) {
    extern __shared__ float2 sm[];  // [rows][nch | 1]
    __shared__ int s_j[kMaxOutRows];
    const int R = P.rows;
    const int64_t g0 = (int64_t)blockIdx.x * R;
    const int nch = P.ch.nch, SP = nch | 1;  // odd row pitch: a warp's column accesses hit distinct banks
    for (int gg = threadIdx.x; gg < R; gg += blockDim.x) s_j[gg] = g0 + gg < P.mtot ? P.iperm[g0 + gg] : 0;
    __syncthreads();
    // four row loads in flight per thread before their shared-memory stores
    constexpr int U = 4;
    for (int e0 = threadIdx.x; e0 < R * nch; e0 += U * blockDim.x) {
        float2 v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int e = e0 + u * blockDim.x;
            const int gg = fdiv(e, P.m_nch), c = e - gg * nch;
            v[u] = e < R * nch && g0 + gg < P.mtot ? P.src[(int64_t)s_j[gg] * nch + c] : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int e = e0 + u * blockDim.x;
            const int gg = fdiv(e, P.m_nch), c = e - gg * nch;
            if (e < R * nch) sm[gg * SP + c] = v[u];
        }
    }
    __syncthreads();
    const int B = P.ch.B, L = P.ch.L, Kc = P.ch.K ? P.ch.K : 1;
    for (int e = threadIdx.x; e < R * B; e += blockDim.x) {
        const int b = e >> P.lrows, gg = e & (R - 1);
        const int64_t g = g0 + gg;
        if (g >= P.mtot) continue;
        float2 acc = make_float2(0.f, 0.f);
        if (L == 1 && !P.ch.K) {
            acc = sm[gg * SP + b];
        } else {
            const int f = P.sframe[s_j[gg]];
            const int t = P.tB ? (int)((g - P.frame_off[f]) % P.readout) : 0;
            for (int l = 0; l < L; ++l) {
                float2 accl = make_float2(0.f, 0.f);
                for (int k = 0; k < Kc; ++k) {
                    float2 v = sm[gg * SP + (l * B + b) * Kc + k];
                    if (P.ch.K) v = cmul(v, P.basis[(int64_t)f * P.ch.K + k]);
                    accl.x += v.x;
                    accl.y += v.y;
                }
                if (P.tB) accl = cmul(accl, P.tB[(int64_t)l * P.readout + t]);
                acc.x += accl.x;
                acc.y += accl.y;
            }
        }
        if (P.weight) {
            const float w = P.weight[g];
            acc.x *= w;
            acc.y *= w;
        }
        float2 *dst = P.dst + (int64_t)b * P.mtot + g;
        if (P.accumulate) {
            const float2 o = *dst;
            acc.x += o.x;
            acc.y += o.y;
        }
        *dst = acc;
    }
}


// ------------------------------------------------------------------------------------
// interp: one warp per bin-sorted sample, lanes = (tap group, channel)
// ------------------------------------------------------------------------------------
struct InterpIL {
    Geom g;
    const float *cos0, *cos1, *cos2;
    const int *sframe;
    int64_t mtot;
    const float2 *grid;   // interleaved
    float2 *res;          // [M][nch]
    Chan ch;
    int cw;               // lanes per channel chunk (power of two <= 32)
    // trajectory gradient
    const float2 *vt;     // [M][B] values (weight applied)
    const float2 *basis;
    const float2 *tB;
    const int *perm;
    const int64_t *frame_off;
    int readout;
    float chain[kMaxDim];
    float *grad;          // (M, ndim) in original sample order
    int accumulate;
    const float *wtap;    // plan taps: records of tap_rec(D, WM) words (weights, then first taps mod n_os)
    const int *xtap;
};

// Per-sample tap weights and FFT-layout positions, computed by lanes (axis, i)
// and left in shared memory for the warp: w[a][i], p[a][i] (and dw/dc).
template <int D, int WM, bool DERIV>
__device__ __forceinline__ void warp_taps(const InterpIL &P, int64_t j, float *sw, int *sp, float *sd, int lane) {
    if (lane < D * WM) {
        int a = lane / WM, i = lane - a * WM;
        const float *cs = a == 0 ? P.cos0 : (a == 1 ? P.cos1 : P.cos2);
        float c = cs[j];
        int w = P.g.w[a];
        long long x0 = start_index(c, w, P.g.cart[a]);
        float wv = 0.f, dv = 0.f;
        if (P.g.cart[a]) {
            wv = i == 0 ? 1.f : 0.f;
        } else if (i < w) {
            float halfw = 0.5f * (float)w;
            float u = ((float)(x0 + i) - c) / halfw;
            if (DERIV) {
                float d;
                wv = kb_eval_deriv(u, P.g.beta[a], &d);
                dv = -d / halfw;
            } else {
                wv = kb_eval(u, P.g.beta[a]);
            }
        }
        int q = pmod(x0 + i - P.g.sh[a], P.g.nos[a]);
        sw[a * WM + i] = wv;
        sp[a * WM + i] = q;
        if (DERIV) sd[a * WM + i] = dv;
    }
}

template <int D>
__host__ __device__ constexpr int ipow(int b) { return D == 1 ? b : (D == 2 ? b * b : b * b * b); }

// Per-sample plan record of the spread and interp: D * WM kernel weights, then
// the D wrapped first taps (int bits), padded to a multiple of 4 words so that
// every record starts on a 16-byte boundary (runs of records can be moved with
// bulk copies).
__host__ __device__ constexpr int tap_rec(int D, int WM) { return (D * WM + D + 3) / 4 * 4; }

// Per-sample tap list in the warp's shared memory: the tap's offset and weight
// for every tap of the WM^D box; taps beyond the kernel widths get weight 0 and
// offset 0 (an in-bounds address).  The offset is the element offset point * nch
// when that fits in 32 bits (WIDE = false), else the point index.  Lanes build
// 32 taps at a time.
template <int D, int WM, bool WIDE, typename WT>
__device__ __forceinline__ void build_tap_list(const InterpIL &P, const float *sw, const int *sp, int nch,
                                               int *s_off, WT *s_wt, int lane) {
    constexpr int NT = ipow<D>(WM);
    const int nx = P.g.nos[0], nxy = P.g.nos[0] * P.g.nos[1];
    for (int t = lane; t < NT; t += 32) {
        const int ix = t % WM, iy = (t / WM) % WM, iz = t / (WM * WM);
        const bool ok = ix < P.g.w[0] && (D < 2 || iy < P.g.w[1]) && (D < 3 || iz < P.g.w[2]);
        float w = 0.f;
        int off = 0;
        if (ok) {
            w = sw[ix] * (D > 1 ? sw[WM + iy] : 1.f) * (D > 2 ? sw[2 * WM + iz] : 1.f);
            off = sp[ix] + (D > 1 ? sp[WM + iy] * nx : 0) + (D > 2 ? sp[2 * WM + iz] * nxy : 0);
            if (!WIDE) off *= nch;
        }
        s_off[t] = off;
        if constexpr (sizeof(WT) == sizeof(float2))
            s_wt[t] = make_float2(w, w);  // the broadcast operand of a packed FFMA2
        else
            s_wt[t] = w;
    }
}

// Per-sample x rows of a 4-wide kernel box in the warp's shared memory, one row per
// (y, z) tap pair: the row's offset (the y and z parts of the tap offset, scaled like
// build_tap_list's) and its weight w_y * w_z as a (w, w) pair.  Lanes < rows build
// one row each.  With the four x taps' positions and weights in registers, the
// gather reads 12 bytes of shared memory per row of four taps instead of 12 bytes
// per tap.
template <int D, bool WIDE>
__device__ __forceinline__ void build_rows(const InterpIL &P, const float *sw, const int *sp, int nch,
                                           int *s_roff, float2 *s_rw, int lane) {
    constexpr int WM = 4, NR = D == 3 ? 16 : 4;
    if (lane < NR) {
        const int iy = lane & 3, iz = lane >> 2;
        const bool ok = iy < P.g.w[1] && (D < 3 || iz < P.g.w[2]);
        float w = 0.f;
        int off = 0;
        if (ok) {
            w = sw[WM + iy] * (D > 2 ? sw[2 * WM + iz] : 1.f);
            off = sp[WM + iy] * P.g.nos[0] + (D > 2 ? sp[2 * WM + iz] * (P.g.nos[0] * P.g.nos[1]) : 0);
            if (!WIDE) off *= nch;
        }
        s_roff[lane] = off;
        s_rw[lane] = make_float2(w, w);
    }
}

// XROWS: the launch has one channel per lane (channel chunks of 32) and a box 4
// taps wide in 2D or 3D; the kernel then takes the x-row form and keeps no
// per-tap list.  CH: the grid's channel count when fixed at compile time (x-row
// form only), else 0.
template <int D, int WM, bool WIDE, bool XROWS, int CH = 0>
__global__ void __launch_bounds__(kTileWarps * 32, 3) interp_il_kernel(const InterpIL P) {
    constexpr int NT = ipow<D>(WM);
    // up to 64 taps the weights are kept as (w, w) pairs for FFMA2 and, with one
    // channel per lane, the gather loop takes 4 taps per 16-byte offset load
    constexpr bool PAIRS = NT <= 64;
    constexpr bool VEC = PAIRS && NT % 4 == 0;
    constexpr bool VEC16 = PAIRS && NT % 16 == 0;
    constexpr bool ROWS = XROWS && PAIRS && WM == 4 && D >= 2;
    static_assert(ROWS || !XROWS, "the x-row form needs a 2D / 3D box 4 taps wide");
    static_assert(CH == 0 || (ROWS && !WIDE), "a compile-time channel count is for the 32-bit x-row form");
    constexpr int NR = ROWS ? NT / 4 : 4;    // x rows of the box
    constexpr int NL = ROWS ? 4 : NT;        // entries of the per-tap list
    using WT = typename std::conditional<PAIRS, float2, float>::type;
    __shared__ __align__(16) float s_w[kTileWarps][3 * WM];
    __shared__ __align__(16) int s_p[kTileWarps][3 * WM];
    __shared__ __align__(16) int s_off[kTileWarps][NL];
    __shared__ __align__(16) WT s_wt[kTileWarps][NL];
    __shared__ __align__(16) int s_roff[kTileWarps][NR];
    __shared__ __align__(16) float2 s_rw[kTileWarps][NR];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cw = P.cw, lcw = log2i(cw), tg_n = 32 >> lcw;
    const int cl = lane & (cw - 1), tg = lane >> lcw;
    const int nch = P.ch.nch;
    // each CTA takes a contiguous run of bin-sorted samples: its warps gather
    // from the same few tiles, which stay in L1
    const int64_t per = (P.mtot + gridDim.x - 1) / gridDim.x;
    const int64_t jbeg = (int64_t)blockIdx.x * per, jend = min(P.mtot, jbeg + per);
    // the plan taps (weights, first taps) and frame of the warp's next sample are
    // loaded into registers while the current sample gathers
    constexpr int DW = D * WM;
    float pw = 0.f;
    int px = 0, pf = 0;
    auto fetch = [&](int64_t jj) {
        if (jj < jend) {
            if (lane < DW) {
                pw = P.wtap[jj * tap_rec(D, WM) + lane];
                px = P.xtap[jj * tap_rec(D, WM) + lane / WM];
            }
            pf = P.ch.K ? 0 : P.sframe[jj];
        }
    };
    fetch(jbeg + warp);
    for (int64_t j = jbeg + warp; j < jend; j += kTileWarps) {
        if (lane < DW) {  // weights as stored, positions from the first tap x0 mod n_os
            const int a = lane / WM, i = lane - a * WM;
            s_w[warp][lane] = pw;
            s_p[warp][lane] = pmod((long long)px + i - P.g.sh[a], P.g.nos[a]);
        }
        const int grp = pf;
        fetch(j + kTileWarps);
        __syncwarp();
        const float2 *G = P.grid + (int64_t)grp * P.g.gvol * nch;
        if constexpr (ROWS)
            build_rows<D, WIDE>(P, s_w[warp], s_p[warp], nch, s_roff[warp], s_rw[warp], lane);
        else
            build_tap_list<D, WM, WIDE>(P, s_w[warp], s_p[warp], nch, s_off[warp], s_wt[warp], lane);
        __syncwarp();
        for (int c0 = 0; c0 < nch; c0 += cw) {
            const int c = c0 + cl;
            const float2 *Gc = G + (c < nch ? c : nch - 1);  // in-bounds address; result discarded
            float2 acc = make_float2(0.f, 0.f);
            if constexpr (ROWS) {
                // 4 rows (16 gathers) in flight; each x position accumulates its
                // column over the rows (weights w_y * w_z), the four columns are
                // combined with the x weights at the end
                const int4 px4 = *reinterpret_cast<const int4 *>(s_p[warp]);
                float2 ax[4] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f),
                                make_float2(0.f, 0.f)};
                const int4 *ro4 = reinterpret_cast<const int4 *>(s_roff[warp]);
                auto run = [&](auto addr) {
#pragma unroll
                    for (int rb = 0; rb < NR / 4; ++rb) {
                        const int4 o = ro4[rb];
                        const int oo[4] = {o.x, o.y, o.z, o.w};
                        float2 v[16];
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
#pragma unroll
                            for (int u = 0; u < 4; ++u) v[4 * q + u] = __ldg(addr(oo[q], u));
                        }
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            const float2 wr = s_rw[warp][4 * rb + q];
#pragma unroll
                            for (int u = 0; u < 4; ++u) ax[u] = __ffma2_rn(wr, v[4 * q + u], ax[u]);
                        }
                    }
                };
                // with a compile-time channel count and the four x taps side by side
                // (not split by the fftshift seam), a row is one pointer and its taps
                // sit at fixed offsets from it
                if (CH > 0 && px4.y == px4.x + 1 && px4.z == px4.x + 2 && px4.w == px4.x + 3) {
                    const float2 *Gx0 = Gc + px4.x * CH;
                    run([&](int o, int u) { return Gx0 + o + u * CH; });
                } else {
                    const float2 *Gx[4] = {WIDE ? Gc + (int64_t)px4.x * nch : Gc + px4.x * nch,
                                           WIDE ? Gc + (int64_t)px4.y * nch : Gc + px4.y * nch,
                                           WIDE ? Gc + (int64_t)px4.z * nch : Gc + px4.z * nch,
                                           WIDE ? Gc + (int64_t)px4.w * nch : Gc + px4.w * nch};
                    run([&](int o, int u) { return WIDE ? Gx[u] + (int64_t)o * nch : Gx[u] + o; });
                }
                const float4 wx4 = *reinterpret_cast<const float4 *>(s_w[warp]);
                const int w0 = P.g.w[0];
                const float wx1 = w0 > 1 ? wx4.y : 0.f, wx2 = w0 > 2 ? wx4.z : 0.f, wx3 = w0 > 3 ? wx4.w : 0.f;
                acc = __fmul2_rn(make_float2(wx4.x, wx4.x), ax[0]);
                acc = __ffma2_rn(make_float2(wx1, wx1), ax[1], acc);
                acc = __ffma2_rn(make_float2(wx2, wx2), ax[2], acc);
                acc = __ffma2_rn(make_float2(wx3, wx3), ax[3], acc);
            } else {
            if (VEC16 && tg_n == 1) {
                // 16 gathers issued before their sums (more loads in flight per warp);
                // taps summed in order 0, 1, 2, ...: the same sums as the loops below
                const int4 *o4 = reinterpret_cast<const int4 *>(s_off[warp]);
                const float4 *w4 = reinterpret_cast<const float4 *>(s_wt[warp]);
                for (int t16 = 0; t16 < NT / 16; ++t16) {
                    float2 v[16];
#pragma unroll
                    for (int g = 0; g < 4; ++g) {
                        const int4 o = o4[4 * t16 + g];
                        const int oo[4] = {o.x, o.y, o.z, o.w};
#pragma unroll
                        for (int u = 0; u < 4; ++u)
                            v[4 * g + u] = WIDE ? __ldg(Gc + (int64_t)oo[u] * nch) : __ldg(Gc + oo[u]);
                    }
#pragma unroll
                    for (int g = 0; g < 4; ++g) {
                        const float4 wa = w4[2 * (4 * t16 + g)], wb = w4[2 * (4 * t16 + g) + 1];
                        acc = __ffma2_rn(make_float2(wa.x, wa.y), v[4 * g + 0], acc);
                        acc = __ffma2_rn(make_float2(wa.z, wa.w), v[4 * g + 1], acc);
                        acc = __ffma2_rn(make_float2(wb.x, wb.y), v[4 * g + 2], acc);
                        acc = __ffma2_rn(make_float2(wb.z, wb.w), v[4 * g + 3], acc);
                    }
                }
            } else if (VEC && tg_n == 1) {
                // taps in order 0, 1, 2, ...: the same sums as the loop below
                const int4 *o4 = reinterpret_cast<const int4 *>(s_off[warp]);
                const float4 *w4 = reinterpret_cast<const float4 *>(s_wt[warp]);
#pragma unroll 4
                for (int t4 = 0; t4 < NT / 4; ++t4) {
                    const int4 o = o4[t4];
                    const float4 wa = w4[2 * t4], wb = w4[2 * t4 + 1];
                    float2 v[4];
                    const int oo[4] = {o.x, o.y, o.z, o.w};
#pragma unroll
                    for (int u = 0; u < 4; ++u)
                        v[u] = WIDE ? __ldg(Gc + (int64_t)oo[u] * nch) : __ldg(Gc + oo[u]);
                    acc = __ffma2_rn(make_float2(wa.x, wa.y), v[0], acc);
                    acc = __ffma2_rn(make_float2(wa.z, wa.w), v[1], acc);
                    acc = __ffma2_rn(make_float2(wb.x, wb.y), v[2], acc);
                    acc = __ffma2_rn(make_float2(wb.z, wb.w), v[3], acc);
                }
            } else {
#pragma unroll 8
                for (int t = tg; t < NT; t += tg_n) {
                    const float2 v = WIDE ? __ldg(Gc + (int64_t)s_off[warp][t] * nch) : __ldg(Gc + s_off[warp][t]);
                    if constexpr (PAIRS)
                        acc = __ffma2_rn(s_wt[warp][t], v, acc);
                    else
                        acc = cfma(s_wt[warp][t], v, acc);
                }
            }
            }
            // reduce over tap groups (lanes that share the channel)
            for (int off = cw; off < 32; off <<= 1) {
                acc.x += __shfl_xor_sync(0xffffffffu, acc.x, off);
                acc.y += __shfl_xor_sync(0xffffffffu, acc.y, off);
            }
            if (tg == 0 && c < nch) P.res[j * nch + c] = acc;
        }
        __syncwarp();
    }
}

template <int D, int WM>
__global__ void __launch_bounds__(kTileWarps * 32) traj_il_kernel(const InterpIL P) {
    __shared__ float s_w[kTileWarps][3 * WM];
    __shared__ float s_d[kTileWarps][3 * WM];
    __shared__ int s_p[kTileWarps][3 * WM];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cw = P.cw, lcw = log2i(cw), tg_n = 32 >> lcw;
    const int cl = lane & (cw - 1), tg = lane >> lcw;
    const int nch = P.ch.nch, B = P.ch.B, Kc = P.ch.K ? P.ch.K : 1;
    const int64_t nx = P.g.nos[0], nxy = (int64_t)P.g.nos[0] * P.g.nos[1];
    const int wa[3] = {P.g.w[0], D > 1 ? P.g.w[1] : 1, D > 2 ? P.g.w[2] : 1};
    const int64_t per = (P.mtot + gridDim.x - 1) / gridDim.x;
    const int64_t jbeg = (int64_t)blockIdx.x * per, jend = min(P.mtot, jbeg + per);
    for (int64_t j = jbeg + warp; j < jend; j += kTileWarps) {
        warp_taps<D, WM, true>(P, j, s_w[warp], s_p[warp], s_d[warp], lane);
        __syncwarp();
        const int f = P.sframe[j];
        const int gs = P.perm[j];
        const int grp = P.ch.K ? 0 : f;
        const int t = P.tB ? (int)((gs - P.frame_off[f]) % P.readout) : 0;
        const float2 *G = P.grid + (int64_t)grp * P.g.gvol * nch;
        float gacc[3] = {0.f, 0.f, 0.f};
        for (int c0 = 0; c0 < nch; c0 += cw) {
            const int c = c0 + cl;
            float2 dsum[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
            if (c < nch) {
                for (int iz = 0; iz < wa[2]; ++iz) {
                    const float wz = D > 2 ? s_w[warp][2 * WM + iz] : 1.f;
                    const float dz = D > 2 ? s_d[warp][2 * WM + iz] : 0.f;
                    const int64_t pz = D > 2 ? s_p[warp][2 * WM + iz] * nxy : 0;
                    for (int iy = 0; iy < wa[1]; ++iy) {
                        const float wy = D > 1 ? s_w[warp][WM + iy] : 1.f;
                        const float dy = D > 1 ? s_d[warp][WM + iy] : 0.f;
                        const int64_t rowp = pz + (D > 1 ? s_p[warp][WM + iy] * nx : 0);
                        for (int ix = tg; ix < wa[0]; ix += tg_n) {
                            const float wx = s_w[warp][ix], dx = s_d[warp][ix];
                            const float2 h = __ldg(G + (rowp + s_p[warp][ix]) * nch + c);
                            dsum[0] = cfma(wz * wy * dx, h, dsum[0]);
                            if (D > 1) dsum[1] = cfma(wz * dy * wx, h, dsum[1]);
                            if (D > 2) dsum[2] = cfma(dz * wy * wx, h, dsum[2]);
                        }
                    }
                }
                // channel factor B_l(t) basis[f, k] and the value v_b
                const int k = c % Kc, lb = c / Kc, b = lb % B, l = lb / B;
                float2 fac = make_float2(1.f, 0.f);
                if (P.tB) fac = P.tB[(int64_t)l * P.readout + t];
                if (P.ch.K) fac = cmul(fac, P.basis[(int64_t)f * P.ch.K + k]);
                const float2 v = P.vt[j * B + b];
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    float2 dd = cmul(dsum[a], fac);
                    gacc[a] += dd.x * v.x + dd.y * v.y;  // Re(conj(D) v)
                }
            }
        }
#pragma unroll
        for (int a = 0; a < 3; ++a)
            for (int off = 16; off > 0; off >>= 1) gacc[a] += __shfl_xor_sync(0xffffffffu, gacc[a], off);
        if (lane < D) {
            float r = (lane == 0 ? gacc[0] : (lane == 1 ? gacc[1] : gacc[2])) * P.chain[lane];
            float *dst = P.grad + (int64_t)gs * D + lane;
            *dst = P.accumulate ? *dst + r : r;
        }
        __syncwarp();
    }
}


// ------------------------------------------------------------------------------------
// spread: owner-computes tiles
// ------------------------------------------------------------------------------------
struct SpreadIL {
    Geom g;
    const float *cos0, *cos1, *cos2;
    const int *bin_start;
    int nframes;
    int ncode;
    const OwnerItem *items;
    const float2 *vals;   // [M][nch]
    const float *wtap;    // per sorted sample, record of tap_rec(D, WM) words: D * WM kernel weights
    const int *xtap;      // wtap + D * WM: the D wrapped first taps (same record stride)
    float2 *grid;         // planar [grp][ch][point]
    Chan ch;
    int cw;               // channels per CTA (power of two <= 32)
    int per_frame;        // 1: bins per (tile, frame); 0: bins merged over frames
};

__device__ __forceinline__ int tile_coord(int bin, int a, const Geom &g) {
    if (a == 0) return bin % g.nbins[0];
    if (a == 1) return (bin / g.nbins[0]) % g.nbins[1];
    return bin / (g.nbins[0] * g.nbins[1]);
}

// the sorted-order range of key (bin, code) for frame f (per_frame) or all frames
__device__ __forceinline__ void bin_range(const SpreadIL &P, int bin, int code, int f, int *s0, int *s1) {
    const int k0 = (bin * P.ncode + code) * P.nframes;
    if (P.per_frame) {
        *s0 = P.bin_start[k0 + f];
        *s1 = P.bin_start[k0 + f + 1];
    } else {
        *s0 = P.bin_start[k0];
        *s1 = P.bin_start[k0 + P.nframes];
    }
}

// Prefix table of the (neighbour delta, edge code) ranges that reach the item's
// tile: the samples of bins t - delta, delta in {0,1}^D, whose edge code contains
// delta.  Entry r, in the fixed order (delta ascending, then code ascending among
// the codes containing delta) in which the plan's owner items count positions,
// holds the first sorted position s_beg[r], the delta s_dlt[r] and the prefix
// s_pre[r] of the range sizes; s_pre[NR] is the total.  A delta that would wrap a
// single-tile axis onto itself gives an empty range.  The calling warp computes
// one range per lane (the loads go out together) and scans the sizes.
template <int D>
__device__ __forceinline__ void neighbour_ranges(const SpreadIL &P, const OwnerItem &it, int *s_pre, int *s_beg,
                                                 int *s_dlt, int lane) {
    constexpr int NR = D == 1 ? 3 : (D == 2 ? 9 : 27);
    int dlt = 0, code = 0;
    {
        int r = 0;
#pragma unroll
        for (int d = 0; d < (1 << D); ++d)
#pragma unroll
            for (int cd = 0; cd < (1 << D); ++cd)
                if ((cd & d) == d) {
                    if (r == lane) {
                        dlt = d;
                        code = cd;
                    }
                    ++r;
                }
    }
    int cnt = 0, s0 = 0;
    if (lane < NR) {
        int bin = 0, stride = 1;
        bool ok = true;
        for (int a = 0; a < D; ++a) {
            const int da = (dlt >> a) & 1, nb = P.g.nbins[a];
            if (da && nb == 1) ok = false;
            int tc = tile_coord(it.tile, a, P.g) - da;
            tc = tc < 0 ? tc + nb : tc;
            bin += tc * stride;
            stride *= nb;
        }
        if (ok) {
            int s1;
            bin_range(P, bin, code, it.frame < 0 ? 0 : it.frame, &s0, &s1);
            cnt = s1 - s0;
        }
    }
    int inc = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane < NR) {
        s_pre[lane] = inc - cnt;
        s_beg[lane] = s0;
        s_dlt[lane] = dlt;
    }
    if (lane == NR - 1) s_pre[NR] = inc;
}

// Per-sample kernel taps for the spread and interp, computed once per plan: in
// the record of sorted sample j (tap_rec(D, WM) words), weights w[a * WM + i]
// and then the wrapped first taps x0m[a].
template <int D, int WM>
__global__ void __launch_bounds__(256) taps_prep_kernel(Geom g, const float *__restrict__ cos0,
                                                        const float *__restrict__ cos1,
                                                        const float *__restrict__ cos2, int64_t mtot,
                                                        float *__restrict__ wout, int *__restrict__ xout) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < mtot; j += stride) {
#pragma unroll
        for (int a = 0; a < D; ++a) {
            const float c = (a == 0 ? cos0 : (a == 1 ? cos1 : cos2))[j];
            const int w = g.w[a];
            const long long x0 = start_index(c, w, g.cart[a]);
            const float inv_halfw = 2.0f / (float)w;
#pragma unroll
            for (int i = 0; i < WM; ++i) {
                float wv = 0.f;
                if (g.cart[a]) wv = i == 0 ? 1.f : 0.f;
                else if (i < w) wv = kb_eval(((float)(x0 + i) - c) * inv_halfw, g.beta[a]);
                wout[j * tap_rec(D, WM) + a * WM + i] = wv;
            }
            xout[j * tap_rec(D, WM) + a] = pmod(x0, g.nos[a]);
        }
    }
}

// Shared tile: for each tile point the real parts of its cw channels, then the
// imaginary parts, then one pad word (pitch 2*cw + 1 floats).  Lanes that are
// channels hit consecutive words in the accumulation; lanes that are points
// hit words an odd pitch apart in the store.
template <int D, int WM>
__global__ void __launch_bounds__(kSpreadWarps * 32) spread_il_kernel(const SpreadIL P) {
    extern __shared__ float acc[];
    constexpr int NT = ipow<D>(WM);
    __shared__ float s_w[kSpreadWarps][3 * WM];
    __shared__ int s_x[kSpreadWarps][3];
    constexpr int NR = D == 1 ? 3 : (D == 2 ? 9 : 27);  // (neighbour, edge code) ranges
    __shared__ int s_pre[NR + 1];   // prefix sums of the range sizes
    __shared__ int s_beg[NR];
    __shared__ int s_dlt[NR];
    const OwnerItem it = P.items[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cw = P.cw, lcw = log2i(cw), tg_n = 32 >> lcw;
    const int cl = lane & (cw - 1), tg = lane >> lcw;
    const int pitch = 2 * cw + 1;
    const int c0 = blockIdx.y * cw;
    const int nch = P.ch.nch;
    const int c = c0 + cl;
    // tile geometry
    int org[3], text[3], wrap[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (a < D) {
            int tc = tile_coord(it.tile, a, P.g);
            org[a] = tile_org(P.g, a, tc);
            text[a] = tile_extent(P.g, a, tc);
            wrap[a] = P.g.nbins[a] == 1 ? text[a] : 0;
        } else {
            org[a] = 0;
            text[a] = 1;
            wrap[a] = 0;
        }
    }
    const int T0 = P.g.tile[0], T1 = D > 1 ? P.g.tile[1] : 1, T2 = D > 2 ? P.g.tile[2] : 1;
    const int tpts = T0 * T1 * T2;
    int *s_pos = reinterpret_cast<int *>(acc + tpts * pitch);  // FFT-layout position of each tile point
    // per-warp compact tap lists (after the tile and the position table)
    int *s_li_base = s_pos + tpts;
    float *s_tw_base = reinterpret_cast<float *>(s_li_base + kSpreadWarps * NT);
    int *s_li_w = s_li_base + warp * NT;
    float *s_tw_w = s_tw_base + warp * NT;
    for (int e = threadIdx.x; e < tpts * pitch; e += blockDim.x) acc[e] = 0.f;
    for (int pt = threadIdx.x; pt < tpts; pt += blockDim.x) {
        int t0 = pt % T0, rest = pt / T0, t1 = rest % T1, t2 = rest / T1;
        int pos = -1;
        if (t0 < text[0] && t1 < text[1] && t2 < text[2]) {
            pos = pmod(org[0] + t0 - P.g.sh[0], P.g.nos[0]);
            if (D > 1) pos += pmod(org[1] + t1 - P.g.sh[1], P.g.nos[1]) * P.g.nos[0];
            if (D > 2) pos += pmod(org[2] + t2 - P.g.sh[2], P.g.nos[2]) * P.g.nos[0] * P.g.nos[1];
        }
        s_pos[pt] = pos;
    }
    // samples of the neighbour bins t - delta, delta in {0,1}^D (no wrap onto
    // itself), whose edge code contains delta: exactly those reaching this tile
    if (warp == 0) neighbour_ranges<D>(P, it, s_pre, s_beg, s_dlt, lane);
    __syncthreads();
    constexpr int DW = D * WM;
    // virtual index v over the concatenated neighbour ranges: it.v0, it.v0 + s, ...
    const int vs = item_stride(it);
    for (int v = it.v0 + warp * vs; v < it.v1; v += kSpreadWarps * vs) {
        // range r: the last one whose prefix is <= v (binary search; empty
        // ranges share their prefix with the next one and are skipped)
        int lo_r = 0, hi_r = NR;  // s_pre[lo_r] <= v < s_pre[hi_r]
        while (hi_r - lo_r > 1) {
            const int mid = (lo_r + hi_r) >> 1;
            if (s_pre[mid] <= v) lo_r = mid; else hi_r = mid;
        }
        const int r = lo_r;
        const int dl = s_dlt[r];
        const int64_t j = (int64_t)s_beg[r] + (v - s_pre[r]);
        if (lane < DW) s_w[warp][lane] = P.wtap[j * tap_rec(D, WM) + lane];
        if (lane < D) s_x[warp][lane] = P.xtap[j * tap_rec(D, WM) + lane];
        float2 val = make_float2(0.f, 0.f);
        if (c < nch) val = P.vals[j * nch + c];
        __syncwarp();
        // tile-local offset of x0 per axis; a sample of the lower neighbour (bit a
        // of r) lies before the origin, across the periodic wrap for the first tile
        int lo[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            lo[a] = 0;
            if (a < D) {
                int d = s_x[warp][a] - org[a];
                if (((dl >> a) & 1) && d >= 0) d -= P.g.nos[a];
                lo[a] = d;
            }
        }
        if (tg_n == 1) {
            // lanes are 32 channels: walk the box of this sample's taps that lies
            // inside the tile, axis by axis (warp-uniform bounds, unrolled taps)
            int i0[3], i1[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                i0[a] = 0;
                i1[a] = 1;
                if (a < D) {
                    i0[a] = wrap[a] ? 0 : max(0, -lo[a]);
                    i1[a] = wrap[a] ? P.g.w[a] : min(P.g.w[a], text[a] - lo[a]);
                }
            }
            float wx[WM];
#pragma unroll
            for (int i = 0; i < WM; ++i) wx[i] = s_w[warp][i];
            float *a0 = acc + cl;
            for (int iz = i0[2]; iz < i1[2]; ++iz) {
                int z = lo[2] + iz;
                if (D > 2 && wrap[2] && z >= wrap[2]) z -= wrap[2];
                const float wz = D > 2 ? s_w[warp][2 * WM + iz] : 1.f;
                for (int iy = i0[1]; iy < i1[1]; ++iy) {
                    int y = lo[1] + iy;
                    if (D > 1 && wrap[1] && y >= wrap[1]) y -= wrap[1];
                    const float wzy = wz * (D > 1 ? s_w[warp][WM + iy] : 1.f);
                    const float vx = wzy * val.x, vy = wzy * val.y;
                    float *row = a0 + (z * T1 + y) * T0 * pitch;
#pragma unroll
                    for (int ix = 0; ix < WM; ++ix) {
                        if (ix < i0[0] || ix >= i1[0]) continue;
                        int x = lo[0] + ix;
                        if (wrap[0] && x >= wrap[0]) x -= wrap[0];
                        atomicAdd(row + x * pitch, wx[ix] * vx);
                        atomicAdd(row + x * pitch + cw, wx[ix] * vy);
                    }
                }
            }
            __syncwarp();
            continue;
        }
        // compact list of this sample's taps that fall inside the tile:
        // (shared-memory row index * pitch, weight)
        int n_in = 0;
        for (int base = 0; base < NT; base += 32) {
            const int t = base + lane;
            const int ix = t % WM, iy = (t / WM) % WM, iz = t / (WM * WM);
            bool ok = t < NT && ix < P.g.w[0] && (D < 2 || iy < P.g.w[1]) && (D < 3 || iz < P.g.w[2]);
            int x = lo[0] + ix, y = D > 1 ? lo[1] + iy : 0, z = D > 2 ? lo[2] + iz : 0;
            if (wrap[0] && x >= wrap[0]) x -= wrap[0];
            if (D > 1 && wrap[1] && y >= wrap[1]) y -= wrap[1];
            if (D > 2 && wrap[2] && z >= wrap[2]) z -= wrap[2];
            ok = ok && x >= 0 && x < text[0] && y >= 0 && y < text[1] && z >= 0 && z < text[2];
            const unsigned m = __ballot_sync(0xffffffffu, ok);
            if (ok) {
                const int k = n_in + __popc(m & ((1u << lane) - 1u));
                s_li_w[k] = ((z * T1 + y) * T0 + x) * pitch;
                s_tw_w[k] = s_w[warp][ix] * (D > 1 ? s_w[warp][WM + iy] : 1.f) *
                                (D > 2 ? s_w[warp][2 * WM + iz] : 1.f);
            }
            n_in += __popc(m);
        }
        __syncwarp();
        if (c < nch) {
            float *a0 = acc + cl;
#pragma unroll 4
            for (int k = tg; k < n_in; k += tg_n) {
                const int li = s_li_w[k];
                const float w = s_tw_w[k];
                atomicAdd(a0 + li, w * val.x);
                atomicAdd(a0 + li + cw, w * val.y);
            }
        }
        __syncwarp();
    }
    __syncthreads();
    // write the tile into the planar grid: plain stores (sole owner) or float2
    // atomics (split tile); consecutive threads take consecutive tile points
    const int grp = P.ch.K ? 0 : (it.frame < 0 ? 0 : it.frame);
    for (int ccl = 0; ccl < cw; ++ccl) {
        const int ch = c0 + ccl;
        if (ch >= nch) break;
        float2 *G = P.grid + ((int64_t)grp * nch + ch) * P.g.gvol;
        for (int pt = threadIdx.x; pt < tpts; pt += blockDim.x) {
            const int pos = s_pos[pt];
            if (pos < 0) continue;
            const float2 vv = make_float2(acc[pt * pitch + ccl], acc[pt * pitch + cw + ccl]);
            if (it.atomic) atomicAdd(G + pos, vv);
            else G[pos] = vv;
        }
    }
}

// Register-tile spread for 3D tiles of up to 8 x 8 x 8 points and 32 channels per
// CTA (tile points are packed 8 per axis whatever the tile extent).  Each of the
// 16 warps owns a 4 x 4 x 2 block of the tile and keeps its 32 points x (its
// lane's channel) in registers, so no two warps ever write the same point and
// no atomics are needed.  Samples go through shared memory in batches: their
// raw rows (channel values, kernel weights, first taps) arrive by cp.async one
// batch ahead; then lanes (axis, t) turn them into tile-relative weight vectors
// w_x[0..8), w_y, w_z (zero outside the support and outside the tile) with a
// 24-bit mask of the non-zero entries, by which each warp picks (ballot) the
// samples that touch its block.  The tile leaves through shared memory,
// coalesced along x.
constexpr int kRegTile = 8;                   // packed tile extent per axis
// Launch shape of the register spread for CPW channels per lane group: the 32
// lanes of a warp are G = 32 / CPW groups of CPW channels, each group owning one
// of the 16 blocks of 4 x 4 x 2 points, so a CTA has 16 / G warps.
// Staging: two raw buffers (values [B][CPW] f2, plan records [B][REC] words
// (the kernel weights, then the first taps), neighbour bits [B] i), filled by
// cp.async one batch ahead, then one set of derived arrays (tile weights [B][24]
// f2, each weight held twice as the broadcast operand of a packed FFMA2; masks
// [B] u), written and read within one batch.  With 32 channels one CTA fills an
// SM (registers); smaller groups use smaller batches so that 2 (16 channels) or
// 4 (8) CTAs share an SM.
template <int CPW, int REC>
struct RegCfg {
    static constexpr int G = 32 / CPW;
    static constexpr int NW = 16 / G;
    static constexpr int Batch = CPW == 32 ? 224 : (CPW == 16 ? 128 : 80);
    static constexpr int MinBlocks = CPW == 32 ? 1 : (CPW == 16 ? 2 : 4);
    static constexpr size_t OffR = (size_t)Batch * CPW * sizeof(float2);
    static constexpr size_t OffD = OffR + (size_t)Batch * REC * sizeof(int);
    static constexpr size_t Buf = OffD + (size_t)Batch * sizeof(int);
    static constexpr size_t OffTW = 2 * Buf;
    static constexpr size_t OffM = OffTW + (size_t)Batch * 24 * sizeof(float2);
    static constexpr size_t Stage = OffM + (size_t)Batch * sizeof(unsigned);
    static constexpr size_t Out = (size_t)kRegTile * kRegTile * kRegTile * (CPW + 1) * sizeof(float2);
    static constexpr size_t Smem = Out > Stage ? Out : Stage;
    static_assert(Buf % 16 == 0 && OffTW % 16 == 0, "16-byte aligned staging arrays");
    static_assert(Smem * MinBlocks + MinBlocks * 1024 <= 228 * 1024, "shared memory of the CTAs of one SM");
};



// Rows y in [YLO, YHI], z in [ZLO, ZHI] of a 4 x 4 x 2 register block:
// acc[x + 4 (y + 4 z)] += wx[x] (wy[y] (wz[z] v)), weights as (w, w) pairs.
template <int YLO, int YHI, int ZLO, int ZHI>
__device__ __forceinline__ void reg3_rows(float2 (&acc)[32], const float2 (&wx2)[4], const float2 (&wy)[4],
                                          const float2 (&wz)[2], float2 v) {
#pragma unroll
    for (int pz = ZLO; pz <= ZHI; ++pz) {
        const float2 vz = __fmul2_rn(wz[pz], v);
#pragma unroll
        for (int py = YLO; py <= YHI; ++py) {
            const float2 vv = __fmul2_rn(wy[py], vz);
#pragma unroll
            for (int px = 0; px < 4; ++px) {
                const int q2 = px + 4 * (py + 4 * pz);
                acc[q2] = __ffma2_rn(wx2[px], vv, acc[q2]);
            }
        }
    }
}

template <int WM, int CPW>
__global__ void __launch_bounds__(RegCfg<CPW, tap_rec(3, WM)>::NW * 32, RegCfg<CPW, tap_rec(3, WM)>::MinBlocks)
    spread_reg3_kernel(const SpreadIL P) {
    constexpr int D = 3, DW = D * WM, REC = tap_rec(D, WM);
    using C = RegCfg<CPW, REC>;
    constexpr int G = C::G, NW = C::NW;
    extern __shared__ __align__(16) unsigned char ub[];
    constexpr int NR = 27;
    __shared__ int s_pre[NR + 1];
    __shared__ int s_beg[NR];
    __shared__ int s_dlt[NR];
    const OwnerItem it = P.items[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nch = P.ch.nch;
    const int cl = lane % CPW, grpl = lane / CPW;  // channel and block group of this lane
    const int c0 = blockIdx.y * CPW;
    int org[3], text[3], wrap[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const int tc = tile_coord(it.tile, a, P.g);
        org[a] = tile_org(P.g, a, tc);
        text[a] = tile_extent(P.g, a, tc);
        wrap[a] = P.g.nbins[a] == 1 ? text[a] : 0;
    }
    if (warp == 0) neighbour_ranges<3>(P, it, s_pre, s_beg, s_dlt, lane);
    __syncthreads();
    const int nvis = item_visits(it), vs = item_stride(it);
    const int nbat = (nvis + C::Batch - 1) / C::Batch;
    auto batch_size = [&](int bb) { return (nvis - bb + nbat - 1) / nbat; };
    // issue the copies of batch bb into buffer buf.  A warp takes rounds of 32
    // samples (warp, warp + NW, ... in units of 32): lane l resolves sample q0 + l
    // (its sorted position and neighbour delta), then the warp copies the round's
    // plan records and value rows in 16-byte pieces, consecutive lanes on
    // consecutive pieces of a row
    auto issue = [&](int bb, int buf) {
        unsigned char *B = ub + buf * C::Buf;
        float2 *rv = reinterpret_cast<float2 *>(B);
        int *rr = reinterpret_cast<int *>(B + C::OffR);
        int *rd = reinterpret_cast<int *>(B + C::OffD);
        const int nb = batch_size(bb);
        for (int q0 = warp * 32; q0 < nb; q0 += NW * 32) {
            const int q = q0 + lane, nq = min(32, nb - q0);
            int j = 0;
            if (q < nb) {
                // batch bb takes visits bb, bb + nbat, bb + 2 nbat, ...: every batch
                // mixes the neighbour ranges, so all warps find work in it
                const int v = it.v0 + (bb + q * nbat) * vs;
                // range: the last one whose prefix is <= v (empty ranges share the
                // prefix of the next one and are skipped)
                int lo = 0, hi = NR;
                while (hi - lo > 1) {
                    const int m = (lo + hi) >> 1;
                    if (s_pre[m] <= v) lo = m;
                    else hi = m;
                }
                j = s_beg[lo] + (v - s_pre[lo]);
                rd[q] = s_dlt[lo];
            }
            // plan records: REC / 4 pieces per sample.  Lanes past the round's last
            // piece copy nothing (a zero-size copy still writes its destination)
            constexpr int RP = REC / 4;
            for (int e0 = 0; e0 < nq * RP; e0 += 32) {
                const int e = e0 + lane;
                const bool in = e < nq * RP;
                const int sq = in ? e / RP : 0, part = e - sq * RP;
                const int js = __shfl_sync(0xffffffffu, j, sq);
                if (in) cp_async16(rr + (q0 + sq) * REC + 4 * part, P.wtap + (int64_t)js * REC + 4 * part, true);
            }
            // value rows: channels c0 .. c0 + CPW - 1, zero-filled past nch; lanes past
            // the round's last piece copy nothing
            if (nch % 2 == 0) {
                constexpr int VP = CPW / 2;  // 16-byte pieces (two channels) per row
                for (int e0 = 0; e0 < nq * VP; e0 += 32) {
                    const int e = e0 + lane;
                    const bool in = e < nq * VP;
                    const int sq = in ? e / VP : 0, part = e - sq * VP;
                    const int js = __shfl_sync(0xffffffffu, j, sq);
                    const int ch = c0 + 2 * part;
                    const bool ok = ch < nch;
                    if (in) cp_async16(rv + (q0 + sq) * CPW + 2 * part, P.vals + (ok ? (int64_t)js * nch + ch : 0), ok);
                }
            } else {
                for (int e0 = 0; e0 < nq * CPW; e0 += 32) {
                    const int e = e0 + lane;
                    const bool in = e < nq * CPW;
                    const int sq = in ? e / CPW : 0, part = e - sq * CPW;
                    const int js = __shfl_sync(0xffffffffu, j, sq);
                    const int ch = c0 + part;
                    const bool ok = ch < nch;
                    if (in) cp_async8(rv + (q0 + sq) * CPW + part, P.vals + (ok ? (int64_t)js * nch + ch : 0), ok);
                }
            }
        }
    };
    // this lane's block (block id warp * G + group) and the warp's blocks' bits in the
    // sample masks
    const int bid = warp * G + grpl;
    const int bx0 = (bid & 1) * 4, by0 = ((bid >> 1) & 1) * 4, bz0 = (bid >> 2) * 2;
    unsigned bmx[G], bmy[G], bmz[G];
#pragma unroll
    for (int g = 0; g < G; ++g) {
        const int b2 = warp * G + g;
        bmx[g] = 0xFu << ((b2 & 1) * 4);
        bmy[g] = 0xFu << (8 + ((b2 >> 1) & 1) * 4);
        bmz[g] = 0x3u << (16 + (b2 >> 2) * 2);
    }
    // tile weights: lane (slot, t) builds tile coordinate t of every axis for sample
    // slot (lanes 8 slot .. 8 slot + 7), four samples per warp pass
    const int lt = lane & 7, lslot = lane >> 3;
    float2 acc[32];
#pragma unroll
    for (int q = 0; q < 32; ++q) acc[q] = make_float2(0.f, 0.f);
    if (nbat > 0) issue(0, 0);
    cp_async_commit();
    for (int b = 0; b < nbat; ++b) {
        const int cur = b & 1;
        cp_async_wait_all();
        __syncthreads();  // batch b landed; every warp is done with batch b - 1
        if (b + 1 < nbat) issue(b + 1, cur ^ 1);
        cp_async_commit();
        unsigned char *B = ub + cur * C::Buf;
        const float2 *rv = reinterpret_cast<const float2 *>(B);
        const float *rw = reinterpret_cast<const float *>(B + C::OffR);  // records: weights, then first taps
        const int *rx = reinterpret_cast<const int *>(B + C::OffR) + DW;
        const int *rd = reinterpret_cast<const int *>(B + C::OffD);
        float2 *tw = reinterpret_cast<float2 *>(ub + C::OffTW);
        unsigned *tm = reinterpret_cast<unsigned *>(ub + C::OffM);
        const int nb = batch_size(b);
        for (int q0 = warp * 4; q0 < nb; q0 += NW * 4) {
            const int q = q0 + lslot;
            const bool qv = q < nb;
            int4 x0 = make_int4(0, 0, 0, 0);
            int dl = 0;
            if (qv) {
                // first taps mod n_os (x, y, z); one 16-byte load when they start 16-byte aligned
                if constexpr (DW % 4 == 0) {
                    x0 = *reinterpret_cast<const int4 *>(rx + q * REC);
                } else {
                    x0.x = rx[q * REC];
                    x0.y = rx[q * REC + 1];
                    x0.z = rx[q * REC + 2];
                }
                dl = rd[q];
            }
            unsigned m = 0;  // the sample's 24-bit mask of non-zero tile weights
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                float wv = 0.f;
                if (qv) {
                    int d = (a == 0 ? x0.x : (a == 1 ? x0.y : x0.z)) - org[a];
                    if (((dl >> a) & 1) && d >= 0) d -= P.g.nos[a];
                    int i = lt - d;
                    if (wrap[a] && i < 0) i += wrap[a];
                    if (lt < text[a] && i >= 0 && i < P.g.w[a]) wv = rw[q * REC + a * WM + i];
                    tw[q * 24 + a * 8 + lt] = make_float2(wv, wv);
                }
                const unsigned bal = __ballot_sync(0xffffffffu, wv != 0.f);
                m |= ((bal >> (8 * lslot)) & 0xffu) << (8 * a);
            }
            if (qv && lt == 0) tm[q] = m;
        }
        __syncthreads();  // tile weights and masks of batch b ready
        for (int q0 = 0; q0 < nb; q0 += 32) {
            bool hit = false;
            unsigned zl = 0;  // occupied z rows of the warp's z layer, sample q0 + lane
            unsigned yq = 0;  // occupied y rows of the blocks of the warp's groups (relative to each)
            if (q0 + lane < nb) {
                const unsigned m = tm[q0 + lane];
                zl = (m >> (16 + bz0)) & 3u;
#pragma unroll
                for (int g = 0; g < G; ++g) yq |= (m >> (8 + (((warp * G + g) >> 1) & 1) * 4)) & 0xFu;
#pragma unroll
                for (int g = 0; g < G; ++g) hit = hit || ((m & bmx[g]) && (m & bmy[g]) && (m & bmz[g]));
            }
            const unsigned hm = __ballot_sync(0xffffffffu, hit);
            // ballots are warp-uniform values: the loops below need no convergence barrier
            const unsigned z0 = __ballot_sync(0xffffffffu, zl & 1u), z1 = __ballot_sync(0xffffffffu, zl & 2u);
            // the hits of the round in nine passes by their occupied rows, each pass with
            // its rows fixed at compile time: z rows of the warp's z layer (both, the
            // first, the second; the blocks of a warp share one z layer) times y halves of
            // the blocks (both, the lower, the upper; with several lane groups the union
            // over the warp's blocks).  No per-hit jump on the pattern (a 3-case jump per
            // hit cost 12 instructions a hit); a pattern of one y half skips half the
            // rows.  Single y rows as patterns too would add passes costing more than the
            // rows they skip
            auto pass = [&](unsigned m, auto rows) {
                while (m) {
                    const int k = __ffs(m) - 1, q = q0 + k;
                    m &= m - 1;
                    const float2 v = rv[q * CPW + cl];
                    // weight pairs (w, w): x entries bx0..bx0+3, y 8+by0.., z 16+bz0..; zero
                    // outside the sample's support, so the rows of an occupied z layer are
                    // all updated without a test (a branch per row costs more than the row)
                    const float4 *t4 = reinterpret_cast<const float4 *>(tw + q * 24);
                    const float4 x01 = t4[bx0 >> 1], x23 = t4[(bx0 >> 1) + 1];
                    const float4 y01 = t4[(8 + by0) >> 1], y23 = t4[((8 + by0) >> 1) + 1];
                    const float4 z01 = t4[(16 + bz0) >> 1];
                    const float2 wx2[4] = {make_float2(x01.x, x01.y), make_float2(x01.z, x01.w),
                                           make_float2(x23.x, x23.y), make_float2(x23.z, x23.w)};
                    const float2 wy[4] = {make_float2(y01.x, y01.y), make_float2(y01.z, y01.w),
                                          make_float2(y23.x, y23.y), make_float2(y23.z, y23.w)};
                    const float2 wz[2] = {make_float2(z01.x, z01.y), make_float2(z01.z, z01.w)};
                    rows(wx2, wy, wz, v);
                }
            };
            const unsigned ylo = __ballot_sync(0xffffffffu, yq & 3u), yhi = __ballot_sync(0xffffffffu, yq & 0xCu);
            const unsigned zm[3] = {z0 & z1, z0 & ~z1, ~z0 & z1}, ym[3] = {ylo & yhi, ylo & ~yhi, ~ylo & yhi};
            // z pattern ZI, y pattern YI: rows y Y0..Y1, z Z0..Z1 of the block
#define PFB_PASS(ZI, Y0, Y1, Z0, Z1, YI) \
    pass(hm & zm[ZI] & ym[YI], [&](const float2(&a)[4], const float2(&b)[4], const float2(&c)[2], float2 v) { \
        reg3_rows<Y0, Y1, Z0, Z1>(acc, a, b, c, v); \
    });
            PFB_PASS(0, 0, 3, 0, 1, 0)
            PFB_PASS(0, 0, 1, 0, 1, 1)
            PFB_PASS(0, 2, 3, 0, 1, 2)
            PFB_PASS(1, 0, 3, 0, 0, 0)
            PFB_PASS(1, 0, 1, 0, 0, 1)
            PFB_PASS(1, 2, 3, 0, 0, 2)
            PFB_PASS(2, 0, 3, 1, 1, 0)
            PFB_PASS(2, 0, 1, 1, 1, 1)
            PFB_PASS(2, 2, 3, 1, 1, 2)
#undef PFB_PASS
        }
    }
    // the tile leaves through shared memory: [16 blocks x 32 points][CPW + 1]
    // (odd pitch), then thread pt writes tile point pt of every channel (the points
    // of a warp are 4 rows of 8 x positions, contiguous in the grid between wraps)
    float2 *s_out = reinterpret_cast<float2 *>(ub);
    __syncthreads();  // staging no longer read
#pragma unroll
    for (int q = 0; q < 32; ++q) s_out[(bid * 32 + q) * (CPW + 1) + cl] = acc[q];
    __syncthreads();
    const int grp = P.ch.K ? 0 : (it.frame < 0 ? 0 : it.frame);
    const int nce = min(CPW, nch - c0);
    for (int pt = threadIdx.x; pt < kRegTile * kRegTile * kRegTile; pt += blockDim.x) {
        const int x = pt & 7, y = (pt >> 3) & 7, z = pt >> 6;
        if (x >= text[0] || y >= text[1] || z >= text[2]) continue;
        const int pos = pmod(org[0] + x - P.g.sh[0], P.g.nos[0]) +
                        pmod(org[1] + y - P.g.sh[1], P.g.nos[1]) * P.g.nos[0] +
                        pmod(org[2] + z - P.g.sh[2], P.g.nos[2]) * P.g.nos[0] * P.g.nos[1];
        const int w = (x >> 2) | ((y >> 2) << 1) | ((z >> 1) << 2);
        const int q = (x & 3) | ((y & 3) << 2) | ((z & 1) << 4);
        const float2 *src = s_out + (w * 32 + q) * (CPW + 1);
        float2 *dst = P.grid + ((int64_t)grp * nch + c0) * P.g.gvol + pos;
        if (it.atomic) {
            for (int ce = 0; ce < nce; ++ce, dst += P.g.gvol) atomicAdd(dst, src[ce]);
        } else {
            for (int ce = 0; ce < nce; ++ce, dst += P.g.gvol) *dst = src[ce];
        }
    }
}

// Rows y in [Y0, Y1] of a 4 x 8 register block: acc[x + 4 y] += wx[x] (wy[y] v); t4y
// holds the block's 8 y weights as (w, w) pairs, two per float4.
template <int Y0, int Y1>
__device__ __forceinline__ void reg2_rows(float2 (&acc)[32], const float2 (&wx2)[4], const float4 *t4y, float2 v) {
#pragma unroll
    for (int py = Y0; py <= Y1; ++py) {
        const float4 y = t4y[py >> 1];
        const float2 vv = __fmul2_rn((py & 1) ? make_float2(y.z, y.w) : make_float2(y.x, y.y), v);
#pragma unroll
        for (int px = 0; px < 4; ++px) acc[px + 4 * py] = __ffma2_rn(wx2[px], vv, acc[px + 4 * py]);
    }
}

// Register-tile spread for 2D tiles of up to 16 x 16 points: the 2D form of
// spread_reg3_kernel.  Eight blocks of 4 (x) x 8 (y) points tile the packed
// 16 x 16 tile; a lane group of CPW channels owns one block, its 32 points x
// its lane's channel in registers (no atomics), so a CTA has 8 / (32 / CPW)
// warps and 2 (32 channels), 3 (16) or 4 (8) CTAs share an SM.  A sample's tile
// weights are 16 x-weights and 16 y-weights (lanes (axis, t) build them), its
// occupancy mask holds x in bits 0..15 and y in bits 16..31.
constexpr int kReg2Tile = 16;
constexpr int kReg2Pts = kReg2Tile * kReg2Tile;
template <int CPW>
struct Reg2Cfg {
    static constexpr int G = 32 / CPW;
    static constexpr int NW = 8 / G;
    static constexpr int MinBlocks = CPW == 32 ? 2 : (CPW == 16 ? 3 : 4);
    static constexpr int Batch = CPW == 32 ? 96 : (CPW == 16 ? 96 : 80);
    static constexpr size_t OffW = (size_t)Batch * CPW * sizeof(float2);
    static constexpr size_t OffX = OffW + (size_t)Batch * 16 * sizeof(float);
    static constexpr size_t OffD = OffX + (size_t)Batch * 4 * sizeof(int);
    static constexpr size_t Buf = OffD + (size_t)Batch * sizeof(int);
    static constexpr size_t OffTW = 2 * Buf;
    static constexpr size_t OffM = OffTW + (size_t)Batch * 32 * sizeof(float2);
    static constexpr size_t Stage = OffM + (size_t)Batch * sizeof(unsigned);
    static constexpr size_t Out = (size_t)kReg2Pts * (CPW + 1) * sizeof(float2);
    static constexpr size_t Smem = kReg2Pts * sizeof(int) + (Out > Stage ? Out : Stage);
    static_assert(Buf % 16 == 0 && OffTW % 16 == 0, "16-byte aligned staging arrays");
    static_assert(Smem * MinBlocks + MinBlocks * 1024 <= 228 * 1024, "shared memory of the CTAs of one SM");
};

template <int WM, int CPW>
__global__ void __launch_bounds__(Reg2Cfg<CPW>::NW * 32, Reg2Cfg<CPW>::MinBlocks)
    spread_reg2_kernel(const SpreadIL P) {
    using C = Reg2Cfg<CPW>;
    constexpr int G = C::G, NW = C::NW;
    constexpr int D = 2, DW = D * WM;
    static_assert(DW <= 16, "raw weights of one sample fit 16 entries");
    extern __shared__ __align__(16) unsigned char smraw[];
    int *s_pos = reinterpret_cast<int *>(smraw);
    unsigned char *ub = smraw + kReg2Pts * sizeof(int);
    float2 *s_out = reinterpret_cast<float2 *>(ub);  // [8 blocks x 32 points][CPW + 1], after the last batch
    constexpr int NR = 9;
    __shared__ int s_pre[NR + 1];
    __shared__ int s_beg[NR];
    __shared__ int s_dlt[NR];
    const OwnerItem it = P.items[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nch = P.ch.nch;
    const int cl = lane % CPW, grpl = lane / CPW;
    const int c0 = blockIdx.y * CPW, c = c0 + cl;
    int org[2], text[2], wrap[2];
#pragma unroll
    for (int a = 0; a < 2; ++a) {
        const int tc = tile_coord(it.tile, a, P.g);
        org[a] = tile_org(P.g, a, tc);
        text[a] = tile_extent(P.g, a, tc);
        wrap[a] = P.g.nbins[a] == 1 ? text[a] : 0;
    }
    for (int pt = threadIdx.x; pt < kReg2Pts; pt += blockDim.x) {
        const int t0 = pt & 15, t1 = pt >> 4;
        int pos = -1;
        if (t0 < text[0] && t1 < text[1])
            pos = pmod(org[0] + t0 - P.g.sh[0], P.g.nos[0]) + pmod(org[1] + t1 - P.g.sh[1], P.g.nos[1]) * P.g.nos[0];
        s_pos[pt] = pos;
    }
    if (warp == 0) neighbour_ranges<2>(P, it, s_pre, s_beg, s_dlt, lane);
    __syncthreads();
    const int nvis = item_visits(it), vs = item_stride(it);
    const int nbat = (nvis + C::Batch - 1) / C::Batch;
    auto batch_size = [&](int bb) { return (nvis - bb + nbat - 1) / nbat; };
    auto issue = [&](int bb, int buf) {
        unsigned char *B = ub + buf * C::Buf;
        float2 *rv = reinterpret_cast<float2 *>(B);
        float *rw = reinterpret_cast<float *>(B + C::OffW);
        int *rx = reinterpret_cast<int *>(B + C::OffX);
        int *rd = reinterpret_cast<int *>(B + C::OffD);
        const int nb = batch_size(bb);
        for (int q = warp; q < nb; q += NW) {
            const int v = it.v0 + (bb + q * nbat) * vs;  // batches mix the neighbour ranges
            const unsigned le = __ballot_sync(0xffffffffu, lane < NR && s_pre[lane] <= v);
            const int r = 31 - __clz(le);
            const int64_t j = (int64_t)s_beg[r] + (v - s_pre[r]);
            if (lane < CPW) cp_async8(rv + q * CPW + lane, P.vals + j * nch + (c < nch ? c : 0), c < nch);
            if (lane < DW) cp_async4(rw + q * 16 + lane, P.wtap + j * tap_rec(D, WM) + lane);
            if (lane < D) cp_async4(rx + q * 4 + lane, P.xtap + j * tap_rec(D, WM) + lane);
            if (lane == 0) rd[q] = s_dlt[r];
        }
    };
    // this lane's block: bid = warp * G + group, 4 blocks along x, 2 along y
    const int bid = warp * G + grpl;
    const int bx0 = (bid & 3) * 4, by0 = (bid >> 2) * 8;
    unsigned bmx[G], bmy[G];
#pragma unroll
    for (int g = 0; g < G; ++g) {
        const int b2 = warp * G + g;
        bmx[g] = 0xFu << ((b2 & 3) * 4);
        bmy[g] = 0xFFu << (16 + (b2 >> 2) * 8);
    }
    // lane (a, t): tile coordinate t (0..15) on axis a (lanes 0..15 x, 16..31 y)
    const int la = lane >> 4, lt = lane & 15;
    const int orga = la == 0 ? org[0] : org[1];
    const int texta = la == 0 ? text[0] : text[1];
    const int wrapa = la == 0 ? wrap[0] : wrap[1];
    const int nosa = la == 0 ? P.g.nos[0] : P.g.nos[1];
    const int wa = la == 0 ? P.g.w[0] : P.g.w[1];
    float2 acc[32];
#pragma unroll
    for (int q = 0; q < 32; ++q) acc[q] = make_float2(0.f, 0.f);
    if (nbat > 0) issue(0, 0);
    cp_async_commit();
    for (int b = 0; b < nbat; ++b) {
        const int cur = b & 1;
        cp_async_wait_all();
        __syncthreads();  // batch b landed; every warp is done with batch b - 1
        if (b + 1 < nbat) issue(b + 1, cur ^ 1);
        cp_async_commit();
        unsigned char *B = ub + cur * C::Buf;
        const float2 *rv = reinterpret_cast<const float2 *>(B);
        const float *rw = reinterpret_cast<const float *>(B + C::OffW);
        const int *rx = reinterpret_cast<const int *>(B + C::OffX);
        const int *rd = reinterpret_cast<const int *>(B + C::OffD);
        float2 *tw = reinterpret_cast<float2 *>(ub + C::OffTW);
        unsigned *tm = reinterpret_cast<unsigned *>(ub + C::OffM);
        const int nb = batch_size(b);
        for (int q = warp; q < nb; q += NW) {
            float wv = 0.f;
            int d = rx[q * 4 + la] - orga;
            if (((rd[q] >> la) & 1) && d >= 0) d -= nosa;
            int i = lt - d;
            if (wrapa && i < 0) i += wrapa;
            if (lt < texta && i >= 0 && i < wa) wv = rw[q * 16 + la * WM + i];
            tw[q * 32 + lane] = make_float2(wv, wv);
            const unsigned m = __ballot_sync(0xffffffffu, wv != 0.f);
            if (lane == 0) tm[q] = m;
        }
        __syncthreads();  // tile weights and masks of batch b ready
        for (int q0 = 0; q0 < nb; q0 += 32) {
            bool hit = false;
            unsigned yq = 0;  // occupied y rows of the warp's y block (shared by its groups)
            if (q0 + lane < nb) {
                const unsigned m = tm[q0 + lane];
                yq = (m >> (16 + by0)) & 0xFFu;
#pragma unroll
                for (int g = 0; g < G; ++g) hit = hit || ((m & bmx[g]) && (m & bmy[g]));
            }
            const unsigned hm = __ballot_sync(0xffffffffu, hit);
            // the hits of the round in passes by the occupied quarters (pairs of y rows)
            // of the block, each pass with its rows fixed at compile time: a support of
            // W <= 4 rows covers 2 or 3 of the 4 quarters, so most hits update 4 or 6 of
            // the 8 rows.  Ballots are warp-uniform: the loops need no convergence barrier
            const unsigned q0b = __ballot_sync(0xffffffffu, yq & 0x03u), q1b = __ballot_sync(0xffffffffu, yq & 0x0Cu);
            const unsigned q2b = __ballot_sync(0xffffffffu, yq & 0x30u), q3b = __ballot_sync(0xffffffffu, yq & 0xC0u);
            auto pass = [&](unsigned mk, auto rows) {
                while (mk) {
                    const int q = q0 + __ffs(mk) - 1;
                    mk &= mk - 1;
                    const float2 v = rv[q * CPW + cl];
                    // weight pairs (w, w): x entries bx0..bx0+3, y 16+by0..16+by0+7, zero
                    // outside the support, so the rows of a pass are updated without a test
                    const float4 *t4 = reinterpret_cast<const float4 *>(tw + q * 32);
                    const float4 x01 = t4[bx0 >> 1], x23 = t4[(bx0 >> 1) + 1];
                    const float2 wx2[4] = {make_float2(x01.x, x01.y), make_float2(x01.z, x01.w),
                                           make_float2(x23.x, x23.y), make_float2(x23.z, x23.w)};
                    rows(wx2, t4 + ((16 + by0) >> 1), v);
                }
            };
            // quarter range [lo, hi]: exactly the quarters lo..hi occupied
            auto range = [&](int lo, int hi) {
                const unsigned b[4] = {q0b, q1b, q2b, q3b};
                unsigned r = hm;
#pragma unroll
                for (int i = 0; i < 4; ++i) r &= (i >= lo && i <= hi) ? b[i] : ~b[i];
                return r;
            };
            unsigned done = 0;
#define PFB_PASS2(LO, HI)                                                                              \
    {                                                                                                  \
        const unsigned mk = range(LO, HI);                                                             \
        done |= mk;                                                                                    \
        pass(mk, [&](const float2(&a)[4], const float4 *ty, float2 v) { reg2_rows<2 * LO, 2 * HI + 1>(acc, a, ty, v); }); \
    }
            PFB_PASS2(0, 0) PFB_PASS2(0, 1) PFB_PASS2(0, 2) PFB_PASS2(1, 1) PFB_PASS2(1, 2)
            PFB_PASS2(1, 3) PFB_PASS2(2, 2) PFB_PASS2(2, 3) PFB_PASS2(3, 3)
#undef PFB_PASS2
            // every other pattern (all four quarters, or a support wrapped around a
            // one-tile axis): all 8 rows
            pass(hm & ~done, [&](const float2(&a)[4], const float4 *ty, float2 v) { reg2_rows<0, 7>(acc, a, ty, v); });
        }
    }
    __syncthreads();  // staging no longer read: reuse it for the output tile
#pragma unroll
    for (int q = 0; q < 32; ++q) s_out[(bid * 32 + q) * (CPW + 1) + cl] = acc[q];
    __syncthreads();
    const int grp = P.ch.K ? 0 : (it.frame < 0 ? 0 : it.frame);
    for (int e = threadIdx.x; e < CPW * kReg2Pts; e += blockDim.x) {
        const int ce = e / kReg2Pts, pt = e - ce * kReg2Pts;
        const int ch = c0 + ce;
        if (ch >= nch) break;
        const int pos = s_pos[pt];
        if (pos < 0) continue;
        const int x = pt & 15, y = pt >> 4;
        const int w = (x >> 2) | ((y >> 3) << 2);
        const int q = (x & 3) | ((y & 7) << 2);
        const float2 vv = s_out[(w * 32 + q) * (CPW + 1) + ce];
        float2 *Gp = P.grid + ((int64_t)grp * nch + ch) * P.g.gvol;
        if (it.atomic) atomicAdd(Gp + pos, vv);
        else Gp[pos] = vv;
    }
}

// zero the tiles that several CTAs combine with atomics (planar grid)
template <int D>
__global__ void zero_tiles_kernel(Geom g, const OwnerItem *zero, int nch, float2 *grid, int basis) {
    const OwnerItem it = zero[blockIdx.x];
    int org[3], text[3];
    for (int a = 0; a < 3; ++a) {
        if (a < D) {
            int tc = a == 0 ? it.tile % g.nbins[0]
                            : (a == 1 ? (it.tile / g.nbins[0]) % g.nbins[1] : it.tile / (g.nbins[0] * g.nbins[1]));
            org[a] = tile_org(g, a, tc);
            text[a] = tile_extent(g, a, tc);
        } else {
            org[a] = 0;
            text[a] = 1;
        }
    }
    const int grp = basis ? 0 : (it.frame < 0 ? 0 : it.frame);
    const int tp = text[0] * text[1] * text[2];
    for (int e = threadIdx.x; e < tp * nch; e += blockDim.x) {
        int ch = e / tp, pt = e - ch * tp;
        int t0 = pt % text[0], rest = pt / text[0], t1 = rest % text[1], t2 = rest / text[1];
        int64_t pos = pmod(org[0] + t0 - g.sh[0], g.nos[0]);
        if (D > 1) pos += (int64_t)pmod(org[1] + t1 - g.sh[1], g.nos[1]) * g.nos[0];
        if (D > 2) pos += (int64_t)pmod(org[2] + t2 - g.sh[2], g.nos[2]) * g.nos[0] * g.nos[1];
        grid[((int64_t)grp * nch + ch) * g.gvol + pos] = make_float2(0.f, 0.f);
    }
}

int pow2ceil(int v) {
    int p = 1;
    while (p < v) p <<= 1;
    return p;
}

size_t up256(size_t x) { return (x + 255) / 256 * 256; }

struct WsLayout {
    size_t gridp, gridi, samp, taps, work, total;
};

// taps per axis the kernels are compiled for: 1 (Cartesian / sparse FFT), 4 or 8
int wm_of(const Geom &g) {
    const int w = std::max(g.w[0], std::max(g.w[1], g.w[2]));
    return w == 1 ? 1 : (w <= 4 ? 4 : 8);
}

int layout_ws(pfb_plan *p, const Chan &c, WsLayout *L, cufftHandle *h, size_t *wb) {
    const int64_t P = (int64_t)c.ngrp * c.nch;
    if (fft_fused_ready(p)) {
        // the fused transform needs no library plan or work area
        *h = 0;
        *wb = 0;
    } else {
        int st = get_fft_plan(p->fft_mu, p->fft_plans, p->fft_work, p->g.ndim, p->g.nos, P, h, wb);
        if (st) return st;
    }
    L->gridp = up256((size_t)P * p->g.gvol * sizeof(float2));
    L->gridi = L->gridp;
    L->samp = up256((size_t)p->mtot * c.nch * sizeof(float2));
    L->taps = 0;  // the per-sample taps live in the plan
    L->work = up256(*wb);
    L->total = L->gridp + L->gridi + L->samp + L->taps + L->work;
    return PFB_OK;
}

template <int D, int WM>
int launch_interp_il_t(const InterpIL &P, int blocks, cudaStream_t s) {
    // element offsets point * nch in 32 bits when the grid allows it
    const bool wide = P.g.gvol * (int64_t)P.ch.nch >= (1LL << 31);
    if constexpr (WM == 4 && D >= 2) {
        if (P.cw == 32) {  // one channel per lane: the x-row form
            if (!wide && P.ch.nch == 32) interp_il_kernel<D, WM, false, true, 32><<<blocks, kTileWarps * 32, 0, s>>>(P);
            else if (!wide) interp_il_kernel<D, WM, false, true><<<blocks, kTileWarps * 32, 0, s>>>(P);
            else interp_il_kernel<D, WM, true, true><<<blocks, kTileWarps * 32, 0, s>>>(P);
            PFB_CHECK_LAUNCH();
            return PFB_OK;
        }
    }
    if (!wide) interp_il_kernel<D, WM, false, false><<<blocks, kTileWarps * 32, 0, s>>>(P);
    else interp_il_kernel<D, WM, true, false><<<blocks, kTileWarps * 32, 0, s>>>(P);
    PFB_CHECK_LAUNCH();
    return PFB_OK;
}

template <int D, int WM>
int launch_traj_il_t(const InterpIL &P, int blocks, cudaStream_t s) {
    traj_il_kernel<D, WM><<<blocks, kTileWarps * 32, 0, s>>>(P);
    PFB_CHECK_LAUNCH();
    return PFB_OK;
}

template <int WM, int CPW>
int launch_spread_reg3_t(const SpreadIL &P, int nitems, int nchunks, cudaStream_t s) {
    using C = RegCfg<CPW, tap_rec(3, WM)>;
    auto k = spread_reg3_kernel<WM, CPW>;
    PFB_RAISE_SMEM(k, (int)C::Smem);
    dim3 grid(nitems, nchunks);
    k<<<grid, C::NW * 32, C::Smem, s>>>(P);
    PFB_CHECK_LAUNCH();
    return PFB_OK;
}

template <int WM, int CPW>
int launch_spread_reg2_t(const SpreadIL &P, int nitems, int nchunks, cudaStream_t s) {
    using C = Reg2Cfg<CPW>;
    auto k = spread_reg2_kernel<WM, CPW>;
    PFB_RAISE_SMEM(k, (int)C::Smem);
    dim3 grid(nitems, nchunks);
    k<<<grid, C::NW * 32, C::Smem, s>>>(P);
    PFB_CHECK_LAUNCH();
    return PFB_OK;
}

template <int WM>
int launch_spread_reg2_w(const SpreadIL &P, int nitems, int nch, cudaStream_t s) {
    if (nch <= 8) return launch_spread_reg2_t<WM, 8>(P, nitems, 1, s);
    if (nch <= 16) return launch_spread_reg2_t<WM, 16>(P, nitems, 1, s);
    return launch_spread_reg2_t<WM, 32>(P, nitems, (nch + 31) / 32, s);
}

template <int WM>
int launch_spread_reg3_w(const SpreadIL &P, int nitems, int nch, cudaStream_t s) {
    // channel groups of 8 or 16 keep few-channel spreads on register tiles
    if (nch <= 8) return launch_spread_reg3_t<WM, 8>(P, nitems, 1, s);
    if (nch <= 16) return launch_spread_reg3_t<WM, 16>(P, nitems, 1, s);
    return launch_spread_reg3_t<WM, 32>(P, nitems, (nch + 31) / 32, s);
}

template <int D, int WM>
int launch_spread_il_t(const SpreadIL &P, int nitems, int nchunks, size_t smem, cudaStream_t s) {
    auto k = spread_il_kernel<D, WM>;
    PFB_RAISE_SMEM(k, (int)smem);
    dim3 grid(nitems, nchunks);
    k<<<grid, kSpreadWarps * 32, smem, s>>>(P);
    PFB_CHECK_LAUNCH();
    return PFB_OK;
}

int sample_blocks(int64_t mtot) {
    int64_t b = (mtot + kTileWarps - 1) / kTileWarps;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, 148LL * 64));
}

int flat_blocks(int64_t n) {
    int64_t b = (n + 255) / 256;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, 148LL * 32));
}

void fill_interp(const pfb_plan *p, const Chan &c, InterpIL &P) {
    P.g = p->g;
    P.cos0 = p->d_cos[0];
    P.cos1 = p->d_cos[1];
    P.cos2 = p->d_cos[2];
    P.sframe = p->d_sframe;
    P.perm = p->d_perm;
    P.mtot = p->mtot;
    P.ch = c;
    P.cw = std::min(32, pow2ceil(c.nch));
    P.frame_off = p->d_frame_off;
    P.readout = p->readout;
    P.wtap = p->d_wtap;
    P.xtap = p->d_xtap;
    for (int a = 0; a < kMaxDim; ++a) P.chain[a] = (float)p->g.nos[a] / (float)p->g.n[a];
}


size_t tile_points(const pfb_plan *p) {
    return (size_t)p->g.tile[0] * (p->g.ndim > 1 ? p->g.tile[1] : 1) * (p->g.ndim > 2 ? p->g.tile[2] : 1);
}

constexpr size_t kSpreadSmem = 200 * 1024;

// the spread's channel chunk: as many of the (power-of-two) lanes as fit
// bytes of the per-warp tap lists of the spread (WM^D taps, offset + weight)
size_t spread_list_bytes(const pfb_plan *p) {
    int nt = 1, wm = wm_of(p->g);
    for (int a = 0; a < p->g.ndim; ++a) nt *= wm;
    return (size_t)kSpreadWarps * nt * (sizeof(int) + sizeof(float));
}

size_t spread_smem(const pfb_plan *p, int cw) {
    return tile_points(p) * ((2 * cw + 1) * sizeof(float) + sizeof(int)) + spread_list_bytes(p);
}

int spread_cw(const pfb_plan *p, const Chan &c) {
    int cw = std::min(32, pow2ceil(c.nch));
    while (cw > 1 && spread_smem(p, cw) > kSpreadSmem) cw >>= 1;
    return cw;
}

#define PFB_DISPATCH_DW(ND, WMV, CALL1, CALL4, CALL8)                              \
    switch (ND) {                                                                  \
        case 1: return (WMV) == 1 ? CALL1(1) : ((WMV) == 4 ? CALL4(1) : CALL8(1)); \
        case 2: return (WMV) == 1 ? CALL1(2) : ((WMV) == 4 ? CALL4(2) : CALL8(2)); \
        default: return (WMV) == 1 ? CALL1(3) : ((WMV) == 4 ? CALL4(3) : CALL8(3)); \
    }

}  // namespace

int fast_supported(const pfb_plan *p, const ApplyDesc &d, std::string *why) {
    Chan c = make_chan(p, d);
    // shared-memory staging of the sample transposes: 32 rows x channels
    if ((size_t)kOutRows * c.nch * sizeof(float2) > 96 * 1024 ||
        (size_t)kOutRows * (size_t)c.B * sizeof(float2) > 96 * 1024) {
        if (why) *why = "too many channels for the interleaved path";
        return 0;
    }
    if (spread_smem(p, 1) > kSpreadSmem) {
        if (why) *why = "tile too large";
        return 0;
    }
    if (p->g.gvol >= (1LL << 31)) {
        if (why) *why = "grid too large";
        return 0;
    }
    return 1;
}

int fast_workspace(pfb_plan *p, const ApplyDesc &d, size_t *bytes) {
    Chan c = make_chan(p, d);
    WsLayout L;
    cufftHandle h;
    size_t wb;
    int st = layout_ws(p, c, &L, &h, &wb);
    if (st) return st;
    *bytes = L.total;
    return PFB_OK;
}

// One stage of the pipeline.  The workspace holds the planar grid, the
// interleaved grid, the bin-sorted sample buffer and cuFFT's work area.
//   PFB_STAGE_PAD        src image      -> planar grid
//   PFB_STAGE_FFT        planar grid forward FFT (in place)
//   PFB_STAGE_TRANSPOSE  planar grid    -> interleaved grid
//   PFB_STAGE_INTERP     interleaved grid -> sample buffer (per-channel results)
//   PFB_STAGE_OUT        sample buffer  -> dst k-space
//   PFB_STAGE_VALS       src k-space    -> sample buffer (per-channel values)
//   PFB_STAGE_SPREAD     sample buffer  -> planar grid (owner tiles)
//   PFB_STAGE_IFFT       planar grid inverse FFT (in place)
//   PFB_STAGE_CROP       planar grid    -> dst image
int fast_stage(pfb_plan *p, const ApplyDesc &d, int stage, const void *src, void *dst, void *ws, size_t wsb,
               float factor, bool accumulate, cudaStream_t s) {
    Chan c = make_chan(p, d);
    WsLayout L;
    cufftHandle h;
    size_t wb;
    int st = layout_ws(p, c, &L, &h, &wb);
    if (st) return st;
    if (wsb < L.total) return fail(PFB_ERR_WORKSPACE, "workspace too small");
    float2 *gridp = static_cast<float2 *>(ws);
    float2 *gridi = reinterpret_cast<float2 *>(static_cast<char *>(ws) + L.gridp);
    float2 *samp = reinterpret_cast<float2 *>(static_cast<char *>(ws) + L.gridp + L.gridi);
    const float *wtap = p->d_wtap;
    const int *xtap = p->d_xtap;
    void *work = static_cast<char *>(ws) + L.gridp + L.gridi + L.samp + L.taps;
    const bool basis = d.basis != nullptr;
    const int wmv = wm_of(p->g);
    const int64_t P = (int64_t)c.ngrp * c.nch;
    const bool fused = fft_fused_ready(p) == 1;
    const float *apod[3] = {p->d_apod[0], p->d_apod[1], p->d_apod[2]};
    if (fused) {
        // PAD, FFT and TRANSPOSE are the three forward passes of the fused
        // transform; IFFT is its first adjoint pass(es) and CROP the last
        switch (stage) {
            case PFB_STAGE_PAD:
                return fft_fused_fwd(p, 0, c, d.ncoeff, static_cast<const float2 *>(src), apod, d.b0_space, factor,
                                     gridp, gridi, s);
            case PFB_STAGE_FFT:
                return fft_fused_fwd(p, 1, c, d.ncoeff, nullptr, apod, d.b0_space, 1.f, gridp, gridi, s);
            case PFB_STAGE_TRANSPOSE:
                return fft_fused_fwd(p, 2, c, d.ncoeff, nullptr, apod, d.b0_space, 1.f, gridp, gridi, s);
            case PFB_STAGE_IFFT:
                return fft_fused_adj(p, 0, c, d.ncoeff, nullptr, apod, d.b0_space, 1.f, false, gridp, gridi, s);
            case PFB_STAGE_CROP:
                return fft_fused_adj(p, 1, c, d.ncoeff, static_cast<float2 *>(dst), apod, d.b0_space, factor,
                                     accumulate, gridp, gridi, s);
            default:
                break;
        }
    }
    switch (stage) {
        case PFB_STAGE_PAD:
        case PFB_STAGE_CROP: {
            PadPL Q{};
            Q.g = p->g;
            Q.apod0 = p->d_apod[0];
            Q.apod1 = p->d_apod[1];
            Q.apod2 = p->d_apod[2];
            Q.Cl = d.b0_space;
            Q.ch = c;
            Q.C = d.ncoeff;
            Q.factor = factor;
            Q.accumulate = accumulate ? 1 : 0;
            if (stage == PFB_STAGE_PAD) {
                Q.src = static_cast<const float2 *>(src);
                Q.dst = gridp;
                const int64_t units = (int64_t)p->g.nos[1] * p->g.nos[2] * ((p->g.nos[0] + kRowSeg - 1) / kRowSeg);
                dim3 grid((unsigned)((units + 7) / 8), (unsigned)std::min<int64_t>(P, 65535));
                pad_pl_kernel<<<grid, 256, 0, s>>>(Q);
            } else {
                Q.src = gridp;
                Q.dst = static_cast<float2 *>(dst);
                const int64_t units = (int64_t)p->g.n[1] * p->g.n[2] * ((p->g.n[0] + kRowSeg - 1) / kRowSeg);
                dim3 grid((unsigned)((units + 7) / 8), (unsigned)std::min<int64_t>((int64_t)c.B * d.ncoeff, 65535));
                crop_pl_kernel<<<grid, 256, 0, s>>>(Q);
            }
            PFB_CHECK_LAUNCH();
            return PFB_OK;
        }
        case PFB_STAGE_FFT:
        case PFB_STAGE_IFFT:
            return run_fft(p->fft_mu, h, wb, gridp, stage == PFB_STAGE_FFT ? -1 : +1, work, L.work, s);
        case PFB_STAGE_TRANSPOSE: {
            const int tc = std::min(32, pow2ceil(c.nch));
            if (tc == 32) {
                dim3 g3((unsigned)((p->g.gvol + 63) / 64), (unsigned)((c.nch + 31) / 32), (unsigned)c.ngrp);
                transpose32_kernel<<<g3, 256, 0, s>>>(gridp, gridi, p->g.gvol, c.nch, p->g.gvol % 2 == 0);
            } else {
                const int tp = 1024 / tc;
                dim3 g3((unsigned)((p->g.gvol + tp - 1) / tp), (unsigned)((c.nch + tc - 1) / tc), (unsigned)c.ngrp);
                transpose_kernel<<<g3, 256, 0, s>>>(gridp, gridi, p->g.gvol, c.nch, tc);
            }
            PFB_CHECK_LAUNCH();
            return PFB_OK;
        }
        case PFB_STAGE_INTERP: {
            if (p->mtot == 0) return PFB_OK;
            InterpIL Q{};
            fill_interp(p, c, Q);
            Q.grid = gridi;
            Q.res = samp;
            int blocks = sample_blocks(p->mtot);
#define PFB_I1(DD) launch_interp_il_t<DD, 1>(Q, blocks, s)
#define PFB_I4(DD) launch_interp_il_t<DD, 4>(Q, blocks, s)
#define PFB_I8(DD) launch_interp_il_t<DD, 8>(Q, blocks, s)
            PFB_DISPATCH_DW(p->g.ndim, wmv, PFB_I1, PFB_I4, PFB_I8)
#undef PFB_I1
#undef PFB_I4
#undef PFB_I8
        }
        case PFB_STAGE_OUT:
        case PFB_STAGE_VALS: {
            if (p->mtot == 0) return PFB_OK;
            SampIL O{};
            O.iperm = p->d_iperm;
            O.sframe = p->d_sframe;
            O.frame_off = p->d_frame_off;
            O.mtot = p->mtot;
            O.readout = p->readout;
            O.weight = d.weight;
            O.basis = d.basis;
            O.tB = d.b0_time;
            O.ch = c;
            O.accumulate = accumulate ? 1 : 0;
            set_samp_rows(O, std::max(c.nch, c.B));
            const unsigned blocks = (unsigned)((p->mtot + O.rows - 1) / O.rows);
            if (stage == PFB_STAGE_OUT) {
                O.src = samp;
                O.dst = static_cast<float2 *>(dst);
                size_t smem = (size_t)O.rows * (c.nch | 1) * sizeof(float2);
                PFB_RAISE_SMEM(out_il_kernel, (int)smem);
                out_il_kernel<<<blocks, 256, smem, s>>>(O);
            } else {
                O.src = static_cast<const float2 *>(src);
                O.dst = samp;
                O.factors = 1;
                size_t smem = (size_t)O.rows * (c.B | 1) * sizeof(float2);
                PFB_RAISE_SMEM(vals_il_kernel, (int)smem);
                vals_il_kernel<<<blocks, 256, smem, s>>>(O);
            }
            PFB_CHECK_LAUNCH();
            return PFB_OK;
        }
        case PFB_STAGE_SPREAD: {
            const OwnerItem *items = basis ? p->d_own_all : p->d_own_frame;
            const int nitems = basis ? p->n_own_all : p->n_own_frame;
            const OwnerItem *zero = basis ? p->d_zero_all : p->d_zero_frame;
            const int nzero = basis ? p->n_zero_all : p->n_zero_frame;
            if (nzero > 0) {
                switch (p->g.ndim) {
                    case 1: zero_tiles_kernel<1><<<nzero, 256, 0, s>>>(p->g, zero, c.nch, gridp, basis); break;
                    case 2: zero_tiles_kernel<2><<<nzero, 256, 0, s>>>(p->g, zero, c.nch, gridp, basis); break;
                    default: zero_tiles_kernel<3><<<nzero, 256, 0, s>>>(p->g, zero, c.nch, gridp, basis); break;
                }
                PFB_CHECK_LAUNCH();
            }
            if (nitems == 0) return PFB_OK;
            SpreadIL S{};
            S.g = p->g;
            S.cos0 = p->d_cos[0];
            S.cos1 = p->d_cos[1];
            S.cos2 = p->d_cos[2];
            S.bin_start = p->d_bin_start;
            S.nframes = p->nframes;
            S.ncode = p->ncode;
            S.items = items;
            S.vals = samp;
            S.wtap = wtap;
            S.xtap = xtap;
            S.grid = gridp;
            S.ch = c;
            S.cw = spread_cw(p, c);
            S.per_frame = basis ? 0 : 1;
            if (p->g.ndim == 3 && p->g.tile[0] <= kRegTile && p->g.tile[1] <= kRegTile &&
                p->g.tile[2] <= kRegTile) {
                // register-tile form: channels in groups of 8, 16 or 32 per block, no
                // shared atomics
                return wmv == 1 ? launch_spread_reg3_w<1>(S, nitems, c.nch, s)
                                : (wmv == 4 ? launch_spread_reg3_w<4>(S, nitems, c.nch, s)
                                            : launch_spread_reg3_w<8>(S, nitems, c.nch, s));
            }
            if (p->g.ndim == 2 && p->g.tile[0] <= kReg2Tile && p->g.tile[1] <= kReg2Tile && c.nch > 16) {
                // 2D register tiles (16 x 16 points), 32 channels per lane group (with
                // fewer channels a CTA would have too few warps for the crowded tiles of
                // radial trajectories: the shared-atomic kernel, 16 warps, is faster)
                return wmv == 1 ? launch_spread_reg2_w<1>(S, nitems, c.nch, s)
                                : (wmv == 4 ? launch_spread_reg2_w<4>(S, nitems, c.nch, s)
                                            : launch_spread_reg2_w<8>(S, nitems, c.nch, s));
            }
            const size_t smem = spread_smem(p, S.cw);
            const int nchunks = (c.nch + S.cw - 1) / S.cw;
#define PFB_S1(DD) launch_spread_il_t<DD, 1>(S, nitems, nchunks, smem, s)
#define PFB_S4(DD) launch_spread_il_t<DD, 4>(S, nitems, nchunks, smem, s)
#define PFB_S8(DD) launch_spread_il_t<DD, 8>(S, nitems, nchunks, smem, s)
            PFB_DISPATCH_DW(p->g.ndim, wmv, PFB_S1, PFB_S4, PFB_S8)
#undef PFB_S1
#undef PFB_S4
#undef PFB_S8
        }
        default:
            return fail(PFB_ERR_INVALID, "unknown stage");
    }
}

int fast_fwd(pfb_plan *p, const ApplyDesc &d, const float2 *img, float2 *ksp, void *ws, size_t wsb, float factor,
             bool accumulate, cudaStream_t s) {
    int st;
    if ((st = fast_stage(p, d, PFB_STAGE_PAD, img, nullptr, ws, wsb, factor, false, s))) return st;
    if ((st = fast_stage(p, d, PFB_STAGE_FFT, nullptr, nullptr, ws, wsb, 1.f, false, s))) return st;
    if ((st = fast_stage(p, d, PFB_STAGE_TRANSPOSE, nullptr, nullptr, ws, wsb, 1.f, false, s))) return st;
    if ((st = fast_stage(p, d, PFB_STAGE_INTERP, nullptr, nullptr, ws, wsb, 1.f, false, s))) return st;
    return fast_stage(p, d, PFB_STAGE_OUT, nullptr, ksp, ws, wsb, 1.f, accumulate, s);
}

int fast_adj(pfb_plan *p, const ApplyDesc &d, const float2 *ksp, float2 *img, void *ws, size_t wsb, float factor,
             bool accumulate, cudaStream_t s) {
    int st;
    if ((st = fast_stage(p, d, PFB_STAGE_VALS, ksp, nullptr, ws, wsb, 1.f, false, s))) return st;
    if ((st = fast_stage(p, d, PFB_STAGE_SPREAD, nullptr, nullptr, ws, wsb, 1.f, false, s))) return st;
    if ((st = fast_stage(p, d, PFB_STAGE_IFFT, nullptr, nullptr, ws, wsb, 1.f, false, s))) return st;
    return fast_stage(p, d, PFB_STAGE_CROP, nullptr, img, ws, wsb, factor, accumulate, s);
}

int fast_traj_grad(pfb_plan *p, const ApplyDesc &d, const float2 *img, const float2 *vals, float *grad, void *ws,
                   size_t wsb, float factor, bool accumulate, cudaStream_t s) {
    Chan c = make_chan(p, d);
    WsLayout L;
    cufftHandle h;
    size_t wb;
    int st = layout_ws(p, c, &L, &h, &wb);
    if (st) return st;
    if (wsb < L.total) return fail(PFB_ERR_WORKSPACE, "workspace too small");
    if ((st = fast_stage(p, d, PFB_STAGE_PAD, img, nullptr, ws, wsb, factor, false, s))) return st;
    if ((st = fast_stage(p, d, PFB_STAGE_FFT, nullptr, nullptr, ws, wsb, 1.f, false, s))) return st;
    if ((st = fast_stage(p, d, PFB_STAGE_TRANSPOSE, nullptr, nullptr, ws, wsb, 1.f, false, s))) return st;
    if (p->mtot == 0) return PFB_OK;
    float2 *gridi = reinterpret_cast<float2 *>(static_cast<char *>(ws) + L.gridp);
    float2 *samp = reinterpret_cast<float2 *>(static_cast<char *>(ws) + L.gridp + L.gridi);
    // v transposed to [j][b] with the density weight (no channel factors)
    Chan cb = c;
    cb.L = 1;
    cb.K = 0;
    cb.nch = c.B;
    SampIL V{};
    V.iperm = p->d_iperm;
    V.sframe = p->d_sframe;
    V.frame_off = p->d_frame_off;
    V.mtot = p->mtot;
    V.readout = p->readout;
    V.weight = d.weight;
    V.ch = cb;
    V.src = vals;
    V.dst = samp;
    V.factors = 0;
    set_samp_rows(V, std::max(c.nch, c.B));
    size_t smem = (size_t)V.rows * (c.B | 1) * sizeof(float2);
    PFB_RAISE_SMEM(vals_il_kernel, (int)smem);
    vals_il_kernel<<<(unsigned)((p->mtot + V.rows - 1) / V.rows), 256, smem, s>>>(V);
    PFB_CHECK_LAUNCH();
    InterpIL Q{};
    fill_interp(p, c, Q);
    Q.grid = gridi;
    Q.vt = samp;
    Q.basis = d.basis;
    Q.tB = d.b0_time;
    Q.grad = grad;
    Q.accumulate = accumulate ? 1 : 0;
    const int wmv = wm_of(p->g);
    int blocks = sample_blocks(p->mtot);
#define PFB_T1(DD) launch_traj_il_t<DD, 1>(Q, blocks, s)
#define PFB_T4(DD) launch_traj_il_t<DD, 4>(Q, blocks, s)
#define PFB_T8(DD) launch_traj_il_t<DD, 8>(Q, blocks, s)
    PFB_DISPATCH_DW(p->g.ndim, wmv, PFB_T1, PFB_T4, PFB_T8)
#undef PFB_T1
#undef PFB_T4
#undef PFB_T8
}

// ------------------------------------------------------------------------------------
// plan-time owner items
// ------------------------------------------------------------------------------------
namespace {

void owner_items_for(const pfb_plan *p, bool per_frame, int chunk, std::vector<OwnerItem> &items,
                     std::vector<OwnerItem> &zero) {
    const Geom &g = p->g;
    const int D = g.ndim;
    const int F = p->nframes;
    const auto &bs = p->bin_start;
    items.clear();
    zero.clear();
    const int nfr = per_frame ? F : 1;
    for (int t = 0; t < p->nbins_total; ++t) {
        int tc[3] = {0, 0, 0};
        tc[0] = t % g.nbins[0];
        if (D > 1) tc[1] = (t / g.nbins[0]) % g.nbins[1];
        if (D > 2) tc[2] = t / (g.nbins[0] * g.nbins[1]);
        for (int f = 0; f < nfr; ++f) {
            long long total = 0;
            for (int dlt = 0; dlt < (1 << D); ++dlt) {
                int bin = 0, stride = 1;
                bool ok = true;
                for (int a = 0; a < D; ++a) {
                    int da = (dlt >> a) & 1;
                    if (da && g.nbins[a] == 1) ok = false;
                    int c = tc[a] - da;
                    c = c < 0 ? c + g.nbins[a] : c;
                    bin += c * stride;
                    stride *= g.nbins[a];
                }
                if (!ok) continue;
                // only the samples whose footprint crosses into this tile along
                // every axis of delta: edge codes that contain delta
                for (int code = 0; code < (1 << D); ++code) {
                    if ((code & dlt) != dlt) continue;
                    const int k0 = (bin * p->ncode + code) * F;
                    if (per_frame) total += bs[k0 + f + 1] - bs[k0 + f];
                    else total += bs[k0 + F] - bs[k0];
                }
            }
            int fr = per_frame ? f : -1;
            if (total <= chunk) {
                items.push_back({t, fr, 0, (int)total, 0});
            } else {
                // a crowded tile: S items, item r taking visits r, r + S, r + 2 S, ... (a
                // contiguous piece would mostly be one neighbour range, whose samples
                // reach only the blocks on that side of the tile)
                const int S = (int)((total + chunk - 1) / chunk);
                for (int r = 0; r < S; ++r) items.push_back({t, fr, r, (int)total, S});
                zero.push_back({t, fr, 0, 0, 1});
            }
        }
    }
}

template <typename T>
int upload(const std::vector<T> &h, T **d) {
    if (*d) {
        cudaDeviceSynchronize();  // applies in flight may read the old table
        pool_free(*d, 0);
        *d = nullptr;
    }
    const int st = pool_alloc(reinterpret_cast<void **>(d), std::max<size_t>(h.size(), 1) * sizeof(T));
    if (st) return st;
    if (!h.empty()) PFB_CUDA_TRY(cudaMemcpy(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    return PFB_OK;
}

}  // namespace

int build_owner_items(pfb_plan *p, int chunk) {
    std::vector<OwnerItem> it, z;
    int st;
    owner_items_for(p, true, chunk, it, z);
    if ((st = upload(it, &p->d_own_frame))) return st;
    if ((st = upload(z, &p->d_zero_frame))) return st;
    p->n_own_frame = (int)it.size();
    p->n_zero_frame = (int)z.size();
    owner_items_for(p, false, chunk, it, z);
    if ((st = upload(it, &p->d_own_all))) return st;
    if ((st = upload(z, &p->d_zero_all))) return st;
    p->n_own_all = (int)it.size();
    p->n_zero_all = (int)z.size();
    p->own_chunk = chunk;
    return PFB_OK;
}

int build_plan_taps(pfb_plan *p, cudaStream_t s) {
    if (p->d_wtap) {
        cudaDeviceSynchronize();  // applies in flight may read the old records
        pool_free(p->d_wtap, 0);
    }
    p->d_wtap = nullptr;
    p->d_xtap = nullptr;
    const int D = p->g.ndim, WM = wm_of(p->g);
    const size_t n = (size_t)std::max<int64_t>(p->mtot, 1);
    // one record per sorted sample: weights, then first taps (d_xtap points into it)
    const int st = pool_alloc(reinterpret_cast<void **>(&p->d_wtap), n * tap_rec(D, WM) * sizeof(float));
    if (st) return st;
    p->d_xtap = reinterpret_cast<int *>(p->d_wtap + D * WM);
    if (p->mtot == 0) return PFB_OK;
    const int tb = flat_blocks(p->mtot);
    float *w = p->d_wtap;
    int *x = p->d_xtap;
    switch (D * 10 + WM) {
        case 11: taps_prep_kernel<1, 1><<<tb, 256, 0, s>>>(p->g, p->d_cos[0], p->d_cos[1], p->d_cos[2], p->mtot, w, x); break;
        case 21: taps_prep_kernel<2, 1><<<tb, 256, 0, s>>>(p->g, p->d_cos[0], p->d_cos[1], p->d_cos[2], p->mtot, w, x); break;
        case 31: taps_prep_kernel<3, 1><<<tb, 256, 0, s>>>(p->g, p->d_cos[0], p->d_cos[1], p->d_cos[2], p->mtot, w, x); break;
        case 14: taps_prep_kernel<1, 4><<<tb, 256, 0, s>>>(p->g, p->d_cos[0], p->d_cos[1], p->d_cos[2], p->mtot, w, x); break;
        case 18: taps_prep_kernel<1, 8><<<tb, 256, 0, s>>>(p->g, p->d_cos[0], p->d_cos[1], p->d_cos[2], p->mtot, w, x); break;
        case 24: taps_prep_kernel<2, 4><<<tb, 256, 0, s>>>(p->g, p->d_cos[0], p->d_cos[1], p->d_cos[2], p->mtot, w, x); break;
        case 28: taps_prep_kernel<2, 8><<<tb, 256, 0, s>>>(p->g, p->d_cos[0], p->d_cos[1], p->d_cos[2], p->mtot, w, x); break;
        case 34: taps_prep_kernel<3, 4><<<tb, 256, 0, s>>>(p->g, p->d_cos[0], p->d_cos[1], p->d_cos[2], p->mtot, w, x); break;
        default: taps_prep_kernel<3, 8><<<tb, 256, 0, s>>>(p->g, p->d_cos[0], p->d_cos[1], p->d_cos[2], p->mtot, w, x); break;
    }
    PFB_CHECK_LAUNCH();
    return PFB_OK;
}

void free_owner_items(pfb_plan *p) {
    cudaDeviceSynchronize();  // every apply of the plan has finished
    pool_free(p->d_wtap, 0);  // d_xtap points into the same records
    p->d_wtap = nullptr;
    p->d_xtap = nullptr;
    pool_free(p->d_own_frame, 0);
    pool_free(p->d_zero_frame, 0);
    pool_free(p->d_own_all, 0);
    pool_free(p->d_zero_all, 0);
    p->d_own_frame = p->d_zero_frame = p->d_own_all = p->d_zero_all = nullptr;
    fft_fused_free(p);
}

}  // namespace pfb
