// Adjoint gridding ("spread"): non-Cartesian samples -> oversampled grid.
//
// Restates _grid_nb and its subspace variant
// (src/pyfourier/_subroutines/_grid/_noncart2cart/_{1,2,3}D[_subspace].py):
//   grid[plane, idx(x0 + i)] += prod_axes KB_axis(i) * value(sample, plane)
// with the B0 temporal weights, the subspace basis and the density weight
// folded into the per-sample value.
//
// B200 design.  Samples were bin-sorted at plan time by the tile holding their
// first tap x0, so one CTA owns one run of samples whose footprints all land in
// a (tile + W - 1)^d window.  The CTA accumulates that window for up to
// kMaxCh channels (coil x coefficient x segment planes) in shared memory with
// native shared-memory float atomics, computing the Kaiser-Bessel weights once
// per sample and reusing them across channels, then flushes the window to the
// grid with one 8-byte vector atomic (float2 atomicAdd, sm_90+) per non-zero
// point.  Contention on hot k-space tiles stays inside shared memory.
#include "pfb_common.cuh"

namespace pfb {

namespace {

constexpr int kMaxCh = 8;

struct SpreadParams {
    Geom g;
    int tw[kMaxDim];   // tile + w - 1
    int tvol;
    const float *cos0, *cos1, *cos2;
    const int *perm, *sframe;
    const SpreadItem *items;
    const float2 *y;
    int64_t mtot;
    const float *weight;
    const float2 *basis;
    int K;             // subspace size (0: no basis)
    int C;             // planes per (segment, batch)
    const float2 *tB;
    int L, readout;
    const int64_t *frame_off;
    int64_t B;
    int nch_total;     // channels: L * B * (K ? K : 1)
    int nch;           // channels per CTA
    float2 *grid;
    int fft_layout;
};

template <int D, int WM>
__global__ void __launch_bounds__(256) spread_kernel(const SpreadParams P) {
    extern __shared__ float2 acc[];
    const SpreadItem it = P.items[blockIdx.x];
    const int ch0 = blockIdx.y * P.nch;
    const int nc = min(P.nch, P.nch_total - ch0);
    const int tvol = P.tvol;

    for (int e = threadIdx.x; e < nc * tvol; e += blockDim.x) acc[e] = make_float2(0.f, 0.f);

    // tile origin from the bin index (x fastest)
    int org[kMaxDim] = {0, 0, 0};
    {
        int b = it.bin;
        org[0] = tile_org(P.g, 0, b % P.g.nbins[0]);
        if (D > 1) { b /= P.g.nbins[0]; org[1] = tile_org(P.g, 1, b % P.g.nbins[1]); }
        if (D > 2) { b /= P.g.nbins[1]; org[2] = tile_org(P.g, 2, b); }
    }
    __syncthreads();

    const int Kc = P.K ? P.K : 1;
    for (int j = it.begin + threadIdx.x; j < it.end; j += blockDim.x) {
        const int gs = P.perm[j];
        const int f = it.frame >= 0 ? it.frame : P.sframe[j];
        float wx[WM], wy[WM], wz[WM];
        int lo0, lo1 = 0, lo2 = 0;
        {
            float tmp[kMaxWidth];
            long long x0 = axis_weights(P.cos0[j], P.g.w[0], P.g.cart[0], P.g.beta[0], tmp);
#pragma unroll
            for (int i = 0; i < WM; ++i) wx[i] = tmp[i];
            lo0 = pmod(x0, P.g.nos[0]) - org[0];
            if (D > 1) {
                x0 = axis_weights(P.cos1[j], P.g.w[1], P.g.cart[1], P.g.beta[1], tmp);
#pragma unroll
                for (int i = 0; i < WM; ++i) wy[i] = tmp[i];
                lo1 = pmod(x0, P.g.nos[1]) - org[1];
            } else {
#pragma unroll
                for (int i = 0; i < WM; ++i) wy[i] = i == 0 ? 1.f : 0.f;
            }
            if (D > 2) {
                x0 = axis_weights(P.cos2[j], P.g.w[2], P.g.cart[2], P.g.beta[2], tmp);
#pragma unroll
                for (int i = 0; i < WM; ++i) wz[i] = tmp[i];
                lo2 = pmod(x0, P.g.nos[2]) - org[2];
            } else {
#pragma unroll
                for (int i = 0; i < WM; ++i) wz[i] = i == 0 ? 1.f : 0.f;
            }
        }
        // per-channel input values
        const float wgt = P.weight ? P.weight[gs] : 1.0f;
        int tix = 0;
        if (P.tB) tix = (int)((gs - P.frame_off[f]) % P.readout);
        float2 v[kMaxCh];
#pragma unroll
        for (int c = 0; c < kMaxCh; ++c) {
            v[c] = make_float2(0.f, 0.f);
            if (c < nc) {
                int ch = ch0 + c;
                int k = ch % Kc;
                int b = (ch / Kc) % (int)P.B;
                int l = ch / (Kc * (int)P.B);
                float2 val = P.y[(int64_t)b * P.mtot + gs];
                val.x *= wgt;
                val.y *= wgt;
                if (P.tB) val = cmulc(val, P.tB[(int64_t)l * P.readout + tix]);
                if (P.K) val = cmulc(val, P.basis[(int64_t)f * P.K + k]);
                v[c] = val;
            }
        }
        const int wz_ = D > 2 ? P.g.w[2] : 1;
        const int wy_ = D > 1 ? P.g.w[1] : 1;
        const int wx_ = P.g.w[0];
#pragma unroll
        for (int iz = 0; iz < (D > 2 ? WM : 1); ++iz) {
            if (iz >= wz_) break;
#pragma unroll
            for (int iy = 0; iy < (D > 1 ? WM : 1); ++iy) {
                if (iy >= wy_) break;
                const float wyz = wz[iz] * wy[iy];
                const int row = ((lo2 + iz) * P.tw[1] + (lo1 + iy)) * P.tw[0] + lo0;
#pragma unroll
                for (int ix = 0; ix < WM; ++ix) {
                    if (ix >= wx_) break;
                    const float wt = wyz * wx[ix];
                    float *dst = reinterpret_cast<float *>(acc + row + ix);
#pragma unroll
                    for (int c = 0; c < kMaxCh; ++c) {
                        if (c < nc) {
                            atomicAdd(dst + 2 * c * tvol, wt * v[c].x);
                            atomicAdd(dst + 2 * c * tvol + 1, wt * v[c].y);
                        }
                    }
                }
            }
        }
    }
    __syncthreads();

    // flush the window (wrapping around the periodic grid)
    const int64_t gvol = P.g.gvol;
    for (int e = threadIdx.x; e < nc * tvol; e += blockDim.x) {
        float2 val = acc[e];
        if (val.x == 0.f && val.y == 0.f) continue;
        int c = e / tvol, loc = e - c * tvol;
        int l0 = loc % P.tw[0];
        int rest = loc / P.tw[0];
        int l1 = D > 1 ? rest % P.tw[1] : 0;
        int l2 = D > 2 ? rest / P.tw[1] : 0;
        int sh0 = P.fft_layout ? P.g.sh[0] : 0;
        int p0 = pmod((long long)org[0] + l0 - sh0, P.g.nos[0]);
        int64_t lin = p0;
        if (D > 1) {
            int sh1 = P.fft_layout ? P.g.sh[1] : 0;
            int p1 = pmod((long long)org[1] + l1 - sh1, P.g.nos[1]);
            lin += (int64_t)p1 * P.g.nos[0];
        }
        if (D > 2) {
            int sh2 = P.fft_layout ? P.g.sh[2] : 0;
            int p2 = pmod((long long)org[2] + l2 - sh2, P.g.nos[2]);
            lin += (int64_t)p2 * P.g.nos[0] * P.g.nos[1];
        }
        int ch = ch0 + c;
        int k = ch % Kc;
        int b = (ch / Kc) % (int)P.B;
        int l = ch / (Kc * (int)P.B);
        int64_t plane = ((int64_t)l * P.B + b) * P.C + (P.K ? k : it.frame);
        atomicAdd(P.grid + plane * gvol + lin, val);
    }
}

template <int D, int WM>
int launch_spread_t(const SpreadParams &P, int nitems, int threads, size_t smem, cudaStream_t s) {
    int nchg = (P.nch_total + P.nch - 1) / P.nch;
    auto kern = spread_kernel<D, WM>;
    PFB_RAISE_SMEM(kern, (int)smem);
    dim3 grid(nitems, nchg);
    kern<<<grid, threads, smem, s>>>(P);
    PFB_CHECK_LAUNCH();
    return PFB_OK;
}

}  // namespace

int launch_spread(const pfb_plan *p, const ApplyDesc &d, const float2 *y, float2 *grid,
                  bool fft_layout, cudaStream_t s) {
    const Geom &g = p->g;
    int64_t nplanes = (int64_t)d.nseg * d.batch * d.ncoeff;
    if (nplanes > 0)
        PFB_CUDA_TRY(cudaMemsetAsync(grid, 0, nplanes * g.gvol * sizeof(float2), s));
    if (p->mtot == 0 || d.batch == 0) return PFB_OK;

    SpreadParams P{};
    P.g = g;
    P.tvol = 1;
    for (int a = 0; a < kMaxDim; ++a) {
        P.tw[a] = a < g.ndim ? g.tile[a] + g.w[a] - 1 : 1;
        P.tvol *= P.tw[a];
    }
    P.cos0 = p->d_cos[0];
    P.cos1 = p->d_cos[1];
    P.cos2 = p->d_cos[2];
    P.perm = p->d_perm;
    P.sframe = p->d_sframe;
    const bool use_all = d.basis != nullptr;
    P.items = use_all ? p->d_items_all : p->d_items_frame;
    int nitems = use_all ? p->n_items_all : p->n_items_frame;
    if (nitems == 0) return PFB_OK;
    P.y = y;
    P.mtot = p->mtot;
    P.weight = d.weight;
    P.basis = d.basis;
    P.K = d.basis ? d.ncoeff : 0;
    P.C = d.ncoeff;
    P.tB = d.b0_time;
    P.L = d.nseg;
    P.readout = p->readout;
    P.frame_off = p->d_frame_off;
    P.B = d.batch;
    P.nch_total = (int)((int64_t)d.nseg * d.batch * (d.basis ? d.ncoeff : 1));
    P.grid = grid;
    P.fft_layout = fft_layout ? 1 : 0;

    // channels per CTA: as many as fit ~96 KB of shared memory, at most kMaxCh
    size_t per_ch = (size_t)P.tvol * sizeof(float2);
    int nch = p->spread_channels > 0 ? p->spread_channels : (int)std::max<size_t>(1, (96 * 1024) / per_ch);
    nch = std::min(nch, kMaxCh);
    nch = std::min(nch, P.nch_total);
    if ((size_t)nch * per_ch > 200 * 1024)
        return fail(PFB_ERR_INVALID, "spread tile too large for shared memory; use a smaller tile");
    P.nch = nch;
    size_t smem = (size_t)nch * per_ch;
    int threads = p->spread_threads;
    int wmax = std::max(g.w[0], std::max(g.w[1], g.w[2]));
    bool w4 = wmax <= 4;
    switch (g.ndim) {
        case 1: return w4 ? launch_spread_t<1, 4>(P, nitems, threads, smem, s) : launch_spread_t<1, 8>(P, nitems, threads, smem, s);
        case 2: return w4 ? launch_spread_t<2, 4>(P, nitems, threads, smem, s) : launch_spread_t<2, 8>(P, nitems, threads, smem, s);
        default: return w4 ? launch_spread_t<3, 4>(P, nitems, threads, smem, s) : launch_spread_t<3, 8>(P, nitems, threads, smem, s);
    }
}

}  // namespace pfb
