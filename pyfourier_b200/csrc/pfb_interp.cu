// Forward gridding ("interp") and the trajectory gradient.
//
// Interp restates _degrid_nb and its subspace variant
// (src/pyfourier/_subroutines/_grid/_cart2noncart/_{1,2,3}D[_subspace].py):
//   y[b, g] = sum_l B_l(t) * sum_k basis[f, k] * sum_taps prod_axes KB * grid[(l, b, k), idx]
// (the B0 / basis factors reduce to 1 when absent), times the density weight.
//
// One thread per bin-sorted sample: neighbouring threads read overlapping
// grid windows, so the W^d gathers hit L1/L2 instead of HBM.  The kernel
// weights are computed once per sample and reused for every coil, segment
// and coefficient plane.
//
// The trajectory gradient uses the analytic derivative of the same
// Kaiser-Bessel form: for every sample and axis
//   D_{b,a} = sum_l B_l(t) sum_k basis[f,k] sum_taps dKB_a * prod_{other} KB * H[(l,b,k), idx]
//   grad[g, a] = (n_os,a / N_a) * sum_b Re(conj(D_{b,a}) * v[b, g]) * weight[g]
// which is d/dk of Re(<v, A(k) x>) when H is the forward grid of x.  The
// reference's trajectory backward (src/pyfourier/_nufft/_nufft.py:175-209)
// builds ramped images instead and omits the -2*pi*i/N factor.
#include "pfb_common.cuh"

namespace pfb {

namespace {

struct InterpParams {
    Geom g;
    const float *cos0, *cos1, *cos2;
    const int *perm, *sframe;
    const float2 *grid;
    float2 *y;
    int64_t mtot;
    const float *weight;
    const float2 *basis;
    int K;
    int C;
    const float2 *tB;
    int L, readout;
    const int64_t *frame_off;
    int64_t B;
    int fft_layout;
    int accumulate;
    float chain[kMaxDim];  // n_os / N per axis (traj grad)
    float *grad;
};

template <int D, int WM>
__device__ __forceinline__ void sample_taps(const InterpParams &P, int j, float (&w)[3][WM],
                                            int (&px)[WM], int (&py)[WM], int (&pz)[WM]) {
    const float *cs[3] = {P.cos0, P.cos1, P.cos2};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (a >= D) {
#pragma unroll
            for (int i = 0; i < WM; ++i) w[a][i] = i == 0 ? 1.f : 0.f;
            continue;
        }
        float tmp[kMaxWidth];
        long long x0 = axis_weights(cs[a][j], P.g.w[a], P.g.cart[a], P.g.beta[a], tmp);
        int sh = P.fft_layout ? P.g.sh[a] : 0;
        int base = pmod(x0 - sh, P.g.nos[a]);
#pragma unroll
        for (int i = 0; i < WM; ++i) {
            w[a][i] = tmp[i];
            int q = base + i;
            q = q >= P.g.nos[a] ? q - P.g.nos[a] : q;
            if (a == 0) px[i] = q;
            if (a == 1) py[i] = q;
            if (a == 2) pz[i] = q;
        }
    }
}

template <int D, int WM>
__global__ void __launch_bounds__(256) interp_kernel(const InterpParams P) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int Kc = P.K ? P.K : 1;
    const int wx_ = P.g.w[0];
    const int wy_ = D > 1 ? P.g.w[1] : 1;
    const int wz_ = D > 2 ? P.g.w[2] : 1;
    const int64_t nx = P.g.nos[0], nxy = (int64_t)P.g.nos[0] * P.g.nos[1];
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < P.mtot; j += stride) {
        const int gs = P.perm[j];
        const int f = P.sframe[j];
        float w[3][WM];
        int px[WM], py[WM], pz[WM];
#pragma unroll
        for (int i = 0; i < WM; ++i) { px[i] = 0; py[i] = 0; pz[i] = 0; }
        sample_taps<D, WM>(P, (int)j, w, px, py, pz);
        const float wgt = P.weight ? P.weight[gs] : 1.0f;
        int tix = 0;
        if (P.tB) tix = (int)((gs - P.frame_off[f]) % P.readout);
        for (int64_t b = 0; b < P.B; ++b) {
            float2 acc = make_float2(0.f, 0.f);
            for (int l = 0; l < P.L; ++l) {
                float2 accl = make_float2(0.f, 0.f);
                for (int k = 0; k < Kc; ++k) {
                    int64_t plane = ((int64_t)l * P.B + b) * P.C + (P.K ? k : f);
                    const float2 *G = P.grid + plane * P.g.gvol;
                    float2 s = make_float2(0.f, 0.f);
#pragma unroll
                    for (int iz = 0; iz < (D > 2 ? WM : 1); ++iz) {
                        if (iz >= wz_) break;
#pragma unroll
                        for (int iy = 0; iy < (D > 1 ? WM : 1); ++iy) {
                            if (iy >= wy_) break;
                            const float wyz = w[2][iz] * w[1][iy];
                            const float2 *row = G + pz[iz] * nxy + py[iy] * nx;
#pragma unroll
                            for (int ix = 0; ix < WM; ++ix) {
                                if (ix >= wx_) break;
                                s = cfma(wyz * w[0][ix], __ldg(row + px[ix]), s);
                            }
                        }
                    }
                    if (P.K) s = cmul(s, P.basis[(int64_t)f * P.K + k]);
                    accl.x += s.x;
                    accl.y += s.y;
                }
                if (P.tB) accl = cmul(accl, P.tB[(int64_t)l * P.readout + tix]);
                acc.x += accl.x;
                acc.y += accl.y;
            }
            acc.x *= wgt;
            acc.y *= wgt;
            float2 *dst = P.y + b * P.mtot + gs;
            if (P.accumulate) {
                float2 o = *dst;
                acc.x += o.x;
                acc.y += o.y;
            }
            *dst = acc;
        }
    }
}

template <int D, int WM>
__global__ void __launch_bounds__(256) traj_grad_kernel(const InterpParams P) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int Kc = P.K ? P.K : 1;
    const int64_t nx = P.g.nos[0], nxy = (int64_t)P.g.nos[0] * P.g.nos[1];
    const float *cs[3] = {P.cos0, P.cos1, P.cos2};
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < P.mtot; j += stride) {
        const int gs = P.perm[j];
        const int f = P.sframe[j];
        float w[3][WM], dw[3][WM];
        int pp[3][WM];
        int wa[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            wa[a] = a < D ? P.g.w[a] : 1;
            if (a >= D) {
#pragma unroll
                for (int i = 0; i < WM; ++i) { w[a][i] = i == 0 ? 1.f : 0.f; dw[a][i] = 0.f; pp[a][i] = 0; }
                continue;
            }
            float tv[kMaxWidth], td[kMaxWidth];
            long long x0 = axis_weights_deriv(cs[a][j], P.g.w[a], P.g.cart[a], P.g.beta[a], tv, td);
            int sh = P.fft_layout ? P.g.sh[a] : 0;
            int base = pmod(x0 - sh, P.g.nos[a]);
#pragma unroll
            for (int i = 0; i < WM; ++i) {
                w[a][i] = tv[i];
                dw[a][i] = td[i];
                int q = base + i;
                pp[a][i] = q >= P.g.nos[a] ? q - P.g.nos[a] : q;
            }
        }
        const float wgt = P.weight ? P.weight[gs] : 1.0f;
        int tix = 0;
        if (P.tB) tix = (int)((gs - P.frame_off[f]) % P.readout);
        float gacc[3] = {0.f, 0.f, 0.f};
        for (int64_t b = 0; b < P.B; ++b) {
            float2 Dsum[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
            for (int l = 0; l < P.L; ++l) {
                float2 Dl[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
                for (int k = 0; k < Kc; ++k) {
                    int64_t plane = ((int64_t)l * P.B + b) * P.C + (P.K ? k : f);
                    const float2 *G = P.grid + plane * P.g.gvol;
                    float2 d3[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
                    for (int iz = 0; iz < wa[2]; ++iz) {
                        for (int iy = 0; iy < wa[1]; ++iy) {
                            const float2 *row = G + pp[2][iz] * nxy + pp[1][iy] * nx;
#pragma unroll
                            for (int ix = 0; ix < WM; ++ix) {
                                if (ix >= wa[0]) break;
                                float2 h = __ldg(row + pp[0][ix]);
                                d3[0] = cfma(w[2][iz] * w[1][iy] * dw[0][ix], h, d3[0]);
                                if (D > 1) d3[1] = cfma(w[2][iz] * dw[1][iy] * w[0][ix], h, d3[1]);
                                if (D > 2) d3[2] = cfma(dw[2][iz] * w[1][iy] * w[0][ix], h, d3[2]);
                            }
                        }
                    }
#pragma unroll
                    for (int a = 0; a < 3; ++a) {
                        float2 t = P.K ? cmul(d3[a], P.basis[(int64_t)f * P.K + k]) : d3[a];
                        Dl[a].x += t.x;
                        Dl[a].y += t.y;
                    }
                }
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    float2 t = P.tB ? cmul(Dl[a], P.tB[(int64_t)l * P.readout + tix]) : Dl[a];
                    Dsum[a].x += t.x;
                    Dsum[a].y += t.y;
                }
            }
            float2 v = P.y[b * P.mtot + gs];
#pragma unroll
            for (int a = 0; a < 3; ++a) gacc[a] += Dsum[a].x * v.x + Dsum[a].y * v.y;  // Re(conj(D) v)
        }
        for (int a = 0; a < D; ++a) {
            float r = gacc[a] * wgt * P.chain[a];
            float *dst = P.grad + (int64_t)gs * D + a;
            *dst = P.accumulate ? *dst + r : r;
        }
    }
}

void fill_params(const pfb_plan *p, const ApplyDesc &d, bool fft_layout, InterpParams &P) {
    P.g = p->g;
    P.cos0 = p->d_cos[0];
    P.cos1 = p->d_cos[1];
    P.cos2 = p->d_cos[2];
    P.perm = p->d_perm;
    P.sframe = p->d_sframe;
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
    P.fft_layout = fft_layout ? 1 : 0;
    for (int a = 0; a < kMaxDim; ++a) P.chain[a] = (float)p->g.nos[a] / (float)p->g.n[a];
}

int grid_blocks(int64_t n, int threads) {
    int64_t b = (n + threads - 1) / threads;
    int64_t cap = 148LL * 16;
    return (int)std::max<int64_t>(1, std::min(b, cap));
}

}  // namespace

int launch_interp(const pfb_plan *p, const ApplyDesc &d, const float2 *grid, float2 *y,
                  bool fft_layout, cudaStream_t s, bool accumulate) {
    if (p->mtot == 0 || d.batch == 0) return PFB_OK;
    InterpParams P{};
    fill_params(p, d, fft_layout, P);
    P.grid = grid;
    P.y = y;
    P.accumulate = accumulate ? 1 : 0;
    int threads = p->interp_threads;
    int blocks = grid_blocks(p->mtot, threads);
    int wmax = std::max(p->g.w[0], std::max(p->g.w[1], p->g.w[2]));
    bool w4 = wmax <= 4;
    switch (p->g.ndim) {
        case 1: if (w4) interp_kernel<1, 4><<<blocks, threads, 0, s>>>(P); else interp_kernel<1, 8><<<blocks, threads, 0, s>>>(P); break;
        case 2: if (w4) interp_kernel<2, 4><<<blocks, threads, 0, s>>>(P); else interp_kernel<2, 8><<<blocks, threads, 0, s>>>(P); break;
        default: if (w4) interp_kernel<3, 4><<<blocks, threads, 0, s>>>(P); else interp_kernel<3, 8><<<blocks, threads, 0, s>>>(P); break;
    }
    PFB_CHECK_LAUNCH();
    return PFB_OK;
}

int launch_traj_grad(const pfb_plan *p, const ApplyDesc &d, const float2 *grid, const float2 *v,
                     float *grad, bool fft_layout, cudaStream_t s, bool accumulate) {
    if (p->mtot == 0) return PFB_OK;
    InterpParams P{};
    fill_params(p, d, fft_layout, P);
    P.grid = grid;
    P.y = const_cast<float2 *>(v);
    P.grad = grad;
    P.accumulate = accumulate ? 1 : 0;
    int threads = 128;
    int blocks = grid_blocks(p->mtot, threads);
    int wmax = std::max(p->g.w[0], std::max(p->g.w[1], p->g.w[2]));
    bool w4 = wmax <= 4;
    switch (p->g.ndim) {
        case 1: if (w4) traj_grad_kernel<1, 4><<<blocks, threads, 0, s>>>(P); else traj_grad_kernel<1, 8><<<blocks, threads, 0, s>>>(P); break;
        case 2: if (w4) traj_grad_kernel<2, 4><<<blocks, threads, 0, s>>>(P); else traj_grad_kernel<2, 8><<<blocks, threads, 0, s>>>(P); break;
        default: if (w4) traj_grad_kernel<3, 4><<<blocks, threads, 0, s>>>(P); else traj_grad_kernel<3, 8><<<blocks, threads, 0, s>>>(P); break;
    }
    PFB_CHECK_LAUNCH();
    return PFB_OK;
}

}  // namespace pfb
