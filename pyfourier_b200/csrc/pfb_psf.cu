// Plan-time float64 spread for the Toeplitz point-spread function.
//
// The reference builds the PSF of its Toeplitz Gram with its complex64 adjoint
// NUFFT of the sample weights at twice the coordinates
// (src/pyfourier/_sparsegram/_plan.py:201-208).  Here that spread runs in
// float64 -- kernel weights, products and sums -- once per plan; the applies stay
// complex64.  Tap arithmetic is the reference's (_grid/_plan.py:192-210):
// x0 = ceil(c - W/2) from the float32 grid coordinate promoted to float64, grid
// index (x0 + i) mod n_os, weight KB(((x0 + i) - c) / (W/2), beta) with the
// Abramowitz-Stegun I0 forms evaluated in float64 (not rounded to float32
// tables); Cartesian axes take the rounded position with weight 1.
//
// One thread per sample in the caller's (original) order, so that the samples
// of a warp lie along a readout rather than in one crowded tile; float64
// atomics accumulate into the grid.
#include "pfb_common.cuh"

namespace pfb {
namespace {

__device__ __forceinline__ double kb_eval_f64(double u, double beta) {
    if (fabs(u) > 1.0) return 0.0;
    const double a = beta * sqrt(1.0 - u * u);
    if (a < 3.75) {
        const double t = a / 3.75, t2 = t * t;
        return 1.0 + t2 * (3.5156229 + t2 * (3.0899424 + t2 * (1.2067492 +
               t2 * (0.2659732 + t2 * (0.0360768 + t2 * 0.0045813)))));
    }
    const double ti = 3.75 / a;
    return exp(a) / sqrt(a) *
           (0.39894228 + ti * (0.01328592 + ti * (0.00225319 + ti * (-0.00157565 +
            ti * (0.00916281 + ti * (-0.02057706 + ti * (0.02635537 +
            ti * (-0.01647633 + ti * 0.00392377))))))));
}

struct SpreadF64 {
    Geom g;
    const float *cos0, *cos1, *cos2;  // bin-sorted oversampled-grid coordinates
    const int *iperm;                 // sample -> sorted position
    const int *sframe;                // sorted position -> frame
    int64_t mtot;
    int nframes, nch;
    const double2 *vals;              // (nch, mtot) in sample order
    double2 *grid;                    // (nch, nframes, *nos), reference (unshifted) layout
};

__global__ void __launch_bounds__(256) spread_f64_kernel(const SpreadF64 P) {
    const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= P.mtot) return;
    const int j = P.iperm[m];
    const int f = P.sframe[j];
    double wv[3][kMaxWidth];
    int64_t ix[3][kMaxWidth];
    int wa[3] = {1, 1, 1};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        wv[a][0] = 1.0;
        ix[a][0] = 0;
        if (a >= P.g.ndim) continue;
        const float *cs = a == 0 ? P.cos0 : (a == 1 ? P.cos1 : P.cos2);
        const double c = (double)cs[j];
        const int nos = P.g.nos[a];
        if (P.g.cart[a]) {
            ix[a][0] = pmod((long long)rint(c), nos);
            continue;
        }
        const int w = P.g.w[a];
        wa[a] = w;
        const double x0 = ceil(c - 0.5 * (double)w);
        for (int t = 0; t < w; ++t) {
            wv[a][t] = kb_eval_f64(((x0 + t) - c) / (0.5 * (double)w), (double)P.g.beta[a]);
            ix[a][t] = pmod((long long)x0 + t, nos);
        }
    }
    const int64_t nx = P.g.nos[0], nxy = nx * P.g.nos[1];
    for (int ch = 0; ch < P.nch; ++ch) {
        const double2 v = P.vals[(int64_t)ch * P.mtot + m];
        if (v.x == 0.0 && v.y == 0.0) continue;
        double2 *G = P.grid + ((int64_t)ch * P.nframes + f) * P.g.gvol;
        for (int tz = 0; tz < wa[2]; ++tz)
            for (int ty = 0; ty < wa[1]; ++ty) {
                const double wzy = wv[2][tz] * wv[1][ty];
                const int64_t row = ix[2][tz] * nxy + ix[1][ty] * nx;
                for (int tx = 0; tx < wa[0]; ++tx) {
                    const double w = wzy * wv[0][tx];
                    atomicAdd(&G[row + ix[0][tx]].x, w * v.x);
                    atomicAdd(&G[row + ix[0][tx]].y, w * v.y);
                }
            }
    }
}

}  // namespace
}  // namespace pfb

using namespace pfb;

extern "C" int pfb_spread_f64(pfb_plan *p, const void *values, int nch, void *grid, void *stream) {
    if (!p || !values || !grid || nch < 1) return fail(PFB_ERR_INVALID, "bad argument");
    if (p->mtot == 0) return PFB_OK;
    if (p->mtot > INT32_MAX) return fail(PFB_ERR_UNSUPPORTED, "more than 2^31 samples");
    int prev = -1;
    PFB_CUDA_TRY(cudaGetDevice(&prev));
    if (prev != p->device) PFB_CUDA_TRY(cudaSetDevice(p->device));
    SpreadF64 P{};
    P.g = p->g;
    P.cos0 = p->d_cos[0];
    P.cos1 = p->d_cos[1];
    P.cos2 = p->d_cos[2];
    P.iperm = p->d_iperm;
    P.sframe = p->d_sframe;
    P.mtot = p->mtot;
    P.nframes = p->nframes;
    P.nch = nch;
    P.vals = static_cast<const double2 *>(values);
    P.grid = static_cast<double2 *>(grid);
    const unsigned blocks = (unsigned)((p->mtot + 255) / 256);
    spread_f64_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(P);
    cudaError_t e = cudaGetLastError();
    if (prev != p->device) cudaSetDevice(prev);
    if (e != cudaSuccess) return fail(PFB_ERR_CUDA, std::string("spread_f64_kernel: ") + cudaGetErrorString(e));
    return PFB_OK;
}
