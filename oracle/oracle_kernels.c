/*
 * CPU oracle for the pyfourier NUFFT hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * This file is a plain-C restatement of the reference's Numba CPU kernels.
 * It exists to check the CUDA product path and to time a CPU baseline; the
 * product library never links, loads or calls it.  Only tests/, the smoke
 * check in __graft_entry__.py and the cpu-baseline leg of bench.py use it.
 *
 * Parity is pinned by the .npz fixtures in tests/golden, which were produced by running the
 * reference's own Numba kernels (tests/golden/make_golden.py).
 *
 * Reference functions restated here (paths inside the pyfourier project):
 *   orc_kaiser_bessel          src/pyfourier/_subroutines/_grid/_plan.py:157-189
 *   orc_kernel_scaling         src/pyfourier/_subroutines/_grid/_plan.py:118-141
 *   orc_prepare_interpolator   src/pyfourier/_subroutines/_grid/_plan.py:192-210
 *   orc_grid                   src/pyfourier/_subroutines/_grid/_noncart2cart/_{1,2,3}D.py (_grid_nb)
 *   orc_grid_subspace          src/pyfourier/_subroutines/_grid/_noncart2cart/_{1,2,3}D_subspace.py
 *   orc_degrid                 src/pyfourier/_subroutines/_grid/_cart2noncart/_{1,2,3}D.py (_degrid_nb)
 *   orc_degrid_subspace        src/pyfourier/_subroutines/_grid/_cart2noncart/_{1,2,3}D_subspace.py
 *
 * The 1D and 2D reference kernels are the 3D loop nest with unit-width outer
 * axes; here every kernel is written once as the 3D nest and the caller passes
 * width-1 tables (index 0, value 1) for the missing axes.  Multiplying by the
 * unit value is exact, so the arithmetic is unchanged.
 *
 * Parallel structure mirrors the reference's nb.prange loops:
 *   spread (grid): parallel over (frame, batch) or (coeff, batch), serial over samples;
 *   interp (degrid): parallel over (frame, batch, sample).
 */
#include <math.h>
#include <stdint.h>
#include <complex.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef float complex cf32;

/* Kaiser-Bessel kernel with the Abramowitz-Stegun 9.8.1 / 9.8.2 polynomial
 * approximation of I0; zero outside |x| <= 1. */
double orc_kaiser_bessel(double x, double beta)
{
    if (fabs(x) > 1.0)
        return 0.0;
    double a = beta * sqrt(1.0 - x * x);
    double t = a / 3.75;
    if (a < 3.75) {
        double t2 = t * t;
        return 1.0 + 3.5156229 * t2 + 3.0899424 * pow(t, 4) + 1.2067492 * pow(t, 6) +
               0.2659732 * pow(t, 8) + 0.0360768 * pow(t, 10) + 0.0045813 * pow(t, 12);
    }
    return pow(a, -0.5) * exp(a) *
           (0.39894228 + 0.01328592 * pow(t, -1) + 0.00225319 * pow(t, -2) -
            0.00157565 * pow(t, -3) + 0.00916281 * pow(t, -4) - 0.02057706 * pow(t, -5) +
            0.02635537 * pow(t, -6) - 0.01647633 * pow(t, -7) + 0.00392377 * pow(t, -8));
}

/* Sum over the W^d node-centred kernel samples (product over axes). */
double orc_kernel_scaling(int ndim, const int *width, const double *beta)
{
    double vals[3][16];
    int w[3] = {1, 1, 1};
    for (int ax = 0; ax < ndim; ++ax) {
        w[ax] = width[ax];
        double start = ceil(-width[ax] / 2.0);
        for (int e = 0; e < width[ax]; ++e)
            vals[ax][e] = (width[ax] == 1) ? 1.0
                                           : orc_kaiser_bessel((start + e) / (width[ax] / 2.0), beta[ax]);
    }
    for (int ax = ndim; ax < 3; ++ax)
        vals[ax][0] = 1.0;
    double s = 0.0;
    for (int i = 0; i < w[0]; ++i)
        for (int j = 0; j < w[1]; ++j)
            for (int k = 0; k < w[2]; ++k)
                s += vals[0][i] * vals[1][j] * vals[2][k];
    return s;
}

/* Per-axis interpolator tables: value (npts, W) float32, index (npts, W) int32. */
void orc_prepare_interpolator(float *value, int32_t *index, const float *coord, int64_t npts,
                              int width, double beta, int grid_shape)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < npts; ++i) {
        double c = (double)coord[i];
        double x0 = ceil(c - width / 2.0);
        for (int xi = 0; xi < width; ++xi) {
            double v = orc_kaiser_bessel(((x0 + xi) - c) / (width / 2.0), beta);
            value[i * width + xi] = (float)v;
            /* Python-sign modulo: result in [0, grid_shape) */
            double m = fmod(x0 + xi, (double)grid_shape);
            if (m < 0)
                m += grid_shape;
            index[i * width + xi] = (int32_t)m;
        }
    }
}

/* Spread: cart (F, B, nz, ny, nx) += taps * noncart (F, B, M).
 * Tables are (F, M, w_ax) in (z, y, x) order. */
void orc_grid(cf32 *cart, const cf32 *noncart, const float *zval, const float *yval,
              const float *xval, const int32_t *zidx, const int32_t *yidx, const int32_t *xidx,
              int64_t nframes, int64_t batch, int64_t npts, int wz, int wy, int wx, int nz, int ny,
              int nx)
{
    const int64_t plane = (int64_t)nz * ny * nx;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t i = 0; i < nframes * batch; ++i) {
        int64_t frame = i / batch, b = i % batch;
        cf32 *out = cart + (frame * batch + b) * plane;
        const cf32 *in = noncart + (frame * batch + b) * npts;
        for (int64_t p = 0; p < npts; ++p) {
            int64_t t = frame * npts + p;
            for (int iz = 0; iz < wz; ++iz) {
                int32_t idz = zidx[t * wz + iz];
                float vz = zval[t * wz + iz];
                for (int iy = 0; iy < wy; ++iy) {
                    int32_t idy = yidx[t * wy + iy];
                    float vy = vz * yval[t * wy + iy];
                    for (int ix = 0; ix < wx; ++ix) {
                        int32_t idx = xidx[t * wx + ix];
                        float v = vy * xval[t * wx + ix];
                        out[((int64_t)idz * ny + idy) * nx + idx] += v * in[p];
                    }
                }
            }
        }
    }
}

/* Spread with subspace projection: cart (K, B, nz, ny, nx) += v * basis[k, f] * noncart (F, B, M).
 * basis is (K, F) -- the reference conj-transposes the user's (F, K) basis first. */
void orc_grid_subspace(cf32 *cart, const cf32 *noncart, const float *zval, const float *yval,
                       const float *xval, const int32_t *zidx, const int32_t *yidx,
                       const int32_t *xidx, const cf32 *basis, int64_t ncoeff, int64_t nframes,
                       int64_t batch, int64_t npts, int wz, int wy, int wx, int nz, int ny, int nx)
{
    const int64_t plane = (int64_t)nz * ny * nx;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t i = 0; i < ncoeff * batch; ++i) {
        int64_t coeff = i / batch, b = i % batch;
        cf32 *out = cart + (coeff * batch + b) * plane;
        for (int64_t frame = 0; frame < nframes; ++frame) {
            const cf32 *in = noncart + (frame * batch + b) * npts;
            cf32 bk = basis[coeff * nframes + frame];
            for (int64_t p = 0; p < npts; ++p) {
                int64_t t = frame * npts + p;
                for (int iz = 0; iz < wz; ++iz) {
                    int32_t idz = zidx[t * wz + iz];
                    float vz = zval[t * wz + iz];
                    for (int iy = 0; iy < wy; ++iy) {
                        int32_t idy = yidx[t * wy + iy];
                        float vy = vz * yval[t * wy + iy];
                        for (int ix = 0; ix < wx; ++ix) {
                            int32_t idx = xidx[t * wx + ix];
                            float v = vy * xval[t * wx + ix];
                            out[((int64_t)idz * ny + idy) * nx + idx] += v * bk * in[p];
                        }
                    }
                }
            }
        }
    }
}

/* Interp: noncart (F, B, M) += taps * cart (F, B, nz, ny, nx). */
void orc_degrid(cf32 *noncart, const cf32 *cart, const float *zval, const float *yval,
                const float *xval, const int32_t *zidx, const int32_t *yidx, const int32_t *xidx,
                int64_t nframes, int64_t batch, int64_t npts, int wz, int wy, int wx, int nz, int ny,
                int nx)
{
    const int64_t plane = (int64_t)nz * ny * nx;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nframes * batch * npts; ++i) {
        int64_t frame = i / (batch * npts);
        int64_t rem = i % (batch * npts);
        int64_t b = rem / npts, p = rem % npts;
        int64_t t = frame * npts + p;
        const cf32 *g = cart + (frame * batch + b) * plane;
        cf32 acc = noncart[i];
        for (int iz = 0; iz < wz; ++iz) {
            int32_t idz = zidx[t * wz + iz];
            float vz = zval[t * wz + iz];
            for (int iy = 0; iy < wy; ++iy) {
                int32_t idy = yidx[t * wy + iy];
                float vy = vz * yval[t * wy + iy];
                for (int ix = 0; ix < wx; ++ix) {
                    int32_t idx = xidx[t * wx + ix];
                    float v = vy * xval[t * wx + ix];
                    acc += v * g[((int64_t)idz * ny + idy) * nx + idx];
                }
            }
        }
        noncart[i] = acc;
    }
}

/* Interp with adjoint subspace projection:
 * noncart (F, B, M) += v * basis_adj[f, k] * cart (K, B, ...); basis_adj is (F, K). */
void orc_degrid_subspace(cf32 *noncart, const cf32 *cart, const float *zval, const float *yval,
                         const float *xval, const int32_t *zidx, const int32_t *yidx,
                         const int32_t *xidx, const cf32 *basis_adj, int64_t ncoeff,
                         int64_t nframes, int64_t batch, int64_t npts, int wz, int wy, int wx,
                         int nz, int ny, int nx)
{
    const int64_t plane = (int64_t)nz * ny * nx;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nframes * batch * npts; ++i) {
        int64_t frame = i / (batch * npts);
        int64_t rem = i % (batch * npts);
        int64_t b = rem / npts, p = rem % npts;
        int64_t t = frame * npts + p;
        cf32 acc = noncart[i];
        for (int iz = 0; iz < wz; ++iz) {
            int32_t idz = zidx[t * wz + iz];
            float vz = zval[t * wz + iz];
            for (int iy = 0; iy < wy; ++iy) {
                int32_t idy = yidx[t * wy + iy];
                float vy = vz * yval[t * wy + iy];
                for (int ix = 0; ix < wx; ++ix) {
                    int32_t idx = xidx[t * wx + ix];
                    float v = vy * xval[t * wx + ix];
                    int64_t off = ((int64_t)idz * ny + idy) * nx + idx;
                    for (int64_t k = 0; k < ncoeff; ++k)
                        acc += v * basis_adj[frame * ncoeff + k] * cart[(k * batch + b) * plane + off];
                }
            }
        }
        noncart[i] = acc;
    }
}

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* Float64 spread for the Toeplitz PSF (plan time).  Same tap arithmetic as
 * orc_prepare_interpolator (x0 = ceil(c - W/2), index (x0 + i) mod n_os,
 * weight KB(((x0 + i) - c) / (W/2))) with the weights kept in float64 instead of
 * being rounded to float32 tables; Cartesian axes (cart_xyz[a] != 0) take the
 * rounded position with weight 1.  coord (F, M, ndim) float32 in (x, y, z)
 * order; noncart (F, B, M) complex128; cart (F, B, *os) complex128 accumulated.
 * Parallel over (frame, batch) like orc_grid. */
void orc_grid_f64(double complex *cart, const double complex *noncart, const float *coord, int ndim,
                  int64_t nframes, int64_t batch, int64_t npts, const int *width_xyz, const double *beta_xyz,
                  const int *nos_xyz, const int *cart_xyz)
{
    int w[3] = {1, 1, 1}, nos[3] = {1, 1, 1}, ca[3] = {1, 1, 1};
    double beta[3] = {0, 0, 0};
    for (int a = 0; a < ndim; ++a) {
        w[a] = cart_xyz[a] ? 1 : width_xyz[a];
        nos[a] = nos_xyz[a];
        beta[a] = beta_xyz[a];
        ca[a] = cart_xyz[a];
    }
    const int64_t plane = (int64_t)nos[0] * nos[1] * nos[2];
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t i = 0; i < nframes * batch; ++i) {
        int64_t frame = i / batch, b = i % batch;
        double complex *out = cart + (frame * batch + b) * plane;
        const double complex *in = noncart + (frame * batch + b) * npts;
        for (int64_t p = 0; p < npts; ++p) {
            const float *c = coord + (frame * npts + p) * ndim;
            double wv[3][16];
            int64_t ix[3][16];
            for (int a = 0; a < 3; ++a) {
                if (a >= ndim) {
                    wv[a][0] = 1.0;
                    ix[a][0] = 0;
                    continue;
                }
                double cc = (double)c[a];
                if (ca[a]) {
                    double m = fmod(rint(cc), (double)nos[a]);
                    if (m < 0)
                        m += nos[a];
                    wv[a][0] = 1.0;
                    ix[a][0] = (int64_t)m;
                    continue;
                }
                double x0 = ceil(cc - w[a] / 2.0);
                for (int t = 0; t < w[a]; ++t) {
                    wv[a][t] = orc_kaiser_bessel(((x0 + t) - cc) / (w[a] / 2.0), beta[a]);
                    double m = fmod(x0 + t, (double)nos[a]);
                    if (m < 0)
                        m += nos[a];
                    ix[a][t] = (int64_t)m;
                }
            }
            const double complex v = in[p];
            for (int tz = 0; tz < w[2]; ++tz)
                for (int ty = 0; ty < w[1]; ++ty) {
                    const double wzy = wv[2][tz] * wv[1][ty];
                    const int64_t row = (ix[2][tz] * nos[1] + ix[1][ty]) * nos[0];
                    for (int tx = 0; tx < w[0]; ++tx)
                        out[row + ix[0][tx]] += (wzy * wv[0][tx]) * v;
                }
        }
    }
}
