// Image-side kernels around the oversampled-grid FFT, and the Toeplitz Gram
// pad / mix / crop.  All are HBM-bound streaming kernels: one read of the
// source and one write of the destination, with the index shifts of the
// centred FFT folded into the address computation instead of extra copies.
//
// Centred FFT (src/pyfourier/_subroutines/_fft.py:72-79) of a centred zero-pad
// (src/pyfourier/_subroutines/_resize.py:16-42): image pixel r (0 <= r < N) is
// stored at FFT position (r - N//2) mod n_os, and every other position is zero.
// The inverse path reads the same positions back (fftshift + centred crop).
// Deapodisation (src/pyfourier/_subroutines/_apod.py:16-46) multiplies each
// pixel by the per-axis weights, precomputed in float64 at plan time.
#include "pfb_common.cuh"

namespace pfb {

namespace {

struct PadParams {
    Geom g;
    const float2 *img;
    float2 *grid;
    const float *apod0, *apod1, *apod2;
    const float2 *Cl;      // (L, nvol) or null
    int64_t B;
    int C;
    int L;
    float factor;
    int accumulate;
};

// grid plane (l, b, c), FFT-layout position p -> image pixel r = (p + N//2) mod n_os, valid if r < N
__global__ void deapod_pad_kernel(const PadParams P) {
    const int64_t gvol = P.g.gvol;
    const int64_t total = (int64_t)P.L * P.B * P.C * gvol;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += stride) {
        int64_t plane = e / gvol;
        int64_t pos = e - plane * gvol;
        int p0 = (int)(pos % P.g.nos[0]);
        int64_t rest = pos / P.g.nos[0];
        int p1 = (int)(rest % P.g.nos[1]);
        int p2 = (int)(rest / P.g.nos[1]);
        int r0 = p0 + P.g.n[0] / 2; r0 = r0 >= P.g.nos[0] ? r0 - P.g.nos[0] : r0;
        int r1 = p1 + P.g.n[1] / 2; r1 = r1 >= P.g.nos[1] ? r1 - P.g.nos[1] : r1;
        int r2 = p2 + P.g.n[2] / 2; r2 = r2 >= P.g.nos[2] ? r2 - P.g.nos[2] : r2;
        float2 out = make_float2(0.f, 0.f);
        if (r0 < P.g.n[0] && r1 < P.g.n[1] && r2 < P.g.n[2]) {
            int64_t rl = ((int64_t)r2 * P.g.n[1] + r1) * P.g.n[0] + r0;
            int64_t bc = plane % (P.B * P.C);   // (b, c) image plane
            int l = (int)(plane / (P.B * P.C));
            float2 v = P.img[bc * P.g.nvol + rl];
            float a = P.factor;
            if (P.apod0) a *= P.apod0[r0];
            if (P.apod1) a *= P.apod1[r1];
            if (P.apod2) a *= P.apod2[r2];
            if (P.Cl) v = cmul(v, P.Cl[(int64_t)l * P.g.nvol + rl]);
            out = make_float2(v.x * a, v.y * a);
        }
        P.grid[e] = out;
    }
}

// image (b, c, r) = factor * apod(r) * sum_l conj(C_l(r)) * grid[(l, b, c), (r - N//2) mod n_os]
__global__ void crop_deapod_kernel(const PadParams P) {
    const int64_t nvol = P.g.nvol;
    const int64_t total = P.B * P.C * nvol;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += stride) {
        int64_t bc = e / nvol;
        int64_t rl = e - bc * nvol;
        int r0 = (int)(rl % P.g.n[0]);
        int64_t rest = rl / P.g.n[0];
        int r1 = (int)(rest % P.g.n[1]);
        int r2 = (int)(rest / P.g.n[1]);
        int p0 = r0 - P.g.n[0] / 2; p0 = p0 < 0 ? p0 + P.g.nos[0] : p0;
        int p1 = r1 - P.g.n[1] / 2; p1 = p1 < 0 ? p1 + P.g.nos[1] : p1;
        int p2 = r2 - P.g.n[2] / 2; p2 = p2 < 0 ? p2 + P.g.nos[2] : p2;
        int64_t pos = ((int64_t)p2 * P.g.nos[1] + p1) * P.g.nos[0] + p0;
        float2 acc = make_float2(0.f, 0.f);
        for (int l = 0; l < P.L; ++l) {
            float2 v = P.grid[((int64_t)l * P.B * P.C + bc) * P.g.gvol + pos];
            if (P.Cl) v = cmulc(v, P.Cl[(int64_t)l * nvol + rl]);
            acc.x += v.x;
            acc.y += v.y;
        }
        float a = P.factor;
        if (P.apod0) a *= P.apod0[r0];
        if (P.apod1) a *= P.apod1[r1];
        if (P.apod2) a *= P.apod2[r2];
        acc.x *= a;
        acc.y *= a;
        if (P.accumulate) {
            float2 o = P.img[e];
            acc.x += o.x;
            acc.y += o.y;
        }
        const_cast<float2 *>(P.img)[e] = acc;
    }
}

// Uncentred embedding (the Gram's centred zero-pad followed by an uncentred FFT,
// src/pyfourier/_sparsegram/_sparsegram.py:63-67): pixel r at r + (n_os//2 - N//2).
struct EmbedParams {
    int n[3], nos[3], off[3];
    int64_t nvol, gvol, nplanes;
    const float2 *src;
    float2 *dst;
    float factor;
    const float2 *Cl;  // (L, nvol) B0 spatial coefficients or null
    int L;             // segments (grid planes = L * bk)
    int64_t bk;        // image planes per segment
};

// One CTA per grid row (plane, z, y) at a time: the row's index split is done once,
// the threads walk x (no 64-bit division per element).
__global__ void __launch_bounds__(128) embed_kernel(const EmbedParams P) {
    const int64_t rows_per_plane = (int64_t)P.nos[1] * P.nos[2];
    const int64_t nrows = P.nplanes * rows_per_plane;
    for (int64_t row = blockIdx.x; row < nrows; row += gridDim.x) {
        const int64_t plane = row / rows_per_plane;
        const int rr = (int)(row - plane * rows_per_plane);
        const int q2 = rr / P.nos[1], q1 = rr - q2 * P.nos[1];
        const int r1 = q1 - P.off[1], r2 = q2 - P.off[2];
        float2 *d = P.dst + row * P.nos[0];
        if (r1 < 0 || r1 >= P.n[1] || r2 < 0 || r2 >= P.n[2]) {
            for (int q0 = threadIdx.x; q0 < P.nos[0]; q0 += blockDim.x) d[q0] = make_float2(0.f, 0.f);
            continue;
        }
        // grid plane (l, image plane); the segment multiplies by C_l
        const int64_t l = plane / P.bk, ip = plane - l * P.bk;
        const int64_t rl0 = ((int64_t)r2 * P.n[1] + r1) * P.n[0];
        const float2 *src = P.src + ip * P.nvol + rl0;
        const float2 *cl = P.Cl ? P.Cl + l * P.nvol + rl0 : nullptr;
        for (int q0 = threadIdx.x; q0 < P.nos[0]; q0 += blockDim.x) {
            const int r0 = q0 - P.off[0];
            float2 v = make_float2(0.f, 0.f);
            if (r0 >= 0 && r0 < P.n[0]) {
                v = src[r0];
                if (cl) v = cmul(v, cl[r0]);
            }
            d[q0] = v;
        }
    }
}

// One CTA per image row (plane, z, y) at a time, as embed_kernel.
__global__ void __launch_bounds__(128) extract_kernel(const EmbedParams P) {
    const int64_t rows_per_plane = (int64_t)P.n[1] * P.n[2];
    const int64_t nrows = P.nplanes * rows_per_plane;
    for (int64_t row = blockIdx.x; row < nrows; row += gridDim.x) {
        const int64_t plane = row / rows_per_plane;
        const int rr = (int)(row - plane * rows_per_plane);
        const int r2 = rr / P.n[1], r1 = rr - r2 * P.n[1];
        const int64_t pos0 = ((int64_t)(r2 + P.off[2]) * P.nos[1] + (r1 + P.off[1])) * P.nos[0] + P.off[0];
        const int64_t rl0 = (int64_t)rr * P.n[0];
        float2 *d = P.dst + row * P.n[0];
        for (int r0 = threadIdx.x; r0 < P.n[0]; r0 += blockDim.x) {
            // sum over segments of conj(C_l) times segment l's plane
            float2 v = make_float2(0.f, 0.f);
            for (int l = 0; l < P.L; ++l) {
                float2 g = P.src[((int64_t)l * P.bk + plane) * P.gvol + pos0 + r0];
                if (P.Cl) g = cmulc(g, P.Cl[(int64_t)l * P.nvol + rl0 + r0]);
                v.x += g.x;
                v.y += g.y;
            }
            d[r0] = make_float2(v.x * P.factor, v.y * P.factor);
        }
    }
}

// Per-voxel K x K mix, out[v] = scale * T[v] @ in[v] (T row-major per voxel),
// for every batch item; the K-vector of a voxel lives in K planes of the grid.
// The evident intent of _bmatvec/_bdot.py:16-115 (the shipped _dot_nb computes
// in * colsum(T), not the product).  blockIdx.y strides over batch items, so
// small grids still fill the GPU; T (K*K per voxel) is re-read per y-slice and
// stays in L2.
template <int KM>
__global__ void __launch_bounds__(256) mix_kernel(int64_t gvol, int K, int64_t batch,
                                                  const float2 *__restrict__ T, float2 *__restrict__ grid,
                                                  float scale) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < gvol; v += stride) {
        float2 t[KM][KM];
#pragma unroll
        for (int i = 0; i < KM; ++i)
#pragma unroll
            for (int j = 0; j < KM; ++j) {
                float2 e = (i < K && j < K) ? __ldg(T + (v * K + i) * K + j) : make_float2(0.f, 0.f);
                t[i][j] = make_float2(e.x * scale, e.y * scale);
            }
        for (int64_t b = blockIdx.y; b < batch; b += gridDim.y) {
            float2 x[KM];
#pragma unroll
            for (int j = 0; j < KM; ++j)
                x[j] = j < K ? grid[(b * K + j) * gvol + v] : make_float2(0.f, 0.f);
#pragma unroll
            for (int i = 0; i < KM; ++i) {
                if (i >= K) break;
                float2 acc = make_float2(0.f, 0.f);
#pragma unroll
                for (int j = 0; j < KM; ++j) {
                    float2 p = cmul(t[i][j], x[j]);
                    acc.x += p.x;
                    acc.y += p.y;
                }
                grid[(b * K + i) * gvol + v] = acc;
            }
        }
    }
}

// Elementwise multiply (no subspace): plane (b, c) *= scale * T[c] (T has C planes).
__global__ void diag_kernel(int64_t gvol, int C, int64_t batch, const float2 *__restrict__ T,
                            float2 *__restrict__ grid, float scale) {
    const int64_t total = batch * C * gvol;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += stride) {
        int64_t cv = e % (C * gvol);
        float2 r = cmul(__ldg(T + cv), grid[e]);
        grid[e] = make_float2(r.x * scale, r.y * scale);
    }
}

int blocks_for(int64_t n, int threads) {
    int64_t b = (n + threads - 1) / threads;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, 148LL * 32));
}

}  // namespace

int launch_deapod_pad(const pfb_plan *p, const ApplyDesc &d, const float2 *img, float2 *grid,
                      float factor, cudaStream_t s) {
    PadParams P{};
    P.g = p->g;
    P.img = img;
    P.grid = grid;
    P.apod0 = p->d_apod[0];
    P.apod1 = p->d_apod[1];
    P.apod2 = p->d_apod[2];
    P.Cl = d.b0_space;
    P.B = d.batch;
    P.C = d.ncoeff;
    P.L = d.nseg;
    P.factor = factor;
    int64_t total = (int64_t)d.nseg * d.batch * d.ncoeff * p->g.gvol;
    if (total == 0) return PFB_OK;
    deapod_pad_kernel<<<blocks_for(total, 256), 256, 0, s>>>(P);
    PFB_CHECK_LAUNCH();
    return PFB_OK;
}

int launch_crop_deapod(const pfb_plan *p, const ApplyDesc &d, const float2 *grid, float2 *img,
                       float factor, cudaStream_t s, bool accumulate) {
    PadParams P{};
    P.g = p->g;
    P.img = img;
    P.grid = const_cast<float2 *>(grid);
    P.apod0 = p->d_apod[0];
    P.apod1 = p->d_apod[1];
    P.apod2 = p->d_apod[2];
    P.Cl = d.b0_space;
    P.B = d.batch;
    P.C = d.ncoeff;
    P.L = d.nseg;
    P.factor = factor;
    P.accumulate = accumulate ? 1 : 0;
    int64_t total = d.batch * d.ncoeff * p->g.nvol;
    if (total == 0) return PFB_OK;
    crop_deapod_kernel<<<blocks_for(total, 256), 256, 0, s>>>(P);
    PFB_CHECK_LAUNCH();
    return PFB_OK;
}

static void fill_embed(int ndim, const int *n, const int *nos, EmbedParams &P) {
    P.nvol = P.gvol = 1;
    for (int a = 0; a < 3; ++a) {
        P.n[a] = a < ndim ? n[a] : 1;
        P.nos[a] = a < ndim ? nos[a] : 1;
        // _resize.py:23-24: oshift = max(o//2 - i//2, 0)
        P.off[a] = std::max(P.nos[a] / 2 - P.n[a] / 2, 0);
        P.nvol *= P.n[a];
        P.gvol *= P.nos[a];
    }
}

int launch_embed(int ndim, const int *n, const int *nos, const float2 *img, float2 *grid,
                 int64_t nplanes, const float2 *Cl, int L, cudaStream_t s) {
    EmbedParams P{};
    fill_embed(ndim, n, nos, P);
    P.Cl = Cl;
    P.L = L;
    P.bk = nplanes;
    nplanes *= L;
    P.nplanes = nplanes;
    P.src = img;
    P.dst = grid;
    P.factor = 1.f;
    const int64_t rows = nplanes * P.nos[1] * P.nos[2];
    if (rows == 0 || P.nos[0] == 0) return PFB_OK;
    embed_kernel<<<(unsigned)std::min<int64_t>(rows, 1 << 20), 128, 0, s>>>(P);
    PFB_CHECK_LAUNCH();
    return PFB_OK;
}

int launch_extract(int ndim, const int *n, const int *nos, const float2 *grid, float2 *img,
                   int64_t nplanes, float factor, const float2 *Cl, int L, cudaStream_t s) {
    EmbedParams P{};
    fill_embed(ndim, n, nos, P);
    P.Cl = Cl;
    P.L = L;
    P.bk = nplanes;
    P.nplanes = nplanes;
    P.src = grid;
    P.dst = img;
    P.factor = factor;
    const int64_t rows = nplanes * P.n[1] * P.n[2];
    if (rows == 0 || P.n[0] == 0) return PFB_OK;
    extract_kernel<<<(unsigned)std::min<int64_t>(rows, 1 << 20), 128, 0, s>>>(P);
    PFB_CHECK_LAUNCH();
    return PFB_OK;
}

int launch_mix(int64_t gvol, int K, int lowrank, int64_t batch, const float2 *T, float2 *grid,
               cudaStream_t s, float scale) {
    if (gvol == 0 || batch == 0) return PFB_OK;
    if (!lowrank) {
        diag_kernel<<<blocks_for(batch * K * gvol, 256), 256, 0, s>>>(gvol, K, batch, T, grid, scale);
        PFB_CHECK_LAUNCH();
        return PFB_OK;
    }
    if (K > 8) return fail(PFB_ERR_UNSUPPORTED, "subspace size K > 8 is not supported by the Gram mix");
    const int threads = K <= 4 ? 256 : 128;
    const int bx = blocks_for(gvol, threads);
    // batch slices so that about 8 blocks per SM run (148 SMs)
    const int by = (int)std::max<int64_t>(1, std::min<int64_t>(batch, (148LL * 8 + bx - 1) / bx));
    dim3 grd(bx, by);
    if (K <= 2)
        mix_kernel<2><<<grd, threads, 0, s>>>(gvol, K, batch, T, grid, scale);
    else if (K <= 4)
        mix_kernel<4><<<grd, threads, 0, s>>>(gvol, K, batch, T, grid, scale);
    else
        mix_kernel<8><<<grd, threads, 0, s>>>(gvol, K, batch, T, grid, scale);
    PFB_CHECK_LAUNCH();
    return PFB_OK;
}

}  // namespace pfb
