// Plan construction: coordinate scaling, tile binning and the stable integer
// counting sort of samples by (tile, edge code, frame) (pfb_sort.cu).  Plan-time only; allocations and host syncs here
// are intended.
//
// Reference behaviour restated (paths inside the pyfourier project):
//   coordinate scaling   src/pyfourier/_subroutines/_traj.py:57-65 (float32 ops)
//   first tap x0         src/pyfourier/_subroutines/_grid/_plan.py:201 (float64 ceil)
//   tap index            src/pyfourier/_subroutines/_grid/_plan.py:210 ((x0+i) mod n_os)
//   kernel scaling       src/pyfourier/_subroutines/_grid/_plan.py:118-141
//   deapodisation        src/pyfourier/_subroutines/_apod.py:24-44 (here in float64)
#include <algorithm>
#include <cmath>

#include "pfb_common.cuh"

namespace pfb {

namespace {

struct ScaleParams {
    int ndim;
    int nframes;
    int64_t mtot;
    float s[kMaxDim];
    float shift[kMaxDim];
    int nos[kMaxDim];
    int w[kMaxDim];
    int cart[kMaxDim];
    int tile[kMaxDim];
    int toff[kMaxDim];
    int nbins[kMaxDim];
};

__global__ void scale_and_key_kernel(ScaleParams P, const float *__restrict__ coord,
                                     const int64_t *__restrict__ frame_off, float *__restrict__ cos_out,
                                     int *__restrict__ keys, int *__restrict__ vals, int *__restrict__ bad) {
    int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= P.mtot) return;
    // frame of sample g: largest f with frame_off[f] <= g
    int lo = 0, hi = P.nframes;  // invariant frame_off[lo] <= g < frame_off[hi]
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (frame_off[mid] <= g) lo = mid; else hi = mid;
    }
    int bin = 0;
    int stride = 1;
    int code = 0;  // bit a: the kernel footprint crosses into the next tile along axis a
    for (int a = 0; a < P.ndim; ++a) {
        float c = coord[g * P.ndim + a];
        // float32 multiply then add, each rounded (no contraction into an FMA)
        float cos_ = __fadd_rn(__fmul_rn(c, P.s[a]), P.shift[a]);
        cos_out[(int64_t)a * P.mtot + g] = cos_;
        if (!isfinite(cos_) || fabsf(cos_) > 1.0e9f) {
            atomicExch(bad, 1);
            cos_ = 0.0f;
        }
        long long x0 = start_index(cos_, P.w[a], P.cart[a]);
        int x0m = pmod(x0, P.nos[a]);
        // tile tb covers [tb * tile - toff, (tb + 1) * tile - toff) clipped to the grid
        const int tb = (x0m + P.toff[a]) / P.tile[a];
        bin += tb * stride;
        stride *= P.nbins[a];
        const int org = max(tb * P.tile[a] - P.toff[a], 0);
        const int text = min((tb + 1) * P.tile[a] - P.toff[a], P.nos[a]) - org;
        if (P.nbins[a] > 1 && x0m - org + P.w[a] - 1 >= text) code |= 1 << a;
    }
    // sort key: (tile, edge code) major, frame minor
    keys[g] = ((bin << P.ndim) | code) * P.nframes + lo;
    vals[g] = (int)g;
}

__global__ void gather_sorted_kernel(int ndim, int64_t mtot, int nframes, const float *__restrict__ cos_in,
                                     const int *__restrict__ perm, const int *__restrict__ keys_sorted,
                                     float *__restrict__ c0, float *__restrict__ c1, float *__restrict__ c2,
                                     int *__restrict__ sframe, int *__restrict__ iperm) {
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= mtot) return;
    int g = perm[j];
    iperm[g] = (int)j;
    c0[j] = cos_in[g];
    if (ndim > 1) c1[j] = cos_in[mtot + g];
    if (ndim > 2) c2[j] = cos_in[2 * mtot + g];
    sframe[j] = keys_sorted[j] % nframes;
}

// bin_start[k] = first sorted position whose key >= k (lower bound), k in [0, nkeys].
__global__ void bin_start_kernel(const int *__restrict__ keys_sorted, int64_t mtot, int nkeys,
                                 int *__restrict__ bin_start) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k > nkeys) return;
    int64_t lo = 0, hi = mtot;
    while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if (keys_sorted[mid] < k) lo = mid + 1; else hi = mid;
    }
    bin_start[k] = (int)lo;
}

// Interpolator tables in the reference's layout (original sample order).
__global__ void tables_kernel(Geom g, int axis, int64_t mtot, const float *__restrict__ cos_sorted,
                              const int *__restrict__ perm, int32_t *__restrict__ index,
                              float *__restrict__ value) {
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= mtot) return;
    int gi = perm[j];
    float wv[kMaxWidth];
    long long x0 = axis_weights(cos_sorted[j], g.w[axis], g.cart[axis], g.beta[axis], wv);
    int w = g.w[axis];
    for (int i = 0; i < w; ++i) {
        index[(int64_t)gi * w + i] = pmod(x0 + i, g.nos[axis]);
        value[(int64_t)gi * w + i] = wv[i];
    }
}

double kb_host(double x, double beta) {
    if (std::fabs(x) > 1.0) return 0.0;
    double a = beta * std::sqrt(1.0 - x * x);
    double t = a / 3.75;
    if (a < 3.75) {
        double t2 = t * t;
        return 1.0 + t2 * (3.5156229 + t2 * (3.0899424 + t2 * (1.2067492 +
               t2 * (0.2659732 + t2 * (0.0360768 + t2 * 0.0045813)))));
    }
    double ti = 1.0 / t;
    return std::pow(a, -0.5) * std::exp(a) *
           (0.39894228 + ti * (0.01328592 + ti * (0.00225319 + ti * (-0.00157565 +
            ti * (0.00916281 + ti * (-0.02057706 + ti * (0.02635537 +
            ti * (-0.01647633 + ti * 0.00392377))))))));
}

// Every tile must be at least W - 1 wide, the first and the last (partial) one
// included, so that a kernel footprint spans at most two consecutive tiles per
// axis (the owner-computes spread gathers from the tile and its lower neighbour
// only).  When the grid extent leaves a last tile narrower than that, the tiles
// are shifted by an offset toff (tile t starts at t * tile - toff) that moves
// part of the remainder into a narrower first tile, so the requested extent is
// kept: 250 = 7 + 30 x 8 + 3 for tile 8, W 4 (toff 1).  Only when no offset
// works does the extent change (the nearest one that fits, smaller first).
int fit_tile(int t, int w, int nos, int *toff) {
    t = std::max(1, std::min(t, nos));
    *toff = 0;
    if (w <= 1 || nos <= t) return t;
    // smallest offset o for which extent tt fits, -1 if none
    auto fit = [&](int tt) {
        if (tt < w - 1) return -1;
        if (nos <= tt) return 0;  // one tile: the footprints wrap inside it
        for (int o = 0; o < tt && tt - o >= w - 1; ++o) {
            const int r = (nos + o) % tt;  // width of the last tile (0: full)
            if (r == 0 || r >= w - 1) return o;
        }
        return -1;
    };
    for (int d = 0; d < nos; ++d) {
        int o;
        if (t - d >= 1 && (o = fit(t - d)) >= 0) {
            *toff = o;
            return t - d;
        }
        if (t + d <= nos && (o = fit(t + d)) >= 0) {
            *toff = o;
            return t + d;
        }
    }
    return nos;
}

int default_tile(int ndim, int nos) {
    // 16 x 16 in 2D and 8^3 in 3D: the register-tile spreads' tiles
    int t = ndim == 1 ? 1024 : (ndim == 2 ? 16 : 8);
    return std::max(1, std::min(t, nos));
}

template <typename T>
int dev_alloc(T **p, size_t count) {
    return pool_alloc(reinterpret_cast<void **>(p), (count == 0 ? 1 : count) * sizeof(T));
}

// every apply of the plan has finished first (the device is synchronised, as
// cudaFree would)
void free_plan_buffers(pfb_plan *p) {
    cudaDeviceSynchronize();
    for (int a = 0; a < kMaxDim; ++a) {
        pool_free(p->d_cos[a], 0);
        pool_free(p->d_apod[a], 0);
        p->d_cos[a] = p->d_apod[a] = nullptr;
    }
    pool_free(p->d_perm, 0);
    pool_free(p->d_iperm, 0);
    p->d_iperm = nullptr;
    pool_free(p->d_sframe, 0);
    pool_free(p->d_bin_start, 0);
    pool_free(p->d_items_frame, 0);
    pool_free(p->d_items_all, 0);
    pool_free(p->d_frame_off, 0);
    p->d_perm = p->d_sframe = p->d_bin_start = nullptr;
    p->d_items_frame = p->d_items_all = nullptr;
    p->d_frame_off = nullptr;
}

// keys are ((bin * ncode + code) * nframes + frame): the samples of one tile
// and frame sit in ncode runs (one per edge code)
void build_items(const std::vector<int> &bs, int nbins, int ncode, int nframes, int chunk, bool per_frame,
                 std::vector<SpreadItem> &items) {
    items.clear();
    for (int b = 0; b < nbins; ++b) {
        for (int c = 0; c < ncode; ++c) {
            const int k0 = (b * ncode + c) * nframes;
            if (per_frame) {
                for (int f = 0; f < nframes; ++f) {
                    int s0 = bs[k0 + f], s1 = bs[k0 + f + 1];
                    for (int s = s0; s < s1; s += chunk)
                        items.push_back({s, std::min(s1, s + chunk), b, f});
                }
            } else {
                int s0 = bs[k0], s1 = bs[k0 + nframes];
                for (int s = s0; s < s1; s += chunk)
                    items.push_back({s, std::min(s1, s + chunk), b, -1});
            }
        }
    }
}

}  // namespace

int rebuild_items(pfb_plan *p, int chunk) {
    std::vector<SpreadItem> a, b;
    build_items(p->bin_start, p->nbins_total, p->ncode, p->nframes, chunk, true, a);
    build_items(p->bin_start, p->nbins_total, p->ncode, p->nframes, chunk, false, b);
    if (p->d_items_frame || p->d_items_all) cudaDeviceSynchronize();  // applies in flight may read them
    pool_free(p->d_items_frame, 0);
    pool_free(p->d_items_all, 0);
    p->d_items_frame = p->d_items_all = nullptr;
    int st;
    if ((st = dev_alloc(&p->d_items_frame, a.size()))) return st;
    if ((st = dev_alloc(&p->d_items_all, b.size()))) return st;
    if (!a.empty())
        PFB_CUDA_TRY(cudaMemcpy(p->d_items_frame, a.data(), a.size() * sizeof(SpreadItem), cudaMemcpyHostToDevice));
    if (!b.empty())
        PFB_CUDA_TRY(cudaMemcpy(p->d_items_all, b.data(), b.size() * sizeof(SpreadItem), cudaMemcpyHostToDevice));
    p->n_items_frame = (int)a.size();
    p->n_items_all = (int)b.size();
    p->chunk = chunk;
    return PFB_OK;
}

int plan_create(const float *coord, int ndim, int nframes, const int64_t *frame_offsets,
                int readout_len, const int *shape, const int *os_shape, const int *width,
                const float *beta, const int *is_cart, const int *tile, int device,
                cudaStream_t stream, pfb_plan **out) {
    if (!out) return fail(PFB_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (ndim < 1 || ndim > 3) return fail(PFB_ERR_INVALID, "ndim must be 1, 2 or 3");
    if (nframes < 1 || !frame_offsets) return fail(PFB_ERR_INVALID, "nframes < 1 or no frame offsets");
    if (!shape || !os_shape || !width || !beta) return fail(PFB_ERR_INVALID, "missing per-axis parameters");
    if (frame_offsets[0] != 0) return fail(PFB_ERR_INVALID, "frame_offsets[0] must be 0");
    for (int f = 0; f < nframes; ++f)
        if (frame_offsets[f + 1] < frame_offsets[f]) return fail(PFB_ERR_INVALID, "frame_offsets not ascending");
    int64_t mtot = frame_offsets[nframes];
    if (mtot >= (int64_t)1 << 31) return fail(PFB_ERR_INVALID, "more than 2^31-1 samples per plan");
    if (mtot > 0 && !coord) return fail(PFB_ERR_INVALID, "coord is NULL");
    if (readout_len < 1) return fail(PFB_ERR_INVALID, "readout_len < 1");

    pfb_plan *p = new pfb_plan();
    p->device = device;
    p->nframes = nframes;
    p->mtot = mtot;
    p->readout = readout_len;
    p->frame_off.assign(frame_offsets, frame_offsets + nframes + 1);
    Geom &g = p->g;
    g.ndim = ndim;
    g.gvol = 1;
    g.nvol = 1;
    int64_t nbins_total = 1;
    for (int a = 0; a < kMaxDim; ++a) {
        if (a < ndim) {
            int z = ndim - 1 - a;  // (z, y, x) input index of x-first axis a
            g.n[a] = shape[z];
            g.nos[a] = os_shape[z];
            // width 1 means integer positions with unit weight, whatever is_cart says
            // (_grid/_plan.py:69-72)
            g.cart[a] = (is_cart && is_cart[z] != 0) || width[z] == 1;
            g.w[a] = g.cart[a] ? 1 : width[z];
            g.beta[a] = beta[z];
            g.tile[a] = fit_tile(tile && tile[z] > 0 ? tile[z] : default_tile(ndim, g.nos[a]), g.w[a], g.nos[a],
                                 &g.toff[a]);
        } else {
            g.n[a] = g.nos[a] = g.w[a] = g.tile[a] = 1;
            g.toff[a] = 0;
            g.cart[a] = 1;
            g.beta[a] = 0.f;
        }
        if (g.n[a] < 1 || g.nos[a] < g.n[a]) {
            delete p;
            return fail(PFB_ERR_INVALID, "need 1 <= shape <= os_shape on every axis");
        }
        if (g.w[a] < 1 || g.w[a] > kMaxWidth) {
            delete p;
            return fail(PFB_ERR_INVALID, "kernel width must be in [1, 8]");
        }
        if (g.w[a] > g.nos[a]) {
            delete p;
            return fail(PFB_ERR_INVALID, "kernel width larger than the oversampled grid");
        }
        g.nbins[a] = (g.nos[a] + g.toff[a] + g.tile[a] - 1) / g.tile[a];
        g.sh[a] = g.nos[a] / 2;
        g.gvol *= g.nos[a];
        g.nvol *= g.n[a];
        nbins_total *= g.nbins[a];
    }
    if ((nbins_total << ndim) * nframes >= (int64_t)1 << 30) {
        delete p;
        return fail(PFB_ERR_INVALID, "too many (tile, frame) bins; use a larger tile");
    }
    p->nbins_total = (int)nbins_total;

    // kernel scaling: product over axes of the node-centred sums (_grid/_plan.py:118-141)
    double scale = 1.0;
    for (int a = 0; a < ndim; ++a) {
        if (g.w[a] == 1) continue;
        double start = std::ceil(-g.w[a] / 2.0), s = 0.0;
        for (int e = 0; e < g.w[a]; ++e) s += kb_host((start + e) / (g.w[a] / 2.0), (double)g.beta[a]);
        scale *= s;
    }
    p->scale = scale;

    int st = PFB_OK;
    float *d_cos_tmp = nullptr;
    int *d_keys = nullptr, *d_vals = nullptr, *d_keys_sorted = nullptr, *d_bad = nullptr;
    void *d_temp = nullptr;
    size_t temp_bytes = 0;
    p->ncode = 1 << ndim;
    int nkeys = (int)(nbins_total * p->ncode * nframes);
    const int T = 256;

    // the temporaries go back in the order of the plan stream's work
    auto cleanup = [&](int code) {
        pool_free(d_cos_tmp, stream);
        pool_free(d_keys, stream);
        pool_free(d_vals, stream);
        pool_free(d_keys_sorted, stream);
        pool_free(d_bad, stream);
        pool_free(d_temp, stream);
        if (code != PFB_OK) {
            free_owner_items(p);
            free_plan_buffers(p);
            delete p;
        }
        return code;
    };

#define PFB_TRY_ST(expr) do { st = (expr); if (st != PFB_OK) return cleanup(st); } while (0)
#define PFB_TRY_CU(expr) do { cudaError_t _e = (expr); if (_e != cudaSuccess) \
        return cleanup(fail(PFB_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e))); } while (0)

    PFB_TRY_ST(dev_alloc(&p->d_frame_off, nframes + 1));
    PFB_TRY_CU(cudaMemcpyAsync(p->d_frame_off, frame_offsets, (nframes + 1) * sizeof(int64_t),
                               cudaMemcpyHostToDevice, stream));
    for (int a = 0; a < ndim; ++a) PFB_TRY_ST(dev_alloc(&p->d_cos[a], mtot));
    PFB_TRY_ST(dev_alloc(&p->d_perm, mtot));
    PFB_TRY_ST(dev_alloc(&p->d_iperm, mtot));
    PFB_TRY_ST(dev_alloc(&p->d_sframe, mtot));
    PFB_TRY_ST(dev_alloc(&p->d_bin_start, nkeys + 1));
    PFB_TRY_ST(dev_alloc(&d_cos_tmp, (size_t)ndim * mtot));
    PFB_TRY_ST(dev_alloc(&d_keys, mtot));
    PFB_TRY_ST(dev_alloc(&d_vals, mtot));
    PFB_TRY_ST(dev_alloc(&d_keys_sorted, mtot));
    PFB_TRY_ST(dev_alloc(&d_bad, 1));
    PFB_TRY_CU(cudaMemsetAsync(d_bad, 0, sizeof(int), stream));

    ScaleParams sp{};
    sp.ndim = ndim;
    sp.nframes = nframes;
    sp.mtot = mtot;
    for (int a = 0; a < ndim; ++a) {
        // _traj.py:62-65: scale = ceil(osf*N)/N and shift = ceil(osf*N)//2, float32
        sp.s[a] = (float)g.nos[a] / (float)g.n[a];
        sp.shift[a] = (float)(g.nos[a] / 2);
        sp.nos[a] = g.nos[a];
        sp.w[a] = g.w[a];
        sp.cart[a] = g.cart[a];
        sp.tile[a] = g.tile[a];
        sp.toff[a] = g.toff[a];
        sp.nbins[a] = g.nbins[a];
    }
    if (mtot > 0) {
        unsigned blocks = (unsigned)((mtot + T - 1) / T);
        scale_and_key_kernel<<<blocks, T, 0, stream>>>(sp, coord, p->d_frame_off, d_cos_tmp, d_keys, d_vals, d_bad);
        PFB_TRY_CU(cudaGetLastError());
        int end_bit = 1;
        while ((1LL << end_bit) < (long long)nkeys) ++end_bit;
        temp_bytes = counting_sort_temp_bytes(mtot);
        PFB_TRY_ST(pool_alloc(&d_temp, temp_bytes));
        PFB_TRY_ST(counting_sort_pairs(d_keys, d_vals, d_keys_sorted, p->d_perm, mtot, end_bit, d_temp, temp_bytes,
                                       stream));
        gather_sorted_kernel<<<blocks, T, 0, stream>>>(ndim, mtot, nframes, d_cos_tmp, p->d_perm, d_keys_sorted,
                                                       p->d_cos[0], p->d_cos[1], p->d_cos[2], p->d_sframe,
                                                       p->d_iperm);
        PFB_TRY_CU(cudaGetLastError());
    }
    bin_start_kernel<<<(nkeys + 1 + T - 1) / T, T, 0, stream>>>(d_keys_sorted, mtot, nkeys, p->d_bin_start);
    PFB_TRY_CU(cudaGetLastError());
    p->bin_start.resize(nkeys + 1);
    int bad = 0;
    PFB_TRY_CU(cudaMemcpyAsync(p->bin_start.data(), p->d_bin_start, (nkeys + 1) * sizeof(int),
                               cudaMemcpyDeviceToHost, stream));
    PFB_TRY_CU(cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, stream));
    PFB_TRY_CU(cudaStreamSynchronize(stream));
    if (bad) return cleanup(fail(PFB_ERR_INVALID, "non-finite or out-of-range coordinates"));

    // deapodisation vectors (float64 math, _apod.py:27-41)
    for (int a = 0; a < ndim; ++a) {
        if (g.w[a] == 1) continue;
        int n = g.n[a];
        std::vector<double> v(n);
        for (int i = 0; i < n; ++i) {
            double q = M_PI * g.w[a] * (double)(i - n / 2) / (double)g.nos[a];
            double arg = (double)g.beta[a] * (double)g.beta[a] - q * q;
            double r = std::sqrt(arg);
            v[i] = r / std::sinh(r);
        }
        double dc = v[n / 2];
        std::vector<float> vf(n);
        for (int i = 0; i < n; ++i) {
            double r = v[i] / dc;
            vf[i] = std::isnan(r) ? 1.0f : (float)r;
        }
        PFB_TRY_ST(dev_alloc(&p->d_apod[a], n));
        PFB_TRY_CU(cudaMemcpy(p->d_apod[a], vf.data(), n * sizeof(float), cudaMemcpyHostToDevice));
    }

    int maxbin = 0;
    for (int k = 0; k < nkeys; ++k) maxbin = std::max(maxbin, p->bin_start[k + 1] - p->bin_start[k]);
    p->max_bin = maxbin;
    int chunk = ndim == 3 ? 256 : 512;
    PFB_TRY_ST(rebuild_items(p, chunk));
    // visits per owner item before a crowded tile is split (its items interleave the
    // visits).  Longer items are faster but sum more visits serially in float32 per
    // grid point: 3D radial 200^3 / 32 coils, spread 11.9 / 11.64 / 11.55 ms and the
    // adjoint 4.9e-6 / 4.7e-6 / 1.15e-5 from float64 at 2048 / 4096 / 8192 visits
    PFB_TRY_ST(build_owner_items(p, 4096));
    PFB_TRY_ST(build_plan_taps(p, stream));
    // twiddle tables of the fused transform now, so that no apply allocates
    // (applies may be captured into CUDA graphs)
    fft_fused_ready(p);
#undef PFB_TRY_ST
#undef PFB_TRY_CU
    cleanup(PFB_OK);
    *out = p;
    return PFB_OK;
}

int plan_tables(const pfb_plan *p, int axis_zyx, int32_t *index, float *value, cudaStream_t s) {
    if (axis_zyx < 0 || axis_zyx >= p->g.ndim) return fail(PFB_ERR_INVALID, "axis out of range");
    int a = p->g.ndim - 1 - axis_zyx;
    if (p->mtot == 0) return PFB_OK;
    const int T = 256;
    tables_kernel<<<(unsigned)((p->mtot + T - 1) / T), T, 0, s>>>(p->g, a, p->mtot, p->d_cos[a], p->d_perm,
                                                                  index, value);
    PFB_CHECK_LAUNCH();
    return PFB_OK;
}

void plan_free(pfb_plan *p) {
    {
        std::lock_guard<std::mutex> lk(p->fft_mu);
        for (auto &kv : p->fft_plans) cufftDestroy(kv.second);
        p->fft_plans.clear();
    }
    free_owner_items(p);
    free_plan_buffers(p);
    delete p;
}

}  // namespace pfb
