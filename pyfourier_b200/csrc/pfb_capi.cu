// extern "C" entry points of libpfb200.so (declared in include/pfb200.h).
#include <cmath>
#include <cstring>

#include <map>
#include <mutex>
#include <utility>

#include "pfb_common.cuh"

namespace pfb {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

int raise_smem_limit(const void *kernel, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, size_t> granted;
    int dev = 0;
    PFB_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    size_t &g = granted[{kernel, dev}];
    if (g >= bytes) return PFB_OK;
    PFB_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    g = bytes;
    return PFB_OK;
}

int fail(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

namespace {

// Make `dev` current for the scope of an entry point.
struct DeviceGuard {
    int prev = -1;
    bool ok = true;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) { ok = false; return; }
        if (prev != dev && cudaSetDevice(dev) != cudaSuccess) ok = false;
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

constexpr size_t kAlign = 256;
size_t align_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

}  // namespace

// cuFFT plan over `nplanes` batched grids of extent dims (slowest first).
int get_fft_plan(std::mutex &mu, std::map<int64_t, cufftHandle> &plans, std::map<int64_t, size_t> &work,
                 int ndim, const int *nos_xyz, int64_t nplanes, cufftHandle *out, size_t *wbytes) {
    std::lock_guard<std::mutex> lk(mu);
    auto it = plans.find(nplanes);
    if (it != plans.end()) {
        *out = it->second;
        *wbytes = work[nplanes];
        return PFB_OK;
    }
    cufftHandle h;
    PFB_CUFFT_TRY(cufftCreate(&h));
    cufftResult r = cufftSetAutoAllocation(h, 0);
    if (r != CUFFT_SUCCESS) { cufftDestroy(h); return fail(PFB_ERR_CUFFT, "cufftSetAutoAllocation failed"); }
    long long dims[3];
    for (int a = 0; a < ndim; ++a) dims[a] = nos_xyz[ndim - 1 - a];
    long long dist = 1;
    for (int a = 0; a < ndim; ++a) dist *= dims[a];
    size_t ws = 0;
    r = cufftMakePlanMany64(h, ndim, dims, nullptr, 1, dist, nullptr, 1, dist, CUFFT_C2C,
                            (long long)nplanes, &ws);
    if (r != CUFFT_SUCCESS) {
        cufftDestroy(h);
        return fail(PFB_ERR_CUFFT, "cufftMakePlanMany64 failed with status " + std::to_string((int)r));
    }
    plans[nplanes] = h;
    work[nplanes] = ws;
    *out = h;
    *wbytes = ws;
    return PFB_OK;
}

// The plan's cuFFT handle is shared by every apply on the plan: its stream and
// work area are set per call, so `mu` (the plan's fft_mu) is held from
// cufftSetStream to the end of cufftExecC2C, and concurrent applies of one plan
// from several host threads cannot run one call's transform with another's work
// area.
int run_fft(std::mutex &mu, cufftHandle h, size_t wbytes, float2 *data, int direction, void *work,
            size_t work_avail, cudaStream_t s) {
    if (wbytes > work_avail) return fail(PFB_ERR_WORKSPACE, "workspace too small for the cuFFT work area");
    std::lock_guard<std::mutex> lk(mu);
    PFB_CUFFT_TRY(cufftSetStream(h, s));
    PFB_CUFFT_TRY(cufftSetWorkArea(h, work));
    PFB_CUFFT_TRY(cufftExecC2C(h, reinterpret_cast<cufftComplex *>(data), reinterpret_cast<cufftComplex *>(data),
                               direction < 0 ? CUFFT_FORWARD : CUFFT_INVERSE));
    return PFB_OK;
}

int run_fft_to(std::mutex &mu, cufftHandle h, size_t wbytes, const float2 *src, float2 *dst, int direction,
               void *work, size_t work_avail, cudaStream_t s) {
    if (wbytes > work_avail) return fail(PFB_ERR_WORKSPACE, "workspace too small for the cuFFT work area");
    std::lock_guard<std::mutex> lk(mu);
    PFB_CUFFT_TRY(cufftSetStream(h, s));
    PFB_CUFFT_TRY(cufftSetWorkArea(h, work));
    // a C2C transform leaves an out-of-place input unchanged
    PFB_CUFFT_TRY(cufftExecC2C(h, reinterpret_cast<cufftComplex *>(const_cast<float2 *>(src)),
                               reinterpret_cast<cufftComplex *>(dst), direction < 0 ? CUFFT_FORWARD : CUFFT_INVERSE));
    return PFB_OK;
}

int to_desc(const pfb_plan *p, const pfb_apply_t *o, ApplyDesc &d) {
    if (!o) return fail(PFB_ERR_INVALID, "apply options are NULL");
    d.batch = o->batch;
    d.ncoeff = o->ncoeff;
    d.basis = static_cast<const float2 *>(o->basis);
    d.weight = o->weight;
    d.nseg = o->nseg < 1 ? 1 : o->nseg;
    d.b0_time = static_cast<const float2 *>(o->b0_time);
    d.b0_space = static_cast<const float2 *>(o->b0_space);
    d.norm = o->norm;
    if (d.batch < 0) return fail(PFB_ERR_INVALID, "batch < 0");
    if (d.ncoeff < 1) return fail(PFB_ERR_INVALID, "ncoeff < 1");
    if (!d.basis && d.ncoeff != p->nframes)
        return fail(PFB_ERR_INVALID, "without a basis ncoeff must equal the number of frames");
    if ((d.b0_time == nullptr) != (d.b0_space == nullptr))
        return fail(PFB_ERR_INVALID, "b0_time and b0_space must be given together");
    if (!d.b0_time && d.nseg != 1) return fail(PFB_ERR_INVALID, "nseg > 1 needs B0 coefficients");
    if (o->norm != PFB_NORM_NONE && o->norm != PFB_NORM_ORTHO) return fail(PFB_ERR_INVALID, "unknown norm");
    if (d.batch * (int64_t)d.nseg * (d.basis ? d.ncoeff : 1) > (1LL << 30))
        return fail(PFB_ERR_INVALID, "too many channels");
    return PFB_OK;
}

namespace {

int64_t planes_of(const ApplyDesc &d) { return (int64_t)d.nseg * d.batch * d.ncoeff; }

}  // namespace
}  // namespace pfb

using namespace pfb;

struct pfb_gram {
    int device = 0;
    int ndim = 2;
    int n[3] = {1, 1, 1};
    int nos[3] = {1, 1, 1};
    int64_t nvol = 1, gvol = 1;
    int K = 1;
    int lowrank = 0;
    int nseg = 1;          // B0 time segments (one kernel each)
    float2 *d_T = nullptr;
    std::mutex fft_mu;
    std::map<int64_t, cufftHandle> fft_plans;
    std::map<int64_t, size_t> fft_work;
};

extern "C" {

const char *pfb_last_error(void) { return g_last_error.c_str(); }

const char *pfb_version(void) { return "pyfourier_b200 0.1.0 (sm_100a)"; }

int pfb_plan_create(const float *coord, int ndim, int nframes, const int64_t *frame_offsets, int readout_len,
                    const int *shape, const int *os_shape, const int *width, const float *beta,
                    const int *is_cart, const int *tile, int device, void *stream, pfb_plan **out) {
    // argument checks that need no device come first
    if (!out) return fail(PFB_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (ndim < 1 || ndim > 3) return fail(PFB_ERR_INVALID, "ndim must be 1, 2 or 3");
    if (nframes < 1 || !frame_offsets) return fail(PFB_ERR_INVALID, "nframes < 1 or no frame offsets");
    if (!shape || !os_shape || !width || !beta) return fail(PFB_ERR_INVALID, "missing per-axis parameters");
    DeviceGuard dg(device);
    if (!dg.ok) return fail(PFB_ERR_CUDA, "cannot select device");
    return plan_create(coord, ndim, nframes, frame_offsets, readout_len, shape, os_shape, width, beta, is_cart,
                       tile, device, static_cast<cudaStream_t>(stream), out);
}

int pfb_plan_destroy(pfb_plan *plan) {
    if (!plan) return PFB_OK;
    DeviceGuard dg(plan->device);
    plan_free(plan);
    return PFB_OK;
}

int pfb_plan_info(const pfb_plan *p, pfb_plan_info_t *info) {
    if (!p || !info) return fail(PFB_ERR_INVALID, "NULL argument");
    std::memset(info, 0, sizeof(*info));
    info->ndim = p->g.ndim;
    info->nframes = p->nframes;
    info->total_samples = p->mtot;
    for (int z = 0; z < 3; ++z) {
        int a = p->g.ndim - 1 - z;
        bool used = z < p->g.ndim;
        info->shape[z] = used ? p->g.n[a] : 1;
        info->os_shape[z] = used ? p->g.nos[a] : 1;
        info->width[z] = used ? p->g.w[a] : 1;
        info->tile[z] = used ? p->g.tile[a] : 1;
        info->tile_offset[z] = used ? p->g.toff[a] : 0;
    }
    info->scale = p->scale;
    info->n_items = p->n_items_frame;
    info->max_bin = p->max_bin;
    return PFB_OK;
}

int pfb_plan_set_tuning(pfb_plan *p, int spread_threads, int interp_threads, int spread_channels) {
    if (!p) return fail(PFB_ERR_INVALID, "NULL plan");
    auto ok = [](int t) { return t == 0 || (t >= 32 && t <= 1024 && t % 32 == 0); };
    if (!ok(spread_threads) || !ok(interp_threads))
        return fail(PFB_ERR_INVALID, "threads must be a multiple of 32 in [32, 1024]");
    if (spread_threads > 256 || interp_threads > 256)
        return fail(PFB_ERR_INVALID, "kernels are compiled for at most 256 threads per CTA");
    if (spread_channels < 0 || spread_channels > 8) return fail(PFB_ERR_INVALID, "spread_channels in [0, 8]");
    if (spread_threads) p->spread_threads = spread_threads;
    if (interp_threads) p->interp_threads = interp_threads;
    p->spread_channels = spread_channels;
    return PFB_OK;
}

int pfb_plan_set_chunk(pfb_plan *p, int chunk) {
    if (!p || chunk < 1 || chunk > 16384) return fail(PFB_ERR_INVALID, "chunk must be in [1, 16384]");
    DeviceGuard dg(p->device);
    int st = rebuild_items(p, chunk);
    if (st) return st;
    return build_owner_items(p, chunk);
}

int pfb_plan_tables(const pfb_plan *p, int axis, int32_t *index, float *value, void *stream) {
    if (!p || !index || !value) return fail(PFB_ERR_INVALID, "NULL argument");
    DeviceGuard dg(p->device);
    return plan_tables(p, axis, index, value, static_cast<cudaStream_t>(stream));
}

int pfb_plan_order(const pfb_plan *p, int32_t *order, void *stream) {
    if (!p || !order) return fail(PFB_ERR_INVALID, "NULL argument");
    if (p->mtot == 0) return PFB_OK;
    DeviceGuard dg(p->device);
    PFB_CUDA_TRY(cudaMemcpyAsync(order, p->d_perm, p->mtot * sizeof(int32_t), cudaMemcpyDeviceToDevice,
                                 static_cast<cudaStream_t>(stream)));
    return PFB_OK;
}

int pfb_plan_check(pfb_plan *p, void *stream) {
    if (!p) return fail(PFB_ERR_INVALID, "NULL plan");
    if (!p->d_fft_err) return PFB_OK;
    DeviceGuard dg(p->device);
    int v = 0;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    PFB_CUDA_TRY(cudaMemcpyAsync(&v, p->d_fft_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    PFB_CUDA_TRY(cudaStreamSynchronize(s));
    if (v) {
        PFB_CUDA_TRY(cudaMemsetAsync(p->d_fft_err, 0, sizeof(int), s));
        return fail(PFB_ERR_DEVICE, "a fused-FFT pass gave up waiting for its tile loads: "
                                    "results since the last check are invalid");
    }
    return PFB_OK;
}

int pfb_workspace_size(pfb_plan *p, int64_t nplanes, size_t *bytes) {
    if (!p || !bytes || nplanes < 1) return fail(PFB_ERR_INVALID, "bad argument");
    DeviceGuard dg(p->device);
    cufftHandle h;
    size_t wb = 0;
    int st = get_fft_plan(p->fft_mu, p->fft_plans, p->fft_work, p->g.ndim, p->g.nos, nplanes, &h, &wb);
    if (st) return st;
    *bytes = align_up((size_t)nplanes * p->g.gvol * sizeof(float2)) + align_up(wb);
    return PFB_OK;
}

int pfb_grid_fft(pfb_plan *p, void *grid, int64_t nplanes, int direction, void *workspace, size_t workspace_bytes,
                 void *stream) {
    if (!p || !grid || nplanes < 1) return fail(PFB_ERR_INVALID, "bad argument");
    DeviceGuard dg(p->device);
    cufftHandle h;
    size_t wb = 0;
    int st = get_fft_plan(p->fft_mu, p->fft_plans, p->fft_work, p->g.ndim, p->g.nos, nplanes, &h, &wb);
    if (st) return st;
    return run_fft(p->fft_mu, h, wb, static_cast<float2 *>(grid), direction, workspace, workspace_bytes,
                   static_cast<cudaStream_t>(stream));
}

int pfb_nufft_fwd(pfb_plan *p, const pfb_apply_t *opt, const void *image, void *kspace, void *workspace,
                  size_t workspace_bytes, void *stream) {
    if (!p || !image || !kspace || !workspace) return fail(PFB_ERR_INVALID, "NULL argument");
    DeviceGuard dg(p->device);
    ApplyDesc d;
    int st = to_desc(p, opt, d);
    if (st) return st;
    if (d.batch == 0) return PFB_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int64_t P = planes_of(d);
    // forward: unnormalised FFT ("ortho": 1/sqrt(G)), and 1/scale of _cart2noncart:110
    double fac = 1.0 / p->scale;
    if (d.norm == PFB_NORM_ORTHO) fac /= std::sqrt((double)p->g.gvol);
    // channel-interleaved path when the workspace holds it, else the planar path
    size_t fast_bytes = 0;
    if (fast_supported(p, d, nullptr) && fast_workspace(p, d, &fast_bytes) == PFB_OK && workspace_bytes >= fast_bytes)
        return fast_fwd(p, d, static_cast<const float2 *>(image), static_cast<float2 *>(kspace), workspace,
                        workspace_bytes, (float)fac, opt->flags & PFB_FLAG_ACCUMULATE, s);
    cufftHandle h;
    size_t wb = 0;
    if ((st = get_fft_plan(p->fft_mu, p->fft_plans, p->fft_work, p->g.ndim, p->g.nos, P, &h, &wb))) return st;
    size_t gbytes = align_up((size_t)P * p->g.gvol * sizeof(float2));
    if (workspace_bytes < gbytes + wb) return fail(PFB_ERR_WORKSPACE, "workspace too small");
    float2 *grid = static_cast<float2 *>(workspace);
    void *work = static_cast<char *>(workspace) + gbytes;
    if ((st = launch_deapod_pad(p, d, static_cast<const float2 *>(image), grid, (float)fac, s))) return st;
    if ((st = run_fft(p->fft_mu, h, wb, grid, -1, work, workspace_bytes - gbytes, s))) return st;
    return launch_interp(p, d, grid, static_cast<float2 *>(kspace), true, s, opt->flags & PFB_FLAG_ACCUMULATE);
}

int pfb_nufft_adj(pfb_plan *p, const pfb_apply_t *opt, const void *kspace, void *image, void *workspace,
                  size_t workspace_bytes, void *stream) {
    if (!p || !image || !kspace || !workspace) return fail(PFB_ERR_INVALID, "NULL argument");
    DeviceGuard dg(p->device);
    ApplyDesc d;
    int st = to_desc(p, opt, d);
    if (st) return st;
    if (d.batch == 0) return PFB_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int64_t P = planes_of(d);
    // adjoint: inverse FFT scaled 1/G (None) or 1/sqrt(G) (ortho), and 1/scale of _noncart2cart:119
    double fac = 1.0 / p->scale;
    fac /= (d.norm == PFB_NORM_ORTHO) ? std::sqrt((double)p->g.gvol) : (double)p->g.gvol;
    size_t fast_bytes = 0;
    if (fast_supported(p, d, nullptr) && fast_workspace(p, d, &fast_bytes) == PFB_OK && workspace_bytes >= fast_bytes)
        return fast_adj(p, d, static_cast<const float2 *>(kspace), static_cast<float2 *>(image), workspace,
                        workspace_bytes, (float)fac, opt->flags & PFB_FLAG_ACCUMULATE, s);
    cufftHandle h;
    size_t wb = 0;
    if ((st = get_fft_plan(p->fft_mu, p->fft_plans, p->fft_work, p->g.ndim, p->g.nos, P, &h, &wb))) return st;
    size_t gbytes = align_up((size_t)P * p->g.gvol * sizeof(float2));
    if (workspace_bytes < gbytes + wb) return fail(PFB_ERR_WORKSPACE, "workspace too small");
    float2 *grid = static_cast<float2 *>(workspace);
    void *work = static_cast<char *>(workspace) + gbytes;
    if ((st = launch_spread(p, d, static_cast<const float2 *>(kspace), grid, true, s))) return st;
    if ((st = run_fft(p->fft_mu, h, wb, grid, +1, work, workspace_bytes - gbytes, s))) return st;
    return launch_crop_deapod(p, d, grid, static_cast<float2 *>(image), (float)fac, s,
                              opt->flags & PFB_FLAG_ACCUMULATE);
}

int pfb_apply_workspace_size(pfb_plan *p, const pfb_apply_t *opt, size_t *bytes) {
    if (!p || !bytes) return fail(PFB_ERR_INVALID, "NULL argument");
    DeviceGuard dg(p->device);
    ApplyDesc d;
    int st = to_desc(p, opt, d);
    if (st) return st;
    if (d.batch == 0) {
        *bytes = 0;
        return PFB_OK;
    }
    if (fast_supported(p, d, nullptr)) return fast_workspace(p, d, bytes);
    cufftHandle h;
    size_t wb = 0;
    int64_t P = planes_of(d);
    if ((st = get_fft_plan(p->fft_mu, p->fft_plans, p->fft_work, p->g.ndim, p->g.nos, P, &h, &wb))) return st;
    *bytes = align_up((size_t)P * p->g.gvol * sizeof(float2)) + align_up(wb);
    return PFB_OK;
}

int pfb_nufft_traj_grad(pfb_plan *p, const pfb_apply_t *opt, const void *image, const void *values, float *grad,
                        float factor, void *workspace, size_t workspace_bytes, void *stream) {
    if (!p || !image || !values || !grad || !workspace) return fail(PFB_ERR_INVALID, "NULL argument");
    DeviceGuard dg(p->device);
    ApplyDesc d;
    int st = to_desc(p, opt, d);
    if (st) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const bool acc = opt->flags & PFB_FLAG_ACCUMULATE;
    if (d.batch == 0 || p->mtot == 0) {
        if (!acc && p->mtot > 0) PFB_CUDA_TRY(cudaMemsetAsync(grad, 0, p->mtot * p->g.ndim * sizeof(float), s));
        return PFB_OK;
    }
    size_t fast_bytes = 0;
    if (fast_supported(p, d, nullptr) && fast_workspace(p, d, &fast_bytes) == PFB_OK && workspace_bytes >= fast_bytes)
        return fast_traj_grad(p, d, static_cast<const float2 *>(image), static_cast<const float2 *>(values), grad,
                              workspace, workspace_bytes, factor, acc, s);
    int64_t P = planes_of(d);
    cufftHandle h;
    size_t wb = 0;
    if ((st = get_fft_plan(p->fft_mu, p->fft_plans, p->fft_work, p->g.ndim, p->g.nos, P, &h, &wb))) return st;
    size_t gbytes = align_up((size_t)P * p->g.gvol * sizeof(float2));
    if (workspace_bytes < gbytes + wb) return fail(PFB_ERR_WORKSPACE, "workspace too small");
    float2 *grid = static_cast<float2 *>(workspace);
    void *work = static_cast<char *>(workspace) + gbytes;
    if ((st = launch_deapod_pad(p, d, static_cast<const float2 *>(image), grid, factor, s))) return st;
    if ((st = run_fft(p->fft_mu, h, wb, grid, -1, work, workspace_bytes - gbytes, s))) return st;
    return launch_traj_grad(p, d, grid, static_cast<const float2 *>(values), grad, true, s, acc);
}

int pfb_nufft_stage(pfb_plan *p, const pfb_apply_t *opt, int stage, const void *src, void *dst, float factor,
                    void *workspace, size_t workspace_bytes, void *stream) {
    if (!p || !workspace) return fail(PFB_ERR_INVALID, "NULL argument");
    DeviceGuard dg(p->device);
    ApplyDesc d;
    int st = to_desc(p, opt, d);
    if (st) return st;
    if (d.batch == 0) return PFB_OK;
    if (!fast_supported(p, d, nullptr)) return fail(PFB_ERR_UNSUPPORTED, "options outside the interleaved path");
    if ((stage == PFB_STAGE_PAD || stage == PFB_STAGE_VALS) && !src) return fail(PFB_ERR_INVALID, "src is NULL");
    if ((stage == PFB_STAGE_OUT || stage == PFB_STAGE_CROP) && !dst) return fail(PFB_ERR_INVALID, "dst is NULL");
    return fast_stage(p, d, stage, src, dst, workspace, workspace_bytes, factor, opt->flags & PFB_FLAG_ACCUMULATE,
                      static_cast<cudaStream_t>(stream));
}

int pfb_spread(pfb_plan *p, const pfb_apply_t *opt, const void *kspace, void *grid, int fft_layout, void *stream) {
    if (!p || !kspace || !grid) return fail(PFB_ERR_INVALID, "NULL argument");
    DeviceGuard dg(p->device);
    ApplyDesc d;
    int st = to_desc(p, opt, d);
    if (st) return st;
    return launch_spread(p, d, static_cast<const float2 *>(kspace), static_cast<float2 *>(grid), fft_layout != 0,
                         static_cast<cudaStream_t>(stream));
}

int pfb_interp(pfb_plan *p, const pfb_apply_t *opt, const void *grid, void *kspace, int fft_layout, void *stream) {
    if (!p || !kspace || !grid) return fail(PFB_ERR_INVALID, "NULL argument");
    DeviceGuard dg(p->device);
    ApplyDesc d;
    int st = to_desc(p, opt, d);
    if (st) return st;
    return launch_interp(p, d, static_cast<const float2 *>(grid), static_cast<float2 *>(kspace), fft_layout != 0,
                         static_cast<cudaStream_t>(stream), opt->flags & PFB_FLAG_ACCUMULATE);
}

int pfb_deapod_pad(pfb_plan *p, const pfb_apply_t *opt, const void *image, void *grid, float factor, void *stream) {
    if (!p || !image || !grid) return fail(PFB_ERR_INVALID, "NULL argument");
    DeviceGuard dg(p->device);
    ApplyDesc d;
    int st = to_desc(p, opt, d);
    if (st) return st;
    return launch_deapod_pad(p, d, static_cast<const float2 *>(image), static_cast<float2 *>(grid), factor,
                             static_cast<cudaStream_t>(stream));
}

int pfb_crop_deapod(pfb_plan *p, const pfb_apply_t *opt, const void *grid, void *image, float factor, void *stream) {
    if (!p || !image || !grid) return fail(PFB_ERR_INVALID, "NULL argument");
    DeviceGuard dg(p->device);
    ApplyDesc d;
    int st = to_desc(p, opt, d);
    if (st) return st;
    return launch_crop_deapod(p, d, static_cast<const float2 *>(grid), static_cast<float2 *>(image), factor,
                              static_cast<cudaStream_t>(stream), opt->flags & PFB_FLAG_ACCUMULATE);
}

int pfb_traj_grad(pfb_plan *p, const pfb_apply_t *opt, const void *grid, const void *values, float *grad,
                  int fft_layout, void *stream) {
    if (!p || !grid || !values || !grad) return fail(PFB_ERR_INVALID, "NULL argument");
    DeviceGuard dg(p->device);
    ApplyDesc d;
    int st = to_desc(p, opt, d);
    if (st) return st;
    return launch_traj_grad(p, d, static_cast<const float2 *>(grid), static_cast<const float2 *>(values), grad,
                            fft_layout != 0, static_cast<cudaStream_t>(stream), opt->flags & PFB_FLAG_ACCUMULATE);
}

}  // extern "C"

namespace {
// image grid == FFT grid and no B0 segments: the Gram needs no embedding
bool gram_is_dense(const pfb_gram *g) {
    if (g->nseg != 1) return false;
    for (int a = 0; a < g->ndim; ++a)
        if (g->n[a] != g->nos[a]) return false;
    return true;
}
}  // namespace

extern "C" {

int pfb_gram_create(int ndim, const int *shape, const int *os_shape, int ncoeff, int lowrank, int nseg,
                    const void *kernel, int device, void *stream, pfb_gram **out) {
    if (!out) return fail(PFB_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (ndim < 1 || ndim > 3 || !shape || !os_shape || !kernel || ncoeff < 1 || nseg < 1)
        return fail(PFB_ERR_INVALID, "bad argument");
    if (lowrank && ncoeff > 8) return fail(PFB_ERR_UNSUPPORTED, "subspace size K > 8");
    DeviceGuard dg(device);
    if (!dg.ok) return fail(PFB_ERR_CUDA, "cannot select device");
    pfb_gram *g = new pfb_gram();
    g->device = device;
    g->ndim = ndim;
    for (int a = 0; a < ndim; ++a) {
        g->n[a] = shape[ndim - 1 - a];
        g->nos[a] = os_shape[ndim - 1 - a];
        if (g->n[a] < 1 || g->nos[a] < g->n[a]) {
            delete g;
            return fail(PFB_ERR_INVALID, "need 1 <= shape <= os_shape");
        }
        g->nvol *= g->n[a];
        g->gvol *= g->nos[a];
    }
    g->K = ncoeff;
    g->lowrank = lowrank != 0;
    g->nseg = nseg;
    size_t tbytes = (size_t)nseg * g->gvol * sizeof(float2) *
                    (g->lowrank ? (size_t)ncoeff * ncoeff : (size_t)ncoeff);
    cudaError_t e = cudaMalloc(&g->d_T, tbytes);
    if (e != cudaSuccess) {
        delete g;
        return fail(PFB_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    e = cudaMemcpyAsync(g->d_T, kernel, tbytes, cudaMemcpyDeviceToDevice, static_cast<cudaStream_t>(stream));
    if (e == cudaSuccess) e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        cudaFree(g->d_T);
        delete g;
        return fail(PFB_ERR_CUDA, std::string("kernel copy: ") + cudaGetErrorString(e));
    }
    *out = g;
    return PFB_OK;
}

int pfb_gram_destroy(pfb_gram *g) {
    if (!g) return PFB_OK;
    DeviceGuard dg(g->device);
    {
        std::lock_guard<std::mutex> lk(g->fft_mu);
        for (auto &kv : g->fft_plans) cufftDestroy(kv.second);
    }
    cudaFree(g->d_T);
    delete g;
    return PFB_OK;
}

int pfb_gram_workspace_size(pfb_gram *g, int64_t batch, size_t *bytes) {
    if (!g || !bytes || batch < 1) return fail(PFB_ERR_INVALID, "bad argument");
    DeviceGuard dg(g->device);
    int64_t P = (int64_t)g->nseg * batch * g->K;
    cufftHandle h;
    size_t wb = 0;
    int st = get_fft_plan(g->fft_mu, g->fft_plans, g->fft_work, g->ndim, g->nos, P, &h, &wb);
    if (st) return st;
    // a dense Gram transforms in the output array: only the cuFFT work area
    *bytes = gram_is_dense(g) ? std::max<size_t>(align_up(wb), 256)
                              : align_up((size_t)P * g->gvol * sizeof(float2)) + align_up(wb);
    return PFB_OK;
}

int pfb_gram_apply(pfb_gram *g, const void *image, void *out, int64_t batch, const void *b0_space,
                   void *workspace, size_t workspace_bytes, void *stream) {
    if (!g || !image || !out || !workspace) return fail(PFB_ERR_INVALID, "NULL argument");
    if (batch < 0) return fail(PFB_ERR_INVALID, "batch < 0");
    if (g->nseg > 1 && !b0_space) return fail(PFB_ERR_INVALID, "a Gram with B0 segments needs b0_space");
    if (batch == 0) return PFB_OK;
    DeviceGuard dg(g->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int L = g->nseg;
    const int64_t bk = batch * g->K;  // image planes
    const int64_t P = L * bk;         // grid planes (segment-major)
    cufftHandle h;
    size_t wb = 0;
    int st = get_fft_plan(g->fft_mu, g->fft_plans, g->fft_work, g->ndim, g->nos, P, &h, &wb);
    if (st) return st;
    if (gram_is_dense(g)) {
        // grid == image, one segment: FFT image -> out, mix in place with the 1/G
        // of the two transforms folded in, inverse FFT in place (3 passes, no
        // embed / extract copies)
        if (workspace_bytes < wb) return fail(PFB_ERR_WORKSPACE, "workspace too small");
        float2 *o = static_cast<float2 *>(out);
        if ((st = run_fft_to(g->fft_mu, h, wb, static_cast<const float2 *>(image), o, -1, workspace, workspace_bytes, s)))
            return st;
        if ((st = launch_mix(g->gvol, g->K, g->lowrank, batch, g->d_T, o, s, (float)(1.0 / (double)g->gvol))))
            return st;
        return run_fft(g->fft_mu, h, wb, o, +1, workspace, workspace_bytes, s);
    }
    size_t gbytes = align_up((size_t)P * g->gvol * sizeof(float2));
    if (workspace_bytes < gbytes + wb) return fail(PFB_ERR_WORKSPACE, "workspace too small");
    float2 *grid = static_cast<float2 *>(workspace);
    void *work = static_cast<char *>(workspace) + gbytes;
    const float2 *Cl = static_cast<const float2 *>(b0_space);
    if ((st = launch_embed(g->ndim, g->n, g->nos, static_cast<const float2 *>(image), grid, bk, Cl, L, s)))
        return st;
    if ((st = run_fft(g->fft_mu, h, wb, grid, -1, work, workspace_bytes - gbytes, s))) return st;
    const size_t tplane = (size_t)g->gvol * (g->lowrank ? (size_t)g->K * g->K : (size_t)g->K);
    for (int l = 0; l < L; ++l)  // segment l's kernel on segment l's planes
        if ((st = launch_mix(g->gvol, g->K, g->lowrank, batch, g->d_T + l * tplane, grid + l * bk * g->gvol, s)))
            return st;
    if ((st = run_fft(g->fft_mu, h, wb, grid, +1, work, workspace_bytes - gbytes, s))) return st;
    // forward and inverse FFT scalings multiply to 1/G whatever `norm` is
    return launch_extract(g->ndim, g->n, g->nos, grid, static_cast<float2 *>(out), bk,
                          (float)(1.0 / (double)g->gvol), Cl, L, s);
}

}  // extern "C"
