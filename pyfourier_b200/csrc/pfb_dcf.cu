// Pipe-Menon density compensation (src/pyfourier/_dcomp/pipemenon.py:9-115):
// starting from the caller's weights (ones in the reference, :76), niter times
//     w <- w / |A A^H w|,
// A the plan's NUFFT with norm "ortho" (_GHG, :99-115), one channel over all
// frames of the plan.  All iterations run on the caller's stream through the
// library's own forward / adjoint pipelines; between them one kernel divides by
// the magnitude and rebuilds the complex input of the next adjoint.  Nothing is
// allocated and the host never waits, so the whole loop can be issued once.
#include <cmath>

#include "pfb_common.cuh"

namespace pfb {
namespace {

// wc = (w, 0)
__global__ void dcf_load_kernel(const float *__restrict__ w, float2 *__restrict__ wc, int64_t m) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < m; j += stride)
        wc[j] = make_float2(w[j], 0.f);
}

// w = w / |k|, wc = (w, 0); a zero |k| gives inf as in the reference's division
__global__ void dcf_update_kernel(const float2 *__restrict__ k, float *__restrict__ w, float2 *__restrict__ wc,
                                  int64_t m) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < m; j += stride) {
        const float2 v = k[j];
        const float a = w[j] / hypotf(v.x, v.y);
        w[j] = a;
        wc[j] = make_float2(a, 0.f);
    }
}

size_t align_up(size_t x) { return (x + 255) / 256 * 256; }

unsigned dcf_blocks(int64_t m) {
    const int64_t b = (m + 255) / 256;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(b, 148LL * 16));
}

pfb_apply_t dcf_opt(const pfb_plan *p) {
    pfb_apply_t o{};
    o.batch = 1;
    o.ncoeff = p->nframes;
    o.nseg = 1;
    o.norm = PFB_NORM_ORTHO;
    return o;
}

struct DcfLayout {
    size_t apply, image, kspace, wc, total;
};

int dcf_layout(pfb_plan *p, DcfLayout *L) {
    pfb_apply_t o = dcf_opt(p);
    int st = pfb_apply_workspace_size(p, &o, &L->apply);
    if (st) return st;
    L->apply = align_up(L->apply);
    L->image = align_up((size_t)p->nframes * (size_t)p->g.nvol * sizeof(float2));
    L->kspace = align_up((size_t)std::max<int64_t>(p->mtot, 1) * sizeof(float2));
    L->wc = L->kspace;
    L->total = L->apply + L->image + L->kspace + L->wc;
    return PFB_OK;
}

}  // namespace
}  // namespace pfb

extern "C" {

int pfb_dcf_workspace_size(pfb_plan *p, size_t *bytes) {
    using namespace pfb;
    if (!p || !bytes) return fail(PFB_ERR_INVALID, "NULL argument");
    DcfLayout L;
    int st = dcf_layout(p, &L);
    if (st) return st;
    *bytes = L.total;
    return PFB_OK;
}

int pfb_pipe_menon_dcf(pfb_plan *p, float *weights, int niter, void *workspace, size_t workspace_bytes,
                       void *stream) {
    using namespace pfb;
    if (!p || !weights || !workspace) return fail(PFB_ERR_INVALID, "NULL argument");
    if (niter < 0) return fail(PFB_ERR_INVALID, "niter < 0");
    DcfLayout L;
    int st = dcf_layout(p, &L);
    if (st) return st;
    if (workspace_bytes < L.total) return fail(PFB_ERR_WORKSPACE, "workspace too small");
    if (niter == 0 || p->mtot == 0) return PFB_OK;
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) return fail(PFB_ERR_CUDA, "cudaGetDevice failed");
    if (prev != p->device && cudaSetDevice(p->device) != cudaSuccess)
        return fail(PFB_ERR_CUDA, "cannot select the plan's device");
    struct Restore {
        int dev;
        ~Restore() {
            int cur = -1;
            if (dev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != dev) cudaSetDevice(dev);
        }
    } restore{prev};
    char *ws = static_cast<char *>(workspace);
    void *apply = ws;
    float2 *image = reinterpret_cast<float2 *>(ws + L.apply);
    float2 *kspace = reinterpret_cast<float2 *>(ws + L.apply + L.image);
    float2 *wc = reinterpret_cast<float2 *>(ws + L.apply + L.image + L.kspace);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const pfb_apply_t o = dcf_opt(p);
    const unsigned nb = dcf_blocks(p->mtot);
    dcf_load_kernel<<<nb, 256, 0, s>>>(weights, wc, p->mtot);
    PFB_CHECK_LAUNCH();
    for (int it = 0; it < niter; ++it) {
        if ((st = pfb_nufft_adj(p, &o, wc, image, apply, L.apply, stream))) return st;
        if ((st = pfb_nufft_fwd(p, &o, image, kspace, apply, L.apply, stream))) return st;
        dcf_update_kernel<<<nb, 256, 0, s>>>(kspace, weights, wc, p->mtot);
        PFB_CHECK_LAUNCH();
    }
    return PFB_OK;
}

}  // extern "C"
