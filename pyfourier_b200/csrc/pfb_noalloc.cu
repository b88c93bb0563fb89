// pfb_nufft_adj_noalloc: the adjoint NUFFT for callers that cannot allocate
// device memory.
//
// Who needs it: code that runs where cudaMalloc is not allowed or not wanted at
// apply time -- inside a host framework that owns all device memory through its
// own pool, on a real-time reconstruction loop with a fixed memory budget, or
// in a process that must never grow its footprint after set-up.  Such a
// caller cannot provide the workspace that pfb_nufft_adj needs.
//
// This entry point keeps its scratch (the oversampled grid and cuFFT's work
// area) in one file-scope device array of PFB_NOALLOC_SCRATCH_BYTES bytes.  The
// caller still passes the input k-space and the output image.
//
// Rules of use:
//   * Set-up, once per device, with the plan's device current: call it with
//     opt->batch == 0.  That call only looks up the array's device address
//     (cudaGetSymbolAddress).  CUDA loads this file's device code lazily, so
//     the lookup is the moment the 64 MiB array is reserved on that device; it
//     stays reserved until the process exits.  Make the set-up call before any
//     stream capture.  Without it, the first real call does the same lookup.
//   * The cuFFT plan for the call's number of grid planes must already exist:
//     call pfb_workspace_size(plan, nplanes, ...) once during set-up (that call
//     may allocate; this one does not).  Without it the call returns
//     PFB_ERR_INVALID.
//   * Requests whose grid plus cuFFT work area exceed the array are rejected
//     with PFB_ERR_INVALID and a message naming both sizes.
//   * All calls share the one array and it keeps the last call's contents.  The
//     grid part is cleared on every call before the spread adds into it.  Calls
//     that overlap on the GPU (different streams, or different threads without
//     ordering) race on the array and give wrong results: serialise them.
//
// The address is looked up on every call (after the first, a table lookup in
// the runtime that allocates nothing), so a device reset that reloads the
// module never leaves a stale pointer behind.  Argument checks are the same
// as pfb_nufft_adj's (pfb::to_desc).
//
// It calls no cudaMalloc, cudaFree or allocating library routine.
#include <cmath>
#include <mutex>
#include <string>

#include "pfb_common.cuh"

namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[PFB_NOALLOC_SCRATCH_BYTES];

// Device address of the scratch array on the current device.
int scratch_address(void **out) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
        return pfb::fail(PFB_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    *out = p;
    return PFB_OK;
}

size_t up256(size_t x) { return (x + 255) / 256 * 256; }

}  // namespace

extern "C" int pfb_nufft_adj_noalloc(pfb_plan *p, const pfb_apply_t *o, const void *kspace, void *image,
                                     void *stream) {
    using namespace pfb;
    if (!p || !o) return fail(PFB_ERR_INVALID, "NULL argument");
    ApplyDesc d;
    int st = to_desc(p, o, d);
    if (st) return st;
    if (d.batch > 0 && (!kspace || !image)) return fail(PFB_ERR_INVALID, "NULL argument");

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

    void *base = nullptr;
    if ((st = scratch_address(&base))) return st;
    if (d.batch == 0) return PFB_OK;  // set-up call: the array is now resident on this device

    const int64_t nplanes = (int64_t)d.nseg * d.batch * d.ncoeff;
    cufftHandle h;
    size_t wbytes = 0;
    {
        std::lock_guard<std::mutex> lk(p->fft_mu);
        auto it = p->fft_plans.find(nplanes);
        if (it == p->fft_plans.end())
            return fail(PFB_ERR_INVALID, "no cuFFT plan for " + std::to_string(nplanes) +
                                             " planes: call pfb_workspace_size(plan, nplanes) once during set-up");
        h = it->second;
        wbytes = p->fft_work[nplanes];
    }
    const size_t gbytes = up256((size_t)nplanes * (size_t)p->g.gvol * sizeof(float2));
    const size_t need = gbytes + up256(wbytes);
    if (need > (size_t)PFB_NOALLOC_SCRATCH_BYTES)
        return fail(PFB_ERR_INVALID, "request needs " + std::to_string(need) + " bytes of scratch; the static "
                                     "array holds " + std::to_string((size_t)PFB_NOALLOC_SCRATCH_BYTES));
    float2 *grid = static_cast<float2 *>(base);
    void *work = static_cast<unsigned char *>(base) + gbytes;
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    double fac = 1.0 / p->scale;
    fac /= (d.norm == PFB_NORM_ORTHO) ? std::sqrt((double)p->g.gvol) : (double)p->g.gvol;
    // launch_spread clears the grid part of the scratch before adding into it
    if ((st = launch_spread(p, d, static_cast<const float2 *>(kspace), grid, true, s))) return st;
    // run_fft holds the plan's fft_mu across cufftSetStream / SetWorkArea / Exec
    if ((st = run_fft(p->fft_mu, h, wbytes, grid, +1, work, up256(wbytes), s))) return st;
    return launch_crop_deapod(p, d, grid, static_cast<float2 *>(image), (float)fac, s,
                              (o->flags & PFB_FLAG_ACCUMULATE) != 0);
}
