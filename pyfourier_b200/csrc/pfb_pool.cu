// Device memory of plans: one library-owned CUDA memory pool per device whose
// release threshold is unlimited, so the blocks a destroyed plan gives back stay
// reserved for the next plan.  Building and destroying plans back to back (every
// Pipe-Menon call builds one, as the reference's pipe_menon_dcf takes
// coordinates, src/pyfourier/_dcomp/pipemenon.py:69-96) then costs stream-ordered
// pool operations instead of cudaMalloc / cudaFree.  pfb_release_cached_memory
// hands the kept blocks back to the device.
#include <cstdint>
#include <mutex>

#include "pfb_common.cuh"

namespace pfb {
namespace {

constexpr int kMaxDevices = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_pool[kMaxDevices] = {};

// the device's pool, created on first use (nullptr if the device has none)
cudaMemPool_t device_pool(int dev) {
    if (dev < 0 || dev >= kMaxDevices) return nullptr;
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (!g_pool[dev]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) return nullptr;
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        g_pool[dev] = pool;
    }
    return g_pool[dev];
}

}  // namespace

int pool_alloc(void **p, size_t bytes) {
    *p = nullptr;
    int dev = 0;
    PFB_CUDA_TRY(cudaGetDevice(&dev));
    cudaMemPool_t pool = device_pool(dev);
    if (!pool) return fail(PFB_ERR_CUDA, "no memory pool on the current device");
    if (bytes == 0) bytes = 1;
    // ordered on the legacy default stream, which is synchronised so that the block
    // can be used on any stream
    cudaError_t e = cudaMallocFromPoolAsync(p, bytes, pool, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) {
        *p = nullptr;
        return fail(e == cudaErrorMemoryAllocation ? PFB_ERR_NOMEM : PFB_ERR_CUDA,
                    std::string("pool allocation: ") + cudaGetErrorString(e));
    }
    return PFB_OK;
}

void pool_free(void *p, cudaStream_t s) {
    if (p) cudaFreeAsync(p, s);
}

}  // namespace pfb

extern "C" int pfb_release_cached_memory(int device) {
    using namespace pfb;
    cudaMemPool_t pool = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        if (device < 0 || device >= kMaxDevices) return fail(PFB_ERR_INVALID, "bad device");
        pool = g_pool[device];
    }
    if (!pool) return PFB_OK;
    int prev = -1;
    PFB_CUDA_TRY(cudaGetDevice(&prev));
    if (prev != device) PFB_CUDA_TRY(cudaSetDevice(device));
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemPoolTrimTo(pool, 0);
    if (prev != device) cudaSetDevice(prev);
    if (e != cudaSuccess) return fail(PFB_ERR_CUDA, std::string("pool trim: ") + cudaGetErrorString(e));
    return PFB_OK;
}
