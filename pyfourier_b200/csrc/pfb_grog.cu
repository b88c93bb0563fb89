// GROG pre-interpolation (src/pyfourier/_preinterp/_grog.py:22-250, the apply of
// :399-439): every non-Cartesian sample's coil vector is moved onto its nearest
// grid point by the GRAPPA operator of its quantised offset,
//     out[b, :, m] = in[b, :, m] @ G[op(m), slice(b)],
// G a table of nc x nc complex64 operators (nsteps^ndim of them, per
// calibration slice in 2D).  The reference computes one (sample, batch) vector
// product per thread and reads the nc x nc operator of every sample from
// memory.  Here the plan sorts the samples by operator once; an apply then
//   1. transposes the coil-major input (b, c, m) into coil vectors in sorted
//      order, rows[b][j][c] (coalesced reads along m, one contiguous row write
//      per sample),
//   2. walks the chunks of <= kChunk rows that share an operator with
//      persistent CTAs: the rows are staged in shared memory (double-buffered
//      cp.async), each lane keeps one operator column in registers and computes
//      one output coil of every row (row values are shared-memory broadcasts),
//      written back in place,
//   3. transposes back to (b, c, m), writing zeros for samples outside the grid.
// An operator is read from memory once per run of chunks that share it instead
// of once per sample.

#include <algorithm>
#include <vector>

#include "pfb_common.cuh"

struct GrogChunk {
    int op;         // operator index in [0, ntable)
    int cnt;        // rows in the chunk (1 .. kChunk)
    int64_t start;  // first sorted row
};

struct pfb_grog {
    int device = 0;
    int64_t M = 0;   // samples
    int64_t Mk = 0;  // samples inside the grid (sorted rows)
    int nc = 0;      // coils
    int nslices = 1; // operator sets (2D: one per calibration slice)
    int ntable = 0;  // operators per set
    int *d_pos = nullptr;   // sample -> sorted row, -1 outside the grid
    float2 *d_G = nullptr;  // (ntable, nslices, nc, nc), [i][j] = source coil i -> target coil j
    GrogChunk *d_chunks = nullptr;
    int nchunks = 0;
    int nsm = 148;  // SMs of the device (persistent grid of the apply)
};

namespace pfb {
namespace {

constexpr int kChunk = 128;  // rows per apply work item (even: rows are taken in pairs)
constexpr int kTile = 64;    // samples per transpose tile
constexpr int kMaxCoils = 64;

struct Guard {
    int prev = -1;
    bool ok = true;
    explicit Guard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) { ok = false; return; }
        if (prev != dev && cudaSetDevice(dev) != cudaSuccess) ok = false;
    }
    ~Guard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

// sort keys: the operator index, or ntable for samples outside the grid
__global__ void grog_keys_kernel(const int *__restrict__ lut, int64_t M, int ntable, int *__restrict__ keys,
                                 int *__restrict__ idx, int *__restrict__ bad) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; m < M; m += stride) {
        int k = lut[m];
        if (k < -1 || k >= ntable) {
            atomicExch(bad, 1);
            k = ntable;
        }
        keys[m] = k < 0 ? ntable : k;
        idx[m] = (int)m;
    }
}

// off[k] = first sorted position with key >= k, k = 0 .. nkeys (each written once)
__global__ void grog_bounds_kernel(const int *__restrict__ keys, int64_t M, int nkeys, int *__restrict__ off) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j <= M; j += stride) {
        const int lo = j == 0 ? 0 : keys[j - 1] + 1;
        const int hi = j == M ? nkeys : keys[j];
        for (int k = lo; k <= hi; ++k) off[k] = (int)j;
    }
}

__global__ void grog_pos_kernel(const int *__restrict__ perm, int64_t M, int64_t Mk, int *__restrict__ pos) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < M; j += stride)
        pos[perm[j]] = j < Mk ? (int)j : -1;
}

// Pass 1: in (B, nc, M) -> rows (B, Mk, nc) in sorted order.  One CTA per tile of
// kTile consecutive samples of one batch item (blockIdx.y strides the batch): the
// tile and its sorted positions are staged in shared memory, then each warp writes
// whole rows (no global load waits between the row stores).
__global__ void __launch_bounds__(256) grog_rows_kernel(const float2 *__restrict__ in, const int *__restrict__ pos,
                                                        int nc, int64_t M, int64_t Mk, int64_t batch,
                                                        float2 *__restrict__ rows) {
    __shared__ float2 tile[kMaxCoils][kTile + 1];
    __shared__ int spos[kTile];
    const int64_t m0 = (int64_t)blockIdx.x * kTile;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int64_t b = blockIdx.y; b < batch; b += gridDim.y) {
        __syncthreads();
        if (threadIdx.x < kTile) spos[threadIdx.x] = m0 + threadIdx.x < M ? pos[m0 + threadIdx.x] : -1;
        for (int e = threadIdx.x; e < nc * kTile; e += blockDim.x) {
            const int c = e / kTile, t = e % kTile;
            const int64_t m = m0 + t;
            tile[c][t] = m < M ? in[((int64_t)b * nc + c) * M + m] : make_float2(0.f, 0.f);
        }
        __syncthreads();
        for (int t = warp; t < kTile; t += 8) {
            const int p = spos[t];
            if (p < 0) continue;
            float2 *r = rows + ((int64_t)b * Mk + p) * nc;
            for (int c = lane; c < nc; c += 32) r[c] = tile[c][t];
        }
    }
}

// Pass 3: rows (B, Mk, nc) -> out (B, nc, M); samples outside the grid get zeros.
// Each warp issues the row loads of its kTile / 8 samples back to back.
__global__ void __launch_bounds__(256) grog_cols_kernel(const float2 *__restrict__ rows, const int *__restrict__ pos,
                                                        int nc, int64_t M, int64_t Mk, int64_t batch,
                                                        float2 *__restrict__ out) {
    __shared__ float2 tile[kMaxCoils][kTile + 1];
    __shared__ int spos[kTile];
    constexpr int kPerWarp = kTile / 8;
    const int64_t m0 = (int64_t)blockIdx.x * kTile;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int64_t b = blockIdx.y; b < batch; b += gridDim.y) {
        __syncthreads();
        if (threadIdx.x < kTile) spos[threadIdx.x] = m0 + threadIdx.x < M ? pos[m0 + threadIdx.x] : -1;
        __syncthreads();
        float2 v[kPerWarp][2];
#pragma unroll
        for (int q = 0; q < kPerWarp; ++q) {
            const int p = spos[warp + 8 * q];
            const float2 *r = rows + ((int64_t)b * Mk + (p < 0 ? 0 : p)) * nc;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int c = lane + 32 * h;
                v[q][h] = (p >= 0 && c < nc) ? r[c] : make_float2(0.f, 0.f);
            }
        }
#pragma unroll
        for (int q = 0; q < kPerWarp; ++q)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int c = lane + 32 * h;
                if (c < nc) tile[c][warp + 8 * q] = v[q][h];
            }
        __syncthreads();
        for (int e = threadIdx.x; e < nc * kTile; e += blockDim.x) {
            const int c = e / kTile, t = e % kTile;
            const int64_t m = m0 + t;
            if (m < M) out[((int64_t)b * nc + c) * M + m] = tile[c][t];
        }
    }
}

__device__ __forceinline__ void cmac(float2 &acc, float2 a, float2 g) {
    acc.x = fmaf(a.x, g.x, acc.x);
    acc.x = fmaf(-a.y, g.y, acc.x);
    acc.y = fmaf(a.x, g.y, acc.y);
    acc.y = fmaf(a.y, g.x, acc.y);
}

// Pass 2 for 32 < nc <= 64: one CTA (8 warps) per chunk of rows sharing one
// operator, rows in place; lane j computes output coils j and j + 32 with the
// operator in shared memory.  Rows are stored with an even stride so that two
// coils load as one 16-byte broadcast.
__global__ void __launch_bounds__(256) grog_apply_smem_kernel(const GrogChunk *__restrict__ chunks,
                                                              const float2 *__restrict__ G, int nc, int nslices,
                                                              int64_t Mk, int64_t batch, float2 *__restrict__ rows) {
    extern __shared__ float4 smem4[];
    const int ncs = (nc + 1) & ~1;
    float2 *srow = reinterpret_cast<float2 *>(smem4);  // kChunk x ncs
    float2 *sG = srow + kChunk * ncs;                  // nc x nc
    const GrogChunk ck = chunks[blockIdx.x];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int64_t b = blockIdx.y; b < batch; b += gridDim.y) {
        const int sl = nslices > 1 ? (int)b : 0;
        const float2 *Gop = G + ((int64_t)ck.op * nslices + sl) * nc * nc;
        float2 *R = rows + ((int64_t)b * Mk + ck.start) * nc;
        __syncthreads();  // the previous batch item's readers are done with shared memory
        for (int e = threadIdx.x; e < nc * nc; e += blockDim.x) sG[e] = __ldg(Gop + e);
        const int tot = ck.cnt * nc;
        for (int e = threadIdx.x; e < tot; e += blockDim.x) {
            const int r = e / nc, i = e - r * nc;
            srow[r * ncs + i] = R[e];
        }
        if (nc & 1)
            for (int r = threadIdx.x; r < ck.cnt; r += blockDim.x) srow[r * ncs + nc] = make_float2(0.f, 0.f);
        __syncthreads();
        const int j1 = lane + 32;
        for (int r = warp; r < ck.cnt; r += 8) {
            const float4 *src = reinterpret_cast<const float4 *>(srow + r * ncs);
            float2 acc0 = make_float2(0.f, 0.f), acc1 = make_float2(0.f, 0.f);
            for (int i2 = 0; 2 * i2 < nc; ++i2) {
                const float4 v = src[i2];
                const int i = 2 * i2;
                const float2 a0 = make_float2(v.x, v.y), a1 = make_float2(v.z, v.w);
                const bool has1 = i + 1 < nc;
                cmac(acc0, a0, sG[i * nc + lane]);
                if (has1) cmac(acc0, a1, sG[(i + 1) * nc + lane]);
                if (j1 < nc) {
                    cmac(acc1, a0, sG[i * nc + j1]);
                    if (has1) cmac(acc1, a1, sG[(i + 1) * nc + j1]);
                }
            }
            R[r * nc + lane] = acc0;
            if (j1 < nc) R[r * nc + j1] = acc1;
        }
    }
}

// Pass 2 for nc <= 32: persistent CTAs (8 warps, 2 per SM) each walking a
// contiguous range of virtual chunks v = b * nchunks + c, so that consecutive
// chunks mostly share an operator: its column stays in registers (lane j holds
// G[:, j]) and is reloaded only when the operator changes.  The rows of chunk
// v + 1 are copied into the second shared-memory buffer with cp.async while
// chunk v is computed; each warp takes two rows at a time (four independent
// accumulation chains per lane).
__global__ void __launch_bounds__(256, 2) grog_apply_reg_kernel(const GrogChunk *__restrict__ chunks, int nchunks,
                                                                const float2 *__restrict__ G, int nc, int nslices,
                                                                int64_t Mk, int64_t batch,
                                                                float2 *__restrict__ rows) {
    extern __shared__ float4 smem4[];
    const int ncs = (nc + 1) & ~1;
    float2 *buf = reinterpret_cast<float2 *>(smem4);  // 2 x kChunk x ncs
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t nv = (int64_t)nchunks * batch;
    const int64_t v0 = nv * blockIdx.x / gridDim.x, v1 = nv * (blockIdx.x + 1) / gridDim.x;
    if (v0 >= v1) return;
    if (nc & 1)  // zero pad column of every row of both buffers (never a cp.async target)
        for (int r = threadIdx.x; r < 2 * kChunk; r += blockDim.x) buf[r * ncs + nc] = make_float2(0.f, 0.f);
    auto stage = [&](int64_t v, float2 *dst) {
        const int64_t b = v / nchunks;
        const GrogChunk ck = chunks[v - b * nchunks];
        const float2 *R = rows + ((int64_t)b * Mk + ck.start) * nc;
        const int tot = ck.cnt * nc;
        for (int e = threadIdx.x; e < tot; e += blockDim.x) {
            const int r = e / nc;
            cp_async8(dst + r * ncs + (e - r * nc), R + e, true);
        }
        cp_async_commit();
    };
    stage(v0, buf);
    int cur_op = -1, cur_sl = -1;
    float2 gcol[32];
    for (int64_t v = v0; v < v1; ++v) {
        const float2 *cb = buf + ((v - v0) & 1) * kChunk * ncs;
        cp_async_wait_all();
        __syncthreads();  // chunk v has landed; every warp is done with the other buffer
        if (v + 1 < v1) stage(v + 1, buf + ((v + 1 - v0) & 1) * kChunk * ncs);
        const int64_t b = v / nchunks;
        const GrogChunk ck = chunks[v - b * nchunks];
        const int sl = nslices > 1 ? (int)b : 0;
        if (ck.op != cur_op || sl != cur_sl) {
            const float2 *Gop = G + ((int64_t)ck.op * nslices + sl) * nc * nc;
#pragma unroll
            for (int i = 0; i < 32; ++i)
                gcol[i] = (i < nc && lane < nc) ? __ldg(Gop + i * nc + lane) : make_float2(0.f, 0.f);
            cur_op = ck.op;
            cur_sl = sl;
        }
        float2 *R = rows + ((int64_t)b * Mk + ck.start) * nc;
        for (int r = 2 * warp; r < ck.cnt; r += 16) {  // rows r, r + 1 (r + 1 < kChunk: kChunk is even)
            const float4 *s0 = reinterpret_cast<const float4 *>(cb + r * ncs);
            const float4 *s1 = reinterpret_cast<const float4 *>(cb + (r + 1) * ncs);
            float2 a0 = make_float2(0.f, 0.f), a1 = make_float2(0.f, 0.f);
#pragma unroll
            for (int i2 = 0; i2 < 16; ++i2) {
                if (2 * i2 >= nc) break;
                const float4 x0 = s0[i2], x1 = s1[i2];
                cmac(a0, make_float2(x0.x, x0.y), gcol[2 * i2]);
                cmac(a1, make_float2(x1.x, x1.y), gcol[2 * i2]);
                cmac(a0, make_float2(x0.z, x0.w), gcol[2 * i2 + 1]);
                cmac(a1, make_float2(x1.z, x1.w), gcol[2 * i2 + 1]);
            }
            if (lane < nc) {
                R[r * nc + lane] = a0;
                if (r + 1 < ck.cnt) R[(r + 1) * nc + lane] = a1;
            }
        }
    }
}

unsigned ytiles(int64_t batch) { return (unsigned)std::min<int64_t>(std::max<int64_t>(batch, 1), 65535); }

}  // namespace
}  // namespace pfb

using namespace pfb;

extern "C" {

int pfb_grog_create(const int *lut, int64_t nsamples, int ntable, int ncoils, int nslices, const void *table,
                    int device, void *stream, pfb_grog **out) {
    if (!out) return fail(PFB_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!table || nsamples < 0 || ntable < 1 || nslices < 1 || (nsamples > 0 && !lut))
        return fail(PFB_ERR_INVALID, "bad argument");
    if (ncoils < 1 || ncoils > kMaxCoils) return fail(PFB_ERR_UNSUPPORTED, "GROG supports 1 to 64 coils");
    if (nsamples >= (1LL << 31) - 1) return fail(PFB_ERR_UNSUPPORTED, "more than 2^31 - 2 samples");
    Guard dg(device);
    if (!dg.ok) return fail(PFB_ERR_CUDA, "cannot select device");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    pfb_grog *g = new pfb_grog();
    g->device = device;
    g->M = nsamples;
    g->nc = ncoils;
    g->nslices = nslices;
    g->ntable = ntable;
    if (cudaDeviceGetAttribute(&g->nsm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) g->nsm = 148;
    int *keys = nullptr, *keys_s = nullptr, *idx = nullptr, *perm = nullptr, *off = nullptr, *bad = nullptr;
    void *temp = nullptr;
    auto cleanup = [&](int st) {
        cudaFree(keys);
        cudaFree(keys_s);
        cudaFree(idx);
        cudaFree(perm);
        cudaFree(off);
        cudaFree(bad);
        cudaFree(temp);
        if (st) {
            cudaFree(g->d_pos);
            cudaFree(g->d_G);
            cudaFree(g->d_chunks);
            delete g;
        }
        return st;
    };
#define GROG_TRY(expr)                                                                                 \
    do {                                                                                               \
        cudaError_t _e = (expr);                                                                       \
        if (_e != cudaSuccess)                                                                         \
            return cleanup(fail(PFB_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)));   \
    } while (0)
    const size_t gbytes = (size_t)ntable * nslices * ncoils * ncoils * sizeof(float2);
    GROG_TRY(cudaMalloc(&g->d_G, gbytes));
    GROG_TRY(cudaMemcpyAsync(g->d_G, table, gbytes, cudaMemcpyDeviceToDevice, s));
    const int64_t M = nsamples;
    std::vector<int> hoff(ntable + 2, 0);
    if (M > 0) {
        GROG_TRY(cudaMalloc(&keys, M * sizeof(int)));
        GROG_TRY(cudaMalloc(&keys_s, M * sizeof(int)));
        GROG_TRY(cudaMalloc(&idx, M * sizeof(int)));
        GROG_TRY(cudaMalloc(&perm, M * sizeof(int)));
        GROG_TRY(cudaMalloc(&off, (ntable + 2) * sizeof(int)));
        GROG_TRY(cudaMalloc(&bad, sizeof(int)));
        GROG_TRY(cudaMalloc(&g->d_pos, M * sizeof(int)));
        GROG_TRY(cudaMemsetAsync(bad, 0, sizeof(int), s));
        const unsigned blocks = (unsigned)std::min<int64_t>((M + 255) / 256, 148LL * 32);
        grog_keys_kernel<<<blocks, 256, 0, s>>>(lut, M, ntable, keys, idx, bad);
        GROG_TRY(cudaGetLastError());
        int end_bit = 1;
        while ((1LL << end_bit) <= (long long)ntable) ++end_bit;
        const size_t tb = counting_sort_temp_bytes(M);
        GROG_TRY(cudaMalloc(&temp, tb));
        {
            const int sst = counting_sort_pairs(keys, idx, keys_s, perm, M, end_bit, temp, tb, s);
            if (sst) return cleanup(sst);
        }
        grog_bounds_kernel<<<(unsigned)std::min<int64_t>((M + 256) / 256, 148LL * 32), 256, 0, s>>>(
            keys_s, M, ntable + 1, off);
        GROG_TRY(cudaGetLastError());
        int hbad = 0;
        GROG_TRY(cudaMemcpyAsync(hoff.data(), off, (ntable + 2) * sizeof(int), cudaMemcpyDeviceToHost, s));
        GROG_TRY(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
        GROG_TRY(cudaStreamSynchronize(s));
        if (hbad) return cleanup(fail(PFB_ERR_INVALID, "operator index outside [-1, ntable)"));
        g->Mk = hoff[ntable];
        grog_pos_kernel<<<blocks, 256, 0, s>>>(perm, M, g->Mk, g->d_pos);
        GROG_TRY(cudaGetLastError());
    }
    std::vector<GrogChunk> ch;
    for (int k = 0; k < ntable; ++k)
        for (int64_t j = hoff[k]; j < hoff[k + 1]; j += kChunk)
            ch.push_back(GrogChunk{k, (int)std::min<int64_t>(kChunk, hoff[k + 1] - j), j});
    g->nchunks = (int)ch.size();
    if (!ch.empty()) {
        GROG_TRY(cudaMalloc(&g->d_chunks, ch.size() * sizeof(GrogChunk)));
        GROG_TRY(cudaMemcpyAsync(g->d_chunks, ch.data(), ch.size() * sizeof(GrogChunk), cudaMemcpyHostToDevice, s));
    }
    GROG_TRY(cudaStreamSynchronize(s));
#undef GROG_TRY
    cleanup(PFB_OK);
    *out = g;
    return PFB_OK;
}

int pfb_grog_destroy(pfb_grog *g) {
    if (!g) return PFB_OK;
    Guard dg(g->device);
    cudaFree(g->d_pos);
    cudaFree(g->d_G);
    cudaFree(g->d_chunks);
    delete g;
    return PFB_OK;
}

int pfb_grog_workspace_size(pfb_grog *g, int64_t batch, size_t *bytes) {
    if (!g || !bytes || batch < 0) return fail(PFB_ERR_INVALID, "bad argument");
    *bytes = std::max<size_t>(align256((size_t)batch * g->Mk * g->nc * sizeof(float2)), 256);
    return PFB_OK;
}

int pfb_grog_apply(pfb_grog *g, const void *in, void *out, int64_t batch, void *workspace, size_t workspace_bytes,
                   void *stream) {
    if (!g || !in || !out || !workspace) return fail(PFB_ERR_INVALID, "NULL argument");
    if (batch < 0) return fail(PFB_ERR_INVALID, "batch < 0");
    if (g->nslices > 1 && batch != g->nslices)
        return fail(PFB_ERR_INVALID, "per-slice operators need batch == number of operator slices");
    if (batch == 0 || g->M == 0) return PFB_OK;
    size_t need = 0;
    pfb_grog_workspace_size(g, batch, &need);
    if (workspace_bytes < need) return fail(PFB_ERR_WORKSPACE, "workspace too small");
    Guard dg(g->device);
    if (!dg.ok) return fail(PFB_ERR_CUDA, "cannot select device");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    float2 *rows = static_cast<float2 *>(workspace);
    const dim3 tgrid((unsigned)((g->M + kTile - 1) / kTile), ytiles(batch));
    if (g->Mk > 0) {
        grog_rows_kernel<<<tgrid, 256, 0, s>>>(static_cast<const float2 *>(in), g->d_pos, g->nc, g->M, g->Mk, batch,
                                               rows);
        PFB_CHECK_LAUNCH();
        const int ncs = (g->nc + 1) & ~1;
        if (g->nc <= 32) {
            const size_t sm = 2 * (size_t)kChunk * ncs * sizeof(float2);
            PFB_RAISE_SMEM(grog_apply_reg_kernel, (int)(2 * kChunk * 32 * sizeof(float2)));
            const int64_t nv = (int64_t)g->nchunks * batch;
            const unsigned nblk = (unsigned)std::max<int64_t>(1, std::min<int64_t>(nv, 2LL * g->nsm));
            grog_apply_reg_kernel<<<nblk, 256, sm, s>>>(g->d_chunks, g->nchunks, g->d_G, g->nc, g->nslices, g->Mk,
                                                        batch, rows);
        } else {
            const size_t sm = ((size_t)kChunk * ncs + (size_t)g->nc * g->nc) * sizeof(float2);
            // 64 coils need 96 KB of dynamic shared memory
            PFB_RAISE_SMEM(grog_apply_smem_kernel, (int)(((size_t)kChunk * kMaxCoils + kMaxCoils * kMaxCoils) *
                                                    sizeof(float2)));
            const dim3 agrid((unsigned)g->nchunks, ytiles(batch));
            grog_apply_smem_kernel<<<agrid, 256, sm, s>>>(g->d_chunks, g->d_G, g->nc, g->nslices, g->Mk, batch,
                                                          rows);
        }
        PFB_CHECK_LAUNCH();
    }
    grog_cols_kernel<<<tgrid, 256, 0, s>>>(rows, g->d_pos, g->nc, g->M, g->Mk, batch, static_cast<float2 *>(out));
    PFB_CHECK_LAUNCH();
    return PFB_OK;
}

}  // extern "C"
