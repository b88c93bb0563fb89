// Stable integer counting sort of the plan's bin keys (plan time).
//
// The samples are bucketed by the integer key ((tile << d | edge code) * F +
// frame), whose tile part uses the reference's grid-index arithmetic
// (x0 = ceil(c_os - W/2) mod n_os, _grid/_plan.py:192-210).  The sort is a
// least-significant-digit sequence of counting sorts over 8-bit digits: each
// pass histograms the digit per chunk of samples, scans the (digit, chunk)
// counts into output offsets (a segmented prefix sum over all CTAs), and
// scatters every sample to
// offset[digit][chunk] + (its rank among the chunk's samples with the same
// digit that precede it).  Every pass is stable, so equal keys keep the order
// of the caller's samples and the result is deterministic (bit for bit the
// same permutation on every run).
#include <algorithm>

#include "pfb_common.cuh"

namespace pfb {
namespace {

constexpr int kSortThreads = 256;
constexpr int kSortRounds = 16;                      // 256-sample rounds per chunk
constexpr int kSortChunk = kSortThreads * kSortRounds;  // samples per CTA
constexpr int kDigits = 256;
constexpr int kSortWarps = kSortThreads / 32;
static_assert(kSortThreads == kDigits, "one thread per digit in the per-chunk tables");

// counts[d * nchunks + chunk] = samples of `chunk` whose digit is d
__global__ void __launch_bounds__(kSortThreads) digit_count_kernel(const int *__restrict__ keys, int n, int shift,
                                                                   int nchunks, int *__restrict__ counts) {
    __shared__ int h[kDigits];
    h[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kSortChunk;
    for (int r = 0; r < kSortRounds; ++r) {
        const int64_t i = base + r * kSortThreads + threadIdx.x;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & (kDigits - 1)], 1);
    }
    __syncthreads();
    counts[(int64_t)threadIdx.x * nchunks + blockIdx.x] = h[threadIdx.x];
}

// Exclusive prefix sum of `len` ints in place, one CTA of 1024 threads: each
// thread sums a contiguous segment, the segment sums are scanned in shared
// memory, then each thread rewrites its segment.
__global__ void __launch_bounds__(1024) exclusive_scan_kernel(int *__restrict__ a, int64_t len) {
    __shared__ int s[1024];
    const int t = threadIdx.x;
    const int64_t seg = (len + 1023) / 1024;
    const int64_t b = t * seg, e = min(len, b + seg);
    int sum = 0;
    for (int64_t i = b; i < e; ++i) sum += a[i];
    s[t] = sum;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        const int v = t >= off ? s[t - off] : 0;
        __syncthreads();
        s[t] += v;
        __syncthreads();
    }
    int run = s[t] - sum;  // exclusive prefix of this segment
    for (int64_t i = b; i < e; ++i) {
        const int v = a[i];
        a[i] = run;
        run += v;
    }
}

// Exclusive prefix sum of a long array in three steps: per-segment sums
// (kScanSeg elements per CTA), an exclusive scan of the segment sums in one CTA
// (exclusive_scan_kernel), then each CTA rescans its segment from its offset.
constexpr int kScanSeg = 4096;
__global__ void __launch_bounds__(256) segment_sum_kernel(const int *__restrict__ a, int64_t len,
                                                          int *__restrict__ sums) {
    __shared__ int s[256];
    const int64_t b = (int64_t)blockIdx.x * kScanSeg;
    int v = 0;
    for (int i = threadIdx.x; i < kScanSeg; i += 256) {
        const int64_t k = b + i;
        if (k < len) v += a[k];
    }
    s[threadIdx.x] = v;
    __syncthreads();
    for (int off = 128; off > 0; off >>= 1) {
        if (threadIdx.x < off) s[threadIdx.x] += s[threadIdx.x + off];
        __syncthreads();
    }
    if (threadIdx.x == 0) sums[blockIdx.x] = s[0];
}

// segment-local exclusive scan plus the segment's offset; thread t owns the 16
// consecutive elements t * 16 .. t * 16 + 15 of the segment
__global__ void __launch_bounds__(256) segment_scan_kernel(int *__restrict__ a, int64_t len,
                                                           const int *__restrict__ offs) {
    constexpr int PER = kScanSeg / 256;
    __shared__ int s[256];
    const int64_t b = (int64_t)blockIdx.x * kScanSeg + threadIdx.x * PER;
    int v[PER];
    int sum = 0;
#pragma unroll
    for (int i = 0; i < PER; ++i) {
        v[i] = b + i < len ? a[b + i] : 0;
        sum += v[i];
    }
    s[threadIdx.x] = sum;
    __syncthreads();
    for (int off = 1; off < 256; off <<= 1) {
        const int t = threadIdx.x >= off ? s[threadIdx.x - off] : 0;
        __syncthreads();
        s[threadIdx.x] += t;
        __syncthreads();
    }
    int run = offs[blockIdx.x] + s[threadIdx.x] - sum;
#pragma unroll
    for (int i = 0; i < PER; ++i) {
        if (b + i < len) a[b + i] = run;
        run += v[i];
    }
}

// Stable scatter of one pass.  A chunk is walked in rounds of 256 samples in
// sample order (thread t holds sample base + 256 r + t); within a round a
// sample's rank among equal digits is the count in earlier warps plus the
// count in its own warp below its lane.
__global__ void __launch_bounds__(kSortThreads) digit_scatter_kernel(const int *__restrict__ keys_in,
                                                                     const int *__restrict__ vals_in, int n,
                                                                     int shift, int nchunks,
                                                                     const int *__restrict__ offsets,
                                                                     int *__restrict__ keys_out,
                                                                     int *__restrict__ vals_out) {
    __shared__ int run[kDigits];               // next free slot per digit for this chunk
    __shared__ int wcount[kSortWarps][kDigits];
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    run[t] = offsets[(int64_t)t * nchunks + blockIdx.x];
    for (int w = 0; w < kSortWarps; ++w) wcount[w][t] = 0;
    __syncthreads();
    const unsigned lt = (1u << lane) - 1u;
    const int64_t base = (int64_t)blockIdx.x * kSortChunk;
    for (int r = 0; r < kSortRounds; ++r) {
        const int64_t i = base + r * kSortThreads + t;
        const bool ok = i < n;
        const int key = ok ? keys_in[i] : 0;
        const int val = ok ? vals_in[i] : 0;
        const int d = ok ? (key >> shift) & (kDigits - 1) : -1;  // -1: no sample (not counted)
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        if (ok && (peers & lt) == 0) wcount[warp][d] = __popc(peers);  // group leader records the count
        __syncthreads();
        if (ok) {
            int pos = run[d] + __popc(peers & lt);
            for (int w = 0; w < warp; ++w) pos += wcount[w][d];
            keys_out[pos] = key;
            vals_out[pos] = val;
        }
        __syncthreads();
        int tot = 0;
        for (int w = 0; w < kSortWarps; ++w) {
            tot += wcount[w][t];
            wcount[w][t] = 0;
        }
        run[t] += tot;
        __syncthreads();
    }
}

}  // namespace

size_t counting_sort_temp_bytes(int64_t n) {
    const int64_t nchunks = (n + kSortChunk - 1) / kSortChunk;
    const int64_t nseg = ((int64_t)kDigits * nchunks + kScanSeg - 1) / kScanSeg;
    // two key / value buffers, the (digit, chunk) counts and their segment sums
    return (size_t)(2 * n + (int64_t)kDigits * nchunks + nseg + 64) * sizeof(int);
}

int counting_sort_pairs(const int *keys, const int *vals, int *keys_out, int *vals_out, int64_t n, int end_bit,
                        void *temp, size_t temp_bytes, cudaStream_t s) {
    if (n <= 0) return PFB_OK;
    if (n >= (int64_t)1 << 31) return fail(PFB_ERR_INVALID, "counting sort: too many samples");
    if (temp_bytes < counting_sort_temp_bytes(n)) return fail(PFB_ERR_WORKSPACE, "counting sort: temp too small");
    const int nchunks = (int)((n + kSortChunk - 1) / kSortChunk);
    int *ka = static_cast<int *>(temp);
    int *va = ka + n;
    int *counts = va + n;
    const int64_t ncount = (int64_t)kDigits * nchunks;
    const int nseg = (int)((ncount + kScanSeg - 1) / kScanSeg);
    int *segs = counts + ncount;
    const int passes = std::max(1, (end_bit + 7) / 8);
    // pass p reads (in) and writes (out); the last pass writes keys_out / vals_out
    const int *kin = keys, *vin = vals;
    for (int p = 0; p < passes; ++p) {
        const bool last = p == passes - 1;
        // ping-pong so that the last pass lands in the caller's buffers
        int *kout = last ? keys_out : (((passes - 1 - p) & 1) ? ka : keys_out);
        int *vout = last ? vals_out : (((passes - 1 - p) & 1) ? va : vals_out);
        digit_count_kernel<<<nchunks, kSortThreads, 0, s>>>(kin, (int)n, 8 * p, nchunks, counts);
        PFB_CHECK_LAUNCH();
        segment_sum_kernel<<<nseg, 256, 0, s>>>(counts, ncount, segs);
        PFB_CHECK_LAUNCH();
        exclusive_scan_kernel<<<1, 1024, 0, s>>>(segs, nseg);
        PFB_CHECK_LAUNCH();
        segment_scan_kernel<<<nseg, 256, 0, s>>>(counts, ncount, segs);
        PFB_CHECK_LAUNCH();
        digit_scatter_kernel<<<nchunks, kSortThreads, 0, s>>>(kin, vin, (int)n, 8 * p, nchunks, counts, kout, vout);
        PFB_CHECK_LAUNCH();
        kin = kout;
        vin = vout;
    }
    return PFB_OK;
}

}  // namespace pfb
