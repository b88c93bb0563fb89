// Fused, pruned FFT of the channel-interleaved NUFFT pipeline (2D and 3D).
//
// The reference's glue around the library FFT (src/pyfourier/_subroutines/_fft.py:72-79
// via _nufft/_nufft.py:218-287) is pad -> centred FFT -> (interpolate) and
// (spread) -> centred inverse FFT -> crop, with deapodisation (_apod.py:16-46) and
// the B0 spatial factors applied on the image side.  Here the multi-dimensional
// transform is run axis by axis as batched 1D transforms in shared memory, and
// the passes are pruned and fused with their neighbours:
//
//   forward 3D: image --(z pass: deapodise, C_l, zero-pad, FFT)--> T1[plane][kz][y][x]
//               --(y pass)--> T2[plane][kz][ky][x] --(x pass)--> interleaved grid
//   adjoint 3D: planar grid --(x pass: IFFT, crop x)--> T1[plane][kz][ky][x]
//               --(y pass: crop y)--> T2[plane][kz][y][x]
//               --(z pass: crop z, sum_l conj(C_l), deapodise)--> image
//
// (2D drops the z pass.)  Rows and columns that are all zero are never read or
// written, so a forward transform of an N^3 image onto an n^3 grid moves about
// N^3 + 2 n N^2 + 2 n^2 N + n^3 elements per plane instead of the 2 n^3 per pass
// of an unpruned transform, and the pad, crop and channel transpose cost nothing
// extra.
//
// Each 1D transform is a mixed-radix Stockham autosort FFT (radices 8, 10, 5, 4, 3, 7,
// 2, and two stages of radix 15, 16, 25 or 10 for the 240-, 250-, 160- and 256-point
// transforms; Govindaraju et al., "High performance discrete Fourier transforms on
// graphics processors", SC 2008):
// stage s with radix r and ns = product of the earlier radices reads
// x_q = src[i + q n / r], multiplies by exp(-2 pi i j q / (ns r)) (j = i mod ns),
// takes the r-point DFT and writes dst[(i - j) r + j + k ns].  A CTA holds 16 vectors
// (columns of shared memory); a thread takes two adjacent columns of a butterfly, or
// one column for radices 15, 16 and 25.  Inverse passes run the forward transform
// and read its output reversed, IDFT(x)[k] = DFT(x)[(n - k) mod n], or (the
// copy-based x pass) conjugate on load and store.
// Twiddles are computed in double precision on the host.

#include <cuda.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "pfb_common.cuh"

namespace pfb {
namespace {

constexpr int kCols = 16;                 // vectors per CTA
constexpr int kPitch = kCols + 2;         // shared row pitch (float2): 16-byte aligned rows
constexpr int kThreads = 256;
constexpr int kStreams = kThreads / kCols;        // load / store: 16 lanes per row
constexpr int kPairStreams = kThreads / (kCols / 2);  // butterflies: a thread takes 2 columns
constexpr int kMaxN = 512;                // longest axis handled here (else the library FFT)

// Complex add / subtract / scale-and-add as packed (re, im) FP32 instructions: the
// same roundings as the componentwise forms (a - b is b * -1 + a, the product exact).
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
// -i * a
__device__ __forceinline__ float2 cmi(float2 a) { return make_float2(a.y, -a.x); }
__device__ __forceinline__ float2 caxpy(float s, float2 a, float2 y) { return __ffma2_rn(make_float2(s, s), a, y); }

// forward r-point DFTs, b_k = sum_q a_q exp(-2 pi i q k / r), in place
template <int R>
__device__ __forceinline__ void dft(float2 *a);

template <>
__device__ __forceinline__ void dft<2>(float2 *a) {
    const float2 t = a[1];
    a[1] = csub(a[0], t);
    a[0] = cadd(a[0], t);
}

template <>
__device__ __forceinline__ void dft<4>(float2 *a) {
    const float2 t0 = cadd(a[0], a[2]), t1 = csub(a[0], a[2]);
    const float2 t2 = cadd(a[1], a[3]), t3 = cmi(csub(a[1], a[3]));
    a[0] = cadd(t0, t2);
    a[2] = csub(t0, t2);
    a[1] = cadd(t1, t3);
    a[3] = csub(t1, t3);
}

template <>
__device__ __forceinline__ void dft<8>(float2 *a) {
    float2 e[4] = {a[0], a[2], a[4], a[6]}, o[4] = {a[1], a[3], a[5], a[7]};
    dft<4>(e);
    dft<4>(o);
    const float h = 0.70710678118654757f;  // sqrt(1/2)
    // o_k * exp(-2 pi i k / 8)
    const float2 o1 = make_float2(h * (o[1].x + o[1].y), h * (o[1].y - o[1].x));
    const float2 o2 = cmi(o[2]);
    const float2 o3 = make_float2(h * (o[3].y - o[3].x), -h * (o[3].x + o[3].y));
    a[0] = cadd(e[0], o[0]);
    a[4] = csub(e[0], o[0]);
    a[1] = cadd(e[1], o1);
    a[5] = csub(e[1], o1);
    a[2] = cadd(e[2], o2);
    a[6] = csub(e[2], o2);
    a[3] = cadd(e[3], o3);
    a[7] = csub(e[3], o3);
}

template <>
__device__ __forceinline__ void dft<3>(float2 *a) {
    const float s = 0.86602540378443871f;  // sin(2 pi / 3)
    const float2 t = cadd(a[1], a[2]), d = csub(a[1], a[2]);
    const float2 m = caxpy(-0.5f, t, a[0]);
    const float2 u = make_float2(s * d.y, -s * d.x);  // -i s d
    a[0] = cadd(a[0], t);
    a[1] = cadd(m, u);
    a[2] = csub(m, u);
}

template <>
__device__ __forceinline__ void dft<5>(float2 *a) {
    // cos and sin of 2 pi / 5 and 4 pi / 5
    const float c1 = 0.30901699437494745f, c2 = -0.80901699437494734f;
    const float s1 = 0.95105651629515353f, s2 = 0.58778525229247325f;
    const float2 t1 = cadd(a[1], a[4]), t2 = cadd(a[2], a[3]);
    const float2 t3 = csub(a[1], a[4]), t4 = csub(a[2], a[3]);
    const float2 p1 = caxpy(c2, t2, caxpy(c1, t1, a[0]));
    const float2 p2 = caxpy(c1, t2, caxpy(c2, t1, a[0]));
    const float2 q1 = caxpy(s2, t4, make_float2(s1 * t3.x, s1 * t3.y));
    const float2 q2 = caxpy(-s1, t4, make_float2(s2 * t3.x, s2 * t3.y));
    a[0] = cadd(a[0], cadd(t1, t2));
    a[1] = cadd(p1, cmi(q1));
    a[4] = csub(p1, cmi(q1));
    a[2] = cadd(p2, cmi(q2));
    a[3] = csub(p2, cmi(q2));
}

template <>
__device__ __forceinline__ void dft<7>(float2 *a) {
    // cos and sin of 2 pi k / 7
    const float C[7] = {1.f, 0.62348980185873359f, -0.22252093395631434f, -0.90096886790241903f,
                        -0.90096886790241915f, -0.22252093395631459f, 0.62348980185873337f};
    const float S[7] = {0.f, 0.7818314824680298f, 0.97492791218182362f, 0.43388373911755823f,
                        -0.43388373911755801f, -0.97492791218182362f, -0.78183148246802991f};
    float2 t[4], d[4];
#pragma unroll
    for (int k = 1; k <= 3; ++k) {
        t[k] = cadd(a[k], a[7 - k]);
        d[k] = csub(a[k], a[7 - k]);
    }
    const float2 a0 = a[0];
    a[0] = cadd(a0, cadd(t[1], cadd(t[2], t[3])));
#pragma unroll
    for (int m = 1; m <= 3; ++m) {
        float2 p = a0, q = make_float2(0.f, 0.f);
#pragma unroll
        for (int k = 1; k <= 3; ++k) {
            p = caxpy(C[(k * m) % 7], t[k], p);
            q = caxpy(S[(k * m) % 7], d[k], q);
        }
        a[m] = cadd(p, cmi(q));
        a[7 - m] = csub(p, cmi(q));
    }
}

template <>
__device__ __forceinline__ void dft<10>(float2 *a) {
    float2 e[5] = {a[0], a[2], a[4], a[6], a[8]}, o[5] = {a[1], a[3], a[5], a[7], a[9]};
    dft<5>(e);
    dft<5>(o);
    // exp(-2 pi i k / 10), k = 1..4
    const float c1 = 0.80901699437494745f, s1 = 0.58778525229247314f;
    const float c2 = 0.30901699437494745f, s2 = 0.95105651629515353f;
    const float2 w[5] = {make_float2(1.f, 0.f), make_float2(c1, -s1), make_float2(c2, -s2), make_float2(-c2, -s2),
                         make_float2(-c1, -s1)};
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const float2 t = k ? cmul(o[k], w[k]) : o[0];
        a[k] = cadd(e[k], t);
        a[k + 5] = csub(e[k], t);
    }
}

// N = N1 N2 point DFT by one mixed-radix split: with n = n1 + N1 n2 and
// k = N2 k1 + k2, b_k = sum_n1 W_N1^(n1 k1) W_N^(n1 k2) sum_n2 W_N2^(n2 k2) a_n:
// N1 inner N2-point DFTs, the twiddles W_N^(n1 k2), N2 outer N1-point DFTs.
// C / S hold cos / sin of 2 pi m / N, m = 0..N-1 (constant-folded once unrolled).
template <int N1, int N2>
__device__ __forceinline__ void dft_split(float2 *a, const float *C, const float *S) {
    constexpr int N = N1 * N2;
    float2 y[N1][N2];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) {
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) y[n1][n2] = a[n1 + N1 * n2];
        dft<N2>(y[n1]);
    }
#pragma unroll
    for (int n1 = 1; n1 < N1; ++n1)
#pragma unroll
        for (int k2 = 1; k2 < N2; ++k2) {
            const int m = (n1 * k2) % N;
            y[n1][k2] = cmul(y[n1][k2], make_float2(C[m], -S[m]));
        }
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) {
        float2 z[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; ++n1) z[n1] = y[n1][k2];
        dft<N1>(z);
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) a[N2 * k1 + k2] = z[k1];
    }
}

template <>
__device__ __forceinline__ void dft<16>(float2 *a) {
    // cos and sin of 2 pi m / 16, m = 0..7 (the split uses m = k2 < 8)
    const float C[8] = {1.f, 0.92387953251128674f, 0.70710678118654757f, 0.38268343236508984f,
                        0.f, -0.38268343236508973f, -0.70710678118654746f, -0.92387953251128674f};
    const float S[8] = {0.f, 0.38268343236508978f, 0.70710678118654746f, 0.92387953251128674f,
                        1.f, 0.92387953251128674f, 0.70710678118654757f, 0.38268343236508989f};
    dft_split<2, 8>(a, C, S);
}

template <>
__device__ __forceinline__ void dft<15>(float2 *a) {
    // cos and sin of 2 pi m / 15
    const float C[15] = {1.f, 0.91354545764260087f, 0.66913060635885824f, 0.30901699437494745f,
                         -0.10452846326765333f, -0.49999999999999978f, -0.80901699437494734f,
                         -0.97814760073380569f, -0.97814760073380569f, -0.80901699437494756f,
                         -0.50000000000000044f, -0.10452846326765423f, 0.30901699437494723f,
                         0.66913060635885846f, 0.91354545764260098f};
    const float S[15] = {0.f, 0.40673664307580015f, 0.74314482547739413f, 0.95105651629515353f,
                         0.9945218953682734f, 0.86602540378443871f, 0.58778525229247325f,
                         0.20791169081775931f, -0.20791169081775907f, -0.58778525229247303f,
                         -0.86602540378443837f, -0.99452189536827329f, -0.95105651629515364f,
                         -0.74314482547739402f, -0.40673664307580015f};
    dft_split<3, 5>(a, C, S);
}

template <>
__device__ __forceinline__ void dft<25>(float2 *a) {
    // cos and sin of 2 pi m / 25
    const float C[25] = {1.f, 0.96858316112863108f, 0.87630668004386358f, 0.72896862742141155f,
                         0.53582679497899655f, 0.30901699437494745f, 0.062790519529313527f,
                         -0.1873813145857246f, -0.42577929156507272f, -0.63742398974868975f,
                         -0.80901699437494734f, -0.92977648588825135f, -0.99211470131447776f,
                         -0.99211470131447788f, -0.92977648588825146f, -0.80901699437494778f,
                         -0.63742398974868952f, -0.42577929156507216f, -0.18738131458572463f,
                         0.062790519529312833f, 0.30901699437494723f, 0.53582679497899677f,
                         0.72896862742141122f, 0.87630668004386314f, 0.96858316112863097f};
    const float S[25] = {0.f, 0.24868988716485479f, 0.48175367410171532f, 0.68454710592868862f,
                         0.84432792550201508f, 0.95105651629515353f, 0.99802672842827156f,
                         0.98228725072868872f, 0.90482705246601947f, 0.77051324277578925f,
                         0.58778525229247325f, 0.36812455268467814f, 0.12533323356430454f,
                         -0.12533323356430429f, -0.36812455268467792f, -0.58778525229247269f,
                         -0.77051324277578936f, -0.9048270524660198f, -0.98228725072868872f,
                         -0.99802672842827156f, -0.95105651629515364f, -0.84432792550201496f,
                         -0.68454710592868895f, -0.4817536741017161f, -0.24868988716485535f};
    dft_split<5, 5>(a, C, S);
}

// One Stockham stage over the CTA's 16 columns (rows PITCH float2 apart); a
// thread takes two adjacent columns (one float4) of each of its butterflies.
template <int R, int PITCH>
__device__ __forceinline__ void fft_stage(const float2 *__restrict__ src, float2 *__restrict__ dst, int m, int ns,
                                          unsigned magic, const float2 *__restrict__ tw, int stream, int cp) {
    for (int i = stream; i < m; i += kPairStreams) {
        const int j = ns == 1 ? 0 : i - (int)__umulhi((unsigned)i, magic) * ns;
        float2 a[R], b[R];
#pragma unroll
        for (int q = 0; q < R; ++q) {
            const float4 v = *reinterpret_cast<const float4 *>(src + (i + q * m) * PITCH + 2 * cp);
            a[q] = make_float2(v.x, v.y);
            b[q] = make_float2(v.z, v.w);
        }
        if (j != 0) {
#pragma unroll
            for (int q = 1; q < R; ++q) {
                const float2 w = __ldg(tw + j * (R - 1) + (q - 1));
                a[q] = cmul(a[q], w);
                b[q] = cmul(b[q], w);
            }
        }
        dft<R>(a);
        dft<R>(b);
        const int base = (i - j) * R + j;
#pragma unroll
        for (int k = 0; k < R; ++k)
            *reinterpret_cast<float4 *>(dst + (base + k * ns) * PITCH + 2 * cp) = make_float4(a[k].x, a[k].y, b[k].x, b[k].y);
    }
}

// The stage plan of a transform length: the radix order 8, 10, 5, 4, 3, 7, 2, each
// as often as it divides, except for the lengths of the benchmark grids, which run
// two stages (one CTA barrier and one shared-memory round trip fewer than the three
// the radix order gives): 240 = 16 x 15, 250 = 25 x 10, 160 = 16 x 10 and
// 256 = 16 x 16.  make_axis builds the twiddle table from the same plan, so the
// compile-time and table-driven forms agree; radices 15, 16 and 25 only occur in
// the compile-time form.
constexpr int kRadixOrder[7] = {8, 10, 5, 4, 3, 7, 2};
struct StagePlan {
    int nst = 0;
    int radix[kFftMaxStages] = {};
    int ns[kFftMaxStages] = {};
    int twoff[kFftMaxStages] = {};  // relative to the axis's first twiddle
};
constexpr StagePlan stage_plan(int n) {
    StagePlan p{};
    int rad[kFftMaxStages] = {};
    int nr = 0;
    if (n == 240) {
        rad[0] = 16;
        rad[1] = 15;
        nr = 2;
    } else if (n == 250) {
        rad[0] = 25;
        rad[1] = 10;
        nr = 2;
    } else if (n == 160) {
        rad[0] = 16;
        rad[1] = 10;
        nr = 2;
    } else if (n == 256) {
        rad[0] = 16;
        rad[1] = 16;
        nr = 2;
    } else {
        int m = n;
        for (int k = 0; k < 7; ++k) {
            const int r = kRadixOrder[k];
            while (m % r == 0 && nr < kFftMaxStages) {
                rad[nr++] = r;
                m /= r;
            }
        }
    }
    int ns = 1, off = 0;
    for (int s = 0; s < nr; ++s) {
        p.radix[s] = rad[s];
        p.ns[s] = ns;
        p.twoff[s] = off;
        off += ns * (rad[s] - 1);
        ns *= rad[s];
    }
    p.nst = nr;
    return p;
}

// One Stockham stage with the radix, stage extent and butterfly count known at
// compile time: the loop over butterflies unrolls, j = i mod ns and every
// shared-memory index reduce to constants plus the thread's stream.
// Source of a stage: position pos of the column pair cp as (col 2cp, col 2cp + 1).
// Rows of PITCH float2, position-major (the layout every stage writes).
template <int PITCH>
struct PitchLoad {
    const float2 *src;
    __device__ __forceinline__ float4 operator()(int pos, int cp) const {
        return *reinterpret_cast<const float4 *>(src + pos * PITCH + 2 * cp);
    }
    // position pos of column c alone
    __device__ __forceinline__ float2 one(int pos, int c) const { return src[pos * PITCH + c]; }
};

// Source of the first stage of an x pass: 16 rows (one per vector) of `pitch`
// float2 as loaded from global memory (row-major); position pos holds element
// x = (pos + rot) mod n of its row, zero where x >= len (the pruned input)
struct RowMajorLoad {
    const float2 *src;
    int pitch, n, rot, len;
    __device__ __forceinline__ float4 operator()(int pos, int cp) const {
        int x = pos + rot;
        if (x >= n) x -= n;
        if (x >= len) return make_float4(0.f, 0.f, 0.f, 0.f);
        const float2 a = src[(2 * cp) * pitch + x], b = src[(2 * cp + 1) * pitch + x];
        return make_float4(a.x, a.y, b.x, b.y);
    }
    __device__ __forceinline__ float2 one(int pos, int c) const {
        int x = pos + rot;
        if (x >= n) x -= n;
        if (x >= len) return make_float2(0.f, 0.f);
        return src[c * pitch + x];
    }
};

// Radices whose stages run with one column per thread (16 columns x 16 butterfly
// streams): a butterfly of two columns would hold 30 to 50 complex values
constexpr bool one_col_radix(int r) { return r >= 15; }
constexpr int kColStreams = kThreads / kCols;

// A Stockham stage with one column per thread: thread t takes column t mod 16 of
// butterflies t / 16, t / 16 + 16, ...  Same positions, twiddles and results as
// the two-column form.
template <int R, int NS, int M, int PITCH, class L>
__device__ __forceinline__ void fft_stage1_cl(const L &ld, float2 *__restrict__ dst, const float2 *__restrict__ tw) {
    constexpr int IT = (M + kColStreams - 1) / kColStreams;
    const int c = threadIdx.x & (kCols - 1), stream = threadIdx.x / kCols;
#pragma unroll
    for (int it = 0; it < IT; ++it) {
        const int i = stream + it * kColStreams;
        if (M % kColStreams != 0 && i >= M) break;
        const int j = NS == 1 ? 0 : i % NS;
        float2 a[R];
#pragma unroll
        for (int q = 0; q < R; ++q) a[q] = ld.one(i + q * M, c);
        if (NS > 1 && j != 0) {
#pragma unroll
            for (int q = 1; q < R; ++q) a[q] = cmul(a[q], __ldg(tw + j * (R - 1) + (q - 1)));
        }
        dft<R>(a);
        const int base = (i - j) * R + j;
#pragma unroll
        for (int k = 0; k < R; ++k) dst[(base + k * NS) * PITCH + c] = a[k];
    }
}

template <int R, int NS, int M, int PITCH, class L>
__device__ __forceinline__ void fft_stage_cl(const L &ld, float2 *__restrict__ dst, const float2 *__restrict__ tw,
                                             int stream, int cp) {
    constexpr int IT = (M + kPairStreams - 1) / kPairStreams;
#pragma unroll
    for (int it = 0; it < IT; ++it) {
        const int i = stream + it * kPairStreams;
        if (M % kPairStreams != 0 && i >= M) break;
        const int j = NS == 1 ? 0 : i % NS;
        float2 a[R], b[R];
#pragma unroll
        for (int q = 0; q < R; ++q) {
            const float4 v = ld(i + q * M, cp);
            a[q] = make_float2(v.x, v.y);
            b[q] = make_float2(v.z, v.w);
        }
        if (NS > 1 && j != 0) {
#pragma unroll
            for (int q = 1; q < R; ++q) {
                const float2 w = __ldg(tw + j * (R - 1) + (q - 1));
                a[q] = cmul(a[q], w);
                b[q] = cmul(b[q], w);
            }
        }
        dft<R>(a);
        dft<R>(b);
        const int base = (i - j) * R + j;
#pragma unroll
        for (int k = 0; k < R; ++k)
            *reinterpret_cast<float4 *>(dst + (base + k * NS) * PITCH + 2 * cp) =
                make_float4(a[k].x, a[k].y, b[k].x, b[k].y);
    }
}

template <int R, int NS, int M, int PITCH>
__device__ __forceinline__ void fft_stage_c(const float2 *__restrict__ src, float2 *__restrict__ dst,
                                            const float2 *__restrict__ tw, int stream, int cp) {
    fft_stage_cl<R, NS, M, PITCH>(PitchLoad<PITCH>{src}, dst, tw, stream, cp);
}

template <int N, int S, int PITCH>
__device__ __forceinline__ void fft_stages_c(float2 *&src, float2 *&dst, const float2 *tw, int stream, int cp) {
    constexpr StagePlan P = stage_plan(N);
    if constexpr (S < P.nst) {
        constexpr int R = P.radix[S], NS = P.ns[S];
        if constexpr (one_col_radix(R))
            fft_stage1_cl<R, NS, N / R, PITCH>(PitchLoad<PITCH>{src}, dst, tw + P.twoff[S]);
        else
            fft_stage_c<R, NS, N / R, PITCH>(src, dst, tw + P.twoff[S], stream, cp);
        __syncthreads();
        float2 *t = src;
        src = dst;
        dst = t;
        fft_stages_c<N, S + 1, PITCH>(src, dst, tw, stream, cp);
    }
}

// forward FFT of the 16 columns held in A (B is scratch; rows PITCH float2
// apart); returns the buffer holding the result.  Ends with the CTA
// synchronised.  The transform lengths of the benchmark grids run a compile-time
// stage plan; other lengths the table-driven loop below (same stages, same
// twiddles, same results).
template <int PITCH = kPitch>
__device__ __forceinline__ float2 *fft_run(float2 *A, float2 *B, const FftAxis &fa) {
    {
        float2 *src = A, *dst = B;
        const int cp = threadIdx.x & (kCols / 2 - 1), stream = threadIdx.x / (kCols / 2);
        switch (fa.n) {
            case 250: fft_stages_c<250, 0, PITCH>(src, dst, fa.tw, stream, cp); return src;
            case 240: fft_stages_c<240, 0, PITCH>(src, dst, fa.tw, stream, cp); return src;
            case 160: fft_stages_c<160, 0, PITCH>(src, dst, fa.tw, stream, cp); return src;
            case 256: fft_stages_c<256, 0, PITCH>(src, dst, fa.tw, stream, cp); return src;
            case 512: fft_stages_c<512, 0, PITCH>(src, dst, fa.tw, stream, cp); return src;
            default: break;
        }
    }
    float2 *src = A, *dst = B;
    const int cp = threadIdx.x & (kCols / 2 - 1), stream = threadIdx.x / (kCols / 2);
    for (int s = 0; s < fa.nst; ++s) {
        const int r = fa.radix[s], ns = fa.ns[s], m = fa.n / r;
        const unsigned mg = fa.magic[s];
        const float2 *tw = fa.tw + fa.twoff[s];
        switch (r) {
            case 2: fft_stage<2, PITCH>(src, dst, m, ns, mg, tw, stream, cp); break;
            case 3: fft_stage<3, PITCH>(src, dst, m, ns, mg, tw, stream, cp); break;
            case 4: fft_stage<4, PITCH>(src, dst, m, ns, mg, tw, stream, cp); break;
            case 5: fft_stage<5, PITCH>(src, dst, m, ns, mg, tw, stream, cp); break;
            case 7: fft_stage<7, PITCH>(src, dst, m, ns, mg, tw, stream, cp); break;
            case 10: fft_stage<10, PITCH>(src, dst, m, ns, mg, tw, stream, cp); break;
            default: fft_stage<8, PITCH>(src, dst, m, ns, mg, tw, stream, cp); break;
        }
        __syncthreads();
        float2 *t = src;
        src = dst;
        dst = t;
    }
    return src;
}

// Forward FFT of length N whose first stage reads its input through `ld` and
// writes B; the later stages ping-pong between B and A (rows PITCH float2 apart).
// Returns the buffer holding the result; ends with the CTA synchronised.
template <int N, int PITCH, class L>
__device__ __forceinline__ float2 *fft_run_first_n(const L &ld, float2 *A, float2 *B, const float2 *tw) {
    constexpr StagePlan SP = stage_plan(N);
    const int cp = threadIdx.x & (kCols / 2 - 1), stream = threadIdx.x / (kCols / 2);
    if constexpr (one_col_radix(SP.radix[0]))
        fft_stage1_cl<SP.radix[0], SP.ns[0], N / SP.radix[0], PITCH>(ld, B, tw + SP.twoff[0]);
    else
        fft_stage_cl<SP.radix[0], SP.ns[0], N / SP.radix[0], PITCH>(ld, B, tw + SP.twoff[0], stream, cp);
    __syncthreads();
    float2 *src = B, *dst = A;
    fft_stages_c<N, 1, PITCH>(src, dst, tw, stream, cp);
    return src;
}

// The same for the transform lengths with a compile-time stage plan; nullptr for
// any other length (the caller only launches with those)
template <int PITCH, class L>
__device__ __forceinline__ float2 *fft_run_first(const L &ld, float2 *A, float2 *B, const FftAxis &fa) {
    switch (fa.n) {
        case 250: return fft_run_first_n<250, PITCH>(ld, A, B, fa.tw);
        case 240: return fft_run_first_n<240, PITCH>(ld, A, B, fa.tw);
        case 160: return fft_run_first_n<160, PITCH>(ld, A, B, fa.tw);
        case 256: return fft_run_first_n<256, PITCH>(ld, A, B, fa.tw);
        case 512: return fft_run_first_n<512, PITCH>(ld, A, B, fa.tw);
        default: return nullptr;
    }
}
bool first_stage_length(int n) { return n == 250 || n == 240 || n == 160 || n == 256 || n == 512; }

// Transform along an outer axis (y or z) of 16 adjacent x positions.
//   mode 0: buffer -> buffer; 1: image -> buffer (forward first pass: deapodisation,
//   C_l, factor); 2: buffer -> image (adjoint last pass: sum over segments of
//   conj(C_l) times the transform, deapodisation, factor, optional accumulate).
// Forward passes read lin = N elements placed at FFT positions (i - N/2) mod n
// and write all n; inverse passes read all n and write lout = N, element o from
// FFT position (o - N/2) mod n.  Strides are in elements; for the image side they
// are the image strides.
struct ColPass {
    FftAxis fa;
    int inv, mode;
    int lin, lout, nax;
    int X, nmid, nplanes;
    int64_t in_plane, in_mid, in_ax;
    int64_t out_plane, out_mid, out_ax;
    const float2 *src;
    float2 *dst;
    Chan ch;
    int C;
    int64_t nvol;
    const float *apod_ax, *apod_mid, *apod_x;
    const float2 *Cl;
    float factor;
    int accumulate;
    int *err;   // device flag of the plan (TMA form: a wait that gave up)
    int nsm;    // SMs of the device (TMA form: persistent grid)
};

// VEC: a thread moves two adjacent columns (16 bytes) in the copy, finish and
// store loops; the host selects it when every base and stride is even in
// elements (16-byte aligned pairs) and X is even.
template <bool VEC>
__global__ void __launch_bounds__(kThreads, 3) col_pass_kernel(const ColPass P) {
    extern __shared__ float2 fsm[];
    const int n = P.fa.n;
    float2 *A = fsm, *Bf = fsm + n * kPitch, *Acc = fsm + 2 * n * kPitch;
    const int nxc = (P.X + kCols - 1) / kCols;
    int blk = blockIdx.x;
    const int xc = blk % nxc;
    blk /= nxc;
    const int mid = blk % P.nmid;
    const int plane = blk / P.nmid;
    // element loops: NC columns per thread starting at column col, NS streams over positions
    constexpr int NC = VEC ? 2 : 1;
    constexpr int NS = kThreads * NC / kCols;
    const int col = (threadIdx.x % (kCols / NC)) * NC, stream = threadIdx.x / (kCols / NC);
    const int x = xc * kCols + col;
    const bool xin = x < P.X;  // VEC: X is even, so both columns of the pair are in or out
    const int xs = xin ? x : P.X - NC;  // in-bounds address for columns past the edge
    const int hn = P.nax / 2;
    const int Kc = P.ch.K ? P.ch.K : 1;
    const int nl = P.mode == 2 ? P.ch.L : 1;
    // per-column factors of the image side (deapodisation across the mid and x axes)
    float amid[NC];
#pragma unroll
    for (int k = 0; k < NC; ++k) {
        amid[k] = P.factor;
        if (P.mode != 0 && P.apod_mid) amid[k] *= P.apod_mid[mid];
        if (P.mode != 0 && P.apod_x) amid[k] *= P.apod_x[xs + k];
    }
    for (int l = 0; l < nl; ++l) {
        int64_t in_base;
        const float2 *cl = nullptr;
        if (P.mode == 1) {  // grid plane (grp, ch) <- image plane (b, c), segment ll
            const int grp = plane / P.ch.nch, chn = plane - grp * P.ch.nch;
            const int k = chn % Kc, lb = chn / Kc, b = lb % P.ch.B, ll = lb / P.ch.B;
            const int c = P.ch.K ? k : grp;
            in_base = ((int64_t)b * P.C + c) * P.nvol + mid * P.in_mid;
            if (P.Cl) cl = P.Cl + (int64_t)ll * P.nvol + mid * P.in_mid;
        } else if (P.mode == 2) {  // image plane (b, c) <- grid plane of segment l
            const int b = plane / P.C, c = plane - b * P.C;
            const int grp = P.ch.K ? 0 : c;
            const int chn = P.ch.K ? (l * P.ch.B + b) * Kc + c : l * P.ch.B + b;
            in_base = ((int64_t)grp * P.ch.nch + chn) * P.in_plane + mid * P.in_mid;
        } else {
            in_base = (int64_t)plane * P.in_plane + mid * P.in_mid;
        }
        // all copies of the column block in flight at once (C_l into the scratch
        // buffer); positions without input are zero-filled.  Offsets along the
        // axis stay in 32 bits (at most 512 x 512^2 elements within a plane).
        const float2 *srcp = P.src + in_base + xs;
        const float2 *clp = cl ? cl + xs : nullptr;
        const int in_ax = (int)P.in_ax;
        for (int p = stream; p < n; p += NS) {
            int i = p;
            if (!P.inv) {
                i = p + hn;
                if (i >= n) i -= n;
            }
            const bool valid = i < P.lin;
            const int off = (valid ? i : 0) * in_ax;
            if (VEC) {
                cp_async16(A + p * kPitch + col, srcp + off, valid);
                if (clp) cp_async16(Bf + p * kPitch + col, clp + off, valid);
            } else {
                cp_async8(A + p * kPitch + col, srcp + off, valid);
                if (clp) cp_async8(Bf + p * kPitch + col, clp + off, valid);
            }
        }
        cp_async_commit();
        cp_async_wait_all();
        if (P.mode == 1 || P.inv) {
            // each thread finishes the elements it copied
            for (int p = stream; p < n; p += NS) {
                int i = p;
                if (!P.inv) {
                    i = p + hn;
                    if (i >= n) i -= n;
                }
                if (i >= P.lin) continue;
#pragma unroll
                for (int k = 0; k < NC; ++k) {
                    float2 v = A[p * kPitch + col + k];
                    if (P.mode == 1) {
                        if (cl) v = cmul(v, Bf[p * kPitch + col + k]);
                        const float a = P.apod_ax ? amid[k] * P.apod_ax[i] : amid[k];
                        v = make_float2(v.x * a, v.y * a);
                    }
                    if (P.inv) v.y = -v.y;
                    A[p * kPitch + col + k] = v;
                }
            }
        }
        __syncthreads();
        const float2 *R = fft_run(A, Bf, P.fa);
        if (P.mode == 2) {
            const int64_t out_base = (int64_t)plane * P.nvol + mid * P.out_mid;
            for (int o = stream; o < P.lout; o += NS) {
                int pp = o - hn;
                if (pp < 0) pp += n;
                const int64_t oo = (int64_t)o * P.out_ax + mid * P.out_mid;
                float2 v[NC];
#pragma unroll
                for (int k = 0; k < NC; ++k) {
                    v[k] = R[pp * kPitch + col + k];
                    v[k].y = -v[k].y;
                    if (P.Cl) v[k] = cmulc(v[k], P.Cl[(int64_t)l * P.nvol + oo + xs + k]);
                    if (l > 0) v[k] = cadd(v[k], Acc[o * kPitch + col + k]);
                }
                if (l + 1 < nl) {
#pragma unroll
                    for (int k = 0; k < NC; ++k) Acc[o * kPitch + col + k] = v[k];
                } else if (xin) {
                    // last segment: deapodise, scale and write the image
#pragma unroll
                    for (int k = 0; k < NC; ++k) {
                        const float a = P.apod_ax ? amid[k] * P.apod_ax[o] : amid[k];
                        v[k] = make_float2(v[k].x * a, v[k].y * a);
                    }
                    float2 *d = P.dst + out_base + (int64_t)o * P.out_ax + x;
                    if (VEC) {
                        float4 r = make_float4(v[0].x, v[0].y, v[NC - 1].x, v[NC - 1].y);
                        if (P.accumulate) {
                            const float4 old = *reinterpret_cast<const float4 *>(d);
                            r.x += old.x;
                            r.y += old.y;
                            r.z += old.z;
                            r.w += old.w;
                        }
                        *reinterpret_cast<float4 *>(d) = r;
                    } else {
                        if (P.accumulate) v[0] = cadd(v[0], *d);
                        *d = v[0];
                    }
                }
            }
            if (l + 1 < nl) __syncthreads();  // the next segment reloads A
        } else {
            float2 *dstp = P.dst + (int64_t)plane * P.out_plane + mid * P.out_mid + x;
            const int out_ax = (int)P.out_ax;
            for (int o = stream; o < P.lout; o += NS) {
                int pp = o;
                if (P.inv) {
                    pp = o - hn;
                    if (pp < 0) pp += n;
                }
                float2 *d = dstp + o * out_ax;
                if (VEC) {
                    float4 r = *reinterpret_cast<const float4 *>(R + pp * kPitch + col);
                    if (P.inv) {
                        r.y = -r.y;
                        r.w = -r.w;
                    }
                    if (xin) *reinterpret_cast<float4 *>(d) = r;
                } else {
                    float2 v = R[pp * kPitch + col];
                    if (P.inv) v.y = -v.y;
                    if (xin) *d = v;
                }
            }
        }
    }
}

// ------------------------------------------------------------------------------------
// Column pass on the tensor memory accelerator: a persistent CTA walks column
// tiles (16 adjacent x positions x the whole axis, one (mid, plane)), each loaded
// by TMA into one slot of a two-slot ring while the previous tile transforms.
// Rows are dense in shared memory (16 float2 = 128 bytes, the box layout), so
// forward passes also leave by TMA store.  Inverse passes run the forward
// transform and read its output reversed, IDFT(x)[k] = DFT(x)[(n - k) mod n],
// which needs no conjugation of the input or output.
// ------------------------------------------------------------------------------------
constexpr int kTmaPitch = kCols;        // float2 per shared row: one 128-byte TMA box row
constexpr int kTmaMaxBoxes = 8;         // load boxes per tile
constexpr int kWaitLimit = 1 << 20;     // mbarrier polls before a wait gives up

struct ColTma {
    FftAxis fa;
    int inv, mode;          // as ColPass: 0 buffer -> buffer, 1 image -> buffer, 2 buffer -> image
    int lin, lout, hn;      // rows read / written; hn: rotation of the fftshift (nax / 2)
    int X, nxc, nmid, nplanes;
    int ntiles;             // output blocks (16 x positions of one (mid, plane))
    int nseg;               // tiles per output block: the B0 segments summed by an adjoint last pass, else 1
    int nbox;               // load boxes per tile: smem row, source row (before the +hn rotation fold)
    int box_smem[kTmaMaxBoxes], box_src[kTmaMaxBoxes];
    int br;                 // rows per load box
    int nsbox, sbr;         // forward stores: boxes and rows per box (overlapping last box)
    int64_t out_plane, out_mid, out_ax;  // plain stores (inverse passes)
    float2 *dst;
    Chan ch;
    int C;
    int64_t nvol;
    const float *apod_ax, *apod_mid, *apod_x;
    const float2 *Cl;       // B0 segment factors on the image side (nseg x nvol), or null
    int64_t img_mid, img_ax;  // image strides of Cl (the image side's mid and axis strides)
    float factor;
    int accumulate;
    int *err;               // set to 1 when a wait gives up (the results are then invalid)
};

__device__ __forceinline__ unsigned smem_u32(const void *p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// bounded wait for the phase with the given parity to complete
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity) {
    const unsigned a = smem_u32(bar);
    for (int it = 0; it < kWaitLimit; ++it) {
        unsigned done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
// 4D tiled TMA load into this CTA's shared memory, completing on `bar`
__device__ __forceinline__ void tma_load4(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                          uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(smem_u32(dst)),
        "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}
// 4D tiled TMA store from shared memory (bulk-group completion)
__device__ __forceinline__ void tma_store4(const CUtensorMap *map, int c0, int c1, int c2, int c3, const void *src) {
    asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4}], [%5];" ::"l"(map),
                 "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(src))
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

struct TileInfo {
    int xc, mid, plane, l;  // l: segment of an adjoint last pass (0 otherwise)
};

// src_map: the pass's source as 4D (2X floats, rows, mid, source plane); dst_map:
// the destination of forward passes (2X floats, n rows, mid, plane).
// NSLOT ring slots: 2 (the next tile loads while this one transforms; 2 CTAs per
// SM) or 1 (3 CTAs per SM overlap instead: slower, 1.30 against 1.21 ms for the
// 200^3 z pass, 1.45 against 1.21 ms for the y pass)
// SEG: B0 factors and segment sums (forward first passes with C_l, adjoint last
// passes over several segments); the plain instantiation keeps its simpler loops.
template <int NSLOT, bool SEG>
__global__ void __launch_bounds__(kThreads, NSLOT == 1 ? 3 : 2)
    col_tma_kernel(const __grid_constant__ CUtensorMap src_map, const __grid_constant__ CUtensorMap dst_map,
                   const ColTma P) {
    extern __shared__ __align__(128) float2 tsm[];
    __shared__ __align__(8) uint64_t full[2];
    __shared__ TileInfo info[2];
    const int n = P.fa.n;
    // slot s of the ring at tsm + s * n rows, the transform's scratch buffer after them
    float2 *scr = tsm + NSLOT * n * kTmaPitch;
    const int col = (threadIdx.x % (kCols / 2)) * 2, stream = threadIdx.x / (kCols / 2);
    constexpr int NS = kThreads * 2 / kCols;  // row streams: a thread moves two adjacent columns
    const unsigned box_bytes = (unsigned)P.br * kTmaPitch * sizeof(float2);
    const bool fwd_store = P.mode != 2 && !P.inv;
    // thread 0: load segment l of output block t into slot s (tile coordinates go with
    // it through shared memory)
    auto issue = [&](int t, int l, int s) {
        const int r = t / P.nxc, xc = t - r * P.nxc;
        const int plane = r / P.nmid, mid = r - plane * P.nmid;
        int sp = plane;  // source plane
        if (P.mode == 1) {  // grid plane (grp, ch) <- image plane (b, c)
            const int Kc = P.ch.K ? P.ch.K : 1;
            const int grp = plane / P.ch.nch, chn = plane - grp * P.ch.nch;
            const int k = chn % Kc, b = (chn / Kc) % P.ch.B;
            sp = b * P.C + (P.ch.K ? k : grp);
        } else if (P.mode == 2) {  // image plane (b, c) <- grid plane (grp, chn) of segment l
            const int b = plane / P.C, c = plane - b * P.C;
            const int Kc = P.ch.K ? P.ch.K : 1;
            sp = (P.ch.K ? 0 : c) * P.ch.nch + (P.ch.K ? (l * P.ch.B + b) * Kc + c : l * P.ch.B + b);
        }
        info[s] = TileInfo{xc, mid, plane, l};
        mbar_expect_tx(&full[s], box_bytes * P.nbox);
        for (int b = 0; b < P.nbox; ++b)
            tma_load4(tsm + (s * n + P.box_smem[b]) * kTmaPitch, &src_map, xc * 2 * kCols, P.box_src[b], mid, sp,
                      &full[s]);
    };
    // the CTA's k-th tile: segment k mod nseg of its output block k / nseg (the
    // segments of one block are consecutive, so one CTA sums them)
    auto block_of = [&](int kk, int &l) {
        const int q = SEG ? kk / P.nseg : kk;
        l = kk - q * P.nseg;
        return (int)blockIdx.x + q * (int)gridDim.x;
    };
    if (threadIdx.x == 0) {
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int s = 0; s < NSLOT; ++s) {
            int l;
            const int t = block_of(s, l);
            if (t < P.ntiles) issue(t, l, s);
        }
    }
    bool store_pending = false;  // thread 0: a TMA store of the scratch buffer may still be reading it
    for (int k = 0;; ++k) {
        int lk;
        const int t = block_of(k, lk);
        if (t >= P.ntiles) break;
        const int s = NSLOT == 1 ? 0 : k & 1;
        bool ok = mbar_wait(&full[s], (NSLOT == 1 ? k : k >> 1) & 1);
        const TileInfo ti = info[s];
        float2 *A = tsm + s * n * kTmaPitch;
        const int x = ti.xc * kCols + col;
        const bool xin = x < P.X;
        const int xs = xin ? x : P.X - 2;
        float amid0 = P.factor, amid1 = P.factor;
        if (P.mode != 0) {
            if (P.apod_mid) {
                amid0 *= P.apod_mid[ti.mid];
                amid1 *= P.apod_mid[ti.mid];
            }
            if (P.apod_x) {
                amid0 *= P.apod_x[xs];
                amid1 *= P.apod_x[xs + 1];
            }
        }
        if (SEG && ok && P.mode == 1) {
            // B0 factors of the plane's segment, then deapodise, on the rows that hold
            // image data (the others were filled with zeros)
            const float2 *clp = nullptr;
            if (P.Cl) {
                const int Kc = P.ch.K ? P.ch.K : 1;
                const int chn = ti.plane % P.ch.nch;
                const int ll = chn / Kc / P.ch.B;
                clp = P.Cl + (int64_t)ll * P.nvol + (int64_t)ti.mid * P.img_mid + xs;
            }
            // kU rows per thread at a time: their factor loads are all in flight
            // before the first product
            constexpr int kU = 4;
            for (int p0 = stream; p0 < n; p0 += kU * NS) {
                int ii[kU];
                float aa[kU];
                float4 cc[kU];
#pragma unroll
                for (int u = 0; u < kU; ++u) {
                    const int p = p0 + u * NS;
                    int i = p + P.hn;
                    if (i >= n) i -= n;
                    ii[u] = p < n && i < P.lin ? i : -1;
                    const int ic = ii[u] < 0 ? 0 : ii[u];
                    aa[u] = P.apod_ax ? P.apod_ax[ic] : 1.f;
                    cc[u] = clp ? __ldg(reinterpret_cast<const float4 *>(clp + (int64_t)ic * P.img_ax))
                                : make_float4(0.f, 0.f, 0.f, 0.f);
                }
#pragma unroll
                for (int u = 0; u < kU; ++u) {
                    if (ii[u] < 0) continue;
                    float4 *q = reinterpret_cast<float4 *>(A + (p0 + u * NS) * kTmaPitch + col);
                    float4 v = *q;
                    if (clp) {
                        const float2 v0 = cmul(make_float2(v.x, v.y), make_float2(cc[u].x, cc[u].y));
                        const float2 v1 = cmul(make_float2(v.z, v.w), make_float2(cc[u].z, cc[u].w));
                        v = make_float4(v0.x, v0.y, v1.x, v1.y);
                    }
                    const float a0 = aa[u] * amid0, a1 = aa[u] * amid1;
                    v.x *= a0;
                    v.y *= a0;
                    v.z *= a1;
                    v.w *= a1;
                    *q = v;
                }
            }
        } else if (ok && P.mode == 1) {
            // deapodise the rows that hold image data (the others were filled with zeros)
            for (int p = stream; p < n; p += NS) {
                int i = p + P.hn;
                if (i >= n) i -= n;
                if (i >= P.lin) continue;
                const float a = P.apod_ax ? P.apod_ax[i] : 1.f;
                float4 *q = reinterpret_cast<float4 *>(A + p * kTmaPitch + col);
                float4 v = *q;
                const float a0 = a * amid0, a1 = a * amid1;
                v.x *= a0;
                v.y *= a0;
                v.z *= a1;
                v.w *= a1;
                *q = v;
            }
        }
        // the previous tile's TMA store has read the scratch buffer before the
        // transform below writes it; every thread agrees on the wait's outcome
        if (threadIdx.x == 0 && store_pending) {
            bulk_wait_read0();
            store_pending = false;
        }
        ok = __syncthreads_and(ok);
        if (!ok) {
            if (threadIdx.x == 0) {
                atomicExch(P.err, 1);
                // the other slot's load, if one is in flight
                int l1;
                if (NSLOT == 2 && block_of(k + 1, l1) < P.ntiles) mbar_wait(&full[s ^ 1], ((k + 1) >> 1) & 1);
                if (store_pending) bulk_wait_read0();
            }
            return;
        }
        const float2 *R = fft_run<kTmaPitch>(A, scr, P.fa);
        int ln;
        const int tn = block_of(k + NSLOT, ln);  // the next tile for this slot
        if (fwd_store) {
            // rows 0..n-1 of the result are the output rows: TMA store from shared memory
            fence_async_smem();
            __syncthreads();
            if (threadIdx.x == 0) {
                for (int b = 0; b < P.nsbox; ++b) {
                    const int r0 = b + 1 < P.nsbox ? b * P.sbr : n - P.sbr;
                    tma_store4(&dst_map, ti.xc * 2 * kCols, r0, ti.mid, ti.plane, R + r0 * kTmaPitch);
                }
                bulk_commit();
                // refill the slot now unless the store reads it; a store of the scratch
                // buffer is waited for before the next transform
                if (R == A) bulk_wait_read0();
                else store_pending = true;
                if (tn < P.ntiles) issue(tn, ln, s);
            }
            continue;
        } else {
            // output row o holds inverse-transform position pp = (o - hn) mod n, i.e. the
            // forward transform's position (n - pp) mod n
            const int64_t obase = P.mode == 2 ? (int64_t)ti.plane * P.nvol + (int64_t)ti.mid * P.out_mid
                                              : (int64_t)ti.plane * P.out_plane + (int64_t)ti.mid * P.out_mid;
            if (SEG) {
                // kU rows per thread at a time: the factor and partial-sum loads of an
                // adjoint last pass are all in flight before the first product
                constexpr int kU = 3;
                const bool seg_sum = P.mode == 2 && (P.accumulate || ti.l > 0);
                const float2 *clp =
                    P.mode == 2 && P.Cl ? P.Cl + (int64_t)ti.l * P.nvol + (int64_t)ti.mid * P.out_mid : nullptr;
                for (int o0 = stream; o0 < P.lout; o0 += kU * NS) {
                    float4 cc[kU], old[kU];
                    float aa[kU];
#pragma unroll
                    for (int u = 0; u < kU; ++u) {
                        const int o = o0 + u * NS;
                        const int oc = o < P.lout ? o : 0;
                        if (P.mode == 2 && xin) {
                            const int64_t off = (int64_t)oc * P.out_ax + x;
                            cc[u] = clp ? __ldg(reinterpret_cast<const float4 *>(clp + off))
                                        : make_float4(0.f, 0.f, 0.f, 0.f);
                            // segments after the first add to the sum this thread stored for
                            // the ones before (same addresses, same thread: a plain load)
                            old[u] = seg_sum ? *reinterpret_cast<const float4 *>(P.dst + obase + off)
                                             : make_float4(0.f, 0.f, 0.f, 0.f);
                            aa[u] = P.apod_ax ? P.apod_ax[oc] : 1.f;
                        }
                    }
#pragma unroll
                    for (int u = 0; u < kU; ++u) {
                        const int o = o0 + u * NS;
                        if (o >= P.lout || !xin) continue;
                        int pp = o - P.hn;
                        if (pp < 0) pp += n;
                        const int q = pp == 0 ? 0 : n - pp;
                        float4 w = *reinterpret_cast<const float4 *>(R + q * kTmaPitch + col);
                        if (P.mode == 2) {
                            if (clp) {  // times conj(C_l) of the tile's segment
                                const float2 v0 = cmulc(make_float2(w.x, w.y), make_float2(cc[u].x, cc[u].y));
                                const float2 v1 = cmulc(make_float2(w.z, w.w), make_float2(cc[u].z, cc[u].w));
                                w = make_float4(v0.x, v0.y, v1.x, v1.y);
                            }
                            const float a0 = aa[u] * amid0, a1 = aa[u] * amid1;
                            w.x *= a0;
                            w.y *= a0;
                            w.z *= a1;
                            w.w *= a1;
                            if (seg_sum) {
                                w.x += old[u].x;
                                w.y += old[u].y;
                                w.z += old[u].z;
                                w.w += old[u].w;
                            }
                        }
                        *reinterpret_cast<float4 *>(P.dst + obase + (int64_t)o * P.out_ax + x) = w;
                    }
                }
            } else {
                for (int o = stream; o < P.lout; o += NS) {
                    int pp = o - P.hn;
                    if (pp < 0) pp += n;
                    const int q = pp == 0 ? 0 : n - pp;
                    float4 v = *reinterpret_cast<const float4 *>(R + q * kTmaPitch + col);
                    if (!xin) continue;
                    float4 *d = reinterpret_cast<float4 *>(P.dst + obase + (int64_t)o * P.out_ax + x);
                    if (P.mode == 2) {
                        const float a = P.apod_ax ? P.apod_ax[o] : 1.f;
                        const float a0 = a * amid0, a1 = a * amid1;
                        v.x *= a0;
                        v.y *= a0;
                        v.z *= a1;
                        v.w *= a1;
                        if (P.accumulate) {
                            const float4 old = *d;
                            v.x += old.x;
                            v.y += old.y;
                            v.z += old.z;
                            v.w += old.w;
                        }
                    }
                    *d = v;
                }
            }
            // the slot and the scratch buffer are read; the generic accesses are ordered
            // before the slot's next TMA load
            fence_async_smem();
            __syncthreads();
        }
        // refill this slot with the tile after next
        if (threadIdx.x == 0 && tn < P.ntiles) issue(tn, ln, s);
    }
    if (threadIdx.x == 0 && store_pending) bulk_wait_read0();
}

// ------------------------------------------------------------------------------------
// x passes on TMA (row_tma_kernel).  A tile is 16 consecutive vectors (rows along x);
// each row arrives by 2D tensor-map boxes, `pitch` float2 apart in shared memory, into
// one slot of a two-slot ring while the previous tile transforms.  The first radix
// stage reads that row-major layout (RowMajorLoad: the fftshift rotation and the zero
// padding fold into its index) and writes the position-major layout of the later
// stages.  Forward: rows of T (N0 long, [plane][kz][ky][x]) -> the interleaved grid,
// the 16 vectors being 16 consecutive channels of one (group, kz, ky), stored by TMA
// as boxes of 16 channels x kx (rows 16 float2 wide).  Adjoint: rows of the planar
// grid (n long) -> rows of T cropped to N0, read back reversed (IDFT(x)[k] =
// DFT(x)[(n - k) mod n], no conjugation) from rows of 18 float2 (conflict-free column
// reads) and stored coalesced along x.
// ------------------------------------------------------------------------------------
struct RowTma {
    FftAxis fa;
    int N0, len, rot;   // input row length; first-stage rotation (forward N0 / 2, adjoint 0)
    int hn;             // adjoint crop rotation (N0 / 2)
    int nvec, ntiles;
    int nch, nos1, nos2;
    int pitch;          // x extent of the load box = float2 between the loaded rows (>= len;
                        // the columns past len are zero-filled)
    int nsbox, sbr;     // forward stores: boxes along kx and rows per box (last box overlapping)
    int slot;           // float2 per ring slot
    float2 *dst;        // adjoint output
    int *err;
};

__device__ __forceinline__ void tma_load2(void *dst, const CUtensorMap *map, int c0, int c1, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(smem_u32(dst)),
        "l"(map), "r"(c0), "r"(c1), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tma_load3(void *dst, const CUtensorMap *map, int c0, int c1, int c2, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_u32(dst)),
        "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}

template <bool INV>
__global__ void __launch_bounds__(kThreads, 2)
    row_tma_kernel(const __grid_constant__ CUtensorMap src_map, const __grid_constant__ CUtensorMap dst_map,
                   const RowTma P) {
    constexpr int PITCH = INV ? kPitch : kTmaPitch;
    extern __shared__ __align__(128) float2 tsm[];
    __shared__ __align__(8) uint64_t full[2];
    const int n = P.fa.n;
    float2 *scr = tsm + 2 * P.slot;
    // thread 0: load tile t into slot s as one box of 16 rows of P.pitch (rows past the
    // last vector and columns past the row length are zero-filled).  A tensor copy's
    // shared-memory destination must be 128-byte aligned: the slots are; a slot that
    // is not (never by construction) sets the error flag and is not loaded
    auto issue = [&](int t, int s) {
        float2 *dst = tsm + s * P.slot;
        const int u0 = t * kCols;
        if (smem_u32(dst) & 127u) {
            atomicExch(P.err, 1);
            mbar_expect_tx(&full[s], 0);
            return;
        }
        mbar_expect_tx(&full[s], (unsigned)(kCols * P.pitch * sizeof(float2)));
        if (INV) {
            tma_load2(dst, &src_map, 0, u0, &full[s]);  // 16 consecutive rows of the planar grid
        } else {
            // 16 consecutive channels of one (group, kz, ky): planes grp nch + chn0 ..
            const int chn0 = u0 % P.nch;
            int r = u0 / P.nch;
            const int ky = r % P.nos1;
            r /= P.nos1;
            const int kz = r % P.nos2, grp = r / P.nos2;
            tma_load3(dst, &src_map, 0, kz * P.nos1 + ky, grp * P.nch + chn0, &full[s]);
        }
    };
    if (threadIdx.x == 0) {
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int s = 0; s < 2; ++s) {
            const int t = blockIdx.x + s * gridDim.x;
            if (t < P.ntiles) issue(t, s);
        }
    }
    int k = 0;
    bool store_pending = false;  // thread 0: a TMA store of the scratch buffer may still be reading it
    for (int t = blockIdx.x; t < P.ntiles; t += gridDim.x, ++k) {
        const int s = k & 1;
        bool ok = mbar_wait(&full[s], (k >> 1) & 1);
        float2 *S = tsm + s * P.slot;
        if (threadIdx.x == 0 && store_pending) {
            bulk_wait_read0();
            store_pending = false;
        }
        ok = __syncthreads_and(ok);
        if (!ok) {
            if (threadIdx.x == 0) {
                atomicExch(P.err, 1);
                if (t + (int)gridDim.x < P.ntiles) mbar_wait(&full[s ^ 1], ((k + 1) >> 1) & 1);
                if (store_pending) bulk_wait_read0();
            }
            return;
        }
        const RowMajorLoad ld{S, P.pitch, n, P.rot, P.len};
        const float2 *R = fft_run_first<PITCH>(ld, S, scr, P.fa);
        const int u0 = t * kCols;
        const int tn = t + 2 * gridDim.x;
        if (!INV) {
            // rows kx of the result are 16 channels of point (kz, ky, kx): TMA store
            fence_async_smem();
            __syncthreads();
            if (threadIdx.x == 0) {
                const int chn0 = u0 % P.nch;
                int r = u0 / P.nch;
                const int ky = r % P.nos1;
                r /= P.nos1;
                const int kz = r % P.nos2, grp = r / P.nos2;
                for (int b = 0; b < P.nsbox; ++b) {
                    const int r0 = b + 1 < P.nsbox ? b * P.sbr : n - P.sbr;
                    tma_store4(&dst_map, chn0, r0, kz * P.nos1 + ky, grp, R + r0 * PITCH);
                }
                bulk_commit();
                // refill the slot now unless the store reads it; a store of the scratch
                // buffer is waited for before the next transform
                if (R == S) bulk_wait_read0();
                else store_pending = true;
                if (tn < P.ntiles) issue(tn, s);
            }
            continue;
        }
        // adjoint: element x < N0 of vector v is inverse-transform position
        // pp = (x - hn) mod n, i.e. forward position (n - pp) mod n
        {
            const int v = threadIdx.x >> 4, lx = threadIdx.x & 15;
            const int u = u0 + v;
            if (u < P.nvec) {
                float2 *d = P.dst + (int64_t)u * P.N0;
                for (int x = lx; x < P.N0; x += 16) {
                    int pp = x - P.hn;
                    if (pp < 0) pp += n;
                    const int q = pp == 0 ? 0 : n - pp;
                    d[x] = R[q * PITCH + v];
                }
            }
        }
        // the slot and the scratch buffer are read; the generic accesses are ordered
        // before the slot's next TMA load
        fence_async_smem();
        __syncthreads();
        if (threadIdx.x == 0 && tn < P.ntiles) issue(tn, s);
    }
    if (threadIdx.x == 0 && store_pending) bulk_wait_read0();
}

// Transform along x.  Forward: rows of T (N0 long, [plane][kz][ky][x]) -> the
// interleaved grid [grp][point][ch]; the 16 vectors of a CTA are consecutive
// (grp, kz, ky, ch) with ch fastest, so a half-warp stores 16 channels of one
// point.  Inverse: rows of the planar grid ([plane][kz][ky][kx], n0 long) -> rows
// of T cropped to N0.
struct RowPass {
    FftAxis fa;
    int N0;
    int64_t nvec;
    int nch, nos1, nos2;
    int64_t gvol;
    const float2 *src;
    float2 *dst;
    int *err;  // device flag of the plan (TMA form: a wait that gave up)
    int nsm;   // SMs of the device (TMA form: persistent grid)
};

__global__ void __launch_bounds__(kThreads) row_fwd_kernel(const RowPass P) {
    extern __shared__ float2 fsm[];
    const int n = P.fa.n;
    float2 *A = fsm, *Bf = fsm + n * kPitch;
    const int64_t u0 = (int64_t)blockIdx.x * kCols;
    const int hn = P.N0 / 2;
    {
        const int v = threadIdx.x >> 4, lx = threadIdx.x & 15;
        const int64_t u = u0 + v;
        const bool ok = u < P.nvec;
        int64_t src_off = 0;
        if (ok) {
            const int chn = (int)(u % P.nch);
            int64_t r = u / P.nch;
            const int ky = (int)(r % P.nos1);
            r /= P.nos1;
            const int kz = (int)(r % P.nos2);
            const int64_t grp = r / P.nos2;
            src_off = (((grp * P.nch + chn) * P.nos2 + kz) * P.nos1 + ky) * P.N0;
        }
        for (int p = lx; p < n; p += 16) {
            int x = p + hn;
            if (x >= n) x -= n;
            const bool valid = ok && x < P.N0;
            cp_async8(A + p * kPitch + v, P.src + src_off + (valid ? x : 0), valid);
        }
        cp_async_commit();
        cp_async_wait_all();
    }
    __syncthreads();
    const float2 *R = fft_run(A, Bf, P.fa);
    if (P.nch % 2 == 0) {
        // even channel count: vectors u, u + 1 (u even) are channels ch, ch + 1 of the
        // same point, stored together as one float4
        const int v = (threadIdx.x & 7) * 2;
        const int64_t u = u0 + v;
        if (u < P.nvec) {
            const int chn = (int)(u % P.nch);
            int64_t r = u / P.nch;
            const int ky = (int)(r % P.nos1);
            r /= P.nos1;
            const int kz = (int)(r % P.nos2);
            const int64_t grp = r / P.nos2;
            const int64_t base = (grp * P.gvol + ((int64_t)kz * P.nos1 + ky) * n) * P.nch + chn;
            for (int kx = threadIdx.x >> 3; kx < n; kx += 2 * kStreams)
                *reinterpret_cast<float4 *>(P.dst + base + (int64_t)kx * P.nch) =
                    *reinterpret_cast<const float4 *>(R + kx * kPitch + v);
        }
    } else {
        const int v = threadIdx.x & 15;
        const int64_t u = u0 + v;
        if (u < P.nvec) {
            const int chn = (int)(u % P.nch);
            int64_t r = u / P.nch;
            const int ky = (int)(r % P.nos1);
            r /= P.nos1;
            const int kz = (int)(r % P.nos2);
            const int64_t grp = r / P.nos2;
            const int64_t base = (grp * P.gvol + ((int64_t)kz * P.nos1 + ky) * n) * P.nch + chn;
            for (int kx = threadIdx.x >> 4; kx < n; kx += kStreams) P.dst[base + (int64_t)kx * P.nch] = R[kx * kPitch + v];
        }
    }
}

__global__ void __launch_bounds__(kThreads) row_inv_kernel(const RowPass P) {
    extern __shared__ float2 fsm[];
    const int n = P.fa.n;
    float2 *A = fsm, *Bf = fsm + n * kPitch;
    const int64_t u0 = (int64_t)blockIdx.x * kCols;
    const int hn = P.N0 / 2;
    const int v = threadIdx.x >> 4, lx = threadIdx.x & 15;
    const int64_t u = u0 + v;
    const bool ok = u < P.nvec;
    const int64_t ub = ok ? u : 0;
    for (int p = lx; p < n; p += 16) cp_async8(A + p * kPitch + v, P.src + ub * n + p, ok);
    cp_async_commit();
    cp_async_wait_all();
    for (int p = lx; p < n; p += 16) A[p * kPitch + v].y = -A[p * kPitch + v].y;  // conjugate (inverse)
    __syncthreads();
    const float2 *R = fft_run(A, Bf, P.fa);
    if (ok) {
        for (int x = lx; x < P.N0; x += 16) {
            int pp = x - hn;
            if (pp < 0) pp += n;
            float2 val = R[pp * kPitch + v];
            val.y = -val.y;
            P.dst[u * P.N0 + x] = val;
        }
    }
}

constexpr double kPi = 3.14159265358979323846;

// Appends the axis's twiddles to tw: its stages' offsets are relative to *base,
// the axis's first twiddle in tw (the kernels get the table from there).
bool make_axis(int n, FftAxis *fa, std::vector<float2> &tw, size_t *base) {
    if (n < 1 || n > kMaxN) return false;
    *fa = FftAxis{};
    fa->n = n;
    const StagePlan sp = stage_plan(n);
    int prod = 1;
    for (int s = 0; s < sp.nst; ++s) prod *= sp.radix[s];
    if (prod != n) return false;
    *base = tw.size();
    fa->nst = sp.nst;
    for (int s = 0; s < sp.nst; ++s) {
        const int r = sp.radix[s], ns = sp.ns[s];
        fa->radix[s] = r;
        fa->ns[s] = ns;
        fa->twoff[s] = (int)(tw.size() - *base);
        if (fa->twoff[s] != sp.twoff[s]) return false;
        fa->magic[s] = ns > 1 ? (unsigned)(0xFFFFFFFFull / (unsigned long long)ns + 1ull) : 0u;
        for (int j = 0; j < ns; ++j)
            for (int q = 1; q < r; ++q) {
                const double ang = -2.0 * kPi * (double)j * (double)q / ((double)ns * (double)r);
                tw.push_back(make_float2((float)std::cos(ang), (float)std::sin(ang)));
            }
    }
    return true;
}

// the accumulator over segments only when there are several
size_t col_smem(int n, int mode, int nseg) {
    return (size_t)(mode == 2 && nseg > 1 ? 3 : 2) * n * kPitch * sizeof(float2);
}
size_t row_smem(int n) { return (size_t)2 * n * kPitch * sizeof(float2); }

// cuTensorMapEncodeTiled through the runtime's driver entry point (the driver
// library itself is not linked)
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
    static const EncodeTiledFn fn = [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<EncodeTiledFn>(f);
    }();
    return fn;
}

// 4D map over complex64 data seen as float32 pairs: (2 X floats, rows, mid,
// planes) with the given element strides, boxes of 16 complex x br rows.  Rows
// past `rows` read as zeros.  Strides of unit extents are unused: any legal value.
bool encode_col_map(CUtensorMap *m, const void *base, int X, int rows, int nmid, int64_t nplanes, int64_t s_row,
                    int64_t s_mid, int64_t s_plane, int br) {
    const EncodeTiledFn fn = encode_tiled();
    if (!fn) return false;
    if (nmid == 1) s_mid = s_row;
    if (nplanes == 1) s_plane = s_row;
    const cuuint64_t dim[4] = {(cuuint64_t)2 * X, (cuuint64_t)rows, (cuuint64_t)nmid, (cuuint64_t)nplanes};
    const cuuint64_t str[3] = {(cuuint64_t)s_row * 8, (cuuint64_t)s_mid * 8, (cuuint64_t)s_plane * 8};
    for (cuuint64_t v : str)
        if (v == 0 || v % 16 != 0 || v >= (1ull << 40)) return false;
    const cuuint32_t box[4] = {2 * kCols, (cuuint32_t)br, 1, 1};
    const cuuint32_t es[4] = {1, 1, 1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<void *>(base), dim, str, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// rows per box for segments of lengths a and b (b may be 0): the largest common
// divisor <= 256 when it is at least 32 rows, else the shortest segment (<= 256)
// with the last box of a segment overlapping the one before it
int box_rows(int a, int b) {
    const int m = std::min(256, b > 0 ? std::min(a, b) : a);
    for (int d = m; d >= 32; --d)
        if (a % d == 0 && (b == 0 || b % d == 0)) return d;
    return m;
}

// The column pass on TMA when its layout allows it (every stride and base
// 16-byte aligned, even X); returns 1 if launched, 0 to take the copy-based
// kernel, or an error.  An adjoint last pass over B0 segments walks the segments
// of each output block as consecutive tiles of one CTA.
int launch_col_tma(const ColPass &P, int64_t ntiles, cudaStream_t s) {
    const int n = P.fa.n;
    if (!P.err || P.nsm <= 0 || P.X % 2 != 0 || n > kMaxN) return 0;
    auto a16 = [](const void *q) { return ((uintptr_t)q & 15u) == 0; };
    if (!a16(P.src) || !a16(P.dst)) return 0;
    if (P.Cl && (P.mode == 0 || !a16(P.Cl))) return 0;
    const int nseg = P.mode == 2 ? P.ch.L : 1;
    if (nseg < 1) return 0;
    const int64_t src_plane = P.mode == 1 ? P.nvol : P.in_plane;
    const int64_t dst_plane = P.mode == 2 ? P.nvol : P.out_plane;
    for (int64_t v : {P.in_ax, P.in_mid, src_plane, P.out_ax, P.out_mid, dst_plane})
        if (v % 2 != 0) return 0;
    ColTma T{};
    T.fa = P.fa;
    T.inv = P.inv;
    T.mode = P.mode;
    T.lin = P.lin;
    T.lout = P.lout;
    T.hn = P.nax / 2;
    T.X = P.X;
    T.nxc = (P.X + kCols - 1) / kCols;
    T.nmid = P.nmid;
    T.nplanes = P.nplanes;
    if (ntiles >= (1LL << 31) - 2LL * P.nsm * 4) return 0;
    T.ntiles = (int)ntiles;
    T.nseg = nseg;
    // load boxes: forward passes rotate (smem row p <- source row (p + hn) mod n),
    // inverse passes read the rows in order
    const int seg0 = P.inv ? n : n - T.hn, seg1 = P.inv ? 0 : T.hn;
    T.br = box_rows(seg0, seg1);
    if (T.br > P.lin) return 0;
    int nb = 0;
    for (int sg = 0; sg < 2; ++sg) {
        const int len = sg == 0 ? seg0 : seg1;
        const int s0 = sg == 0 ? 0 : seg0, r0 = sg == 0 ? (P.inv ? 0 : T.hn) : 0;
        for (int r = 0; r < len; r += T.br) {
            if (nb >= kTmaMaxBoxes) return 0;
            const int o = std::min(r, len - T.br);
            T.box_smem[nb] = s0 + o;
            T.box_src[nb] = r0 + o;
            ++nb;
        }
    }
    T.nbox = nb;
    if (!P.inv && P.mode != 2) {
        if (P.lout != n) return 0;
        T.sbr = box_rows(n, 0);
        T.nsbox = (n + T.sbr - 1) / T.sbr;
    }
    T.out_plane = P.out_plane;
    T.out_mid = P.out_mid;
    T.out_ax = P.out_ax;
    T.dst = P.dst;
    T.ch = P.ch;
    T.C = P.C;
    T.nvol = P.nvol;
    T.apod_ax = P.apod_ax;
    T.apod_mid = P.apod_mid;
    T.apod_x = P.apod_x;
    T.Cl = P.Cl;
    T.img_mid = P.in_mid;  // read for forward first passes (image -> buffer)
    T.img_ax = P.in_ax;
    T.factor = P.factor;
    T.accumulate = P.accumulate;
    T.err = P.err;
    const int64_t src_planes = P.mode == 1 ? (int64_t)P.ch.B * P.C
                                           : (P.mode == 2 ? (int64_t)P.ch.ngrp * P.ch.nch : P.nplanes);
    CUtensorMap smap, dmap;
    if (!encode_col_map(&smap, P.src, P.X, P.lin, P.nmid, src_planes, P.in_ax, P.in_mid, src_plane, T.br)) return 0;
    if (T.nsbox > 0) {
        if (!encode_col_map(&dmap, P.dst, P.X, n, P.nmid, P.nplanes, P.out_ax, P.out_mid, P.out_plane, T.sbr))
            return 0;
    } else {
        dmap = smap;  // not read
    }
    constexpr int kSlots = 2;
    const size_t smem = (size_t)(kSlots + 1) * n * kTmaPitch * sizeof(float2);
    auto kern = P.Cl || nseg > 1 ? col_tma_kernel<kSlots, true> : col_tma_kernel<kSlots, false>;
    PFB_RAISE_SMEM(kern, (int)smem);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem) != cudaSuccess || per_sm < 1)
        return 0;
    const int64_t grid = std::min<int64_t>(ntiles, (int64_t)P.nsm * per_sm);
    kern<<<(unsigned)grid, kThreads, smem, s>>>(smap, dmap, T);
    PFB_CHECK_LAUNCH();
    return 1;
}

int launch_col(const ColPass &P, cudaStream_t s) {
    const int64_t blocks = (int64_t)P.nplanes * P.nmid * ((P.X + kCols - 1) / kCols);
    if (blocks == 0) return PFB_OK;
    {
        const int st = launch_col_tma(P, blocks, s);
        if (st == 1) return PFB_OK;
        if (st != 0) return st;
    }
    if (blocks >= (1LL << 31)) return fail(PFB_ERR_UNSUPPORTED, "too many vectors for the fused FFT");
    const size_t smem = col_smem(P.fa.n, P.mode, P.ch.L);
    // two-column moves when every base and stride keeps the pairs 16-byte aligned
    auto a16 = [](const void *q) { return ((uintptr_t)q & 15u) == 0; };
    const bool img_in = P.mode == 1, img_out = P.mode == 2;
    bool vec = P.X % 2 == 0 && a16(P.src) && a16(P.dst) && (!P.Cl || a16(P.Cl)) && P.in_mid % 2 == 0 &&
               P.in_ax % 2 == 0 && P.out_mid % 2 == 0 && P.out_ax % 2 == 0;
    vec = vec && (img_in || img_out ? P.nvol % 2 == 0 : true);
    vec = vec && (img_in ? true : P.in_plane % 2 == 0) && (img_out ? true : P.out_plane % 2 == 0);
    auto k = vec ? col_pass_kernel<true> : col_pass_kernel<false>;
    PFB_RAISE_SMEM(k, (int)smem);
    k<<<(unsigned)blocks, kThreads, smem, s>>>(P);
    PFB_CHECK_LAUNCH();
    return PFB_OK;
}

// Tiled tensor map over 8-byte elements (complex64 as one element): rank dims
// (innermost first), rank - 1 byte strides, a box per dimension.  Rows past an
// extent read as zeros.
bool encode_map8(CUtensorMap *m, const void *base, int rank, const cuuint64_t *dim, const cuuint64_t *stride,
                 const cuuint32_t *box) {
    const EncodeTiledFn fn = encode_tiled();
    if (!fn || rank < 1 || rank > 5) return false;
    for (int i = 0; i < rank - 1; ++i)
        if (stride[i] == 0 || stride[i] % 16 != 0 || stride[i] >= (1ull << 40)) return false;
    for (int i = 0; i < rank; ++i)
        if (dim[i] == 0 || box[i] == 0 || box[i] > 256) return false;
    if ((box[0] * 8) % 16 != 0) return false;
    const cuuint32_t es[5] = {1, 1, 1, 1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_INT64, (cuuint32_t)rank, const_cast<void *>(base), dim, stride, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The x pass on TMA when the layout allows it (a transform length with a
// compile-time stage plan, even row lengths, 16-byte aligned bases, 32-bit vector
// indices; forward: a multiple of 16 channels); returns 1 if launched, 0 to take
// the copy-based kernel, or an error.
int launch_row_tma(const RowPass &P, bool inv, cudaStream_t s) {
    const int n = P.fa.n;
    if (!P.err || P.nsm <= 0 || !first_stage_length(n) || P.N0 % 2 != 0 || n % 2 != 0) return 0;
    if (P.nvec <= 0 || P.nvec >= (1LL << 31) - (int64_t)kCols * 4 * P.nsm) return 0;
    if (!inv && (P.nch % kCols != 0)) return 0;
    auto a16 = [](const void *q) { return ((uintptr_t)q & 15u) == 0; };
    if (!a16(P.src) || !a16(P.dst)) return 0;
    RowTma T{};
    T.fa = P.fa;
    T.N0 = P.N0;
    T.len = inv ? n : P.N0;
    T.rot = inv ? 0 : P.N0 / 2;
    T.hn = P.N0 / 2;
    T.nvec = (int)P.nvec;
    T.ntiles = (int)((P.nvec + kCols - 1) / kCols);
    T.nch = P.nch;
    T.nos1 = P.nos1;
    T.nos2 = P.nos2;
    // one box per tile, x extent = row pitch >= the row length with pitch = 2 (mod 8):
    // the first stage's column reads (8 column pairs x 4 positions per warp) then touch
    // each bank at most twice; a box is at most 256 wide
    T.pitch = T.len;
    while (T.pitch % 8 != 2) ++T.pitch;
    if (T.pitch > 256) return 0;
    const int pitch_out = inv ? kPitch : kTmaPitch;
    T.slot = std::max(kCols * T.pitch, n * pitch_out);
    T.slot = (T.slot + 15) / 16 * 16;  // 128-byte aligned slots
    T.dst = P.dst;
    T.err = P.err;
    CUtensorMap smap, dmap;
    if (inv) {
        // rows of the planar grid, 16 consecutive ones per tile
        const cuuint64_t dim[2] = {(cuuint64_t)n, (cuuint64_t)P.nvec};
        const cuuint64_t str[1] = {(cuuint64_t)n * 8};
        const cuuint32_t box[2] = {(cuuint32_t)T.pitch, (cuuint32_t)kCols};
        if (!encode_map8(&smap, P.src, 2, dim, str, box)) return 0;
    } else {
        // rows of T: x, row (kz, ky) of a plane, plane (group, channel); 16 planes per tile
        const int64_t planes = P.nvec / ((int64_t)P.nos1 * P.nos2);
        const cuuint64_t dim[3] = {(cuuint64_t)P.N0, (cuuint64_t)P.nos2 * P.nos1, (cuuint64_t)planes};
        const cuuint64_t str[2] = {(cuuint64_t)P.N0 * 8, (cuuint64_t)P.N0 * P.nos2 * P.nos1 * 8};
        const cuuint32_t box[3] = {(cuuint32_t)T.pitch, 1, (cuuint32_t)kCols};
        if (!encode_map8(&smap, P.src, 3, dim, str, box)) return 0;
    }
    if (!inv) {
        T.sbr = n <= 256 ? n : 256;
        T.nsbox = (n + T.sbr - 1) / T.sbr;
        const int64_t ngrp = P.nvec / ((int64_t)P.nch * P.nos1 * P.nos2);
        const cuuint64_t dim[4] = {(cuuint64_t)P.nch, (cuuint64_t)n, (cuuint64_t)P.nos2 * P.nos1, (cuuint64_t)ngrp};
        const cuuint64_t str[3] = {(cuuint64_t)P.nch * 8, (cuuint64_t)n * P.nch * 8, (cuuint64_t)P.gvol * P.nch * 8};
        const cuuint32_t box[4] = {(cuuint32_t)kCols, (cuuint32_t)T.sbr, 1, 1};
        if (!encode_map8(&dmap, P.dst, 4, dim, str, box)) return 0;
    } else {
        dmap = smap;  // not read
    }
    const size_t smem = (size_t)3 * T.slot * sizeof(float2);
    auto k = inv ? row_tma_kernel<true> : row_tma_kernel<false>;
    PFB_RAISE_SMEM(k, (int)smem);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kThreads, smem) != cudaSuccess || per_sm < 1)
        return 0;
    const int grid = (int)std::min<int64_t>(T.ntiles, (int64_t)P.nsm * per_sm);
    k<<<grid, kThreads, smem, s>>>(smap, dmap, T);
    PFB_CHECK_LAUNCH();
    return 1;
}

int launch_row(const RowPass &P, bool inv, cudaStream_t s) {
    const int64_t blocks = (P.nvec + kCols - 1) / kCols;
    if (blocks == 0) return PFB_OK;
    {
        const int st = launch_row_tma(P, inv, s);
        if (st == 1) return PFB_OK;
        if (st != 0) return st;
    }
    if (blocks >= (1LL << 31)) return fail(PFB_ERR_UNSUPPORTED, "too many vectors for the fused FFT");
    const size_t smem = row_smem(P.fa.n);
    auto k = inv ? row_inv_kernel : row_fwd_kernel;
    PFB_RAISE_SMEM(k, (int)smem);
    k<<<(unsigned)blocks, kThreads, smem, s>>>(P);
    PFB_CHECK_LAUNCH();
    return PFB_OK;
}

}  // namespace

int fft_fused_ready(pfb_plan *p) {
    std::lock_guard<std::mutex> lk(p->fft_mu);
    if (p->fft_fused >= 0) return p->fft_fused;
    p->fft_fused = 0;
    const int D = p->g.ndim;
    if (D < 2) return 0;
    std::vector<float2> tw;
    size_t tw_base[3] = {0, 0, 0};
    for (int a = 0; a < D; ++a)
        if (!make_axis(p->g.nos[a], &p->fft_ax[a], tw, &tw_base[a])) return 0;
    if (tw.empty()) tw.push_back(make_float2(1.f, 0.f));
    if (pool_alloc(reinterpret_cast<void **>(&p->d_fft_tw), tw.size() * sizeof(float2)) != PFB_OK) return 0;
    if (cudaMemcpy(p->d_fft_tw, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice) != cudaSuccess) {
        pool_free(p->d_fft_tw, 0);
        p->d_fft_tw = nullptr;
        return 0;
    }
    for (int a = 0; a < D; ++a) p->fft_ax[a].tw = p->d_fft_tw + tw_base[a];
    // the TMA column pass's flag and persistent grid (optional: without them the
    // copy-based column pass runs)
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&p->fft_nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        p->fft_nsm = 0;
    if (pool_alloc(reinterpret_cast<void **>(&p->d_fft_err), sizeof(int)) != PFB_OK) {
        p->d_fft_err = nullptr;
    } else if (cudaMemset(p->d_fft_err, 0, sizeof(int)) != cudaSuccess) {
        pool_free(p->d_fft_err, 0);
        p->d_fft_err = nullptr;
    }
    p->fft_fused = 1;
    return 1;
}

void fft_fused_free(pfb_plan *p) {
    std::lock_guard<std::mutex> lk(p->fft_mu);
    // called with the device synchronised (plan destruction)
    pool_free(p->d_fft_tw, 0);
    p->d_fft_tw = nullptr;
    pool_free(p->d_fft_err, 0);
    p->d_fft_err = nullptr;
    p->fft_fused = -1;
}

int fft_fused_fwd(pfb_plan *p, int pass, const Chan &c, int C, const float2 *img, const float *const *apod,
                  const float2 *Cl, float factor, float2 *gridp, float2 *gridi, cudaStream_t s) {
    const Geom &g = p->g;
    const int D = g.ndim;
    const int P = c.ngrp * c.nch;
    const int64_t N0 = g.n[0], N1 = g.n[1], n1 = g.nos[1], n2 = g.nos[2];
    if (pass == 0) {  // image -> first intermediate: z pass (3D) into gridi, or y pass (2D) into gridp
        ColPass Q{};
        Q.err = p->d_fft_err;
        Q.nsm = p->fft_nsm;
        Q.inv = 0;
        Q.mode = 1;
        Q.X = (int)N0;
        Q.nplanes = P;
        Q.src = img;
        Q.ch = c;
        Q.C = C;
        Q.nvol = g.nvol;
        Q.Cl = Cl;
        Q.factor = factor;
        Q.apod_x = apod[0];
        if (D == 3) {
            Q.fa = p->fft_ax[2];
            Q.lin = Q.nax = g.n[2];
            Q.lout = (int)n2;
            Q.nmid = (int)N1;
            Q.in_mid = N0;
            Q.in_ax = N1 * N0;
            Q.out_plane = n2 * N1 * N0;
            Q.out_mid = N0;
            Q.out_ax = N1 * N0;
            Q.apod_ax = apod[2];
            Q.apod_mid = apod[1];
            Q.dst = gridi;
        } else {
            Q.fa = p->fft_ax[1];
            Q.lin = Q.nax = (int)N1;
            Q.lout = (int)n1;
            Q.nmid = 1;
            Q.in_mid = 0;
            Q.in_ax = N0;
            Q.out_plane = n1 * N0;
            Q.out_mid = 0;
            Q.out_ax = N0;
            Q.apod_ax = apod[1];
            Q.apod_mid = nullptr;
            Q.dst = gridp;
        }
        return launch_col(Q, s);
    }
    if (pass == 1) {  // 3D: y pass, gridi -> gridp
        if (D != 3) return PFB_OK;
        ColPass Q{};
        Q.err = p->d_fft_err;
        Q.nsm = p->fft_nsm;
        Q.fa = p->fft_ax[1];
        Q.inv = 0;
        Q.mode = 0;
        Q.lin = Q.nax = (int)N1;
        Q.lout = (int)n1;
        Q.X = (int)N0;
        Q.nmid = (int)n2;
        Q.nplanes = P;
        Q.in_plane = n2 * N1 * N0;
        Q.in_mid = N1 * N0;
        Q.in_ax = N0;
        Q.out_plane = n2 * n1 * N0;
        Q.out_mid = n1 * N0;
        Q.out_ax = N0;
        Q.src = gridi;
        Q.dst = gridp;
        return launch_col(Q, s);
    }
    // x pass: gridp rows -> interleaved grid
    RowPass R{};
    R.err = p->d_fft_err;
    R.nsm = p->fft_nsm;
    R.fa = p->fft_ax[0];
    R.N0 = (int)N0;
    R.nch = c.nch;
    R.nos1 = (int)n1;
    R.nos2 = D == 3 ? (int)n2 : 1;
    R.nvec = (int64_t)c.ngrp * R.nos2 * R.nos1 * c.nch;
    R.gvol = g.gvol;
    R.src = gridp;
    R.dst = gridi;
    return launch_row(R, false, s);
}

int fft_fused_adj(pfb_plan *p, int pass, const Chan &c, int C, float2 *img, const float *const *apod,
                  const float2 *Cl, float factor, bool accumulate, float2 *gridp, float2 *gridi, cudaStream_t s) {
    const Geom &g = p->g;
    const int D = g.ndim;
    const int P = c.ngrp * c.nch;
    const int64_t N0 = g.n[0], N1 = g.n[1], n1 = g.nos[1], n2 = g.nos[2];
    if (pass == 0) {
        // x pass: planar grid rows -> gridi, cropped to N0
        RowPass R{};
        R.err = p->d_fft_err;
        R.nsm = p->fft_nsm;
        R.fa = p->fft_ax[0];
        R.N0 = (int)N0;
        R.nos1 = (int)n1;
        R.nos2 = D == 3 ? (int)n2 : 1;
        R.nvec = (int64_t)P * R.nos2 * R.nos1;
        R.src = gridp;
        R.dst = gridi;
        int st = launch_row(R, true, s);
        if (st || D != 3) return st;
        // 3D: y pass, gridi -> gridp, cropped to N1
        ColPass Q{};
        Q.err = p->d_fft_err;
        Q.nsm = p->fft_nsm;
        Q.fa = p->fft_ax[1];
        Q.inv = 1;
        Q.mode = 0;
        Q.lin = (int)n1;
        Q.lout = Q.nax = (int)N1;
        Q.X = (int)N0;
        Q.nmid = (int)n2;
        Q.nplanes = P;
        Q.in_plane = n2 * n1 * N0;
        Q.in_mid = n1 * N0;
        Q.in_ax = N0;
        Q.out_plane = n2 * N1 * N0;
        Q.out_mid = N1 * N0;
        Q.out_ax = N0;
        Q.src = gridi;
        Q.dst = gridp;
        return launch_col(Q, s);
    }
    // last pass -> image: z pass (3D, from gridp) or y pass (2D, from gridi)
    ColPass Q{};
    Q.err = p->d_fft_err;
    Q.nsm = p->fft_nsm;
    Q.inv = 1;
    Q.mode = 2;
    Q.X = (int)N0;
    Q.nplanes = c.B * C;
    Q.ch = c;
    Q.C = C;
    Q.nvol = g.nvol;
    Q.Cl = Cl;
    Q.factor = factor;
    Q.accumulate = accumulate ? 1 : 0;
    Q.apod_x = apod[0];
    Q.dst = img;
    if (D == 3) {
        Q.fa = p->fft_ax[2];
        Q.lin = (int)n2;
        Q.lout = Q.nax = g.n[2];
        Q.nmid = (int)N1;
        Q.in_plane = n2 * N1 * N0;
        Q.in_mid = N0;
        Q.in_ax = N1 * N0;
        Q.out_mid = N0;
        Q.out_ax = N1 * N0;
        Q.apod_ax = apod[2];
        Q.apod_mid = apod[1];
        Q.src = gridp;
    } else {
        Q.fa = p->fft_ax[1];
        Q.lin = (int)n1;
        Q.lout = Q.nax = (int)N1;
        Q.nmid = 1;
        Q.in_plane = n1 * N0;
        Q.in_mid = 0;
        Q.in_ax = N0;
        Q.out_mid = 0;
        Q.out_ax = N0;
        Q.apod_ax = apod[1];
        Q.apod_mid = nullptr;
        Q.src = gridi;
    }
    return launch_col(Q, s);
}

}  // namespace pfb
