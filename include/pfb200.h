/*
 * pfb200.h -- C ABI of libpfb200.so, the B200 (sm_100a) NUFFT hot path of
 * pyfourier.  Plain C types only: device pointers, sizes and a CUDA stream
 * passed as void*.  Every entry point returns a status code (PFB_OK == 0);
 * pfb_last_error() gives the message of the last failure on the calling thread.
 *
 * Conventions
 *   - complex data is complex64 (interleaved float re, im);
 *   - per-axis parameters (shape, os_shape, width, beta, is_cart) are in the
 *     reference's (z, y, x) order; coordinates are per sample in (x, y, z)
 *     order, in cycles/FOV, i.e. in [-N/2, N/2) (reference
 *     src/pyfourier/_nufft/_plan.py:89-93, :134-136);
 *   - samples of all frames are concatenated; frame f owns global samples
 *     [frame_offsets[f], frame_offsets[f+1]) (frames may differ in length);
 *   - non-Cartesian data is (batch, total samples); images are
 *     (batch, ncoeff, *shape); oversampled grids are
 *     (nseg, batch, ncoeff, *os_shape) -- see pfb_apply_t;
 *   - all calls are asynchronous on the given stream, allocate nothing during
 *     an apply (the caller passes the workspace) and may be captured in a CUDA
 *     graph, except where noted (plan creation synchronises the stream).
 *
 * Each entry point names the reference interface it replaces (paths inside
 * the pyfourier project).
 */
#ifndef PFB200_H
#define PFB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PFB_OK 0
#define PFB_ERR_INVALID 1     /* bad argument, shape or size */
#define PFB_ERR_CUDA 2        /* CUDA runtime error */
#define PFB_ERR_CUFFT 3       /* cuFFT error */
#define PFB_ERR_NOMEM 4       /* device allocation failed */
#define PFB_ERR_UNSUPPORTED 5 /* valid request this build does not implement */
#define PFB_ERR_WORKSPACE 6   /* workspace too small */
#define PFB_ERR_DEVICE 7      /* a kernel's bounded wait gave up; see pfb_plan_check */

#define PFB_NORM_NONE 0  /* forward unscaled, adjoint scaled by 1/prod(os_shape) */
#define PFB_NORM_ORTHO 1 /* both scaled by 1/sqrt(prod(os_shape)) */

typedef struct pfb_plan pfb_plan;
typedef struct pfb_gram pfb_gram;
typedef struct pfb_grog pfb_grog;

/* Options of an operator apply.
 *   batch    B: product of the leading batch axes (coils, slices, ...);
 *   ncoeff   C: number of image planes per batch item: K with a subspace basis,
 *            otherwise the number of frames of the plan;
 *   basis    (F, K) complex64 device array or NULL (reference `basis`,
 *            src/pyfourier/_nufft/_fwd.py:66-68);
 *   weight   per-sample float32 device array (total samples) or NULL
 *            (reference `weight`, broadcast over the batch axes);
 *   nseg     L, number of B0 time segments (1 without field map);
 *   b0_time  (L, readout_len) complex64 temporal interpolator or NULL;
 *   b0_space (L, prod(shape)) complex64 spatial coefficients or NULL;
 *   norm     PFB_NORM_NONE or PFB_NORM_ORTHO;
 *   flags    PFB_FLAG_* bits. */
typedef struct {
    int64_t batch;
    int32_t ncoeff;
    int32_t nseg;
    const void *basis;
    const float *weight;
    const void *b0_time;
    const void *b0_space;
    int32_t norm;
    int32_t flags;
} pfb_apply_t;

/* pfb_apply_t.flags */
#define PFB_FLAG_ACCUMULATE 1 /* add into the output instead of overwriting it */

/* Plan information returned by pfb_plan_info. */
typedef struct {
    int32_t ndim;
    int32_t nframes;
    int64_t total_samples;
    int32_t shape[3];    /* (z, y, x), unused axes 1 */
    int32_t os_shape[3];
    int32_t width[3];
    int32_t tile[3];
    double scale;        /* sum of node-centred kernel samples */
    int32_t n_items;     /* spread work items (per-frame binning) */
    int32_t max_bin;     /* largest number of samples starting in one tile */
    int32_t tile_offset[3]; /* tile t of an axis covers [t*tile - off, (t+1)*tile - off) */
} pfb_plan_info_t;

const char *pfb_last_error(void);
const char *pfb_version(void);

/* Build a plan on `device`.  Replaces plan_nufft's interpolator build
 * (src/pyfourier/_nufft/_plan.py:117-155 and the Interpolator,
 * src/pyfourier/_subroutines/_grid/_plan.py:14-114): scales the coordinates
 * onto the oversampled grid with the reference's float32 arithmetic
 * (src/pyfourier/_subroutines/_traj.py:57-65), then bins the samples by the
 * tile of their first kernel tap with a stable radix sort.  The kernel weights
 * are recomputed in every apply instead of being stored.
 *   coord          device float32 (total, ndim), (x, y, z) per sample;
 *   frame_offsets  host int64 (nframes + 1);
 *   readout_len    samples per readout, the period of the B0 time index;
 *   shape, os_shape, width, is_cart: host int32 (ndim), (z, y, x);
 *   beta           host float32 (ndim), (z, y, x);
 *   tile           host int32 (ndim) tile extent or NULL for the default;
 * Synchronises `stream` (plan-time only). */
int pfb_plan_create(const float *coord, int ndim, int nframes, const int64_t *frame_offsets,
                    int readout_len, const int *shape, const int *os_shape, const int *width,
                    const float *beta, const int *is_cart, const int *tile, int device,
                    void *stream, pfb_plan **out);
int pfb_plan_destroy(pfb_plan *plan);
int pfb_plan_info(const pfb_plan *plan, pfb_plan_info_t *info);

/* Tuning knobs (threads per CTA for spread / interp, channels per spread CTA,
 * 0 keeps the current value). */
int pfb_plan_set_tuning(pfb_plan *plan, int spread_threads, int interp_threads,
                        int spread_channels);

/* Maximum number of samples per spread work item (the split of crowded tiles),
 * in [1, 16384]. */
int pfb_plan_set_chunk(pfb_plan *plan, int chunk);

/* Materialise the reference's interpolator tables for one axis (0 = z ... in
 * (z, y, x) order like Interpolator.index / .value,
 * src/pyfourier/_subroutines/_grid/_plan.py:75-86): index int32 and value
 * float32, both (total samples, width[axis]), in the original sample order.
 * Debug / parity aid; not used by the operators. */
int pfb_plan_tables(const pfb_plan *plan, int axis, int32_t *index, float *value, void *stream);

/* The plan's sample order after the stable counting sort by bin key: order[j] =
 * the sample (caller's index) at sorted position j, int32 (total samples) on the
 * device.  Equal keys keep the caller's order.  Debug / parity aid; the
 * reference has no sorted order (its kernels walk the samples as given,
 * src/pyfourier/_subroutines/_grid/_noncart2cart/_3D.py:29-50). */
int pfb_plan_order(const pfb_plan *plan, int32_t *order, void *stream);

/* Device-side status of the plan's applies: PFB_ERR_DEVICE if a kernel gave up
 * a bounded wait since the last check (its results are invalid; the flag is
 * cleared), else PFB_OK.  Synchronises `stream`.  The reference has no
 * counterpart (its kernels never wait on asynchronous copies). */
int pfb_plan_check(pfb_plan *plan, void *stream);

/* Plans take their device memory from a library-owned pool per device that keeps
 * the blocks destroyed plans give back (repeated plan builds, e.g. one per
 * Pipe-Menon call, then allocate nothing from the driver).  Hand the kept blocks
 * of `device` back to the driver; synchronises the device.  The reference has no
 * counterpart (its plans are NumPy / CuPy arrays). */
int pfb_release_cached_memory(int device);

/* Workspace bytes for an apply over `nplanes` oversampled grid planes
 * (nplanes = nseg * batch * ncoeff).  May create the cuFFT plan. */
int pfb_workspace_size(pfb_plan *plan, int64_t nplanes, size_t *bytes);

/* Workspace bytes for pfb_nufft_fwd / pfb_nufft_adj / pfb_nufft_traj_grad with
 * these options on their fastest path (the channel-interleaved grid plus a
 * bin-sorted sample buffer).  A workspace of pfb_workspace_size bytes is also
 * accepted by those calls; they then take the slower planar path.  May create
 * the cuFFT plan. */
int pfb_apply_workspace_size(pfb_plan *plan, const pfb_apply_t *opt, size_t *bytes);

/* Forward NUFFT: image (batch, ncoeff, *shape) -> kspace (batch, total samples).
 * Replaces _nufft_fwd / _do_nufft (src/pyfourier/_nufft/_nufft.py:11-90, :218-251):
 * apodize -> zero-pad -> centred FFT -> interpolate / scale, B0 segment sum,
 * weight. */
int pfb_nufft_fwd(pfb_plan *plan, const pfb_apply_t *opt, const void *image, void *kspace,
                  void *workspace, size_t workspace_bytes, void *stream);

/* Adjoint NUFFT: kspace (batch, total samples) -> image (batch, ncoeff, *shape).
 * Replaces _nufft_adj / _do_nufft_adj (src/pyfourier/_nufft/_nufft.py:93-169, :254-287). */
int pfb_nufft_adj(pfb_plan *plan, const pfb_apply_t *opt, const void *kspace, void *image,
                  void *workspace, size_t workspace_bytes, void *stream);

/* Adjoint NUFFT that allocates nothing and takes no workspace.  It has no
 * counterpart in the reference.  It exists for callers that cannot call
 * cudaMalloc at apply time: code running inside a host framework that owns all
 * device memory through its own pool, real-time loops with a fixed memory
 * budget, processes that must not grow after set-up.  Same result as
 * pfb_nufft_adj and the same argument checks; its scratch (grid + cuFFT work
 * area) is one static device array of PFB_NOALLOC_SCRATCH_BYTES.  Larger
 * requests are rejected (PFB_ERR_INVALID).  Set-up, once per device: a call
 * with opt->batch == 0 (kspace and image may then be NULL) looks up the array's
 * address; CUDA loads the array lazily, so that call is when the 64 MiB are
 * reserved on the device, until the process exits.  Make it before any stream
 * capture (otherwise the first real call does it).  pfb_workspace_size(plan,
 * nplanes) must also have been called once to create the cuFFT plan.  All calls
 * share the array: calls that overlap on the GPU race and must be serialised
 * by the caller. */
#define PFB_NOALLOC_SCRATCH_BYTES (64u << 20)
int pfb_nufft_adj_noalloc(pfb_plan *plan, const pfb_apply_t *opt, const void *kspace, void *image,
                          void *stream);

/* ---- stages (each replaces one reference subroutine) ---------------------------- */

/* Spread onto the oversampled grid: grid (nseg, batch, ncoeff, *os_shape)
 * = sum of kernel-weighted samples (not divided by scale).  `fft_layout` 1 stores
 * the grid ifftshift-ed (ready for an uncentred FFT), 0 stores it centred like
 * the reference.  Replaces _noncart2cart + _grid_nb
 * (src/pyfourier/_subroutines/_grid/_noncart2cart/__init__.py:25-119). The grid
 * is overwritten. */
int pfb_spread(pfb_plan *plan, const pfb_apply_t *opt, const void *kspace, void *grid,
               int fft_layout, void *stream);

/* Interpolate from the oversampled grid: kspace (batch, total) = sum of
 * kernel-weighted grid values (not divided by scale; weight, B0 and basis
 * applied).  Replaces _cart2noncart + _degrid_nb
 * (src/pyfourier/_subroutines/_grid/_cart2noncart/__init__.py:25-110). */
int pfb_interp(pfb_plan *plan, const pfb_apply_t *opt, const void *grid, void *kspace,
               int fft_layout, void *stream);

/* Deapodise + zero-pad (+ B0 spatial coefficients) into the FFT-ready grid,
 * multiplied by `factor`.  Replaces _apodize + _resize + ifftshift
 * (src/pyfourier/_subroutines/_apod.py:16-46, _resize.py:16-42, _fft.py:72-79). */
int pfb_deapod_pad(pfb_plan *plan, const pfb_apply_t *opt, const void *image, void *grid,
                   float factor, void *stream);

/* Crop + deapodise (+ conj B0 coefficients summed over segments) from the
 * FFT-layout grid, multiplied by `factor`.  Replaces fftshift + _resize + _apodize. */
int pfb_crop_deapod(pfb_plan *plan, const pfb_apply_t *opt, const void *grid, void *image,
                    float factor, void *stream);

/* In-place batched FFT of nplanes FFT-layout grids (direction -1 forward,
 * +1 inverse, both unnormalised).  Uses the workspace for cuFFT's work area. */
int pfb_grid_fft(pfb_plan *plan, void *grid, int64_t nplanes, int direction, void *workspace,
                 size_t workspace_bytes, void *stream);

/* Trajectory gradient: grad (total, ndim) float32 in (x, y, z) order, in
 * coordinate units (cycles/FOV), = sum over batch of Re(conj(D) * v) with
 * D = sum_taps dW/dk * grid, v = kspace-shaped values (batch, total).
 * Uses the analytic derivative of the Kaiser-Bessel form.  Replaces the
 * trajectory backward of the reference (src/pyfourier/_nufft/_nufft.py:175-209),
 * which omits the -2*pi*i/N factor; this is the exact derivative of the
 * discretised operator.  grad is overwritten. */
int pfb_traj_grad(pfb_plan *plan, const pfb_apply_t *opt, const void *grid, const void *values,
                  float *grad, int fft_layout, void *stream);

/* Trajectory gradient of a forward NUFFT, from the image side: grad (total, ndim)
 * float32 = d/dk sum_b Re(conj(A(k) x)_b v_b) where A(k) x is the forward NUFFT
 * of `image` (batch, ncoeff, *shape) with the deapodisation / scaling `factor`
 * given here (1/scale, times 1/sqrt(prod(os_shape)) for "ortho"), and v =
 * `values` (batch, total).  Padding, cuFFT and the gradient kernel in one call;
 * the kernel weights are recomputed, nothing is stored.  grad is overwritten
 * (or accumulated with PFB_FLAG_ACCUMULATE). */
int pfb_nufft_traj_grad(pfb_plan *plan, const pfb_apply_t *opt, const void *image, const void *values,
                        float *grad, float factor, void *workspace, size_t workspace_bytes, void *stream);

/* One stage of the fast pipelines, for per-kernel timing and for callers that
 * interleave their own work between stages.  The workspace (of
 * pfb_apply_workspace_size bytes) carries the intermediates between calls:
 * forward = PAD, FFT, TRANSPOSE, INTERP, OUT; adjoint = VALS, SPREAD, IFFT, CROP.
 *   PAD:    src image -> planar grid (deapodised, padded, times `factor`)
 *   FFT / IFFT: the planar grid in place
 *   TRANSPOSE: planar grid -> channel-interleaved grid
 *   INTERP: interleaved grid -> per-channel sample results;  OUT: results -> dst k-space
 *   VALS:   src k-space -> per-channel sample values;  SPREAD: values -> grid
 *   CROP:   grid -> dst image (cropped, deapodised, times `factor`)
 * For 2D and 3D grids whose axes are at most 512 long with factors 2, 3, 5, 7
 * the transform is the fused pruned FFT: PAD, FFT and TRANSPOSE are then its
 * three forward passes (image -> z pass -> y pass -> x pass writing the
 * interleaved grid; 2D: y pass, nothing, x pass) and IFFT / CROP its adjoint
 * passes (x and y passes / last pass writing the image); the chain of stages
 * computes the same result either way.
 * Stages of the forward path replace _do_nufft's steps
 * (src/pyfourier/_nufft/_nufft.py:235-246), those of the adjoint _do_nufft_adj's
 * (:271-282). */
#define PFB_STAGE_PAD 0
#define PFB_STAGE_FFT 1
#define PFB_STAGE_INTERP 2
#define PFB_STAGE_OUT 3
#define PFB_STAGE_VALS 4
#define PFB_STAGE_SPREAD 5
#define PFB_STAGE_IFFT 6
#define PFB_STAGE_CROP 7
#define PFB_STAGE_TRANSPOSE 8
int pfb_nufft_stage(pfb_plan *plan, const pfb_apply_t *opt, int stage, const void *src, void *dst,
                    float factor, void *workspace, size_t workspace_bytes, void *stream);

/* ---- density compensation (src/pyfourier/_dcomp) ------------------------------ */

/* Pipe-Menon density compensation, replacing pipe_menon_dcf
 * (src/pyfourier/_dcomp/pipemenon.py:9-96, _GHG :99-115): niter times
 *     w <- w / |A A^H w|
 * with A the plan's NUFFT (norm "ortho"), one channel over all the plan's
 * frames.  weights: device float32 (total samples) in the original sample
 * order, updated in place; the caller sets the start (ones in the reference).
 * The iterations run back to back on `stream` without host synchronisation.
 * Workspace: pfb_dcf_workspace_size bytes. */
int pfb_dcf_workspace_size(pfb_plan *plan, size_t *bytes);
int pfb_pipe_menon_dcf(pfb_plan *plan, float *weights, int niter, void *workspace, size_t workspace_bytes,
                       void *stream);

/* ---- Toeplitz and Cartesian Gram (src/pyfourier/_sparsegram, src/pyfourier/_gram) -- */

/* Create a Gram operator from its Toeplitz kernel on the 2x grid, or from the
 * Cartesian sampling mask on the image grid (os_shape == shape: the dense Gram).
 *   ndim, shape (z, y, x): image extent N; os_shape (z, y, x): embedding grid;
 *   ncoeff  K (low rank) or number of kernel planes (elementwise);
 *   lowrank 1: kernel is (prod(os_shape), K, K) with out[v] = T[v] @ in[v];
 *           0: kernel is (ncoeff, prod(os_shape)) applied elementwise;
 *   nseg    B0 time segments L (1 without field map): the kernel then holds
 *           L such kernels, one per segment;
 *   kernel  device complex64, uncentred (ifftshift-ed) layout, copied.
 * Replaces GramMatrix (src/pyfourier/_sparsegram/_plan.py:253-270,
 * src/pyfourier/_gram/_plan.py:160-177). */
/* Plan-time float64 spread for the Toeplitz PSF: grid[ch, frame(m), idx] +=
 * KB64 taps of sample m * values[ch, m], for every sample m of the plan (in the
 * plan's sample order) and ch < nch.  values (nch, total samples) and grid
 * (nch, nframes, *os_shape) are device complex128; the grid is in the
 * reference's table layout (index (x0 + i) mod n_os, no FFT shift), not divided
 * by the kernel scale, and accumulated (the caller zeroes it).  Kernel weights,
 * products and sums are float64.  Replaces the complex64 spread inside the PSF
 * construction (src/pyfourier/_sparsegram/_plan.py:201-208, the adjoint NUFFT
 * of the sample weights). */
int pfb_spread_f64(pfb_plan *plan, const void *values, int nch, void *grid, void *stream);

int pfb_gram_create(int ndim, const int *shape, const int *os_shape, int ncoeff, int lowrank,
                    int nseg, const void *kernel, int device, void *stream, pfb_gram **out);
int pfb_gram_destroy(pfb_gram *gram);
int pfb_gram_workspace_size(pfb_gram *gram, int64_t batch, size_t *bytes);

/* Apply: image (batch, ncoeff, *shape) -> out (same).  Zero-pad into the 2x grid,
 * FFT, per-voxel K x K mix (or elementwise product), inverse FFT, crop.  With
 * B0 segments, out = sum_l conj(C_l) G_l(C_l x) with b0_space = C (L, prod(shape)),
 * complex64 (NULL without segments).  When os_shape == shape and nseg == 1 there is
 * no embedding: FFT image -> out, mix in out, inverse FFT in out; the workspace
 * then only holds the cuFFT work area.
 * Replaces _sparsegram / _do_sparsegram / _bdot
 * (src/pyfourier/_sparsegram/_sparsegram.py:11-81, _bmatvec/_bdot.py:16-115) and
 * _gram / _do_gram (src/pyfourier/_gram/_gram.py:11-133). */
int pfb_gram_apply(pfb_gram *gram, const void *image, void *out, int64_t batch, const void *b0_space,
                   void *workspace, size_t workspace_bytes, void *stream);

/* ---- GROG pre-interpolation (src/pyfourier/_preinterp/_grog.py) ------------------ */

/* Create a GROG operator set for one trajectory.
 *   lut      device int32 (nsamples): operator index of each sample in [0, ntable),
 *            -1 for samples outside the grid (their output is zero);
 *   ntable   operators per set (nsteps^ndim);
 *   ncoils   nc, 1 .. 64;
 *   nslices  operator sets: 2D GROG trains one set per calibration slice and applies
 *            set b to batch item b; 1 otherwise;
 *   table    device complex64 (ntable, nslices, nc, nc), [i][j] maps source coil i to
 *            target coil j; copied.
 * Sorts the samples by operator (once).  Replaces the operator lookup of
 * src/pyfourier/_preinterp/_grog.py:172-185 and the kernel launch of :399-439. */
int pfb_grog_create(const int *lut, int64_t nsamples, int ntable, int ncoils, int nslices, const void *table,
                    int device, void *stream, pfb_grog **out);
int pfb_grog_destroy(pfb_grog *grog);
/* Workspace of an apply: batch x (samples inside the grid) x nc complex64. */
int pfb_grog_workspace_size(pfb_grog *grog, int64_t batch, size_t *bytes);

/* Apply: in (batch, nc, nsamples) complex64 -> out (same), out[b, :, m] =
 * in[b, :, m] @ table[lut[m], slice b]; zeros where lut[m] == -1.  in and out must not
 * overlap.  Replaces _interp / do_interpolation (src/pyfourier/_preinterp/_grog.py:399-439;
 * the shipped per-sample product computes in * colsum(G), the evident intent is
 * in @ G). */
int pfb_grog_apply(pfb_grog *grog, const void *in, void *out, int64_t batch, void *workspace,
                   size_t workspace_bytes, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* PFB200_H */
