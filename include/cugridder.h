/*
 * cugridder.h -- C ABI of libcugridder.so, the B200 (sm_100a) gridder.
 *
 * Drop-in for the ms2dirty / dirty2ms path of RapidsAtHKUST/cuGridder.
 * The first eight functions have exactly the reference's names, argument
 * order, argument meaning and return convention (include/cugridder.h:37-47
 * of the reference; definitions src/astro/cugridder.cu:541-571):
 *
 *   - uvw is a HOST array [nrow][3] (u, v, w in metres), row-major;
 *   - vis is a HOST array of nrow complex values (input of ms2dirty,
 *     output of dirty2ms);
 *   - dirty is a HOST array [nxdirty][nydirty] complex, row-major
 *     (output of ms2dirty, input of dirty2ms);
 *   - wgt (the _2 variants) is a HOST array of nrow real weights; both
 *     directions MULTIPLY by it (the reference's dirty2ms "divide" invoker
 *     launches the multiply kernel, src/utils.cu:661-668);
 *   - fov is the field of view in degrees on both axes; freq in Hz;
 *   - the phase is exp(+2 pi i f/c (u l + v m + sign w (n-1))) for ms2dirty
 *     and its conjugate for dirty2ms, l = (x - nx/2) fov/nx,
 *     m = (y - ny/2) fov/ny (src/astro/precomp.cu:48-72);
 *   - return 0 on success, 1 when epsilon was below the precision floor and
 *     was clipped (the reference's ier = 1), >= 2 on error.  The library
 *     never calls exit().
 *
 * Complex arrays are interleaved (re, im) pairs, layout-compatible with
 * std::complex<T>, C99 _Complex and numpy complex64/complex128.
 */
#ifndef CUGRIDDER_B200_H
#define CUGRIDDER_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { double re, im; } cg_c128;
typedef struct { float re, im; } cg_c64;

/* status codes */
#define CG_OK 0
#define CG_WARN_EPS_CLIPPED 1 /* epsilon below the floor, clipped (reference ier = 1) */
#define CG_ERR_ARG 2          /* invalid argument (sizes, null pointers, non-finite uvw) */
#define CG_ERR_CUDA 3         /* CUDA runtime error */
#define CG_ERR_CUFFT 4        /* cuFFT error */
#define CG_ERR_NOMEM 5        /* device memory exhausted */
#define CG_ERR_SIZE 6         /* problem too large for this build (index range) */
#define CG_ERR_NOGPU 7        /* no CUDA device */

/* ---------------- reference-compatible entry points ----------------
 * FP64: ms2dirty_1/_2, dirty2ms_1/_2 (reference cugridder.h:37-47 with
 * PCS=double, CPX=std::complex<double>). */
int ms2dirty_2(int nrow, int nxdirty, int nydirty, double fov, double freq, double *uvw,
               cg_c128 *vis, double *wgt, cg_c128 *dirty, double epsilon, double sigma,
               int sign);
int ms2dirty_1(int nrow, int nxdirty, int nydirty, double fov, double freq, double *uvw,
               cg_c128 *vis, cg_c128 *dirty, double epsilon, double sigma, int sign);
int dirty2ms_1(int nrow, int nxdirty, int nydirty, double fov, double freq, double *uvw,
               cg_c128 *vis, cg_c128 *dirty, double epsilon, double sigma, int sign);
int dirty2ms_2(int nrow, int nxdirty, int nydirty, double fov, double freq, double *uvw,
               cg_c128 *vis, double *wgt, cg_c128 *dirty, double epsilon, double sigma,
               int sign);

/* FP32 twins ms2dirtyf_1/_2, dirty2msf_1/_2 (reference cugridder.h:21-31,
 * -DSINGLE: PCS=float).  uvw arrives in float as in the reference; the
 * library widens it to FP64 for the coordinate scaling and the
 * integer/fraction split, and grids in FP32. */
int ms2dirtyf_2(int nrow, int nxdirty, int nydirty, float fov, float freq, float *uvw,
                cg_c64 *vis, float *wgt, cg_c64 *dirty, float epsilon, float sigma, int sign);
int ms2dirtyf_1(int nrow, int nxdirty, int nydirty, float fov, float freq, float *uvw,
                cg_c64 *vis, cg_c64 *dirty, float epsilon, float sigma, int sign);
int dirty2msf_1(int nrow, int nxdirty, int nydirty, float fov, float freq, float *uvw,
                cg_c64 *vis, cg_c64 *dirty, float epsilon, float sigma, int sign);
int dirty2msf_2(int nrow, int nxdirty, int nydirty, float fov, float freq, float *uvw,
                cg_c64 *vis, float *wgt, cg_c64 *dirty, float epsilon, float sigma, int sign);

/* ---------------- precision-split host entry points ----------------
 * No reference counterpart: same argument order as ms2dirty_2 / dirty2ms_2,
 * but uvw stays FP64 while vis, wgt and dirty are FP32 (complex64 / float).
 * wgt may be NULL. */
int cg_ms2dirty_mixed(int64_t nrow, int nxdirty, int nydirty, double fov, double freq,
                      const double *uvw, const cg_c64 *vis, const float *wgt, cg_c64 *dirty,
                      double epsilon, double sigma, int sign);
int cg_dirty2ms_mixed(int64_t nrow, int nxdirty, int nydirty, double fov, double freq,
                      const double *uvw, cg_c64 *vis, const float *wgt, const cg_c64 *dirty,
                      double epsilon, double sigma, int sign);

/* ---------------- plan API: device pointers, stream ordered ----------------
 * Replaces the reference's gridder_setting / gridder_execution /
 * gridder_destroy (reference cugridder.h:33-36; cugridder.cu:90-257) with a
 * reusable plan whose workspace stays resident in HBM across calls.
 *
 * precision: CG_PREC_FP64  uvw f64, vis/dirty complex128, wgt f64
 *            CG_PREC_FP32  uvw f64, vis/dirty complex64,  wgt f32
 * stream:    a cudaStream_t (NULL = legacy default stream).  Calls are
 *            stream ordered; each call performs one small device-to-host read
 *            (the w range) and therefore synchronizes the stream once.
 * All pointers passed to cg_plan_ms2dirty / cg_plan_dirty2ms are DEVICE
 * pointers. d_wgt may be NULL. */
#define CG_PREC_FP64 0
#define CG_PREC_FP32 1

typedef struct cg_plan_s cg_plan;

typedef struct {
    int kw;            /* kernel width W */
    double beta;       /* ES beta */
    int nf1, nf2;      /* grid sizes: nf1 <- nydirty, nf2 <- nxdirty */
    int nw;            /* number of w planes of the last call */
    double i_center, i_half_width, o_center, o_half_width, gamma, h;
    double pixelsize_x, pixelsize_y;
    int nhive[3];
    int64_t nrow;      /* rows of the last call */
    size_t workspace_bytes;
} cg_plan_info;

int cg_plan_create(cg_plan **plan, int nxdirty, int nydirty, double fov, double epsilon,
                   double sigma, int sign, int precision, void *stream);
int cg_plan_set_stream(cg_plan *plan, void *stream);
int cg_plan_ms2dirty(cg_plan *plan, int64_t nrow, double freq, const double *d_uvw,
                     const void *d_vis, const void *d_wgt, void *d_dirty);
int cg_plan_dirty2ms(cg_plan *plan, int64_t nrow, double freq, const double *d_uvw,
                     const void *d_dirty, const void *d_wgt, void *d_vis);
int cg_plan_get_info(const cg_plan *plan, cg_plan_info *info);

/* Multi-channel calls (no reference counterpart: the reference's C API takes
 * one frequency, cursl.py:78 uses freq[0] only and the channel loop of
 * w_s_gridder_test.cu:206-224 is broken).  freqs: HOST array of nchan
 * frequencies; d_vis / d_wgt are [nrow][nchan] (d_wgt may be NULL).
 * ms2dirty sums every (row, channel) visibility into one image, as NIFTY's
 * ms2dirty does; dirty2ms fills every (row, channel).  The channels are
 * flattened into nrow * nchan rows of one call (uvw scaled by f_c / f_0). */
int cg_plan_ms2dirty_chan(cg_plan *plan, int64_t nrow, int nchan, const double *freqs,
                          const double *d_uvw, const void *d_vis, const void *d_wgt,
                          void *d_dirty);
int cg_plan_dirty2ms_chan(cg_plan *plan, int64_t nrow, int nchan, const double *freqs,
                          const double *d_uvw, const void *d_dirty, const void *d_wgt,
                          void *d_vis);
int cg_plan_destroy(cg_plan *plan);

/* ---------------- inspection (tests / tools) ----------------
 * After a call, copies an internal device buffer of the plan to HOST memory:
 *   CG_BUF_HIVE_START  int32  [nhive0*nhive1*nhive2 + 1]  first sorted row of
 *                      each 8x8x1 hive: the reference's hive_count
 *                      (conv_interp_invoker.cu:121-224)
 *   CG_BUF_PERM        int32  [nrow]  original row index of each sorted row
 *   CG_BUF_SORTED_KEYS int64  [nrow]  hive-major cell key of each sorted row
 *                      (the reference's histogram_3d_sparse key,
 *                      utils.cu:105-132)
 *   CG_BUF_GRID        complex (precision) [nw][nf2][nf1], the grid after the
 *                      stage selected by cg_plan_set_stop_stage
 *   CG_BUF_FSERIES_1 / _2  f64 [nf1/2+1] / [nf2/2+1] kernel Fourier series
 *                      (deconv.cu:12-26, with the (-1)^k fold)
 *   CG_BUF_FSERIES_W   f64 [(nx/2+1)*(ny/2+1)] w kernel correction on the
 *                      quarter image (deconv.cu:49-65)
 * bytes must be at least the size of the buffer; returns CG_ERR_ARG if not. */
#define CG_BUF_HIVE_START 1
#define CG_BUF_PERM 2
#define CG_BUF_SORTED_KEYS 3
#define CG_BUF_GRID 4
#define CG_BUF_FSERIES_1 5
#define CG_BUF_FSERIES_2 6
#define CG_BUF_FSERIES_W 7
int cg_plan_copy_buffer(cg_plan *plan, int which, void *host_dst, size_t bytes,
                        size_t *bytes_needed);

/* Spreading / interpolation method: 1 = tiled shared-memory kernels
 * (default); 2 = tensor-core gridding (split-TF32 mma.sync per hive) for FP32
 * with W <= 8, tiled kernels otherwise; 0 = direct kernels with global
 * atomics / gathers (cross-check). */
int cg_plan_set_method(cg_plan *plan, int method);

/* Gridding kernel of a plan (no reference counterpart; the reference always
 * uses ES with W from epsilon).
 *   CG_KERNEL_ES:   exp(beta sqrt(1 - (2d/W)^2)); W = 0 takes W and beta
 *                   from epsilon (the default), W in 2..16 forces that width
 *                   with the reference's beta for it; coef is ignored.
 *   CG_KERNEL_POLY: a piecewise polynomial of width W (2..16): segment i
 *                   (d in [i - W/2, i + 1 - W/2)) is
 *                   sum_n coef[i*8 + n] * (2 (d + W/2 - i) - 1)^n, n < 8 --
 *                   the Horner form of a learned kernel.  The kernel's
 *                   Fourier series is computed by the same Gauss-Legendre
 *                   quadrature as for ES, and the grid sizes follow from W.
 * Takes effect from the next call. */
#define CG_KERNEL_ES 0
#define CG_KERNEL_POLY 1
int cg_plan_set_kernel(cg_plan *plan, int kind, int W, const double *coef);

/* The same choice for the host-pointer entry points (the eight reference
 * functions and cg_*_mixed), process-wide: their cached plans switch kernel
 * on their next call.  Default: CG_KERNEL_ES with W from epsilon, the
 * reference's behaviour.  No reference counterpart. */
int cg_set_host_kernel(int kind, int W, const double *coef);

/* Memory-limited mode (no reference counterpart; the reference's equivalent
 * is its plane-cube loop, ra_exec.cu:292-389 / 522-613).  When the whole
 * grid (nw planes) would exceed `bytes`, the plan keeps only as many planes
 * as fit and runs gridding + FFT + w-DFT (ms2dirty) or plane fill + FFT +
 * degridding (dirty2ms) window by window; results equal the resident path
 * up to summation order.  0 (default) = no limit. */
int cg_plan_set_grid_budget(cg_plan *plan, size_t bytes);

/* Fixed-uvw mode (no reference counterpart): the caller promises that the
 * uvw array behind d_uvw does not change between calls.  A call whose d_uvw,
 * nrow and freq equal the previous call's (either direction) then reuses its
 * w range, geometry, quarter tables and binning: no host synchronisation and
 * no allocation, so after one warm call the plan's calls can be captured in
 * a CUDA graph on the plan's stream.  Off by default; per-stage timing
 * disables the reuse. */
int cg_plan_set_fixed_uvw(cg_plan *plan, int on);

/* Autotuning (no reference counterpart): when on, the first call per
 * direction for a grid geometry times a fixed list of candidate tilings of
 * its spreading / interpolation launch (tile size, plane batch, warps or
 * threads per CTA) on the call's own data and keeps the fastest for later
 * calls.  Off by default for plans made with cg_plan_create (the
 * environment variable CG_AUTOTUNE=1 turns it on for plans created
 * afterwards); on by default for the cached plans behind the host entry
 * points (ms2dirty_1 ... cg_dirty2ms_mixed), which callers cannot reach with
 * this call, unless CG_AUTOTUNE=0.  The tuning call synchronizes, so capture a plan's calls into a
 * CUDA graph only after it.  cg_plan_get_tiling reports the tiling in the
 * layout of cg_batch_get_tiling. */
int cg_plan_set_autotune(cg_plan *plan, int on);
int cg_plan_get_tiling(const cg_plan *plan, int *tiling, float *tuned_ms);

/* Stops the next calls after a stage (testing): 0 = run to the end,
 * 1 = after binning, 2 = after gridding (ms2dirty) / plane fill (dirty2ms),
 * 3 = after the FFT. */
int cg_plan_set_stop_stage(cg_plan *plan, int stage);

/* Status of the plan's asynchronous work (no reference counterpart: the
 * reference synchronizes after every kernel and exit()s on errors,
 * include/utils.h:18-27).  Waits for the plan's stream, then returns
 * CG_ERR_CUDA (message in cg_last_error) if a bounded staging wait of the
 * TMA degridding ran out since the last check, which leaves that call's
 * visibilities incomplete, and clears the condition; else CG_OK.  A
 * dirty2ms call that is not being captured into a CUDA graph runs this
 * check itself before it returns; a captured call's condition is reported
 * by this function or by the plan's next call. */
int cg_plan_status(cg_plan *plan);

/* Per-stage CUDA-event timers of a plan (profiling; off by default).
 * Stages of ms2dirty: 0 w range, 1 quarter tables, 2 binning, 3 sorted
 * stream, 4 gridding, 5 FFT, 6 w-DFT + corrections.  Stages of dirty2ms:
 * 0 w range, 1 quarter tables, 2 binning, 3 plane fill, 4 FFT, 5 sorted
 * stream, 6 degridding.  cg_plan_set_timing resets the totals;
 * cg_plan_get_timing synchronizes the plan's stream and returns the summed
 * milliseconds per stage of direction 0 (ms2dirty) or 1 (dirty2ms). */
int cg_plan_set_timing(cg_plan *plan, int on);
int cg_plan_get_timing(cg_plan *plan, int direction, double *stage_ms, int cap, int *nstages,
                       long long *ncalls);

/* Allocation-free hive binning (no reference counterpart).  Runs the binning
 * stage of a plan call -- w range, stable sort of the rows by the hive-major
 * cell key, hive offsets -- on DEVICE uvw [nrow][3] and writes the same
 * d_perm [nrow] (original row of each sorted row, as CG_BUF_PERM) and
 * d_hive_start [n_hives + 1] (as CG_BUF_HIVE_START) that a plan with the same
 * nxdirty, nydirty, fov, epsilon, sigma, sign and precision computes.
 * It allocates nothing: its scratch is a fixed 15 MiB device array inside the
 * library, so nrow is limited to cg_bin_static_max_rows() (524,288) and
 * larger nrow returns CG_ERR_SIZE.  When hive_start_len < n_hives + 1 (or
 * d_hive_start is NULL) it stores n_hives, returns CG_ERR_SIZE and writes no
 * output.  Synchronizes `stream` once (w range read-back).  The first call on
 * a device looks up the scratch address (module load); make it before any
 * stream capture.  Overlapping calls on one device race on the shared
 * scratch. */
int cg_bin_static(int64_t nrow, int nxdirty, int nydirty, double fov, double freq,
                  const double *d_uvw, double epsilon, double sigma, int sign, int precision,
                  int *d_perm, int *d_hive_start, int64_t hive_start_len, int64_t *n_hives,
                  void *stream);
int64_t cg_bin_static_max_rows(void);

/* ---------------- learned kernel: training primitives ----------------
 * No reference counterpart.  Device pointers, stream ordered, FP32 unless
 * noted.  The learned kernel family is
 *   phi(d) = exp(beta0 (sqrt(1 - t^2) - 1) + net(2 t^2 - 1)),  t = 2d/W, |t| < 1,
 * net a 1-32-32-1 tanh MLP with cg_learn_theta_size() parameters laid out
 * W1[32], b1[32], W2[32][32] (row = output unit), b2[32], w3[32], b3.
 *   phi_forward:  phi[i] = phi(d[i])
 *   phi_backward: dtheta += sum_i dphi[i] * d phi(d[i]) / d theta
 *                 (accumulates; the caller zeroes dtheta)
 *   spread2d:     grid[s][ix][iy] += c[s][j] phx[s][j][l] phy[s][j][m] at
 *                 ix = gx0 + l, iy = gy0 + m mod nf (complex interleaved;
 *                 accumulates)
 *   spread2d_adjoint: dphx[s][j][l] = sum_m <ggrid, c> phy, dphy likewise,
 *                 <a, b> = a.re b.re + a.im b.im
 *   dft2 (FP64):  F[s][i] = sum_j c[s][j] exp(2 pi i (k1[s][i] X[s][j] +
 *                 k2[s][i] Y[s][j]) / nf), the direct-sum target. */
int cg_learn_theta_size(void);
int cg_learn_phi_forward(const float *theta, float beta0, int W, int64_t n, const float *d,
                         float *phi, void *stream);
int cg_learn_phi_backward(const float *theta, float beta0, int W, int64_t n, const float *d,
                          const float *dphi, float *dtheta, void *stream);
int cg_learn_spread2d(int nsets, int M, int W, int nf, const float *c, const int *gx0,
                      const int *gy0, const float *phx, const float *phy, float *grid,
                      void *stream);
int cg_learn_spread2d_adjoint(int nsets, int M, int W, int nf, const float *c, const int *gx0,
                              const int *gy0, const float *phx, const float *phy,
                              const float *ggrid, float *dphx, float *dphy, void *stream);
int cg_learn_dft2(int nsets, int M, int nf, const double *X, const double *Y, const double *c,
                  int nk, const int *k1, const int *k2, double *F, void *stream);

/* ---------------- on-device FP64 direct DFT ----------------
 * The exact sums that ms2dirty / dirty2ms approximate (the reference's
 * explicit_gridder, precomp.cu:246-321, with the library's conventions:
 * weights multiply, w enters with `sign`, n - 1 = -(l^2+m^2)/(1+n)), for
 * error checks on large problems.  DEVICE pointers, stream ordered, FP64.
 *   cg_explicit_ms2dirty: d_out[q] = sum_j wgt_j vis_j
 *       exp(2 pi i f/c (u_j l + v_j m + sign w_j (n-1))) / n for pixel
 *       d_pix[q] (flat index x*ny + y), q < npix; npix < 0: every pixel,
 *       d_out [nx][ny].
 *   cg_explicit_dirty2ms: d_out[q] = wgt_j sum_{x,y} dirty[x][y] / n
 *       exp(-2 pi i f/c (...)) for row j = d_rows[q], q < nvis; nvis < 0:
 *       every row.
 * d_wgt may be NULL.  Outputs are overwritten; out-of-range indices give 0. */
int cg_explicit_ms2dirty(int64_t nrow, int nxdirty, int nydirty, double fov, double freq,
                         const double *d_uvw, const cg_c128 *d_vis, const double *d_wgt, int sign,
                         int64_t npix, const int64_t *d_pix, cg_c128 *d_out, void *stream);
int cg_explicit_dirty2ms(int64_t nrow, int nxdirty, int nydirty, double fov, double freq,
                         const double *d_uvw, const cg_c128 *d_dirty, const double *d_wgt, int sign,
                         int64_t nvis, const int64_t *d_rows, cg_c128 *d_out, void *stream);

/* ---------------- generic NUFFT, type 1 and 2, 1-3 dimensions ----------------
 * The reference's generic front end (cunufft_setting, cuft.cu:327-504, and
 * the flow of test/nufft_{1d,2d_1,2d_2,3d_1,3d_2}_test.cu) on this library's
 * ES kernel, Gauss-Legendre deconvolution, sorting and cuFFT.
 *   type 1: fk[k3][k2][k1] = sum_j c_j exp(i iflag ((k1 - N1/2) x_j +
 *           (k2 - N2/2) y_j + (k3 - N3/2) z_j)), k1 fastest;
 *   type 2: c_j = sum_k fk[k3][k2][k1] exp(i iflag (...)).
 * nmodes: dim entries N1 (, N2 (, N3)).  Coordinates: DEVICE FP64 arrays in
 * radians (period 2 pi); c / fk: DEVICE complex arrays of the plan precision.
 * setpts sorts the points (keep the coordinate arrays alive until then
 * only); execute may be called many times per setpts. */
typedef struct cg_nufft_s cg_nufft;
int cg_nufft_create(cg_nufft **plan, int type, int dim, const int64_t *nmodes, int iflag,
                    double epsilon, double sigma, int precision, void *stream);
int cg_nufft_setpts(cg_nufft *plan, int64_t M, const double *d_x, const double *d_y,
                    const double *d_z);
int cg_nufft_execute(cg_nufft *plan, void *d_c, void *d_fk);
int cg_nufft_get_info(const cg_nufft *plan, int *kw, int64_t *nf);
int cg_nufft_destroy(cg_nufft *plan);

/* ---------------- batched solves ----------------
 * No reference counterpart (its C API images one dataset per call).  A batch
 * images n independent datasets -- each with its own image size, field of
 * view, rows and channels -- in one call.  All pointers of a dataset are
 * DEVICE pointers that must stay valid (and uvw unchanged) for the life of
 * the batch; vis / wgt are [nrow][nchan] (wgt may be NULL), freqs a HOST array
 * of nchan frequencies (copied at creation).  ms2dirty sums a dataset's
 * channels into its image; dirty2ms fills every (row, channel).  All
 * datasets are spread (interpolated) by ONE persistent launch over a
 * (dataset, tile) work queue; the stages before and after it run per dataset
 * over the batch's streams.  The first call per direction runs eagerly and
 * autotunes that launch's tiling; the second is captured into a CUDA graph
 * and later calls replay it (CG_BATCH_GRAPH=0 disables the graph).  Calls
 * are ordered on `stream`. */
typedef struct {
    int64_t nrow;
    int nchan;
    const double *freqs;
    int nxdirty, nydirty;
    double fov;
    const double *d_uvw;
    void *d_vis;
    const void *d_wgt;
    void *d_dirty;
} cg_dataset;
typedef struct cg_batch_s cg_batch;
int cg_batch_create(cg_batch **batch, int n, const cg_dataset *datasets, double epsilon,
                    double sigma, int sign, int precision, void *stream);
int cg_batch_ms2dirty(cg_batch *batch);
int cg_batch_dirty2ms(cg_batch *batch);
/* Gridding kernel of every dataset (arguments as cg_plan_set_kernel); only
 * before the first call. */
int cg_batch_set_kernel(cg_batch *batch, int kind, int W, const double *coef);
/* Tiling picked by the autotuner on the first call of each direction
 * (CG_BATCH_AUTOTUNE=0 keeps the defaults): tiling[0..3] = gridding warp
 * tile x, y, plane batch, warps per CTA; tiling[4..7] = degridding tile x,
 * y, plane batch, threads per CTA (0 = default).  tuned_ms (may be NULL)
 * receives the winning launch times in ms (0 = not tuned). */
int cg_batch_get_tiling(const cg_batch *batch, int *tiling, float *tuned_ms);
int cg_batch_destroy(cg_batch *batch);

/* Host-pointer calls above keep one cached plan per precision so that
 * repeated calls reuse device workspace; this frees it. */
int cg_release_cache(void);

/* Number of kernels libcugridder.so has launched in this process (its own
 * kernels; cuFFT's are not counted). */
long long cg_kernel_launches(void);

const char *cg_last_error(void);
int cg_version(void);

#ifdef __cplusplus
}
#endif
#endif /* CUGRIDDER_B200_H */
