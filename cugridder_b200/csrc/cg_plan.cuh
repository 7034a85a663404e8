// Plan object behind the C ABI.  Replaces the reference's CURAFFT_PLAN +
// ragridder_plan pair (curafft_plan.h:74-150, ragridder_plan.h:36-56), which
// is created, filled and freed inside every call (cugridder.cu:309-388); here
// the plan owns its device workspace and cuFFT plan and keeps them resident
// across calls.
#pragma once
#include <mutex>

#include "cg_internal.cuh"

struct cg_dev_buf {
  void* p = nullptr;
  size_t cap = 0;
};

// Per-stage CUDA-event timers (two event sets, so one call's events are read
// back at the next call's w-range synchronization instead of adding a sync).
constexpr int kMaxStages = 8;
struct cg_stage_timer {
  bool on = false;
  bool created = false;
  cudaEvent_t ev[2][kMaxStages + 1];
  int n[2] = {0, 0};
  int dir[2] = {0, 0};
  bool pending[2] = {false, false};
  int cur = 0;
  double acc[2][kMaxStages] = {};
  long long calls[2] = {0, 0};
};

struct cg_plan_s {
  int device = 0;
  cudaStream_t stream = nullptr;
  // user configuration
  int nx = 0, ny = 0, sign = -1, precision = CG_PREC_FP64;
  double fov = 0, eps = 0, sigma = 2.0;
  int eps_status = CG_OK;  // CG_WARN_EPS_CLIPPED when epsilon was clipped
  // kernel (setup_conv_opts, conv_interp_invoker.cu:49-119)
  int kw = 0;
  double beta = 0, es_c = 0;
  int nf1 = 0, nf2 = 0;
  cg::Quad quad;
  // last call
  cg::Geom geom{};
  int64_t nrow = 0;
  int key_bytes = 4;
  int stop_stage = 0;
  int grid_method = 1;  // 0 direct, 1 tiled SIMT, 2 tensor-core (cg_plan_set_method, CG_GRID_METHOD)
  cg::TileTune tune{};  // tiling of the tiled kernels (0 = default)
  // autotuning (cg_plan_set_autotune, CG_AUTOTUNE): the first call per
  // direction times the candidate tilings of its spreading / interpolation
  // launch; tuned_key holds the geometry (nf1, nf2, nw, W) each was tuned for
  int autotune = 0;
  bool tma_armed = false;  // the TMA degridding error word has been cleared once
  int tma_default = 2;  // untuned tiling: TMA-staged degridding variant where it applies (CG_DEGRID_TMA: 0 off, 1, 2)
  int tuned_key[2][4] = {};
  float tuned_ms[2] = {0.f, 0.f};
  // gridding kernel: CG_KERNEL_ES (W from epsilon) or CG_KERNEL_POLY (W and
  // piecewise-polynomial coefficients given by cg_plan_set_kernel)
  int kernel_kind = CG_KERNEL_ES;
  int poly_w = 0;
  int es_w = 0;  // CG_KERNEL_ES with a forced width (0: from epsilon)
  double poly[cg::kMaxW * cg::kPolyCoef] = {};
  // device buffers
  cg_dev_buf mm, K1, K2, K3q, zq, grid, recs, perm, skeys, hive_start, binws, fftwork, io_uvw,
      io_vis, io_wgt, io_dirty, polyf, polyd, recs_tmp, chan_uvw, chan_scale, coltw, acc, roots;
  // row split of heavy warp tiles in gridding (chunks per tile and their
  // scan, the scan's workspace, the partial tiles)
  cg_dev_buf split_chunks, split_sums, split_parts;
  unsigned long long* h_mm = nullptr;  // pinned, 2 words + flag
  // cuFFT: full 2-D batched plan, and the 1-D plans of the band-pruned path
  cufftHandle fft = 0;
  bool fft_valid = false;
  int fft_nf1 = 0, fft_nf2 = 0, fft_nw = 0;
  size_t fft_work_bytes = 0;
  cufftHandle fft_rows = 0, fft_cols = 0;
  bool rows_valid = false, cols_valid = false;
  int rows_n = 0, rows_batch = 0, cols_n = 0, cols_stride = 0, cols_batch = 0;
  int fft_pruning = 1;  // 0: always the full 2-D transform (CG_FFT_PRUNE=0)
  int col_fft = 1;      // 0: cuFFT for the column transforms too (CG_COL_FFT=0)
  int four_step = 0;    // four-step column transform (CG_COL_FFT_REG=4 at creation)
  int roots_n = 0;      // length of the root table in roots
  int row_fft = 0;      // 1: register-resident row kernel instead of cuFFT rows (CG_ROW_FFT=1; slower on B200)
  int coltw_n = 0;      // length of the twiddle table in coltw
  // memory-limited mode (cg_plan_set_grid_budget): the grid holds plane_batch
  // planes at a time when the whole grid exceeds grid_budget bytes
  size_t grid_budget = 0;
  // fixed-uvw mode (cg_plan_set_fixed_uvw): calls with the same uvw pointer,
  // nrow and freq as the last one reuse its geometry and binning (no host
  // synchronisation, so such calls can be captured in a CUDA graph)
  int fixed_uvw = 0;
  bool bins_valid = false;
  // the quarter tables (K3q, zq) hold those of quarter_key: they depend only on
  // the image geometry, the w-derived shift and scales and the kernel's
  // quadrature (reset when the plan is reconfigured)
  bool quarter_valid = false;
  double quarter_key[7] = {};
  // the u, v, w ranges (range words 0-5), row count and frequency the current
  // geometry was built from (spec_valid), for dirty2ms_speculate: a plane fill
  // and FFT started on that geometry (spec_pending) and confirmed by the
  // call's range pass (spec_hit)
  bool spec_valid = false, spec_pending = false, spec_hit = false;
  unsigned long long spec_mm[6] = {};
  int64_t spec_nrow = -1;
  double spec_freq = 0;
  const double* last_uvw = nullptr;
  int64_t last_nrow = -1;
  double last_freq = 0;
  int plane_batch = 0;  // 0: the whole grid is resident
  cufftHandle fft1 = 0; // one-plane 2-D transform of the memory-limited mode
  bool fft1_valid = false;
  int fft1_nf1 = 0, fft1_nf2 = 0;
  cg_stage_timer timer;
  // host entry points: every input is copied on io_stream, one copy after the
  // other in the order the stages need them (uvw, then the visibilities or
  // the image, then the weights), each at the link's full bandwidth; the
  // plan's stream waits for uvw before the w range, on main_ready (when set)
  // before the first stage that reads the visibilities or the image, and on
  // inputs_ready (when set) before the first stage that reads the weights
  cudaStream_t io_stream = nullptr;
  cudaEvent_t io_event = nullptr, io_ev_uvw = nullptr, io_ev_main = nullptr;
  cudaEvent_t inputs_ready = nullptr, main_ready = nullptr;
  // uvw_ready (when set): the plan's stream waits on it before the first
  // stage that reads uvw.  host_mm (when set): the u/v/w range words and the
  // non-finite flag, computed on the host from the caller's uvw (the layout
  // of launch_wminmax's output), so prepare() needs no device pass and no
  // synchronization.  With both, dirty2ms runs the plane fill and the FFT on
  // aux_stream as soon as the image is in, concurrently with the binning.
  cudaEvent_t uvw_ready = nullptr;
  const unsigned long long* host_mm = nullptr;
  cudaStream_t aux_stream = nullptr;
  cudaEvent_t aux_ev0 = nullptr, aux_ev1 = nullptr;
  std::mutex mu;
};

namespace cg {
int setup_conv_opts(double eps, double sigma, double eps_floor, int& kw, double& beta, double& c);
int get_num_cells(int ms, double sigma, int kw);
void set_nhg_w(double S, double X, int kw, double sigma, int& nf, double& h, double& gam);
// Geometry of one call (setup_gridder_plan, cugridder.cu:29-86): fills g's
// pixel sizes, f/c, sign, the w range's centre and half width (from the
// range words h_mm[4..5] of launch_wminmax; zero width when nrow == 0), o_c,
// the w planes (set_nhg_w) and the hive counts.  g.N1, N2, nf1, nf2, kw,
// beta and es_c must be set.  Shared by the plan path and the allocation-free
// binning, so that both key the same rows alike.
int call_geometry(double fov, double freq, int sign, double sigma, int64_t nrow,
                  const unsigned long long* h_mm, Geom& g);
void make_quad(int kw, double beta, double c, const double* poly, Quad& q);
void fseries_uv(const Quad& q, int nf, double* out);
int plan_configure(cg_plan_s* P, int nx, int ny, double fov, double eps, double sigma, int sign,
                   int precision);
int ensure(cg_dev_buf& b, size_t bytes);
void release(cg_dev_buf& b);
size_t workspace_bytes(const cg_plan_s* P);
int timer_begin(cg_plan_s* P, int dir);
void timer_mark(cg_plan_s* P);
void timer_flush(cg_plan_s* P, int set);
}  // namespace cg
