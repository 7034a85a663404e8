// Host orchestration of ms2dirty / dirty2ms (improved W-stacking).
//
// Reference flow: ms2dirty_exec -> gridder_setting -> exec_vis2dirty
// (cugridder.cu:276-404, :90-210; ra_exec.cu:184-468) and dirty2ms_exec ->
// exec_dirty2vis (cugridder.cu:406-538; ra_exec.cu:470-680).  The scalar plan
// math below restates setup_conv_opts, get_num_cells, next235beven,
// set_nhg_w and setup_gridder_plan; everything else runs as stream-ordered
// kernels with no intermediate device synchronization (one small read of the
// w range per call).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "cg_launch.cuh"
#include "cg_plan.cuh"

namespace cg {

// ------------------------------------------------------------ scalar plan math
// next235beven: common_utils.cu:76-101
static int next235beven(int n, int b) {
  if (n <= 2) return 2;
  if (n % 2 == 1) n += 1;
  int nplus = n - 2, numdiv = 2;
  while ((numdiv > 1) || (nplus % b != 0)) {
    nplus += 2;
    numdiv = nplus;
    while (numdiv % 2 == 0) numdiv /= 2;
    while (numdiv % 3 == 0) numdiv /= 3;
    while (numdiv % 5 == 0) numdiv /= 5;
  }
  return nplus;
}

// beta / W of the ES kernel for width kw (conv_interp_invoker.cu:87-114)
static double es_beta_over_w(int kw, double sigma) {
  double betaoverns = 2.30;
  if (kw == 2) betaoverns = 2.20;
  if (kw == 3) betaoverns = 2.26;
  if (kw == 4) betaoverns = 2.38;
  if (sigma != 2.0) betaoverns = 0.97 * kPi * (1 - 1 / (2 * sigma));
  return betaoverns;
}

// setup_conv_opts: conv_interp_invoker.cu:49-119
int setup_conv_opts(double eps, double sigma, double eps_floor, int& kw, double& beta,
                           double& c) {
  int st = CG_OK;
  if (!(sigma > 1.0)) return CG_ERR_ARG;
  if (!(eps >= eps_floor)) {  // also catches NaN / non-positive eps
    eps = eps_floor;
    st = CG_WARN_EPS_CLIPPED;
  }
  kw = (int)std::ceil(-std::log10(eps / 10.0));
  if (sigma != 2.0) kw = (int)std::ceil(-std::log(eps) / (kPi * std::sqrt(1.0 - 1.0 / sigma)));
  kw = std::max(2, kw);
  kw = std::min(kMaxW, kw);
  beta = es_beta_over_w(kw, sigma) * (double)kw;
  c = 4.0 / (double)(kw * kw);
  return st;
}

// get_num_cells: conv_interp_invoker.cu:30-47
int get_num_cells(int ms, double sigma, int kw) {
  int nf = (int)(sigma * ms);
  if (nf < 2 * kw) nf = 2 * kw;
  return next235beven(nf, 1);
}

// set_nhg_w: utils.cu:670-709
void set_nhg_w(double S, double X, int kw, double sigma, int& nf, double& h, double& gam) {
  int nss = kw + 1;
  double Xsafe = X, Ssafe = S;
  if (X == 0.0) {
    if (S == 0.0) {
      Xsafe = 1.0;
      Ssafe = 1.0;
    } else {
      Xsafe = std::max(Xsafe, 1 / S);
    }
  } else {
    Ssafe = std::max(Ssafe, 1 / X);
  }
  double nfd = 2.0 * sigma * Ssafe * Xsafe / kPi + nss;
  if (!std::isfinite(nfd)) nfd = 0.0;
  double capped = std::min(nfd, 1.0e9);
  nf = (int)capped;
  nf = nf % 2 + nf;
  if (nf < 2 * kw) nf = 2 * kw;
  h = 2 * kPi / nf;
  gam = (double)nf / (2.0 * sigma * Ssafe);
}

// Gauss-Legendre nodes on [-1,1] (Newton on the Legendre recurrence),
// decreasing order; the fseries uses the first (positive) half of 2p nodes
// (deconv.cu:80-93).
static void gauss_legendre(int n, double* x, double* w) {
  for (int k = 0; k < n; k++) {
    double z = std::cos(kPi * (k + 0.75) / (n + 0.5)), pp = 0;
    for (int it = 0; it < 100; it++) {
      double p0 = 1.0, p1 = z;
      for (int j = 2; j <= n; j++) {
        double p2 = ((2.0 * j - 1.0) * z * p1 - (j - 1.0) * p0) / j;
        p0 = p1;
        p1 = p2;
      }
      pp = n * (z * p1 - p0) / (z * z - 1.0);
      double dz = p1 / pp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    double p0 = 1.0, p1 = z;
    for (int j = 2; j <= n; j++) {
      double p2 = ((2.0 * j - 1.0) * z * p1 - (j - 1.0) * p0) / j;
      p0 = p1;
      p1 = p2;
    }
    pp = n * (z * p1 - p0) / (z * z - 1.0);
    x[k] = z;
    w[k] = 2.0 / ((1.0 - z * z) * pp * pp);
  }
}

// piecewise-polynomial kernel value at d (segment floor(d + W/2)); 0 outside
static double poly_phi(const double* poly, int kw, double d) {
  const double u = d + 0.5 * kw;
  const int s = (int)std::floor(u);
  if (s < 0 || s >= kw) return 0.0;
  const double t = 2.0 * (u - s) - 1.0;
  const double* a = poly + s * kPolyCoef;
  double v = a[kPolyCoef - 1];
  for (int n = kPolyCoef - 2; n >= 0; n--) v = v * t + a[n];
  return v;
}

// quadrature of the kernel Fourier series (deconv.cu:80-93): ES, or the
// piecewise-polynomial kernel when poly is given
void make_quad(int kw, double beta, double c, const double* poly, Quad& q) {
  double alpha = kw / 2.0;
  int p = (int)(2 + 3.0 * alpha);
  double x[2 * kMaxQuad], w[2 * kMaxQuad];
  gauss_legendre(2 * p, x, w);
  q.p = p;
  for (int n = 0; n < p; n++) {
    double xn = x[n] * alpha;
    double phi = poly ? poly_phi(poly, kw, xn)
                      : ((std::fabs(xn) <= alpha) ? std::exp(beta * std::sqrt(1.0 - c * xn * xn)) : 0.0);
    q.x[n] = xn;
    q.g[n] = alpha * w[n] * phi;
  }
}

// fwkerhalf{1,2} (deconv.cu:12-26): (-1)^k folded into the cosine
void fseries_uv(const Quad& q, int nf, double* out) {
  int N = nf / 2 + 1;
  for (int k = 0; k < N; k++) {
    double s = 0;
    for (int i = 0; i < q.p; i++) s += q.g[i] * std::cos((q.x[i] - N + 1) / (double)(N - 1) * kPi * k);
    out[k] = 2 * s;
  }
}

// ------------------------------------------------------------ buffers
int ensure(cg_dev_buf& b, size_t bytes) {
  if (bytes == 0) bytes = 256;
  if (b.cap >= bytes) return CG_OK;
  if (b.p) {
    cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
  }
  CG_CUDA(cudaMalloc(&b.p, bytes));
  b.cap = bytes;
  return CG_OK;
}

void release(cg_dev_buf& b) {
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.cap = 0;
}

size_t workspace_bytes(const cg_plan_s* P) {
  const cg_dev_buf* bs[] = {&P->mm,   &P->K1,    &P->K2,         &P->K3q,   &P->zq,
                            &P->grid, &P->recs,  &P->recs_tmp, &P->perm,       &P->skeys, &P->hive_start,
                            &P->binws, &P->fftwork, &P->io_uvw, &P->io_vis, &P->io_wgt,
                            &P->io_dirty, &P->split_chunks, &P->split_sums, &P->split_parts};
  size_t s = 0;
  for (auto b : bs) s += b->cap;
  return s;
}

// ------------------------------------------------------------ stage timers
int timer_begin(cg_plan_s* P, int dir) {
  cg_stage_timer& T = P->timer;
  if (!T.on) return CG_OK;
  if (!T.created) {
    for (int s = 0; s < 2; s++)
      for (int i = 0; i <= kMaxStages; i++) CG_CUDA(cudaEventCreate(&T.ev[s][i]));
    T.created = true;
  }
  T.cur ^= 1;
  T.n[T.cur] = 0;
  T.dir[T.cur] = dir;
  T.pending[T.cur] = true;
  timer_mark(P);
  return CG_OK;
}

void timer_mark(cg_plan_s* P) {
  cg_stage_timer& T = P->timer;
  if (!T.on || !T.created || T.n[T.cur] > kMaxStages) return;
  cudaEventRecord(T.ev[T.cur][T.n[T.cur]], P->stream);
  T.n[T.cur]++;
}

// reads a finished event set (its stream work is complete) into the totals
void timer_flush(cg_plan_s* P, int set) {
  cg_stage_timer& T = P->timer;
  if (!T.created || !T.pending[set]) return;
  for (int i = 1; i < T.n[set]; i++) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, T.ev[set][i - 1], T.ev[set][i]) == cudaSuccess)
      T.acc[T.dir[set]][i - 1] += ms;
  }
  cudaGetLastError();
  T.calls[T.dir[set]]++;
  T.pending[set] = false;
}

int plan_configure(cg_plan_s* P, int nx, int ny, double fov, double eps, double sigma, int sign,
                   int precision) {
  if (nx <= 0 || ny <= 0 || (nx & 1) || (ny & 1)) {
    set_last_error("nxdirty and nydirty must be positive and even");
    return CG_ERR_ARG;
  }
  if (!(fov > 0.0) || !std::isfinite(fov)) {
    set_last_error("fov must be positive and finite");
    return CG_ERR_ARG;
  }
  if (precision != CG_PREC_FP64 && precision != CG_PREC_FP32) return CG_ERR_ARG;
  bool same = P->kw > 0 && P->nx == nx && P->ny == ny && P->fov == fov && P->eps == eps &&
              P->sigma == sigma && P->sign == sign && P->precision == precision;
  if (same) return CG_OK;
  double floor_eps = (precision == CG_PREC_FP64) ? 1.1e-16 : 6e-8;  // utils.h:34-38
  int kw;
  double beta, c;
  int st = setup_conv_opts(eps, sigma, floor_eps, kw, beta, c);
  if (st > 1) {
    set_last_error("sigma must be > 1");
    return st;
  }
  const bool poly = P->kernel_kind == CG_KERNEL_POLY;
  if (poly) {  // the kernel's own width replaces the width chosen from epsilon
    kw = P->poly_w;
    beta = 0.0;
    c = 0.0;
  } else if (P->es_w > 0) {  // ES at a forced width: the same beta rule for that W
    kw = P->es_w;
    beta = es_beta_over_w(kw, sigma) * kw;
    c = 4.0 / (double)(kw * kw);
  }
  int nf1 = get_num_cells(ny, sigma, kw), nf2 = get_num_cells(nx, sigma, kw);
  if (nf1 > 65535 || nf2 > 65535) {
    set_last_error("grid larger than 65535 cells per axis");
    return CG_ERR_SIZE;
  }
  P->nx = nx;
  P->ny = ny;
  P->fov = fov;
  P->eps = eps;
  P->sigma = sigma;
  P->sign = sign;
  P->precision = precision;
  P->eps_status = st;
  P->bins_valid = false;
  P->quarter_valid = false;
  P->spec_valid = false;
  P->kw = kw;
  P->beta = beta;
  P->es_c = c;
  P->nf1 = nf1;
  P->nf2 = nf2;
  make_quad(kw, beta, c, poly ? P->poly : nullptr, P->quad);
  if (poly) {
    float pf[kMaxW * kPolyCoef];
    for (int i = 0; i < kw * kPolyCoef; i++) pf[i] = (float)P->poly[i];
    CG_TRY(ensure(P->polyd, sizeof(double) * kw * kPolyCoef));
    CG_TRY(ensure(P->polyf, sizeof(float) * kw * kPolyCoef));
    CG_CUDA(cudaMemcpy(P->polyd.p, P->poly, sizeof(double) * kw * kPolyCoef, cudaMemcpyHostToDevice));
    CG_CUDA(cudaMemcpy(P->polyf.p, pf, sizeof(float) * kw * kPolyCoef, cudaMemcpyHostToDevice));
  }
  std::vector<double> k1(nf1 / 2 + 1), k2(nf2 / 2 + 1);
  fseries_uv(P->quad, nf1, k1.data());
  fseries_uv(P->quad, nf2, k2.data());
  CG_TRY(ensure(P->K1, k1.size() * 8));
  CG_TRY(ensure(P->K2, k2.size() * 8));
  CG_CUDA(cudaMemcpy(P->K1.p, k1.data(), k1.size() * 8, cudaMemcpyHostToDevice));
  CG_CUDA(cudaMemcpy(P->K2.p, k2.data(), k2.size() * 8, cudaMemcpyHostToDevice));
  size_t nq = (size_t)(ny / 2 + 1) * (nx / 2 + 1);
  CG_TRY(ensure(P->K3q, nq * 8));
  CG_TRY(ensure(P->zq, nq * 8));
  return CG_OK;
}

// ------------------------------------------------------------ per-call geometry
// setup_gridder_plan (cugridder.cu:29-86) with the w range from the device.
// the band-pruned transform pays off for this geometry (else the full 2-D one runs)
static bool fft_is_pruned(const cg_plan_s* P, const Geom& g) {
  const int nrows = g.band_r1 - g.band_r0 + 1;
  const double full = 2.0 * g.nf1 * g.nf2;
  const double pruned = (double)nrows * g.nf1 + (double)g.N1 * g.nf2;
  return P->fft_pruning && pruned <= 0.8 * full;
}

static bool cols_all_env() {
  static const bool v = getenv("CG_FFT_COLS_ALL") && atoi(getenv("CG_FFT_COLS_ALL")) != 0;
  return v;
}

// The forward transform's columns go through the one-pass register-resident
// kernel, which skips loading the rows outside the image (so the plane fill
// need not zero them in the image's columns)
static bool fill_skip_ok(const cg_plan_s* P, const Geom& g, int rowperm) {
  if (rowperm || P->precision != CG_PREC_FP32 || !P->col_fft || P->plane_batch ||
      cols_all_env() || !fft_is_pruned(P, g) || g.N1 % 2 != 0)
    return false;
  const char* e = getenv("CG_COL_FFT_REG");
  if (e && atoi(e) != 1) return false;  // the other column kernels load every row
  return col_fft_supported(g.nf2, g.N1 / 2, g.N1 / 2);
}

// L2 of the four-step column transform when it will run for this geometry
// (FP32 plans with the column kernels, band-pruned transform, resident
// planes, image halves in whole 16-column groups), else 0.  Chosen with
// CG_COL_FFT_REG=4, and by default for L = 16384, beyond the one-pass kernels.
static int four_step_rows(const cg_plan_s* P, const Geom& g) {
  if (!(P->four_step || g.nf2 == 16384) || P->precision != CG_PREC_FP32 || !P->col_fft ||
      P->plane_batch || cols_all_env() || !fft_is_pruned(P, g) || g.N1 % 2 != 0)
    return 0;
  return four_step_supported(g.nf2, g.N1 / 2, g.N1 / 2) ? g.nf2 / 64 : 0;
}

int call_geometry(double fov, double freq, int sign, double sigma, int64_t nrow,
                  const unsigned long long* h_mm, Geom& g) {
  g.pixx = fov / 180.0 * kPi / (double)g.N2;
  g.pixy = fov / 180.0 * kPi / (double)g.N1;
  g.foc = freq / kSpeedOfLight;
  g.sign = sign;
  double wmin = 0, wmax = 0;
  if (nrow > 0) {
    const double rmin = decode_ordered(h_mm[4]), rmax = decode_ordered(h_mm[5]);
    // same rounding chain as eff_coords(); monotone in w
    auto scale = [&](double w) { return (w * (g.foc * (double)g.sign)) * (2 * kPi); };
    const double a = scale(rmin), b = scale(rmax);
    wmin = std::min(a, b);
    wmax = std::max(a, b);
  }
  const double l_min = 0 - 0.5 * g.pixx * g.N2;
  const double m_min = 0 - 0.5 * g.pixy * g.N1;
  const double temp = 1.0 - std::pow(l_min, 2) - std::pow(m_min, 2);
  const double n_lm = temp <= 0 ? 0 : std::sqrt(temp);
  g.i_center = (wmax + wmin) / 2.0;
  g.i_half_width = (wmax - wmin) / 2.0;
  const double o_min = n_lm - 1;
  g.o_center = o_min / 2.0;
  g.o_half_width = std::fabs(o_min / 2.0);
  set_nhg_w(g.o_half_width, g.i_half_width, g.kw, sigma, g.nw, g.h, g.gamma);
  if (g.nw > 65535) {
    set_last_error("number of w planes too large");
    return CG_ERR_SIZE;
  }
  g.nhx = (g.nf1 - 1) / 8 + 1;
  g.nhy = (g.nf2 - 1) / 8 + 1;
  g.nhz = g.nw;
  return CG_OK;
}

static int prepare(cg_plan_s* P, int64_t nrow, double freq, const double* d_uvw) {
  if (nrow < 0 || nrow > 2147483647LL) {
    set_last_error("nrow out of range");
    return nrow < 0 ? CG_ERR_ARG : CG_ERR_SIZE;
  }
  if (!(freq > 0.0) || !std::isfinite(freq)) {
    set_last_error("freq must be positive and finite");
    return CG_ERR_ARG;
  }
  cudaStream_t st = P->stream;
  CG_TRY(ensure(P->mm, 128));
  if (!P->h_mm) CG_CUDA(cudaMallocHost(&P->h_mm, 128));
  unsigned long long* d_mm = (unsigned long long*)P->mm.p;
  int* d_bad = (int*)(d_mm + 6);
  if (P->host_mm) {
    // ranges computed on the host from the caller's uvw: no device pass, no
    // synchronization (host entry points, which check the TMA status per call)
    memcpy(P->h_mm, P->host_mm, 7 * sizeof(unsigned long long));
    ((int*)P->h_mm)[18] = 0;
  } else {
    if (P->uvw_ready) CG_CUDA(cudaStreamWaitEvent(st, P->uvw_ready, 0));
    CG_TRY(launch_wminmax(d_uvw, nrow, d_mm, d_bad, st));
    CG_CUDA(cudaMemcpyAsync(P->h_mm, d_mm, 80, cudaMemcpyDeviceToHost, st));
    CG_CUDA(cudaStreamSynchronize(st));
  }
  if (P->spec_pending) {  // a plane fill and FFT started on the last call's geometry
    P->spec_pending = false;
    P->spec_hit = nrow == P->spec_nrow && freq == P->spec_freq &&
                  std::equal(P->spec_mm, P->spec_mm + 6, P->h_mm) &&
                  ((const int*)(P->h_mm + 6))[0] == 0;
    // otherwise its grid and tables are rebuilt below: let it finish first
    if (!P->spec_hit) CG_CUDA(cudaStreamSynchronize(P->aux_stream));
  }
  timer_flush(P, P->timer.cur ^ 1);
  if (P->tma_armed && ((const int*)P->h_mm)[18]) {  // word 72: a TMA staging wait ran out
    // only a call captured into a CUDA graph (or one whose status was not
    // read) leaves the word set: non-captured calls report it themselves
    CG_CUDA(cudaMemsetAsync((char*)P->mm.p + 72, 0, sizeof(int), st));
    set_last_error("degridding: a TMA staging wait timed out in an earlier call");
    return CG_ERR_CUDA;
  }
  if (((int*)(P->h_mm + 6))[0]) {
    set_last_error("non-finite uvw coordinate");
    return CG_ERR_ARG;
  }
  Geom g{};
  g.N1 = P->ny;
  g.N2 = P->nx;
  g.nf1 = P->nf1;
  g.nf2 = P->nf2;
  g.kw = P->kw;
  g.beta = P->beta;
  g.es_c = P->es_c;
  const bool poly = P->kernel_kind == CG_KERNEL_POLY;
  g.polyf = poly ? (const float*)P->polyf.p : nullptr;
  g.polyd = poly ? (const double*)P->polyd.p : nullptr;
  CG_TRY(call_geometry(P->fov, freq, P->sign, P->sigma, nrow, P->h_mm, g));
  // band of grid rows (g1 <- u) / columns (g0 <- v) reached by the taps: the
  // grid coordinate is monotone in u (v) while the scaled value stays inside
  // [-pi, pi); otherwise the data wraps and the band is the whole axis.
  g.band_r0 = 0;
  g.band_r1 = g.nf2 - 1;
  g.band_c0 = 0;
  g.band_c1 = g.nf1 - 1;
  if (nrow > 0) {
    const int lo = (g.kw - 1) / 2 + 1, hi = (g.kw + 1) / 2 + 1;  // tap halo, one cell of margin
    auto band = [&](double umin, double umax, double pix, int nf, int& b0, int& b1) {
      const double a = ((umin * g.foc) * (2 * kPi)) * pix, b = ((umax * g.foc) * (2 * kPi)) * pix;
      if (!(a > -kPi + 1e-9 && b < kPi - 1e-9)) return;
      const double xa = (a * kM_1_2PI + 0.5) * nf, xb = (b * kM_1_2PI + 0.5) * nf;
      const int r0 = (int)std::floor(xa) - lo, r1 = (int)std::floor(xb) + hi;
      if (r0 < 0 || r1 >= nf) return;
      b0 = r0;
      b1 = r1;
    };
    band(decode_ordered(P->h_mm[0]), decode_ordered(P->h_mm[1]), g.pixx, g.nf2, g.band_r0, g.band_r1);
    band(decode_ordered(P->h_mm[2]), decode_ordered(P->h_mm[3]), g.pixy, g.nf1, g.band_c0, g.band_c1);
  }
  P->geom = g;
  P->nrow = nrow;
  int64_t nh = (int64_t)g.nhx * g.nhy * g.nhz;
  P->key_bytes = ((unsigned long long)nh * 64ULL <= 0xFFFFFFFFULL) ? 4 : 8;
  size_t tsz = (P->precision == CG_PREC_FP64) ? 8 : 4;
  size_t G = (size_t)g.nf1 * g.nf2 * g.nw;
  P->plane_batch = 0;
  if (P->grid_budget > 0 && G * 2 * tsz > P->grid_budget) {
    // memory-limited mode: as many whole planes as the budget holds
    const size_t plane_bytes = (size_t)g.nf1 * g.nf2 * 2 * tsz;
    const size_t pb = P->grid_budget / plane_bytes;
    if (pb < 1) {
      set_last_error("grid budget smaller than one w plane");
      return CG_ERR_NOMEM;
    }
    P->plane_batch = (int)std::min<size_t>(pb, (size_t)g.nw);
    CG_TRY(ensure(P->grid, (size_t)P->plane_batch * plane_bytes));
  } else {
    CG_TRY(ensure(P->grid, G * 2 * tsz));
  }
  // hive offsets followed by the scan scratch of the counting path
  CG_TRY(ensure(P->hive_start, (size_t)(nh + 1 + hive_sums_ints(nh)) * 4));
  CG_TRY(ensure(P->perm, (size_t)nrow * 4));
  CG_TRY(ensure(P->skeys, (size_t)nrow * P->key_bytes));
  CG_TRY(ensure(P->binws, bin_workspace_bytes(nrow, P->key_bytes)));
  CG_TRY(ensure(P->recs, (size_t)nrow * (tsz == 8 ? sizeof(Rec<double>) : sizeof(Rec<float>))));
  CG_TRY(ensure(P->recs_tmp, (size_t)nrow * (tsz == 8 ? sizeof(Rec<double>) : sizeof(Rec<float>))));
  P->geom.rowperm = four_step_rows(P, P->geom);
  P->geom.fill_skip = fill_skip_ok(P, P->geom, P->geom.rowperm) ? 1 : 0;
  P->geom.grid_skip = P->geom.fill_skip;
  std::copy(P->h_mm, P->h_mm + 6, P->spec_mm);
  P->spec_nrow = nrow;
  P->spec_freq = freq;
  P->spec_valid = nrow > 0;
  return CG_OK;
}

static int fft_exec(cg_plan_s* P, void* d_grid, int direction) {
  const Geom& g = P->geom;
  if (!P->fft_valid || P->fft_nf1 != g.nf1 || P->fft_nf2 != g.nf2 || P->fft_nw != g.nw ||
      P->precision == -1) {
    if (P->fft_valid) {
      cufftDestroy(P->fft);
      P->fft_valid = false;
    }
    CG_CUFFT(cufftCreate(&P->fft));
    P->fft_valid = true;
    CG_CUFFT(cufftSetAutoAllocation(P->fft, 0));
    long long n[2] = {g.nf2, g.nf1};
    size_t ws = 0;
    cufftType t = (P->precision == CG_PREC_FP64) ? CUFFT_Z2Z : CUFFT_C2C;
    CG_CUFFT(cufftMakePlanMany64(P->fft, 2, n, nullptr, 1, 0, nullptr, 1, 0, t, g.nw, &ws));
    if (ws > P->fftwork.cap) {
      CG_CUDA(cudaStreamSynchronize(P->stream));
      CG_TRY(ensure(P->fftwork, ws));
      if (P->rows_valid) CG_CUFFT(cufftSetWorkArea(P->fft_rows, P->fftwork.p));
      if (P->cols_valid) CG_CUFFT(cufftSetWorkArea(P->fft_cols, P->fftwork.p));
    }
    CG_CUFFT(cufftSetWorkArea(P->fft, P->fftwork.p));
    P->fft_nf1 = g.nf1;
    P->fft_nf2 = g.nf2;
    P->fft_nw = g.nw;
    P->fft_work_bytes = ws;
  }
  CG_CUFFT(cufftSetStream(P->fft, P->stream));
  if (P->precision == CG_PREC_FP64)
    CG_CUFFT(cufftExecZ2Z(P->fft, (cufftDoubleComplex*)d_grid, (cufftDoubleComplex*)d_grid, direction));
  else
    CG_CUFFT(cufftExecC2C(P->fft, (cufftComplex*)d_grid, (cufftComplex*)d_grid, direction));
  return CG_OK;
}

// work-queue head of the tiled kernels: a word of the small scratch buffer
static int* queue_counter(cg_plan_s* P) { return (int*)((char*)P->mm.p + 64); }
// error word of the TMA-staged degridding (read back by the next prepare)
static int* tma_error_word(cg_plan_s* P) { return (int*)((char*)P->mm.p + 72); }

// Degridding launch for tiling tt: threads -1 / -2 select the TMA-staged
// kernel's variant 1 / 2 (FP32 where it applies), anything else the tiled
// kernel; untuned plans take variant tma_default (0: the tiled kernel).
template <typename T>
static int degrid_dispatch(cg_plan_s* P, const TileTune& tt, T* d_vis) {
  const Geom& g = P->geom;
  const int variant = tt.dthreads < 0 ? -tt.dthreads : (tt.dthreads == 0 ? P->tma_default : 0);
  if (variant > 0) {
    if constexpr (sizeof(T) == 4) {
      if (P->grid_method == kGridTiled && degrid_tma_supported(g, variant)) {
        if (!P->tma_armed) {
          CG_CUDA(cudaMemsetAsync(tma_error_word(P), 0, sizeof(int), P->stream));
          P->tma_armed = true;
        }
        return launch_degrid_tma((const Rec<float>*)P->recs.p, (const int*)P->perm.p,
                                 (const int*)P->hive_start.p, P->nrow, g,
                                 (const float*)P->grid.p, (float*)d_vis, queue_counter(P),
                                 tma_error_word(P), P->stream, variant);
      }
    }
    if (tt.dthreads < 0) return CG_ERR_ARG;  // a tuning candidate that does not apply
  }
  return launch_degrid<T>((const Rec<T>*)P->recs.p, (const int*)P->perm.p,
                          (const int*)P->hive_start.p, P->nrow, g, (const T*)P->grid.p, d_vis,
                          P->grid_method, queue_counter(P), P->stream, &tt);
}

// 1-D cuFFT plans of the band-pruned transform (work areas shared with the
// 2-D plan's buffer; the plans run one after another on the plan's stream).
static int make_1d_plan(cg_plan_s* P, cufftHandle& h, bool& valid, int n, int stride, int batch) {
  if (valid) {
    cufftDestroy(h);
    valid = false;
  }
  CG_CUFFT(cufftCreate(&h));
  valid = true;
  CG_CUFFT(cufftSetAutoAllocation(h, 0));
  long long nn[1] = {n}, emb[1] = {n};
  size_t ws = 0;
  cufftType t = (P->precision == CG_PREC_FP64) ? CUFFT_Z2Z : CUFFT_C2C;
  if (stride == 1)
    CG_CUFFT(cufftMakePlanMany64(h, 1, nn, nullptr, 1, 0, nullptr, 1, 0, t, batch, &ws));
  else
    CG_CUFFT(cufftMakePlanMany64(h, 1, nn, emb, stride, 1, emb, stride, 1, t, batch, &ws));
  if (ws > P->fftwork.cap) {
    // grow the shared work buffer; every plan must point at the new one
    CG_CUDA(cudaStreamSynchronize(P->stream));
    CG_TRY(ensure(P->fftwork, ws));
    if (P->fft_valid) CG_CUFFT(cufftSetWorkArea(P->fft, P->fftwork.p));
    if (P->rows_valid && &h != &P->fft_rows) CG_CUFFT(cufftSetWorkArea(P->fft_rows, P->fftwork.p));
    if (P->cols_valid && &h != &P->fft_cols) CG_CUFFT(cufftSetWorkArea(P->fft_cols, P->fftwork.p));
  }
  CG_CUFFT(cufftSetWorkArea(h, P->fftwork.p));
  return CG_OK;
}

static int exec_c2c(cg_plan_s* P, cufftHandle h, void* data, int direction) {
  CG_CUFFT(cufftSetStream(h, P->stream));
  if (P->precision == CG_PREC_FP64)
    CG_CUFFT(cufftExecZ2Z(h, (cufftDoubleComplex*)data, (cufftDoubleComplex*)data, direction));
  else
    CG_CUFFT(cufftExecC2C(h, (cufftComplex*)data, (cufftComplex*)data, direction));
  return CG_OK;
}

// Separable 2-D transform restricted to what the pipeline uses:
//   ms2dirty: rows of the data band (other rows are zero), then only the N1
//             columns the image keeps (two column ranges of N1/2);
//   dirty2ms: the N1 non-zero columns first, then only the rows the
//             degridding reads.
// Falls back to the full 2-D transform when the band saves little.
static int fft_exec_pruned(cg_plan_s* P, void* d_grid, int direction) {
  const Geom& g = P->geom;
  if (!fft_is_pruned(P, g)) return fft_exec(P, d_grid, direction);
  // rows plan: batch rounded up to 64 rows (extra rows are zero or unused)
  int r0, batch;
  fft_row_band(g, r0, batch);
  if (!P->rows_valid || P->rows_n != g.nf1 || P->rows_batch != batch) {
    CG_TRY(make_1d_plan(P, P->fft_rows, P->rows_valid, g.nf1, 1, batch));
    P->rows_n = g.nf1;
    P->rows_batch = batch;
  }
  // CG_FFT_COLS_ALL=1 (tuning): one column transform over every grid column
  const bool cols_all = cols_all_env();
  const int half = cols_all ? g.nf1 : g.N1 / 2;
  if (!P->cols_valid || P->cols_n != g.nf2 || P->cols_stride != g.nf1 || P->cols_batch != half) {
    CG_TRY(make_1d_plan(P, P->fft_cols, P->cols_valid, g.nf2, g.nf1, half));
    P->cols_n = g.nf2;
    P->cols_stride = g.nf1;
    P->cols_batch = half;
  }
  const size_t esz = (P->precision == CG_PREC_FP64) ? 16 : 8;
  const size_t plane = (size_t)g.nf1 * g.nf2;
  char* base = (char*)d_grid;
  auto rows = [&](int p) { return exec_c2c(P, P->fft_rows, base + esz * (p * plane + (size_t)r0 * g.nf1), direction); };
  auto cols = [&](int p) {
    int s1 = exec_c2c(P, P->fft_cols, base + esz * (p * plane), direction);
    if (s1 > 1 || cols_all) return s1;
    return exec_c2c(P, P->fft_cols, base + esz * (p * plane + (size_t)(g.nf1 - half)), direction);
  };
  // four-step column transform (two in-place passes over 16-column groups;
  // the w stage and the plane fill address rows through row_of)
  if (g.rowperm) {
    if (P->roots_n != g.nf2) {
      CG_TRY(ensure(P->roots, sizeof(float2) * g.nf2));
      CG_TRY(make_fft_roots(g.nf2, (float2*)P->roots.p, P->stream));
      P->roots_n = g.nf2;
    }
    auto cols4 = [&]() {
      return launch_col_fft_four_step((float2*)d_grid, g.nf2, g.nf1, plane, g.nw, 0, half,
                                      g.nf1 - half, half, direction == CUFFT_INVERSE ? 1 : -1,
                                      (const float2*)P->roots.p, P->stream);
    };
    if (direction == CUFFT_INVERSE) {
      for (int p = 0; p < g.nw; p++) CG_TRY(rows(p));
      CG_TRY(cols4());
    } else {
      CG_TRY(cols4());
      for (int p = 0; p < g.nw; p++) CG_TRY(rows(p));
    }
    return CG_OK;
  }
  // FP32 power-of-two columns: the shared-memory column transform over every
  // plane in one launch (the image's two column ranges of N1/2)
  if (P->col_fft && !cols_all && P->precision == CG_PREC_FP32 &&
      col_fft_supported(g.nf2, half, half)) {
    if (P->coltw_n != g.nf2) {
      CG_TRY(ensure(P->coltw, sizeof(float2) * col_fft_twiddle_count(g.nf2)));
      CG_TRY(make_col_fft_twiddles(g.nf2, (float2*)P->coltw.p, P->stream));
      P->coltw_n = g.nf2;
    }
    // image rows of a column under the CMCL map: [0, N2 - N2/2) and [nf2 - N2/2, nf2);
    // the rows between are zero before the forward transform (plane fill)
    // and unread after the inverse one (w-DFT).  Rows outside the band of
    // the row transforms, [r0, r0 + batch), are zero before the inverse
    // transform (gridding wrote zeros, the row pass left them) and unread
    // after the forward one (row pass and degridding stay in the band).
    const int mid0 = g.N2 - g.N2 / 2, mid1 = g.nf2 - g.N2 / 2;
    auto all_cols = [&]() {
      return launch_col_fft((float2*)d_grid, g.nf2, g.nf1, plane, g.nw, 0, half, g.nf1 - half, half,
                            direction == CUFFT_INVERSE ? 1 : -1, (const float2*)P->coltw.p,
                            P->stream, mid0, mid1, direction == CUFFT_INVERSE ? (2 | 4) : (1 | 8),
                            r0, r0 + batch);
    };
    // rows by cuFFT, or (CG_ROW_FFT=1, slower on B200) by the register-resident
    // row kernel on square grids (the same twiddles), which skips the columns
    // outside the image, [N1 - N1/2, nf1 - N1/2): zero before the forward row
    // pass and unread after the inverse one
    const bool row_kernel = g.nf1 == g.nf2 && half == g.N1 - g.N1 / 2 && P->row_fft;
    auto all_rows = [&]() -> int {
      if (row_kernel)
        return launch_row_fft((float2*)d_grid, g.nf1, plane, g.nw, r0, batch,
                              direction == CUFFT_INVERSE ? 1 : -1, (const float2*)P->coltw.p,
                              P->stream, half, g.nf1 - half, direction == CUFFT_INVERSE ? 2 : 1);
      for (int p = 0; p < g.nw; p++) CG_TRY(rows(p));
      return CG_OK;
    };
    if (direction == CUFFT_INVERSE) {
      CG_TRY(all_rows());
      CG_TRY(all_cols());
    } else {
      CG_TRY(all_cols());
      CG_TRY(all_rows());
    }
    return CG_OK;
  }
  for (int p = 0; p < g.nw; p++) {
    if (direction == CUFFT_INVERSE) {
      CG_TRY(rows(p));
      CG_TRY(cols(p));
    } else {
      CG_TRY(cols(p));
      CG_TRY(rows(p));
    }
  }
  return CG_OK;
}

static int64_t nh_of(const Geom& g) { return (int64_t)g.nhx * g.nhy * g.nhz; }

// one-plane 2-D transform used by the memory-limited mode
static int fft_one_plane(cg_plan_s* P, void* d_plane, int direction) {
  const Geom& g = P->geom;
  if (!P->fft1_valid || P->fft1_nf1 != g.nf1 || P->fft1_nf2 != g.nf2) {
    if (P->fft1_valid) cufftDestroy(P->fft1);
    P->fft1_valid = false;
    CG_CUFFT(cufftPlan2d(&P->fft1, g.nf2, g.nf1,
                         P->precision == CG_PREC_FP64 ? CUFFT_Z2Z : CUFFT_C2C));
    P->fft1_valid = true;
    P->fft1_nf1 = g.nf1;
    P->fft1_nf2 = g.nf2;
  }
  return exec_c2c(P, P->fft1, d_plane, direction);
}

// Memory-limited ms2dirty after the sorted stream: per plane window, spread
// the window's taps, transform its planes and add its share of the w-DFT to
// an FP64 accumulator image; the per-pixel corrections come last.
template <typename T>
static int ms2dirty_windows(cg_plan_s* P, T* d_dirty) {
  const Geom& g = P->geom;
  cudaStream_t st = P->stream;
  const size_t plane = (size_t)g.nf1 * g.nf2;
  const size_t npix = (size_t)g.N1 * g.N2;
  CG_TRY(ensure(P->acc, npix * 16));
  CG_CUDA(cudaMemsetAsync(P->acc.p, 0, npix * 16, st));
  T* fwb = (T*)P->grid.p;
  for (int p0 = 0; p0 < g.nw; p0 += P->plane_batch) {
    const int p1 = std::min(g.nw, p0 + P->plane_batch);
    CG_TRY(launch_grid_window<T>((const Rec<T>*)P->recs.p, P->nrow, g, p0, p1, fwb, st));
    for (int p = p0; p < p1; p++) CG_TRY(fft_one_plane(P, fwb + 2 * (p - p0) * plane, CUFFT_INVERSE));
    CG_TRY(launch_wdft_window<T>(fwb, g, p0, p1, (const double*)P->zq.p, (double*)P->acc.p, st));
  }
  return launch_wdft_finish<T>((const double*)P->acc.p, g, (const double*)P->K1.p,
                               (const double*)P->K2.p, (const double*)P->K3q.p,
                               (const double*)P->zq.p, d_dirty, st);
}

// Memory-limited dirty2ms after the sorted stream: per plane window, fill,
// transform and add each row's window share into vis (zeroed first).
template <typename T>
static int dirty2ms_windows(cg_plan_s* P, const T* d_dirty, T* d_vis) {
  const Geom& g = P->geom;
  cudaStream_t st = P->stream;
  const size_t plane = (size_t)g.nf1 * g.nf2;
  CG_CUDA(cudaMemsetAsync(d_vis, 0, (size_t)P->nrow * 2 * sizeof(T), st));
  T* fwb = (T*)P->grid.p;
  for (int p0 = 0; p0 < g.nw; p0 += P->plane_batch) {
    const int p1 = std::min(g.nw, p0 + P->plane_batch);
    CG_TRY(launch_plane_fill_window<T>(d_dirty, g, p0, p1, (const double*)P->K1.p,
                                       (const double*)P->K2.p, (const double*)P->K3q.p,
                                       (const double*)P->zq.p, fwb, st));
    for (int p = p0; p < p1; p++) CG_TRY(fft_one_plane(P, fwb + 2 * (p - p0) * plane, CUFFT_FORWARD));
    CG_TRY(launch_degrid_window<T>((const Rec<T>*)P->recs.p, (const int*)P->perm.p, P->nrow, g,
                                   p0, p1, fwb, d_vis, st));
  }
  return CG_OK;
}

// Autotuning: on the first call per direction for a geometry, time every
// candidate tiling of the spreading (dir 0) or interpolation (dir 1) launch
// -- each launch rewrites its whole output, so the repeats are harmless --
// and keep the fastest in P->tune.
template <typename T>
static int autotune_launch(cg_plan_s* P, int dir, T* d_vis) {
  const Geom& g = P->geom;
  const int key[4] = {g.nf1, g.nf2, g.nw, g.kw};
  if (!P->autotune || P->grid_method != kGridTiled ||
      std::equal(key, key + 4, P->tuned_key[dir]))
    return CG_OK;
  cudaStream_t st = P->stream;
  const SplitScratch split{&P->split_chunks, &P->split_sums, &P->split_parts};
  auto launch = [&](const TileTune& tt) {
    return dir == 0 ? launch_grid<T>((const Rec<T>*)P->recs.p, (const int*)P->hive_start.p,
                                     P->nrow, g, (T*)P->grid.p, P->grid_method,
                                     queue_counter(P), st, &tt, &split)
                    : degrid_dispatch<T>(P, tt, d_vis);
  };
  cudaEvent_t e0, e1;
  CG_CUDA(cudaEventCreate(&e0));
  CG_CUDA(cudaEventCreate(&e1));
  const int (*cand)[4] = nullptr;
  const int ncand = tile_candidates(dir, &cand);
  float best = -1.f;
  TileTune best_tt = P->tune;
  int rc = CG_OK;
  for (int c = 0; c < ncand && rc == CG_OK; c++) {
    TileTune tt = P->tune;
    set_tile_candidate(tt, dir, cand[c]);
    float ms = 0.f;
    bool ok = true;
    for (int rep = 0; rep < 2 && ok && rc == CG_OK; rep++) {  // the first launch warms up
      if (cudaEventRecord(e0, st) != cudaSuccess) rc = CG_ERR_CUDA;
      ok = launch(tt) == CG_OK;
      if (cudaEventRecord(e1, st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
          cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
        rc = CG_ERR_CUDA;
    }
    if (!ok) {  // a tiling that does not fit on an SM launched nothing
      cudaGetLastError();
      continue;
    }
    if (best < 0.f || ms < best) {
      best = ms;
      best_tt = tt;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != CG_OK) {
    set_last_error("autotuning: CUDA event failure");
    return rc;
  }
  P->tune = best_tt;
  P->tuned_ms[dir] = std::max(best, 0.f);
  std::copy(key, key + 4, P->tuned_key[dir]);
  return CG_OK;
}

// host entry points: wait for the inputs copied on the second stream (all
// of them; or, main_only, the visibilities / the image)
static int wait_inputs(cg_plan_s* P, bool main_only = false) {
  cudaEvent_t e = main_only && P->main_ready ? P->main_ready : P->inputs_ready;
  if (e) CG_CUDA(cudaStreamWaitEvent(P->stream, e, 0));
  return CG_OK;
}
// host entry points: wait for uvw (before the binning)
static int wait_uvw(cg_plan_s* P) {
  if (P->uvw_ready) CG_CUDA(cudaStreamWaitEvent(P->stream, P->uvw_ready, 0));
  return CG_OK;
}

// the stages after gridding: FFT, then w-DFT with the corrections
template <typename T>
static int ms2dirty_tail(cg_plan_s* P, T* d_dirty) {
  const Geom& g = P->geom;
  CG_TRY(fft_exec_pruned(P, P->grid.p, CUFFT_INVERSE));
  timer_mark(P);  // 5: FFT
  if (P->stop_stage == 3) return CG_OK;
  CG_TRY(launch_wdft_deconv<T>((const T*)P->grid.p, g, (const double*)P->K1.p,
                               (const double*)P->K2.p, (const double*)P->K3q.p,
                               (const double*)P->zq.p, d_dirty, P->stream));
  timer_mark(P);  // 6: w-DFT + corrections
  return CG_OK;
}

// part 0: the whole call; 1: the stages before gridding; 2: those after it
// Quarter tables of the call's geometry; a call whose geometry equals the
// last one's (same image, pixel sizes, w shift and scales, quadrature) finds
// them already in place.
static int quarter_tables(cg_plan_s* P, cudaStream_t st) {
  const Geom& g = P->geom;
  const double key[7] = {(double)g.N1, (double)g.N2, g.pixx, g.pixy, g.o_center, g.gamma, g.h};
  if (P->quarter_valid && std::equal(key, key + 7, P->quarter_key)) return CG_OK;
  CG_TRY(launch_quarter(g, P->quad, (double*)P->K3q.p, (double*)P->zq.p, st));
  std::copy(key, key + 7, P->quarter_key);
  P->quarter_valid = true;
  return CG_OK;
}

template <typename T>
static int ms2dirty_t(cg_plan_s* P, const double* d_uvw, const T* d_vis, const T* d_wgt,
                      T* d_dirty, bool reuse, int part = 0) {
  if (part == 2) return ms2dirty_tail<T>(P, d_dirty);
  const Geom& g = P->geom;
  cudaStream_t st = P->stream;
  int64_t M = P->nrow;
  timer_mark(P);  // stage 0: w range + geometry
  if (!reuse) CG_TRY(quarter_tables(P, st));
  timer_mark(P);  // 1: quarter tables
  if (!reuse) {
    CG_TRY(wait_uvw(P));
    CG_TRY(launch_bin(d_uvw, M, g, P->key_bytes, P->binws.p, P->binws.cap, (int*)P->perm.p,
                      P->skeys.p, (int*)P->hive_start.p, st,
                      (int*)P->hive_start.p + (nh_of(g) + 1)));
  }
  timer_mark(P);  // 2: binning
  if (P->stop_stage == 1) return CG_OK;
  CG_TRY(wait_inputs(P));
  CG_TRY(launch_build_stream<T>((const int*)P->perm.p, M, d_uvw, d_vis, d_wgt, g, true,
                                (Rec<T>*)P->recs_tmp.p, (Rec<T>*)P->recs.p, st));
  timer_mark(P);  // 3: sorted stream
  if (P->plane_batch) {  // memory-limited mode: gridding, FFT and w-DFT per plane window
    CG_TRY(ms2dirty_windows<T>(P, d_dirty));
    timer_mark(P);  // 4: gridding (all windows)
    timer_mark(P);  // 5: FFT (inside the windows)
    timer_mark(P);  // 6
    return CG_OK;
  }
  if (part == 1) return CG_OK;
  CG_TRY(autotune_launch<T>(P, 0, (T*)nullptr));
  Geom gg = g;
  if (P->stop_stage != 0) gg.grid_skip = 0;  // the grid is inspected: every row written
  const SplitScratch split{&P->split_chunks, &P->split_sums, &P->split_parts};
  CG_TRY(launch_grid<T>((const Rec<T>*)P->recs.p, (const int*)P->hive_start.p, M, gg,
                        (T*)P->grid.p, P->grid_method, queue_counter(P), st, &P->tune, &split));
  timer_mark(P);  // 4: gridding
  if (P->stop_stage == 2) return CG_OK;
  return ms2dirty_tail<T>(P, d_dirty);
}

// part 0: the whole call; 1: the stages before degridding
template <typename T>
static int speculate_t(cg_plan_s* P, const T* d_dirty) {
  const Geom& g = P->geom;
  CG_CUDA(cudaStreamWaitEvent(P->aux_stream, P->main_ready, 0));  // the image
  cudaStream_t st = P->stream;
  P->stream = P->aux_stream;  // the FFT helpers launch on P->stream
  int rc = launch_plane_fill<T>(d_dirty, g, (const double*)P->K1.p, (const double*)P->K2.p,
                                (const double*)P->K3q.p, (const double*)P->zq.p, (T*)P->grid.p,
                                P->aux_stream);
  if (rc == CG_OK) rc = fft_exec_pruned(P, P->grid.p, CUFFT_FORWARD);
  P->stream = st;
  CG_TRY(rc);
  CG_CUDA(cudaEventRecord(P->aux_ev1, P->aux_stream));
  P->spec_pending = true;
  return CG_OK;
}

int dirty2ms_speculate(cg_plan_s* P, int64_t nrow, double freq, const void* d_dirty) {
  P->spec_pending = false;
  P->spec_hit = false;
  // the geometry, its quarter tables and the grid of the last call, which had
  // this call's rows and frequency
  if (!P->spec_valid || !P->quarter_valid || nrow <= 0 || nrow != P->spec_nrow ||
      freq != P->spec_freq || P->plane_batch || P->stop_stage || P->timer.on || !P->aux_stream ||
      !P->main_ready || !P->grid.p || P->fixed_uvw)
    return CG_OK;
  return P->precision == CG_PREC_FP64 ? speculate_t<double>(P, (const double*)d_dirty)
                                      : speculate_t<float>(P, (const float*)d_dirty);
}

template <typename T>
static int dirty2ms_t(cg_plan_s* P, const double* d_uvw, const T* d_dirty, const T* d_wgt,
                      T* d_vis, bool reuse, int part = 0) {
  const Geom& g = P->geom;
  cudaStream_t st = P->stream;
  int64_t M = P->nrow;
  timer_mark(P);  // stage 0: w range + geometry
  if (!reuse) CG_TRY(quarter_tables(P, st));
  timer_mark(P);  // 1: quarter tables
  if (P->spec_hit) {
    // the plane fill and FFT of this very geometry already run on aux_stream
    // (dirty2ms_speculate); uvw is in (the range pass waited for it)
    P->spec_hit = false;
    CG_TRY(launch_bin(d_uvw, M, g, P->key_bytes, P->binws.p, P->binws.cap, (int*)P->perm.p,
                      P->skeys.p, (int*)P->hive_start.p, st,
                      (int*)P->hive_start.p + (nh_of(g) + 1)));
    CG_TRY(wait_inputs(P));  // the weights
    CG_TRY(launch_build_stream<T>((const int*)P->perm.p, M, d_uvw, (const T*)nullptr, d_wgt, g,
                                  false, (Rec<T>*)P->recs_tmp.p, (Rec<T>*)P->recs.p, st));
    CG_CUDA(cudaStreamWaitEvent(st, P->aux_ev1, 0));  // the transformed grid
    CG_TRY(autotune_launch<T>(P, 1, d_vis));
    CG_TRY(degrid_dispatch<T>(P, P->tune, d_vis));
    return CG_OK;
  }
  // Host entry points whose ranges came from the host: the plane fill and
  // the FFT need only the image and the geometry, so they run on aux_stream
  // as soon as the image is in, while this stream waits for uvw, bins the
  // rows and builds the stream; degridding waits for both.
  if (P->host_mm && P->main_ready && P->aux_stream && !P->plane_batch && !P->stop_stage &&
      !P->timer.on && part == 0 && !reuse) {
    CG_CUDA(cudaEventRecord(P->aux_ev0, st));  // the quarter tables
    CG_CUDA(cudaStreamWaitEvent(P->aux_stream, P->aux_ev0, 0));
    CG_CUDA(cudaStreamWaitEvent(P->aux_stream, P->main_ready, 0));  // the image
    P->stream = P->aux_stream;  // the FFT helpers launch on P->stream
    int rc = launch_plane_fill<T>(d_dirty, g, (const double*)P->K1.p, (const double*)P->K2.p,
                                  (const double*)P->K3q.p, (const double*)P->zq.p, (T*)P->grid.p,
                                  P->aux_stream);
    if (rc == CG_OK) rc = fft_exec_pruned(P, P->grid.p, CUFFT_FORWARD);
    P->stream = st;
    CG_TRY(rc);
    CG_CUDA(cudaEventRecord(P->aux_ev1, P->aux_stream));
    CG_TRY(wait_uvw(P));
    CG_TRY(launch_bin(d_uvw, M, g, P->key_bytes, P->binws.p, P->binws.cap, (int*)P->perm.p,
                      P->skeys.p, (int*)P->hive_start.p, st,
                      (int*)P->hive_start.p + (nh_of(g) + 1)));
    CG_TRY(wait_inputs(P));  // the weights
    CG_TRY(launch_build_stream<T>((const int*)P->perm.p, M, d_uvw, (const T*)nullptr, d_wgt, g,
                                  false, (Rec<T>*)P->recs_tmp.p, (Rec<T>*)P->recs.p, st));
    CG_CUDA(cudaStreamWaitEvent(st, P->aux_ev1, 0));  // the transformed grid
    CG_TRY(autotune_launch<T>(P, 1, d_vis));
    CG_TRY(degrid_dispatch<T>(P, P->tune, d_vis));
    return CG_OK;
  }
  if (!reuse) {
    CG_TRY(wait_uvw(P));
    CG_TRY(launch_bin(d_uvw, M, g, P->key_bytes, P->binws.p, P->binws.cap, (int*)P->perm.p,
                      P->skeys.p, (int*)P->hive_start.p, st,
                      (int*)P->hive_start.p + (nh_of(g) + 1)));
  }
  timer_mark(P);  // 2: binning
  if (P->stop_stage == 1) return CG_OK;
  CG_TRY(wait_inputs(P, P->plane_batch == 0));  // the image (the weights before the stream)
  if (P->plane_batch) {  // memory-limited mode: fill, FFT and degridding per plane window
    CG_TRY(launch_build_stream<T>((const int*)P->perm.p, M, d_uvw, (const T*)nullptr, d_wgt, g,
                                  false, (Rec<T>*)P->recs_tmp.p, (Rec<T>*)P->recs.p, st));
    CG_TRY(dirty2ms_windows<T>(P, d_dirty, d_vis));
    for (int i = 0; i < 4; i++) timer_mark(P);  // stages 3-6 are inside the windows
    return CG_OK;
  }
  CG_TRY(launch_plane_fill<T>(d_dirty, g, (const double*)P->K1.p, (const double*)P->K2.p,
                              (const double*)P->K3q.p, (const double*)P->zq.p, (T*)P->grid.p, st));
  timer_mark(P);  // 3: plane fill
  if (P->stop_stage == 2) return CG_OK;
  CG_TRY(fft_exec_pruned(P, P->grid.p, CUFFT_FORWARD));
  timer_mark(P);  // 4: FFT
  if (P->stop_stage == 3) return CG_OK;
  CG_TRY(wait_inputs(P));  // the weights
  CG_TRY(launch_build_stream<T>((const int*)P->perm.p, M, d_uvw, (const T*)nullptr, d_wgt, g,
                                false, (Rec<T>*)P->recs_tmp.p, (Rec<T>*)P->recs.p, st));
  timer_mark(P);  // 5: sorted stream
  if (part == 1) return CG_OK;
  CG_TRY(autotune_launch<T>(P, 1, d_vis));
  CG_TRY(degrid_dispatch<T>(P, P->tune, d_vis));
  timer_mark(P);  // 6: degridding
  return CG_OK;
}

// Status of the TMA-staged degridding launched on the plan's stream: waits
// for the stream, reads and clears the error word.  CG_ERR_CUDA when a
// staging wait ran out (that call's visibilities are incomplete).
int tma_status(cg_plan_s* P) {
  if (!P->tma_armed) return CG_OK;
  CG_CUDA(cudaMemcpyAsync(P->h_mm + 9, tma_error_word(P), sizeof(int), cudaMemcpyDeviceToHost,
                          P->stream));
  CG_CUDA(cudaStreamSynchronize(P->stream));
  if (*(const int*)(P->h_mm + 9)) {
    CG_CUDA(cudaMemsetAsync(tma_error_word(P), 0, sizeof(int), P->stream));
    CG_CUDA(cudaStreamSynchronize(P->stream));
    set_last_error("degridding: a TMA staging wait timed out; the visibilities are incomplete");
    return CG_ERR_CUDA;
  }
  return CG_OK;
}

// fixed-uvw mode: the last call's geometry and binning still describe this one
static bool reuse_geometry(const cg_plan_s* P, int64_t nrow, double freq, const double* d_uvw) {
  return P->fixed_uvw && P->bins_valid && !P->timer.on && P->stop_stage == 0 &&
         P->last_uvw == d_uvw && P->last_nrow == nrow && P->last_freq == freq;
}
static void remember_geometry(cg_plan_s* P, int64_t nrow, double freq, const double* d_uvw) {
  P->bins_valid = P->fixed_uvw && P->stop_stage == 0;
  P->last_uvw = d_uvw;
  P->last_nrow = nrow;
  P->last_freq = freq;
}

// A call can be split at its spreading step (batched solves): true when the
// plan's mode has that step as one tiled launch over resident planes.
static bool splittable(const cg_plan_s* P) {
  return !P->plane_batch && P->grid_method == kGridTiled && !P->timer.on && P->stop_stage == 0;
}

static int ms2dirty_run(cg_plan_s* P, int part, int64_t nrow, double freq, const double* d_uvw,
                        const void* d_vis, const void* d_wgt, void* d_dirty, bool* split) {
  const bool fp64 = P->precision == CG_PREC_FP64;
  if (part == 2) {
    CG_CUDA(cudaSetDevice(P->device));
    const int st = fp64 ? ms2dirty_t<double>(P, d_uvw, nullptr, nullptr, (double*)d_dirty, true, 2)
                        : ms2dirty_t<float>(P, d_uvw, nullptr, nullptr, (float*)d_dirty, true, 2);
    return st != CG_OK ? st : P->eps_status;
  }
  if (split) *split = false;
  if (!d_dirty || (nrow > 0 && (!d_uvw || !d_vis))) {
    set_last_error("null pointer");
    return CG_ERR_ARG;
  }
  CG_CUDA(cudaSetDevice(P->device));
  const bool reuse = reuse_geometry(P, nrow, freq, d_uvw);
  CG_TRY(timer_begin(P, 0));
  if (!reuse) CG_TRY(prepare(P, nrow, freq, d_uvw));
  size_t tsz = fp64 ? 8 : 4;
  if (nrow == 0) {
    CG_CUDA(cudaMemsetAsync(d_dirty, 0, (size_t)P->nx * P->ny * 2 * tsz, P->stream));
    remember_geometry(P, nrow, freq, d_uvw);
    return P->eps_status;
  }
  if (part == 1 && !splittable(P)) part = 0;
  if (split) *split = part == 1;
  int st = fp64 ? ms2dirty_t<double>(P, d_uvw, (const double*)d_vis, (const double*)d_wgt, (double*)d_dirty, reuse, part)
                : ms2dirty_t<float>(P, d_uvw, (const float*)d_vis, (const float*)d_wgt, (float*)d_dirty, reuse, part);
  if (st == CG_OK) remember_geometry(P, nrow, freq, d_uvw);
  return st != CG_OK ? st : P->eps_status;
}

static int dirty2ms_run(cg_plan_s* P, int part, int64_t nrow, double freq, const double* d_uvw,
                        const void* d_dirty, const void* d_wgt, void* d_vis, bool* split) {
  if (split) *split = false;
  if (!d_dirty || (nrow > 0 && (!d_uvw || !d_vis))) {
    set_last_error("null pointer");
    return CG_ERR_ARG;
  }
  CG_CUDA(cudaSetDevice(P->device));
  const bool reuse = reuse_geometry(P, nrow, freq, d_uvw);
  CG_TRY(timer_begin(P, 1));
  if (!reuse) CG_TRY(prepare(P, nrow, freq, d_uvw));
  if (nrow == 0) {
    remember_geometry(P, nrow, freq, d_uvw);
    return P->eps_status;
  }
  if (part == 1 && !splittable(P)) part = 0;
  if (split) *split = part == 1;
  int st = (P->precision == CG_PREC_FP64)
               ? dirty2ms_t<double>(P, d_uvw, (const double*)d_dirty, (const double*)d_wgt, (double*)d_vis, reuse, part)
               : dirty2ms_t<float>(P, d_uvw, (const float*)d_dirty, (const float*)d_wgt, (float*)d_vis, reuse, part);
  if (st == CG_OK) remember_geometry(P, nrow, freq, d_uvw);
  // a call that is not being captured reports a timed-out TMA staging wait
  // itself (one more stream synchronization, only when the TMA kernel ran)
  if (st == CG_OK && part == 0 && P->tma_armed) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CG_CUDA(cudaStreamIsCapturing(P->stream, &cs));
    if (cs == cudaStreamCaptureStatusNone) st = tma_status(P);
  }
  return st != CG_OK ? st : P->eps_status;
}

int ms2dirty_device(cg_plan_s* P, int64_t nrow, double freq, const double* d_uvw,
                    const void* d_vis, const void* d_wgt, void* d_dirty) {
  return ms2dirty_run(P, 0, nrow, freq, d_uvw, d_vis, d_wgt, d_dirty, nullptr);
}

int dirty2ms_device(cg_plan_s* P, int64_t nrow, double freq, const double* d_uvw,
                    const void* d_dirty, const void* d_wgt, void* d_vis) {
  return dirty2ms_run(P, 0, nrow, freq, d_uvw, d_dirty, d_wgt, d_vis, nullptr);
}

int ms2dirty_split(cg_plan_s* P, int part, int64_t nrow, double freq, const double* d_uvw,
                   const void* d_vis, const void* d_wgt, void* d_dirty, bool* split) {
  return ms2dirty_run(P, part, nrow, freq, d_uvw, d_vis, d_wgt, d_dirty, split);
}

int dirty2ms_split(cg_plan_s* P, int64_t nrow, double freq, const double* d_uvw,
                   const void* d_dirty, const void* d_wgt, void* d_vis, bool* split) {
  return dirty2ms_run(P, 1, nrow, freq, d_uvw, d_dirty, d_wgt, d_vis, split);
}

template <typename T>
int plan_grid_job(const cg_plan_s* P, const TileTune& tt, T* d_vis, GridJob<T>* job) {
  const Geom& g = P->geom;
  GridJob<T> J{};
  J.recs = (const Rec<T>*)P->recs.p;
  J.hive_start = (const int*)P->hive_start.p;
  J.perm = (const int*)P->perm.p;
  J.fw = (T*)P->grid.p;
  J.vis = d_vis;
  J.M = P->nrow;
  J.g = g;
  J.wt = warp_tiling<T>(g, &tt);
  // x-sliding windows for a tuning candidate with wx < 0, or CG_GRID_SLIDE=1
  // (as for a single plan); st.TY = 0 where they do not apply
  J.st = SlideTile{};
  const char* sl = getenv("CG_GRID_SLIDE");
  if ((tt.wx < 0 || (sl && atoi(sl) != 0)) && !slide_tiling(g, sizeof(T), &tt, J.st))
    J.st = SlideTile{};
  J.dt = grid_tiling<T>(g, true, &tt);
  J.nslots = degrid_slots(J.dt, g.kw);
  *job = J;
  return CG_OK;
}
template int plan_grid_job<float>(const cg_plan_s*, const TileTune&, float*, GridJob<float>*);
template int plan_grid_job<double>(const cg_plan_s*, const TileTune&, double*, GridJob<double>*);

}  // namespace cg
