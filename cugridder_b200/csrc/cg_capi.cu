// extern "C" entry points of libcugridder.so.
//
// The eight reference-compatible functions (reference include/cugridder.h:37-47,
// src/astro/cugridder.cu:541-571) take HOST pointers and are synchronous, as in
// the reference.  Unlike the reference, which mallocs, copies and frees every
// device buffer and cuFFT plan inside each call (cugridder.cu:309-388), they
// share one cached plan per precision so repeated calls reuse HBM workspace;
// cg_release_cache() frees it.  Errors are returned, never exit()ed.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <limits>
#include <sched.h>
#include <string>
#include <condition_variable>
#include <functional>
#include <thread>
#include <vector>

#include "cg_plan.cuh"

#include <atomic>

namespace cg {
static thread_local std::string g_last_error;
void set_last_error(const char* msg) { g_last_error = msg ? msg : ""; }
static std::atomic<long long> g_launches{0};
void count_launches(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

cudaError_t kernel_occupancy(const void* func, int threads, size_t smem, int* per_sm) {
  struct Key {
    const void* f;
    int t;
    size_t s;
    int dev;
    bool operator<(const Key& o) const {
      return f != o.f ? f < o.f : t != o.t ? t < o.t : s != o.s ? s < o.s : dev < o.dev;
    }
  };
  static std::mutex mu;
  static std::map<Key, int> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  const Key k{func, threads, smem, dev};
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(k);
    if (it != cache.end()) {
      *per_sm = it->second;
      return cudaSuccess;
    }
  }
  std::lock_guard<std::mutex> lk(mu);
  // the opt-in only ever grows: every launch shape cached before stays valid
  static std::map<std::pair<const void*, int>, size_t> opt_in;
  size_t& cur = opt_in[{func, dev}];
  if (smem > 48 * 1024 && smem > cur) {
    const cudaError_t e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    cur = smem;
  }
  int n = 0;
  const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, func, threads, smem);
  if (e != cudaSuccess) return e;
  cache[k] = n;
  *per_sm = n;
  return cudaSuccess;
}
}  // namespace cg

using cg::ensure;

namespace {

std::mutex g_cache_mu;
cg_plan_s* g_cache[2] = {nullptr, nullptr};

// gridding kernel of the host-pointer entry points (cg_set_host_kernel)
struct HostKernel {
  int kind = CG_KERNEL_ES;
  int w = 0;  // ES: forced width (0 = from epsilon); POLY: width
  double poly[cg::kMaxW * cg::kPolyCoef] = {};
} g_host_kernel;

// bring a cached plan's kernel in line with g_host_kernel (caller holds g_cache_mu)
void apply_host_kernel(cg_plan_s* P) {
  const HostKernel& k = g_host_kernel;
  const bool poly = k.kind == CG_KERNEL_POLY;
  const bool same = P->kernel_kind == k.kind &&
                    (poly ? (P->poly_w == k.w &&
                             memcmp(P->poly, k.poly, sizeof(double) * k.w * cg::kPolyCoef) == 0)
                          : P->es_w == k.w);
  if (same) return;
  P->kernel_kind = k.kind;
  if (poly) {
    P->poly_w = k.w;
    memcpy(P->poly, k.poly, sizeof(k.poly));
  } else {
    P->es_w = k.w;
  }
  P->kw = 0;  // reconfigure on the next plan_configure
}

int ensure_device() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    cg::set_last_error("no CUDA device");
    return CG_ERR_NOGPU;
  }
  return CG_OK;
}

void destroy_plan(cg_plan_s* P) {
  if (!P) return;
  cudaSetDevice(P->device);
  if (P->fft_valid) cufftDestroy(P->fft);
  if (P->rows_valid) cufftDestroy(P->fft_rows);
  if (P->cols_valid) cufftDestroy(P->fft_cols);
  if (P->fft1_valid) cufftDestroy(P->fft1);
  cg_dev_buf* bs[] = {&P->mm,   &P->K1,    &P->K2,     &P->K3q,    &P->zq,     &P->grid,
                      &P->recs, &P->perm,  &P->skeys,  &P->hive_start, &P->binws, &P->fftwork,
                      &P->io_uvw, &P->io_vis, &P->io_wgt, &P->io_dirty, &P->polyf, &P->polyd, &P->recs_tmp,
                      &P->chan_uvw, &P->chan_scale, &P->coltw, &P->acc, &P->roots,
                      &P->split_chunks, &P->split_sums, &P->split_parts};
  for (auto b : bs) cg::release(*b);
  if (P->h_mm) cudaFreeHost(P->h_mm);
  if (P->io_stream) cudaStreamDestroy(P->io_stream);
  if (P->io_event) cudaEventDestroy(P->io_event);
  if (P->aux_stream) cudaStreamDestroy(P->aux_stream);
  if (P->aux_ev0) cudaEventDestroy(P->aux_ev0);
  if (P->aux_ev1) cudaEventDestroy(P->aux_ev1);
  if (P->io_ev_uvw) cudaEventDestroy(P->io_ev_uvw);
  if (P->io_ev_main) cudaEventDestroy(P->io_ev_main);
  if (P->timer.created)
    for (int s = 0; s < 2; s++)
      for (int i = 0; i <= kMaxStages; i++) cudaEventDestroy(P->timer.ev[s][i]);
  delete P;
}

cg_plan_s* cached_plan(int precision, int& status) {
  status = ensure_device();
  if (status) return nullptr;
  cg_plan_s*& P = g_cache[precision];
  int dev = 0;
  cudaGetDevice(&dev);
  if (P && P->device != dev) {
    destroy_plan(P);
    P = nullptr;
  }
  if (!P) {
    P = new cg_plan_s();
    P->device = dev;
    P->stream = nullptr;
    // the reference-compatible calls cannot reach cg_plan_set_autotune, and
    // their cached plan serves every later call of the same geometry: tune
    // on the first call (CG_AUTOTUNE=0 turns it off)
    P->autotune = 1;
    if (const char* m = getenv("CG_AUTOTUNE")) P->autotune = atoi(m) != 0;
    if (const char* m = getenv("CG_DEGRID_TMA")) P->tma_default = atoi(m);
  }
  return P;
}

__global__ void k_widen_uvw(const float* __restrict__ in, double* __restrict__ out, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (double)in[i];
}

// Multi-channel rows: row r of channel c is the visibility at frequency f_c.
// Its phase 2 pi f_c/c (u l + v m + w (n-1)) equals that of a row with
// uvw * (f_c / f_0) at frequency f_0, so the channels are flattened into
// nrow * nchan rows (index r * nchan + c, the layout of vis[nrow][nchan]) of
// one call at f_0 = freqs[0]; channel 0 keeps its coordinates bit for bit.
__global__ void k_expand_chan(const double* __restrict__ uvw, int64_t nrow, int nchan,
                              const double* __restrict__ scale, double* __restrict__ out) {
  const int64_t n = nrow * nchan;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = q / nchan;
    const double s = scale[q - r * nchan];
#pragma unroll
    for (int k = 0; k < 3; k++) out[3 * q + k] = uvw[3 * r + k] * s;
  }
}

int expand_channels(cg_plan_s* P, int64_t nrow, int nchan, const double* freqs,
                    const double* d_uvw, const double** d_out) {
  if (nchan < 1 || !freqs || nrow < 0) {
    cg::set_last_error("nchan must be >= 1 with nchan frequencies");
    return CG_ERR_ARG;
  }
  if (nrow * (int64_t)nchan > 2147483647LL) {
    cg::set_last_error("nrow * nchan out of range");
    return CG_ERR_SIZE;
  }
  std::vector<double> sc(nchan);
  for (int c = 0; c < nchan; c++) {
    if (!(freqs[c] > 0.0) || !std::isfinite(freqs[c])) {
      cg::set_last_error("frequencies must be positive and finite");
      return CG_ERR_ARG;
    }
    sc[c] = c == 0 ? 1.0 : freqs[c] / freqs[0];
  }
  if (nchan == 1 || nrow == 0) {
    *d_out = d_uvw;
    return CG_OK;
  }
  CG_TRY(ensure(P->chan_scale, sizeof(double) * nchan));
  CG_TRY(ensure(P->chan_uvw, sizeof(double) * 3 * (size_t)nrow * nchan));
  CG_CUDA(cudaMemcpyAsync(P->chan_scale.p, sc.data(), sizeof(double) * nchan,
                          cudaMemcpyHostToDevice, P->stream));
  int64_t n = nrow * nchan;
  int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
  k_expand_chan<<<blocks, 256, 0, P->stream>>>(d_uvw, nrow, nchan, (const double*)P->chan_scale.p,
                                                (double*)P->chan_uvw.p);
  cg::count_launches(1);
  CG_CUDA(cudaGetLastError());
  *d_out = (const double*)P->chan_uvw.p;
  return CG_OK;
}

// order-preserving integer key of a double (the device's ordered_key)
unsigned long long ordered_key_host(double x) {
  unsigned long long b;
  memcpy(&b, &x, sizeof(b));
  return (b & 0x8000000000000000ULL) ? ~b : (b | 0x8000000000000000ULL);
}

// The u, v, w ranges and the non-finite flag of the caller's uvw ([nrow][3],
// float or double) computed on the host, in the layout launch_wminmax writes
// (order-preserving keys of u_min, u_max, v_min, v_max, w_min, w_max, then
// the flag): min and max are exact, so the values equal the device pass's.
// Threads split the rows; it runs while the DMA engine copies the inputs.
template <typename F>
void scan_uvw_host(const F* uvw, int64_t nrow, unsigned long long out[7]) {
  struct Part {
    double lo[3], hi[3];
    int bad;
  };
  // Branch-free compares (a NaN never replaces a bound, as fmin/fmax) and
  // one running sum of x - x, which is NaN as soon as any x is not finite:
  // this loop vectorizes, where fmin / isfinite per element do not.
  auto scan = [&](int64_t r0, int64_t r1, Part& p) {
    double lo0 = std::numeric_limits<double>::max(), lo1 = lo0, lo2 = lo0;
    double hi0 = -lo0, hi1 = -lo0, hi2 = -lo0, acc = 0.0;
    for (int64_t i = r0; i < r1; i++) {
      const double x0 = (double)uvw[3 * i], x1 = (double)uvw[3 * i + 1], x2 = (double)uvw[3 * i + 2];
      acc += (x0 - x0) + (x1 - x1) + (x2 - x2);
      lo0 = x0 < lo0 ? x0 : lo0;
      hi0 = x0 > hi0 ? x0 : hi0;
      lo1 = x1 < lo1 ? x1 : lo1;
      hi1 = x1 > hi1 ? x1 : hi1;
      lo2 = x2 < lo2 ? x2 : lo2;
      hi2 = x2 > hi2 ? x2 : hi2;
    }
    p.lo[0] = lo0; p.lo[1] = lo1; p.lo[2] = lo2;
    p.hi[0] = hi0; p.hi[1] = hi1; p.hi[2] = hi2;
    p.bad = !(acc == 0.0);
  };
  int ncpu = 1;
  {
    cpu_set_t cs;
    if (sched_getaffinity(0, sizeof(cs), &cs) == 0) ncpu = std::max(1, CPU_COUNT(&cs));
  }
  const int nt = nrow < (1 << 20) ? 1 : std::min(16, ncpu);
  std::vector<Part> parts(nt);
  std::vector<std::thread> th;
  for (int t = 1; t < nt; t++)
    th.emplace_back(scan, nrow * t / nt, nrow * (t + 1) / nt, std::ref(parts[t]));
  scan(0, nrow / nt, parts[0]);
  for (auto& x : th) x.join();
  Part r = parts[0];
  for (int t = 1; t < nt; t++) {
    for (int a = 0; a < 3; a++) {
      r.lo[a] = parts[t].lo[a] < r.lo[a] ? parts[t].lo[a] : r.lo[a];
      r.hi[a] = parts[t].hi[a] > r.hi[a] ? parts[t].hi[a] : r.hi[a];
    }
    r.bad |= parts[t].bad;
  }
  for (int a = 0; a < 3; a++) {
    out[2 * a] = nrow > 0 ? ordered_key_host(r.lo[a]) : ~0ULL;
    out[2 * a + 1] = nrow > 0 ? ordered_key_host(r.hi[a]) : 0ULL;
  }
  out[6] = (unsigned long long)(r.bad ? 1 : 0);
}

// ---------------------------------------------------------------- pageable host buffers
// The reference's callers (its Python binding passes numpy arrays) hand the
// host entry points ordinary pageable memory, which the DMA engine cannot
// read directly: a plain cudaMemcpyAsync then copies through the driver's
// own staging at about 10 GB/s.  Here worker threads copy each chunk into
// one of a few pinned staging buffers while the DMA engine moves the
// previous chunk, so both run at once.

// A fixed team of worker threads running one job over all of them at a time.
class CopyTeam {
 public:
  explicit CopyTeam(int n) : n_(n) {
    for (int i = 1; i < n_; i++) th_.emplace_back([this, i] { work(i); });
  }
  ~CopyTeam() {
    {
      std::lock_guard<std::mutex> lk(m_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : th_) t.join();
  }
  int size() const { return n_; }
  // fn(i) for i in [0, n), the caller running i = 0; returns when all are done
  void run(const std::function<void(int)>& fn) {
    {
      std::lock_guard<std::mutex> lk(m_);
      job_ = &fn;
      pending_ = n_ - 1;
      gen_++;
    }
    cv_.notify_all();
    fn(0);
    std::unique_lock<std::mutex> lk(m_);
    done_.wait(lk, [this] { return pending_ == 0; });
    job_ = nullptr;
  }

 private:
  void work(int i) {
    long seen = 0;
    for (;;) {
      const std::function<void(int)>* job;
      {
        std::unique_lock<std::mutex> lk(m_);
        cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen_;
        job = job_;
      }
      (*job)(i);
      std::lock_guard<std::mutex> lk(m_);
      if (--pending_ == 0) done_.notify_one();
    }
  }
  int n_;
  std::vector<std::thread> th_;
  std::mutex m_;
  std::condition_variable cv_, done_;
  const std::function<void(int)>* job_ = nullptr;
  long gen_ = 0;
  int pending_ = 0;
  bool stop_ = false;
};

int host_threads() {
  cpu_set_t cs;
  int ncpu = 1;
  if (sched_getaffinity(0, sizeof(cs), &cs) == 0) ncpu = std::max(1, CPU_COUNT(&cs));
  return std::min(16, ncpu);
}

// Pinned staging: kBufs buffers of kChunk bytes, each with the event of the
// last copy that used it.  Used by one call at a time (the caller holds
// g_cache_mu); allocated on the first pageable copy.
struct Staging {
  static constexpr size_t kChunk = 8u << 20;
  static constexpr int kBufs = 4;
  void* buf[kBufs] = {};
  cudaEvent_t ev[kBufs] = {};
  int dev = -1;
  std::unique_ptr<CopyTeam> team;
};
Staging g_staging;

int staging_ready() {
  int dev = 0;
  CG_CUDA(cudaGetDevice(&dev));
  Staging& S = g_staging;
  if (S.buf[0] && S.dev == dev) return CG_OK;
  for (int b = 0; b < Staging::kBufs; b++) {
    if (!S.buf[b]) CG_CUDA(cudaHostAlloc(&S.buf[b], Staging::kChunk, cudaHostAllocPortable));
    if (S.ev[b]) cudaEventDestroy(S.ev[b]);  // events belong to the device current at creation
    CG_CUDA(cudaEventCreateWithFlags(&S.ev[b], cudaEventDisableTiming));
  }
  S.dev = dev;
  if (!S.team) S.team.reset(new CopyTeam(host_threads()));
  return CG_OK;
}

// whole-team memcpy of n bytes
void team_copy(void* dst, const void* src, size_t n) {
  CopyTeam& T = *g_staging.team;
  const int k = T.size();
  T.run([&](int i) {
    const size_t a = n * i / k, b = n * (i + 1) / k;
    if (b > a) std::memcpy((char*)dst + a, (const char*)src + a, b - a);
  });
}

// pageable: memory the DMA engine cannot read directly (not pinned or
// registered, not device or managed memory); small copies go direct
bool staged(const void* host, size_t bytes) {
  if (bytes < (2u << 20)) return false;
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, host) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeUnregistered;
}

// host -> device on stream st; returns when the last chunk is handed to the
// DMA engine (the copies complete in stream order)
int copy_h2d(void* dst, const void* src, size_t bytes, cudaStream_t st) {
  if (!staged(src, bytes)) {
    CG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
    return CG_OK;
  }
  CG_TRY(staging_ready());
  Staging& S = g_staging;
  int k = 0;
  for (size_t off = 0; off < bytes; off += Staging::kChunk, k++) {
    const int b = k % Staging::kBufs;
    const size_t n = std::min(Staging::kChunk, bytes - off);
    CG_CUDA(cudaEventSynchronize(S.ev[b]));  // the copy that last read buffer b is done
    team_copy(S.buf[b], (const char*)src + off, n);
    CG_CUDA(cudaMemcpyAsync((char*)dst + off, S.buf[b], n, cudaMemcpyHostToDevice, st));
    CG_CUDA(cudaEventRecord(S.ev[b], st));
  }
  return CG_OK;
}

// device -> host on stream st (after the work queued on it); returns when
// every byte is in dst
int copy_d2h(void* dst, const void* src, size_t bytes, cudaStream_t st) {
  if (!staged(dst, bytes)) {
    CG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
    CG_CUDA(cudaStreamSynchronize(st));
    return CG_OK;
  }
  CG_TRY(staging_ready());
  Staging& S = g_staging;
  const size_t nchunks = (bytes + Staging::kChunk - 1) / Staging::kChunk;
  auto issue = [&](size_t k) -> int {
    const int b = (int)(k % Staging::kBufs);
    const size_t off = k * Staging::kChunk, n = std::min(Staging::kChunk, bytes - off);
    CG_CUDA(cudaMemcpyAsync(S.buf[b], (const char*)src + off, n, cudaMemcpyDeviceToHost, st));
    CG_CUDA(cudaEventRecord(S.ev[b], st));
    return CG_OK;
  };
  // keep kBufs - 1 chunks in flight ahead of the one being drained
  const size_t ahead = std::min<size_t>(nchunks, Staging::kBufs - 1);
  for (size_t k = 0; k < ahead; k++) CG_TRY(issue(k));
  for (size_t k = 0; k < nchunks; k++) {
    const int b = (int)(k % Staging::kBufs);
    const size_t off = k * Staging::kChunk, n = std::min(Staging::kChunk, bytes - off);
    if (k + ahead < nchunks) CG_TRY(issue(k + ahead));  // buffer (k + ahead) % kBufs was drained
    CG_CUDA(cudaEventSynchronize(S.ev[b]));
    team_copy((char*)dst + off, S.buf[b], n);
  }
  return CG_OK;
}

// Host-pointer driver shared by every host entry point.
// uvw_is_float: uvw given in float (reference -DSINGLE API), widened on device.
int host_call(bool to_dirty, int precision, int64_t nrow, int nx, int ny, double fov,
              double freq, const void* uvw, bool uvw_is_float, void* vis, const void* wgt,
              void* dirty, double eps, double sigma, int sign) {
  if (nrow < 0 || (nrow > 0 && (!uvw || !vis)) || !dirty) {
    cg::set_last_error("invalid argument");
    return CG_ERR_ARG;
  }
  std::lock_guard<std::mutex> lock(g_cache_mu);
  int st;
  cg_plan_s* P = cached_plan(precision, st);
  if (!P) return st;
  CG_CUDA(cudaSetDevice(P->device));
  apply_host_kernel(P);
  CG_TRY(cg::plan_configure(P, nx, ny, fov, eps, sigma, sign, precision));
  size_t tsz = precision == CG_PREC_FP64 ? 8 : 4;
  size_t n_uvw = (size_t)nrow * 3;
  CG_TRY(ensure(P->io_uvw, n_uvw * 8 + (uvw_is_float ? n_uvw * 4 : 0)));
  CG_TRY(ensure(P->io_vis, (size_t)nrow * 2 * tsz));
  CG_TRY(ensure(P->io_wgt, (size_t)nrow * tsz));
  CG_TRY(ensure(P->io_dirty, (size_t)nx * ny * 2 * tsz));
  cudaStream_t s = P->stream;
  if (!P->io_stream) {
    CG_CUDA(cudaStreamCreateWithFlags(&P->io_stream, cudaStreamNonBlocking));
    CG_CUDA(cudaStreamCreateWithFlags(&P->aux_stream, cudaStreamNonBlocking));
    CG_CUDA(cudaEventCreateWithFlags(&P->io_event, cudaEventDisableTiming));
    CG_CUDA(cudaEventCreateWithFlags(&P->io_ev_uvw, cudaEventDisableTiming));
    CG_CUDA(cudaEventCreateWithFlags(&P->io_ev_main, cudaEventDisableTiming));
    CG_CUDA(cudaEventCreateWithFlags(&P->aux_ev0, cudaEventDisableTiming));
    CG_CUDA(cudaEventCreateWithFlags(&P->aux_ev1, cudaEventDisableTiming));
  }
  cudaStream_t s2 = P->io_stream;
  // every return below leaves all streams idle (the host buffers may be
  // reused as soon as the call returns) and the plan without the waits
  struct Finish {
    cg_plan_s* P;
    ~Finish() {
      P->inputs_ready = nullptr;
      P->main_ready = nullptr;
      P->uvw_ready = nullptr;
      P->host_mm = nullptr;
      P->spec_pending = false;
      P->spec_hit = false;
      cudaStreamSynchronize(P->io_stream);
      cudaStreamSynchronize(P->aux_stream);
      cudaStreamSynchronize(P->stream);
    }
  } finish{P};
  double* d_uvw = (double*)P->io_uvw.p;
  // All copies on the second stream, one after the other at full bandwidth,
  // in the order the stages need them.  ms2dirty: uvw (binning), then the
  // visibilities and the weights (sorted stream), so the binning runs while
  // they arrive.  dirty2ms: the image first (plane fill and FFT, which need
  // nothing else), then uvw (binning), then the weights (sorted stream).
  // (The previous call left every stream idle: see Finish.)
  auto copy_uvw = [&]() -> int {
    if (nrow <= 0) return CG_OK;
    if (uvw_is_float) {
      float* d_f = (float*)(d_uvw + n_uvw);
      CG_TRY(copy_h2d(d_f, uvw, n_uvw * 4, s2));
      k_widen_uvw<<<592, 256, 0, s2>>>(d_f, d_uvw, (int64_t)n_uvw);
      cg::count_launches(1);
      CG_CUDA(cudaGetLastError());
    } else {
      CG_TRY(copy_h2d(d_uvw, uvw, n_uvw * 8, s2));
    }
    CG_CUDA(cudaEventRecord(P->io_ev_uvw, s2));
    return CG_OK;
  };
  if (to_dirty) {
    CG_TRY(copy_uvw());
    if (nrow > 0)
      CG_TRY(copy_h2d(P->io_vis.p, vis, (size_t)nrow * 2 * tsz, s2));
    CG_CUDA(cudaEventRecord(P->io_ev_main, s2));
  } else {
    CG_TRY(copy_h2d(P->io_dirty.p, dirty, (size_t)nx * ny * 2 * tsz, s2));
    CG_CUDA(cudaEventRecord(P->io_ev_main, s2));
    CG_TRY(copy_uvw());
  }
  if (nrow > 0 && wgt)
    CG_TRY(copy_h2d(P->io_wgt.p, wgt, (size_t)nrow * tsz, s2));
  CG_CUDA(cudaEventRecord(P->io_event, s2));
  P->main_ready = P->io_ev_main;
  P->inputs_ready = P->io_event;
  P->uvw_ready = nrow > 0 ? P->io_ev_uvw : nullptr;
  // dirty2ms: the u/v/w ranges from the caller's uvw while the copies run,
  // so the geometry is known before uvw is in and the plane fill and FFT
  // start as soon as the image is (ms2dirty gains nothing from it: its
  // binning waits for uvw anyway and is done before the visibilities are in)
  unsigned long long host_mm[7];
  const char* hr = getenv("CG_HOST_RANGES");  // 0: the device range pass instead (A/B timing)
  // a pageable uvw was staged before this point, so the device pass on it
  // is already possible and the host scan would only add its own time
  const bool uvw_staged = nrow > 0 && staged(uvw, n_uvw * (uvw_is_float ? 4 : 8));
  // dirty2ms with the last call's rows and frequency: the plane fill and FFT
  // start on its geometry now, and the device range pass confirms it
  const char* sp = getenv("CG_SPECULATE");  // 0: never (A/B timing)
  if (!to_dirty && !(sp && atoi(sp) == 0))
    CG_TRY(cg::dirty2ms_speculate(P, nrow, freq, P->io_dirty.p));
  if (!to_dirty && !(hr && atoi(hr) == 0) && !uvw_staged && !P->spec_pending) {
    if (uvw_is_float)
      scan_uvw_host((const float*)uvw, nrow, host_mm);
    else
      scan_uvw_host((const double*)uvw, nrow, host_mm);
    P->host_mm = host_mm;
  }
  int rs;
  if (to_dirty) {
    rs = cg::ms2dirty_device(P, nrow, freq, d_uvw, P->io_vis.p, wgt ? P->io_wgt.p : nullptr,
                             P->io_dirty.p);
    if (rs > 1) return rs;
    CG_TRY(copy_d2h(dirty, P->io_dirty.p, (size_t)nx * ny * 2 * tsz, s));
  } else {
    rs = cg::dirty2ms_device(P, nrow, freq, d_uvw, P->io_dirty.p, wgt ? P->io_wgt.p : nullptr,
                             P->io_vis.p);
    if (rs > 1) return rs;
    if (nrow > 0) CG_TRY(copy_d2h(vis, P->io_vis.p, (size_t)nrow * 2 * tsz, s));
  }
  CG_CUDA(cudaStreamSynchronize(s));
  return rs;
}

}  // namespace

extern "C" {

// ---------------- reference-compatible FP64 (cugridder.cu:541-571) ----------------
int ms2dirty_2(int nrow, int nxdirty, int nydirty, double fov, double freq, double* uvw,
               cg_c128* vis, double* wgt, cg_c128* dirty, double epsilon, double sigma, int sign) {
  return host_call(true, CG_PREC_FP64, nrow, nxdirty, nydirty, fov, freq, uvw, false, vis, wgt,
                   dirty, epsilon, sigma, sign);
}
int ms2dirty_1(int nrow, int nxdirty, int nydirty, double fov, double freq, double* uvw,
               cg_c128* vis, cg_c128* dirty, double epsilon, double sigma, int sign) {
  return host_call(true, CG_PREC_FP64, nrow, nxdirty, nydirty, fov, freq, uvw, false, vis,
                   nullptr, dirty, epsilon, sigma, sign);
}
int dirty2ms_1(int nrow, int nxdirty, int nydirty, double fov, double freq, double* uvw,
               cg_c128* vis, cg_c128* dirty, double epsilon, double sigma, int sign) {
  return host_call(false, CG_PREC_FP64, nrow, nxdirty, nydirty, fov, freq, uvw, false, vis,
                   nullptr, dirty, epsilon, sigma, sign);
}
int dirty2ms_2(int nrow, int nxdirty, int nydirty, double fov, double freq, double* uvw,
               cg_c128* vis, double* wgt, cg_c128* dirty, double epsilon, double sigma, int sign) {
  return host_call(false, CG_PREC_FP64, nrow, nxdirty, nydirty, fov, freq, uvw, false, vis, wgt,
                   dirty, epsilon, sigma, sign);
}

// ---------------- reference-compatible FP32 (-DSINGLE twins) ----------------
int ms2dirtyf_2(int nrow, int nxdirty, int nydirty, float fov, float freq, float* uvw,
                cg_c64* vis, float* wgt, cg_c64* dirty, float epsilon, float sigma, int sign) {
  return host_call(true, CG_PREC_FP32, nrow, nxdirty, nydirty, fov, freq, uvw, true, vis, wgt,
                   dirty, epsilon, sigma, sign);
}
int ms2dirtyf_1(int nrow, int nxdirty, int nydirty, float fov, float freq, float* uvw,
                cg_c64* vis, cg_c64* dirty, float epsilon, float sigma, int sign) {
  return host_call(true, CG_PREC_FP32, nrow, nxdirty, nydirty, fov, freq, uvw, true, vis,
                   nullptr, dirty, epsilon, sigma, sign);
}
int dirty2msf_1(int nrow, int nxdirty, int nydirty, float fov, float freq, float* uvw,
                cg_c64* vis, cg_c64* dirty, float epsilon, float sigma, int sign) {
  return host_call(false, CG_PREC_FP32, nrow, nxdirty, nydirty, fov, freq, uvw, true, vis,
                   nullptr, dirty, epsilon, sigma, sign);
}
int dirty2msf_2(int nrow, int nxdirty, int nydirty, float fov, float freq, float* uvw,
                cg_c64* vis, float* wgt, cg_c64* dirty, float epsilon, float sigma, int sign) {
  return host_call(false, CG_PREC_FP32, nrow, nxdirty, nydirty, fov, freq, uvw, true, vis, wgt,
                   dirty, epsilon, sigma, sign);
}

// ---------------- precision split, host pointers ----------------
int cg_ms2dirty_mixed(int64_t nrow, int nxdirty, int nydirty, double fov, double freq,
                      const double* uvw, const cg_c64* vis, const float* wgt, cg_c64* dirty,
                      double epsilon, double sigma, int sign) {
  return host_call(true, CG_PREC_FP32, nrow, nxdirty, nydirty, fov, freq, uvw, false,
                   (void*)vis, wgt, dirty, epsilon, sigma, sign);
}
int cg_dirty2ms_mixed(int64_t nrow, int nxdirty, int nydirty, double fov, double freq,
                      const double* uvw, cg_c64* vis, const float* wgt, const cg_c64* dirty,
                      double epsilon, double sigma, int sign) {
  return host_call(false, CG_PREC_FP32, nrow, nxdirty, nydirty, fov, freq, uvw, false, vis, wgt,
                   (void*)dirty, epsilon, sigma, sign);
}

// ---------------- plan API ----------------
int cg_plan_create(cg_plan** plan, int nxdirty, int nydirty, double fov, double epsilon,
                   double sigma, int sign, int precision, void* stream) {
  if (!plan) return CG_ERR_ARG;
  *plan = nullptr;
  int st = ensure_device();
  if (st) return st;
  cg_plan_s* P = new cg_plan_s();
  cudaGetDevice(&P->device);
  P->stream = (cudaStream_t)stream;
  if (const char* m = getenv("CG_GRID_METHOD")) {
    const int v = atoi(m);
    P->grid_method = (v >= 0 && v <= 2) ? v : 1;
  }
  if (const char* m = getenv("CG_FFT_PRUNE")) P->fft_pruning = atoi(m) != 0;
  if (const char* m = getenv("CG_COL_FFT")) P->col_fft = atoi(m) != 0;
  if (const char* m = getenv("CG_ROW_FFT")) P->row_fft = atoi(m) != 0;
  if (const char* m = getenv("CG_COL_FFT_REG")) P->four_step = atoi(m) == 4;
  if (const char* m = getenv("CG_AUTOTUNE")) P->autotune = atoi(m) != 0;
  if (const char* m = getenv("CG_DEGRID_TMA")) P->tma_default = atoi(m);
  st = cg::plan_configure(P, nxdirty, nydirty, fov, epsilon, sigma, sign, precision);
  if (st > 1) {
    destroy_plan(P);
    return st;
  }
  *plan = P;
  return st;
}

int cg_plan_set_stream(cg_plan* plan, void* stream) {
  if (!plan) return CG_ERR_ARG;
  plan->stream = (cudaStream_t)stream;
  return CG_OK;
}

int cg_plan_ms2dirty(cg_plan* plan, int64_t nrow, double freq, const double* d_uvw,
                     const void* d_vis, const void* d_wgt, void* d_dirty) {
  if (!plan) return CG_ERR_ARG;
  std::lock_guard<std::mutex> lock(plan->mu);
  return cg::ms2dirty_device(plan, nrow, freq, d_uvw, d_vis, d_wgt, d_dirty);
}

int cg_plan_dirty2ms(cg_plan* plan, int64_t nrow, double freq, const double* d_uvw,
                     const void* d_dirty, const void* d_wgt, void* d_vis) {
  if (!plan) return CG_ERR_ARG;
  std::lock_guard<std::mutex> lock(plan->mu);
  return cg::dirty2ms_device(plan, nrow, freq, d_uvw, d_dirty, d_wgt, d_vis);
}

int cg_plan_status(cg_plan* plan) {
  if (!plan) return CG_ERR_ARG;
  std::lock_guard<std::mutex> lock(plan->mu);
  CG_CUDA(cudaSetDevice(plan->device));
  return cg::tma_status(plan);
}

int cg_plan_ms2dirty_chan(cg_plan* plan, int64_t nrow, int nchan, const double* freqs,
                          const double* d_uvw, const void* d_vis, const void* d_wgt,
                          void* d_dirty) {
  if (!plan) return CG_ERR_ARG;
  std::lock_guard<std::mutex> lock(plan->mu);
  CG_CUDA(cudaSetDevice(plan->device));
  const double* u = nullptr;
  CG_TRY(expand_channels(plan, nrow, nchan, freqs, d_uvw, &u));
  return cg::ms2dirty_device(plan, nrow * nchan, freqs[0], u, d_vis, d_wgt, d_dirty);
}

int cg_plan_dirty2ms_chan(cg_plan* plan, int64_t nrow, int nchan, const double* freqs,
                          const double* d_uvw, const void* d_dirty, const void* d_wgt,
                          void* d_vis) {
  if (!plan) return CG_ERR_ARG;
  std::lock_guard<std::mutex> lock(plan->mu);
  CG_CUDA(cudaSetDevice(plan->device));
  const double* u = nullptr;
  CG_TRY(expand_channels(plan, nrow, nchan, freqs, d_uvw, &u));
  return cg::dirty2ms_device(plan, nrow * nchan, freqs[0], u, d_dirty, d_wgt, d_vis);
}

int cg_plan_get_info(const cg_plan* plan, cg_plan_info* info) {
  if (!plan || !info) return CG_ERR_ARG;
  const cg::Geom& g = plan->geom;
  info->kw = plan->kw;
  info->beta = plan->beta;
  info->nf1 = plan->nf1;
  info->nf2 = plan->nf2;
  info->nw = g.nw;
  info->i_center = g.i_center;
  info->i_half_width = g.i_half_width;
  info->o_center = g.o_center;
  info->o_half_width = g.o_half_width;
  info->gamma = g.gamma;
  info->h = g.h;
  info->pixelsize_x = plan->fov / 180.0 * cg::kPi / (double)plan->nx;
  info->pixelsize_y = plan->fov / 180.0 * cg::kPi / (double)plan->ny;
  info->nhive[0] = g.nhx;
  info->nhive[1] = g.nhy;
  info->nhive[2] = g.nhz;
  info->nrow = plan->nrow;
  info->workspace_bytes = cg::workspace_bytes(plan);
  return CG_OK;
}

int cg_plan_destroy(cg_plan* plan) {
  destroy_plan(plan);
  return CG_OK;
}

int cg_plan_set_method(cg_plan* plan, int method) {
  if (!plan || method < 0 || method > 2) return CG_ERR_ARG;
  plan->grid_method = method;
  return CG_OK;
}

int cg_plan_set_kernel(cg_plan* plan, int kind, int W, const double* coef) {
  if (!plan || (kind != CG_KERNEL_ES && kind != CG_KERNEL_POLY)) return CG_ERR_ARG;
  std::lock_guard<std::mutex> lock(plan->mu);
  if (kind == CG_KERNEL_POLY) {
    if (W < 2 || W > cg::kMaxW || !coef) {
      cg::set_last_error("polynomial kernel needs 2 <= W <= 16 and W*8 coefficients");
      return CG_ERR_ARG;
    }
    for (int i = 0; i < W * cg::kPolyCoef; i++)
      if (!std::isfinite(coef[i])) {
        cg::set_last_error("non-finite kernel coefficient");
        return CG_ERR_ARG;
      }
    memcpy(plan->poly, coef, sizeof(double) * W * cg::kPolyCoef);
    plan->poly_w = W;
  } else {
    if (W != 0 && (W < 2 || W > cg::kMaxW)) {
      cg::set_last_error("ES kernel width must be 0 (from epsilon) or 2..16");
      return CG_ERR_ARG;
    }
    plan->es_w = W;
  }
  plan->kernel_kind = kind;
  CG_CUDA(cudaSetDevice(plan->device));
  plan->kw = 0;  // force plan_configure to recompute W, grid sizes and the Fourier series
  int st = cg::plan_configure(plan, plan->nx, plan->ny, plan->fov, plan->eps, plan->sigma,
                              plan->sign, plan->precision);
  return st > 1 ? st : CG_OK;
}

int cg_set_host_kernel(int kind, int W, const double* coef) {
  if (kind != CG_KERNEL_ES && kind != CG_KERNEL_POLY) return CG_ERR_ARG;
  if (kind == CG_KERNEL_POLY && (W < 2 || W > cg::kMaxW || !coef)) return CG_ERR_ARG;
  if (kind == CG_KERNEL_ES && W != 0 && (W < 2 || W > cg::kMaxW)) return CG_ERR_ARG;
  if (kind == CG_KERNEL_POLY)
    for (int i = 0; i < W * cg::kPolyCoef; i++)
      if (!std::isfinite(coef[i])) return CG_ERR_ARG;
  std::lock_guard<std::mutex> lock(g_cache_mu);
  g_host_kernel = HostKernel();
  g_host_kernel.kind = kind;
  g_host_kernel.w = W;
  if (kind == CG_KERNEL_POLY) memcpy(g_host_kernel.poly, coef, sizeof(double) * W * cg::kPolyCoef);
  return CG_OK;
}

int cg_plan_set_fixed_uvw(cg_plan* plan, int on) {
  if (!plan) return CG_ERR_ARG;
  std::lock_guard<std::mutex> lock(plan->mu);
  plan->fixed_uvw = on != 0;
  plan->bins_valid = false;
  return CG_OK;
}

int cg_plan_set_autotune(cg_plan* plan, int on) {
  if (!plan) return CG_ERR_ARG;
  std::lock_guard<std::mutex> lock(plan->mu);
  plan->autotune = on != 0;
  for (auto& k : plan->tuned_key) std::fill(k, k + 4, 0);
  if (!on) plan->tune = cg::TileTune{};
  return CG_OK;
}

int cg_plan_get_tiling(const cg_plan* plan, int* tiling, float* tuned_ms) {
  if (!plan || !tiling) return CG_ERR_ARG;
  const cg::TileTune& t = plan->tune;
  const int v[8] = {t.wx, t.wy, t.wpb, t.warps, t.dx, t.dy, t.dpb, t.dthreads};
  std::copy(v, v + 8, tiling);
  if (tuned_ms) {
    tuned_ms[0] = plan->tuned_ms[0];
    tuned_ms[1] = plan->tuned_ms[1];
  }
  return CG_OK;
}

int cg_plan_set_grid_budget(cg_plan* plan, size_t bytes) {
  if (!plan) return CG_ERR_ARG;
  std::lock_guard<std::mutex> lock(plan->mu);
  plan->grid_budget = bytes;
  plan->bins_valid = false;
  return CG_OK;
}

int cg_plan_set_stop_stage(cg_plan* plan, int stage) {
  if (!plan || stage < 0 || stage > 3) return CG_ERR_ARG;
  plan->stop_stage = stage;
  return CG_OK;
}

int cg_plan_copy_buffer(cg_plan* plan, int which, void* host_dst, size_t bytes,
                        size_t* bytes_needed) {
  if (!plan) return CG_ERR_ARG;
  const cg::Geom& g = plan->geom;
  size_t tsz = plan->precision == CG_PREC_FP64 ? 8 : 4;
  const void* src = nullptr;
  size_t need = 0;
  switch (which) {
    case CG_BUF_HIVE_START:
      src = plan->hive_start.p;
      need = ((size_t)g.nhx * g.nhy * g.nhz + 1) * 4;
      break;
    case CG_BUF_PERM:
      src = plan->perm.p;
      need = (size_t)plan->nrow * 4;
      break;
    case CG_BUF_SORTED_KEYS:
      src = plan->skeys.p;
      need = (size_t)plan->nrow * 8;
      break;
    case CG_BUF_GRID:
      src = plan->grid.p;
      need = (size_t)g.nf1 * g.nf2 * g.nw * 2 * tsz;
      break;
    case CG_BUF_FSERIES_1:
      src = plan->K1.p;
      need = (size_t)(plan->nf1 / 2 + 1) * 8;
      break;
    case CG_BUF_FSERIES_2:
      src = plan->K2.p;
      need = (size_t)(plan->nf2 / 2 + 1) * 8;
      break;
    case CG_BUF_FSERIES_W:
      src = plan->K3q.p;
      need = (size_t)(plan->ny / 2 + 1) * (plan->nx / 2 + 1) * 8;
      break;
    default:
      return CG_ERR_ARG;
  }
  if (bytes_needed) *bytes_needed = need;
  if (!host_dst) return CG_OK;
  if (bytes < need || !src) return CG_ERR_ARG;
  CG_CUDA(cudaStreamSynchronize(plan->stream));
  if (which == CG_BUF_SORTED_KEYS && plan->key_bytes == 4) {
    // widen 32-bit keys to int64 on the host
    std::vector<uint32_t> tmp(plan->nrow);
    if (plan->nrow) CG_CUDA(cudaMemcpy(tmp.data(), src, (size_t)plan->nrow * 4, cudaMemcpyDeviceToHost));
    int64_t* dst = (int64_t*)host_dst;
    for (int64_t i = 0; i < plan->nrow; i++) dst[i] = (int64_t)tmp[i];
    return CG_OK;
  }
  if (need) CG_CUDA(cudaMemcpy(host_dst, src, need, cudaMemcpyDeviceToHost));
  return CG_OK;
}

int cg_plan_set_timing(cg_plan* plan, int on) {
  if (!plan) return CG_ERR_ARG;
  std::lock_guard<std::mutex> lock(plan->mu);
  plan->timer.on = on != 0;
  for (int d = 0; d < 2; d++) {
    plan->timer.calls[d] = 0;
    for (int i = 0; i < kMaxStages; i++) plan->timer.acc[d][i] = 0;
  }
  plan->timer.pending[0] = plan->timer.pending[1] = false;
  return CG_OK;
}

int cg_plan_get_timing(cg_plan* plan, int direction, double* stage_ms, int cap, int* nstages,
                       long long* ncalls) {
  if (!plan || direction < 0 || direction > 1) return CG_ERR_ARG;
  std::lock_guard<std::mutex> lock(plan->mu);
  CG_CUDA(cudaStreamSynchronize(plan->stream));
  cg::timer_flush(plan, 0);
  cg::timer_flush(plan, 1);
  int n = kMaxStages < cap ? kMaxStages : cap;
  for (int i = 0; i < n; i++) stage_ms[i] = plan->timer.acc[direction][i];
  if (nstages) *nstages = 7;
  if (ncalls) *ncalls = plan->timer.calls[direction];
  return CG_OK;
}

int cg_release_cache(void) {
  std::lock_guard<std::mutex> lock(g_cache_mu);
  for (int i = 0; i < 2; i++) {
    destroy_plan(g_cache[i]);
    g_cache[i] = nullptr;
  }
  return CG_OK;
}

const char* cg_last_error(void) { return cg::g_last_error.c_str(); }

long long cg_kernel_launches(void) { return cg::g_launches.load(); }

int cg_version(void) { return 100; }

}  // extern "C"
