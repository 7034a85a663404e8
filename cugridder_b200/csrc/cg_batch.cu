// Batched solves: many independent datasets (each with its own image size,
// field of view, row count and channels) imaged by one call.  The reference
// has no batched entry point (its C API images one dataset per call,
// cugridder.cu:541-571).
//
// Each dataset gets a plan in fixed-uvw mode.  A call runs in three phases:
//   1. per dataset, forked over a few streams: the stages before the
//      spreading step (binning on the first call, the sorted stream; for
//      dirty2ms also the plane fill and the FFT);
//   2. ONE persistent launch that spreads (ms2dirty) or interpolates
//      (dirty2ms) every dataset: CTAs / warps take (dataset, tile) items from
//      a global work queue, so small datasets fill the gaps of large ones;
//   3. ms2dirty only, per dataset: the FFT and the w-DFT with corrections.
// Datasets whose call cannot be split (no rows, memory-limited windows) run
// whole in phase 1.  The first call per direction runs eagerly and autotunes
// the tiling of the phase-2 launch (tile size, plane batch, threads per
// tile) by timing candidates on the batch's own data; the second call is
// captured into a CUDA graph and every later call replays it.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <numeric>
#include <vector>

#include "cg_launch.cuh"
#include "cg_plan.cuh"
#include "cg_tiles.cuh"

namespace {

constexpr int kBatchStreams = 4;

__global__ void k_chan_scale(const double* __restrict__ uvw, int64_t nrow, int nchan,
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

}  // namespace

struct cg_batch_s {
  int device = 0;
  cudaStream_t stream = nullptr;
  int precision = CG_PREC_FP32;
  std::vector<cg_dataset> ds;
  std::vector<double> f0;             // frequency of each dataset's flattened call
  std::vector<cg_plan_s*> plans;
  std::vector<cg_dev_buf> uvw_chan;   // flattened channel coordinates (nchan > 1)
  std::vector<cg_dev_buf> scales;
  std::vector<cudaStream_t> streams;
  cudaStream_t origin = nullptr;      // capture origin (the caller's stream may be the NULL stream)
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> joins;
  cudaEvent_t t0 = nullptr, t1 = nullptr;  // autotuner timing
  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  int calls[2] = {0, 0};
  int use_graph = 1;
  int autotune = 1;
  // phase 2: which datasets were split, their jobs (device array) and shape
  std::vector<char> split[2];
  std::vector<int> job_of[2];         // dataset index of each job
  std::vector<unsigned char> host_jobs[2];
  cg_dev_buf jobs[2], counter[2];
  cg::MultiShape shape[2] = {};
  bool jobs_ready[2] = {false, false};
  cg::TileTune tune{};
  float tuned_ms[2] = {0.f, 0.f};
  // row-split heavy gridding tiles: host copies of the datasets' hive offsets
  // (read back once: the uvw are fixed), the split tables and their device
  // copies, the partial tiles' scratch
  std::vector<std::vector<int>> hs_host;
  std::vector<cg::SplitItem> split_host;  // chunk items, then one entry per split tile
  std::vector<int> split_flags;
  cg_dev_buf split_dev, flags_dev, parts_dev;
};

namespace {

void destroy_batch(cg_batch_s* B) {
  if (!B) return;
  cudaSetDevice(B->device);
  for (int d = 0; d < 2; d++) {
    if (B->exec[d]) cudaGraphExecDestroy(B->exec[d]);
    cg::release(B->jobs[d]);
    cg::release(B->counter[d]);
  }
  cg::release(B->split_dev);
  cg::release(B->flags_dev);
  cg::release(B->parts_dev);
  for (auto P : B->plans) cg_plan_destroy(P);
  for (auto& b : B->uvw_chan) cg::release(b);
  for (auto& b : B->scales) cg::release(b);
  for (auto s : B->streams) cudaStreamDestroy(s);
  if (B->origin) cudaStreamDestroy(B->origin);
  if (B->fork) cudaEventDestroy(B->fork);
  if (B->t0) cudaEventDestroy(B->t0);
  if (B->t1) cudaEventDestroy(B->t1);
  for (auto e : B->joins) cudaEventDestroy(e);
  delete B;
}

const double* rows_uvw(const cg_batch_s* B, size_t i) {
  return B->ds[i].nchan > 1 ? (const double*)B->uvw_chan[i].p : B->ds[i].d_uvw;
}
int64_t rows_of(const cg_dataset& d) { return d.nrow * (int64_t)std::max(1, d.nchan); }

int fork_streams(cg_batch_s* B, cudaStream_t origin) {
  CG_CUDA(cudaEventRecord(B->fork, origin));
  for (auto s : B->streams) CG_CUDA(cudaStreamWaitEvent(s, B->fork, 0));
  return CG_OK;
}
int join_streams(cg_batch_s* B, cudaStream_t origin) {
  for (size_t k = 0; k < B->streams.size(); k++) {
    CG_CUDA(cudaEventRecord(B->joins[k], B->streams[k]));
    CG_CUDA(cudaStreamWaitEvent(origin, B->joins[k], 0));
  }
  return CG_OK;
}

// Row-split plan of the gridding launch's warp tiles.  A warp grids one tile's
// rows alone, so a tile holding far more than a warp's share of the launch
// (the centre of a dense small grid: 3% of a 19M-visibility dataset in one
// 16 x 8 tile) sets the launch's length.  Tiles with more than R rows, R about
// a quarter of a warp's share, become ceil(rows / R) chunk items at the head
// of the queue, each into a partial tile that k_split_reduce sums in chunk
// order.  Rows per tile come from the hive offsets, read back once (the
// batch's uvw are fixed); a chunk takes its share of the rows the kernel
// itself counts, so the estimate only sets the number of chunks.
// CG_BATCH_SPLIT=0 turns this off, CG_BATCH_SPLIT_ROWS sets R.
template <typename T>
int plan_splits(cg_batch_s* B, std::vector<cg::GridJob<T>>& jobs, const std::vector<int>& order,
                cg::MultiShape* sh, cudaStream_t st) {
  using C = typename std::conditional<sizeof(T) == 4, float2, double2>::type;
  B->split_host.clear();
  B->split_flags.clear();
  const char* off = std::getenv("CG_BATCH_SPLIT");
  if (off && std::atoi(off) == 0) return CG_OK;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  CG_CUDA(cudaStreamIsCapturing(st, &cs));
  if (cs != cudaStreamCaptureStatusNone) return CG_OK;  // planned by the eager first call only
  if (B->hs_host.size() != B->ds.size()) B->hs_host.assign(B->ds.size(), {});
  bool copied = false;
  for (size_t j = 0; j < jobs.size(); j++) {
    const cg::Geom& g = jobs[j].g;
    const size_t nh1 = (size_t)g.nhx * g.nhy * g.nhz + 1;
    std::vector<int>& hs = B->hs_host[order[j]];
    if (hs.size() == nh1) continue;
    hs.resize(nh1);
    CG_CUDA(cudaMemcpyAsync(hs.data(), jobs[j].hive_start, nh1 * sizeof(int),
                            cudaMemcpyDeviceToHost, st));
    copied = true;
  }
  if (copied) CG_CUDA(cudaStreamSynchronize(st));
  std::vector<std::vector<int64_t>> rows(jobs.size());
  int64_t V = 0;
  for (size_t j = 0; j < jobs.size(); j++) {
    const cg::WarpTile& wt = jobs[j].wt;
    rows[j].resize((size_t)wt.nitems);
    for (int t = 0; t < wt.nitems; t++) {
      rows[j][t] = cg::tile_slot_rows(B->hs_host[order[j]].data(), jobs[j].g, wt, t);
      V += rows[j][t];
    }
  }
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess)
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t warps = (int64_t)sms * std::max(1, sh->warps);
  int64_t R = std::max<int64_t>(2048, (V + 4 * warps - 1) / (4 * warps));
  if (const char* e = std::getenv("CG_BATCH_SPLIT_ROWS")) R = std::max<int64_t>(1, std::atoll(e));
  constexpr int kMaxChunks = 1024;
  constexpr size_t kMaxParts = (size_t)1 << 30;  // scratch bytes at most
  struct Heavy {
    int job, tile, nchunks;
    int64_t rows;
  };
  std::vector<Heavy> heavy;
  size_t parts = 0;
  for (;;) {  // R doubles until the partial tiles fit the scratch bound
    heavy.clear();
    parts = 0;
    for (size_t j = 0; j < jobs.size(); j++) {
      const cg::WarpTile& wt = jobs[j].wt;
      for (int t = 0; t < wt.nitems; t++) {
        const int64_t r = rows[j][t];
        if (r <= R) continue;
        const int k = (int)std::min<int64_t>(kMaxChunks, (r + R - 1) / R);
        heavy.push_back({(int)j, t, k, r});
        parts += (size_t)k * wt.TX * wt.TY * wt.PB * sizeof(C);
      }
    }
    if (parts <= kMaxParts) break;
    R *= 2;
  }
  if (heavy.empty()) return CG_OK;
  std::stable_sort(heavy.begin(), heavy.end(), [](const Heavy& a, const Heavy& b) { return a.rows > b.rows; });
  // flags of the jobs that have split tiles, one device array
  std::vector<int64_t> flag0(jobs.size(), -1);
  for (const Heavy& h : heavy)
    if (flag0[h.job] < 0) {
      flag0[h.job] = (int64_t)B->split_flags.size();
      B->split_flags.resize(B->split_flags.size() + jobs[h.job].wt.nitems, 0);
    }
  for (const Heavy& h : heavy) B->split_flags[flag0[h.job] + h.tile] = 1;
  std::vector<cg::SplitItem> tiles;
  long long offc = 0;  // complex cells
  for (const Heavy& h : heavy) {
    const cg::WarpTile& wt = jobs[h.job].wt;
    const long long slot = (long long)wt.TX * wt.TY * wt.PB;
    tiles.push_back({h.job, h.tile, 0, h.nchunks, offc});
    for (int c = 0; c < h.nchunks; c++)
      B->split_host.push_back({h.job, h.tile, c, h.nchunks, offc + c * slot});
    offc += (long long)h.nchunks * slot;
  }
  const size_t nsplit = B->split_host.size();
  if (nsplit + (size_t)sh->grid_items > 2147483647u) return CG_ERR_SIZE;
  B->split_host.insert(B->split_host.end(), tiles.begin(), tiles.end());
  CG_TRY(cg::ensure(B->split_dev, B->split_host.size() * sizeof(cg::SplitItem)));
  CG_TRY(cg::ensure(B->flags_dev, B->split_flags.size() * sizeof(int)));
  CG_TRY(cg::ensure(B->parts_dev, std::max<size_t>(parts, 256)));
  CG_CUDA(cudaMemcpyAsync(B->split_dev.p, B->split_host.data(),
                          B->split_host.size() * sizeof(cg::SplitItem), cudaMemcpyHostToDevice, st));
  CG_CUDA(cudaMemcpyAsync(B->flags_dev.p, B->split_flags.data(), B->split_flags.size() * sizeof(int),
                          cudaMemcpyHostToDevice, st));
  for (size_t j = 0; j < jobs.size(); j++)
    jobs[j].tile_split = flag0[j] < 0 ? nullptr : (const int*)B->flags_dev.p + flag0[j];
  sh->nsplit = (int)nsplit;
  sh->nsplit_tiles = (int)tiles.size();
  sh->d_split = (const cg::SplitItem*)B->split_dev.p;
  sh->d_split_tiles = (const cg::SplitItem*)B->split_dev.p + nsplit;
  sh->d_parts = B->parts_dev.p;
  return CG_OK;
}

// Jobs of the split datasets for tiling tt, heaviest rows-per-item first so
// that the queue ends on light items; fills the shape.
template <typename T>
int build_jobs(cg_batch_s* B, int dir, const cg::TileTune& tt, std::vector<cg::GridJob<T>>& jobs,
               std::vector<int>& order, cg::MultiShape* shape, cudaStream_t st) {
  jobs.clear();
  order.clear();
  for (size_t i = 0; i < B->ds.size(); i++) {
    if (!B->split[dir][i]) continue;
    cg::GridJob<T> J{};
    CG_TRY(cg::plan_grid_job<T>(B->plans[i], tt, (T*)B->ds[i].d_vis, &J));
    jobs.push_back(J);
    order.push_back((int)i);
  }
  if (jobs.empty()) return CG_OK;
  if (dir == 0 && tt.wx < 0)  // a sliding-window candidate needs every dataset's grid to take it
    for (const auto& J : jobs)
      if (J.st.TY == 0) return CG_ERR_ARG;
  std::vector<size_t> idx(jobs.size());
  std::iota(idx.begin(), idx.end(), 0);
  auto density = [&](size_t k) {
    const int items = dir == 0 ? (jobs[k].st.TY > 0 ? jobs[k].st.nitems : jobs[k].wt.nitems)
                               : jobs[k].dt.nitems;
    return (double)jobs[k].M / std::max(1, items);
  };
  std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) { return density(a) > density(b); });
  std::vector<cg::GridJob<T>> sorted;
  std::vector<int> sorted_order;
  for (size_t k : idx) {
    sorted.push_back(jobs[k]);
    sorted_order.push_back(order[k]);
  }
  jobs.swap(sorted);
  order.swap(sorted_order);
  CG_TRY(cg::multi_shape<T>(jobs.data(), (int)jobs.size(), shape));
  if (dir == 0 && !shape->slide) CG_TRY(plan_splits<T>(B, jobs, order, shape, st));
  return CG_OK;
}

template <typename T>
int upload_jobs(cg_batch_s* B, int dir, const std::vector<cg::GridJob<T>>& jobs, cudaStream_t st) {
  const size_t bytes = sizeof(cg::GridJob<T>) * std::max<size_t>(1, jobs.size());
  // the host copy stays alive until the batch is destroyed
  B->host_jobs[dir].resize(bytes);
  if (!jobs.empty()) std::memcpy(B->host_jobs[dir].data(), jobs.data(), sizeof(cg::GridJob<T>) * jobs.size());
  CG_TRY(cg::ensure(B->jobs[dir], bytes));
  CG_TRY(cg::ensure(B->counter[dir], 256));
  if (!jobs.empty())
    CG_CUDA(cudaMemcpyAsync(B->jobs[dir].p, B->host_jobs[dir].data(),
                            sizeof(cg::GridJob<T>) * jobs.size(), cudaMemcpyHostToDevice, st));
  return CG_OK;
}

template <typename T>
int launch_phase2(cg_batch_s* B, int dir, int njobs, const cg::MultiShape& sh, cudaStream_t st) {
  const auto* d_jobs = (const cg::GridJob<T>*)B->jobs[dir].p;
  int* counter = (int*)B->counter[dir].p;
  return dir == 0 ? cg::launch_grid_multi<T>(d_jobs, njobs, sh, counter, st)
                  : cg::launch_degrid_multi<T>(d_jobs, njobs, sh, counter, st);
}

// First call of a direction (eager): time every candidate tiling of the
// phase-2 launch on the batch's data (each launch rewrites its whole output,
// so the repeats are harmless), keep the fastest, upload its jobs.
template <typename T>
int prepare_phase2(cg_batch_s* B, int dir, cudaStream_t st) {
  std::vector<cg::GridJob<T>> jobs;
  std::vector<int> order;
  cg::MultiShape sh{};
  if (B->autotune) {
    const int (*cand)[4] = nullptr;
    const int ncand = cg::tile_candidates(dir, &cand);
    float best = -1.f;
    cg::TileTune best_tt = B->tune;
    for (int c = 0; c < ncand; c++) {
      if (dir == 1 && cand[c][3] < 0) continue;  // the TMA-staged kernel is single-grid only
      // the x-sliding windows run in the batch only when CG_GRID_SLIDE=1 asks
      // for them: on the 32-dataset workload (uv concentrated near each
      // grid's centre, so a few items hold most rows) they measured 3.4x
      // slower than the warp tiles, and each candidate costs two launches
      if (dir == 0 && cand[c][0] < 0) continue;
      cg::TileTune tt = B->tune;
      cg::set_tile_candidate(tt, dir, cand[c]);
      if (build_jobs<T>(B, dir, tt, jobs, order, &sh, st) != CG_OK || jobs.empty()) continue;
      CG_TRY(upload_jobs<T>(B, dir, jobs, st));
      float ms = 0.f;
      bool ok = true;
      for (int rep = 0; rep < 2 && ok; rep++) {  // the first launch warms up
        CG_CUDA(cudaEventRecord(B->t0, st));
        ok = launch_phase2<T>(B, dir, (int)jobs.size(), sh, st) == CG_OK;
        CG_CUDA(cudaEventRecord(B->t1, st));
        CG_CUDA(cudaEventSynchronize(B->t1));
        CG_CUDA(cudaEventElapsedTime(&ms, B->t0, B->t1));
      }
      if (!ok) continue;  // a candidate that does not fit on an SM launched nothing
      if (best < 0.f || ms < best) {
        best = ms;
        best_tt = tt;
      }
    }
    B->tune = best_tt;
    B->tuned_ms[dir] = std::max(best, 0.f);
  }
  CG_TRY(build_jobs<T>(B, dir, B->tune, jobs, order, &sh, st));
  CG_TRY(upload_jobs<T>(B, dir, jobs, st));
  B->job_of[dir] = order;
  B->shape[dir] = sh;
  B->jobs_ready[dir] = true;
  return CG_OK;
}

// One call: phase 1 per dataset over the batch streams, phase 2 as one
// launch on `origin`, phase 3 (ms2dirty) per dataset again.
int run_all(cg_batch_s* B, int dir, cudaStream_t origin) {
  const bool fp64 = B->precision == CG_PREC_FP64;
  const size_t n = B->ds.size();
  std::vector<char> split(n, 0);
  CG_TRY(fork_streams(B, origin));
  for (size_t i = 0; i < n; i++) {
    const cg_dataset& d = B->ds[i];
    cg_plan_s* P = B->plans[i];
    P->stream = B->streams[i % B->streams.size()];
    bool sp = false;
    const int st = dir == 0 ? cg::ms2dirty_split(P, 1, rows_of(d), B->f0[i], rows_uvw(B, i), d.d_vis,
                                                 d.d_wgt, d.d_dirty, &sp)
                            : cg::dirty2ms_split(P, rows_of(d), B->f0[i], rows_uvw(B, i), d.d_dirty,
                                                 d.d_wgt, d.d_vis, &sp);
    if (st > 1) return st;
    split[i] = sp;
  }
  CG_TRY(join_streams(B, origin));
  if (!B->jobs_ready[dir]) {
    B->split[dir] = split;
    CG_TRY(fp64 ? prepare_phase2<double>(B, dir, origin) : prepare_phase2<float>(B, dir, origin));
  } else if (split != B->split[dir]) {
    cg::set_last_error("batch: the datasets' split pattern changed between calls");
    return CG_ERR_ARG;
  }
  const int njobs = (int)B->job_of[dir].size();
  CG_TRY(fp64 ? launch_phase2<double>(B, dir, njobs, B->shape[dir], origin)
              : launch_phase2<float>(B, dir, njobs, B->shape[dir], origin));
  if (dir == 0 && njobs > 0) {
    CG_TRY(fork_streams(B, origin));
    for (int i : B->job_of[0]) {
      const cg_dataset& d = B->ds[i];
      CG_TRY(cg::ms2dirty_split(B->plans[i], 2, rows_of(d), B->f0[i], rows_uvw(B, i), d.d_vis,
                                d.d_wgt, d.d_dirty, nullptr));
    }
    CG_TRY(join_streams(B, origin));
  }
  return CG_OK;
}

}  // namespace

extern "C" {

int cg_batch_create(cg_batch_s** batch, int n, const cg_dataset* ds, double epsilon, double sigma,
                    int sign, int precision, void* stream) {
  if (!batch || n < 1 || !ds) return CG_ERR_ARG;
  *batch = nullptr;
  cg_batch_s* B = new cg_batch_s();
  cudaGetDevice(&B->device);
  B->stream = (cudaStream_t)stream;
  B->precision = precision;
  B->ds.assign(ds, ds + n);
  B->uvw_chan.resize(n);
  B->scales.resize(n);
  if (const char* e = getenv("CG_BATCH_GRAPH")) B->use_graph = atoi(e) != 0;
  if (const char* e = getenv("CG_BATCH_AUTOTUNE")) B->autotune = atoi(e) != 0;
  int rc = CG_OK;
  for (int i = 0; i < n && rc <= 1; i++) {
    const cg_dataset& d = B->ds[i];
    const int nchan = std::max(1, d.nchan);
    if (d.nrow < 0 || !d.freqs || !d.d_dirty || (d.nrow > 0 && (!d.d_uvw || !d.d_vis)) ||
        d.nrow * (int64_t)nchan > 2147483647LL) {
      cg::set_last_error("invalid dataset");
      rc = CG_ERR_ARG;
      break;
    }
    B->f0.push_back(d.freqs[0]);
    cg_plan_s* P = nullptr;
    rc = cg_plan_create(&P, d.nxdirty, d.nydirty, d.fov, epsilon, sigma, sign, precision, stream);
    if (rc > 1) break;
    B->plans.push_back(P);
    P->fixed_uvw = 1;
    if (nchan > 1 && d.nrow > 0) {  // channels flattened once: uvw * f_c / f_0 at f_0
      std::vector<double> sc(nchan);
      for (int c = 0; c < nchan; c++) sc[c] = c == 0 ? 1.0 : d.freqs[c] / d.freqs[0];
      rc = cg::ensure(B->scales[i], sizeof(double) * nchan);
      if (rc == CG_OK) rc = cg::ensure(B->uvw_chan[i], sizeof(double) * 3 * d.nrow * nchan);
      if (rc == CG_OK &&
          cudaMemcpy(B->scales[i].p, sc.data(), sizeof(double) * nchan, cudaMemcpyHostToDevice) != cudaSuccess)
        rc = CG_ERR_CUDA;
      if (rc == CG_OK) {
        const int64_t m = d.nrow * nchan;
        k_chan_scale<<<(int)std::min<int64_t>((m + 255) / 256, 148 * 16), 256, 0, B->stream>>>(
            d.d_uvw, d.nrow, nchan, (const double*)B->scales[i].p, (double*)B->uvw_chan[i].p);
        cg::count_launches(1);
        if (cudaGetLastError() != cudaSuccess) rc = CG_ERR_CUDA;
      }
    }
  }
  const int ns = std::min(kBatchStreams, n);
  for (int k = 0; k < ns && rc <= 1; k++) {
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) rc = CG_ERR_CUDA;
    else B->streams.push_back(s);
    cudaEvent_t e;
    if (rc <= 1 && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) rc = CG_ERR_CUDA;
    else if (rc <= 1) B->joins.push_back(e);
  }
  if (rc <= 1 && cudaEventCreateWithFlags(&B->fork, cudaEventDisableTiming) != cudaSuccess)
    rc = CG_ERR_CUDA;
  if (rc <= 1 && (cudaEventCreate(&B->t0) != cudaSuccess || cudaEventCreate(&B->t1) != cudaSuccess))
    rc = CG_ERR_CUDA;
  if (rc <= 1 && cudaStreamCreateWithFlags(&B->origin, cudaStreamNonBlocking) != cudaSuccess)
    rc = CG_ERR_CUDA;
  if (rc > 1) {
    destroy_batch(B);
    return rc;
  }
  *batch = B;
  return CG_OK;
}

static int batch_call(cg_batch_s* B, int dir) {
  if (!B) return CG_ERR_ARG;
  CG_CUDA(cudaSetDevice(B->device));
  const int k = B->calls[dir]++;
  // first call: geometry, binning, plans, autotuning
  if (!B->use_graph || k == 0) return run_all(B, dir, B->stream);
  if (!B->exec[dir]) {
    // captured on the batch's own origin stream: the caller's stream may be
    // the legacy NULL stream, which cannot be captured; the graph is then
    // launched on the caller's stream, which orders it like the eager calls
    cudaGraph_t graph = nullptr;
    CG_CUDA(cudaStreamBeginCapture(B->origin, cudaStreamCaptureModeRelaxed));
    const int st = run_all(B, dir, B->origin);
    const cudaError_t e = cudaStreamEndCapture(B->origin, &graph);
    if (st > 1 || e != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      cudaGetLastError();
      cg::set_last_error("batch graph capture failed");
      return st > 1 ? st : CG_ERR_CUDA;
    }
    const cudaError_t ei = cudaGraphInstantiate(&B->exec[dir], graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) {
      B->exec[dir] = nullptr;
      cg::set_last_error(cudaGetErrorString(ei));
      return CG_ERR_CUDA;
    }
  }
  CG_CUDA(cudaGraphLaunch(B->exec[dir], B->stream));
  return CG_OK;
}

int cg_batch_ms2dirty(cg_batch_s* batch) { return batch_call(batch, 0); }
int cg_batch_dirty2ms(cg_batch_s* batch) { return batch_call(batch, 1); }

int cg_batch_set_kernel(cg_batch_s* batch, int kind, int W, const double* coef) {
  if (!batch) return CG_ERR_ARG;
  if (batch->calls[0] || batch->calls[1]) {
    cg::set_last_error("batch: set the kernel before the first call");
    return CG_ERR_ARG;
  }
  for (auto P : batch->plans) CG_TRY(cg_plan_set_kernel(P, kind, W, coef));
  return CG_OK;
}

int cg_batch_get_tiling(const cg_batch_s* batch, int* tiling, float* tuned_ms) {
  if (!batch || !tiling) return CG_ERR_ARG;
  const cg::TileTune& t = batch->tune;
  const int v[8] = {t.wx, t.wy, t.wpb, t.warps, t.dx, t.dy, t.dpb, t.dthreads};
  for (int i = 0; i < 8; i++) tiling[i] = v[i];
  if (tuned_ms) {
    tuned_ms[0] = batch->tuned_ms[0];
    tuned_ms[1] = batch->tuned_ms[1];
  }
  return CG_OK;
}

int cg_batch_destroy(cg_batch_s* batch) {
  destroy_batch(batch);
  return CG_OK;
}

}  // extern "C"
