// Batched solves: many independent datasets (each with its own image size,
// field of view, row count and channels) imaged by one call.  Each dataset
// gets a plan in fixed-uvw mode; the datasets are spread over a few
// streams forked from the caller's stream, so small datasets overlap.  The
// first call per direction runs eagerly (w ranges, geometry, binning,
// allocation, cuFFT plans); the second is captured into a CUDA graph over
// all streams and every later call replays that graph -- one launch for the
// whole batch.  The reference has no batched entry point (its C API images
// one dataset per call, cugridder.cu:541-571).
#include <algorithm>
#include <cmath>
#include <vector>

#include "cg_launch.cuh"
#include "cg_plan.cuh"

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
  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  int calls[2] = {0, 0};
  int use_graph = 1;
};

namespace {

void destroy_batch(cg_batch_s* B) {
  if (!B) return;
  cudaSetDevice(B->device);
  for (int d = 0; d < 2; d++)
    if (B->exec[d]) cudaGraphExecDestroy(B->exec[d]);
  for (auto P : B->plans) cg_plan_destroy(P);
  for (auto& b : B->uvw_chan) cg::release(b);
  for (auto& b : B->scales) cg::release(b);
  for (auto s : B->streams) cudaStreamDestroy(s);
  if (B->origin) cudaStreamDestroy(B->origin);
  if (B->fork) cudaEventDestroy(B->fork);
  for (auto e : B->joins) cudaEventDestroy(e);
  delete B;
}

const double* rows_uvw(const cg_batch_s* B, size_t i) {
  return B->ds[i].nchan > 1 ? (const double*)B->uvw_chan[i].p : B->ds[i].d_uvw;
}

// every dataset's call, forked from `origin` over the batch streams and
// joined back into it
int run_all(cg_batch_s* B, int dir, cudaStream_t origin) {
  CG_CUDA(cudaEventRecord(B->fork, origin));
  for (auto s : B->streams) CG_CUDA(cudaStreamWaitEvent(s, B->fork, 0));
  for (size_t i = 0; i < B->ds.size(); i++) {
    const cg_dataset& d = B->ds[i];
    cg_plan_s* P = B->plans[i];
    P->stream = B->streams[i % B->streams.size()];
    const int64_t rows = d.nrow * (int64_t)std::max(1, d.nchan);
    const int st = dir == 0 ? cg::ms2dirty_device(P, rows, B->f0[i], rows_uvw(B, i), d.d_vis, d.d_wgt, d.d_dirty)
                            : cg::dirty2ms_device(P, rows, B->f0[i], rows_uvw(B, i), d.d_dirty, d.d_wgt, d.d_vis);
    if (st > 1) return st;
  }
  for (size_t k = 0; k < B->streams.size(); k++) {
    CG_CUDA(cudaEventRecord(B->joins[k], B->streams[k]));
    CG_CUDA(cudaStreamWaitEvent(origin, B->joins[k], 0));
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
  // first call: geometry, binning, plans
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
int cg_batch_destroy(cg_batch_s* batch) {
  destroy_batch(batch);
  return CG_OK;
}

}  // extern "C"
