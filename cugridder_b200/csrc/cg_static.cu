// Allocation-free hive binning: the binning stage of ms2dirty / dirty2ms
// (the w-range pass, the stable radix sort on the hive-major cell key and the
// hive offsets) with every scratch buffer carved from one file-scope device
// array instead of plan workspace.  No cudaMalloc, no cudaFree, no
// allocating library; outputs go to caller-owned device buffers.
//
// Setup: the first call on a device looks up the array's device address with
// cudaGetSymbolAddress (with that device current) and caches it; that lookup
// loads the module, so the first call on each device should come before any
// stream capture.  The array is shared by all callers in the process:
// overlapping calls on one device (two streams, two host threads) race on it.
#include <cmath>
#include <mutex>

#include "cg_launch.cuh"
#include "cg_plan.cuh"

namespace {

constexpr int64_t kStaticMaxRows = 1 << 19;  // 524,288 rows
constexpr size_t kStaticBytes = 15u << 20;   // 15 MiB: mm words + radix workspace + sorted keys
constexpr size_t kMmBytes = 256;             // w/u/v range words and the non-finite flag
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_bin_scratch[kStaticBytes];

std::mutex g_mu;
void* g_scratch[kMaxDevices] = {};

inline size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

int scratch_for_device(int dev, void** out) {
  if (dev < 0 || dev >= kMaxDevices) {
    cg::set_last_error("device ordinal out of range for the static scratch table");
    return CG_ERR_ARG;
  }
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_bin_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      cg::set_last_error(e != cudaSuccess ? cudaGetErrorString(e) : "null symbol address");
      return CG_ERR_CUDA;
    }
    g_scratch[dev] = p;
  }
  *out = g_scratch[dev];
  return CG_OK;
}

}  // namespace

extern "C" {

int64_t cg_bin_static_max_rows(void) { return kStaticMaxRows; }

int cg_bin_static(int64_t nrow, int nxdirty, int nydirty, double fov, double freq,
                  const double* d_uvw, double epsilon, double sigma, int sign, int precision,
                  int* d_perm, int* d_hive_start, int64_t hive_start_len, int64_t* n_hives,
                  void* stream) {
  using namespace cg;
  if (n_hives) *n_hives = 0;
  if (nrow < 0) {
    set_last_error("nrow must be >= 0");
    return CG_ERR_ARG;
  }
  if (nrow > kStaticMaxRows) {
    set_last_error("nrow exceeds cg_bin_static_max_rows() (524288): the static scratch is fixed");
    return CG_ERR_SIZE;
  }
  if (nxdirty <= 0 || nydirty <= 0 || (nxdirty & 1) || (nydirty & 1)) {
    set_last_error("nxdirty and nydirty must be positive and even");
    return CG_ERR_ARG;
  }
  if (!(fov > 0.0) || !std::isfinite(fov) || !(freq > 0.0) || !std::isfinite(freq)) {
    set_last_error("fov and freq must be positive and finite");
    return CG_ERR_ARG;
  }
  if (precision != CG_PREC_FP64 && precision != CG_PREC_FP32) {
    set_last_error("precision must be CG_PREC_FP64 or CG_PREC_FP32");
    return CG_ERR_ARG;
  }
  if (nrow > 0 && (!d_uvw || !d_perm)) {
    set_last_error("null pointer");
    return CG_ERR_ARG;
  }
  int dev = 0;
  CG_CUDA(cudaGetDevice(&dev));
  void* scratch = nullptr;
  CG_TRY(scratch_for_device(dev, &scratch));
  cudaStream_t st = (cudaStream_t)stream;

  // geometry: the same steps as the plan path (setup_conv_opts,
  // get_num_cells, setup_gridder_plan in cugridder.cu:29-86)
  const double floor_eps = (precision == CG_PREC_FP64) ? 1.1e-16 : 6e-8;
  int kw;
  double beta, c;
  const int eps_status = setup_conv_opts(epsilon, sigma, floor_eps, kw, beta, c);
  if (eps_status > 1) {
    set_last_error("sigma must be > 1");
    return eps_status;
  }
  Geom g{};
  g.N1 = nydirty;
  g.N2 = nxdirty;
  g.nf1 = get_num_cells(nydirty, sigma, kw);
  g.nf2 = get_num_cells(nxdirty, sigma, kw);
  if (g.nf1 > 65535 || g.nf2 > 65535) {
    set_last_error("grid larger than 65535 cells per axis");
    return CG_ERR_SIZE;
  }
  g.kw = kw;
  g.beta = beta;
  g.es_c = c;

  unsigned long long* d_mm = (unsigned long long*)scratch;
  int* d_bad = (int*)(d_mm + 6);
  unsigned long long h_mm[7] = {};
  CG_TRY(launch_wminmax(d_uvw, nrow, d_mm, d_bad, st));  // resets the range words and the flag
  CG_CUDA(cudaMemcpyAsync(h_mm, d_mm, 52, cudaMemcpyDeviceToHost, st));
  CG_CUDA(cudaStreamSynchronize(st));
  if (((int*)(h_mm + 6))[0]) {
    set_last_error("non-finite uvw coordinate");
    return CG_ERR_ARG;
  }
  CG_TRY(call_geometry(fov, freq, sign, sigma, nrow, h_mm, g));
  const int64_t nh = (int64_t)g.nhx * g.nhy * g.nhz;
  if (n_hives) *n_hives = nh;
  if (!d_hive_start || hive_start_len < nh + 1) {
    set_last_error("hive_start_len must be at least n_hives + 1");
    return CG_ERR_SIZE;
  }

  // carve the radix-sort workspace and the sorted keys after the range words
  const int key_bytes = ((unsigned long long)nh * 64ULL <= 0xFFFFFFFFULL) ? 4 : 8;
  const size_t ws = bin_workspace_bytes(nrow, key_bytes);
  const size_t need = kMmBytes + align256(ws) + align256((size_t)nrow * key_bytes);
  if (need > kStaticBytes) {  // cannot happen for nrow <= kStaticMaxRows
    set_last_error("static scratch too small");
    return CG_ERR_SIZE;
  }
  char* base = (char*)scratch + kMmBytes;
  void* d_ws = base;
  void* d_keys = base + align256(ws);
  CG_TRY(launch_bin(d_uvw, nrow, g, key_bytes, d_ws, ws, d_perm, d_keys, d_hive_start, st));
  return eps_status;
}

}  // extern "C"
