// Internal declarations of the B200 gridder (libcugridder.so).
//
// Naming follows the reference (RapidsAtHKUST/cuGridder): N1 = nydirty is the
// fast image axis and grid dim 0 (size nf1, fed by v), N2 = nxdirty is the
// slow image axis and grid dim 1 (size nf2, fed by u); nw = nf3 is the number
// of w planes (cugridder.cu:191,347).  The grid is stored plane-major,
// fw[p][g1][g0] with g0 fastest, as in the reference (conv.cu:596-598).
#pragma once
#include <cuda_runtime.h>
#include <cufft.h>
#include <cstddef>
#include <cstdint>

#include "../../include/cugridder.h"

namespace cg {

constexpr double kPi = 3.14159265358979323846;
// constants exactly as the reference's include/utils.h:29-30
constexpr double kM_1_2PI = 0.159154943091895336;
constexpr double kM_2PI = 6.28318530717958648;
constexpr double kSpeedOfLight = 299792458.0;
constexpr int kMaxW = 16;
constexpr int kMaxQuad = 32;  // GL nodes used by the kernel Fourier series (p <= 26)

// Per-call geometry, passed by value to every kernel.
struct Geom {
  int N1, N2;        // image sizes (N1 = ny fast, N2 = nx)
  int nf1, nf2, nw;  // grid sizes
  int kw;            // kernel width W
  double beta, es_c; // ES kernel exp(beta*sqrt(1 - c d^2)), |d| < W/2
  double pixx, pixy; // pixel sizes (radians): pixx with u / image x, pixy with v / image y
  double foc;        // freq / c
  int sign;
  double i_center, i_half_width, o_center, o_half_width, gamma, h;
  int nhx, nhy, nhz; // 8 x 8 x 1 hives
  // grid rows (g1) / columns (g0) the data can touch, inclusive; the full
  // range when the data wraps around the grid edge
  int band_r0, band_r1, band_c0, band_c1;
  // piecewise-polynomial kernel (learned kernel): W segments x kPolyCoef
  // coefficients in the working precision; null pointers select ES
  const float* polyf;
  const double* polyd;
  // the forward column transform does not load the rows outside the image in
  // the image's columns (one-pass column kernel): the plane fill leaves them
  int fill_skip;
  // the same skips for ms2dirty: the row pass reads only the rows of
  // fft_row_band and the column kernel loads no other row, so gridding may
  // leave the rows outside it unwritten (tiles and bands wholly outside)
  int grid_skip;
  // four-step column transform active (its L2 = nf2 / 64; 0 = off): grid
  // index g along dim 1 sits at row g / 64 + rowperm * (g % 64) between the
  // column transform and the w stage (see row_of)
  int rowperm;
};

// Grid rows [r0, r0 + n) that the band-pruned transform's row pass covers:
// the data band, its row count rounded up to 64 (the row plan's batch).
__host__ __device__ inline void fft_row_band(const Geom& g, int& r0, int& n) {
  const int nrows = g.band_r1 - g.band_r0 + 1;
  n = ((nrows + 63) / 64) * 64;
  if (n > g.nf2) n = g.nf2;
  r0 = g.band_r0 < g.nf2 - n ? g.band_r0 : g.nf2 - n;
}

// storage row of grid index g along dim 1 (identity unless rowperm)
__host__ __device__ __forceinline__ int row_of(const Geom& g, int g1) {
  return g.rowperm ? g1 / 64 + g.rowperm * (g1 % 64) : g1;
}

constexpr int kPolyCoef = 8;  // degree-7 Horner polynomial per segment

// Kernel Fourier-series quadrature: phi_hat(k) = sum_i g[i] * 2 cos(x[i] k)
struct Quad {
  int p;
  double x[kMaxQuad];
  double g[kMaxQuad];
};

// Sorted visibility record: cell index (bx,by,bz) and the fractional offset
// inside the cell in the working precision, plus a complex payload
// (the weighted, phase-shifted visibility for gridding; the output factor
// wgt*exp(-i o_c w) for degridding).
template <typename T>
struct alignas(16) Rec {
  T f[3];
  uint32_t bxy;  // bx | by << 16
  uint32_t bz;
  T c[2];
};

// Tiling of the grid for the tiled spreading / interpolation kernels: tiles of
// TX x TY cells (multiples of the 8x8 hive) times batches of PB planes.
struct TileCfg {
  int TX, TY, PB;
  int ntx, nty, npb, nitems;  // tiles per queue row, queue rows, plane batches, items
  int bx0, by0;               // grid tile of queue item 0 (the data band's first tile)
  int threads;
  size_t smem;
};

// Warp-owned tiles of the gridding kernel: TX x TY cells times PB planes per
// warp, cell (x, y, z) at z * PS + y * RS + x (complex units), y-major: PS =
// TX + 1 is the plane stride inside a tile row and RS >= PB * PS the row stride.
struct WarpTile {
  int TX, TY, PB, RS, PS, slots;
  int ntx, nty, npb, nitems;
  int warps;  // per CTA
  size_t warp_bytes, smem;
};

// Tiling choices of one plan (0 = default): gridding warp tiles (wx x wy
// cells, wpb planes, warps per CTA) and degridding tiles (dx x dy cells,
// dpb planes, threads per CTA).
struct TileTune {
  int wx, wy, wpb, warps;
  int dx, dy, dpb, dthreads;
};

// ---- pipeline entry points (cg_pipeline.cu) ----
}  // namespace cg

struct cg_plan_s;

namespace cg {
int ms2dirty_device(cg_plan_s* P, int64_t nrow, double freq, const double* d_uvw,
                    const void* d_vis, const void* d_wgt, void* d_dirty);
int dirty2ms_device(cg_plan_s* P, int64_t nrow, double freq, const double* d_uvw,
                    const void* d_dirty, const void* d_wgt, void* d_vis);
// Host entry points: when the plan's last call had this call's row count and
// frequency, start dirty2ms's plane fill and FFT on aux_stream with that
// call's geometry as soon as the image (P->main_ready) is in, before uvw.  The
// call's own range pass then confirms the geometry (same u, v, w ranges) or
// discards the work and redoes it.
int dirty2ms_speculate(cg_plan_s* P, int64_t nrow, double freq, const void* d_dirty);
// Calls split at the spreading step (batched solves): ms2dirty part 1 runs
// the stages before gridding, part 2 those after it; dirty2ms_split runs the
// stages before degridding.  *split = false when the call ran whole (no
// rows, memory-limited windows, a non-tiled method, timing or stop stages).
int ms2dirty_split(cg_plan_s* P, int part, int64_t nrow, double freq, const double* d_uvw,
                   const void* d_vis, const void* d_wgt, void* d_dirty, bool* split);
int dirty2ms_split(cg_plan_s* P, int64_t nrow, double freq, const double* d_uvw,
                   const void* d_dirty, const void* d_wgt, void* d_vis, bool* split);
// Waits for the plan's stream and reports (and clears) a timed-out TMA
// staging wait of the degridding: CG_ERR_CUDA, else CG_OK.
int tma_status(cg_plan_s* P);
}  // namespace cg

#define CG_CUDA(call)                                  \
  do {                                                 \
    cudaError_t e_ = (call);                           \
    if (e_ != cudaSuccess) {                           \
      cg::set_last_error(cudaGetErrorString(e_));      \
      return (e_ == cudaErrorMemoryAllocation) ? CG_ERR_NOMEM : CG_ERR_CUDA; \
    }                                                  \
  } while (0)

#define CG_CUFFT(call)                                 \
  do {                                                 \
    cufftResult r_ = (call);                           \
    if (r_ != CUFFT_SUCCESS) {                         \
      cg::set_last_error("cuFFT error");               \
      return (r_ == CUFFT_ALLOC_FAILED) ? CG_ERR_NOMEM : CG_ERR_CUFFT; \
    }                                                  \
  } while (0)

#define CG_TRY(expr)            \
  do {                          \
    int s_ = (expr);            \
    if (s_ > 1) return s_;      \
  } while (0)

namespace cg {
// Dynamic shared-memory opt-in and blocks per SM of a kernel at a launch
// shape, computed once and cached: later launches (including those recorded
// while a stream is being captured into a CUDA graph) make no attribute or
// occupancy queries.  Returns a CUDA error code.
cudaError_t kernel_occupancy(const void* func, int threads, size_t smem, int* per_sm);
void set_last_error(const char* msg);
// number of kernels this library has launched (process-wide)
void count_launches(long long n);
}
