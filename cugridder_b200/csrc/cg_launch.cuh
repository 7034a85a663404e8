// Launchers of the device kernels (one per pipeline stage).  All take the
// stream explicitly and return a status code; none synchronizes.
#pragma once
#include "cg_internal.cuh"

struct cg_dev_buf;

namespace cg {

// ---- binning (cg_bin.cu) ----
int launch_wminmax(const double* d_uvw, int64_t M, unsigned long long* d_mm, int* d_bad,
                   cudaStream_t st);
double decode_ordered(unsigned long long k);

// Stable LSD radix sort of the reference's hive-major cell keys.
// Workspace sizes in bytes for M rows and a key of key_bytes (4 or 8).
size_t bin_workspace_bytes(int64_t M, int key_bytes);
// d_hs_sums: scratch of hive_sums_ints(nh) ints for the counting hive
// offsets; nullptr selects a binary search over the sorted keys instead.
int launch_bin(const double* d_uvw, int64_t M, const Geom& g, int key_bytes, void* d_ws,
               size_t ws_bytes, int* d_perm, void* d_sorted_keys, int* d_hive_start,
               cudaStream_t st, int* d_hs_sums = nullptr);
inline int64_t hive_sums_ints(int64_t nh) { return (nh + 1 + 4095) / 4096; }
// Exclusive scan of n int32 counters (in place allowed); d_sums holds
// hive_sums_ints(n - 1) ints.
int launch_scan_exclusive(const int* d_in, int64_t n, int* d_out, int* d_sums, cudaStream_t st);
int launch_sort_u32(uint32_t* d_keys, int64_t M, int bits, void* d_ws, size_t ws_bytes,
                    int* d_perm, uint32_t* d_sorted, cudaStream_t st);

template <typename T>
int launch_build_stream(const int* d_perm, int64_t M, const double* d_uvw, const T* d_vis,
                        const T* d_wgt, const Geom& g, bool grid_dir, Rec<T>* d_tmp,
                        Rec<T>* d_recs, cudaStream_t st);

// ---- spreading / interpolation (cg_spread.cu) ----
// Device scratch of a plan's row-split warp tiles (see launch_grid): the
// buffers grow on first use and are kept by the plan.
struct SplitScratch {
  cg_dev_buf* chunks;  // per tile: chunks, then their exclusive scan (int)
  cg_dev_buf* sums;    // the scan's workspace
  cg_dev_buf* parts;   // partial tiles
};
// method 0: direct (global atomics / global gathers); 1: tiled (shared memory).
// d_counter: one device int used as the work-queue head of the tiled kernels.
constexpr int kGridDirect = 0;
constexpr int kGridTiled = 1;
constexpr int kGridMma = 2;  // tensor-core gridding (FP32, W <= 8); degridding uses tiled
// x-sliding warp windows (cg_grid_slide.cu): tt->wy band rows (8/16/32),
// tt->wpb hive columns per segment, tt->warps per CTA (0 = defaults).
// CG_ERR_ARG when they do not apply (W outside 4..8, an axis not a multiple
// of 8 cells, or a window that does not fit on an SM).
template <typename T>
int launch_grid_slide(const Rec<T>* d_recs, const int* d_hive_start, const Geom& g, T* d_fw,
                      int* d_counter, cudaStream_t st, const TileTune* tt);
int launch_grid_mma(const Rec<float>* d_recs, const int* d_hive_start, const Geom& g, float* d_fw,
                    cudaStream_t st);
template <typename T>
TileCfg grid_tiling(const Geom& g, bool degrid, const TileTune* tt = nullptr);
template <typename T>
WarpTile warp_tiling(const Geom& g, const TileTune* tt = nullptr);
int degrid_slots(const TileCfg& tc, int W);
// Autotuner candidates of direction dir (0 gridding, 1 degridding): rows of
// {x, y, planes, warps or threads}; set_tile_candidate writes one into tt.
int tile_candidates(int dir, const int (**cand)[4]);
void set_tile_candidate(TileTune& tt, int dir, const int* c);

// Shape of the x-sliding gridding (cg_grid_slide.cu) for one grid: bands of
// TY rows, segments of SEG hive columns, the circular window's row stride RS
// (complex elements), nslots segment slots per column, the items, warps per
// CTA and the per-warp shared-memory layout.
struct SlideTile {
  int TY, logTY, SEG;
  int RS;
  int nslots;
  int nbands, nsegs, nitems;
  int warps;
  size_t stage_off;
  size_t warp_bytes, smem;
};
// Shape for grid g in working precision tsz from the tuned fields of tt
// (wx < 0 selects the sliding kernel; wy band rows, wpb segment columns,
// warps) or the defaults; false where the sliding kernel does not apply.
bool slide_tiling(const Geom& g, size_t tsz, const TileTune* tt, SlideTile& tc);

// Row chunk of a heavy warp tile in a multi-grid gridding launch: chunk
// `chunk` of `nchunks` of tile `tile` of job `job` spreads its share of the
// tile's rows into a partial tile (TX x TY x PB complex cells of the job's
// tiling) at complex offset `off` of the launch's scratch.  Chunks of one tile
// are consecutive slots; the reduce pass sums them in chunk order into the
// grid, so results do not depend on which warp ran which chunk.
struct SplitItem {
  int job, tile, chunk, nchunks;
  long long off;
};

// One grid of a multi-grid launch (batched solves): the plan's sorted stream,
// hive offsets and grid, its tilings and its first work item in the launch.
template <typename T>
struct GridJob {
  const Rec<T>* recs;
  const int* hive_start;
  const int* perm;
  T* fw;
  T* vis;  // degridding output (rows in the caller's order)
  int64_t M;
  Geom g;
  WarpTile wt;
  SlideTile st;     // sliding-window gridding shape (st.TY = 0: warp tiles)
  TileCfg dt;
  int nslots;       // segment slots of the degridding tiles
  int grid_item0;   // first gridding item of this job (prefix over jobs)
  const int* tile_split;  // per warp tile: nonzero = gridded by split items (nullptr: none)
  int degrid_item0; // first degridding item of this job
};
// Launch shape shared by all jobs of a multi-grid launch.
struct MultiShape {
  int kw;
  bool poly;
  int warps;          // gridding warps per CTA
  size_t warp_bytes;  // gridding bytes per warp (largest of the jobs)
  int threads;        // degridding threads per CTA
  size_t dsmem;       // degridding bytes per CTA (largest of the jobs)
  int grid_items, degrid_items;
  bool partial_hives;  // some job's grid has an axis that is not a multiple of 8 cells
  bool slide;          // gridding by x-sliding windows (every job's st set)
  // row-split heavy warp tiles: nsplit chunk items (first in the queue),
  // nsplit_tiles reduce entries (chunk 0 of each split tile), the partial
  // tiles' scratch (complex cells of the working precision)
  int nsplit, nsplit_tiles;
  const SplitItem* d_split;
  const SplitItem* d_split_tiles;
  void* d_parts;
};
// Fill the item prefixes and the shared shape of jobs (host array).
template <typename T>
int multi_shape(GridJob<T>* jobs, int njobs, MultiShape* shape);
template <typename T>
int launch_grid_multi(const GridJob<T>* d_jobs, int njobs, const MultiShape& sh, int* d_counter,
                      cudaStream_t st);
// the same launch for jobs gridded by x-sliding windows (sh.slide)
template <typename T>
int launch_grid_slide_multi(const GridJob<T>* d_jobs, int njobs, const MultiShape& sh,
                            int* d_counter, cudaStream_t st);
// the multi-grid job of a plan whose last call was split at its spreading
// step (cg_plan.cuh's cg_plan_s; tilings from tt)
template <typename T>
int plan_grid_job(const cg_plan_s* P, const TileTune& tt, T* d_vis, GridJob<T>* job);
template <typename T>
int launch_degrid_multi(const GridJob<T>* d_jobs, int njobs, const MultiShape& sh, int* d_counter,
                        cudaStream_t st);
// tt: tiling choices (nullptr = defaults); sp: scratch for the row split of
// heavy warp tiles (nullptr: no split)
template <typename T>
int launch_grid(const Rec<T>* d_recs, const int* d_hive_start, int64_t M, const Geom& g, T* d_fw,
                int method, int* d_counter, cudaStream_t st, const TileTune* tt = nullptr,
                const SplitScratch* sp = nullptr);
template <typename T>
int launch_degrid(const Rec<T>* d_recs, const int* d_perm, const int* d_hive_start, int64_t M,
                  const Geom& g, const T* d_fw, T* d_vis, int method, int* d_counter,
                  cudaStream_t st, const TileTune* tt = nullptr);

// ---- degridding with TMA-staged tiles (cg_degrid_tma.cu; FP32, W 4..8) ----
// d_err: a device int set to 1 when a staging wait ran out (the host checks it)
// variant 1: 512 threads and two stages per CTA; 2: 256 threads and one
// stage, two CTAs per SM; 3: 32 x 8 tiles, 128 threads, three CTAs per SM;
// 4: 16 x 8 tiles, 128 threads (many planes)
bool degrid_tma_supported(const Geom& g, int variant);
int launch_degrid_tma(const Rec<float>* d_recs, const int* d_perm, const int* d_hive_start,
                      int64_t M, const Geom& g, const float* d_fw, float* d_vis, int* d_counter,
                      int* d_err, cudaStream_t st, int variant);

// ---- column FFTs in shared memory (cg_fft.cu) ----
bool col_fft_supported(int L, int na, int nb);
size_t col_fft_twiddle_count(int L);
int make_col_fft_twiddles(int L, float2* d_tw, cudaStream_t st);
// Four-step column transforms (FP32, L = 64 * L2, L in 1024..16384, na and nb
// multiples of 16): inverse (sign +1) leaves index g at row
// g / 64 + L2 (g % 64); forward (sign -1) expects its input there and
// leaves natural order.  d_roots: e^{2 pi i n / L}, n < L (make_fft_roots).
bool four_step_supported(int L, int na, int nb);
int make_fft_roots(int L, float2* d_roots, cudaStream_t st);
int launch_col_fft_four_step(float2* grid, int L, int nf1, size_t plane, int nplanes, int c0a,
                             int na, int c0b, int nb, int sign, const float2* d_roots,
                             cudaStream_t st);
// Row transforms (FP32, power-of-two L = nf1, the columns' twiddle table
// when nf1 = nf2) of rows [r0, r0 + nrows) (nrows even) of nplanes planes;
// elements [mid0, mid1) skipped as for launch_col_fft.
int launch_row_fft(float2* grid, int L, size_t plane, int nplanes, int r0, int nrows, int sign,
                   const float2* d_tw, cudaStream_t st, int mid0 = 0, int mid1 = 0, int skip = 0);
// Flags of skip (the default register-resident kernel; the other variants
// transform every row): rows [mid0, mid1) of the columns zero on input (1:
// not loaded) or unused on output (2: not stored); rows outside [b0, b1)
// zero on input (4) or unused on output (8).
int launch_col_fft(float2* grid, int L, int nf1, size_t plane, int nplanes, int c0a, int na,
                   int c0b, int nb, int sign, const float2* d_tw, cudaStream_t st, int mid0 = 0,
                   int mid1 = 0, int skip = 0, int b0 = 0, int b1 = 0);

// ---- memory-limited mode: plane windows [p0, p1) (cg_spread.cu, cg_wstage.cu) ----
template <typename T>
int launch_grid_window(const Rec<T>* d_recs, int64_t M, const Geom& g, int p0, int p1, T* d_fwb,
                       cudaStream_t st);
template <typename T>
int launch_degrid_window(const Rec<T>* d_recs, const int* d_perm, int64_t M, const Geom& g,
                         int p0, int p1, const T* d_fwb, T* d_vis, cudaStream_t st);
template <typename T>
int launch_wdft_window(const T* d_fwb, const Geom& g, int p0, int p1, const double* d_zq,
                       double* d_acc, cudaStream_t st);
template <typename T>
int launch_wdft_finish(const double* d_acc, const Geom& g, const double* d_K1, const double* d_K2,
                       const double* d_K3q, const double* d_zq, T* d_dirty, cudaStream_t st);
template <typename T>
int launch_plane_fill_window(const T* d_dirty, const Geom& g, int p0, int p1, const double* d_K1,
                             const double* d_K2, const double* d_K3q, const double* d_zq, T* d_fwb,
                             cudaStream_t st);

// ---- w stage (cg_wstage.cu) ----
int launch_quarter(const Geom& g, const Quad& q, double* d_K3q, double* d_zq, cudaStream_t st);
template <typename T>
int launch_wdft_deconv(const T* d_fw, const Geom& g, const double* d_K1, const double* d_K2,
                       const double* d_K3q, const double* d_zq, T* d_dirty, cudaStream_t st);
template <typename T>
int launch_plane_fill(const T* d_dirty, const Geom& g, const double* d_K1, const double* d_K2,
                      const double* d_K3q, const double* d_zq, T* d_fw, cudaStream_t st);

}  // namespace cg
