// Gridding (spreading) and degridding (interpolation) with the ES kernel.
//
// Reference: conv_3d_outputdriven_t1 (conv.cu:522-627) -- one thread per grid
// cell tests every point of 9 neighbouring 8x8 hives and evaluates the
// kernel per (cell, point) pair -- and interp_3d_nputsdriven
// (interp.cu:132-210) -- one thread per unsorted point, W^3 gathers.  Both
// compute the periodic 3-D convolution
//   fw[p][g1][g0] = sum_j c_j phi(g0 - X0_j) phi(g1 - X1_j) phi(p - X2_j)
// with phi(d) = exp(beta sqrt(1 - c d^2)) for |d| < W/2.
//
// Method "tiled" (default): the grid is cut into tiles of TX x TY cells times
// batches of PB planes, handed out by a work queue to persistent CTAs.
//   gridding  : the CTA accumulates its tile in shared memory (FP32/FP64
//               shared atomics) from the rows of its own hives plus a one-hive
//               ring (each row clipped to the tile, periodic shifts applied),
//               then writes every cell of the tile once, coalesced -- the grid
//               needs no memset and no global atomics.
//   degridding: the CTA stages its tile plus the kernel halo (wrapped) in
//               shared memory and interpolates each row of its own hives once.
// Method "direct": input-driven over the sorted stream with global atomics /
// global gathers (kept as a cross-check).
#include <algorithm>
#include <cstdlib>
#include <type_traits>

#include "cg_coords.cuh"
#include "cg_launch.cuh"

namespace cg {

// ======================================================================= direct
template <typename T, int W>
__global__ void __launch_bounds__(256) k_grid_direct(const Rec<T>* __restrict__ recs, int64_t M,
                                                     Geom g, T* __restrict__ fw) {
  const T beta = (T)g.beta, c = (T)g.es_c;
  const int nf1 = g.nf1, nf2 = g.nf2, nw = g.nw;
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < M;
       s += (int64_t)gridDim.x * blockDim.x) {
    const Rec<T> r = recs[s];
    T kx[W], ky[W], kz[W];
    const int bx = (int)(r.bxy & 0xFFFFu), by = (int)(r.bxy >> 16), bz = (int)r.bz;
    if (bx >= nf1 || by >= nf2 || bz >= nw) continue;  // cells always in range; never indexes wild
    const int ox = bx + taps<T, W>(r.f[0], beta, c, kx);
    const int oy = by + taps<T, W>(r.f[1], beta, c, ky);
    const int oz = bz + taps<T, W>(r.f[2], beta, c, kz);
#pragma unroll 1
    for (int a = 0; a < W; a++) {
      const int zz = wrapi(oz + a, nw);
      const T cr = r.c[0] * kz[a], ci = r.c[1] * kz[a];
#pragma unroll 1
      for (int b = 0; b < W; b++) {
        const int yy = wrapi(oy + b, nf2);
        const T vr = cr * ky[b], vi = ci * ky[b];
        T* row = fw + 2 * (((size_t)zz * nf2 + yy) * nf1);
#pragma unroll
        for (int e = 0; e < W; e++) {
          const int xx = wrapi(ox + e, nf1);
          atomicAdd(row + 2 * xx, vr * kx[e]);
          atomicAdd(row + 2 * xx + 1, vi * kx[e]);
        }
      }
    }
  }
}

template <typename T, int W>
__global__ void __launch_bounds__(256) k_degrid_direct(const Rec<T>* __restrict__ recs,
                                                       const int* __restrict__ perm, int64_t M,
                                                       Geom g, const T* __restrict__ fw,
                                                       T* __restrict__ vis) {
  const T beta = (T)g.beta, c = (T)g.es_c;
  const int nf1 = g.nf1, nf2 = g.nf2, nw = g.nw;
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < M;
       s += (int64_t)gridDim.x * blockDim.x) {
    const Rec<T> r = recs[s];
    T kx[W], ky[W], kz[W];
    const int bx = (int)(r.bxy & 0xFFFFu), by = (int)(r.bxy >> 16), bz = (int)r.bz;
    if (bx >= nf1 || by >= nf2 || bz >= nw) continue;
    const int ox = bx + taps<T, W>(r.f[0], beta, c, kx);
    const int oy = by + taps<T, W>(r.f[1], beta, c, ky);
    const int oz = bz + taps<T, W>(r.f[2], beta, c, kz);
    T sr = 0, si = 0;
#pragma unroll 1
    for (int a = 0; a < W; a++) {
      const int zz = wrapi(oz + a, nw);
      T pr = 0, pi = 0;
#pragma unroll 1
      for (int b = 0; b < W; b++) {
        const int yy = wrapi(oy + b, nf2);
        const T* row = fw + 2 * (((size_t)zz * nf2 + yy) * nf1);
        T qr = 0, qi = 0;
#pragma unroll
        for (int e = 0; e < W; e++) {
          const int xx = wrapi(ox + e, nf1);
          qr += row[2 * xx] * kx[e];
          qi += row[2 * xx + 1] * kx[e];
        }
        pr += qr * ky[b];
        pi += qi * ky[b];
      }
      sr += pr * kz[a];
      si += pi * kz[a];
    }
    const int64_t i = perm[s];
    if (i < 0 || i >= M) continue;
    vis[2 * i] = sr * r.c[0] - si * r.c[1];
    vis[2 * i + 1] = sr * r.c[1] + si * r.c[0];
  }
}

// ======================================================================= tiled
// halo of the taps: a row in cell b touches cells [b - lo, b + hi]
template <int W>
struct Halo {
  static constexpr int lo = (W - 1) / 2;
  static constexpr int hi = (W + 1) / 2;
};

__device__ __forceinline__ int floordiv8(int a) { return a >= 0 ? a >> 3 : -((7 - a) >> 3); }

// Segment table of one work item: contiguous runs of sorted rows (hives that
// are neighbours along x share one run) with the periodic shift of their cells.
struct SegTable {
  int* start;
  int* pref;  // exclusive prefix of the run lengths, pref[nslots] = total
  int* sx;
  int* sy;
  int* sz;
};

// Build the runs for hive rows hy in [hya, hyb], planes hz in [za, zb] (raw,
// possibly outside the grid: wrapped with a shift of -+nf / -+nw) and hive
// columns [hxa, hxb].  Three slots per (hz, hy) row (left wrap, inside, right
// wrap).  Returns the number of slots.  Must be called by all threads.
__device__ int build_segments(const Geom& g, const int* __restrict__ hive_start, int hxa, int hxb,
                              int hya, int hyb, int za, int zb, SegTable t, int* s_warp) {
  const int ny_raw = hyb - hya + 1, nz_raw = zb - za + 1;
  const int rows = ny_raw * nz_raw;
  const int nslots = rows * 3;
  const int nhx = g.nhx, nhy = g.nhy, nw = g.nw;
  for (int base = 0; base < rows; base += blockDim.x) {
    const int r = base + threadIdx.x;
    int cnt[3] = {0, 0, 0};
    if (r < rows) {
      const int hy_raw = hya + r % ny_raw, hz_raw = za + r / ny_raw;
      int hy = hy_raw, shy = 0;
      if (hy < 0) { hy += nhy; shy = -g.nf2; }
      else if (hy >= nhy) { hy -= nhy; shy = g.nf2; }
      int hz = hz_raw, shz = 0;
      if (hz < 0) { hz += nw; shz = -nw; }
      else if (hz >= nw) { hz -= nw; shz = nw; }
      const int64_t rowbase = ((int64_t)hz * nhy + hy) * nhx;
      // part k: raw hx range and actual offset
      const int lo_k[3] = {hxa, max(hxa, 0), max(hxa, nhx)};
      const int hi_k[3] = {min(hxb, -1), min(hxb, nhx - 1), hxb};
      const int off_k[3] = {nhx, 0, -nhx};
      const int shx_k[3] = {-g.nf1, 0, g.nf1};
#pragma unroll
      for (int k = 0; k < 3; k++) {
        const int slot = r * 3 + k;
        int st = 0, c = 0;
        if (lo_k[k] <= hi_k[k]) {
          const int64_t h0 = rowbase + lo_k[k] + off_k[k];
          const int64_t h1 = rowbase + hi_k[k] + off_k[k];
          st = hive_start[h0];
          c = hive_start[h1 + 1] - st;
        }
        t.start[slot] = st;
        t.sx[slot] = shx_k[k];
        t.sy[slot] = shy;
        t.sz[slot] = shz;
        cnt[k] = c;
      }
    }
    // exclusive scan of the per-row sums across the block
    const int sum = cnt[0] + cnt[1] + cnt[2];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int inc = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += y;
    }
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    if (warp == 0) {
      const int nwarps = blockDim.x >> 5;
      int v = lane < nwarps ? s_warp[lane] : 0, vi = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, vi, o);
        if (lane >= o) vi += y;
      }
      s_warp[lane] = vi - v;
      if (lane == 31) s_warp[32] = vi;
    }
    __syncthreads();
    const int carry = (base == 0) ? 0 : t.pref[base * 3];
    const int ex = carry + s_warp[warp] + inc - sum;
    const int total = s_warp[32];
    if (r < rows) {
      t.pref[r * 3] = ex;
      t.pref[r * 3 + 1] = ex + cnt[0];
      t.pref[r * 3 + 2] = ex + cnt[0] + cnt[1];
    }
    __syncthreads();
    if (threadIdx.x == 0) t.pref[min(base + (int)blockDim.x, rows) * 3] = carry + total;
    __syncthreads();
  }
  return nslots;
}

__device__ __forceinline__ int find_segment(const int* __restrict__ pref, int nslots, int q) {
  int lo = 0, hi = nslots;  // pref[lo] <= q < pref[hi]
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (pref[mid] <= q) lo = mid; else hi = mid;
  }
  return lo;
}

// ---------------------------------------------------------------- gridding
// Shared accumulator: planar re / im arrays, row stride RS = TX + 8 so that
// the bank of cell (x, y) is (x + 8 y) mod 32: the rows of a warp (spread over
// one 8x8 hive) hit distinct banks.
__host__ __device__ __forceinline__ int acc_row_stride(int TX) { return TX + 8; }

template <typename T, int W>
__global__ void __launch_bounds__(512) k_grid_tiled(const Rec<T>* __restrict__ recs,
                                                    const int* __restrict__ hive_start, Geom g,
                                                    TileCfg tc, int nslots_max,
                                                    T* __restrict__ fw, int* __restrict__ counter) {
  extern __shared__ __align__(16) unsigned char smem[];
  constexpr int lo = Halo<W>::lo, hi = Halo<W>::hi;
  const int TX = tc.TX, TY = tc.TY, PB = tc.PB;
  const int RS = acc_row_stride(TX);
  const int nacc = RS * TY * PB;
  T* acc_re = (T*)smem;
  T* acc_im = acc_re + nacc;
  int* tb = (int*)(acc_im + nacc);
  const int ts = nslots_max + 1;
  SegTable t{tb, tb + ts, tb + 2 * ts, tb + 3 * ts, tb + 4 * ts};
  __shared__ int s_warp[33];
  __shared__ int s_item;
  const T beta = (T)g.beta, c = (T)g.es_c;
  const int nf1 = g.nf1, nf2 = g.nf2, nw = g.nw;
  const size_t plane = (size_t)nf1 * nf2;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const int ncell = TX * TY * PB;

  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int item = s_item;
    if (item >= tc.nitems) break;
    const int tix = item % tc.ntx, tiy = (item / tc.ntx) % tc.nty, tib = item / (tc.ntx * tc.nty);
    const int tx0 = tix * TX, ty0 = tiy * TY, p0 = tib * PB;
    const int tx1 = min(tx0 + TX, nf1), ty1 = min(ty0 + TY, nf2), p1 = min(p0 + PB, nw);
    const int wx = tx1 - tx0;
    const int nslots = build_segments(g, hive_start, floordiv8(tx0 - hi), floordiv8(tx1 - 1 + lo),
                                      floordiv8(ty0 - hi), floordiv8(ty1 - 1 + lo), p0 - hi,
                                      p1 - 1 + lo, t, s_warp);
    const int total = t.pref[nslots];
    if (total == 0) {
      // no row reaches this tile: write zeros straight to the grid
      for (int i = threadIdx.x; i < ncell; i += blockDim.x) {
        const int x = i % TX, y = (i / TX) % TY, z = i / (TX * TY);
        if (x < wx && ty0 + y < ty1 && p0 + z < p1) {
          const size_t o = (size_t)(p0 + z) * plane + (size_t)(ty0 + y) * nf1 + tx0 + x;
          fw[2 * o] = (T)0;
          fw[2 * o + 1] = (T)0;
        }
      }
      __syncthreads();
      continue;
    }
    for (int i = threadIdx.x; i < nacc; i += blockDim.x) {
      acc_re[i] = (T)0;
      acc_im[i] = (T)0;
    }
    __syncthreads();
    // within a chunk of blockDim rows, lane-major order keeps the lanes of a
    // warp on different cells; every row is visited exactly once
    for (int q0 = 0; q0 < total; q0 += blockDim.x) {
      const int q = q0 + lane * nwarp + warp;
      if (q >= total) continue;
      const int sgi = find_segment(t.pref, nslots, q);
      const int idx = t.start[sgi] + (q - t.pref[sgi]);
      const Rec<T> r = recs[idx];
      const int bx = (int)(r.bxy & 0xFFFFu) + t.sx[sgi];
      const int by = (int)(r.bxy >> 16) + t.sy[sgi];
      const int bz = (int)r.bz + t.sz[sgi];
      const int ox = bx + tap_offset<W>(r.f[0]);
      const int oy = by + tap_offset<W>(r.f[1]);
      const int oz = bz + tap_offset<W>(r.f[2]);
      const int xa = max(ox, tx0), xb = min(ox + W, tx1);
      const int ya = max(oy, ty0), yb = min(oy + W, ty1);
      const int za = max(oz, p0), zb = min(oz + W, p1);
      if (xa >= xb || ya >= yb || za >= zb) continue;
      T kx[W], ky[W], kz[W];
      taps<T, W>(r.f[0], beta, c, kx);
      taps<T, W>(r.f[1], beta, c, ky);
      taps<T, W>(r.f[2], beta, c, kz);
      for (int z = za; z < zb; z++) {
        const T cr = r.c[0] * kz[z - oz], ci = r.c[1] * kz[z - oz];
        for (int y = ya; y < yb; y++) {
          const T vr = cr * ky[y - oy], vi = ci * ky[y - oy];
          const int rowo = ((z - p0) * TY + (y - ty0)) * RS - tx0;
#pragma unroll
          for (int e = 0; e < W; e++) {
            const int x = ox + e;
            if (x >= xa && x < xb) {
              atomicAdd(acc_re + rowo + x, vr * kx[e]);
              atomicAdd(acc_im + rowo + x, vi * kx[e]);
            }
          }
        }
      }
    }
    __syncthreads();
    // flush: every cell of the tile written once, coalesced along x
    for (int i = threadIdx.x; i < ncell; i += blockDim.x) {
      const int x = i % TX, y = (i / TX) % TY, z = i / (TX * TY);
      if (x < wx && ty0 + y < ty1 && p0 + z < p1) {
        const size_t o = (size_t)(p0 + z) * plane + (size_t)(ty0 + y) * nf1 + tx0 + x;
        const int a = (z * TY + y) * RS + x;
        fw[2 * o] = acc_re[a];
        fw[2 * o + 1] = acc_im[a];
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- degridding
template <typename T, int W>
__global__ void __launch_bounds__(512) k_degrid_tiled(const Rec<T>* __restrict__ recs,
                                                      const int* __restrict__ perm,
                                                      const int* __restrict__ hive_start, int64_t M,
                                                      Geom g, TileCfg tc, int nslots_max,
                                                      const T* __restrict__ fw,
                                                      T* __restrict__ vis, int* __restrict__ counter) {
  extern __shared__ __align__(16) unsigned char smem[];
  constexpr int lo = Halo<W>::lo, hi = Halo<W>::hi;
  const int TX = tc.TX, TY = tc.TY, PB = tc.PB;
  const int nw = g.nw, nf1 = g.nf1, nf2 = g.nf2;
  const bool all_planes = (PB >= nw);
  const int SX = TX + lo + hi, SY = TY + lo + hi, SZ = all_planes ? nw : PB + lo + hi;
  const int SXP = SX + 1;  // padded row stride (complex elements)
  const int nstage = SX * SY * SZ;
  T* stg = (T*)smem;
  int* tb = (int*)(stg + 2 * (size_t)SXP * SY * SZ);
  const int ts = nslots_max + 1;
  SegTable t{tb, tb + ts, tb + 2 * ts, tb + 3 * ts, tb + 4 * ts};
  __shared__ int s_warp[33];
  __shared__ int s_item;
  const T beta = (T)g.beta, c = (T)g.es_c;
  const size_t plane = (size_t)nf1 * nf2;

  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int item = s_item;
    if (item >= tc.nitems) break;
    const int tix = item % tc.ntx, tiy = (item / tc.ntx) % tc.nty, tib = item / (tc.ntx * tc.nty);
    const int tx0 = tix * TX, ty0 = tiy * TY, p0 = all_planes ? 0 : tib * PB;
    const int tx1 = min(tx0 + TX, nf1), ty1 = min(ty0 + TY, nf2);
    const int p1 = all_planes ? nw : min(p0 + PB, nw);
    const int gx0 = tx0 - lo, gy0 = ty0 - lo, gz0 = all_planes ? 0 : p0 - lo;
    // runs of the tile's own hives (each row belongs to exactly one tile)
    const int nslots = build_segments(g, hive_start, tx0 >> 3, (tx1 - 1) >> 3, ty0 >> 3,
                                      (ty1 - 1) >> 3, p0, p1 - 1, t, s_warp);
    const int total = t.pref[nslots];
    if (total == 0) continue;  // uniform across the block: nothing to interpolate here
    // stage the tile + halo (periodic); row stride SXP = SX + 1 complex
    using V = typename std::conditional<sizeof(T) == 4, float2, double2>::type;
    V* stv = reinterpret_cast<V*>(stg);
    const V* fwv = reinterpret_cast<const V*>(fw);
    for (int i = threadIdx.x; i < nstage; i += blockDim.x) {
      const int sx = i % SX, sy = (i / SX) % SY, sz = i / (SX * SY);
      const int gx = modi(gx0 + sx, nf1), gy = modi(gy0 + sy, nf2), gz = modi(gz0 + sz, nw);
      stv[(sz * SY + sy) * SXP + sx] = fwv[(size_t)gz * plane + (size_t)gy * nf1 + gx];
    }
    __syncthreads();
    for (int q = threadIdx.x; q < total; q += blockDim.x) {
      const int sgi = find_segment(t.pref, nslots, q);
      const int sidx = t.start[sgi] + (q - t.pref[sgi]);
      const Rec<T> r = recs[sidx];
      const int bx = (int)(r.bxy & 0xFFFFu), by = (int)(r.bxy >> 16), bz = (int)r.bz;
      T kx[W], ky[W], kz[W];
      const int lx = bx + taps<T, W>(r.f[0], beta, c, kx) - gx0;
      const int ly = by + taps<T, W>(r.f[1], beta, c, ky) - gy0;
      const int lz = bz + taps<T, W>(r.f[2], beta, c, kz) - gz0;
      if (lx < 0 || ly < 0 || lx + W > SX || ly + W > SY) continue;  // cannot happen: tile rows only
      T sr = 0, si = 0;
      for (int a = 0; a < W; a++) {
        int zz = lz + a;
        zz = all_planes ? wrapi(zz, nw) : min(max(zz, 0), SZ - 1);
        T pr = 0, pi = 0;
        for (int b = 0; b < W; b++) {
          const T* row = stg + 2 * ((zz * SY + (ly + b)) * SXP + lx);
          T qr = 0, qi = 0;
#pragma unroll
          for (int e = 0; e < W; e++) {
            qr += row[2 * e] * kx[e];
            qi += row[2 * e + 1] * kx[e];
          }
          pr += qr * ky[b];
          pi += qi * ky[b];
        }
        sr += pr * kz[a];
        si += pi * kz[a];
      }
      const int64_t i = perm[sidx];
      if (i < 0 || i >= M) continue;
      vis[2 * i] = sr * r.c[0] - si * r.c[1];
      vis[2 * i + 1] = sr * r.c[1] + si * r.c[0];
    }
    __syncthreads();
  }
}

// ======================================================================= launch
static int env_int(const char* name, int dflt) {
  const char* v = getenv(name);
  return v ? atoi(v) : dflt;
}

static int num_sms() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) n = 148;
  }
  return n;
}

static int slots_for(int TY, int PB, int W) { return ((TY >> 3) + 2) * (PB + W + 1) * 3; }

// Tile shape: 32 x 32 cells by default, the plane batch covering all planes
// when the shared-memory footprint allows, otherwise halved until it fits.
// CG_TILE_X / CG_TILE_Y / CG_TILE_PLANES / CG_TILE_THREADS override (tuning).
template <typename T>
TileCfg grid_tiling(const Geom& g, bool degrid) {
  const size_t budget = 220 * 1024;
  const int W = g.kw;
  TileCfg tc{};
  int TX = env_int("CG_TILE_X", 32), TY = env_int("CG_TILE_Y", 32);
  TX = std::max(8, (TX / 8) * 8);
  TY = std::max(8, (TY / 8) * 8);
  int PB = env_int("CG_TILE_PLANES", 0);
  auto bytes = [&](int tx, int ty, int pb) -> size_t {
    size_t cells = degrid ? (size_t)(tx + W + 1) * (ty + W) * (pb >= g.nw ? g.nw : pb + W)
                          : (size_t)acc_row_stride(tx) * ty * pb;
    return cells * 2 * sizeof(T) + (size_t)(slots_for(ty, pb, W) + 1) * 4 * 5;
  };
  if (PB <= 0) {
    PB = g.nw;
    while (PB > 1 && bytes(TX, TY, PB) > budget) PB = (PB + 1) / 2;
  }
  if (PB > g.nw) PB = g.nw;
  // a staged plane batch must not wrap onto itself
  if (degrid && PB < g.nw && PB + W > g.nw) PB = g.nw;
  while (bytes(TX, TY, PB) > budget && (TX > 8 || TY > 8)) {
    if (TY >= TX) TY -= 8; else TX -= 8;
  }
  tc.TX = TX;
  tc.TY = TY;
  tc.PB = PB;
  tc.ntx = (g.nf1 + TX - 1) / TX;
  tc.nty = (g.nf2 + TY - 1) / TY;
  tc.npb = (g.nw + PB - 1) / PB;
  tc.nitems = tc.ntx * tc.nty * tc.npb;
  tc.threads = env_int("CG_TILE_THREADS", 512);
  tc.smem = bytes(TX, TY, PB);
  return tc;
}

template <typename T, int W>
static int grid_w(const Rec<T>* d_recs, const int* d_hive_start, int64_t M, const Geom& g, T* d_fw,
                  int method, int* d_counter, cudaStream_t st) {
  if (method == kGridDirect) {
    size_t G = (size_t)g.nf1 * g.nf2 * g.nw;
    CG_CUDA(cudaMemsetAsync(d_fw, 0, G * 2 * sizeof(T), st));
    if (M == 0) return CG_OK;
    int blocks = (int)((M + 255) / 256);
    if (blocks > 148 * 64) blocks = 148 * 64;
    k_grid_direct<T, W><<<blocks, 256, 0, st>>>(d_recs, M, g, d_fw);
    count_launches(1);
    CG_CUDA(cudaGetLastError());
    return CG_OK;
  }
  TileCfg tc = grid_tiling<T>(g, false);
  int nslots = slots_for(tc.TY, tc.PB, W);
  CG_CUDA(cudaFuncSetAttribute(k_grid_tiled<T, W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)tc.smem));
  int per_sm = 0;
  CG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_grid_tiled<T, W>, tc.threads,
                                                        tc.smem));
  if (per_sm < 1) {
    set_last_error("tiled gridding does not fit on an SM");
    return CG_ERR_ARG;
  }
  int blocks = std::min(tc.nitems, per_sm * num_sms());
  CG_CUDA(cudaMemsetAsync(d_counter, 0, sizeof(int), st));
  k_grid_tiled<T, W><<<blocks, tc.threads, tc.smem, st>>>(d_recs, d_hive_start, g, tc, nslots,
                                                          d_fw, d_counter);
  count_launches(1);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

template <typename T, int W>
static int degrid_w(const Rec<T>* d_recs, const int* d_perm, const int* d_hive_start, int64_t M,
                    const Geom& g, const T* d_fw, T* d_vis, int method, int* d_counter,
                    cudaStream_t st) {
  if (M == 0) return CG_OK;
  if (method == kGridDirect) {
    int blocks = (int)((M + 255) / 256);
    if (blocks > 148 * 64) blocks = 148 * 64;
    k_degrid_direct<T, W><<<blocks, 256, 0, st>>>(d_recs, d_perm, M, g, d_fw, d_vis);
    count_launches(1);
    CG_CUDA(cudaGetLastError());
    return CG_OK;
  }
  TileCfg tc = grid_tiling<T>(g, true);
  int nslots = slots_for(tc.TY, tc.PB, W);
  CG_CUDA(cudaFuncSetAttribute(k_degrid_tiled<T, W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)tc.smem));
  int per_sm = 0;
  CG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_degrid_tiled<T, W>, tc.threads,
                                                        tc.smem));
  if (per_sm < 1) {
    set_last_error("tiled degridding does not fit on an SM");
    return CG_ERR_ARG;
  }
  int blocks = std::min(tc.nitems, per_sm * num_sms());
  CG_CUDA(cudaMemsetAsync(d_counter, 0, sizeof(int), st));
  k_degrid_tiled<T, W><<<blocks, tc.threads, tc.smem, st>>>(d_recs, d_perm, d_hive_start, M, g, tc,
                                                            nslots, d_fw, d_vis, d_counter);
  count_launches(1);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

#define CG_W_SWITCH(W_, CALL)                  \
  switch (W_) {                                \
    case 2: return CALL(2);                    \
    case 3: return CALL(3);                    \
    case 4: return CALL(4);                    \
    case 5: return CALL(5);                    \
    case 6: return CALL(6);                    \
    case 7: return CALL(7);                    \
    case 8: return CALL(8);                    \
    case 9: return CALL(9);                    \
    case 10: return CALL(10);                  \
    case 11: return CALL(11);                  \
    case 12: return CALL(12);                  \
    case 13: return CALL(13);                  \
    case 14: return CALL(14);                  \
    case 15: return CALL(15);                  \
    case 16: return CALL(16);                  \
    default: return CG_ERR_ARG;                \
  }

template <typename T>
int launch_grid(const Rec<T>* d_recs, const int* d_hive_start, int64_t M, const Geom& g, T* d_fw,
                int method, int* d_counter, cudaStream_t st) {
#define CG_GRID_CALL(w) grid_w<T, w>(d_recs, d_hive_start, M, g, d_fw, method, d_counter, st)
  CG_W_SWITCH(g.kw, CG_GRID_CALL)
#undef CG_GRID_CALL
}

template <typename T>
int launch_degrid(const Rec<T>* d_recs, const int* d_perm, const int* d_hive_start, int64_t M,
                  const Geom& g, const T* d_fw, T* d_vis, int method, int* d_counter,
                  cudaStream_t st) {
#define CG_DEGRID_CALL(w) \
  degrid_w<T, w>(d_recs, d_perm, d_hive_start, M, g, d_fw, d_vis, method, d_counter, st)
  CG_W_SWITCH(g.kw, CG_DEGRID_CALL)
#undef CG_DEGRID_CALL
}

template TileCfg grid_tiling<float>(const Geom&, bool);
template TileCfg grid_tiling<double>(const Geom&, bool);
template int launch_grid<float>(const Rec<float>*, const int*, int64_t, const Geom&, float*, int,
                                int*, cudaStream_t);
template int launch_grid<double>(const Rec<double>*, const int*, int64_t, const Geom&, double*, int,
                                 int*, cudaStream_t);
template int launch_degrid<float>(const Rec<float>*, const int*, const int*, int64_t, const Geom&,
                                  const float*, float*, int, int*, cudaStream_t);
template int launch_degrid<double>(const Rec<double>*, const int*, const int*, int64_t,
                                   const Geom&, const double*, double*, int, int*, cudaStream_t);

}  // namespace cg
