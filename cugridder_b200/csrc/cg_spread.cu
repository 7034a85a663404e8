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
#include "cg_plan.cuh"
#include "cg_tiles.cuh"

namespace cg {

// ======================================================================= direct
template <typename T, int W>
__global__ void __launch_bounds__(256) k_grid_direct(const Rec<T>* __restrict__ recs, int64_t M,
                                                     Geom g, T* __restrict__ fw) {
  const T beta = (T)g.beta, c = (T)g.es_c;
  const T* __restrict__ poly = geom_poly<T>(g);
  const int nf1 = g.nf1, nf2 = g.nf2, nw = g.nw;
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < M;
       s += (int64_t)gridDim.x * blockDim.x) {
    const Rec<T> r = recs[s];
    T kx[W], ky[W], kz[W];
    const int bx = (int)(r.bxy & 0xFFFFu), by = (int)(r.bxy >> 16), bz = (int)r.bz;
    if (bx >= nf1 || by >= nf2 || bz >= nw) continue;  // cells always in range; never indexes wild
    const int ox = bx + taps<T, W>(r.f[0], beta, c, poly, kx);
    const int oy = by + taps<T, W>(r.f[1], beta, c, poly, ky);
    const int oz = bz + taps<T, W>(r.f[2], beta, c, poly, kz);
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
  const T* __restrict__ poly = geom_poly<T>(g);
  const int nf1 = g.nf1, nf2 = g.nf2, nw = g.nw;
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < M;
       s += (int64_t)gridDim.x * blockDim.x) {
    const Rec<T> r = recs[s];
    T kx[W], ky[W], kz[W];
    const int bx = (int)(r.bxy & 0xFFFFu), by = (int)(r.bxy >> 16), bz = (int)r.bz;
    if (bx >= nf1 || by >= nf2 || bz >= nw) continue;
    const int ox = bx + taps<T, W>(r.f[0], beta, c, poly, kx);
    const int oy = by + taps<T, W>(r.f[1], beta, c, poly, ky);
    const int oz = bz + taps<T, W>(r.f[2], beta, c, poly, kz);
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


// ---------------------------------------------------------------- gridding
// Warp-owned tiles: every warp accumulates its own TX x TY x PB tile in
// shared memory, so no two threads ever update the same cell concurrently
// and no atomics are needed; the result is deterministic.  Candidate rows
// (own hives plus a one-hive ring, clipped to the tile) are pre-scanned 32 at
// a time; each overlapping row is then spread by the whole warp: lane l takes
// the tap pairs p = l + 32 r, (dy, dz) = (p % W, p / W), and walks the W taps
// along x.  Cell (x, y, z) of a warp tile lives at z*PS + y*RS + x (complex
// units) with RS = 1 and PS = W (mod 16): the 16 lanes of a half-warp touch
// 16 distinct 8-byte bank pairs.

__device__ __forceinline__ int warp_excl_scan(int x, int& total) {
  const int lane = threadIdx.x & 31;
  int inc = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  total = __shfl_sync(0xffffffffu, inc, 31);
  return inc - x;
}

// warp-level version of build_segments (same slot layout)
__device__ int warp_build_segments(const Geom& g, const int* __restrict__ hive_start, int hxa,
                                   int hxb, int hya, int hyb, int za, int zb, SegTable t) {
  const int lane = threadIdx.x & 31;
  const int ny_raw = hyb - hya + 1, nz_raw = zb - za + 1;
  const int rows = ny_raw * nz_raw;
  const int nhx = g.nhx, nhy = g.nhy, nw = g.nw;
  int carry = 0;
  for (int base = 0; base < rows; base += 32) {
    const int r = base + lane;
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
      const int lo_k[3] = {hxa, max(hxa, 0), max(hxa, nhx)};
      const int hi_k[3] = {min(hxb, -1), min(hxb, nhx - 1), hxb};
      const int off_k[3] = {nhx, 0, -nhx};
      const int shx_k[3] = {-g.nf1, 0, g.nf1};
#pragma unroll
      for (int k = 0; k < 3; k++) {
        const int slot = r * 3 + k;
        int st = 0, c = 0;
        if (lo_k[k] <= hi_k[k]) {
          st = hive_start[rowbase + lo_k[k] + off_k[k]];
          c = hive_start[rowbase + hi_k[k] + off_k[k] + 1] - st;
        }
        t.start[slot] = st;
        t.shift[slot] = pack_shift(shx_k[k], shy, shz);
        cnt[k] = c;
      }
    }
    int tot;
    const int ex = carry + warp_excl_scan(cnt[0] + cnt[1] + cnt[2], tot);
    if (r < rows) {
      t.pref[r * 3] = ex;
      t.pref[r * 3 + 1] = ex + cnt[0];
      t.pref[r * 3 + 2] = ex + cnt[0] + cnt[1];
    }
    carry += tot;
  }
  if (lane == 0) t.pref[rows * 3] = carry;
  __syncwarp();
  return rows * 3;
}

template <typename T>
struct Cplx;
template <>
struct Cplx<float> { using type = float2; };
template <>
struct Cplx<double> { using type = double2; };

// Lane layout constants of the warp-tiled spreading for support W.
template <int W>
struct WarpSpread {
  static constexpr int NP = W * W;           // (dy, dz) tap pairs
  static constexpr int NR = (NP + 31) / 32;  // rounds of pairs
  // The last, partly filled round of pairs leaves lanes idle for all W x
  // steps (W = 6: 4 of 36 pairs, 28 lanes idle).  When it is cheaper, those
  // REM pairs' REM * W taps are instead spread one tap per lane ("tail").
  static constexpr int NFULL = NP / 32, REM = NP % 32;
  static constexpr int NTAIL = (REM * W + 31) / 32;
  static constexpr bool kTail = REM > 0 && 12 * NTAIL < 12 + 5 * W;
  static constexpr int NRR = kTail ? NFULL : NR;  // rounds walked pair by pair
  static constexpr int NKV = (3 * W + 31) / 32;   // kernel-value registers per lane
};

// piecewise-polynomial kernel (kPoly): the coefficients of each lane's
// kernel-value slots (segment i of slot s = axis * W + i), loaded once per warp
template <typename T, int W, bool kPoly>
__device__ __forceinline__ void load_lane_poly(const T* __restrict__ poly,
                                               T (&pc)[kPoly ? WarpSpread<W>::NKV : 1][kPolyCoef]) {
  if constexpr (kPoly) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < WarpSpread<W>::NKV; k++) {
      const int sl = lane + 32 * k, i = sl % W;
#pragma unroll
      for (int n = 0; n < kPolyCoef; n++) pc[k][n] = (sl < 3 * W) ? poly[i * kPolyCoef + n] : (T)0;
    }
  }
}

// One warp tile (work item `item` of tiling tc): accumulate the tile in the
// warp's shared-memory region `wsmem` and write every cell of it to fw.
// kExactWrap: halo hive bounds from the wrapped cells (raw_hive_lo/hi), needed
// when an axis of the grid is not a multiple of 8 cells; otherwise floordiv8.
// part != nullptr: row chunk `chunk` of `nchunks` of the tile -- rows
// [total * chunk / nchunks, total * (chunk + 1) / nchunks) of its `total` --
// into a partial tile at part (cell (x, y, z) at (z * TY + y) * TX + x),
// written whole (zeros where no row reaches) instead of the grid cells.
template <typename T, int W, bool kPoly, bool kExactWrap>
__device__ __forceinline__ void grid_warp_tile(
    const Rec<T>* __restrict__ recs, const int* __restrict__ hive_start, const Geom& g,
    const WarpTile& tc, T* __restrict__ fw, int item, unsigned char* wsmem,
    const T (&pc)[kPoly ? WarpSpread<W>::NKV : 1][kPolyCoef], int chunk = 0, int nchunks = 1,
    typename Cplx<T>::type* __restrict__ part = nullptr) {
  using C = typename Cplx<T>::type;
  using WS = WarpSpread<W>;
  constexpr int lo = Halo<W>::lo, hi = Halo<W>::hi;
  constexpr int NP = WS::NP, NFULL = WS::NFULL, REM = WS::REM, NTAIL = WS::NTAIL;
  constexpr bool kTail = WS::kTail;
  constexpr int NRR = WS::NRR, NKV = WS::NKV;
  const int lane = threadIdx.x & 31;
  const int TX = tc.TX, TY = tc.TY, PB = tc.PB, RS = tc.RS, PS = tc.PS;
  C* acc = reinterpret_cast<C*>(wsmem);
  int* tb = reinterpret_cast<int*>(wsmem + (size_t)TY * RS * sizeof(C));
  const int ts = tc.slots + 1;
  SegTable t{tb, tb + ts, tb + 2 * ts};
  const T beta = (T)g.beta, c = (T)g.es_c, halfw = (T)W * (T)0.5;
  const int nf1 = g.nf1, nf2 = g.nf2, nw = g.nw;
  const size_t plane = (size_t)nf1 * nf2;
  C* fwc = reinterpret_cast<C*>(fw);
  const C zero = {(T)0, (T)0};
  {
    const int tix = item % tc.ntx, tiy = (item / tc.ntx) % tc.nty, tib = item / (tc.ntx * tc.nty);
    const int tx0 = tix * TX, ty0 = tiy * TY, p0 = tib * PB;
    const int tx1 = min(tx0 + TX, nf1), ty1 = min(ty0 + TY, nf2), p1 = min(p0 + PB, nw);
    const int wx = tx1 - tx0, wy = ty1 - ty0, wz = p1 - p0;
    auto zero_part = [&]() {
      for (int i = lane; i < TX * TY * PB; i += 32) part[i] = zero;
    };
    if (g.grid_skip) {  // a tile wholly outside the rows the transform reads holds no rows
      int r0, n;
      fft_row_band(g, r0, n);
      if (ty1 <= r0 || ty0 >= r0 + n) {
        if (part) zero_part();
        return;
      }
    }
    // FP32 cells are written two at a time (16 bytes) when every pair is aligned:
    // an even tile width and grid row length and a 16-byte aligned grid
    const bool flush_pairs = sizeof(T) == 4 && ((wx | nf1) & 1) == 0 &&
                             (reinterpret_cast<uintptr_t>(fw) & 15) == 0;
    int nslots;
    if constexpr (kExactWrap)
      nslots = warp_build_segments(
          g, hive_start, raw_hive_lo(tx0 - hi, nf1, g.nhx), raw_hive_hi(tx1 - 1 + lo, nf1, g.nhx),
          raw_hive_lo(ty0 - hi, nf2, g.nhy), raw_hive_hi(ty1 - 1 + lo, nf2, g.nhy), p0 - hi,
          p1 - 1 + lo, t);
    else
      nslots = warp_build_segments(g, hive_start, floordiv8(tx0 - hi), floordiv8(tx1 - 1 + lo),
                                   floordiv8(ty0 - hi), floordiv8(ty1 - 1 + lo), p0 - hi,
                                   p1 - 1 + lo, t);
    const int total = t.pref[nslots];
    __syncwarp();  // every lane has read the table head before it can be rebuilt
    int qb = 0, qe = total;  // the rows of this item
    if (part) {
      qb = (int)((int64_t)total * chunk / nchunks);
      qe = (int)((int64_t)total * (chunk + 1) / nchunks);
      if (qb == qe) {
        zero_part();
        return;
      }
    }
    if (total == 0) {
      if (flush_pairs) {
        const int hx = wx >> 1;
        const TileDiv div_x(hx), div_xy(hx * wy);
        for (int i = lane; i < hx * wy * wz; i += 32) {
          const int z = div_xy(i), r = i - z * hx * wy, y = div_x(r), x = 2 * (r - y * hx);
          *reinterpret_cast<float4*>(fwc + (size_t)(p0 + z) * plane + (size_t)(ty0 + y) * nf1 + tx0 + x) =
              make_float4(0.f, 0.f, 0.f, 0.f);
        }
        return;
      }
      const TileDiv div_x(wx), div_xy(wx * wy);
      for (int i = lane; i < wx * wy * wz; i += 32) {
        const int z = div_xy(i), r = i - z * wx * wy, y = div_x(r), x = r - y * wx;
        fwc[(size_t)(p0 + z) * plane + (size_t)(ty0 + y) * nf1 + tx0 + x] = zero;
      }
      return;
    }
    for (int i = lane; i < TY * RS; i += 32) acc[i] = zero;
    __syncwarp();
    // Candidates are pre-scanned 32 at a time (one per lane); the next
    // chunk's records are loaded while the current chunk is spread.  Within a
    // chunk, the next row's broadcast and kernel values are computed before
    // the current row's shared-memory updates, so the two overlap.
    struct Cand {
      T f0, f1, f2, c0, c1;
      int bx, by, bz;  // cell + periodic shift of the hive slot
      bool ok;
    };
    auto load_cand = [&](int q) {
      Cand cd{};
      cd.ok = q < qe;
      if (cd.ok) {
        const int sgi = find_segment(t.pref, nslots, q);
        const Rec<T> r = recs[t.start[sgi] + (q - t.pref[sgi])];
        cd.f0 = r.f[0]; cd.f1 = r.f[1]; cd.f2 = r.f[2]; cd.c0 = r.c[0]; cd.c1 = r.c[1];
        const int sc = t.shift[sgi];
        cd.bx = (int)(r.bxy & 0xFFFFu) + unpack_shift(sc, nf1);
        cd.by = (int)(r.bxy >> 16) + unpack_shift(sc >> 2, nf2);
        cd.bz = (int)r.bz + unpack_shift(sc >> 4, nw);
      }
      return cd;
    };
    struct Prep {
      T kv[NKV];
      T vr0, vi0;
      int vx, vy, vz;
    };
    Cand nextc = load_cand(qb + lane);
    for (int q0 = qb; q0 < qe; q0 += 32) {
      const Cand cc = nextc;
      if (q0 + 32 < qe) nextc = load_cand(q0 + 32 + lane);
      const int ox = cc.bx + tap_offset<W>(cc.f0);
      const int oy = cc.by + tap_offset<W>(cc.f1);
      const int oz = cc.bz + tap_offset<W>(cc.f2);
      const bool take = cc.ok && max(ox, tx0) < min(ox + W, tx1) &&
                        max(oy, ty0) < min(oy + W, ty1) && max(oz, p0) < min(oz + W, p1);
      unsigned mask = __ballot_sync(0xffffffffu, take);
      // broadcast of row `src` and its kernel values: lane slot s = axis * W + i, s < 3W
      auto prepare = [&](int src) {
        Prep pr;
        const T g0 = __shfl_sync(0xffffffffu, cc.f0, src), g1 = __shfl_sync(0xffffffffu, cc.f1, src);
        const T g2 = __shfl_sync(0xffffffffu, cc.f2, src);
        pr.vr0 = __shfl_sync(0xffffffffu, cc.c0, src);
        pr.vi0 = __shfl_sync(0xffffffffu, cc.c1, src);
        pr.vx = __shfl_sync(0xffffffffu, ox, src) - tx0;
        pr.vy = __shfl_sync(0xffffffffu, oy, src) - ty0;
        pr.vz = __shfl_sync(0xffffffffu, oz, src) - p0;
#pragma unroll
        for (int k = 0; k < NKV; k++) {
          const int sl = lane + 32 * k;
          const int axis = sl / W, i = sl - axis * W;
          const T f = axis == 0 ? g0 : (axis == 1 ? g1 : g2);
          if constexpr (kPoly)
            pr.kv[k] = (sl < 3 * W) ? poly_eval(pc[k], poly_arg<W>(f)) : (T)0;
          else
            pr.kv[k] = (sl < 3 * W) ? es_kernel<T>((T)(tap_offset<W>(f) + i) - f, beta, c, halfw) : (T)0;
        }
        return pr;
      };
      // spread one prepared row into the warp tile
      auto apply = [&](const Prep& cur) {
        const T* kv = cur.kv;
        const T vr0 = cur.vr0, vi0 = cur.vi0;
        const int vx = cur.vx, vy = cur.vy, vz = cur.vz;
        T kx[W];
#pragma unroll
        for (int e = 0; e < W; e++) kx[e] = __shfl_sync(0xffffffffu, kv[0], e);
        // x taps inside the tile: the bits xlo .. xhi-1 (a taken row overlaps it)
        const int xlo = max(0, -vx), xhi = min(W, wx - vx);
        const unsigned xmask = ((1u << xhi) - 1u) & ~((1u << xlo) - 1u);
#pragma unroll
        for (int rr = 0; rr < NRR; rr++) {
          const int pp = lane + 32 * rr;
          const int dz = pp % W, dy = pp / W;  // lane = dy * W + dz = cell offset (mod 16)
          const T ky = __shfl_sync(0xffffffffu, kv[0], W + dy);
          const int zs = 2 * W + dz;
          T kz = __shfl_sync(0xffffffffu, kv[0], zs & 31);
          if (NKV > 1) {
            const T kz1 = __shfl_sync(0xffffffffu, kv[NKV - 1], zs & 31);
            kz = zs >= 32 ? kz1 : kz;
          }
          const int y = vy + dy, z = vz + dz;
          if (pp < NP && y >= 0 && y < wy && z >= 0 && z < wz) {
            const T k = ky * kz;
            const T vr = vr0 * k, vi = vi0 * k;
            C* a = acc + z * PS + y * RS + vx;
            // FP32 W <= 8 and FP64 W <= 6: the taps' loads first, then the
            // FMAs, then the stores (FP32 W = 6: 11.7 -> 11.0 ms at 4096^2 /
            // 20M rows).  Above that a load, FMA and store per tap: FP64
            // W = 10 with its loads first spilled and took twice as long, in
            // groups of 2 or 4 taps 107 and 94 ms against 93 per tap.
            constexpr bool kLoadFirst = sizeof(T) == 4 ? W <= 8 : W <= 6;
            if constexpr (kLoadFirst) {
              C cur[W];
#pragma unroll
              for (int e = 0; e < W; e++)
                if (xmask & (1u << e)) cur[e] = a[e];
#pragma unroll
              for (int e = 0; e < W; e++) {
                cur[e] = tap_fma(cur[e], vr, vi, kx[e]);
              }
#pragma unroll
              for (int e = 0; e < W; e++)
                if (xmask & (1u << e)) a[e] = cur[e];
            } else {
#pragma unroll
              for (int e = 0; e < W; e++) {
                if (xmask & (1u << e)) {
                  C cur = a[e];
                  cur = tap_fma(cur, vr, vi, kx[e]);
                  a[e] = cur;
                }
              }
            }
          }
        }
        if constexpr (kTail) {
          // lane -> (pair, x tap) of the remaining pairs; all cells distinct
#pragma unroll
          for (int it = 0; it < NTAIL; it++) {
            const int t = lane + 32 * it;
            const int pp = 32 * NFULL + t / W, e = t - (t / W) * W;
            const int dz = pp % W, dy = pp / W;
            const T ky = __shfl_sync(0xffffffffu, kv[0], W + dy);
            const int zs = 2 * W + dz;
            T kz = __shfl_sync(0xffffffffu, kv[0], zs & 31);
            if (NKV > 1) {
              const T kz1 = __shfl_sync(0xffffffffu, kv[NKV - 1], zs & 31);
              kz = zs >= 32 ? kz1 : kz;
            }
            const T kxe = __shfl_sync(0xffffffffu, kv[0], e);
            const int x = vx + e, y = vy + dy, z = vz + dz;
            if (t < REM * W && x >= 0 && x < wx && y >= 0 && y < wy && z >= 0 && z < wz) {
              const T k = ky * kz;
              const T vr = vr0 * k, vi = vi0 * k;
              C* a = acc + z * PS + y * RS + x;
              C cur = *a;
              cur = tap_fma(cur, vr, vi, kxe);
              *a = cur;
            }
          }
        }
      };
      if constexpr (kPoly) {
        // polynomial kernel values are cheap: no look-ahead
        while (mask) {
          const Prep cur = prepare(__ffs(mask) - 1);
          mask &= mask - 1;
          apply(cur);
          __syncwarp();
        }
      } else {
        // ES values (exp, sqrt) of the next row are computed ahead
        if (!mask) continue;
        Prep cur = prepare(__ffs(mask) - 1);
        mask &= mask - 1;
        while (true) {
          const bool more = mask != 0;
          Prep nxt;
          if (more) {
            nxt = prepare(__ffs(mask) - 1);
            mask &= mask - 1;
          }
          apply(cur);
          __syncwarp();
          if (!more) break;
          cur = nxt;
        }
      }
    }
    // flush the tile, coalesced along x
    if (part) {
      const TileDiv div_x(TX), div_xy(TX * TY);
      for (int i = lane; i < TX * TY * PB; i += 32) {
        const int z = div_xy(i), r = i - z * TX * TY, y = div_x(r), x = r - y * TX;
        part[i] = acc[z * PS + y * RS + x];
      }
    } else if (flush_pairs) {
      const int hx = wx >> 1;
      const TileDiv div_x(hx), div_xy(hx * wy);
      for (int i = lane; i < hx * wy * wz; i += 32) {
        const int z = div_xy(i), r = i - z * hx * wy, y = div_x(r), x = 2 * (r - y * hx);
        const C* a = acc + z * PS + y * RS + x;
        const C a0 = a[0], a1 = a[1];
        *reinterpret_cast<float4*>(fwc + (size_t)(p0 + z) * plane + (size_t)(ty0 + y) * nf1 + tx0 + x) =
            make_float4((float)a0.x, (float)a0.y, (float)a1.x, (float)a1.y);
      }
    } else {
      const TileDiv div_x(wx), div_xy(wx * wy);
      for (int i = lane; i < wx * wy * wz; i += 32) {
        const int z = div_xy(i), r = i - z * wx * wy, y = div_x(r), x = r - y * wx;
        fwc[(size_t)(p0 + z) * plane + (size_t)(ty0 + y) * nf1 + tx0 + x] = acc[z * PS + y * RS + x];
      }
    }
    __syncwarp();
  }
}

// Tile t of chunk slot `slot` (chunk_off: exclusive scan of the tiles'
// chunks, entry nitems = their total, slot below it): the last t with
// chunk_off[t] <= slot.
__device__ __forceinline__ int chunk_tile(const int* __restrict__ chunk_off, int nitems, int slot) {
  int lo = 0, hi = nitems;  // chunk_off[lo] <= slot < chunk_off[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (chunk_off[mid] <= slot) lo = mid; else hi = mid;
  }
  return lo;
}

// With row splitting (chunk_off set), warps first take chunk slots below
// min(cap, chunks' total) from an atomic queue: slot s is chunk
// s - chunk_off[t] of tile t, into partial tile s, when all of t's chunks fit
// below cap.  Then each warp takes every nwarps-th tile, as without
// splitting, and skips the tiles whose chunks ran.  The static stride keeps
// a CTA's warps on neighbouring tiles, which share halo rows in L1: an atomic
// queue over the tiles too took FP64 W = 10 gridding at 4096^2 from 93 to
// 108 ms.
template <typename T, int W, bool kPoly, bool kExactWrap>
__global__ void __launch_bounds__(512) k_grid_warp(const Rec<T>* __restrict__ recs,
                                                   const int* __restrict__ hive_start, Geom g,
                                                   WarpTile tc, T* __restrict__ fw,
                                                   int* __restrict__ counter,
                                                   const int* __restrict__ chunk_off, int cap,
                                                   typename Cplx<T>::type* __restrict__ parts) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  T pc[kPoly ? WarpSpread<W>::NKV : 1][kPolyCoef];
  load_lane_poly<T, W, kPoly>(geom_poly<T>(g), pc);
  unsigned char* wsmem = smem + (size_t)wib * tc.warp_bytes;
  const int nslot = chunk_off ? min(cap, chunk_off[tc.nitems]) : 0;
  const size_t slot_cells = (size_t)tc.TX * tc.TY * tc.PB;
  const int nwarps = gridDim.x * tc.warps;
  bool chunks = nslot > 0;
  int next = blockIdx.x * tc.warps + wib;  // this warp's next tile of the tile pass
  // one call site of the (large, inlined) tile routine for both passes
  for (;;) {
    int t, chunk = 0, nchunks = 1;
    typename Cplx<T>::type* part = nullptr;
    if (chunks) {
      int item = 0;
      if (lane == 0) item = atomicAdd(counter, 1);
      item = __shfl_sync(0xffffffffu, item, 0);
      if (item >= nslot) {
        chunks = false;
        continue;
      }
      t = chunk_tile(chunk_off, tc.nitems, item);
      const int k0 = chunk_off[t], k1 = chunk_off[t + 1];
      if (k1 > cap) continue;  // the tile's chunks do not fit: gridded whole below
      chunk = item - k0;
      nchunks = k1 - k0;
      part = parts + (size_t)item * slot_cells;
    } else {
      if (next >= tc.nitems) break;
      t = next;
      next += nwarps;
      if (chunk_off) {
        const int k0 = chunk_off[t], k1 = chunk_off[t + 1];
        if (k1 > k0 && k1 <= cap) continue;  // gridded by its chunks
      }
    }
    grid_warp_tile<T, W, kPoly, kExactWrap>(recs, hive_start, g, tc, fw, t, wsmem, pc, chunk, nchunks,
                                            part);
  }
}

// Chunks of each warp tile: 0 for a tile with at most R rows in its hive
// slots, else ceil(rows / R), at most kMaxTileChunks; entry nitems is 0 (the
// scan then leaves the chunks' total there).
constexpr int kMaxTileChunks = 1024;
__global__ void k_tile_chunks(const int* __restrict__ hive_start, Geom g, WarpTile tc, int R,
                              int* __restrict__ chunks) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t > tc.nitems) return;
  if (t == tc.nitems) {
    chunks[t] = 0;
    return;
  }
  const int64_t rows = tile_slot_rows(hive_start, g, tc, t);
  chunks[t] = rows > R ? (int)min((rows + R - 1) / R, (int64_t)kMaxTileChunks) : 0;
}

// Sum of a split tile's nchunks partial tiles (base: chunk 0; chunks
// slot_cells apart) in chunk order, into the tile's grid cells.
template <typename T>
__device__ __forceinline__ void split_reduce_tile(const WarpTile& tc, const Geom& g, int item,
                                                  const typename Cplx<T>::type* __restrict__ base,
                                                  int nchunks, T* __restrict__ fw) {
  using C = typename Cplx<T>::type;
  const int tix = item % tc.ntx, tiy = (item / tc.ntx) % tc.nty, tib = item / (tc.ntx * tc.nty);
  const int tx0 = tix * tc.TX, ty0 = tiy * tc.TY, p0 = tib * tc.PB;
  const int wx = min(tx0 + tc.TX, g.nf1) - tx0, wy = min(ty0 + tc.TY, g.nf2) - ty0;
  const int wz = min(p0 + tc.PB, g.nw) - p0;
  const size_t slot = (size_t)tc.TX * tc.TY * tc.PB;
  const size_t plane = (size_t)g.nf1 * g.nf2;
  C* fwc = reinterpret_cast<C*>(fw);
  for (int i = threadIdx.x; i < wx * wy * wz; i += blockDim.x) {
    const int z = i / (wx * wy), r = i - z * wx * wy, y = r / wx, x = r - y * wx;
    const size_t cell = ((size_t)z * tc.TY + y) * tc.TX + x;
    C s = base[cell];
    for (int k = 1; k < nchunks; k++) {
      const C v = base[(size_t)k * slot + cell];
      s.x += v.x;
      s.y += v.y;
    }
    fwc[(size_t)(p0 + z) * plane + (size_t)(ty0 + y) * g.nf1 + tx0 + x] = s;
  }
}

// One block per chunk slot below cap; the block of a split tile's chunk 0
// reduces the tile.
template <typename T>
__global__ void __launch_bounds__(256) k_split_reduce_plan(const int* __restrict__ chunk_off,
                                                           WarpTile tc, Geom g, int cap,
                                                           const typename Cplx<T>::type* __restrict__ parts,
                                                           T* __restrict__ fw) {
  const int s = blockIdx.x;
  if (s >= chunk_off[tc.nitems]) return;
  const int t = chunk_tile(chunk_off, tc.nitems, s);
  const int k0 = chunk_off[t], k1 = chunk_off[t + 1];
  if (s != k0 || k1 > cap) return;
  split_reduce_tile<T>(tc, g, t, parts + (size_t)k0 * tc.TX * tc.TY * tc.PB, k1 - k0, fw);
}

// index of the job holding global work item `item` (item0 ascending, item0[0] = 0)
template <typename J, typename F>
__device__ __forceinline__ int find_job(const J* __restrict__ jobs, int njobs, int item, F item0) {
  int lo = 0, hi = njobs;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (item0(jobs[mid]) <= item) lo = mid; else hi = mid;
  }
  return lo;
}

// Many grids in one persistent launch: warps take (job, tile) items from a
// global queue; every job shares W and the kernel.  warp_bytes is the largest
// per-warp footprint of the jobs' tilings.
// Items [0, nsplit) are the row chunks of the heavy tiles (splits), the
// others the jobs' tiles in job order; a tile with split chunks is skipped
// there.
template <typename T, int W, bool kPoly, bool kExactWrap>
__global__ void __launch_bounds__(512) k_grid_warp_multi(const GridJob<T>* __restrict__ jobs,
                                                         int njobs, int nitems, size_t warp_bytes,
                                                         int* __restrict__ counter,
                                                         const SplitItem* __restrict__ splits,
                                                         int nsplit,
                                                         typename Cplx<T>::type* __restrict__ parts) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  T pc[kPoly ? WarpSpread<W>::NKV : 1][kPolyCoef];
  load_lane_poly<T, W, kPoly>(geom_poly<T>(jobs[0].g), pc);
  unsigned char* wsmem = smem + (size_t)wib * warp_bytes;
  for (;;) {
    int item = 0;
    if (lane == 0) item = atomicAdd(counter, 1);
    item = __shfl_sync(0xffffffffu, item, 0);
    if (item >= nsplit + nitems) break;
    // one call site of the (large, inlined) tile routine for chunks and tiles
    int j, tile, chunk = 0, nchunks = 1;
    typename Cplx<T>::type* part = nullptr;
    if (item < nsplit) {
      const SplitItem si = splits[item];
      j = si.job;
      tile = si.tile;
      chunk = si.chunk;
      nchunks = si.nchunks;
      part = parts + si.off;
    } else {
      item -= nsplit;
      j = find_job(jobs, njobs, item, [](const GridJob<T>& x) { return x.grid_item0; });
      tile = item - jobs[j].grid_item0;
      if (jobs[j].tile_split && jobs[j].tile_split[tile]) continue;  // gridded by its split items
    }
    const GridJob<T>& J = jobs[j];
    grid_warp_tile<T, W, kPoly, kExactWrap>(J.recs, J.hive_start, J.g, J.wt, J.fw, tile, wsmem, pc,
                                            chunk, nchunks, part);
  }
}

// Sum of the partial tiles of each split tile (tiles[blockIdx.x]: chunk 0 of
// its nchunks, chunks at consecutive slots) in chunk order, into its cells.
template <typename T>
__global__ void __launch_bounds__(256) k_split_reduce(const GridJob<T>* __restrict__ jobs,
                                                      const SplitItem* __restrict__ tiles,
                                                      const typename Cplx<T>::type* __restrict__ parts) {
  const SplitItem si = tiles[blockIdx.x];
  const GridJob<T>& J = jobs[si.job];
  split_reduce_tile<T>(J.wt, J.g, si.tile, parts + si.off, si.nchunks, J.fw);
}

// ---------------------------------------------------------------- degridding
// One degridding tile (work item `item` of tiling tc), staged in `smem`.
// Called by every thread of the block with the same item.
template <typename T, int W>
__device__ __forceinline__ void degrid_tile(const Rec<T>* __restrict__ recs,
                                            const int* __restrict__ perm,
                                            const int* __restrict__ hive_start, int64_t M,
                                            const Geom& g, const TileCfg& tc, int nslots_max,
                                            const T* __restrict__ fw, T* __restrict__ vis,
                                            int item, unsigned char* smem, int* s_warp) {
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
  SegTable t{tb, tb + ts, tb + 2 * ts};
  const T beta = (T)g.beta, c = (T)g.es_c;
  const T* __restrict__ poly = geom_poly<T>(g);
  const size_t plane = (size_t)nf1 * nf2;
  {
    const int tix = tc.bx0 + item % tc.ntx, tiy = tc.by0 + (item / tc.ntx) % tc.nty,
              tib = item / (tc.ntx * tc.nty);
    const int tx0 = tix * TX, ty0 = tiy * TY, p0 = all_planes ? 0 : tib * PB;
    const int tx1 = min(tx0 + TX, nf1), ty1 = min(ty0 + TY, nf2);
    const int p1 = all_planes ? nw : min(p0 + PB, nw);
    const int gx0 = tx0 - lo, gy0 = ty0 - lo, gz0 = all_planes ? 0 : p0 - lo;
    // runs of the tile's own hives (each row belongs to exactly one tile)
    const int nslots = build_segments(g, hive_start, tx0 >> 3, (tx1 - 1) >> 3, ty0 >> 3,
                                      (ty1 - 1) >> 3, p0, p1 - 1, t, s_warp);
    const int total = t.pref[nslots];
    if (total == 0) return;  // uniform across the block: nothing to interpolate here
    // stage the tile + halo (periodic); row stride SXP = SX + 1 complex
    using V = typename std::conditional<sizeof(T) == 4, float2, double2>::type;
    V* stv = reinterpret_cast<V*>(stg);
    const V* fwv = reinterpret_cast<const V*>(fw);
    const TileDiv div_x(SX), div_xy(SX * SY);
    for (int i = threadIdx.x; i < nstage; i += blockDim.x) {
      const int sz = div_xy(i), r = i - sz * SX * SY, sy = div_x(r), sx = r - sy * SX;
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
      const int lx = bx + taps<T, W>(r.f[0], beta, c, poly, kx) - gx0;
      const int ly = by + taps<T, W>(r.f[1], beta, c, poly, ky) - gy0;
      const int lz = bz + taps<T, W>(r.f[2], beta, c, poly, kz) - gz0;
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

template <typename T, int W>
__global__ void __launch_bounds__(512) k_degrid_tiled(const Rec<T>* __restrict__ recs,
                                                      const int* __restrict__ perm,
                                                      const int* __restrict__ hive_start, int64_t M,
                                                      Geom g, TileCfg tc, int nslots_max,
                                                      const T* __restrict__ fw,
                                                      T* __restrict__ vis, int* __restrict__ counter) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_warp[33];
  __shared__ int s_item;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int item = s_item;
    if (item >= tc.nitems) break;
    // the tile's first block-wide barrier orders this read before the next write of s_item
    degrid_tile<T, W>(recs, perm, hive_start, M, g, tc, nslots_max, fw, vis, item, smem, s_warp);
  }
}

// Many grids in one persistent launch: blocks take (job, tile) items from a
// global queue; every job shares W and the kernel, smem is the largest
// footprint of the jobs' tilings.
template <typename T, int W>
__global__ void __launch_bounds__(512, sizeof(T) == 4 ? 2 : 1) k_degrid_tiled_multi(const GridJob<T>* __restrict__ jobs,
                                                            int njobs, int nitems,
                                                            int* __restrict__ counter) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_warp[33];
  __shared__ int s_item;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int item = s_item;
    if (item >= nitems) break;
    const int j = find_job(jobs, njobs, item, [](const GridJob<T>& x) { return x.degrid_item0; });
    const GridJob<T>& J = jobs[j];
    degrid_tile<T, W>(J.recs, J.perm, J.hive_start, J.M, J.g, J.dt, J.nslots, J.fw, J.vis,
                      item - J.degrid_item0, smem, s_warp);
  }
}

// ======================================================================= launch
static int slots_for(int TY, int PB, int W) { return ((TY >> 3) + 2) * (PB + W + 1) * 3; }

// Tile shape: 32 x 32 cells by default, the plane batch covering all planes
// when the shared-memory footprint allows, otherwise halved until it fits.
// CG_TILE_X / CG_TILE_Y / CG_TILE_PLANES / CG_TILE_THREADS override (tuning).
template <typename T>
TileCfg grid_tiling(const Geom& g, bool degrid, const TileTune* tt) {
  const size_t budget = 220 * 1024;
  const int W = g.kw;
  TileCfg tc{};
  // degridding: 32 x 16 tiles keep two CTAs per SM for FP32 at W <= 7 (one
  // stages its tile while the other interpolates); 32 x 32 left one CTA per SM
  int TX = env_int("CG_TILE_X", 32), TY = env_int("CG_TILE_Y", degrid ? 16 : 32);
  int PB = env_int("CG_TILE_PLANES", 0);
  int threads = env_int("CG_TILE_THREADS", 512);
  if (tt && degrid) {
    if (tt->dx > 0) TX = tt->dx;
    if (tt->dy > 0) TY = tt->dy;
    if (tt->dpb > 0) PB = tt->dpb;
    if (tt->dthreads > 0) threads = tt->dthreads;
  }
  TX = std::max(8, (TX / 8) * 8);
  TY = std::max(8, (TY / 8) * 8);
  threads = std::min(512, std::max(64, (threads / 32) * 32));
  auto bytes = [&](int tx, int ty, int pb) -> size_t {
    size_t cells = degrid ? (size_t)(tx + W + 1) * (ty + W) * (pb >= g.nw ? g.nw : pb + W)
                          : (size_t)(tx + 8) * ty * pb;
    return cells * 2 * sizeof(T) + (size_t)(slots_for(ty, pb, W) + 1) * 4 * kSegInts;
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
  // degridding: only the tiles of the cells the data can reach (the full grid
  // when the data wraps around an edge); the others hold no rows
  if (degrid && 0 <= g.band_c0 && g.band_c0 <= g.band_c1 && g.band_c1 < g.nf1) {
    tc.bx0 = g.band_c0 / TX;
    tc.ntx = g.band_c1 / TX - tc.bx0 + 1;
  }
  if (degrid && 0 <= g.band_r0 && g.band_r0 <= g.band_r1 && g.band_r1 < g.nf2) {
    tc.by0 = g.band_r0 / TY;
    tc.nty = g.band_r1 / TY - tc.by0 + 1;
  }
  tc.npb = (g.nw + PB - 1) / PB;
  tc.nitems = tc.ntx * tc.nty * tc.npb;
  tc.threads = threads;
  tc.smem = bytes(TX, TY, PB);
  return tc;
}

int degrid_slots(const TileCfg& tc, int W) { return slots_for(tc.TY, tc.PB, W); }

// Autotuner candidates.  Gridding warp tiles (x, y, planes, warps per CTA):
// planes 64 = all planes of the grid; 0 = the default.  Degridding tiles
// (x, y, planes, threads per CTA).  The first of each list is the default.
// x = -1: the x-sliding windows (cg_grid_slide.cu) with y band rows, planes =
// hive columns per segment.
static const int kGridCand[][4] = {{16, 16, 0, 0},  {16, 8, 0, 0},   {16, 8, 64, 0},
                                   {16, 8, 64, 12}, {16, 16, 64, 0}, {32, 8, 0, 0},
                                   {16, 16, 5, 16}, {16, 16, 0, 12}, {16, 8, 10, 16},
                                   {16, 8, 13, 12}, {16, 16, 8, 10}, {16, 8, 64, 13},
                                   {16, 8, 64, 14}, {-1, 8, 8, 0},   {-1, 8, 12, 0},
                                   {-1, 8, 16, 0},  {-1, 8, 10, 0},  {-1, 8, 12, 14},
                                   {-1, 8, 16, 14}};
// threads -1 .. -4: the TMA-staged kernel's variants (all planes; 32 x 16
// tiles with 512 threads and two stages / 256 threads and one stage; 32 x 8
// and 16 x 8 tiles with 128 threads and one stage) where they apply.
static const int kDegridCand[][4] = {{32, 16, 0, 512}, {32, 32, 0, 512}, {32, 8, 0, 512},
                                     {16, 16, 0, 512}, {64, 16, 0, 512}, {32, 16, 0, 256},
                                     {16, 16, 0, 256}, {32, 16, 8, 512}, {32, 16, 0, -1},
                                     {32, 16, 0, -2}, {32, 8, 0, -3}, {16, 8, 0, -4}};

int tile_candidates(int dir, const int (**cand)[4]) {
  if (dir == 0) {
    *cand = kGridCand;
    return (int)(sizeof(kGridCand) / sizeof(kGridCand[0]));
  }
  *cand = kDegridCand;
  return (int)(sizeof(kDegridCand) / sizeof(kDegridCand[0]));
}

void set_tile_candidate(TileTune& tt, int dir, const int* c) {
  if (dir == 0) {
    tt.wx = c[0]; tt.wy = c[1]; tt.wpb = c[2]; tt.warps = c[3];
  } else {
    tt.dx = c[0]; tt.dy = c[1]; tt.dpb = c[2]; tt.dthreads = c[3];
  }
}

// dynamic shared memory of one warp-tiled gridding CTA at most (the SM
// offers 227 KB to one CTA)
constexpr size_t kWarpSmemMax = 227 * 1024;

// Warp tiles: shape from the tuned fields, CG_WTILE_X / CG_WTILE_Y /
// CG_WTILE_PLANES / CG_WTILE_WARPS, else the defaults below.
template <typename T>
WarpTile warp_tiling(const Geom& g, const TileTune* tt) {
  WarpTile tc{};
  const int W = g.kw;
  // An untuned plan (no field set) gets the shape the autotuner picks for
  // dense data: 16 x 8 cells, every plane, as many warps as fit up to 12.
  // The fields a tuning candidate leaves at 0 keep their candidate-list
  // meaning: 16 x 16 cells, 7 planes, warps up to 8 in 110 KB.
  const bool cand = tt && (tt->wx || tt->wy || tt->wpb || tt->warps);
  int tx = env_int("CG_WTILE_X", 16), ty = env_int("CG_WTILE_Y", cand ? 16 : 8);
  int PB = env_int("CG_WTILE_PLANES", 0);
  int warps = env_int("CG_WTILE_WARPS", 0);
  if (tt) {
    if (tt->wx > 0) tx = tt->wx;
    if (tt->wy > 0) ty = tt->wy;
    if (tt->wpb > 0) PB = tt->wpb;
    if (tt->warps > 0) warps = tt->warps;
  }
  tc.TX = std::max(16, (tx / 16) * 16);
  tc.TY = std::max(8, (ty / 8) * 8);
  tc.PS = tc.TX + 1;  // = 1 (mod 16): consecutive dz of a lane group hit consecutive banks
  if (PB <= 0) PB = cand ? std::min(g.nw, 7) : g.nw;
  PB = std::min(PB, g.nw);
  tc.PB = PB;
  int rs = PB * tc.PS;
  rs += ((W % 16) - (rs % 16) + 16) % 16;  // RS = W (mod 16): consecutive dy, W lanes apart
  tc.RS = rs;
  // hive rows of a tile: (TY / 8 + 2) along y, one more when the last hive row
  // is partial (its low halo then spans two hive rows), times PB + halo
  // planes, 3 runs each
  tc.slots = ((tc.TY >> 3) + 2 + (g.nf2 % 8 != 0)) * (PB + (W - 1) / 2 + (W + 1) / 2) * 3;
  tc.warp_bytes =
      ((size_t)tc.TY * tc.RS * 2 * sizeof(T) + (size_t)(tc.slots + 1) * kSegInts * 4 + 15) & ~(size_t)15;
  if (warps <= 0)
    warps = cand ? (int)std::max<size_t>(1, std::min<size_t>(8, (110 * 1024) / tc.warp_bytes))
                 : (int)std::max<size_t>(1, std::min<size_t>(12, kWarpSmemMax / tc.warp_bytes));
  warps = std::min(warps, 16);
  while (warps > 1 && tc.warp_bytes * warps > kWarpSmemMax) warps--;
  tc.warps = warps;
  tc.smem = tc.warp_bytes * warps;
  tc.ntx = (g.nf1 + tc.TX - 1) / tc.TX;
  tc.nty = (g.nf2 + tc.TY - 1) / tc.TY;
  tc.npb = (g.nw + PB - 1) / PB;
  tc.nitems = tc.ntx * tc.nty * tc.npb;
  return tc;
}

template <typename T, int W>
static int grid_w(const Rec<T>* d_recs, const int* d_hive_start, int64_t M, const Geom& g, T* d_fw,
                  int method, int* d_counter, cudaStream_t st, const TileTune* tt,
                  const SplitScratch* sp) {
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
  // x-sliding windows: a tuning candidate with wx < 0, or CG_GRID_SLIDE=1
  if ((tt && tt->wx < 0) || env_int("CG_GRID_SLIDE", 0)) {
    const int s = launch_grid_slide<T>(d_recs, d_hive_start, g, d_fw, d_counter, st, tt);
    if (s != CG_ERR_ARG || (tt && tt->wx < 0)) return s;
  }
  WarpTile tc = warp_tiling<T>(g, tt);
  const bool exact = (g.nf1 % 8) != 0 || (g.nf2 % 8) != 0;
  auto* kern = geom_poly_host<T>(g) ? (exact ? k_grid_warp<T, W, true, true> : k_grid_warp<T, W, true, false>)
                                    : (exact ? k_grid_warp<T, W, false, true> : k_grid_warp<T, W, false, false>);
  int per_sm = 0;
  CG_CUDA(kernel_occupancy((const void*)kern, tc.warps * 32, tc.smem, &per_sm));
  if (per_sm < 1) {
    set_last_error("warp-tiled gridding does not fit on an SM");
    return CG_ERR_ARG;
  }
  const int blocks = per_sm * num_sms();
  // Row split: a warp grids one tile's rows alone, so a tile holding far more
  // than a warp's share of the launch (the centre of a dense small grid) sets
  // its length.  A tile with more than R rows in its hive slots, R about a
  // quarter of a warp's share (each row sits in about 8 tiles' slots), runs
  // as ceil(rows / R) chunks into partial tiles that k_split_reduce_plan sums
  // in chunk order.  CG_SPLIT=0 turns it off, CG_SPLIT_ROWS sets R.
  using C = typename Cplx<T>::type;
  const int* chunk_off = nullptr;
  int cap = 0;
  C* parts = nullptr;
  if (sp && env_int("CG_SPLIT", 1) && tc.nitems > 0 && M > 0) {
    const int64_t warps = (int64_t)blocks * tc.warps;
    int64_t R = std::max<int64_t>(2048, (2 * M + warps - 1) / warps);
    if (const char* e = getenv("CG_SPLIT_ROWS")) R = std::max<int64_t>(1, atoll(e));
    R = std::min<int64_t>(R, 2147483647);
    const size_t slot_bytes = (size_t)tc.TX * tc.TY * tc.PB * sizeof(C);
    cap = (int)std::max<size_t>(64, ((size_t)64 << 20) / slot_bytes);  // 64 MB of partial tiles
    CG_TRY(ensure(*sp->chunks, (size_t)(tc.nitems + 1) * sizeof(int)));
    CG_TRY(ensure(*sp->sums, (size_t)hive_sums_ints(tc.nitems) * sizeof(int)));
    CG_TRY(ensure(*sp->parts, (size_t)cap * slot_bytes));
    int* chunks = (int*)sp->chunks->p;
    k_tile_chunks<<<(tc.nitems + 1 + 255) / 256, 256, 0, st>>>(d_hive_start, g, tc, (int)R, chunks);
    count_launches(1);
    CG_CUDA(cudaGetLastError());
    CG_TRY(launch_scan_exclusive(chunks, (int64_t)tc.nitems + 1, chunks, (int*)sp->sums->p, st));
    chunk_off = chunks;
    parts = (C*)sp->parts->p;
  }
  if (chunk_off) CG_CUDA(cudaMemsetAsync(d_counter, 0, sizeof(int), st));
  kern<<<blocks, tc.warps * 32, tc.smem, st>>>(d_recs, d_hive_start, g, tc, d_fw, d_counter, chunk_off,
                                               cap, parts);
  count_launches(1);
  CG_CUDA(cudaGetLastError());
  if (chunk_off) {
    k_split_reduce_plan<T><<<cap, 256, 0, st>>>(chunk_off, tc, g, cap, parts, d_fw);
    count_launches(1);
    CG_CUDA(cudaGetLastError());
  }
  return CG_OK;
}

template <typename T, int W>
static int degrid_w(const Rec<T>* d_recs, const int* d_perm, const int* d_hive_start, int64_t M,
                    const Geom& g, const T* d_fw, T* d_vis, int method, int* d_counter,
                    cudaStream_t st, const TileTune* tt) {
  if (M == 0) return CG_OK;
  if (method == kGridDirect) {
    int blocks = (int)((M + 255) / 256);
    if (blocks > 148 * 64) blocks = 148 * 64;
    k_degrid_direct<T, W><<<blocks, 256, 0, st>>>(d_recs, d_perm, M, g, d_fw, d_vis);
    count_launches(1);
    CG_CUDA(cudaGetLastError());
    return CG_OK;
  }
  TileCfg tc = grid_tiling<T>(g, true, tt);
  int nslots = slots_for(tc.TY, tc.PB, W);
  int per_sm = 0;
  CG_CUDA(kernel_occupancy((const void*)k_degrid_tiled<T, W>, tc.threads, tc.smem, &per_sm));
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
                int method, int* d_counter, cudaStream_t st, const TileTune* tt,
                const SplitScratch* sp) {
  if (method == kGridMma) {
    // tensor-core path: FP32, ES kernel and W <= 8; everything else on the SIMT kernels
    if (sizeof(T) == 4 && !g.polyf) {
      int s = launch_grid_mma((const Rec<float>*)d_recs, d_hive_start, g, (float*)d_fw, st);
      if (s != CG_ERR_ARG) return s;
    }
    method = kGridTiled;
  }
#define CG_GRID_CALL(w) grid_w<T, w>(d_recs, d_hive_start, M, g, d_fw, method, d_counter, st, tt, sp)
  CG_W_SWITCH(g.kw, CG_GRID_CALL)
#undef CG_GRID_CALL
}

template <typename T>
int launch_degrid(const Rec<T>* d_recs, const int* d_perm, const int* d_hive_start, int64_t M,
                  const Geom& g, const T* d_fw, T* d_vis, int method, int* d_counter,
                  cudaStream_t st, const TileTune* tt) {
  if (method == kGridMma) method = kGridTiled;
#define CG_DEGRID_CALL(w) \
  degrid_w<T, w>(d_recs, d_perm, d_hive_start, M, g, d_fw, d_vis, method, d_counter, st, tt)
  CG_W_SWITCH(g.kw, CG_DEGRID_CALL)
#undef CG_DEGRID_CALL
}

// ================================================================== multi-grid
template <typename T>
int multi_shape(GridJob<T>* jobs, int njobs, MultiShape* sh) {
  if (njobs < 1) return CG_ERR_ARG;
  *sh = MultiShape{};
  sh->kw = jobs[0].g.kw;
  sh->poly = geom_poly_host<T>(jobs[0].g) != nullptr;
  sh->threads = jobs[0].dt.threads;
  int64_t gi = 0, di = 0;
  int warps = 16;
  // sliding-window gridding when every job has its window shape
  sh->slide = true;
  for (int j = 0; j < njobs; j++) sh->slide = sh->slide && jobs[j].st.TY > 0;
  for (int j = 0; j < njobs; j++) {
    GridJob<T>& J = jobs[j];
    if (J.g.kw != sh->kw || (geom_poly_host<T>(J.g) != nullptr) != sh->poly ||
        J.dt.threads != sh->threads) {
      set_last_error("multi-grid jobs differ in kernel width, kernel or threads");
      return CG_ERR_ARG;
    }
    J.grid_item0 = (int)gi;
    J.degrid_item0 = (int)di;
    gi += sh->slide ? J.st.nitems : J.wt.nitems;
    di += J.dt.nitems;
    sh->warp_bytes = std::max(sh->warp_bytes, sh->slide ? J.st.warp_bytes : J.wt.warp_bytes);
    if ((J.g.nf1 % 8) != 0 || (J.g.nf2 % 8) != 0) sh->partial_hives = true;
    sh->dsmem = std::max(sh->dsmem, J.dt.smem);
    warps = std::min(warps, sh->slide ? J.st.warps : J.wt.warps);
  }
  if (gi > 2147483647LL || di > 2147483647LL) return CG_ERR_SIZE;
  sh->grid_items = (int)gi;
  sh->degrid_items = (int)di;
  sh->warps = std::max(1, warps);
  while (sh->warps > 1 && sh->warp_bytes * sh->warps > kWarpSmemMax) sh->warps--;
  return CG_OK;
}

template <typename T, int W>
static int grid_multi_w(const GridJob<T>* d_jobs, int njobs, const MultiShape& sh, int* d_counter,
                        cudaStream_t st) {
  auto* kern = sh.poly ? (sh.partial_hives ? k_grid_warp_multi<T, W, true, true> : k_grid_warp_multi<T, W, true, false>)
                       : (sh.partial_hives ? k_grid_warp_multi<T, W, false, true> : k_grid_warp_multi<T, W, false, false>);
  const size_t smem = sh.warp_bytes * sh.warps;
  int per_sm = 0;
  CG_CUDA(kernel_occupancy((const void*)kern, sh.warps * 32, smem, &per_sm));
  if (per_sm < 1) {
    set_last_error("multi-grid gridding does not fit on an SM");
    return CG_ERR_ARG;
  }
  const int items = sh.grid_items + sh.nsplit;
  const int blocks = std::min((items + sh.warps - 1) / sh.warps, per_sm * num_sms());
  using C = typename Cplx<T>::type;
  CG_CUDA(cudaMemsetAsync(d_counter, 0, sizeof(int), st));
  kern<<<std::max(1, blocks), sh.warps * 32, smem, st>>>(d_jobs, njobs, sh.grid_items, sh.warp_bytes,
                                                         d_counter, sh.d_split, sh.nsplit,
                                                         (C*)sh.d_parts);
  count_launches(1);
  CG_CUDA(cudaGetLastError());
  if (sh.nsplit_tiles > 0) {
    k_split_reduce<T><<<sh.nsplit_tiles, 256, 0, st>>>(d_jobs, sh.d_split_tiles, (const C*)sh.d_parts);
    count_launches(1);
    CG_CUDA(cudaGetLastError());
  }
  return CG_OK;
}

template <typename T, int W>
static int degrid_multi_w(const GridJob<T>* d_jobs, int njobs, const MultiShape& sh,
                          int* d_counter, cudaStream_t st) {
  int per_sm = 0;
  CG_CUDA(kernel_occupancy((const void*)k_degrid_tiled_multi<T, W>, sh.threads, sh.dsmem, &per_sm));
  if (per_sm < 1) {
    set_last_error("multi-grid degridding does not fit on an SM");
    return CG_ERR_ARG;
  }
  const int blocks = std::min(sh.degrid_items, per_sm * num_sms());
  CG_CUDA(cudaMemsetAsync(d_counter, 0, sizeof(int), st));
  k_degrid_tiled_multi<T, W><<<std::max(1, blocks), sh.threads, sh.dsmem, st>>>(
      d_jobs, njobs, sh.degrid_items, d_counter);
  count_launches(1);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

template <typename T>
int launch_grid_multi(const GridJob<T>* d_jobs, int njobs, const MultiShape& sh, int* d_counter,
                      cudaStream_t st) {
  if (njobs < 1 || sh.grid_items < 1) return CG_OK;
  if (sh.slide) return launch_grid_slide_multi<T>(d_jobs, njobs, sh, d_counter, st);
#define CG_GRID_MULTI_CALL(w) grid_multi_w<T, w>(d_jobs, njobs, sh, d_counter, st)
  CG_W_SWITCH(sh.kw, CG_GRID_MULTI_CALL)
#undef CG_GRID_MULTI_CALL
}

template <typename T>
int launch_degrid_multi(const GridJob<T>* d_jobs, int njobs, const MultiShape& sh, int* d_counter,
                        cudaStream_t st) {
  if (njobs < 1 || sh.degrid_items < 1) return CG_OK;
#define CG_DEGRID_MULTI_CALL(w) degrid_multi_w<T, w>(d_jobs, njobs, sh, d_counter, st)
  CG_W_SWITCH(sh.kw, CG_DEGRID_MULTI_CALL)
#undef CG_DEGRID_MULTI_CALL
}

// ================================================================ plane windows
// Memory-limited mode: the grid holds only planes [p0, p1) (plane p at
// fwb + (p - p0) * plane).  Spreading skips taps outside the window; the
// interpolation adds each window's share of a row into vis, so a call
// visits every window once.  Sorted-stream order, one row per thread.
template <typename T, int W>
__global__ void __launch_bounds__(256) k_grid_window(const Rec<T>* __restrict__ recs, int64_t M,
                                                     Geom g, int p0, int p1, T* __restrict__ fwb) {
  const T beta = (T)g.beta, c = (T)g.es_c;
  const T* __restrict__ poly = geom_poly<T>(g);
  const int nf1 = g.nf1, nf2 = g.nf2, nw = g.nw;
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < M;
       s += (int64_t)gridDim.x * blockDim.x) {
    const Rec<T> r = recs[s];
    T kx[W], ky[W], kz[W];
    const int bx = (int)(r.bxy & 0xFFFFu), by = (int)(r.bxy >> 16), bz = (int)r.bz;
    if (bx >= nf1 || by >= nf2 || bz >= nw) continue;
    const int oz = bz + taps<T, W>(r.f[2], beta, c, poly, kz);
    bool any = false;
#pragma unroll
    for (int a = 0; a < W; a++) {
      const int zz = wrapi(oz + a, nw);
      any |= zz >= p0 && zz < p1;
    }
    if (!any) continue;
    const int ox = bx + taps<T, W>(r.f[0], beta, c, poly, kx);
    const int oy = by + taps<T, W>(r.f[1], beta, c, poly, ky);
#pragma unroll 1
    for (int a = 0; a < W; a++) {
      const int zz = wrapi(oz + a, nw);
      if (zz < p0 || zz >= p1) continue;
      const T cr = r.c[0] * kz[a], ci = r.c[1] * kz[a];
#pragma unroll 1
      for (int b = 0; b < W; b++) {
        const int yy = wrapi(oy + b, nf2);
        const T vr = cr * ky[b], vi = ci * ky[b];
        T* row = fwb + 2 * (((size_t)(zz - p0) * nf2 + yy) * nf1);
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
__global__ void __launch_bounds__(256) k_degrid_window(const Rec<T>* __restrict__ recs,
                                                       const int* __restrict__ perm, int64_t M,
                                                       Geom g, int p0, int p1,
                                                       const T* __restrict__ fwb,
                                                       T* __restrict__ vis) {
  const T beta = (T)g.beta, c = (T)g.es_c;
  const T* __restrict__ poly = geom_poly<T>(g);
  const int nf1 = g.nf1, nf2 = g.nf2, nw = g.nw;
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < M;
       s += (int64_t)gridDim.x * blockDim.x) {
    const Rec<T> r = recs[s];
    T kx[W], ky[W], kz[W];
    const int bx = (int)(r.bxy & 0xFFFFu), by = (int)(r.bxy >> 16), bz = (int)r.bz;
    if (bx >= nf1 || by >= nf2 || bz >= nw) continue;
    const int oz = bz + taps<T, W>(r.f[2], beta, c, poly, kz);
    bool any = false;
#pragma unroll
    for (int a = 0; a < W; a++) {
      const int zz = wrapi(oz + a, nw);
      any |= zz >= p0 && zz < p1;
    }
    if (!any) continue;
    const int ox = bx + taps<T, W>(r.f[0], beta, c, poly, kx);
    const int oy = by + taps<T, W>(r.f[1], beta, c, poly, ky);
    T sr = 0, si = 0;
#pragma unroll 1
    for (int a = 0; a < W; a++) {
      const int zz = wrapi(oz + a, nw);
      if (zz < p0 || zz >= p1) continue;
      T pr = 0, pi = 0;
#pragma unroll 1
      for (int b = 0; b < W; b++) {
        const int yy = wrapi(oy + b, nf2);
        const T* row = fwb + 2 * (((size_t)(zz - p0) * nf2 + yy) * nf1);
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
    vis[2 * i] += sr * r.c[0] - si * r.c[1];
    vis[2 * i + 1] += sr * r.c[1] + si * r.c[0];
  }
}

template <typename T>
int launch_grid_window(const Rec<T>* d_recs, int64_t M, const Geom& g, int p0, int p1, T* d_fwb,
                       cudaStream_t st) {
  CG_CUDA(cudaMemsetAsync(d_fwb, 0, (size_t)(p1 - p0) * g.nf1 * g.nf2 * 2 * sizeof(T), st));
  if (M == 0) return CG_OK;
  const int blocks = (int)std::min<int64_t>((M + 255) / 256, 148 * 64);
#define CG_GW_CALL(w)                                                              \
  (k_grid_window<T, w><<<blocks, 256, 0, st>>>(d_recs, M, g, p0, p1, d_fwb),     \
   count_launches(1), cudaGetLastError() == cudaSuccess ? CG_OK : CG_ERR_CUDA)
  CG_W_SWITCH(g.kw, CG_GW_CALL)
#undef CG_GW_CALL
}

template <typename T>
int launch_degrid_window(const Rec<T>* d_recs, const int* d_perm, int64_t M, const Geom& g,
                         int p0, int p1, const T* d_fwb, T* d_vis, cudaStream_t st) {
  if (M == 0) return CG_OK;
  const int blocks = (int)std::min<int64_t>((M + 255) / 256, 148 * 64);
#define CG_DW_CALL(w)                                                                         \
  (k_degrid_window<T, w><<<blocks, 256, 0, st>>>(d_recs, d_perm, M, g, p0, p1, d_fwb, d_vis), \
   count_launches(1), cudaGetLastError() == cudaSuccess ? CG_OK : CG_ERR_CUDA)
  CG_W_SWITCH(g.kw, CG_DW_CALL)
#undef CG_DW_CALL
}

template int launch_grid_window<float>(const Rec<float>*, int64_t, const Geom&, int, int, float*,
                                       cudaStream_t);
template int launch_grid_window<double>(const Rec<double>*, int64_t, const Geom&, int, int,
                                        double*, cudaStream_t);
template int launch_degrid_window<float>(const Rec<float>*, const int*, int64_t, const Geom&, int,
                                         int, const float*, float*, cudaStream_t);
template int launch_degrid_window<double>(const Rec<double>*, const int*, int64_t, const Geom&,
                                          int, int, const double*, double*, cudaStream_t);

template TileCfg grid_tiling<float>(const Geom&, bool, const TileTune*);
template TileCfg grid_tiling<double>(const Geom&, bool, const TileTune*);
template WarpTile warp_tiling<float>(const Geom&, const TileTune*);
template WarpTile warp_tiling<double>(const Geom&, const TileTune*);
template int multi_shape<float>(GridJob<float>*, int, MultiShape*);
template int multi_shape<double>(GridJob<double>*, int, MultiShape*);
template int launch_grid_multi<float>(const GridJob<float>*, int, const MultiShape&, int*,
                                      cudaStream_t);
template int launch_grid_multi<double>(const GridJob<double>*, int, const MultiShape&, int*,
                                       cudaStream_t);
template int launch_degrid_multi<float>(const GridJob<float>*, int, const MultiShape&, int*,
                                        cudaStream_t);
template int launch_degrid_multi<double>(const GridJob<double>*, int, const MultiShape&, int*,
                                         cudaStream_t);
template int launch_grid<float>(const Rec<float>*, const int*, int64_t, const Geom&, float*, int,
                                int*, cudaStream_t, const TileTune*, const SplitScratch*);
template int launch_grid<double>(const Rec<double>*, const int*, int64_t, const Geom&, double*, int,
                                 int*, cudaStream_t, const TileTune*, const SplitScratch*);
template int launch_degrid<float>(const Rec<float>*, const int*, const int*, int64_t, const Geom&,
                                  const float*, float*, int, int*, cudaStream_t, const TileTune*);
template int launch_degrid<double>(const Rec<double>*, const int*, const int*, int64_t,
                                   const Geom&, const double*, double*, int, int*, cudaStream_t,
                                   const TileTune*);

}  // namespace cg
