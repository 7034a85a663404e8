// Tile helpers shared by the tiled spreading / interpolation kernels: the
// kernel halo, and the segment table that lists a tile's sorted rows as
// contiguous runs of hives (with the periodic shift of each run).
#pragma once
#include "cg_internal.cuh"

namespace cg {

// halo of the taps: a row in cell b touches cells [b - lo, b + hi]
template <int W>
struct Halo {
  static constexpr int lo = (W - 1) / 2;
  static constexpr int hi = (W + 1) / 2;
};

__device__ __forceinline__ int floordiv8(int a) { return a >= 0 ? a >> 3 : -((7 - a) >> 3); }

// Raw hive bounds of the cells [a, b] of one axis that a tile and its kernel
// halo reach (the tile inside [0, nf), the halo outside it by less than nf),
// for build_segments' single periodic wrap of hive indices: a raw hive h < 0
// stands for hive h + nh with its cells shifted by -nf, a raw hive h >= nh for
// hive h - nh shifted by +nf.  The bounds come from the WRAPPED cells:
// cells a + nf .. nf - 1 below, 0 .. b - nf above.  When nf % 8 != 0 the last
// hive is partial and the low halo's wrapped cells can span two hives
// (nh - 2 and nh - 1), which floor(a / 8) would miss; when nf % 8 == 0 the
// bounds equal floordiv8(a) and floordiv8(b), which the gridding kernels then
// use instead (a separate instantiation, so that the common grid sizes keep
// the code generation they were tuned with).
__device__ __forceinline__ int raw_hive_lo(int a, int nf, int nh) {
  return a < 0 ? ((a + nf) >> 3) - nh : a >> 3;
}
__device__ __forceinline__ int raw_hive_hi(int b, int nf, int nh) {
  return b >= nf ? nh + ((b - nf) >> 3) : b >> 3;
}

// Rows in the hive slots of warp tile `item` of tiling wt (the hives of the
// tile and of its kernel halo, each counted once per periodic axis), from the
// exclusive hive offsets hs in (plane, hive row, hive column) order: the
// number of rows the tile's segment table lists, up to the partial-hive edge
// cases (it sets how many chunks a heavy tile is split into, nothing else).
__host__ __device__ inline int64_t tile_slot_rows(const int* hs, const Geom& g, const WarpTile& wt,
                                                  int item) {
  const int nhx = g.nhx, nhy = g.nhy, nhz = g.nhz;
  const int lo = (g.kw - 1) / 2, hi = (g.kw + 1) / 2;
  auto fdiv8 = [](int a) { return a >= 0 ? a >> 3 : -((7 - a) >> 3); };
  // [a, b] of a periodic axis of n as at most two intervals inside [0, n)
  auto wrap = [](int a, int b, int n, int* iv) {
    if (b - a + 1 >= n) {
      iv[0] = 0; iv[1] = n - 1;
      return 1;
    }
    a = ((a % n) + n) % n;
    b = ((b % n) + n) % n;
    if (a <= b) {
      iv[0] = a; iv[1] = b;
      return 1;
    }
    iv[0] = a; iv[1] = n - 1; iv[2] = 0; iv[3] = b;
    return 2;
  };
  const int tix = item % wt.ntx, tiy = (item / wt.ntx) % wt.nty, tib = item / (wt.ntx * wt.nty);
  const int tx0 = tix * wt.TX, ty0 = tiy * wt.TY, p0 = tib * wt.PB;
  const int tx1 = tx0 + wt.TX < g.nf1 ? tx0 + wt.TX : g.nf1;
  const int ty1 = ty0 + wt.TY < g.nf2 ? ty0 + wt.TY : g.nf2;
  const int p1 = p0 + wt.PB < g.nw ? p0 + wt.PB : g.nw;
  int ix[4], iy[4], iz[4];
  const int nx = wrap(fdiv8(tx0 - hi), fdiv8(tx1 - 1 + lo), nhx, ix);
  const int ny = wrap(fdiv8(ty0 - hi), fdiv8(ty1 - 1 + lo), nhy, iy);
  const int nz = wrap(p0 - hi, p1 - 1 + lo, nhz, iz);
  int64_t n = 0;
  for (int a = 0; a < nz; a++)
    for (int z = iz[2 * a]; z <= iz[2 * a + 1]; z++)
      for (int b = 0; b < ny; b++)
        for (int y = iy[2 * b]; y <= iy[2 * b + 1]; y++) {
          const int64_t r = ((int64_t)z * nhy + y) * nhx;
          for (int c = 0; c < nx; c++) n += hs[r + ix[2 * c + 1] + 1] - hs[r + ix[2 * c]];
        }
  return n;
}

// n / d for a tile index: 0 <= n, 0 < d, n * d < 2^32.  m = floor((2^32 - 1) / d) + 1
// exceeds 2^32 / d by e = m - 2^32 / d < 1, so n * m / 2^32 = n / d + n * e / 2^32 and
// the excess n * e / 2^32 < n / 2^32 < 1 / d never carries floor(n / d) over: the
// multiply-high is exact (d = 1 would overflow m and is answered directly).
struct TileDiv {
  unsigned m;
  int d;
  __device__ __forceinline__ explicit TileDiv(int d_) : m(0xFFFFFFFFu / (unsigned)d_ + 1u), d(d_) {}
  __device__ __forceinline__ int operator()(int n) const {
    return d == 1 ? n : (int)__umulhi((unsigned)n, m);
  }
};

// Segment table of one work item: contiguous runs of sorted rows (hives that
// are neighbours along x share one run) with the periodic shift of their cells.
struct SegTable {
  int* start;
  int* pref;   // exclusive prefix of the run lengths, pref[nslots] = total
  int* shift;  // periodic shift of the run's cells, 2 bits per axis (see pack_shift)
};
constexpr int kSegInts = 3;  // ints per slot of a segment table

// shift of one axis (0, -n or +n) as a 2-bit code, three axes in one int
__device__ __forceinline__ int shift_code(int s) { return s < 0 ? 1 : (s > 0 ? 2 : 0); }
__device__ __forceinline__ int pack_shift(int sx, int sy, int sz) {
  return shift_code(sx) | (shift_code(sy) << 2) | (shift_code(sz) << 4);
}
__device__ __forceinline__ int unpack_shift(int code, int n) {
  const int c = code & 3;
  return c == 1 ? -n : (c == 2 ? n : 0);
}

// Build the runs for hive rows hy in [hya, hyb], planes hz in [za, zb] (raw,
// possibly outside the grid: wrapped with a shift of -+nf / -+nw) and hive
// columns [hxa, hxb].  Three slots per (hz, hy) row (left wrap, inside, right
// wrap).  Returns the number of slots.  Must be called by all threads.
__device__ inline int build_segments(const Geom& g, const int* __restrict__ hive_start, int hxa, int hxb,
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
        t.shift[slot] = pack_shift(shx_k[k], shy, shz);
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

}  // namespace cg
