// Gridding (spreading) by x-sliding warp windows.
//
// Same sum as k_grid_warp (conv_3d_outputdriven_t1, conv.cu:522-627):
//   fw[p][g1][g0] = sum_j c_j phi(g0 - X0_j) phi(g1 - X1_j) phi(p - X2_j),
// periodic in all three axes, every grid cell written exactly once, no
// atomics, a deterministic result.
//
// Work item = (band of TY grid rows g1, segment of SEG hive columns along
// g0), all w planes.  The warp walks the segment's hive columns left to right
// (rows are sorted hive-major with the hive column fastest, so each hive of a
// column is one contiguous run of the sorted stream) and accumulates into a
// circular window of kXW = 16 columns x TY rows x nw planes in shared memory.
// A row in hive column c has its taps in cells [8c - lo, 8c + 7 + hi]; once
// column c is done, no later column reaches below 8(c + 1) - lo, so the 8
// cells [8c - 4, 8c + 4) are final (4 >= lo for W <= 8): they are flushed to
// HBM and their window slots zeroed.  The window then holds at most
// 8 + 4 + hi <= 16 columns, and a segment needs one warm-up column (c =
// first - 1) whose cells are not flushed.  Consequences against the tiled
// kernel: a row is visited once along x (only the band edges in g1 revisit
// it: (TY + W - 1) / TY visits), and along w every plane is resident, so the
// plane index wraps inside the lane instead of revisiting rows with a shift.
//
// Lanes take the (dy, dz) tap pairs of a row that fall inside the band: pair
// p = lane -> (dy, dz) = (dya + p / W, p % W), so a row that only partly
// overlaps the band needs one round of 32 pairs; the pairs beyond 32 are
// spread one tap per lane.  Cell (x, y, z) is at y * RS + z * PS + (x & 15)
// with PS = 17 and RS = W (mod 16): lane p then hits bank p + const (mod 16),
// conflict-free for every row whose taps do not wrap around the w axis.
//
// Applies to W in 4..8 with nf1 and nf2 multiples of 8 (whole hive columns
// and rows); launch_grid_slide returns CG_ERR_ARG otherwise and the plan
// keeps the tiled kernel.
#include <algorithm>
#include <cstdlib>

#include "cg_coords.cuh"
#include "cg_launch.cuh"
#include "cg_tiles.cuh"

namespace cg {
namespace {

constexpr int kXW = 16;      // window columns (circular)
constexpr int kPS = kXW + 1;  // plane stride (complex units)
constexpr int kFlushL = 4;    // flushed cells of column c: [8c - 4, 8c + 4)


template <typename T>
struct Cx;
template <>
struct Cx<float> { using type = float2; };
template <>
struct Cx<double> { using type = double2; };

__device__ __forceinline__ int warp_scan_excl(int x, int& total) {
  const int lane = threadIdx.x & 31;
  int inc = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  total = __shfl_sync(0xffffffffu, inc, 31);
  return inc - x;
}

// zero-fill the cells [x0, x0 + n) (n even, x0 even, may start below 0:
// wrapped) of rows [y0, y0 + wy) on every plane
template <typename T>
__device__ __forceinline__ void zero_region(T* __restrict__ fw, const Geom& g, int x0, int n, int y0,
                                            int wy) {
  using C = typename Cx<T>::type;
  C* fwc = reinterpret_cast<C*>(fw);
  const int lane = threadIdx.x & 31;
  const int np = n >> 1;
  const size_t plane = (size_t)g.nf1 * g.nf2;
  const int total = np * wy * g.nw;
  for (int i = lane; i < total; i += 32) {
    const int q = i % np, r = i / np, y = r % wy, z = r / wy;
    int x = x0 + 2 * q;
    if (x < 0) x += g.nf1;
    C* dst = fwc + (size_t)z * plane + (size_t)(y0 + y) * g.nf1 + x;
    if constexpr (sizeof(T) == 4) {
      *reinterpret_cast<float4*>(dst) = make_float4(0.f, 0.f, 0.f, 0.f);
    } else {
      dst[0] = make_double2(0.0, 0.0);
      dst[1] = make_double2(0.0, 0.0);
    }
  }
}

// per-lane candidate slot of the staging area: float: (f0, f1, f2, c0),
// (c1, ox, oy, oz) as two 16-byte words; double: four 16-byte words
template <typename T>
constexpr int kCandBytes = sizeof(T) == 4 ? 32 : 64;

template <typename T>
__device__ __forceinline__ void stage_cand(unsigned char* stg, int lane, T f0, T f1, T f2, T c0,
                                           T c1, int ox, int oy, int oz) {
  if constexpr (sizeof(T) == 4) {
    float4* c = reinterpret_cast<float4*>(stg) + 2 * lane;
    c[0] = make_float4(f0, f1, f2, c0);
    c[1] = make_float4(c1, __int_as_float(ox), __int_as_float(oy), __int_as_float(oz));
  } else {
    double2* c = reinterpret_cast<double2*>(stg) + 4 * lane;
    c[0] = make_double2(f0, f1);
    c[1] = make_double2(f2, c0);
    c[2] = make_double2(c1, 0.0);
    reinterpret_cast<int4*>(c + 3)[0] = make_int4(ox, oy, oz, 0);
  }
}

template <typename T>
__device__ __forceinline__ void read_cand(const unsigned char* stg, int src, T& f0, T& f1, T& f2,
                                          T& c0, T& c1, int& ox, int& oy, int& oz) {
  if constexpr (sizeof(T) == 4) {
    const float4* c = reinterpret_cast<const float4*>(stg) + 2 * src;
    const float4 a = c[0], b = c[1];
    f0 = a.x; f1 = a.y; f2 = a.z; c0 = a.w; c1 = b.x;
    ox = __float_as_int(b.y); oy = __float_as_int(b.z); oz = __float_as_int(b.w);
  } else {
    const double2* c = reinterpret_cast<const double2*>(stg) + 4 * src;
    const double2 a = c[0], b = c[1], d = c[2];
    const int4 o = reinterpret_cast<const int4*>(c + 3)[0];
    f0 = a.x; f1 = a.y; f2 = b.x; c0 = b.y; c1 = d.x;
    ox = o.x; oy = o.y; oz = o.z;
  }
}

// the x kernel values kvs[0 .. 7] (W <= 8) with 16-byte broadcast loads
template <typename T>
__device__ __forceinline__ void read_kx(const T* kvs, T (&kx)[8]) {
  if constexpr (sizeof(T) == 4) {
    const float4 a = reinterpret_cast<const float4*>(kvs)[0], b = reinterpret_cast<const float4*>(kvs)[1];
    kx[0] = a.x; kx[1] = a.y; kx[2] = a.z; kx[3] = a.w;
    kx[4] = b.x; kx[5] = b.y; kx[6] = b.z; kx[7] = b.w;
  } else {
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const double2 v = reinterpret_cast<const double2*>(kvs)[q];
      kx[2 * q] = v.x;
      kx[2 * q + 1] = v.y;
    }
  }
}

// the 3W kernel values of staged candidate src: lane l < 3W evaluates tap
// l % W of axis l / W (its fraction is word l / W of the candidate's slot)
template <typename T, int W, bool kPoly>
__device__ __forceinline__ void eval_kv(const unsigned char* stg, int src, T* kv, int lane,
                                        int axis, int tap, const T (&pc)[kPolyCoef], T beta,
                                        T ces, T halfw) {
  // every lane evaluates (lanes from 3W on repeat axis 2), only 3W store:
  // straight-line code that can interleave with the taps around it
  const T f = reinterpret_cast<const T*>(stg + src * kCandBytes<T>)[axis < 3 ? axis : 2];
  T v;
  if constexpr (kPoly)
    v = poly_eval(pc, poly_arg<W>(f));
  else
    v = es_kernel<T>((T)(tap_offset<W>(f) + tap) - f, beta, ces, halfw);
  if (lane < 3 * W) kv[lane] = v;
}

template <typename T, int W, bool kPoly>
__device__ __forceinline__ void slide_item(const Rec<T>* __restrict__ recs,
                                           const int* __restrict__ hive_start, const Geom& g,
                                           const SlideTile& tc, T* __restrict__ fw, int item,
                                           unsigned char* wsmem, const T (&pc)[kPolyCoef]) {
  using C = typename Cx<T>::type;
  constexpr int lo = Halo<W>::lo, hi = Halo<W>::hi;
  const int lane = threadIdx.x & 31;
  const int TY = tc.TY, RS = tc.RS, nw = g.nw, nf1 = g.nf1, nf2 = g.nf2;
  const int nhx = g.nhx, nhy = g.nhy;
  C* acc = reinterpret_cast<C*>(wsmem);
  int* t_start = reinterpret_cast<int*>(wsmem + (size_t)TY * RS * sizeof(C));
  int* t_pref = t_start + tc.nslots;      // nslots + 1
  int* t_shy = t_pref + tc.nslots + 1;
  // staging of the current chunk's candidates (one 32- or 64-byte slot per
  // lane) and of two rows' kernel values (double-buffered: the next row's are
  // evaluated while the current row is spread): every lane reads them with
  // broadcast loads, where register shuffles took one crossbar operation per
  // value
  unsigned char* stg = wsmem + tc.stage_off;
  T* kvs = reinterpret_cast<T*>(stg + 32 * kCandBytes<T>);
  const int kv_axis = lane / W, kv_tap = lane - kv_axis * W;
  const size_t plane = (size_t)nf1 * nf2;
  C* fwc = reinterpret_cast<C*>(fw);
  const T beta = (T)g.beta, ces = (T)g.es_c, halfw = (T)W * (T)0.5;

  // items are handed out from the grid's centre outward (bands, then the
  // segments inside a band): uv data is densest around u = v = 0, the centre
  // of the grid, so the heaviest items start first and the launch ends on
  // light ones
  const int kb = item / tc.nsegs, ks = item - kb * tc.nsegs;
  const int band = tc.nbands / 2 + ((kb & 1) ? -((kb + 1) >> 1) : (kb >> 1));
  const int lane_dq = lane / W, lane_dz = lane - lane_dq * W;  // pair offsets, first pass of pairs
  const int lane_dq2 = (lane + 32) / W, lane_dz2 = lane + 32 - lane_dq2 * W;  // second pass of pairs
  // W <= 6: tap lane of the pairs beyond 32, pair 32 + lane / W, x tap lane % W
  const int tail_e = lane % W, tail_p = 32 + lane / W;
  const int tail_dq = tail_p / W, tail_dz = tail_p - tail_dq * W;
  const int seg = tc.nsegs / 2 + ((ks & 1) ? -((ks + 1) >> 1) : (ks >> 1));
  const int y0 = band * TY, y1 = min(y0 + TY, nf2), wy = y1 - y0;
  if (g.grid_skip) {  // a band wholly outside the rows the transform reads holds no rows
    int r0, n;
    fft_row_band(g, r0, n);
    if (y1 <= r0 || y0 >= r0 + n) return;
  }
  const int hs = seg * tc.SEG, he = min(hs + tc.SEG, nhx);
  const int hya = floordiv8(y0 - hi), hyb = floordiv8(y1 - 1 + lo);
  const int nyr = hyb - hya + 1;
  const int nslots = nyr * nw;

  // rows of the item: the hive columns [hs - 1, he) of every slot
  {
    int any = 0;
    for (int s = lane; s < nslots; s += 32) {
      const int hz = s / nyr;
      int hy = hya + (s - hz * nyr);
      hy += hy < 0 ? nhy : (hy >= nhy ? -nhy : 0);
      const int64_t rb = ((int64_t)hz * nhy + hy) * nhx;
      int cnt = hive_start[rb + he] - hive_start[rb + max(hs - 1, 0)];
      if (hs == 0) cnt += hive_start[rb + nhx] - hive_start[rb + nhx - 1];
      any |= cnt > 0;
    }
    if (!__any_sync(0xffffffffu, any)) {
      zero_region<T>(fw, g, 8 * hs - kFlushL, 8 * (he - hs), y0, wy);
      return;
    }
  }
  {
    const int n = TY * RS;
    for (int i = lane; i < n; i += 32) acc[i] = C{(T)0, (T)0};
  }
  __syncwarp();

  for (int c = hs - 1; c < he; c++) {
    const int cc = c < 0 ? c + nhx : c;
    const int sx = c < 0 ? -nf1 : 0;
    // segment table of column c: slot s = (hive row hya + s % nyr, plane s / nyr)
    int carry = 0;
    for (int base = 0; base < nslots; base += 32) {
      const int s = base + lane;
      int cnt = 0;
      if (s < nslots) {
        const int hz = s / nyr;
        const int hyr = hya + (s - hz * nyr);
        int hy = hyr, shy = 0;
        if (hy < 0) { hy += nhy; shy = -nf2; }
        else if (hy >= nhy) { hy -= nhy; shy = nf2; }
        const int64_t h = ((int64_t)hz * nhy + hy) * nhx + cc;
        const int st = hive_start[h];
        cnt = hive_start[h + 1] - st;
        t_start[s] = st;
        t_shy[s] = shy;
      }
      int tot;
      const int ex = carry + warp_scan_excl(cnt, tot);
      if (s < nslots) t_pref[s] = ex;
      carry += tot;
    }
    if (lane == 0) t_pref[nslots] = carry;
    __syncwarp();
    const int total = carry;

    for (int q0 = 0; q0 < total; q0 += 32) {
      const int q = q0 + lane;
      bool ok = q < total;
      T f0 = 0, f1 = 0, f2 = 0, c0 = 0, c1 = 0;
      int ox = 0, oy = 0, oz = 0;
      if (ok) {
        int lo_s = 0, hi_s = nslots;  // t_pref[lo_s] <= q < t_pref[hi_s]
        while (hi_s - lo_s > 1) {
          const int mid = (lo_s + hi_s) >> 1;
          if (t_pref[mid] <= q) lo_s = mid; else hi_s = mid;
        }
        const Rec<T> r = recs[t_start[lo_s] + (q - t_pref[lo_s])];
        f0 = r.f[0]; f1 = r.f[1]; f2 = r.f[2]; c0 = r.c[0]; c1 = r.c[1];
        ox = (int)(r.bxy & 0xFFFFu) + sx + tap_offset<W>(f0);
        oy = (int)(r.bxy >> 16) + t_shy[lo_s] + tap_offset<W>(f1);
        oz = (int)r.bz + tap_offset<W>(f2);
        ok = oy < y1 && oy + W > y0;
      }
      stage_cand<T>(stg, lane, f0, f1, f2, c0, c1, ox, oy, oz);
      unsigned mask = __ballot_sync(0xffffffffu, ok);
      __syncwarp();
      if (mask)
        eval_kv<T, W, kPoly>(stg, __ffs(mask) - 1, kvs, lane, kv_axis, kv_tap, pc, beta, ces, halfw);
      int buf = 0;
      __syncwarp();
      while (mask) {
        const int src = __ffs(mask) - 1;
        mask &= mask - 1;
        const T* kv = kvs + buf * 32;
        // the next row's kernel values into the other buffer: independent of
        // this row's taps, so their latency overlaps
        if (mask)
          eval_kv<T, W, kPoly>(stg, __ffs(mask) - 1, kvs + (buf ^ 1) * 32, lane, kv_axis, kv_tap,
                               pc, beta, ces, halfw);
        T g0, g1, g2, vr0, vi0;
        int vx, vy, vz;
        read_cand<T>(stg, src, g0, g1, g2, vr0, vi0, vx, vy, vz);
        vy -= y0;
        T kx[8];
        read_kx<T>(kv, kx);
        const int dya = max(0, -vy), dyb = min(W, wy - vy);
        const int np = (dyb - dya) * W;
        const int xs = vx & (kXW - 1);
        // pair (dya + dq, dz): its W taps along x
        auto spread = [&](int dq, int dz) {
          const int dy = dya + dq;
          const T ky = kv[W + dy];
          const T kz = kv[2 * W + dz];
          int z = vz + dz;
          z += z < 0 ? nw : (z >= nw ? -nw : 0);
          const T k = ky * kz;
          const T vr = vr0 * k, vi = vi0 * k;
          C* a = acc + (vy + dy) * RS + z * kPS;
          // all W loads first, then the FMAs, then the stores: the loads are
          // in flight together (FP32, and FP64 up to W = 6; FP64 W = 7, 8 take
          // a load, FMA and store per tap, at half the registers)
          if constexpr (sizeof(T) == 8 && W > 6) {
            if (xs + W <= kXW) {
              C* b = a + xs;
#pragma unroll
              for (int e = 0; e < W; e++) {
                C cv = b[e];
                cv.x += vr * kx[e];
                cv.y += vi * kx[e];
                b[e] = cv;
              }
            } else {
#pragma unroll
              for (int e = 0; e < W; e++) {
                C* c = a + ((xs + e) & (kXW - 1));
                C cv = *c;
                cv.x += vr * kx[e];
                cv.y += vi * kx[e];
                *c = cv;
              }
            }
            return;
          }
          C cur[W];
          if (xs + W <= kXW) {  // the row's taps do not wrap the window (same for all lanes)
            C* b = a + xs;
#pragma unroll
            for (int e = 0; e < W; e++) cur[e] = b[e];
#pragma unroll
            for (int e = 0; e < W; e++) {
              cur[e] = tap_fma(cur[e], vr, vi, kx[e]);
            }
#pragma unroll
            for (int e = 0; e < W; e++) b[e] = cur[e];
          } else {
#pragma unroll
            for (int e = 0; e < W; e++) cur[e] = a[(xs + e) & (kXW - 1)];
#pragma unroll
            for (int e = 0; e < W; e++) {
              cur[e] = tap_fma(cur[e], vr, vi, kx[e]);
            }
#pragma unroll
            for (int e = 0; e < W; e++) a[(xs + e) & (kXW - 1)] = cur[e];
          }
        };
        if (lane < np) spread(lane_dq, lane_dz);  // pair lane: (dya + lane / W, lane % W)
        if constexpr (W >= 7) {
          // W = 7, 8: up to 49 / 64 pairs; pairs 32 .. np - 1 take a second
          // pass of the same form, pair lane + 32 per lane
          if (np > 32 && lane < np - 32) spread(lane_dq2, lane_dz2);
        } else if (np > 32) {  // W <= 6: at most 4 more pairs (24 taps), one tap per lane
          if (lane < (np - 32) * W) {
            const int e = tail_e, dz = tail_dz, dy = dya + tail_dq;
            {
              const T ky = kv[W + dy], kz = kv[2 * W + dz], kxe = kv[e];
              int z = vz + dz;
              z += z < 0 ? nw : (z >= nw ? -nw : 0);
              const T k = ky * kz;
              C* cell = acc + (vy + dy) * RS + z * kPS + ((xs + e) & (kXW - 1));
              C cur = *cell;
              cur = tap_fma(cur, vr0 * k, vi0 * k, kxe);
              *cell = cur;
            }
          }
        }
        __syncwarp();
        buf ^= 1;
      }
    }

    {
      // cells [8c - 4, 8c + 4) of every row and plane are final: flush them
      // and zero their slots.  The warm-up column (c = hs - 1) only zeroes
      // them: they belong to the previous segment, and their slots are those
      // of cells [8c + 12, 8c + 20) that the next columns reach.
      const bool write = c >= hs;
      const int x0 = 8 * c - kFlushL;
      const int n = TY * nw * 4;  // cell pairs
      for (int i = lane; i < n; i += 32) {
        const int pr = i & 3, rest = i >> 2;
        const int y = rest & (TY - 1), z = rest >> tc.logTY;
        if (y >= wy) continue;
        const int x = x0 + 2 * pr;
        const int slot = x & (kXW - 1);
        C* a = acc + y * RS + z * kPS + slot;
        const C a0 = a[0], a1 = a[1];
        a[0] = C{(T)0, (T)0};
        a[1] = C{(T)0, (T)0};
        if (!write) continue;
        const int gx = x < 0 ? x + nf1 : x;
        C* dst = fwc + (size_t)z * plane + (size_t)(y0 + y) * nf1 + gx;
        if constexpr (sizeof(T) == 4) {
          *reinterpret_cast<float4*>(dst) = make_float4(a0.x, a0.y, a1.x, a1.y);
        } else {
          dst[0] = a0;
          dst[1] = a1;
        }
      }
    }
    __syncwarp();
  }
}

template <typename T, int W, bool kPoly>
__global__ void __launch_bounds__(512) k_grid_slide(const Rec<T>* __restrict__ recs,
                                                    const int* __restrict__ hive_start, Geom g,
                                                    SlideTile tc, T* __restrict__ fw,
                                                    int* __restrict__ counter) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  // piecewise-polynomial kernel: lane l < 3W evaluates segment l % W
  T pc[kPolyCoef];
#pragma unroll
  for (int n = 0; n < kPolyCoef; n++) pc[n] = (T)0;
  if constexpr (kPoly) {
    const T* poly = geom_poly<T>(g);
    if (lane < 3 * W) {
      const int i = lane % W;
#pragma unroll
      for (int n = 0; n < kPolyCoef; n++) pc[n] = poly[i * kPolyCoef + n];
    }
  }
  unsigned char* wsmem = smem + (size_t)wib * tc.warp_bytes;
  for (;;) {
    int item = 0;
    if (lane == 0) item = atomicAdd(counter, 1);
    item = __shfl_sync(0xffffffffu, item, 0);
    if (item >= tc.nitems) break;
    slide_item<T, W, kPoly>(recs, hive_start, g, tc, fw, item, wsmem, pc);
  }
}

// Many grids in one persistent launch (batched solves): warps take (job,
// item) pairs from one queue, every job with its own geometry and window
// shape (jobs[j].st) in a per-warp region of warp_bytes, the largest of the
// jobs'.  Every job shares W and the kernel.
template <typename T, int W, bool kPoly>
__global__ void __launch_bounds__(512) k_grid_slide_multi(const GridJob<T>* __restrict__ jobs,
                                                          int njobs, int nitems,
                                                          size_t warp_bytes,
                                                          int* __restrict__ counter) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  T pc[kPolyCoef];
#pragma unroll
  for (int n = 0; n < kPolyCoef; n++) pc[n] = (T)0;
  if constexpr (kPoly) {
    const T* poly = geom_poly<T>(jobs[0].g);
    if (lane < 3 * W) {
      const int i = lane % W;
#pragma unroll
      for (int n = 0; n < kPolyCoef; n++) pc[n] = poly[i * kPolyCoef + n];
    }
  }
  unsigned char* wsmem = smem + (size_t)wib * warp_bytes;
  for (;;) {
    int item = 0;
    if (lane == 0) item = atomicAdd(counter, 1);
    item = __shfl_sync(0xffffffffu, item, 0);
    if (item >= nitems) break;
    int lo = 0, hi = njobs;  // jobs[lo].grid_item0 <= item < jobs[hi].grid_item0
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (jobs[mid].grid_item0 <= item) lo = mid; else hi = mid;
    }
    const GridJob<T>& J = jobs[lo];
    slide_item<T, W, kPoly>(J.recs, J.hive_start, J.g, J.st, J.fw, item - J.grid_item0, wsmem, pc);
  }
}

constexpr size_t kSlideSmemMax = 227 * 1024;

int env_or(const char* name, int dflt) {
  const char* v = getenv(name);
  return v ? atoi(v) : dflt;
}

}  // namespace

// Band rows, hive columns per segment and warps per CTA: the tuned values,
// else CG_SLIDE_TY / CG_SLIDE_SEG / CG_SLIDE_WARPS, else 8 / 12 / as many as
// fit.  Short segments keep the densest items (around the grid centre) well
// below a warp's share of the work; each costs one warm-up hive column.
bool slide_tiling(const Geom& g, size_t tsz, const TileTune* tt, SlideTile& tc) {
  const int W = g.kw;
  if (W < 4 || W > 8 || (g.nf1 % 8) != 0 || (g.nf2 % 8) != 0 || g.nf1 < kXW) return false;
  int TY = (tt && tt->wy > 0 && tt->wx < 0) ? tt->wy : env_or("CG_SLIDE_TY", 8);
  if (TY != 8 && TY != 16 && TY != 32) return false;
  int SEG = (tt && tt->wpb > 0 && tt->wx < 0) ? tt->wpb : env_or("CG_SLIDE_SEG", 12);
  SEG = std::max(1, std::min(SEG, g.nhx));
  tc.TY = TY;
  tc.logTY = TY == 8 ? 3 : (TY == 16 ? 4 : 5);
  tc.SEG = SEG;
  int rs = g.nw * kPS;
  rs += ((W % 16) - (rs % 16) + 16) % 16;  // RS = W (mod 16)
  tc.RS = rs;
  const int nyr = (TY >> 3) + 2;
  tc.nslots = nyr * g.nw;
  tc.nbands = (g.nf2 + TY - 1) / TY;
  tc.nsegs = (g.nhx + SEG - 1) / SEG;
  if ((int64_t)tc.nbands * tc.nsegs > 2147483647LL) return false;
  tc.nitems = tc.nbands * tc.nsegs;
  tc.stage_off = ((size_t)TY * rs * 2 * tsz + (size_t)(3 * tc.nslots + 1) * 4 + 15) & ~(size_t)15;
  // candidate slots (32 per warp) and two buffers of 32 kernel values
  tc.warp_bytes = tc.stage_off + 32 * (tsz == 4 ? 32 : 64) + 64 * tsz;
  int warps = (tt && tt->warps > 0 && tt->wx < 0) ? tt->warps : env_or("CG_SLIDE_WARPS", 0);
  if (warps <= 0) warps = (int)std::max<size_t>(1, std::min<size_t>(16, kSlideSmemMax / tc.warp_bytes));
  warps = std::min(warps, 16);
  while (warps > 1 && tc.warp_bytes * warps > kSlideSmemMax) warps--;
  if (tc.warp_bytes * warps > kSlideSmemMax) return false;
  tc.warps = warps;
  tc.smem = tc.warp_bytes * warps;
  return true;
}

namespace {

int sms_of_device() {
  int dev = 0, n = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) n = 148;
  return n;
}

template <typename T, int W>
int launch_w(const Rec<T>* d_recs, const int* d_hive_start, const Geom& g, T* d_fw,
             int* d_counter, cudaStream_t st, const SlideTile& tc) {
  auto* kern = geom_poly_host<T>(g) ? k_grid_slide<T, W, true> : k_grid_slide<T, W, false>;
  int per_sm = 0;
  CG_CUDA(kernel_occupancy((const void*)kern, tc.warps * 32, tc.smem, &per_sm));
  if (per_sm < 1) return CG_ERR_ARG;
  static int sms = 0;
  if (!sms) sms = sms_of_device();
  const int blocks = std::min((tc.nitems + tc.warps - 1) / tc.warps, per_sm * sms);
  CG_CUDA(cudaMemsetAsync(d_counter, 0, sizeof(int), st));
  kern<<<std::max(1, blocks), tc.warps * 32, tc.smem, st>>>(d_recs, d_hive_start, g, tc, d_fw,
                                                            d_counter);
  count_launches(1);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

}  // namespace

template <typename T>
int launch_grid_slide(const Rec<T>* d_recs, const int* d_hive_start, const Geom& g, T* d_fw,
                      int* d_counter, cudaStream_t st, const TileTune* tt) {
  SlideTile tc{};
  if (!slide_tiling(g, sizeof(T), tt, tc)) return CG_ERR_ARG;
  switch (g.kw) {
    case 4: return launch_w<T, 4>(d_recs, d_hive_start, g, d_fw, d_counter, st, tc);
    case 5: return launch_w<T, 5>(d_recs, d_hive_start, g, d_fw, d_counter, st, tc);
    case 6: return launch_w<T, 6>(d_recs, d_hive_start, g, d_fw, d_counter, st, tc);
    case 7: return launch_w<T, 7>(d_recs, d_hive_start, g, d_fw, d_counter, st, tc);
    case 8: return launch_w<T, 8>(d_recs, d_hive_start, g, d_fw, d_counter, st, tc);
    default: return CG_ERR_ARG;
  }
}

template <typename T, int W>
static int slide_multi_w(const GridJob<T>* d_jobs, int njobs, const MultiShape& sh, int* d_counter,
                         cudaStream_t st) {
  auto* kern = sh.poly ? k_grid_slide_multi<T, W, true> : k_grid_slide_multi<T, W, false>;
  const size_t smem = sh.warp_bytes * sh.warps;
  int per_sm = 0;
  CG_CUDA(kernel_occupancy((const void*)kern, sh.warps * 32, smem, &per_sm));
  if (per_sm < 1) {
    set_last_error("multi-grid sliding gridding does not fit on an SM");
    return CG_ERR_ARG;
  }
  static int sms = 0;
  if (!sms) sms = sms_of_device();
  const int blocks = std::min((sh.grid_items + sh.warps - 1) / sh.warps, per_sm * sms);
  CG_CUDA(cudaMemsetAsync(d_counter, 0, sizeof(int), st));
  kern<<<std::max(1, blocks), sh.warps * 32, smem, st>>>(d_jobs, njobs, sh.grid_items,
                                                         sh.warp_bytes, d_counter);
  count_launches(1);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

template <typename T>
int launch_grid_slide_multi(const GridJob<T>* d_jobs, int njobs, const MultiShape& sh,
                            int* d_counter, cudaStream_t st) {
  if (njobs < 1 || sh.grid_items < 1) return CG_OK;
  switch (sh.kw) {
    case 4: return slide_multi_w<T, 4>(d_jobs, njobs, sh, d_counter, st);
    case 5: return slide_multi_w<T, 5>(d_jobs, njobs, sh, d_counter, st);
    case 6: return slide_multi_w<T, 6>(d_jobs, njobs, sh, d_counter, st);
    case 7: return slide_multi_w<T, 7>(d_jobs, njobs, sh, d_counter, st);
    case 8: return slide_multi_w<T, 8>(d_jobs, njobs, sh, d_counter, st);
    default: return CG_ERR_ARG;
  }
}

template int launch_grid_slide_multi<float>(const GridJob<float>*, int, const MultiShape&, int*,
                                            cudaStream_t);
template int launch_grid_slide_multi<double>(const GridJob<double>*, int, const MultiShape&, int*,
                                             cudaStream_t);
template int launch_grid_slide<float>(const Rec<float>*, const int*, const Geom&, float*, int*,
                                      cudaStream_t, const TileTune*);
template int launch_grid_slide<double>(const Rec<double>*, const int*, const Geom&, double*, int*,
                                       cudaStream_t, const TileTune*);

}  // namespace cg
