// Degridding with TMA-staged grid tiles (FP32 grids, all planes per tile).
//
// Same interpolation as k_degrid_tiled (interp_3d_nputsdriven,
// interp.cu:132-210, restated tile by tile): a persistent CTA per SM takes
// tiles of TX x TY cells (all nw planes) from a work queue, stages the tile
// plus the kernel halo in shared memory and interpolates every row of the
// tile's own hives from there, one row per thread.  Staging here is one
// cp.async.bulk.tensor.3d box per tile into one of two shared-memory stages:
// while the rows of one tile are interpolated, the next tile's box is already
// in flight.  Tiles whose halo wraps around the grid edge are staged element
// by element (periodic indices); empty tiles are skipped before any staging.
//
// TMA rules kept by construction: the box starts at an even x (16-byte
// aligned for 8-byte elements) and is an even number of elements wide; every
// start coordinate is >= 0 and the box lies inside the grid (interior tiles
// only); the global strides are multiples of 16 bytes; the stages are
// 1024-byte aligned.  Every wait on the stage barriers is bounded; a wait
// that runs out sets *err and the CTA stops taking tiles, so the call's
// visibilities are incomplete and the call reports the error.  The bound of
// the stage waits is a launch argument: CG_TMA_STAGE_WAIT_TRIES (test only)
// lowers it, down to 0 tries, which makes the first staged box's wait run
// out; the drain of boxes still in flight always keeps the full bound.
#include <cuda.h>

#include <algorithm>
#include <cstdlib>

#include "cg_coords.cuh"
#include "cg_launch.cuh"
#include "cg_tiles.cuh"

namespace cg {
namespace {

constexpr int kWaitTries = 1 << 20;  // bounded barrier wait (well under a second)

struct TmaTile {
  int TX, TY;        // tile cells (multiples of 8)
  int SX, SY, SZ;    // staged box: SX even >= TX + W + 1, SY = TY + W, SZ = nw
  int ntx, nty;      // tiles of the grid
  int bx0, by0, nbx; // the tiles of the data band: nbx per band row, from tile (bx0, by0)
  int nitems;        // tiles of the data band (the queue's items)
  int nslots;        // segment slots of a tile's own hives
  size_t stage_bytes;  // one stage, rounded up to 1024 bytes
};

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes)
               : "memory");
}

// bounded wait (at most `tries` polls) for phase `parity` of the barrier;
// false if it ran out
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity, int tries = kWaitTries) {
  for (int i = 0; i < tries; i++) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tma_load_3d(unsigned dst, const CUtensorMap* map, int x, int y,
                                            int z, unsigned bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
      : "memory");
}

// NT threads per CTA; NS stages: 2 = the next tile's box in flight while the
// current one is interpolated (one CTA per SM), 1 = one box at a time (two
// CTAs per SM overlap each other's staging and interpolation)
template <int W, int NT, int NS>
__global__ void __launch_bounds__(NT, NS == 1 ? (NT <= 128 ? 3 : 2) : 1) k_degrid_tma(
    const __grid_constant__ CUtensorMap map, const Rec<float>* __restrict__ recs,
    const int* __restrict__ perm, const int* __restrict__ hive_start, int64_t M, Geom g,
    TmaTile tc, const float2* __restrict__ fw, float* __restrict__ vis, int* __restrict__ counter,
    int* __restrict__ err, int stage_tries) {
  extern __shared__ unsigned char smem_raw[];
  constexpr int lo = Halo<W>::lo;
  unsigned char* base =
      smem_raw + ((1024 - (smem_u32(smem_raw) & 1023)) & 1023);  // 1024-byte aligned
  float2* stage[2] = {reinterpret_cast<float2*>(base),
                      reinterpret_cast<float2*>(base + (NS - 1) * tc.stage_bytes)};
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(base + NS * tc.stage_bytes);
  int* tb = reinterpret_cast<int*>(bars + 2);
  const int ts = tc.nslots + 1;
  SegTable t{tb, tb + ts, tb + 2 * ts};
  __shared__ int s_warp[33];
  __shared__ int s_next;
  const int nw = g.nw, nf1 = g.nf1, nf2 = g.nf2;
  const int SX = tc.SX, SY = tc.SY, SZ = tc.SZ;
  const size_t plane = (size_t)nf1 * nf2;
  const float beta = (float)g.beta, c = (float)g.es_c;
  const float* __restrict__ poly = geom_poly<float>(g);
  const unsigned box_bytes = (unsigned)((size_t)SX * SY * SZ * sizeof(float2));

  if (threadIdx.x == 0) {
    mbar_init(smem_u32(&bars[0]), 1);
    mbar_init(smem_u32(&bars[1]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  // warp 0: the next tile that holds rows (or nitems when the queue is empty)
  auto fetch = [&]() {
    const int lane = threadIdx.x & 31;
    for (;;) {
      int item = 0;
      if (lane == 0) item = atomicAdd(counter, 1);
      item = __shfl_sync(0xffffffffu, item, 0);
      if (item >= tc.nitems) return tc.nitems;
      const int tix = tc.bx0 + item % tc.nbx, tiy = tc.by0 + item / tc.nbx;
      const int tx0 = tix * tc.TX, ty0 = tiy * tc.TY;
      const int hx0 = tx0 >> 3, hx1 = (min(tx0 + tc.TX, nf1) - 1) >> 3;
      const int hy0 = ty0 >> 3, nhyr = ((min(ty0 + tc.TY, nf2) - 1) >> 3) - hy0 + 1;
      int any = 0;
      for (int r = lane; r < nhyr * nw && !any; r += 32) {
        const int hy = hy0 + r % nhyr, z = r / nhyr;
        const int64_t rb = ((int64_t)z * g.nhy + hy) * g.nhx;
        any = hive_start[rb + hx1 + 1] > hive_start[rb + hx0];
      }
      if (__any_sync(0xffffffffu, any)) return item;
    }
  };
  // box origin of a tile (x rounded down to even) and whether it lies inside the grid
  auto origin = [&](int item, int& gx0, int& gy0) {
    const int tix = tc.bx0 + item % tc.nbx, tiy = tc.by0 + item / tc.nbx;
    gx0 = (tix * tc.TX - lo) & ~1;
    gy0 = tiy * tc.TY - lo;
    return gx0 >= 0 && gy0 >= 0 && gx0 + SX <= nf1 && gy0 + SY <= nf2;
  };
  // all threads: element-by-element staging with periodic indices
  auto stage_wrapped = [&](int item, float2* dst) {
    int gx0, gy0;
    origin(item, gx0, gy0);
    const int n = SX * SY * SZ;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const int sx = i % SX, sy = (i / SX) % SY, sz = i / (SX * SY);
      dst[i] = fw[(size_t)sz * plane + (size_t)modi(gy0 + sy, nf2) * nf1 + modi(gx0 + sx, nf1)];
    }
  };
  // thread 0: the box of an interior tile into stage s
  auto issue = [&](int item, int s) {
    int gx0, gy0;
    origin(item, gx0, gy0);
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    const unsigned bar = smem_u32(&bars[s]);
    mbar_expect_tx(bar, box_bytes);
    tma_load_3d(smem_u32(stage[s]), &map, gx0, gy0, 0, bar);
  };

  if (threadIdx.x < 32) {
    const int it = fetch();
    if (threadIdx.x == 0) s_next = it;
  }
  __syncthreads();
  int cur = s_next, s = 0;
  unsigned phase[2] = {0u, 0u};
  bool pending[2] = {false, false};  // a box issued into the stage and not yet waited for
  int gx_dummy, gy_dummy;
  bool cur_tma = cur < tc.nitems && origin(cur, gx_dummy, gy_dummy);
  if (cur < tc.nitems) {
    if (cur_tma) {
      if (threadIdx.x == 0) issue(cur, 0);
      pending[0] = true;
    } else {
      stage_wrapped(cur, stage[0]);
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    }
  }
  __syncthreads();
  while (cur < tc.nitems) {
    // the next tile: fetched by warp 0, its box issued into the other stage
    if (threadIdx.x < 32) {
      const int it = fetch();
      if (threadIdx.x == 0) s_next = it;
    }
    __syncthreads();
    const int next = s_next;
    const bool next_tma = next < tc.nitems && origin(next, gx_dummy, gy_dummy);
    if (NS == 2 && next_tma) {
      if (threadIdx.x == 0) issue(next, s ^ 1);
      pending[s ^ 1] = true;
    }
    // the current tile's box
    bool ok = true;
    if (cur_tma) {
      ok = mbar_wait(smem_u32(&bars[s]), phase[s], stage_tries);
      if (ok) {
        phase[s] ^= 1u;
        pending[s] = false;
      }
    }
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) atomicExch(err, 1);
      break;
    }
    // runs of the tile's own hives, all planes
    const int tix = tc.bx0 + cur % tc.nbx, tiy = tc.by0 + cur / tc.nbx;
    const int tx0 = tix * tc.TX, ty0 = tiy * tc.TY;
    const int tx1 = min(tx0 + tc.TX, nf1), ty1 = min(ty0 + tc.TY, nf2);
    int gx0, gy0;
    origin(cur, gx0, gy0);
    const int nslots = build_segments(g, hive_start, tx0 >> 3, (tx1 - 1) >> 3, ty0 >> 3,
                                      (ty1 - 1) >> 3, 0, nw - 1, t, s_warp);
    const int total = t.pref[nslots];
    const float2* st = stage[s];
    for (int q = threadIdx.x; q < total; q += blockDim.x) {
      const int sgi = find_segment(t.pref, nslots, q);
      const int sidx = t.start[sgi] + (q - t.pref[sgi]);
      const Rec<float> r = recs[sidx];
      const int bx = (int)(r.bxy & 0xFFFFu), by = (int)(r.bxy >> 16), bz = (int)r.bz;
      float kx[W], ky[W], kz[W];
      const int lx = bx + taps<float, W>(r.f[0], beta, c, poly, kx) - gx0;
      const int ly = by + taps<float, W>(r.f[1], beta, c, poly, ky) - gy0;
      const int lz = bz + taps<float, W>(r.f[2], beta, c, poly, kz);
      if (lx < 0 || ly < 0 || lx + W > SX || ly + W > SY) continue;  // cannot happen: tile rows only
      // complex sums of cells times real kernel values, one packed FMA each
      float2 s2 = make_float2(0.f, 0.f);
#pragma unroll
      for (int a = 0; a < W; a++) {
        const int zz = wrapi(lz + a, nw);
        float2 p2 = make_float2(0.f, 0.f);
#pragma unroll
        for (int b = 0; b < W; b++) {
          const float2* row = st + ((size_t)zz * SY + (ly + b)) * SX + lx;
          float2 q2 = make_float2(0.f, 0.f);
#pragma unroll
          for (int e = 0; e < W; e++) {
            const float2 v = row[e];
            q2 = tap_fma(q2, v.x, v.y, kx[e]);
          }
          p2 = tap_fma(p2, q2.x, q2.y, ky[b]);
        }
        s2 = tap_fma(s2, p2.x, p2.y, kz[a]);
      }
      const float sr = s2.x, si = s2.y;
      const int64_t i = perm[sidx];
      if (i < 0 || i >= M) continue;
      vis[2 * i] = sr * r.c[0] - si * r.c[1];
      vis[2 * i + 1] = sr * r.c[1] + si * r.c[0];
    }
    // generic reads of stage s before the box that will overwrite it
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();  // stage s and the segment table are free again
    if (NS == 2) s ^= 1;
    cur = next;
    cur_tma = next_tma;
    if (cur < tc.nitems) {
      if (!cur_tma) {
        stage_wrapped(cur, stage[s]);
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncthreads();
      } else if (NS == 1) {
        if (threadIdx.x == 0) issue(cur, 0);
        pending[0] = true;
      }
    }
  }
  // after a timed-out wait boxes may still be in flight: wait for them, with
  // the full bound whatever stage_tries is, before the CTA's shared memory is
  // released
  if (threadIdx.x == 0)
    for (int k = 0; k < 2; k++)
      if (pending[k]) mbar_wait(smem_u32(&bars[k]), phase[k]);
}

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                 const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                 const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                 CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn() {
  static EncodeTiled fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(p);
  }
  return fn;
}

// shared memory of one CTA with NS stages
size_t tma_smem(const TmaTile& tc, int ns) {
  return 1024 + ns * tc.stage_bytes + 16 + (size_t)(tc.nslots + 1) * kSegInts * 4;
}

// variant 1: 32 x 16 tiles, 512 threads, two stages; variant 2: 32 x 16
// tiles, 256 threads, one stage; variant 3: 32 x 8 tiles, 128 threads, one
// stage (three CTAs per SM); variant 4: 16 x 8 tiles, 128 threads, one stage
// (many planes: two CTAs per SM up to ~38 planes at W = 8)
bool tma_tiling(const Geom& g, TmaTile& tc, int variant) {
  const int W = g.kw;
  const int tx = variant == 4 ? 16 : 32, ty = variant >= 3 ? 8 : 16;
  tc.TX = tx;
  tc.TY = ty;
  tc.SX = (tx + W + 1 + 1) & ~1;
  tc.SY = ty + W;
  tc.SZ = g.nw;
  tc.ntx = (g.nf1 + tx - 1) / tx;
  tc.nty = (g.nf2 + ty - 1) / ty;
  // only the tiles of the cells the data can reach (the full grid when the
  // data wraps around an edge): the others hold no rows
  int bx0 = 0, bx1 = tc.ntx - 1, by0 = 0, by1 = tc.nty - 1;
  if (0 <= g.band_c0 && g.band_c0 <= g.band_c1 && g.band_c1 < g.nf1) {
    bx0 = g.band_c0 / tx;
    bx1 = g.band_c1 / tx;
  }
  if (0 <= g.band_r0 && g.band_r0 <= g.band_r1 && g.band_r1 < g.nf2) {
    by0 = g.band_r0 / ty;
    by1 = g.band_r1 / ty;
  }
  tc.bx0 = bx0;
  tc.by0 = by0;
  tc.nbx = bx1 - bx0 + 1;
  tc.nitems = tc.nbx * (by1 - by0 + 1);
  tc.nslots = ((ty >> 3) + 1) * g.nw * 3;
  tc.stage_bytes = ((size_t)tc.SX * tc.SY * tc.SZ * sizeof(float2) + 1023) & ~(size_t)1023;
  // box dimensions <= 256, grid rows 16-byte multiples; two stages on one
  // SM (variant 1), two (variants 2, 4) or three (variant 3) one-stage CTAs per SM
  const size_t limit = variant == 1 ? 220 * 1024 : (variant == 3 ? 74 * 1024 : 110 * 1024);
  return variant >= 1 && variant <= 4 && g.nw <= 256 && tc.SX <= 256 && tc.SY <= 256 &&
         (g.nf1 % 2) == 0 && g.nf1 >= tc.SX && g.nf2 >= tc.SY &&
         tma_smem(tc, variant == 1 ? 2 : 1) <= limit;
}

template <int W, int NT, int NS>
int launch_w(const Rec<float>* d_recs, const int* d_perm, const int* d_hive_start, int64_t M,
             const Geom& g, const TmaTile& tc, const float* d_fw, float* d_vis, int* d_counter,
             int* d_err, cudaStream_t st) {
  EncodeTiled enc = encode_fn();
  if (!enc) return CG_ERR_ARG;
  CUtensorMap map;
  const cuuint64_t dims[3] = {(cuuint64_t)g.nf1, (cuuint64_t)g.nf2, (cuuint64_t)g.nw};
  const cuuint64_t strides[2] = {(cuuint64_t)g.nf1 * sizeof(float2),
                                 (cuuint64_t)g.nf1 * g.nf2 * sizeof(float2)};
  const cuuint32_t box[3] = {(cuuint32_t)tc.SX, (cuuint32_t)tc.SY, (cuuint32_t)tc.SZ};
  const cuuint32_t estr[3] = {1, 1, 1};
  if (enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, (void*)d_fw, dims, strides, box, estr,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return CG_ERR_ARG;
  const size_t smem = tma_smem(tc, NS);
  int per_sm = 0;
  CG_CUDA(kernel_occupancy((const void*)k_degrid_tma<W, NT, NS>, NT, smem, &per_sm));
  if (per_sm < 1) return CG_ERR_ARG;
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) sms = 148;
  }
  const int blocks = std::min(tc.nitems, per_sm * sms);
  int stage_tries = kWaitTries;
  if (const char* e = getenv("CG_TMA_STAGE_WAIT_TRIES")) stage_tries = std::max(0, std::min(atoi(e), kWaitTries));
  CG_CUDA(cudaMemsetAsync(d_counter, 0, sizeof(int), st));
  k_degrid_tma<W, NT, NS><<<blocks, NT, smem, st>>>(map, d_recs, d_perm, d_hive_start, M, g, tc,
                                                    (const float2*)d_fw, d_vis, d_counter, d_err,
                                                    stage_tries);
  count_launches(1);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

}  // namespace

bool degrid_tma_supported(const Geom& g, int variant) {
  TmaTile tc{};
  if (g.kw < 4 || g.kw > 8 || !tma_tiling(g, tc, variant)) return false;
  const char* e = getenv("CG_DEGRID_TMA");
  return !(e && atoi(e) == 0) && encode_fn() != nullptr;
}

int launch_degrid_tma(const Rec<float>* d_recs, const int* d_perm, const int* d_hive_start,
                      int64_t M, const Geom& g, const float* d_fw, float* d_vis, int* d_counter,
                      int* d_err, cudaStream_t st, int variant) {
  if (M == 0) return CG_OK;
  TmaTile tc{};
  if (!tma_tiling(g, tc, variant)) return CG_ERR_ARG;
#define CG_TMA_CALL(w)                                                                        \
  (variant >= 3   ? launch_w<w, 128, 1>(d_recs, d_perm, d_hive_start, M, g, tc, d_fw, d_vis,  \
                                        d_counter, d_err, st)                               \
   : variant == 2 ? launch_w<w, 256, 1>(d_recs, d_perm, d_hive_start, M, g, tc, d_fw, d_vis,  \
                                        d_counter, d_err, st)                               \
                  : launch_w<w, 512, 2>(d_recs, d_perm, d_hive_start, M, g, tc, d_fw, d_vis,  \
                                        d_counter, d_err, st))
  switch (g.kw) {
    case 4: return CG_TMA_CALL(4);
    case 5: return CG_TMA_CALL(5);
    case 6: return CG_TMA_CALL(6);
    case 7: return CG_TMA_CALL(7);
    case 8: return CG_TMA_CALL(8);
    default: return CG_ERR_ARG;
  }
#undef CG_TMA_CALL
}

}  // namespace cg
