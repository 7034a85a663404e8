// Tensor-core gridding (FP32 precision-split path, W <= 8).
//
// Same periodic 3-D ES convolution as conv_3d_outputdriven_t1 (reference
// conv.cu:522-627), re-cast as one small GEMM per 8x8x1 hive of the sorted
// stream.  All rows of a hive share the hive's plane, so their taps fall in
// one block of EZ planes x EXT rows x EXT columns around the hive
// (EXT = 8 + W - 1, EZ = W for even W; one more for odd W).  For the rows j
// of the hive:
//
//   G[(z, y, re/im), x] = sum_j A[(z, y, re/im), j] * B[j, x]
//   A = Re/Im(c_j) * kz_j[z] * ky_j[y],   B = kx_j[x]
//
// i.e. M = 2*EZ*EXT (padded to 16), N = EXT (padded to 16), K = rows of the
// hive (in chunks of 8).  The products run on the tensor cores as split-TF32
// mma.sync.m16n8k8: every FP32 operand is split into two TF32 parts and all
// four part products are summed (residual ~2^-22 relative); each chunk's
// products go into a zeroed fragment that is added to the FP32 register
// accumulator with IEEE adds, so the tensor core's own accumulation depth
// stays 32 terms.  No per-tap shared-memory read-modify-write is needed;
// each hive's block is committed once to the zero-filled
// grid with vector reductions (red.global.add.v2.f32).  Hives with fewer than
// kMmaMinRows rows are spread directly by the warp (lanes over taps).
#include <algorithm>
#include <cstdint>
#include <cstdlib>

#include "cg_coords.cuh"
#include "cg_launch.cuh"

namespace cg {

// hives with fewer rows are spread directly (CG_MMA_MIN_ROWS overrides)
constexpr int kMmaMinRows = 4;

__device__ __forceinline__ uint32_t f2tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo) {
  hi = f2tf32(x);
  lo = f2tf32(x - __uint_as_float(hi));
}

// D += A * B, m16n8k8, A row-major 16x8 (tf32), B col-major 8x8 (tf32), D f32
__device__ __forceinline__ void mma_tf32(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2,
                                         uint32_t a3, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ void red_add_v2(float* p, float a, float b) {
  asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(p), "f"(a), "f"(b) : "memory");
}

template <int W>
struct MmaShape {
  static constexpr int ODD = W & 1;
  static constexpr int OMIN = ODD ? -(W / 2) : 1 - W / 2;  // smallest tap offset
  static constexpr int EXT = 8 + W - 1 + ODD;               // block extent along x, y
  static constexpr int EZ = W + ODD;                        // block extent along z
  static constexpr int M = 2 * EZ * EXT;
  static constexpr int MT = (M + 15) / 16;
  static constexpr int NT = (EXT + 7) / 8;
  static constexpr int TXS = NT * 8;                        // padded table width
  // m-tiles per pass: large blocks run in two passes to bound the registers
  static constexpr int MTB = MT > 10 ? (MT + 1) / 2 : MT;
};

// Per-warp shared tables of one chunk of 8 rows:
//   ckz[j][ri][z]  Re/Im(c_j) * kz_j[z - oz_j]   (0 outside the taps)
//   kyt[j][y], kxt[j][x]                         (0 outside the taps)
template <int W>
struct ChunkTables {
  float ckz[8][2][MmaShape<W>::EZ];
  float kyt[8][MmaShape<W>::TXS];
  float kxt[8][MmaShape<W>::TXS];
  float kval[8][3][W];  // kernel values of the chunk's rows (axis x, y, z)
  float frac[8][3];
  float cpl[8][2];
  int off[8][3];        // first tap, block-relative
};

template <int W>
__global__ void __launch_bounds__(256) k_grid_mma(const Rec<float>* __restrict__ recs,
                                                  const int* __restrict__ hive_start, Geom g,
                                                  float* __restrict__ fw, int min_rows,
                                                  int64_t nchunks, int64_t perm_mul) {
  using S = MmaShape<W>;
  __shared__ ChunkTables<W> tabs[8];  // one per warp (256 threads)
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  ChunkTables<W>& tb = tabs[wib];
  const int gid = lane >> 2, tig = lane & 3;
  const float beta = (float)g.beta, ec = (float)g.es_c, halfw = (float)W * 0.5f;
  const int nf1 = g.nf1, nf2 = g.nf2, nw = g.nw, nhx = g.nhx, nhy = g.nhy;
  const int64_t nh = (int64_t)nhx * nhy * g.nhz;
  const int64_t gwarp = (int64_t)blockIdx.x * (blockDim.x >> 5) + wib;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);

  // chunks of 32 hives, visited in a multiplicative permutation of their
  // order so that the dense part of the grid is spread over all warps
  for (int64_t c = gwarp; c < nchunks; c += nwarps) {
    const int64_t hbase = ((c * perm_mul) % nchunks) * 32;
    const int64_t hl = hbase + lane;
    int s0 = 0, cnt = 0;
    if (hl < nh) {
      s0 = hive_start[hl];
      cnt = hive_start[hl + 1] - s0;
    }
    unsigned todo = __ballot_sync(0xffffffffu, cnt > 0);
    while (todo) {
      const int src = __ffs(todo) - 1;
      todo &= todo - 1;
      const int64_t h = hbase + src;
      const int start = __shfl_sync(0xffffffffu, s0, src);
      const int n = __shfl_sync(0xffffffffu, cnt, src);
      const int hx = (int)(h % nhx), hy = (int)((h / nhx) % nhy), hz = (int)(h / ((int64_t)nhx * nhy));
      // block origin in grid cells (may be negative: wrapped at commit)
      const int bx0 = hx * 8 + S::OMIN, by0 = hy * 8 + S::OMIN, bz0 = hz + S::OMIN;

      if (n < min_rows) {
        // direct: lanes over the W^3 taps of one row at a time
        for (int j = 0; j < n; j++) {
          const Rec<float> r = recs[start + j];
          const int bx = (int)(r.bxy & 0xFFFFu), by = (int)(r.bxy >> 16), bz = (int)r.bz;
          const int ox = bx + tap_offset<W>(r.f[0]), oy = by + tap_offset<W>(r.f[1]);
          const int oz = bz + tap_offset<W>(r.f[2]);
          // kernel values: lane s < 3W holds axis s / W, tap s % W
          float kv = 0.f;
          if (lane < 3 * W) {
            const int ax = lane / W, i = lane - ax * W;
            const float f = ax == 0 ? r.f[0] : (ax == 1 ? r.f[1] : r.f[2]);
            kv = es_kernel<float>((float)(tap_offset<W>(f) + i) - f, beta, ec, halfw);
          }
          for (int t0 = 0; t0 < W * W * W; t0 += 32) {
            const int t = t0 + lane;
            const int dx = t % W, dy = (t / W) % W, dz = t / (W * W);
            const float kx = __shfl_sync(0xffffffffu, kv, dx);
            const float ky = __shfl_sync(0xffffffffu, kv, W + dy);
            const float kz = __shfl_sync(0xffffffffu, kv, min(2 * W + dz, 31));
            if (t < W * W * W) {
              const float k = kx * ky * kz;
              const int gx = modi(ox + dx, nf1), gy = modi(oy + dy, nf2), gz = modi(oz + dz, nw);
              const size_t o = ((size_t)gz * nf2 + gy) * nf1 + gx;
              red_add_v2(fw + 2 * o, r.c[0] * k, r.c[1] * k);
            }
          }
        }
        continue;
      }

      for (int mbase = 0; mbase < S::MT; mbase += S::MTB) {
      float acc[S::MTB][S::NT][4];
#pragma unroll
      for (int mt = 0; mt < S::MTB; mt++)
#pragma unroll
        for (int nt = 0; nt < S::NT; nt++)
#pragma unroll
          for (int e = 0; e < 4; e++) acc[mt][nt][e] = 0.f;

      for (int c0 = 0; c0 < n; c0 += 8) {
        // ---- tables of this chunk (zero-padded; rows beyond n are zero)
        __syncwarp();
        if (lane < 8) {
          float fr[3] = {0.f, 0.f, 0.f}, cr = 0.f, ci = 0.f;
          int of[3] = {-64, -64, -64};  // rows beyond n: no taps inside the block
          if (c0 + lane < n) {
            const Rec<float> r = recs[start + c0 + lane];
            fr[0] = r.f[0]; fr[1] = r.f[1]; fr[2] = r.f[2];
            cr = r.c[0]; ci = r.c[1];
            of[0] = (int)(r.bxy & 0xFFFFu) + tap_offset<W>(fr[0]) - bx0;
            of[1] = (int)(r.bxy >> 16) + tap_offset<W>(fr[1]) - by0;
            of[2] = hz + tap_offset<W>(fr[2]) - bz0;
          }
#pragma unroll
          for (int a = 0; a < 3; a++) {
            tb.frac[lane][a] = fr[a];
            tb.off[lane][a] = of[a];
          }
          tb.cpl[lane][0] = cr;
          tb.cpl[lane][1] = ci;
        }
        __syncwarp();
        for (int e = lane; e < 8 * 3 * W; e += 32) {
          const int j = e / (3 * W), ax = (e / W) % 3, i = e % W;
          const float f = tb.frac[j][ax];
          (&tb.kval[0][0][0])[e] = es_kernel<float>((float)(tap_offset<W>(f) + i) - f, beta, ec, halfw);
        }
        __syncwarp();
        {
          constexpr int NCKZ = 8 * 2 * S::EZ, NKT = 8 * S::TXS;
          for (int e = lane; e < NCKZ + 2 * NKT; e += 32) {
            float v = 0.f;
            if (e < NCKZ) {
              const int j = e / (2 * S::EZ), ri = (e / S::EZ) & 1, z = e % S::EZ;
              const int i = z - tb.off[j][2];
              if (i >= 0 && i < W) v = tb.cpl[j][ri] * tb.kval[j][2][i];
              (&tb.ckz[0][0][0])[e] = v;
            } else {
              const int e2 = e - NCKZ, ax = e2 / NKT;  // 0: y table, 1: x table
              const int j = (e2 % NKT) / S::TXS, q = e2 % S::TXS;
              const int i = q - tb.off[j][ax == 0 ? 1 : 0];
              if (i >= 0 && i < W) v = tb.kval[j][ax == 0 ? 1 : 0][i];
              if (ax == 0) (&tb.kyt[0][0])[e2 % NKT] = v;
              else (&tb.kxt[0][0])[e2 % NKT] = v;
            }
          }
        }
        __syncwarp();
        // ---- B fragments (x): b0 = B[k = tig][n = gid], b1 = B[k = tig + 4][n = gid]
        uint32_t bh[S::NT][2], bl[S::NT][2];
#pragma unroll
        for (int nt = 0; nt < S::NT; nt++) {
          split_tf32(tb.kxt[tig][nt * 8 + gid], bh[nt][0], bl[nt][0]);
          split_tf32(tb.kxt[tig + 4][nt * 8 + gid], bh[nt][1], bl[nt][1]);
        }
        // ---- A fragments (z, y, re/im) and the products
#pragma unroll
        for (int mtl = 0; mtl < S::MTB; mtl++) {
          const int mt = mbase + mtl;
          if (mt >= S::MT) break;
          const int r0 = mt * 16 + gid, r1 = r0 + 8;
          const int ri = r0 & 1;  // r1 has the same parity
          const int zy0 = r0 >> 1, zy1 = r1 >> 1;
          const int z0 = zy0 / S::EXT, y0 = zy0 % S::EXT, z1 = zy1 / S::EXT, y1 = zy1 % S::EXT;
          const bool v0 = r0 < S::M, v1 = r1 < S::M;
          float a[4];
          a[0] = v0 ? tb.ckz[tig][ri][z0] * tb.kyt[tig][y0] : 0.f;
          a[1] = v1 ? tb.ckz[tig][ri][z1] * tb.kyt[tig][y1] : 0.f;
          a[2] = v0 ? tb.ckz[tig + 4][ri][z0] * tb.kyt[tig + 4][y0] : 0.f;
          a[3] = v1 ? tb.ckz[tig + 4][ri][z1] * tb.kyt[tig + 4][y1] : 0.f;
          uint32_t ah[4], al[4];
#pragma unroll
          for (int e = 0; e < 4; e++) split_tf32(a[e], ah[e], al[e]);
#pragma unroll
          for (int nt = 0; nt < S::NT; nt++) {
            // the chunk's four split products (smallest first) into a zeroed
            // temporary; the running sum is kept with IEEE adds
            float t[4] = {0.f, 0.f, 0.f, 0.f};
            mma_tf32(t, al[0], al[1], al[2], al[3], bl[nt][0], bl[nt][1]);
            mma_tf32(t, al[0], al[1], al[2], al[3], bh[nt][0], bh[nt][1]);
            mma_tf32(t, ah[0], ah[1], ah[2], ah[3], bl[nt][0], bl[nt][1]);
            mma_tf32(t, ah[0], ah[1], ah[2], ah[3], bh[nt][0], bh[nt][1]);
#pragma unroll
            for (int e = 0; e < 4; e++) acc[mtl][nt][e] += t[e];
          }
        }
      }
      // ---- commit: rows r (re) and r + 1 (im) of a cell live in lanes gid, gid + 1
#pragma unroll
      for (int mtl = 0; mtl < S::MTB; mtl++) {
        const int mt = mbase + mtl;
        if (mt >= S::MT) break;
#pragma unroll
        for (int nt = 0; nt < S::NT; nt++) {
          float im[4];
#pragma unroll
          for (int e = 0; e < 4; e++) im[e] = __shfl_down_sync(0xffffffffu, acc[mtl][nt][e], 4);
          if ((gid & 1) == 0) {
#pragma unroll
            for (int hr = 0; hr < 2; hr++) {
              const int r = mt * 16 + gid + 8 * hr;
              if (r >= S::M) continue;
              const int zy = r >> 1, z = zy / S::EXT, y = zy % S::EXT;
              const int gz = modi(bz0 + z, nw), gy = modi(by0 + y, nf2);
              const size_t rowo = ((size_t)gz * nf2 + gy) * nf1;
#pragma unroll
              for (int cx = 0; cx < 2; cx++) {
                const int x = nt * 8 + 2 * tig + cx;
                const float re = acc[mtl][nt][2 * hr + cx], iv = im[2 * hr + cx];
                if (x < S::EXT && (re != 0.f || iv != 0.f))
                  red_add_v2(fw + 2 * (rowo + modi(bx0 + x, nf1)), re, iv);
              }
            }
          }
        }
      }
      }  // m-tile passes
    }
  }
}

template <int W>
static int grid_mma_w(const Rec<float>* d_recs, const int* d_hive_start, const Geom& g,
                      float* d_fw, cudaStream_t st) {
  const size_t G = (size_t)g.nf1 * g.nf2 * g.nw;
  CG_CUDA(cudaMemsetAsync(d_fw, 0, G * 2 * sizeof(float), st));
  int per_sm = 0;
  CG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_grid_mma<W>, 256, 0));
  if (per_sm < 1) per_sm = 1;
  int sms = 0, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t nh = (int64_t)g.nhx * g.nhy * g.nhz;
  int64_t blocks = std::min<int64_t>((int64_t)per_sm * sms, (nh + 255) / 256);
  if (blocks < 1) blocks = 1;
  const char* env = getenv("CG_MMA_MIN_ROWS");
  const int min_rows = env ? atoi(env) : kMmaMinRows;
  const int64_t nchunks = (nh + 31) / 32;
  // a prime multiplier coprime with the chunk count (a permutation mod nchunks)
  int64_t mul = 1;
  const int64_t primes[] = {1000003, 999983, 1299709, 15485863, 32452843};
  for (int64_t p : primes)
    if (nchunks % p != 0) {
      mul = p % nchunks;
      if (mul == 0) mul = 1;
      break;
    }
  k_grid_mma<W><<<(int)blocks, 256, 0, st>>>(d_recs, d_hive_start, g, d_fw, min_rows, nchunks,
                                             mul);
  count_launches(1);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

// Returns CG_ERR_ARG (nothing launched) when the kernel width is not covered;
// the caller then uses the SIMT kernels.
int launch_grid_mma(const Rec<float>* d_recs, const int* d_hive_start, const Geom& g, float* d_fw,
                    cudaStream_t st) {
  switch (g.kw) {
    case 4: return grid_mma_w<4>(d_recs, d_hive_start, g, d_fw, st);
    case 5: return grid_mma_w<5>(d_recs, d_hive_start, g, d_fw, st);
    case 6: return grid_mma_w<6>(d_recs, d_hive_start, g, d_fw, st);
    case 7: return grid_mma_w<7>(d_recs, d_hive_start, g, d_fw, st);
    case 8: return grid_mma_w<8>(d_recs, d_hive_start, g, d_fw, st);
    default: return CG_ERR_ARG;
  }
}

}  // namespace cg
