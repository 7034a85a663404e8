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
// Method 0 here ("direct"): input-driven over the hive-sorted stream; each
// row evaluates 3W kernel values once and adds its W^3 taps with
// hardware float/double atomics (gridding) or gathers them (degridding).
#include "cg_coords.cuh"
#include "cg_launch.cuh"

namespace cg {

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
    if (bx >= nf1 || by >= nf2 || bz >= nw) continue;  // cells always in range; never indexes wild
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

template <typename T, int W>
static int grid_w(const Rec<T>* d_recs, const int* d_hive_start, int64_t M, const Geom& g, T* d_fw,
                  int method, cudaStream_t st) {
  (void)d_hive_start;
  (void)method;
  if (M == 0) return CG_OK;
  int blocks = (int)((M + 255) / 256);
  if (blocks > 148 * 64) blocks = 148 * 64;
  k_grid_direct<T, W><<<blocks, 256, 0, st>>>(d_recs, M, g, d_fw);
  count_launches(1);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

template <typename T, int W>
static int degrid_w(const Rec<T>* d_recs, const int* d_perm, const int* d_hive_start, int64_t M,
                    const Geom& g, const T* d_fw, T* d_vis, int method, cudaStream_t st) {
  (void)d_hive_start;
  (void)method;
  if (M == 0) return CG_OK;
  int blocks = (int)((M + 255) / 256);
  if (blocks > 148 * 64) blocks = 148 * 64;
  k_degrid_direct<T, W><<<blocks, 256, 0, st>>>(d_recs, d_perm, M, g, d_fw, d_vis);
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
                int method, cudaStream_t st) {
#define CG_GRID_CALL(w) grid_w<T, w>(d_recs, d_hive_start, M, g, d_fw, method, st)
  CG_W_SWITCH(g.kw, CG_GRID_CALL)
#undef CG_GRID_CALL
}

template <typename T>
int launch_degrid(const Rec<T>* d_recs, const int* d_perm, const int* d_hive_start, int64_t M,
                  const Geom& g, const T* d_fw, T* d_vis, int method, cudaStream_t st) {
#define CG_DEGRID_CALL(w) degrid_w<T, w>(d_recs, d_perm, d_hive_start, M, g, d_fw, d_vis, method, st)
  CG_W_SWITCH(g.kw, CG_DEGRID_CALL)
#undef CG_DEGRID_CALL
}

template int launch_grid<float>(const Rec<float>*, const int*, int64_t, const Geom&, float*, int,
                                cudaStream_t);
template int launch_grid<double>(const Rec<double>*, const int*, int64_t, const Geom&, double*, int,
                                 cudaStream_t);
template int launch_degrid<float>(const Rec<float>*, const int*, const int*, int64_t, const Geom&,
                                  const float*, float*, int, cudaStream_t);
template int launch_degrid<double>(const Rec<double>*, const int*, const int*, int64_t,
                                   const Geom&, const double*, double*, int, cudaStream_t);

}  // namespace cg
