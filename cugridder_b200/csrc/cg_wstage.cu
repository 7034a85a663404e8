// The w stage of improved W-stacking, fused per pixel.
//
// ms2dirty (reference: four kernels and four HBM passes, each followed by a
// device synchronize):
//   w_term_dft     cuft.cu:597-645   sum_p fw[p] exp(i z' (p - nw/2))
//   deconv_2d      deconv.cu:250-294 / (phi_hat1 phi_hat2), CMCL order
//   w_term_deconv  deconv.cu:401-432 * exp(i (z - o_c) i_c) / phi_hat3(z')
//   div_n_lm       ra_exec.cu:23-37  / n
// are one kernel here: each thread reads the nw plane values of its pixel
// once and writes the finished pixel once.
//
// dirty2ms (div_n_lm, w_term_deconv flag -1, deconv_2d type 2, w_term_idft
// cuft.cu:647-689) is one "plane fill" kernel that writes every cell of every
// plane exactly once (image values with their plane phase, zero padding
// elsewhere), so the grid needs no separate memset.
//
// Pixel geometry: row = image x (N2 axis, pixsize_x), col = image y (N1 axis,
// pixsize_y); z = n - 1 uses the cancellation-free form
// -(l^2+m^2)/(1+sqrt(1-l^2-m^2)) inside the horizon and the reference's
// sqrt(|.|) - 1 beyond it (precomp.cu:215-226); n = sqrt(1-l^2-m^2) as in
// div_n_lm (NaN beyond the horizon, like the reference).
#include "cg_coords.cuh"
#include "cg_launch.cuh"

namespace cg {

template <typename T>
struct Vec2;
template <>
struct Vec2<float> { using type = float2; };
template <>
struct Vec2<double> { using type = double2; };

// Quarter-image tables (k_generation precomp.cu:215-244 and
// fourier_series_appro deconv.cu:49-65): z = n-1 and phi_hat3(z'),
// z' = (z - o_c) * gamma * h (pre_stage_2 cuft.cu:82-104).
__global__ void k_quarter(Geom g, Quad q, double* __restrict__ K3q, double* __restrict__ zq) {
  const int nc = g.N1 / 2 + 1, nr = g.N2 / 2 + 1;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < (int64_t)nr * nc;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int r = (int)(idx / nc), cc = (int)(idx % nc);
    double l = r * g.pixx, m = cc * g.pixy;
    double e2 = l * l + m * m;
    double t = 1.0 - e2;
    double z = (t >= 0.0) ? -e2 / (1.0 + sqrt(t)) : sqrt(-t) - 1.0;
    double zp = (z - g.o_center) * g.gamma * g.h;
    double s = 0.0;
    for (int i = 0; i < q.p; i++) s += q.g[i] * 2.0 * cos(q.x[i] * zp);
    K3q[idx] = s;
    zq[idx] = z;
  }
}

int launch_quarter(const Geom& g, const Quad& q, double* d_K3q, double* d_zq, cudaStream_t st) {
  int64_t n = (int64_t)(g.N1 / 2 + 1) * (g.N2 / 2 + 1);
  int blocks = (int)((n + 255) / 256);
  if (blocks > 148 * 32) blocks = 148 * 32;
  k_quarter<<<blocks, 256, 0, st>>>(g, q, d_K3q, d_zq);
  count_launches(1);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

// per-pixel correction: 1 / (phi_hat1 phi_hat2 phi_hat3 n) * exp(i flag (z - o_c) i_c)
__device__ __forceinline__ void pixel_factor(const Geom& g, int row, int col,
                                             const double* __restrict__ K1,
                                             const double* __restrict__ K2,
                                             const double* __restrict__ K3q,
                                             const double* __restrict__ zq, double flag,
                                             double& fr, double& fi, double& zp) {
  const int dr = abs(row - g.N2 / 2), dc = abs(col - g.N1 / 2);
  const int iq = dr * (g.N1 / 2 + 1) + dc;
  const double z = zq[iq];
  zp = (z - g.o_center) * g.gamma * g.h;
  const double l = (row - g.N2 / 2) * g.pixx, m = (col - g.N1 / 2) * g.pixy;
  const double n = sqrt(1.0 - l * l - m * m);
  const double scale = 1.0 / (K1[dc] * K2[dr] * K3q[iq] * n);
  double sn, cs;
  sincos((z - g.o_center) * g.i_center * flag, &sn, &cs);
  fr = cs * scale;
  fi = sn * scale;
}

template <typename T>
__global__ void k_wdft_deconv(const T* __restrict__ fw, Geom g, const double* __restrict__ K1,
                              const double* __restrict__ K2, const double* __restrict__ K3q,
                              const double* __restrict__ zq, T* __restrict__ dirty) {
  using V = typename Vec2<T>::type;
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = blockIdx.y;
  if (col >= g.N1) return;
  const size_t plane = (size_t)g.nf1 * g.nf2;
  const size_t idx = (size_t)row_of(g, cmcl(row, g.N2, g.nf2)) * g.nf1 + cmcl(col, g.N1, g.nf1);
  double fr, fi, zp;
  pixel_factor(g, row, col, K1, K2, K3q, zq, 1.0, fr, fi, zp);
  // sum_p fw[p] exp(i zp (p - nw/2)), phase by rotation
  double sn, cs, pr, pi;
  sincos(zp, &sn, &cs);
  sincos(zp * (double)(-(g.nw / 2)), &pi, &pr);
  double sr = 0.0, si = 0.0;
  const V* f = reinterpret_cast<const V*>(fw) + idx;
  // planes in groups of kAhead: the group's loads are issued before the
  // rotation recurrence consumes them
  constexpr int kAhead = 8;
  for (int p0 = 0; p0 < g.nw; p0 += kAhead) {
    V v[kAhead];
#pragma unroll
    for (int k = 0; k < kAhead; k++)
      if (p0 + k < g.nw) v[k] = f[(size_t)(p0 + k) * plane];
#pragma unroll
    for (int k = 0; k < kAhead; k++) {
      if (p0 + k < g.nw) {
        sr += (double)v[k].x * pr - (double)v[k].y * pi;
        si += (double)v[k].x * pi + (double)v[k].y * pr;
        double t = pr * cs - pi * sn;
        pi = pr * sn + pi * cs;
        pr = t;
      }
    }
  }
  V out;
  out.x = (T)(sr * fr - si * fi);
  out.y = (T)(sr * fi + si * fr);
  reinterpret_cast<V*>(dirty)[(size_t)row * g.N1 + col] = out;
}

template <typename T>
int launch_wdft_deconv(const T* d_fw, const Geom& g, const double* d_K1, const double* d_K2,
                       const double* d_K3q, const double* d_zq, T* d_dirty, cudaStream_t st) {
  dim3 block(128);
  dim3 grid((g.N1 + 127) / 128, g.N2);
  k_wdft_deconv<T><<<grid, block, 0, st>>>(d_fw, g, d_K1, d_K2, d_K3q, d_zq, d_dirty);
  count_launches(1);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

template <typename T>
__global__ void k_plane_fill(const T* __restrict__ dirty, Geom g, const double* __restrict__ K1,
                             const double* __restrict__ K2, const double* __restrict__ K3q,
                             const double* __restrict__ zq, T* __restrict__ fw) {
  using V = typename Vec2<T>::type;
  const int g0 = blockIdx.x * blockDim.x + threadIdx.x;
  const int g1 = blockIdx.y;
  if (g0 >= g.nf1) return;
  const size_t plane = (size_t)g.nf1 * g.nf2;
  V* f = reinterpret_cast<V*>(fw) + (size_t)row_of(g, g1) * g.nf1 + g0;
  const int col = inv_cmcl(g0, g.N1, g.nf1), row = inv_cmcl(g1, g.N2, g.nf2);
  if (col < 0 || row < 0) {
    // cells in the image's columns but outside its rows are neither loaded
    // nor kept by the one-pass forward column transform, and cells outside
    // the image's columns are read only by the row pass, in its rows: no
    // zeros needed elsewhere
    if (g.fill_skip) {
      if (col >= 0) return;
      int r0, n;
      fft_row_band(g, r0, n);
      if (g1 < r0 || g1 >= r0 + n) return;
    }
    V zero;
    zero.x = (T)0;
    zero.y = (T)0;
    for (int p = 0; p < g.nw; p++) f[(size_t)p * plane] = zero;
    return;
  }
  double fr, fi, zp;
  pixel_factor(g, row, col, K1, K2, K3q, zq, -1.0, fr, fi, zp);
  const V d = reinterpret_cast<const V*>(dirty)[(size_t)row * g.N1 + col];
  const double br = (double)d.x * fr - (double)d.y * fi;
  const double bi = (double)d.x * fi + (double)d.y * fr;
  // plane p gets b * exp(-i zp (p - nw/2))  (w_term_idft, flag = -1)
  double sn, cs, pr, pi;
  sincos(-zp, &sn, &cs);
  sincos(-zp * (double)(-(g.nw / 2)), &pi, &pr);
  for (int p = 0; p < g.nw; p++) {
    V o;
    o.x = (T)(br * pr - bi * pi);
    o.y = (T)(br * pi + bi * pr);
    f[(size_t)p * plane] = o;
    double t = pr * cs - pi * sn;
    pi = pr * sn + pi * cs;
    pr = t;
  }
}

template <typename T>
int launch_plane_fill(const T* d_dirty, const Geom& g, const double* d_K1, const double* d_K2,
                      const double* d_K3q, const double* d_zq, T* d_fw, cudaStream_t st) {
  dim3 block(128);
  dim3 grid((g.nf1 + 127) / 128, g.nf2);
  k_plane_fill<T><<<grid, block, 0, st>>>(d_dirty, g, d_K1, d_K2, d_K3q, d_zq, d_fw);
  count_launches(1);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

// Memory-limited mode: the w-DFT of k_wdft_deconv split over plane windows.
// acc[pixel] (FP64) += sum_{p in [p0, p1)} fwb[p - p0] exp(i zp (p - nw/2));
// k_wdft_finish then applies the per-pixel correction.
template <typename T>
__global__ void k_wdft_accum(const T* __restrict__ fwb, Geom g, int p0, int p1,
                             const double* __restrict__ zq, double2* __restrict__ acc) {
  using V = typename Vec2<T>::type;
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = blockIdx.y;
  if (col >= g.N1) return;
  const size_t plane = (size_t)g.nf1 * g.nf2;
  const size_t idx = (size_t)cmcl(row, g.N2, g.nf2) * g.nf1 + cmcl(col, g.N1, g.nf1);
  const int dr = abs(row - g.N2 / 2), dc = abs(col - g.N1 / 2);
  const double zp = (zq[dr * (g.N1 / 2 + 1) + dc] - g.o_center) * g.gamma * g.h;
  double sn, cs, pr, pi;
  sincos(zp, &sn, &cs);
  sincos(zp * (double)(p0 - g.nw / 2), &pi, &pr);
  double sr = 0.0, si = 0.0;
  const V* f = reinterpret_cast<const V*>(fwb) + idx;
  for (int p = p0; p < p1; p++) {
    const V v = f[(size_t)(p - p0) * plane];
    sr += (double)v.x * pr - (double)v.y * pi;
    si += (double)v.x * pi + (double)v.y * pr;
    const double t = pr * cs - pi * sn;
    pi = pr * sn + pi * cs;
    pr = t;
  }
  double2& a = acc[(size_t)row * g.N1 + col];
  a.x += sr;
  a.y += si;
}

template <typename T>
__global__ void k_wdft_finish(const double2* __restrict__ acc, Geom g, const double* __restrict__ K1,
                              const double* __restrict__ K2, const double* __restrict__ K3q,
                              const double* __restrict__ zq, T* __restrict__ dirty) {
  using V = typename Vec2<T>::type;
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = blockIdx.y;
  if (col >= g.N1) return;
  double fr, fi, zp;
  pixel_factor(g, row, col, K1, K2, K3q, zq, 1.0, fr, fi, zp);
  const double2 a = acc[(size_t)row * g.N1 + col];
  V out;
  out.x = (T)(a.x * fr - a.y * fi);
  out.y = (T)(a.x * fi + a.y * fr);
  reinterpret_cast<V*>(dirty)[(size_t)row * g.N1 + col] = out;
}

// planes [p0, p1) of k_plane_fill (plane p at fwb + (p - p0) * plane)
template <typename T>
__global__ void k_plane_fill_window(const T* __restrict__ dirty, Geom g, int p0, int p1,
                                    const double* __restrict__ K1, const double* __restrict__ K2,
                                    const double* __restrict__ K3q, const double* __restrict__ zq,
                                    T* __restrict__ fwb) {
  using V = typename Vec2<T>::type;
  const int g0 = blockIdx.x * blockDim.x + threadIdx.x;
  const int g1 = blockIdx.y;
  if (g0 >= g.nf1) return;
  const size_t plane = (size_t)g.nf1 * g.nf2;
  V* f = reinterpret_cast<V*>(fwb) + (size_t)g1 * g.nf1 + g0;
  const int col = inv_cmcl(g0, g.N1, g.nf1), row = inv_cmcl(g1, g.N2, g.nf2);
  if (col < 0 || row < 0) {
    V zero;
    zero.x = (T)0;
    zero.y = (T)0;
    for (int p = p0; p < p1; p++) f[(size_t)(p - p0) * plane] = zero;
    return;
  }
  double fr, fi, zp;
  pixel_factor(g, row, col, K1, K2, K3q, zq, -1.0, fr, fi, zp);
  const V d = reinterpret_cast<const V*>(dirty)[(size_t)row * g.N1 + col];
  const double br = (double)d.x * fr - (double)d.y * fi;
  const double bi = (double)d.x * fi + (double)d.y * fr;
  double sn, cs, pr, pi;
  sincos(-zp, &sn, &cs);
  sincos(-zp * (double)(p0 - g.nw / 2), &pi, &pr);
  for (int p = p0; p < p1; p++) {
    V o;
    o.x = (T)(br * pr - bi * pi);
    o.y = (T)(br * pi + bi * pr);
    f[(size_t)(p - p0) * plane] = o;
    const double t = pr * cs - pi * sn;
    pi = pr * sn + pi * cs;
    pr = t;
  }
}

template <typename T>
int launch_wdft_window(const T* d_fwb, const Geom& g, int p0, int p1, const double* d_zq,
                       double* d_acc, cudaStream_t st) {
  dim3 grid((g.N1 + 127) / 128, g.N2);
  k_wdft_accum<T><<<grid, 128, 0, st>>>(d_fwb, g, p0, p1, d_zq, (double2*)d_acc);
  count_launches(1);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

template <typename T>
int launch_wdft_finish(const double* d_acc, const Geom& g, const double* d_K1, const double* d_K2,
                       const double* d_K3q, const double* d_zq, T* d_dirty, cudaStream_t st) {
  dim3 grid((g.N1 + 127) / 128, g.N2);
  k_wdft_finish<T><<<grid, 128, 0, st>>>((const double2*)d_acc, g, d_K1, d_K2, d_K3q, d_zq, d_dirty);
  count_launches(1);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

template <typename T>
int launch_plane_fill_window(const T* d_dirty, const Geom& g, int p0, int p1, const double* d_K1,
                             const double* d_K2, const double* d_K3q, const double* d_zq, T* d_fwb,
                             cudaStream_t st) {
  dim3 grid((g.nf1 + 127) / 128, g.nf2);
  k_plane_fill_window<T><<<grid, 128, 0, st>>>(d_dirty, g, p0, p1, d_K1, d_K2, d_K3q, d_zq, d_fwb);
  count_launches(1);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

template int launch_wdft_window<float>(const float*, const Geom&, int, int, const double*, double*,
                                       cudaStream_t);
template int launch_wdft_window<double>(const double*, const Geom&, int, int, const double*,
                                        double*, cudaStream_t);
template int launch_wdft_finish<float>(const double*, const Geom&, const double*, const double*,
                                       const double*, const double*, float*, cudaStream_t);
template int launch_wdft_finish<double>(const double*, const Geom&, const double*, const double*,
                                        const double*, const double*, double*, cudaStream_t);
template int launch_plane_fill_window<float>(const float*, const Geom&, int, int, const double*,
                                             const double*, const double*, const double*, float*,
                                             cudaStream_t);
template int launch_plane_fill_window<double>(const double*, const Geom&, int, int, const double*,
                                              const double*, const double*, const double*,
                                              double*, cudaStream_t);

template int launch_wdft_deconv<float>(const float*, const Geom&, const double*, const double*,
                                       const double*, const double*, float*, cudaStream_t);
template int launch_wdft_deconv<double>(const double*, const Geom&, const double*, const double*,
                                        const double*, const double*, double*, cudaStream_t);
template int launch_plane_fill<float>(const float*, const Geom&, const double*, const double*,
                                      const double*, const double*, float*, cudaStream_t);
template int launch_plane_fill<double>(const double*, const Geom&, const double*, const double*,
                                       const double*, const double*, double*, cudaStream_t);

}  // namespace cg
