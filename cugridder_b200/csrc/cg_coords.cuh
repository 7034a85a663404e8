// Device helpers: FP64 coordinate scaling, grid-coordinate split and ES
// kernel evaluation.
//
// The coordinate chain uses explicit round-to-nearest intrinsics so that no
// multiply-add is ever contracted: the bin keys are then bit-identical to
// the reference's FP64 formulas, whatever the compiler does elsewhere.
#pragma once
#include "cg_internal.cuh"

namespace cg {

// get_effective_coordinate(..., sign) (precomp.cu:48-72), rescaling_real
// (cugridder.cu:201-202) and the u/v swap of setup_plan (cugridder.cu:191):
// a = v * f/c * 2pi * pixsize_y (grid dim 0), b = u * f/c * 2pi * pixsize_x
// (grid dim 1), w = w * (f/c*sign) * 2pi.
__device__ __forceinline__ void eff_coords(double u, double v, double w, const Geom& g,
                                           double& a, double& b, double& ww) {
  const double twopi = 2 * kPi;
  u = __dmul_rn(u, g.foc);
  v = __dmul_rn(v, g.foc);
  ww = __dmul_rn(w, g.foc * (double)g.sign);
  u = __dmul_rn(u, twopi);
  v = __dmul_rn(v, twopi);
  ww = __dmul_rn(ww, twopi);
  b = __dmul_rn(u, g.pixx);
  a = __dmul_rn(v, g.pixy);
}

// SHIFT_RESCALE(x, N, 0) (conv.h:24): fold into [-pi, pi), map to [0, N).
// A result that rounds onto N (or below 0) is folded back into [0, N); the
// reference would key such a row one hive row off (a measure-zero case).
__device__ __forceinline__ double shift_rescale(double x, int N) {
  double q = floor(__ddiv_rn(x, kM_2PI));
  double t = __dsub_rn(x, __dmul_rn(q, kM_2PI));
  double s = (t >= kPi) ? __dsub_rn(t, kM_2PI) : t;
  double X = __dmul_rn(__dadd_rn(__dmul_rn(s, kM_1_2PI), 0.5), (double)N);
  if (X >= (double)N) X = __dsub_rn(X, (double)N);
  if (X < 0.0) X = __dadd_rn(X, (double)N);
  return X;
}

// Grid coordinates of one row (pre_stage_2, cuft.cu:82-104: w' = (w - i_c)/gamma)
__device__ __forceinline__ void grid_coords(const double* __restrict__ uvw_row, const Geom& g,
                                            double& X0, double& X1, double& X2, double& w_eff) {
  double a, b;
  eff_coords(uvw_row[0], uvw_row[1], uvw_row[2], g, a, b, w_eff);
  double wp = __ddiv_rn(__dsub_rn(w_eff, g.i_center), g.gamma);
  X0 = shift_rescale(a, g.nf1);
  X1 = shift_rescale(b, g.nf2);
  X2 = shift_rescale(wp, g.nw);
}

// ES kernel phi(d) = exp(beta sqrt(1 - c d^2)) for |d| < W/2, else 0
// (conv.cu:591-618, interp.cu:17-23).
template <typename T>
__device__ __forceinline__ T es_kernel(T d, T beta, T c, T halfw);

template <>
__device__ __forceinline__ float es_kernel<float>(float d, float beta, float c, float halfw) {
  return fabsf(d) < halfw ? expf(beta * sqrtf(fmaxf(1.0f - c * d * d, 0.0f))) : 0.0f;
}
template <>
__device__ __forceinline__ double es_kernel<double>(double d, double beta, double c, double halfw) {
  return fabs(d) < halfw ? exp(beta * sqrt(fmax(1.0 - c * d * d, 0.0))) : 0.0;
}

// The W taps of one axis: first tap = b + floor(f - W/2) + 1 with f in [0,1)
// the fraction inside cell b.  The floor is taken exactly: 1 - W/2 for even
// W; -(W-1)/2 or -(W-1)/2 + 1 for odd W depending on f < 1/2.  Returns the
// offset (first tap - b) and fills k[] (taps at |d| >= W/2 get 0).
template <int W, typename T>
__device__ __forceinline__ int tap_offset(T f) {
  return (W % 2 == 0) ? 1 - W / 2 : (f < (T)0.5 ? -(W / 2) : 1 - (W / 2));
}
// Piecewise-polynomial kernel: segment i covers d in [i - W/2, i + 1 - W/2);
// tap i of a row evaluates segment i at z = (first tap - b) + W/2 - f, which
// lies in (0, 1] for every tap, as P_i(2z - 1) = sum_n a[i][n] (2z - 1)^n.
template <typename T>
__device__ __forceinline__ T poly_eval(const T* __restrict__ a, T t) {
  T v = a[kPolyCoef - 1];
#pragma unroll
  for (int n = kPolyCoef - 2; n >= 0; n--) v = fma(v, t, a[n]);
  return v;
}
template <int W, typename T>
__device__ __forceinline__ T poly_arg(T f) {
  return (T)2 * (((T)tap_offset<W>(f) + (T)W * (T)0.5) - f) - (T)1;
}
template <typename T>
__device__ __forceinline__ const T* geom_poly(const Geom& g);
template <>
__device__ __forceinline__ const float* geom_poly<float>(const Geom& g) { return g.polyf; }
template <>
__device__ __forceinline__ const double* geom_poly<double>(const Geom& g) { return g.polyd; }

template <typename T>
inline const T* geom_poly_host(const Geom& g) {
  if constexpr (sizeof(T) == 4) return (const T*)g.polyf; else return (const T*)g.polyd;
}

template <typename T, int W>
__device__ __forceinline__ int taps(T f, T beta, T c, const T* __restrict__ poly, T* k) {
  const T halfw = (T)W * (T)0.5;
  int o = tap_offset<W>(f);
  if (poly) {
    const T t = poly_arg<W>(f);
#pragma unroll
    for (int i = 0; i < W; i++) k[i] = poly_eval(poly + i * kPolyCoef, t);
  } else {
#pragma unroll
    for (int i = 0; i < W; i++) k[i] = es_kernel<T>((T)(o + i) - f, beta, c, halfw);
  }
  return o;
}

// Tap update c + (vr, vi) * k of a complex cell: for FP32 one packed
// fma.rn.f32x2 (sm_100), which rounds each half as fma.rn.f32 does, so the
// result is the same as two scalar FMAs.
__device__ __forceinline__ float2 tap_fma(float2 c, float vr, float vi, float k) {
  float2 r;
  asm("{\n.reg .b64 pv, pk, pc, pr;\n"
      "mov.b64 pv, {%2, %3};\nmov.b64 pk, {%4, %4};\nmov.b64 pc, {%5, %6};\n"
      "fma.rn.f32x2 pr, pv, pk, pc;\nmov.b64 {%0, %1}, pr;\n}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(vr), "f"(vi), "f"(k), "f"(c.x), "f"(c.y));
  return r;
}
__device__ __forceinline__ double2 tap_fma(double2 c, double vr, double vi, double k) {
  return make_double2(fma(vr, k, c.x), fma(vi, k, c.y));
}

// true modulo (any number of periods)
__device__ __forceinline__ int modi(int i, int n) {
  i %= n;
  return i < 0 ? i + n : i;
}

// one-period wrap: i in [-n, 2n)
__device__ __forceinline__ int wrapi(int i, int n) {
  i = (i >= n) ? i - n : i;
  return (i < 0) ? i + n : i;
}

// CMCL index map of deconv_2d (deconv.cu:268-272) and its inverse
__device__ __forceinline__ int cmcl(int k, int N, int nf) { return k >= N / 2 ? k - N / 2 : nf + k - N / 2; }
__device__ __forceinline__ int inv_cmcl(int g, int N, int nf) {
  if (g < N - N / 2) return g + N / 2;
  if (g >= nf - N / 2) return g - nf + N / 2;
  return -1;
}

}  // namespace cg
