// Generic type-1 / type-2 NUFFT in 1, 2 and 3 dimensions: the front end the
// reference exposes as cunufft_setting + curafft_conv / cufft / curafft_deconv
// (cuft.cu:327-545, driven by test/nufft_{1d,2d_1,2d_2,3d_1,3d_2}_test.cu),
// built on this library's pieces: the ES kernel and its Gauss-Legendre
// Fourier series (setup_conv_opts, make_quad, fseries_uv), the stable radix
// sort, and cuFFT for the uniform transform.
//
// Conventions (the reference tests' direct sums):
//   type 1: fk[k3][k2][k1] = sum_j c_j exp(i iflag ((k1 - N1/2) x_j
//                                  + (k2 - N2/2) y_j + (k3 - N3/2) z_j))
//   type 2: c_j = sum_k fk[k3][k2][k1] exp(i iflag (...))
// with coordinates in radians (any real value; period 2 pi), k1 fastest.
// Points are sorted by 16^d cell bins so spreading atomics and
// interpolation gathers stay local.
#include <algorithm>
#include <cmath>
#include <vector>

#include "cg_coords.cuh"
#include "cg_launch.cuh"
#include "cg_plan.cuh"

namespace {

struct NufftGeom {
  int dim;
  int nf[3];
  int64_t N[3];
  double beta, es_c;
};

template <typename T>
struct alignas(16) NRec {
  T f[3];     // fraction inside the cell
  int c[3];   // cell index in [0, nf)
};

template <typename T>
__global__ void k_nufft_points(int64_t M, const double* __restrict__ x, const double* __restrict__ y,
                               const double* __restrict__ z, NufftGeom g, NRec<T>* __restrict__ tmp,
                               uint32_t* __restrict__ keys) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < M;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double* src[3] = {x, y, z};
    NRec<T> r;
    uint32_t key = 0, mul = 1;
#pragma unroll
    for (int d = 0; d < 3; d++) {
      int c = 0;
      T f = (T)0;
      if (d < g.dim) {
        const double X = cg::shift_rescale(src[d][i], g.nf[d]);
        const double fl = floor(X);
        c = (int)fl;
        if (c >= g.nf[d]) c = g.nf[d] - 1;  // never taken: shift_rescale returns [0, nf)
        f = (T)(X - fl);
        const T below1 = sizeof(T) == 4 ? (T)0.99999994f : (T)0.99999999999999989;
        if (f >= (T)1) f = below1;
        key += mul * (uint32_t)(c >> 4);
        mul *= (uint32_t)((g.nf[d] + 15) >> 4);
      }
      r.c[d] = c;
      r.f[d] = f;
    }
    tmp[i] = r;
    keys[i] = key;
  }
}

template <typename T>
__global__ void k_nufft_gather(const int* __restrict__ perm, int64_t M, const NRec<T>* __restrict__ tmp,
                               NRec<T>* __restrict__ recs) {
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < M;
       s += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = perm[s];
    if (i >= 0 && i < M) recs[s] = tmp[i];
  }
}

// kernel values of the taps along one axis (a delta for the absent axes)
template <typename T, int W>
__device__ __forceinline__ int nufft_taps(const NRec<T>& r, int d, const NufftGeom& g, T* k) {
  if (d >= g.dim) {
#pragma unroll
    for (int i = 0; i < W; i++) k[i] = (T)(i == 0 ? 1 : 0);
    return 0;
  }
  return r.c[d] + cg::taps<T, W>(r.f[d], (T)g.beta, (T)g.es_c, nullptr, k);
}

template <typename T>
__device__ __forceinline__ void atomic_add_c(T* p, T re, T im) {
  atomicAdd(p, re);
  atomicAdd(p + 1, im);
}

// type 1 spreading: one thread per sorted point, W^dim taps with atomics
template <typename T, int W, int DIM>
__global__ void __launch_bounds__(256) k_nufft_spread(const NRec<T>* __restrict__ recs,
                                                      const int* __restrict__ perm, int64_t M,
                                                      NufftGeom g, const T* __restrict__ c,
                                                      T* __restrict__ fw) {
  constexpr int WY = DIM >= 2 ? W : 1, WZ = DIM >= 3 ? W : 1;
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < M;
       s += (int64_t)gridDim.x * blockDim.x) {
    const NRec<T> r = recs[s];
    const int64_t j = perm[s];
    if (j < 0 || j >= M) continue;
    const T cr = c[2 * j], ci = c[2 * j + 1];
    T kx[W], ky[W], kz[W];
    const int ox = nufft_taps<T, W>(r, 0, g, kx);
    const int oy = nufft_taps<T, W>(r, 1, g, ky);
    const int oz = nufft_taps<T, W>(r, 2, g, kz);
    for (int a = 0; a < WZ; a++) {
      const int zz = DIM >= 3 ? cg::wrapi(oz + a, g.nf[2]) : 0;
      for (int b = 0; b < WY; b++) {
        const int yy = DIM >= 2 ? cg::wrapi(oy + b, g.nf[1]) : 0;
        const T kyz = ky[b] * kz[a];
        T* row = fw + 2 * (((size_t)zz * g.nf[1] + yy) * g.nf[0]);
#pragma unroll
        for (int e = 0; e < W; e++) {
          const T k = kyz * kx[e];
          atomic_add_c(row + 2 * cg::wrapi(ox + e, g.nf[0]), cr * k, ci * k);
        }
      }
    }
  }
}

// type 2 interpolation: c[perm[s]] = sum over taps of fw * kernel
template <typename T, int W, int DIM>
__global__ void __launch_bounds__(256) k_nufft_interp(const NRec<T>* __restrict__ recs,
                                                      const int* __restrict__ perm, int64_t M,
                                                      NufftGeom g, const T* __restrict__ fw,
                                                      T* __restrict__ c) {
  constexpr int WY = DIM >= 2 ? W : 1, WZ = DIM >= 3 ? W : 1;
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < M;
       s += (int64_t)gridDim.x * blockDim.x) {
    const NRec<T> r = recs[s];
    const int64_t j = perm[s];
    if (j < 0 || j >= M) continue;
    T kx[W], ky[W], kz[W];
    const int ox = nufft_taps<T, W>(r, 0, g, kx);
    const int oy = nufft_taps<T, W>(r, 1, g, ky);
    const int oz = nufft_taps<T, W>(r, 2, g, kz);
    T sr = 0, si = 0;
    for (int a = 0; a < WZ; a++) {
      const int zz = DIM >= 3 ? cg::wrapi(oz + a, g.nf[2]) : 0;
      for (int b = 0; b < WY; b++) {
        const int yy = DIM >= 2 ? cg::wrapi(oy + b, g.nf[1]) : 0;
        const T* row = fw + 2 * (((size_t)zz * g.nf[1] + yy) * g.nf[0]);
        T qr = 0, qi = 0;
#pragma unroll
        for (int e = 0; e < W; e++) {
          const int xx = cg::wrapi(ox + e, g.nf[0]);
          qr += row[2 * xx] * kx[e];
          qi += row[2 * xx + 1] * kx[e];
        }
        const T kyz = ky[b] * kz[a];
        sr += qr * kyz;
        si += qi * kyz;
      }
    }
    c[2 * j] = sr;
    c[2 * j + 1] = si;
  }
}

// modes <-> fine grid with the deconvolution (deconv_2d, deconv.cu:250-294,
// generalised to d dimensions; CMCL index map, (-1)^k folded into K):
//   to_modes: fk[k] = fw[cmcl(k)] / prod_d K_d[|k_d - N_d/2|]
//   to_grid:  fw[cmcl(k)] = fk[k] / prod_d K_d[...]  (fw zeroed beforehand)
template <typename T, bool kToModes>
__global__ void k_nufft_deconv(NufftGeom g, const double* __restrict__ K0,
                               const double* __restrict__ K1, const double* __restrict__ K2,
                               T* __restrict__ fw, T* __restrict__ fk) {
  const int64_t nmodes = g.N[0] * g.N[1] * g.N[2];
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nmodes;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k0 = q % g.N[0], k1 = (q / g.N[0]) % g.N[1], k2 = q / (g.N[0] * g.N[1]);
    const int w0 = cg::cmcl((int)k0, (int)g.N[0], g.nf[0]);
    double kv = K0[abs((int)(k0 - g.N[0] / 2))];
    int w1 = 0, w2 = 0;
    if (g.dim >= 2) {
      w1 = cg::cmcl((int)k1, (int)g.N[1], g.nf[1]);
      kv *= K1[abs((int)(k1 - g.N[1] / 2))];
    }
    if (g.dim >= 3) {
      w2 = cg::cmcl((int)k2, (int)g.N[2], g.nf[2]);
      kv *= K2[abs((int)(k2 - g.N[2] / 2))];
    }
    const size_t o = ((size_t)w2 * g.nf[1] + w1) * g.nf[0] + w0;
    const double inv = 1.0 / kv;
    if (kToModes) {
      fk[2 * q] = (T)((double)fw[2 * o] * inv);
      fk[2 * q + 1] = (T)((double)fw[2 * o + 1] * inv);
    } else {
      fw[2 * o] = (T)((double)fk[2 * q] * inv);
      fw[2 * o + 1] = (T)((double)fk[2 * q + 1] * inv);
    }
  }
}

int blocks_for(int64_t n) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 32));
}

}  // namespace

struct cg_nufft_s {
  int device = 0;
  cudaStream_t stream = nullptr;
  int type = 1, precision = CG_PREC_FP64, iflag = 1;
  NufftGeom g{};
  int kw = 0;
  int eps_status = CG_OK;
  int64_t M = 0;
  bool have_pts = false;
  cg_dev_buf K[3], fw, recs, tmp, keys, skeys, perm, ws;
  cufftHandle fft = 0;
  bool fft_valid = false;
};

namespace {

void free_nufft(cg_nufft_s* P) {
  if (!P) return;
  cudaSetDevice(P->device);
  if (P->fft_valid) cufftDestroy(P->fft);
  cg_dev_buf* bs[] = {&P->K[0], &P->K[1], &P->K[2], &P->fw,   &P->recs,
                      &P->tmp,  &P->keys, &P->skeys, &P->perm, &P->ws};
  for (auto b : bs) cg::release(*b);
  delete P;
}

template <typename T>
int spread_or_interp(cg_nufft_s* P, void* d_c) {
  const NufftGeom& g = P->g;
  const int64_t M = P->M;
  if (M == 0) return CG_OK;
  const NRec<T>* recs = (const NRec<T>*)P->recs.p;
  const int* perm = (const int*)P->perm.p;
  T* fw = (T*)P->fw.p;
  const int blocks = blocks_for(M);
#define CG_NUFFT_CASE(W, D)                                                                     \
  if (P->kw == W && g.dim == D) {                                                               \
    if (P->type == 1)                                                                           \
      k_nufft_spread<T, W, D><<<blocks, 256, 0, P->stream>>>(recs, perm, M, g, (const T*)d_c, fw); \
    else                                                                                        \
      k_nufft_interp<T, W, D><<<blocks, 256, 0, P->stream>>>(recs, perm, M, g, fw, (T*)d_c);     \
    cg::count_launches(1);                                                                      \
    CG_CUDA(cudaGetLastError());                                                                \
    return CG_OK;                                                                               \
  }
#define CG_NUFFT_W(W) CG_NUFFT_CASE(W, 1) CG_NUFFT_CASE(W, 2) CG_NUFFT_CASE(W, 3)
  CG_NUFFT_W(2) CG_NUFFT_W(3) CG_NUFFT_W(4) CG_NUFFT_W(5) CG_NUFFT_W(6) CG_NUFFT_W(7)
  CG_NUFFT_W(8) CG_NUFFT_W(9) CG_NUFFT_W(10) CG_NUFFT_W(11) CG_NUFFT_W(12) CG_NUFFT_W(13)
  CG_NUFFT_W(14) CG_NUFFT_W(15) CG_NUFFT_W(16)
#undef CG_NUFFT_W
#undef CG_NUFFT_CASE
  return CG_ERR_ARG;
}

template <typename T>
int deconv(cg_nufft_s* P, void* d_fk, bool to_modes) {
  const NufftGeom& g = P->g;
  const int64_t n = g.N[0] * g.N[1] * g.N[2];
  const double* K0 = (const double*)P->K[0].p;
  const double* K1 = g.dim >= 2 ? (const double*)P->K[1].p : K0;
  const double* K2 = g.dim >= 3 ? (const double*)P->K[2].p : K0;
  if (to_modes)
    k_nufft_deconv<T, true><<<blocks_for(n), 256, 0, P->stream>>>(g, K0, K1, K2, (T*)P->fw.p, (T*)d_fk);
  else
    k_nufft_deconv<T, false><<<blocks_for(n), 256, 0, P->stream>>>(g, K0, K1, K2, (T*)P->fw.p, (T*)d_fk);
  cg::count_launches(1);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

template <typename T>
int setpts_t(cg_nufft_s* P, int64_t M, const double* x, const double* y, const double* z) {
  const NufftGeom& g = P->g;
  CG_TRY(cg::ensure(P->tmp, sizeof(NRec<T>) * (size_t)std::max<int64_t>(M, 1)));
  CG_TRY(cg::ensure(P->recs, sizeof(NRec<T>) * (size_t)std::max<int64_t>(M, 1)));
  CG_TRY(cg::ensure(P->keys, 4 * (size_t)std::max<int64_t>(M, 1)));
  CG_TRY(cg::ensure(P->skeys, 4 * (size_t)std::max<int64_t>(M, 1)));
  CG_TRY(cg::ensure(P->perm, 4 * (size_t)std::max<int64_t>(M, 1)));
  CG_TRY(cg::ensure(P->ws, cg::bin_workspace_bytes(M, 4)));
  if (M == 0) return CG_OK;
  k_nufft_points<T><<<blocks_for(M), 256, 0, P->stream>>>(M, x, y, z, g, (NRec<T>*)P->tmp.p,
                                                          (uint32_t*)P->keys.p);
  cg::count_launches(1);
  CG_CUDA(cudaGetLastError());
  uint64_t nb = 1;
  for (int d = 0; d < g.dim; d++) nb *= (uint64_t)((g.nf[d] + 15) >> 4);
  int bits = 1;
  while (bits < 32 && (nb >> bits) != 0) bits++;
  CG_TRY(cg::launch_sort_u32((uint32_t*)P->keys.p, M, bits, P->ws.p, P->ws.cap, (int*)P->perm.p,
                             (uint32_t*)P->skeys.p, P->stream));
  k_nufft_gather<T><<<blocks_for(M), 256, 0, P->stream>>>((const int*)P->perm.p, M,
                                                          (const NRec<T>*)P->tmp.p,
                                                          (NRec<T>*)P->recs.p);
  cg::count_launches(1);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

template <typename T>
int execute_t(cg_nufft_s* P, void* d_c, void* d_fk) {
  const NufftGeom& g = P->g;
  const size_t G = (size_t)g.nf[0] * g.nf[1] * g.nf[2];
  CG_CUDA(cudaMemsetAsync(P->fw.p, 0, G * 2 * sizeof(T), P->stream));
  const int dir = P->iflag >= 0 ? CUFFT_INVERSE : CUFFT_FORWARD;
  CG_CUFFT(cufftSetStream(P->fft, P->stream));
  auto fft = [&]() -> int {
    if (sizeof(T) == 8)
      CG_CUFFT(cufftExecZ2Z(P->fft, (cufftDoubleComplex*)P->fw.p, (cufftDoubleComplex*)P->fw.p, dir));
    else
      CG_CUFFT(cufftExecC2C(P->fft, (cufftComplex*)P->fw.p, (cufftComplex*)P->fw.p, dir));
    return CG_OK;
  };
  if (P->type == 1) {
    CG_TRY(spread_or_interp<T>(P, d_c));
    CG_TRY(fft());
    CG_TRY(deconv<T>(P, d_fk, true));
  } else {
    CG_TRY(deconv<T>(P, d_fk, false));
    CG_TRY(fft());
    CG_TRY(spread_or_interp<T>(P, d_c));
  }
  return CG_OK;
}

}  // namespace

extern "C" {

int cg_nufft_create(cg_nufft_s** plan, int type, int dim, const int64_t* nmodes, int iflag,
                    double epsilon, double sigma, int precision, void* stream) {
  if (!plan) return CG_ERR_ARG;
  *plan = nullptr;
  if ((type != 1 && type != 2) || dim < 1 || dim > 3 || !nmodes ||
      (precision != CG_PREC_FP64 && precision != CG_PREC_FP32)) {
    cg::set_last_error("type must be 1 or 2, dim 1..3, precision CG_PREC_FP64/FP32");
    return CG_ERR_ARG;
  }
  for (int d = 0; d < dim; d++)
    if (nmodes[d] < 1 || nmodes[d] > (1 << 28)) {
      cg::set_last_error("mode counts must be in 1..2^28");
      return CG_ERR_ARG;
    }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    cg::set_last_error("no CUDA device");
    return CG_ERR_NOGPU;
  }
  cg_nufft_s* P = new cg_nufft_s();
  cudaGetDevice(&P->device);
  P->stream = (cudaStream_t)stream;
  P->type = type;
  P->iflag = iflag >= 0 ? 1 : -1;
  P->precision = precision;
  int kw;
  double beta, c;
  const double floor_eps = precision == CG_PREC_FP64 ? 1.1e-16 : 6e-8;
  const int st = cg::setup_conv_opts(epsilon, sigma, floor_eps, kw, beta, c);
  if (st > 1) {
    free_nufft(P);
    cg::set_last_error("sigma must be > 1");
    return st;
  }
  P->eps_status = st;
  P->kw = kw;
  NufftGeom& g = P->g;
  g.dim = dim;
  g.beta = beta;
  g.es_c = c;
  double cells = 1;
  for (int d = 0; d < 3; d++) {
    g.N[d] = d < dim ? nmodes[d] : 1;
    g.nf[d] = d < dim ? cg::get_num_cells((int)g.N[d], sigma, kw) : 1;
    cells *= g.nf[d];
  }
  uint64_t nb = 1;
  for (int d = 0; d < dim; d++) nb *= (uint64_t)((g.nf[d] + 15) >> 4);
  if (cells > 4.0e9 || nb >= (1ULL << 32)) {
    free_nufft(P);
    cg::set_last_error("fine grid too large");
    return CG_ERR_SIZE;
  }
  cg::Quad q;
  cg::make_quad(kw, beta, c, nullptr, q);
  int rc = CG_OK;
  for (int d = 0; d < dim && rc == CG_OK; d++) {
    std::vector<double> k(g.nf[d] / 2 + 1);
    cg::fseries_uv(q, g.nf[d], k.data());
    rc = cg::ensure(P->K[d], k.size() * 8);
    if (rc == CG_OK && cudaMemcpy(P->K[d].p, k.data(), k.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess)
      rc = CG_ERR_CUDA;
  }
  const size_t tsz = precision == CG_PREC_FP64 ? 8 : 4;
  if (rc == CG_OK) rc = cg::ensure(P->fw, (size_t)cells * 2 * tsz);
  if (rc == CG_OK) {
    int n[3];
    for (int d = 0; d < dim; d++) n[d] = g.nf[dim - 1 - d];  // slowest first, nf[0] fastest
    if (cufftPlanMany(&P->fft, dim, n, nullptr, 1, 0, nullptr, 1, 0,
                      precision == CG_PREC_FP64 ? CUFFT_Z2Z : CUFFT_C2C, 1) != CUFFT_SUCCESS)
      rc = CG_ERR_CUFFT;
    else
      P->fft_valid = true;
  }
  if (rc != CG_OK) {
    free_nufft(P);
    return rc;
  }
  *plan = P;
  return st;
}

int cg_nufft_setpts(cg_nufft_s* plan, int64_t M, const double* d_x, const double* d_y,
                    const double* d_z) {
  if (!plan || M < 0 || M > 2147483647LL) return CG_ERR_ARG;
  const int dim = plan->g.dim;
  if (M > 0 && (!d_x || (dim >= 2 && !d_y) || (dim >= 3 && !d_z))) {
    cg::set_last_error("null coordinate pointer");
    return CG_ERR_ARG;
  }
  CG_CUDA(cudaSetDevice(plan->device));
  plan->M = M;
  const int r = plan->precision == CG_PREC_FP64 ? setpts_t<double>(plan, M, d_x, d_y, d_z)
                                                 : setpts_t<float>(plan, M, d_x, d_y, d_z);
  plan->have_pts = r == CG_OK;
  return r;
}

int cg_nufft_execute(cg_nufft_s* plan, void* d_c, void* d_fk) {
  if (!plan || !plan->have_pts || !d_fk || (plan->M > 0 && !d_c)) {
    cg::set_last_error("cg_nufft_setpts first; non-null c and fk");
    return CG_ERR_ARG;
  }
  CG_CUDA(cudaSetDevice(plan->device));
  const int r = plan->precision == CG_PREC_FP64 ? execute_t<double>(plan, d_c, d_fk)
                                                 : execute_t<float>(plan, d_c, d_fk);
  return r != CG_OK ? r : plan->eps_status;
}

int cg_nufft_get_info(const cg_nufft_s* plan, int* kw, int64_t* nf) {
  if (!plan) return CG_ERR_ARG;
  if (kw) *kw = plan->kw;
  if (nf)
    for (int d = 0; d < 3; d++) nf[d] = plan->g.nf[d];
  return CG_OK;
}

int cg_nufft_destroy(cg_nufft_s* plan) {
  free_nufft(plan);
  return CG_OK;
}

}  // extern "C"
