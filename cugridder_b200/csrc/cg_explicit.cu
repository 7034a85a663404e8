// On-device FP64 direct DFT ("explicit gridder"): the exact sums that
// ms2dirty / dirty2ms approximate, for error checks at sizes where a CPU DFT
// is too slow.
//
// The reference's explicit_gridder (precomp.cu:246-321) sums
// vis_j exp(2 pi i f/c (l u + m v + (n - 1) w)) / n per pixel without weights
// or sign.  These kernels use the conventions of the library's own
// ms2dirty / dirty2ms (the test_wst.py:15-32 definitions): weights multiply,
// w enters with `sign`, n - 1 is computed as -(l^2 + m^2) / (1 + n) and the
// adjoint carries the conjugate phase and the weight of each row.
//
// Work split: rows (ms2dirty) or pixels (dirty2ms) are cut into chunks along
// grid.y; each block stages one chunk in shared memory and every thread adds
// its chunk's partial sum to its output with FP64 atomics, so the output is
// zeroed first and the result's summation order is not fixed.
#include <algorithm>
#include <cmath>

#include "cg_internal.cuh"

namespace {

constexpr int kThreads = 128;
constexpr int kStage = 256;  // rows / pixels staged per shared-memory round

__device__ __forceinline__ void pixel_lm(int64_t o, int nx, int ny, double pixx, double pixy,
                                         double& l, double& m, double& nm1) {
  const int x = (int)(o / ny), y = (int)(o % ny);
  l = (x - nx / 2) * pixx;
  m = (y - ny / 2) * pixy;
  const double e2 = l * l + m * m;
  nm1 = -e2 / (sqrt(1.0 - e2) + 1.0);
}

// out[q] += sum_{j in chunk} wgt_j vis_j exp(i s (u l + v m + sign w (n-1))) / n
__global__ void __launch_bounds__(kThreads) k_dft_ms2dirty(
    int64_t nrow, int nx, int ny, double pixx, double pixy, double s, int sign,
    const double* __restrict__ uvw, const double2* __restrict__ vis,
    const double* __restrict__ wgt, int64_t npix, const int64_t* __restrict__ pix,
    int64_t chunk, double2* __restrict__ out) {
  __shared__ double su[kStage], sv[kStage], sw[kStage];
  __shared__ double2 sc[kStage];
  const int64_t q = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  const int64_t o = q < npix ? (pix ? pix[q] : q) : -1;
  const bool live = o >= 0 && o < (int64_t)nx * ny;  // bad indices leave their output 0
  double l = 0, m = 0, nm1 = 0;
  if (live) pixel_lm(o, nx, ny, pixx, pixy, l, m, nm1);
  const int64_t j0 = (int64_t)blockIdx.y * chunk, j1 = min(nrow, j0 + chunk);
  double sr = 0, si = 0;
  for (int64_t b = j0; b < j1; b += kStage) {
    const int cnt = (int)((j1 - b) < kStage ? (j1 - b) : kStage);
    __syncthreads();
    for (int t = threadIdx.x; t < cnt; t += kThreads) {
      const int64_t j = b + t;
      su[t] = uvw[3 * j];
      sv[t] = uvw[3 * j + 1];
      sw[t] = (double)sign * uvw[3 * j + 2];
      const double wt = wgt ? wgt[j] : 1.0;
      sc[t] = make_double2(vis[j].x * wt, vis[j].y * wt);
    }
    __syncthreads();
    if (live)
      for (int t = 0; t < cnt; t++) {
        double sn, cs;
        sincos(s * (su[t] * l + sv[t] * m + sw[t] * nm1), &sn, &cs);
        sr += sc[t].x * cs - sc[t].y * sn;
        si += sc[t].x * sn + sc[t].y * cs;
      }
  }
  if (live) {
    const double n = nm1 + 1.0;
    atomicAdd(&out[q].x, sr / n);
    atomicAdd(&out[q].y, si / n);
  }
}

// out[q] += wgt_j sum_{pixels in chunk} dirty / n exp(-i s (u l + v m + sign w (n-1)))
__global__ void __launch_bounds__(kThreads) k_dft_dirty2ms(
    int64_t nrow, int nx, int ny, double pixx, double pixy, double s, int sign,
    const double* __restrict__ uvw, const double2* __restrict__ dirty,
    const double* __restrict__ wgt, int64_t nvis, const int64_t* __restrict__ rows,
    int64_t chunk, double2* __restrict__ out) {
  __shared__ double sl[kStage], sm[kStage], sn1[kStage];
  __shared__ double2 sd[kStage];
  const int64_t q = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  const int64_t jr = q < nvis ? (rows ? rows[q] : q) : -1;
  const bool live = jr >= 0 && jr < nrow;  // bad indices leave their output 0
  const int64_t j = live ? jr : 0;
  double u = 0, v = 0, w = 0;
  if (live) {
    u = uvw[3 * j];
    v = uvw[3 * j + 1];
    w = (double)sign * uvw[3 * j + 2];
  }
  const int64_t npx = (int64_t)nx * ny;
  const int64_t p0 = (int64_t)blockIdx.y * chunk, p1 = min(npx, p0 + chunk);
  double sr = 0, si = 0;
  for (int64_t b = p0; b < p1; b += kStage) {
    const int cnt = (int)((p1 - b) < kStage ? (p1 - b) : kStage);
    __syncthreads();
    for (int t = threadIdx.x; t < cnt; t += kThreads) {
      double l, m, nm1;
      pixel_lm(b + t, nx, ny, pixx, pixy, l, m, nm1);
      sl[t] = l;
      sm[t] = m;
      sn1[t] = nm1;
      const double2 dv = dirty[b + t];
      sd[t] = make_double2(dv.x / (nm1 + 1.0), dv.y / (nm1 + 1.0));
    }
    __syncthreads();
    if (live)
      for (int t = 0; t < cnt; t++) {
        double sn, cs;
        sincos(-s * (u * sl[t] + v * sm[t] + w * sn1[t]), &sn, &cs);
        sr += sd[t].x * cs - sd[t].y * sn;
        si += sd[t].x * sn + sd[t].y * cs;
      }
  }
  if (live) {
    const double wt = wgt ? wgt[j] : 1.0;
    atomicAdd(&out[q].x, sr * wt);
    atomicAdd(&out[q].y, si * wt);
  }
}

int64_t chunk_for(int64_t n, int64_t outputs) {
  // enough chunks to fill the GPU with blocks, at most 65535 along grid.y
  const int64_t xblocks = (outputs + kThreads - 1) / kThreads;
  int64_t want = std::max<int64_t>(1, (148 * 16 + xblocks - 1) / xblocks);
  int64_t chunk = std::max<int64_t>(kStage, (n + want - 1) / want);
  chunk = std::max<int64_t>(chunk, (n + 65534) / 65535);
  return (chunk + kStage - 1) / kStage * kStage;
}

}  // namespace

extern "C" {

int cg_explicit_ms2dirty(int64_t nrow, int nxdirty, int nydirty, double fov, double freq,
                         const double* d_uvw, const cg_c128* d_vis, const double* d_wgt, int sign,
                         int64_t npix, const int64_t* d_pix, cg_c128* d_out, void* stream) {
  if (nrow < 0 || nxdirty <= 0 || nydirty <= 0 || !(fov > 0) || !(freq > 0) || !d_out ||
      (nrow > 0 && (!d_uvw || !d_vis)) || (npix >= 0 && !d_pix && npix > 0)) {
    cg::set_last_error("invalid argument");
    return CG_ERR_ARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t P = npix < 0 ? (int64_t)nxdirty * nydirty : npix;
  if (P == 0) return CG_OK;
  CG_CUDA(cudaMemsetAsync(d_out, 0, sizeof(cg_c128) * P, st));
  if (nrow == 0) return CG_OK;
  const double pixx = fov / 180.0 * cg::kPi / nxdirty, pixy = fov / 180.0 * cg::kPi / nydirty;
  const double s = 2 * cg::kPi * freq / cg::kSpeedOfLight;
  const int64_t chunk = chunk_for(nrow, P);
  dim3 grid((unsigned)((P + kThreads - 1) / kThreads), (unsigned)((nrow + chunk - 1) / chunk));
  if (grid.x > 2147483647u) return CG_ERR_SIZE;
  k_dft_ms2dirty<<<grid, kThreads, 0, st>>>(nrow, nxdirty, nydirty, pixx, pixy, s, sign, d_uvw,
                                            (const double2*)d_vis, d_wgt, P,
                                            npix < 0 ? nullptr : d_pix, chunk, (double2*)d_out);
  cg::count_launches(1);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

int cg_explicit_dirty2ms(int64_t nrow, int nxdirty, int nydirty, double fov, double freq,
                         const double* d_uvw, const cg_c128* d_dirty, const double* d_wgt, int sign,
                         int64_t nvis, const int64_t* d_rows, cg_c128* d_out, void* stream) {
  if (nrow < 0 || nxdirty <= 0 || nydirty <= 0 || !(fov > 0) || !(freq > 0) || !d_dirty ||
      (nrow > 0 && (!d_uvw || !d_out)) || (nvis > 0 && !d_rows)) {
    cg::set_last_error("invalid argument");
    return CG_ERR_ARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t R = nvis < 0 ? nrow : nvis;
  if (R == 0) return CG_OK;
  CG_CUDA(cudaMemsetAsync(d_out, 0, sizeof(cg_c128) * R, st));
  const double pixx = fov / 180.0 * cg::kPi / nxdirty, pixy = fov / 180.0 * cg::kPi / nydirty;
  const double s = 2 * cg::kPi * freq / cg::kSpeedOfLight;
  const int64_t npx = (int64_t)nxdirty * nydirty;
  const int64_t chunk = chunk_for(npx, R);
  dim3 grid((unsigned)((R + kThreads - 1) / kThreads), (unsigned)((npx + chunk - 1) / chunk));
  k_dft_dirty2ms<<<grid, kThreads, 0, st>>>(nrow, nxdirty, nydirty, pixx, pixy, s, sign, d_uvw,
                                            (const double2*)d_dirty, d_wgt, R,
                                            nvis < 0 ? nullptr : d_rows, chunk, (double2*)d_out);
  cg::count_launches(1);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

}  // extern "C"
