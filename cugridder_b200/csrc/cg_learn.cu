// Learned gridding kernel: forward and backward CUDA kernels of the MLP
// phi_theta and the 2-D training problem it is fitted on.
//
// Kernel family (d in grid cells, |d| < W/2, t = 2d/W):
//   phi(d) = exp( beta0 * (sqrt(1 - t^2) - 1) + net(2 t^2 - 1) )
// net: 1 -> 32 -> 32 -> 1 with tanh on both hidden layers.  The ES kernel
// with beta0 = 2.30 W (conv_interp_invoker.cu:49-119) is the prior: with
// net = 0 the family is exactly ES (up to a constant factor), and the MLP
// learns a log-domain correction.  The input 2t^2 - 1 makes phi even.
//
// Parameters theta (float, 1153): W1[32], b1[32], W2[32][32] (row = output
// unit), b2[32], w3[32], b3.
//
// Training problem (one "set"): M points (x_j, y_j) in grid units on an
// nf x nf periodic grid with complex strengths c_j.  Spreading with the
// separable kernel, a 2-D FFT and division by the kernel's Fourier transform
// approximate the type-1 sums F(k1,k2) = sum_j c_j exp(2 pi i (k1 x_j +
// k2 y_j) / nf); the FP64 direct sum on a subset of modes is the target.
//
// The network is 1153 parameters evaluated at ~10^6 points per training
// step: a 32x32 hidden layer is far too small a GEMM for tensor-core tiles to
// pay, so these are SIMT FP32 kernels with the weights in shared memory.
#include <algorithm>
#include <cmath>

#include "cg_internal.cuh"

namespace {

constexpr int kH = 32;
constexpr int kNTheta = kH + kH + kH * kH + kH + kH + 1;  // 1153
constexpr int oW1 = 0, oB1 = kH, oW2 = 2 * kH, oB2 = 2 * kH + kH * kH, oW3 = oB2 + kH,
              oB3 = oW3 + kH;
constexpr int kThreads = 256;     // forward
constexpr int kBwdThreads = 128;  // backward (per-warp staging: 4 x 8.4 KB shared)

// prior(d) = beta0 (sqrt(1 - t^2) - 1), input x = 2 t^2 - 1; false outside the support
__device__ __forceinline__ bool phi_arg(float d, float halfw, float beta0, float& x,
                                        float& prior) {
  const float t = d / halfw;
  const float t2 = t * t;
  if (!(t2 < 1.0f)) return false;
  x = 2.0f * t2 - 1.0f;
  prior = beta0 * (sqrtf(1.0f - t2) - 1.0f);
  return true;
}

__device__ __forceinline__ float mlp_hidden(const float* __restrict__ s, float x, float* h1,
                                            float* h2) {
#pragma unroll
  for (int m = 0; m < kH; m++) h1[m] = tanhf(fmaf(s[oW1 + m], x, s[oB1 + m]));
  float out = s[oB3];
#pragma unroll 4
  for (int k = 0; k < kH; k++) {
    float a = s[oB2 + k];
    const float* row = s + oW2 + k * kH;
#pragma unroll
    for (int m = 0; m < kH; m++) a = fmaf(row[m], h1[m], a);
    h2[k] = tanhf(a);
    out = fmaf(s[oW3 + k], h2[k], out);
  }
  return out;
}

__global__ void __launch_bounds__(kThreads) k_phi_fwd(const float* __restrict__ theta, float beta0,
                                                      float halfw, int64_t n,
                                                      const float* __restrict__ d,
                                                      float* __restrict__ phi) {
  __shared__ float s[kNTheta];
  for (int i = threadIdx.x; i < kNTheta; i += blockDim.x) s[i] = theta[i];
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    float x, prior;
    float v = 0.0f;
    if (phi_arg(d[i], halfw, beta0, x, prior)) {
      float h1[kH], h2[kH];
      v = expf(prior + mlp_hidden(s, x, h1, h2));
    }
    phi[i] = v;
  }
}

// dtheta += sum_i dphi_i * dphi_i/dtheta.  Each warp walks chunks of 32
// points (one per lane).  Per chunk the lanes stage their layer-2 deltas and
// layer-1 activations in shared memory; lane k then accumulates row k of the
// W2 gradient (sum over the chunk of d2[k] h1[m]) and the per-unit sums of
// unit k in registers.  One atomicAdd per parameter per warp at the end.
__global__ void __launch_bounds__(kBwdThreads) k_phi_bwd(const float* __restrict__ theta,
                                                         float beta0, float halfw, int64_t n,
                                                         const float* __restrict__ d,
                                                         const float* __restrict__ dphi,
                                                         float* __restrict__ dtheta) {
  __shared__ float s[kNTheta];
  __shared__ float sa[kBwdThreads / 32][32][kH + 1];
  __shared__ float sb[kBwdThreads / 32][32][kH + 1];
  for (int i = threadIdx.x; i < kNTheta; i += blockDim.x) s[i] = theta[i];
  __syncthreads();
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  float (*A)[kH + 1] = sa[wib];
  float (*B)[kH + 1] = sb[wib];
  float gW2[kH];
#pragma unroll
  for (int m = 0; m < kH; m++) gW2[m] = 0.0f;
  float gW1 = 0, gb1 = 0, gb2 = 0, gw3 = 0, gb3 = 0;
  const int64_t nchunks = (n + 31) / 32;
  const int64_t gw = (int64_t)blockIdx.x * (kBwdThreads / 32) + wib;
  const int64_t nw = (int64_t)gridDim.x * (kBwdThreads / 32);
  for (int64_t ch = gw; ch < nchunks; ch += nw) {
    const int64_t i = ch * 32 + lane;
    float h1[kH], h2[kH];
    float g = 0.0f, x = 0.0f, prior = 0.0f;
    const bool live = (i < n) && phi_arg(d[i], halfw, beta0, x, prior);
    if (live) {
      const float out = mlp_hidden(s, x, h1, h2);
      g = dphi[i] * expf(prior + out);  // dL/d(net output)
    } else {
#pragma unroll
      for (int m = 0; m < kH; m++) { h1[m] = 0.0f; h2[m] = 0.0f; }
    }
    // stage layer-2 deltas (A) and layer-1 activations (B)
#pragma unroll
    for (int k = 0; k < kH; k++) {
      A[lane][k] = g * s[oW3 + k] * (1.0f - h2[k] * h2[k]);
      B[lane][k] = h1[k];
    }
    __syncwarp();
    // layer-1 deltas of this lane's point: (W2^T d2) * (1 - h1^2)
    float d1[kH];
#pragma unroll
    for (int m = 0; m < kH; m++) d1[m] = 0.0f;
#pragma unroll 4
    for (int k = 0; k < kH; k++) {
      const float dk = A[lane][k];
      const float* row = s + oW2 + k * kH;
#pragma unroll
      for (int m = 0; m < kH; m++) d1[m] = fmaf(dk, row[m], d1[m]);
    }
    // row `lane` of the W2 gradient and the b2 sum of unit `lane`
#pragma unroll 4
    for (int p = 0; p < 32; p++) {
      const float dk = A[p][lane];
      gb2 += dk;
#pragma unroll
      for (int m = 0; m < kH; m++) gW2[m] = fmaf(dk, B[p][m], gW2[m]);
    }
    __syncwarp();
    // stage layer-1 deltas (A) and g * h2 (B) for the per-unit sums
#pragma unroll
    for (int m = 0; m < kH; m++) {
      A[lane][m] = d1[m] * (1.0f - h1[m] * h1[m]);
      B[lane][m] = g * h2[m];
    }
    __syncwarp();
#pragma unroll 4
    for (int p = 0; p < 32; p++) {
      const float xp = __shfl_sync(0xffffffffu, x, p);
      const float a = A[p][lane];
      gb1 += a;
      gW1 = fmaf(a, xp, gW1);
      gw3 += B[p][lane];
    }
    float gs = g;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) gs += __shfl_xor_sync(0xffffffffu, gs, o);
    gb3 += gs;
    __syncwarp();
  }
#pragma unroll
  for (int m = 0; m < kH; m++) atomicAdd(&dtheta[oW2 + lane * kH + m], gW2[m]);
  atomicAdd(&dtheta[oW1 + lane], gW1);
  atomicAdd(&dtheta[oB1 + lane], gb1);
  atomicAdd(&dtheta[oB2 + lane], gb2);
  atomicAdd(&dtheta[oW3 + lane], gw3);
  if (lane == 0) atomicAdd(&dtheta[oB3], gb3);
}

// ---------------------------------------------------------------- training problem
__device__ __forceinline__ int wrapn(int i, int n) {
  i %= n;
  return i < 0 ? i + n : i;
}

// grid[s][ix][iy] (complex, iy fastest) += c_j phx[j][l] phy[j][m] at
// ix = gx0_j + l, iy = gy0_j + m (periodic); one thread per (point, l).
__global__ void k_train_spread(int nsets, int M, int W, int nf, const float2* __restrict__ c,
                               const int* __restrict__ gx0, const int* __restrict__ gy0,
                               const float* __restrict__ phx, const float* __restrict__ phy,
                               float2* __restrict__ grid) {
  const int64_t total = (int64_t)nsets * M * W;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t pj = t / W;  // set * M + j
    const int l = (int)(t - pj * W);
    const int s = (int)(pj / M);
    const float2 cj = c[pj];
    const float a = phx[pj * W + l];
    const int ix = wrapn(gx0[pj] + l, nf);
    float* row = reinterpret_cast<float*>(grid + ((int64_t)s * nf + ix) * nf);
    for (int m = 0; m < W; m++) {
      const float w = a * phy[pj * W + m];
      const int iy = wrapn(gy0[pj] + m, nf);
      atomicAdd(row + 2 * iy, cj.x * w);
      atomicAdd(row + 2 * iy + 1, cj.y * w);
    }
  }
}

// adjoint of k_train_spread with respect to the kernel values:
// dphx[j][l] = sum_m <G, c_j> phy[j][m], dphy[j][m] = sum_l <G, c_j> phx[j][l]
// with <G, c> = G.re c.re + G.im c.im the real gradient pairing.
__global__ void k_train_spread_adj(int nsets, int M, int W, int nf, const float2* __restrict__ c,
                                   const int* __restrict__ gx0, const int* __restrict__ gy0,
                                   const float* __restrict__ phx, const float* __restrict__ phy,
                                   const float2* __restrict__ ggrid, float* __restrict__ dphx,
                                   float* __restrict__ dphy) {
  const int64_t total = (int64_t)nsets * M;
  for (int64_t pj = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; pj < total;
       pj += (int64_t)gridDim.x * blockDim.x) {
    const int s = (int)(pj / M);
    const float2 cj = c[pj];
    float px[16], py[16], ay[16];
    for (int m = 0; m < W; m++) {
      py[m] = phy[pj * W + m];
      ay[m] = 0.0f;
    }
    for (int l = 0; l < W; l++) px[l] = phx[pj * W + l];
    for (int l = 0; l < W; l++) {
      const int ix = wrapn(gx0[pj] + l, nf);
      const float2* row = ggrid + ((int64_t)s * nf + ix) * nf;
      float ax = 0.0f;
      for (int m = 0; m < W; m++) {
        const float2 g = row[wrapn(gy0[pj] + m, nf)];
        const float v = g.x * cj.x + g.y * cj.y;
        ax = fmaf(v, py[m], ax);
        ay[m] = fmaf(v, px[l], ay[m]);
      }
      dphx[pj * W + l] = ax;
    }
    for (int m = 0; m < W; m++) dphy[pj * W + m] = ay[m];
  }
}

// FP64 direct sums F[s][i] = sum_j c_j exp(2 pi i (k1_i X_j + k2_i Y_j) / nf)
// for nk modes per set (k1, k2 given per set); one thread per (set, mode).
__global__ void k_train_dft(int nsets, int M, int nf, const double* __restrict__ X,
                            const double* __restrict__ Y, const double2* __restrict__ c, int nk,
                            const int* __restrict__ k1, const int* __restrict__ k2,
                            double2* __restrict__ F) {
  const int64_t total = (int64_t)nsets * nk;
  const double scale = 2.0 * 3.14159265358979323846 / (double)nf;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int s = (int)(t / nk);
    const double a = (double)k1[t], b = (double)k2[t];
    const double* xs = X + (int64_t)s * M;
    const double* ys = Y + (int64_t)s * M;
    const double2* cs = c + (int64_t)s * M;
    double re = 0.0, im = 0.0;
    for (int j = 0; j < M; j++) {
      double sn, cn;
      sincos(scale * (a * xs[j] + b * ys[j]), &sn, &cn);
      const double2 cj = cs[j];
      re += cj.x * cn - cj.y * sn;
      im += cj.x * sn + cj.y * cn;
    }
    F[t] = make_double2(re, im);
  }
}

int grid_blocks(int64_t n, int threads) {
  int64_t b = (n + threads - 1) / threads;
  if (b > 148 * 16) b = 148 * 16;
  return b < 1 ? 1 : (int)b;
}

}  // namespace

extern "C" {

int cg_learn_theta_size(void) { return kNTheta; }

int cg_learn_phi_forward(const float* theta, float beta0, int W, int64_t n, const float* d,
                         float* phi, void* stream) {
  if (W < 2 || W > 16 || n < 0 || (n > 0 && (!theta || !d || !phi))) return CG_ERR_ARG;
  if (n == 0) return CG_OK;
  k_phi_fwd<<<grid_blocks(n, kThreads), kThreads, 0, (cudaStream_t)stream>>>(
      theta, beta0, 0.5f * (float)W, n, d, phi);
  cg::count_launches(1);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

int cg_learn_phi_backward(const float* theta, float beta0, int W, int64_t n, const float* d,
                          const float* dphi, float* dtheta, void* stream) {
  if (W < 2 || W > 16 || n < 0 || (n > 0 && (!theta || !d || !dphi || !dtheta))) return CG_ERR_ARG;
  if (n == 0) return CG_OK;
  const int64_t warps = (n + 31) / 32;
  const int blocks = (int)std::min<int64_t>((warps + 3) / 4, 148 * 8);
  k_phi_bwd<<<blocks, kBwdThreads, 0, (cudaStream_t)stream>>>(theta, beta0, 0.5f * (float)W, n, d,
                                                              dphi, dtheta);
  cg::count_launches(1);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

int cg_learn_spread2d(int nsets, int M, int W, int nf, const float* c, const int* gx0,
                      const int* gy0, const float* phx, const float* phy, float* grid,
                      void* stream) {
  if (nsets < 0 || M < 0 || W < 1 || W > 16 || nf < W) return CG_ERR_ARG;
  const int64_t n = (int64_t)nsets * M * W;
  if (n == 0) return CG_OK;
  k_train_spread<<<grid_blocks(n, 256), 256, 0, (cudaStream_t)stream>>>(
      nsets, M, W, nf, (const float2*)c, gx0, gy0, phx, phy, (float2*)grid);
  cg::count_launches(1);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

int cg_learn_spread2d_adjoint(int nsets, int M, int W, int nf, const float* c, const int* gx0,
                              const int* gy0, const float* phx, const float* phy,
                              const float* ggrid, float* dphx, float* dphy, void* stream) {
  if (nsets < 0 || M < 0 || W < 1 || W > 16 || nf < W) return CG_ERR_ARG;
  const int64_t n = (int64_t)nsets * M;
  if (n == 0) return CG_OK;
  k_train_spread_adj<<<grid_blocks(n, 128), 128, 0, (cudaStream_t)stream>>>(
      nsets, M, W, nf, (const float2*)c, gx0, gy0, phx, phy, (const float2*)ggrid, dphx, dphy);
  cg::count_launches(1);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

int cg_learn_dft2(int nsets, int M, int nf, const double* X, const double* Y, const double* c,
                  int nk, const int* k1, const int* k2, double* F, void* stream) {
  if (nsets < 0 || M < 0 || nk < 0 || nf <= 0) return CG_ERR_ARG;
  const int64_t n = (int64_t)nsets * nk;
  if (n == 0) return CG_OK;
  k_train_dft<<<grid_blocks(n, 128), 128, 0, (cudaStream_t)stream>>>(
      nsets, M, nf, X, Y, (const double2*)c, nk, k1, k2, (double2*)F);
  cg::count_launches(1);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

}  // extern "C"
