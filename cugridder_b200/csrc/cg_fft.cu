// Column FFTs of the w planes (FP32, power-of-two lengths) done in shared
// memory.  cuFFT's strided 1-D transforms along the slow grid axis run at
// ~1.5 TB/s on B200 for 8192-point columns; here a CTA loads CB adjacent
// columns whole (CB x 8 bytes contiguous per grid row), transforms them with
// radix-16 Stockham passes in shared memory and stores them back in place,
// so every grid element crosses HBM once each way.
//
// Transform: X[k] = sum_j x[j] exp(sign 2 pi i j k / L), unnormalised, the
// convention of cufftExecC2C (sign +1 = CUFFT_INVERSE, -1 = CUFFT_FORWARD).
// Shared layout: row j of the column pair at float4 slot j + j / 16 (one pad
// slot per 16 rows keeps the stride-16 stores of the first pass
// conflict-free).
#include <cmath>
#include <vector>

#include "cg_internal.cuh"

namespace cg {
namespace {

constexpr int kFftThreads = 512;

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ int pad16(int j) { return j + (j >> 4); }

// e^{sign 2 pi i k / 16}, k < 16, as (cos, sin) of multiples of pi/8
__device__ __forceinline__ float2 w16(int k, int sign) {
  constexpr float c1 = 0.92387953251128674f, c2 = 0.70710678118654752f, c3 = 0.38268343236508977f;
  const float cs[16] = {1.f, c1, c2, c3, 0.f, -c3, -c2, -c1, -1.f, -c1, -c2, -c3, 0.f, c3, c2, c1};
  const float sn[16] = {0.f, c3, c2, c1, 1.f, c1, c2, c3, 0.f, -c3, -c2, -c1, -1.f, -c1, -c2, -c3};
  return make_float2(cs[k & 15], sign * sn[k & 15]);
}

// in-register DFT of R = 2, 4, 8 or 16 points (radix-2 DIT, bit-reversed input order)
template <int R>
__device__ __forceinline__ void dft_reg(float2* v, int sign) {
  // bit-reversal permutation
#pragma unroll
  for (int i = 0; i < R; i++) {
    int r = 0;
#pragma unroll
    for (int b = 1, t = i; b < R; b <<= 1, t >>= 1) r = (r << 1) | (t & 1);
    if (r > i) {
      const float2 t2 = v[i];
      v[i] = v[r];
      v[r] = t2;
    }
  }
#pragma unroll
  for (int len = 2; len <= R; len <<= 1) {
#pragma unroll
    for (int i = 0; i < R; i += len) {
#pragma unroll
      for (int k = 0; k < len / 2; k++) {
        const float2 w = w16(k * (16 / len), sign);
        const float2 a = v[i + k], b = cmul(v[i + k + len / 2], w);
        v[i + k] = make_float2(a.x + b.x, a.y + b.y);
        v[i + k + len / 2] = make_float2(a.x - b.x, a.y - b.y);
      }
    }
  }
}

// One Stockham pass of radix R over sub-transforms of size Ns, both columns
// of the pair at once (float4 = column 0, column 1 of one row).  In place:
// every thread reads its butterflies, the block syncs, then writes.  The
// pass's twiddles e^{sign 2 pi i m k / (Ns R)} come from its own table
// tw[m * Ns + k] (consecutive lanes read consecutive entries).
template <int L, int R, bool kLast>
__device__ __forceinline__ void stockham_pass(float4* s, int Ns, int sign,
                                              const float2* __restrict__ tw) {
  constexpr int NB = L / R;  // butterflies per column
  constexpr int BPT = (NB + kFftThreads - 1) / kFftThreads;
  if constexpr (kLast) {
    // last pass: butterfly j reads and writes rows j + m * Ns only, so each
    // one is done in place without holding the others in registers
#pragma unroll 1
    for (int j = threadIdx.x; j < NB; j += kFftThreads) {
      float2 a[R], b[R];
#pragma unroll
      for (int m = 0; m < R; m++) {
        const float4 x = s[pad16(j + m * NB)];
        float2 xa = make_float2(x.x, x.y), xb = make_float2(x.z, x.w);
        if (m > 0) {
          const float2 t = tw[m * Ns + j];
          const float2 w = make_float2(t.x, sign * t.y);
          xa = cmul(xa, w);
          xb = cmul(xb, w);
        }
        a[m] = xa;
        b[m] = xb;
      }
      dft_reg<R>(a, sign);
      dft_reg<R>(b, sign);
#pragma unroll
      for (int m = 0; m < R; m++)
        s[pad16(j + m * Ns)] = make_float4(a[m].x, a[m].y, b[m].x, b[m].y);
    }
    __syncthreads();
    return;
  } else {
  float2 a[BPT][R], b[BPT][R];
#pragma unroll
  for (int q = 0; q < BPT; q++) {
    const int j = threadIdx.x + q * kFftThreads;
    if (j < NB) {
      const int k = j & (Ns - 1);
#pragma unroll
      for (int m = 0; m < R; m++) {
        const float4 x = s[pad16(j + m * NB)];
        float2 xa = make_float2(x.x, x.y), xb = make_float2(x.z, x.w);
        if (m > 0 && Ns > 1) {
          const float2 t = tw[m * Ns + k];
          const float2 w = make_float2(t.x, sign * t.y);
          xa = cmul(xa, w);
          xb = cmul(xb, w);
        }
        a[q][m] = xa;
        b[q][m] = xb;
      }
      dft_reg<R>(a[q], sign);
      dft_reg<R>(b[q], sign);
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < BPT; q++) {
    const int j = threadIdx.x + q * kFftThreads;
    if (j < NB) {
      const int k = j & (Ns - 1);
      const int base = (j - k) * R + k;
#pragma unroll
      for (int m = 0; m < R; m++)
        s[pad16(base + m * Ns)] = make_float4(a[q][m].x, a[q][m].y, b[q][m].x, b[q][m].y);
    }
  }
  __syncthreads();
  }
}

// radix of the last pass after the radix-16 passes (1: none)
__host__ __device__ constexpr int last_radix(int L) {
  int ns = 1;
  while (ns * 16 <= L) ns *= 16;
  return L / ns;
}

template <int L>
__global__ void __launch_bounds__(kFftThreads) k_col_fft(float2* __restrict__ grid, int nf1,
                                                         size_t plane, int nplanes, int c0a,
                                                         int na, int c0b, int nb, int sign,
                                                         const float2* __restrict__ tw) {
  extern __shared__ __align__(16) float4 s4[];
  constexpr int CB = 2;
  const int groups_a = na / CB, groups = groups_a + nb / CB;
  const int64_t items = (int64_t)groups * nplanes;
  for (int64_t it = blockIdx.x; it < items; it += gridDim.x) {
    const int p = (int)(it / groups), gi = (int)(it - (int64_t)p * groups);
    const int col0 = gi < groups_a ? c0a + gi * CB : c0b + (gi - groups_a) * CB;
    float2* base = grid + (size_t)p * plane + col0;
    // one 16-byte asynchronous copy per grid row (the two adjacent columns),
    // all in flight before the block waits
#pragma unroll 4
    for (int j = threadIdx.x; j < L; j += kFftThreads) {
      const unsigned dst = (unsigned)__cvta_generic_to_shared(s4 + pad16(j));
      const float2* src = base + (size_t)j * nf1;
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
    }
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    int Ns = 1, toff = 0;
#pragma unroll 1
    for (; Ns * 16 <= L; Ns *= 16) {
      if (Ns * 16 == L)
        stockham_pass<L, 16, true>(s4, Ns, sign, tw + toff);
      else
        stockham_pass<L, 16, false>(s4, Ns, sign, tw + toff);
      if (Ns > 1) toff += 16 * Ns;
    }
    constexpr int RL = last_radix(L);
    if constexpr (RL > 1) stockham_pass<L, RL, true>(s4, Ns, sign, tw + toff);
#pragma unroll 4
    for (int j = threadIdx.x; j < L; j += kFftThreads)
      *reinterpret_cast<float4*>(base + (size_t)j * nf1) = s4[pad16(j)];
    __syncthreads();
  }
}

template <int L>
int launch_l(float2* grid, int nf1, size_t plane, int nplanes, int c0a, int na, int c0b, int nb,
             int sign, const float2* tw, cudaStream_t st) {
  const size_t smem = (size_t)(pad16(L) + 16) * sizeof(float4);
  int per_sm = 0;
  CG_CUDA(kernel_occupancy((const void*)k_col_fft<L>, kFftThreads, smem, &per_sm));
  if (per_sm < 1) return CG_ERR_ARG;
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) sms = 148;
  }
  const int64_t items = (int64_t)(na / 2 + nb / 2) * nplanes;
  const int blocks = (int)std::min<int64_t>(items, (int64_t)per_sm * sms);
  k_col_fft<L><<<blocks, kFftThreads, smem, st>>>(grid, nf1, plane, nplanes, c0a, na, c0b, nb,
                                                 sign, tw);
  count_launches(1);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

}  // namespace

bool col_fft_supported(int L, int na, int nb) {
  return (L == 1024 || L == 2048 || L == 4096 || L == 8192) && na % 2 == 0 && nb % 2 == 0;
}

// Twiddle tables of the passes with Ns > 1, in pass order: table of pass
// (R, Ns) holds e^{2 pi i m k / (Ns R)} at [m * Ns + k], m < R, k < Ns.
size_t col_fft_twiddle_count(int L) {
  size_t n = 0;
  int ns = 1;
  for (; ns * 16 <= L; ns *= 16)
    if (ns > 1) n += 16 * (size_t)ns;
  if (L / ns > 1) n += (size_t)(L / ns) * ns;
  return n;
}

int make_col_fft_twiddles(int L, float2* d_tw, cudaStream_t st) {
  std::vector<float2> h;
  h.reserve(col_fft_twiddle_count(L));
  auto table = [&](int R, int ns) {
    for (int m = 0; m < R; m++)
      for (int k = 0; k < ns; k++) {
        const double a = 2.0 * kPi * (double)m * (double)k / ((double)ns * R);
        h.push_back(make_float2((float)std::cos(a), (float)std::sin(a)));
      }
  };
  int ns = 1;
  for (; ns * 16 <= L; ns *= 16)
    if (ns > 1) table(16, ns);
  if (L / ns > 1) table(L / ns, ns);
  CG_CUDA(cudaMemcpyAsync(d_tw, h.data(), sizeof(float2) * h.size(), cudaMemcpyHostToDevice, st));
  CG_CUDA(cudaStreamSynchronize(st));
  return CG_OK;
}

// In-place column transforms of columns [c0a, c0a + na) and [c0b, c0b + nb)
// of nplanes planes (row stride nf1, plane stride `plane` elements), length L.
int launch_col_fft(float2* grid, int L, int nf1, size_t plane, int nplanes, int c0a, int na,
                   int c0b, int nb, int sign, const float2* d_tw, cudaStream_t st) {
  switch (L) {
    case 1024: return launch_l<1024>(grid, nf1, plane, nplanes, c0a, na, c0b, nb, sign, d_tw, st);
    case 2048: return launch_l<2048>(grid, nf1, plane, nplanes, c0a, na, c0b, nb, sign, d_tw, st);
    case 4096: return launch_l<4096>(grid, nf1, plane, nplanes, c0a, na, c0b, nb, sign, d_tw, st);
    case 8192: return launch_l<8192>(grid, nf1, plane, nplanes, c0a, na, c0b, nb, sign, d_tw, st);
    default: return CG_ERR_ARG;
  }
}

}  // namespace cg
