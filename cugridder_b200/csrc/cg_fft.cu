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
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
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

// Shared-memory element of one grid row of the CB columns a CTA transforms:
// float2 (one column) or float4 (two adjacent columns).
template <int CB>
struct ColVec;
template <>
struct ColVec<1> {
  using type = float2;
  static __device__ __forceinline__ float2 col(const float2& v, int) { return v; }
  static __device__ __forceinline__ float2 make(const float2* a, const float2*, int m) { return a[m]; }
};
template <>
struct ColVec<2> {
  using type = float4;
  static __device__ __forceinline__ float2 col(const float4& v, int c) {
    return c == 0 ? make_float2(v.x, v.y) : make_float2(v.z, v.w);
  }
  static __device__ __forceinline__ float4 make(const float2* a, const float2* b, int m) {
    return make_float4(a[m].x, a[m].y, b[m].x, b[m].y);
  }
};

// One Stockham pass of radix R over sub-transforms of size Ns, on every
// column of the CTA at once.  In place: every thread reads its butterflies,
// the block syncs, then writes.  The pass's twiddles
// e^{sign 2 pi i m k / (Ns R)} come from its own table tw[m * Ns + k]
// (consecutive lanes read consecutive entries).
template <int L, int R, int CB, bool kLast>
__device__ __forceinline__ void stockham_pass(typename ColVec<CB>::type* s, int Ns, int sign,
                                              const float2* __restrict__ tw) {
  using CV = ColVec<CB>;
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
        const auto x = s[pad16(j + m * NB)];
        float2 xa = CV::col(x, 0), xb = CB == 2 ? CV::col(x, 1) : xa;
        if (m > 0) {
          const float2 t = tw[m * Ns + j];
          const float2 w = make_float2(t.x, sign * t.y);
          xa = cmul(xa, w);
          if (CB == 2) xb = cmul(xb, w);
        }
        a[m] = xa;
        b[m] = xb;
      }
      dft_reg<R>(a, sign);
      if (CB == 2) dft_reg<R>(b, sign);
#pragma unroll
      for (int m = 0; m < R; m++) s[pad16(j + m * Ns)] = CV::make(a, b, m);
    }
    __syncthreads();
    return;
  } else {
  float2 a[BPT][R], b[CB == 2 ? BPT : 1][R];
#pragma unroll
  for (int q = 0; q < BPT; q++) {
    const int j = threadIdx.x + q * kFftThreads;
    if (j < NB) {
      const int k = j & (Ns - 1);
#pragma unroll
      for (int m = 0; m < R; m++) {
        const auto x = s[pad16(j + m * NB)];
        float2 xa = CV::col(x, 0);
        float2 xb = CB == 2 ? CV::col(x, 1) : xa;
        if (m > 0 && Ns > 1) {
          const float2 t = tw[m * Ns + k];
          const float2 w = make_float2(t.x, sign * t.y);
          xa = cmul(xa, w);
          if (CB == 2) xb = cmul(xb, w);
        }
        a[q][m] = xa;
        if constexpr (CB == 2) b[q][m] = xb;
      }
      dft_reg<R>(a[q], sign);
      if constexpr (CB == 2) dft_reg<R>(b[q], sign);
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
        s[pad16(base + m * Ns)] = CV::make(a[q], b[CB == 2 ? q : 0], m);
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

template <int L, int CB>
__global__ void __launch_bounds__(kFftThreads, CB == 1 ? 2 : 1) k_col_fft(float2* __restrict__ grid, int nf1,
                                                         size_t plane, int nplanes, int c0a,
                                                         int na, int c0b, int nb, int sign,
                                                         const float2* __restrict__ tw) {
  using V = typename ColVec<CB>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V* sv = reinterpret_cast<V*>(smem_raw);
  const int groups_a = na / CB, groups = groups_a + nb / CB;
  const int64_t items = (int64_t)groups * nplanes;
  for (int64_t it = blockIdx.x; it < items; it += gridDim.x) {
    const int p = (int)(it / groups), gi = (int)(it - (int64_t)p * groups);
    const int col0 = gi < groups_a ? c0a + gi * CB : c0b + (gi - groups_a) * CB;
    float2* base = grid + (size_t)p * plane + col0;
    // one asynchronous copy per grid row (the CB adjacent columns), all in
    // flight before the block waits
#pragma unroll 4
    for (int j = threadIdx.x; j < L; j += kFftThreads) {
      const unsigned dst = (unsigned)__cvta_generic_to_shared(sv + pad16(j));
      const float2* src = base + (size_t)j * nf1;
      if constexpr (CB == 2)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
      else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(src) : "memory");
    }
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    int Ns = 1, toff = 0;
#pragma unroll 1
    for (; Ns * 16 <= L; Ns *= 16) {
      if (Ns * 16 == L)
        stockham_pass<L, 16, CB, true>(sv, Ns, sign, tw + toff);
      else
        stockham_pass<L, 16, CB, false>(sv, Ns, sign, tw + toff);
      if (Ns > 1) toff += 16 * Ns;
    }
    constexpr int RL = last_radix(L);
    if constexpr (RL > 1) stockham_pass<L, RL, CB, true>(sv, Ns, sign, tw + toff);
#pragma unroll 4
    for (int j = threadIdx.x; j < L; j += kFftThreads)
      *reinterpret_cast<V*>(base + (size_t)j * nf1) = sv[pad16(j)];
    __syncthreads();
  }
}

// All passes of a length-L transform of two vectors held in registers:
// thread t holds elements t + m T (m < 16, T = L / 16) of each in a[], b[]
// and gets the outputs back at the same positions.  Radix-16 Stockham passes
// exchange through xch (one vector at a time, padded), then a last radix-RL
// pass runs in registers.
template <int L>
__device__ __forceinline__ void fft_regs(float2 (&a)[16], float2 (&b)[16], int sign,
                                         const float2* __restrict__ tw, float2* xch) {
  constexpr int T = L / 16;
  constexpr int RL = last_radix(L);  // 1: L is a power of 16
  const int t = threadIdx.x;
  auto exchange = [&](float2 (&v)[16], int o0, int Ns) {
#pragma unroll
    for (int m = 0; m < 16; m++) xch[pad16(o0 + m * Ns)] = v[m];
    __syncthreads();
#pragma unroll
    for (int m = 0; m < 16; m++) v[m] = xch[pad16(t + m * T)];
    __syncthreads();
  };
  int Ns = 1, toff = 0;
#pragma unroll 1
  for (; Ns * 16 <= L; Ns *= 16) {
    const int k = t & (Ns - 1);
    if (Ns > 1) {
#pragma unroll
      for (int m = 1; m < 16; m++) {
        const float2 tv = tw[toff + m * Ns + k];
        const float2 w = make_float2(tv.x, sign * tv.y);
        a[m] = cmul(a[m], w);
        b[m] = cmul(b[m], w);
      }
    }
    dft_reg<16>(a, sign);
    dft_reg<16>(b, sign);
    if (Ns * 16 == L) return;  // last pass (L a power of 16): outputs at t + m T
    const int o0 = (t - k) * 16 + k;
    exchange(a, o0, Ns);
    exchange(b, o0, Ns);
    if (Ns > 1) toff += 16 * Ns;
  }
  if constexpr (RL > 1) {
    // last pass, radix RL, Ns = L / RL: butterfly j = t + q T reads and
    // writes positions j + m L / RL, i.e. slots q + m (16 / RL) of this thread
    constexpr int Q = 16 / RL;
#pragma unroll
    for (int q = 0; q < Q; q++) {
      const int j = t + q * T;
      float2 va[RL], vb[RL];
#pragma unroll
      for (int m = 0; m < RL; m++) {
        va[m] = a[q + m * Q];
        vb[m] = b[q + m * Q];
        if (m > 0) {
          const float2 tv = tw[toff + m * (L / RL) + j];
          const float2 w = make_float2(tv.x, sign * tv.y);
          va[m] = cmul(va[m], w);
          vb[m] = cmul(vb[m], w);
        }
      }
      dft_reg<RL>(va, sign);
      dft_reg<RL>(vb, sign);
#pragma unroll
      for (int m = 0; m < RL; m++) {
        a[q + m * Q] = va[m];
        b[q + m * Q] = vb[m];
      }
    }
  }
}

// Register-resident variant: T = L / 16 threads, each holding 16 points of
// both columns of the pair in registers for every pass.  Thread t always
// holds positions t + m T (m < 16): they are the inputs of every radix-16
// pass and of the last radix-RL pass, and the last pass writes its outputs
// back to the same positions, so the item is loaded from and stored to those
// rows directly.  Between passes the Stockham exchange goes through a
// one-column shared buffer (column 0, then column 1).  A second shared
// buffer receives the next item by cp.async while the current one is
// transformed, so loads, passes and stores of consecutive items overlap in
// one CTA.
//
// Rows [mid0, mid1) of every column are outside the image (the CMCL map
// reaches rows [0, mid0) and [mid1, L) only), and rows outside [b0, b1) are
// outside the band of rows the row transforms cover.  skip is a set of flags:
//   1: rows outside the image are zero on input (the plane fill wrote zeros
//      there): not loaded;
//   2: nothing reads rows outside the image afterwards (the w-DFT): not stored;
//   4: rows outside the band are zero on input (the grid holds no data there
//      and the row transforms did not touch them): not loaded;
//   8: nothing reads rows outside the band afterwards (the row transforms and
//      the degridding stay inside it): not stored.
template <int L>
__global__ void __launch_bounds__(L / 16) k_col_fft_reg(float2* __restrict__ grid, int nf1,
                                                        size_t plane, int nplanes, int c0a,
                                                        int na, int c0b, int nb, int sign,
                                                        const float2* __restrict__ tw, int mid0,
                                                        int mid1, int skip, int b0, int b1) {
  constexpr int T = L / 16;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float4* pre = reinterpret_cast<float4*>(smem_raw);                       // L rows x 2 columns
  float2* xch = reinterpret_cast<float2*>(smem_raw + (size_t)L * sizeof(float4));  // padded column
  const int t = threadIdx.x;
  const int groups_a = na / 2, groups = groups_a + nb / 2;
  const int64_t items = (int64_t)groups * nplanes;
  auto base_of = [&](int64_t it) {
    const int p = (int)(it / groups), gi = (int)(it - (int64_t)p * groups);
    const int col0 = gi < groups_a ? c0a + gi * 2 : c0b + (gi - groups_a) * 2;
    return grid + (size_t)p * plane + col0;
  };
  auto outside = [&](int row) { return row >= mid0 && row < mid1; };
  auto no_load = [&](int row) {
    return ((skip & 1) && outside(row)) || ((skip & 4) && (row < b0 || row >= b1));
  };
  auto no_store = [&](int row) {
    return ((skip & 2) && outside(row)) || ((skip & 8) && (row < b0 || row >= b1));
  };
  auto prefetch = [&](int64_t it) {
    const float2* b = base_of(it);
#pragma unroll
    for (int m = 0; m < 16; m++) {
      const int row = t + m * T;
      if (no_load(row)) continue;  // zero rows: not loaded
      const unsigned dst = (unsigned)__cvta_generic_to_shared(pre + row);
      const float2* src = b + (size_t)row * nf1;
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  int64_t it = blockIdx.x;
  if (it < items) prefetch(it);
  for (; it < items; it += gridDim.x) {
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    float2 a[16], b[16];
#pragma unroll
    for (int m = 0; m < 16; m++) {
      const int row = t + m * T;
      const float4 v = no_load(row) ? make_float4(0.f, 0.f, 0.f, 0.f) : pre[row];
      a[m] = make_float2(v.x, v.y);
      b[m] = make_float2(v.z, v.w);
    }
    __syncthreads();  // the prefetch buffer is free again
    if (it + gridDim.x < items) prefetch(it + gridDim.x);
    fft_regs<L>(a, b, sign, tw, xch);
    float2* bs = base_of(it);
#pragma unroll
    for (int m = 0; m < 16; m++) {
      const int row = t + m * T;
      if (no_store(row)) continue;  // rows nothing reads
      *reinterpret_cast<float4*>(bs + (size_t)row * nf1) =
          make_float4(a[m].x, a[m].y, b[m].x, b[m].y);
    }
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// Variant of k_col_fft_reg with one shared buffer of column pairs (float4):
// each exchange moves both columns with 128-bit accesses (half the shared
// memory instructions), and the buffer takes the next item's rows (cp.async)
// once the last exchange of the current item has been read, overlapping that
// load with the last pass and the stores.
template <int L>
__global__ void __launch_bounds__(L / 16) k_col_fft_reg2(float2* __restrict__ grid, int nf1,
                                                         size_t plane, int nplanes, int c0a,
                                                         int na, int c0b, int nb, int sign,
                                                         const float2* __restrict__ tw) {
  constexpr int T = L / 16;
  constexpr int RL = last_radix(L);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float4* sv = reinterpret_cast<float4*>(smem_raw);  // pad16(L) + 16 slots
  const int t = threadIdx.x;
  const int groups_a = na / 2, groups = groups_a + nb / 2;
  const int64_t items = (int64_t)groups * nplanes;
  auto base_of = [&](int64_t it) {
    const int p = (int)(it / groups), gi = (int)(it - (int64_t)p * groups);
    const int col0 = gi < groups_a ? c0a + gi * 2 : c0b + (gi - groups_a) * 2;
    return grid + (size_t)p * plane + col0;
  };
  auto prefetch = [&](int64_t it) {
    const float2* b = base_of(it);
#pragma unroll
    for (int m = 0; m < 16; m++) {
      const int row = t + m * T;
      const unsigned dst = (unsigned)__cvta_generic_to_shared(sv + pad16(row));
      const float2* src = b + (size_t)row * nf1;
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  int64_t it = blockIdx.x;
  if (it < items) prefetch(it);
  for (; it < items; it += gridDim.x) {
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    float2 a[16], b[16];
#pragma unroll
    for (int m = 0; m < 16; m++) {
      const float4 v = sv[pad16(t + m * T)];
      a[m] = make_float2(v.x, v.y);
      b[m] = make_float2(v.z, v.w);
    }
    __syncthreads();
    const bool more = it + gridDim.x < items;
    bool fetched = false;
    int Ns = 1, toff = 0;
#pragma unroll 1
    for (; Ns * 16 <= L; Ns *= 16) {
      const int k = t & (Ns - 1);
      if (Ns > 1) {
#pragma unroll
        for (int m = 1; m < 16; m++) {
          const float2 tv = tw[toff + m * Ns + k];
          const float2 w = make_float2(tv.x, sign * tv.y);
          a[m] = cmul(a[m], w);
          b[m] = cmul(b[m], w);
        }
      }
      dft_reg<16>(a, sign);
      dft_reg<16>(b, sign);
      if (Ns * 16 == L) break;  // last pass: outputs at t + m T
      const int o0 = (t - k) * 16 + k;
#pragma unroll
      for (int m = 0; m < 16; m++)
        sv[pad16(o0 + m * Ns)] = make_float4(a[m].x, a[m].y, b[m].x, b[m].y);
      __syncthreads();
#pragma unroll
      for (int m = 0; m < 16; m++) {
        const float4 v = sv[pad16(t + m * T)];
        a[m] = make_float2(v.x, v.y);
        b[m] = make_float2(v.z, v.w);
      }
      __syncthreads();
      if (Ns > 1) toff += 16 * Ns;
      // after the last exchange the buffer is free: start the next item's rows
      const bool last_exchange = RL > 1 ? (Ns * 16 * 16 > L) : (Ns * 16 * 16 == L);
      if (last_exchange && more) {
        prefetch(it + gridDim.x);
        fetched = true;
      }
    }
    if constexpr (RL > 1) {
      constexpr int Q = 16 / RL;
#pragma unroll
      for (int q = 0; q < Q; q++) {
        const int j = t + q * T;
        float2 va[RL], vb[RL];
#pragma unroll
        for (int m = 0; m < RL; m++) {
          va[m] = a[q + m * Q];
          vb[m] = b[q + m * Q];
          if (m > 0) {
            const float2 tv = tw[toff + m * (L / RL) + j];
            const float2 w = make_float2(tv.x, sign * tv.y);
            va[m] = cmul(va[m], w);
            vb[m] = cmul(vb[m], w);
          }
        }
        dft_reg<RL>(va, sign);
        dft_reg<RL>(vb, sign);
#pragma unroll
        for (int m = 0; m < RL; m++) {
          a[q + m * Q] = va[m];
          b[q + m * Q] = vb[m];
        }
      }
    }
    float2* bs = base_of(it);
#pragma unroll
    for (int m = 0; m < 16; m++)
      *reinterpret_cast<float4*>(bs + (size_t)(t + m * T) * nf1) =
          make_float4(a[m].x, a[m].y, b[m].x, b[m].y);
    if (more && !fetched) {  // one pass only (no exchange): fetch after the stores
      __syncthreads();
      prefetch(it + gridDim.x);
    }
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

template <int L>
int launch_reg2(float2* grid, int nf1, size_t plane, int nplanes, int c0a, int na, int c0b,
                int nb, int sign, const float2* tw, cudaStream_t st) {
  const size_t smem = (size_t)(pad16(L) + 16) * sizeof(float4);
  int per_sm = 0;
  CG_CUDA(kernel_occupancy((const void*)k_col_fft_reg2<L>, L / 16, smem, &per_sm));
  if (per_sm < 1) return CG_ERR_ARG;
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) sms = 148;
  }
  const int64_t items = (int64_t)(na / 2 + nb / 2) * nplanes;
  const int blocks = (int)std::min<int64_t>(items, (int64_t)per_sm * sms);
  k_col_fft_reg2<L><<<blocks, L / 16, smem, st>>>(grid, nf1, plane, nplanes, c0a, na, c0b, nb,
                                                  sign, tw);
  count_launches(1);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

// Cluster variant: four CTAs (a thread-block cluster) transform 8 adjacent
// columns together.  Each CTA loads a quarter of the rows of all 8 columns
// (64 contiguous bytes per grid row instead of 16) into its shared buffer;
// after a cluster barrier every CTA gathers its own column pair, all rows,
// from the four buffers through distributed shared memory, straight into
// the register layout of k_col_fft_reg (thread t holds rows t + m T).  A
// second cluster barrier frees the buffers, so the next item's loads overlap
// this item's passes and stores.  Buffer layout: local row r, 16-byte chunk c
// (column pair c) at slot c ^ ((r >> 1) & 3) of the row's 64 bytes, which
// keeps both the loads and the gathers free of bank conflicts.
constexpr int kColCluster = 4;

template <int L>
__global__ void __cluster_dims__(kColCluster, 1, 1) __launch_bounds__(L / 16)
    k_col_fft_cluster(float2* __restrict__ grid, int nf1, size_t plane, int nplanes, int c0a,
                      int na, int c0b, int nb, int sign, const float2* __restrict__ tw) {
  namespace cgx = cooperative_groups;
  constexpr int T = L / 16;
  constexpr int RL = last_radix(L);
  constexpr int RB = L / kColCluster;  // rows per CTA in the load buffer
  cgx::cluster_group cluster = cgx::this_cluster();
  const int rank = (int)cluster.block_rank();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float4* buf = reinterpret_cast<float4*>(smem_raw);                          // RB rows x 4 chunks
  float2* xch = reinterpret_cast<float2*>(smem_raw + (size_t)RB * 4 * sizeof(float4));  // padded column
  const int t = threadIdx.x;
  const int groups_a = na / 8, groups = groups_a + nb / 8;
  const int64_t items = (int64_t)groups * nplanes;
  const int64_t nclusters = gridDim.x / kColCluster;
  const int64_t cid = blockIdx.x / kColCluster;
  auto base_of = [&](int64_t it) {  // column 0 of the item's 8 columns
    const int p = (int)(it / groups), gi = (int)(it - (int64_t)p * groups);
    const int col0 = gi < groups_a ? c0a + gi * 8 : c0b + (gi - groups_a) * 8;
    return grid + (size_t)p * plane + col0;
  };
  // this CTA's quarter of the rows, 4 chunks of 16 bytes per row
  auto load = [&](int64_t it) {
    const float2* b = base_of(it) + (size_t)rank * RB * nf1;
#pragma unroll
    for (int k = 0; k < (RB * 4) / T; k++) {
      const int idx = t + k * T;
      const int r = idx >> 2, c = idx & 3;
      const unsigned dst =
          (unsigned)__cvta_generic_to_shared(buf + r * 4 + (c ^ ((r >> 1) & 3)));
      const float2* src = b + (size_t)r * nf1 + 2 * c;
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  auto exchange = [&](float2 (&v)[16], int o0, int Ns) {
#pragma unroll
    for (int m = 0; m < 16; m++) xch[pad16(o0 + m * Ns)] = v[m];
    __syncthreads();
#pragma unroll
    for (int m = 0; m < 16; m++) v[m] = xch[pad16(t + m * T)];
    __syncthreads();
  };
  int64_t it = cid;
  if (it < items) load(it);
  for (; it < items; it += nclusters) {
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    cluster.sync();  // every CTA's quarter is in place
    float2 a[16], b[16];
#pragma unroll
    for (int m = 0; m < 16; m++) {
      const int row = t + m * T;
      const int q = row / RB, r = row - q * RB;
      const float4* src = cluster.map_shared_rank(buf, q) + r * 4 + (rank ^ ((r >> 1) & 3));
      const float4 v = *src;
      a[m] = make_float2(v.x, v.y);
      b[m] = make_float2(v.z, v.w);
    }
    cluster.sync();  // every gather is done: the buffers take the next item
    if (it + nclusters < items) load(it + nclusters);
    int Ns = 1, toff = 0;
#pragma unroll 1
    for (; Ns * 16 <= L; Ns *= 16) {
      const int k = t & (Ns - 1);
      if (Ns > 1) {
#pragma unroll
        for (int m = 1; m < 16; m++) {
          const float2 tv = tw[toff + m * Ns + k];
          const float2 w = make_float2(tv.x, sign * tv.y);
          a[m] = cmul(a[m], w);
          b[m] = cmul(b[m], w);
        }
      }
      dft_reg<16>(a, sign);
      dft_reg<16>(b, sign);
      if (Ns * 16 == L) break;
      const int o0 = (t - k) * 16 + k;
      exchange(a, o0, Ns);
      exchange(b, o0, Ns);
      if (Ns > 1) toff += 16 * Ns;
    }
    if constexpr (RL > 1) {
      constexpr int Q = 16 / RL;
#pragma unroll
      for (int q = 0; q < Q; q++) {
        const int j = t + q * T;
        float2 va[RL], vb[RL];
#pragma unroll
        for (int m = 0; m < RL; m++) {
          va[m] = a[q + m * Q];
          vb[m] = b[q + m * Q];
          if (m > 0) {
            const float2 tv = tw[toff + m * (L / RL) + j];
            const float2 w = make_float2(tv.x, sign * tv.y);
            va[m] = cmul(va[m], w);
            vb[m] = cmul(vb[m], w);
          }
        }
        dft_reg<RL>(va, sign);
        dft_reg<RL>(vb, sign);
#pragma unroll
        for (int m = 0; m < RL; m++) {
          a[q + m * Q] = va[m];
          b[q + m * Q] = vb[m];
        }
      }
    }
    float2* bs = base_of(it) + 2 * rank;
#pragma unroll
    for (int m = 0; m < 16; m++)
      *reinterpret_cast<float4*>(bs + (size_t)(t + m * T) * nf1) =
          make_float4(a[m].x, a[m].y, b[m].x, b[m].y);
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  cluster.sync();  // no CTA leaves while another may still read its buffer
}

template <int L>
int launch_cluster(float2* grid, int nf1, size_t plane, int nplanes, int c0a, int na, int c0b,
                   int nb, int sign, const float2* tw, cudaStream_t st) {
  constexpr int RB = L / kColCluster;
  const size_t smem = (size_t)RB * 4 * sizeof(float4) + (size_t)(pad16(L) + 16) * sizeof(float2);
  int per_sm = 0;
  CG_CUDA(kernel_occupancy((const void*)k_col_fft_cluster<L>, L / 16, smem, &per_sm));
  if (per_sm < 1) return CG_ERR_ARG;
  static int max_clusters[4] = {0, 0, 0, 0};
  const int slot = L == 1024 ? 0 : L == 2048 ? 1 : L == 4096 ? 2 : 3;
  if (!max_clusters[slot]) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kColCluster * 148, 1, 1);
    cfg.blockDim = dim3(L / 16, 1, 1);
    cfg.dynamicSmemBytes = smem;
    int n = 0;
    CG_CUDA(cudaOccupancyMaxActiveClusters(&n, (const void*)k_col_fft_cluster<L>, &cfg));
    if (n < 1) return CG_ERR_ARG;
    max_clusters[slot] = n;
  }
  const int64_t items = (int64_t)(na / 8 + nb / 8) * nplanes;
  const int clusters = (int)std::min<int64_t>(items, max_clusters[slot]);
  k_col_fft_cluster<L><<<clusters * kColCluster, L / 16, smem, st>>>(grid, nf1, plane, nplanes,
                                                                     c0a, na, c0b, nb, sign, tw);
  count_launches(1);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

// Row transforms of a band of grid rows, [r0, r0 + nrows) of every plane
// (row stride L = nf1), two rows per item, in the register layout of
// k_col_fft_reg: thread t holds elements t + m T of both rows, loaded by
// cp.async one item ahead and stored straight from registers.  Elements
// [mid0, mid1) (the columns outside the image) are skipped as there: with
// skip = 1 they are zero on input and not loaded, with skip = 2 nothing
// reads them afterwards and they are not stored.
template <int L>
__global__ void __launch_bounds__(L / 16) k_row_fft_reg(float2* __restrict__ grid, size_t plane,
                                                        int nplanes, int r0, int nrows, int sign,
                                                        const float2* __restrict__ tw, int mid0,
                                                        int mid1, int skip) {
  constexpr int T = L / 16;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float4* pre = reinterpret_cast<float4*>(smem_raw);  // element j: (row 0, row 1)
  float2* xch = reinterpret_cast<float2*>(smem_raw + (size_t)L * sizeof(float4));
  const int t = threadIdx.x;
  const int pairs = nrows / 2;
  const int64_t items = (int64_t)pairs * nplanes;
  auto base_of = [&](int64_t it) {
    const int p = (int)(it / pairs), rp = (int)(it - (int64_t)p * pairs);
    return grid + (size_t)p * plane + (size_t)(r0 + 2 * rp) * L;
  };
  auto outside = [&](int j) { return j >= mid0 && j < mid1; };
  auto prefetch = [&](int64_t it) {
    const float2* b = base_of(it);
#pragma unroll
    for (int m = 0; m < 16; m++) {
      const int j = t + m * T;
      if (skip == 1 && outside(j)) continue;  // zero columns: not loaded
      const unsigned dst = (unsigned)__cvta_generic_to_shared(pre + j);
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(b + j) : "memory");
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst + 8), "l"(b + L + j)
                   : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  int64_t it = blockIdx.x;
  if (it < items) prefetch(it);
  for (; it < items; it += gridDim.x) {
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    float2 a[16], b[16];
#pragma unroll
    for (int m = 0; m < 16; m++) {
      const int j = t + m * T;
      const float4 v = (skip == 1 && outside(j)) ? make_float4(0.f, 0.f, 0.f, 0.f) : pre[j];
      a[m] = make_float2(v.x, v.y);
      b[m] = make_float2(v.z, v.w);
    }
    __syncthreads();  // the prefetch buffer is free again
    if (it + gridDim.x < items) prefetch(it + gridDim.x);
    fft_regs<L>(a, b, sign, tw, xch);
    float2* bs = base_of(it);
#pragma unroll
    for (int m = 0; m < 16; m++) {
      const int j = t + m * T;
      if (skip == 2 && outside(j)) continue;  // columns nothing reads
      bs[j] = a[m];
      bs[L + j] = b[m];
    }
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

template <int L>
int launch_row(float2* grid, size_t plane, int nplanes, int r0, int nrows, int sign,
               const float2* tw, cudaStream_t st, int mid0, int mid1, int skip) {
  const size_t smem = (size_t)L * sizeof(float4) + (size_t)(pad16(L) + 16) * sizeof(float2);
  int per_sm = 0;
  CG_CUDA(kernel_occupancy((const void*)k_row_fft_reg<L>, L / 16, smem, &per_sm));
  if (per_sm < 1) return CG_ERR_ARG;
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) sms = 148;
  }
  const int64_t items = (int64_t)(nrows / 2) * nplanes;
  const int blocks = (int)std::min<int64_t>(items, (int64_t)per_sm * sms);
  k_row_fft_reg<L><<<blocks, L / 16, smem, st>>>(grid, plane, nplanes, r0, nrows, sign, tw, mid0,
                                                 mid1, skip);
  count_launches(1);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

template <int L>
int launch_reg(float2* grid, int nf1, size_t plane, int nplanes, int c0a, int na, int c0b, int nb,
               int sign, const float2* tw, cudaStream_t st, int mid0, int mid1, int skip, int b0,
               int b1) {
  const size_t smem = (size_t)L * sizeof(float4) + (size_t)(pad16(L) + 16) * sizeof(float2);
  int per_sm = 0;
  CG_CUDA(kernel_occupancy((const void*)k_col_fft_reg<L>, L / 16, smem, &per_sm));
  if (per_sm < 1) return CG_ERR_ARG;
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) sms = 148;
  }
  const int64_t items = (int64_t)(na / 2 + nb / 2) * nplanes;
  const int blocks = (int)std::min<int64_t>(items, (int64_t)per_sm * sms);
  k_col_fft_reg<L><<<blocks, L / 16, smem, st>>>(grid, nf1, plane, nplanes, c0a, na, c0b, nb,
                                                 sign, tw, mid0, mid1, skip, b0, b1);
  count_launches(1);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

// columns per CTA of the shared-memory-resident kernel: two (16-byte rows),
// or one with CG_COL_FFT_CB=1 (8-byte rows: slower on B200, kept for tests)
inline int col_fft_cb(int L) {
  (void)L;
  const char* e = getenv("CG_COL_FFT_CB");
  return e && atoi(e) == 1 ? 1 : 2;
}

template <int L, int CB>
int launch_lc(float2* grid, int nf1, size_t plane, int nplanes, int c0a, int na, int c0b, int nb,
              int sign, const float2* tw, cudaStream_t st) {
  using V = typename ColVec<CB>::type;
  const size_t smem = (size_t)(pad16(L) + 16) * sizeof(V);
  int per_sm = 0;
  CG_CUDA(kernel_occupancy((const void*)k_col_fft<L, CB>, kFftThreads, smem, &per_sm));
  if (per_sm < 1) return CG_ERR_ARG;
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) sms = 148;
  }
  const int64_t items = (int64_t)(na / CB + nb / CB) * nplanes;
  const int blocks = (int)std::min<int64_t>(items, (int64_t)per_sm * sms);
  k_col_fft<L, CB><<<blocks, kFftThreads, smem, st>>>(grid, nf1, plane, nplanes, c0a, na, c0b, nb,
                                                     sign, tw);
  count_launches(1);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

template <int L>
int launch_l(float2* grid, int nf1, size_t plane, int nplanes, int c0a, int na, int c0b, int nb,
             int sign, const float2* tw, cudaStream_t st, int mid0, int mid1, int skip, int b0,
             int b1) {
  // CG_COL_FFT_REG=0: the shared-memory-resident kernel instead of the register-resident one
  const char* e = getenv("CG_COL_FFT_REG");
  const int reg = e ? atoi(e) : 1;
  if (reg == 3 && na % 8 == 0 && nb % 8 == 0)
    return launch_cluster<L>(grid, nf1, plane, nplanes, c0a, na, c0b, nb, sign, tw, st);
  if (reg == 2) return launch_reg2<L>(grid, nf1, plane, nplanes, c0a, na, c0b, nb, sign, tw, st);
  if (reg != 0)
    return launch_reg<L>(grid, nf1, plane, nplanes, c0a, na, c0b, nb, sign, tw, st, mid0, mid1,
                         skip, b0, b1);
  return col_fft_cb(L) == 1
             ? launch_lc<L, 1>(grid, nf1, plane, nplanes, c0a, na, c0b, nb, sign, tw, st)
             : launch_lc<L, 2>(grid, nf1, plane, nplanes, c0a, na, c0b, nb, sign, tw, st);
}

// ---------------------------------------------------------------- four-step
// Column transforms of length L = 64 * L2 in two in-place passes over 16
// adjacent columns per CTA, so that every load and store is a 128-byte grid
// row segment (the one-pass column kernels move 16 bytes per row).  With
// j = j1 + L2 j2 and k = k2 + 64 k1:
//   X[k2 + 64 k1] = sum_j1 w_L2^(j1 k1) w_L^(j1 k2) sum_j2 x[j1 + L2 j2] w_64^(j2 k2).
// Inverse (x natural): pass 1 = 64-point DFTs over the row sets
// {j1 + L2 j2}, times w_L^(j1 k2), in place; pass 2 = L2-point DFTs over the
// row blocks [L2 k2, L2 k2 + L2), in place, so row k1 + L2 k2 holds
// X[k2 + 64 k1]: index g sits at row perm(g) = g / 64 + L2 (g % 64), which the
// w-DFT reads through.  Forward: the plane fill writes index g at row
// perm(g); pass 1 = L2-point DFTs over the blocks, times w_L^(k2 j1), in
// place; pass 2 = 64-point DFTs over the row sets, in place: natural output.
//
// One item = one row set of N rows (row s * base_mul + r * stride, r < N)
// of 16 columns of one plane.  Thread tid holds points tc + m (N/8) (m < 8)
// of column tid % 16, tc = tid / 16, so the 16 lanes of a half-warp touch one
// 128-byte row segment.  Radix-8 Stockham passes exchange through shared
// memory laid out [position][column]; roots[n] = e^{2 pi i n / L} gives every
// twiddle (conjugated for sign -1).
template <int N>
__device__ __forceinline__ void small_fft8(float2 (&x)[8], int tc, int col, float2* xs, int sign,
                                           const float2* __restrict__ roots, int L) {
  constexpr int T = N / 8;
  constexpr int RL = [] {
    int ns = 1;
    while (ns * 8 <= N) ns *= 8;
    return N / ns;
  }();
  auto w = [&](int e, int den) {  // w_den^e, den divides L
    const float2 r = roots[(int)(((int64_t)e * (L / den)) % L)];
    return make_float2(r.x, sign * r.y);
  };
  int Ns = 1;
#pragma unroll 1
  for (; Ns * 8 <= N; Ns *= 8) {
    const int k = tc & (Ns - 1);
    if (Ns > 1) {
#pragma unroll
      for (int m = 1; m < 8; m++) x[m] = cmul(x[m], w(m * k, Ns * 8));
    }
    dft_reg<8>(x, sign);
    if (Ns * 8 == N) return;  // last pass: outputs at tc + m T
    const int o0 = (tc - k) * 8 + k;
#pragma unroll
    for (int m = 0; m < 8; m++) xs[(o0 + m * Ns) * 16 + col] = x[m];
    __syncthreads();
#pragma unroll
    for (int m = 0; m < 8; m++) x[m] = xs[(tc + m * T) * 16 + col];
    __syncthreads();
  }
  if constexpr (RL > 1) {
    constexpr int Q = 8 / RL;
#pragma unroll
    for (int q = 0; q < Q; q++) {
      const int j = tc + q * T;
      float2 v[RL];
#pragma unroll
      for (int m = 0; m < RL; m++) {
        v[m] = x[q + m * Q];
        if (m > 0) v[m] = cmul(v[m], w(m * j, N));
      }
      dft_reg<RL>(v, sign);
#pragma unroll
      for (int m = 0; m < RL; m++) x[q + m * Q] = v[m];
    }
  }
}

template <int N>
__global__ void __launch_bounds__(2 * N) k_col_step(float2* __restrict__ grid, int nf1,
                                                    size_t plane, int c0a, int na, int c0b,
                                                    int nb, int L, int nsets, int base_mul,
                                                    int stride, int sign,
                                                    const float2* __restrict__ roots,
                                                    int twiddle) {
  constexpr int T = N / 8;
  __shared__ float2 xs[N * 16];
  const int tid = threadIdx.x, col = tid & 15, tc = tid >> 4;
  const int groups_a = na / 16, groups = groups_a + nb / 16;
  const int64_t item = blockIdx.x;
  const int sset = (int)(item % nsets);
  const int64_t rest = item / nsets;
  const int gi = (int)(rest % groups), p = (int)(rest / groups);
  const int col0 = gi < groups_a ? c0a + gi * 16 : c0b + (gi - groups_a) * 16;
  float2* base = grid + (size_t)p * plane + col0 + col;
  const int row0 = sset * base_mul;
  float2 x[8];
#pragma unroll
  for (int m = 0; m < 8; m++) x[m] = base[(size_t)(row0 + (tc + m * T) * stride) * nf1];
  small_fft8<N>(x, tc, col, xs, sign, roots, L);
  if (twiddle) {  // output k of set s times w_L^(s k)
#pragma unroll
    for (int m = 0; m < 8; m++) {
      const int k = tc + m * T;
      const float2 r = roots[(int)(((int64_t)sset * k) % L)];
      x[m] = cmul(x[m], make_float2(r.x, sign * r.y));
    }
  }
#pragma unroll
  for (int m = 0; m < 8; m++) base[(size_t)(row0 + (tc + m * T) * stride) * nf1] = x[m];
}

template <int N>
int launch_step(float2* grid, int nf1, size_t plane, int nplanes, int c0a, int na, int c0b, int nb,
                int L, int nsets, int base_mul, int stride, int sign, const float2* roots,
                int twiddle, cudaStream_t st) {
  const int64_t items = (int64_t)(na / 16 + nb / 16) * nplanes * nsets;
  if (items < 1) return CG_OK;
  if (items > 2147483647LL) return CG_ERR_SIZE;
  k_col_step<N><<<(unsigned)items, 2 * N, 0, st>>>(grid, nf1, plane, c0a, na, c0b, nb, L, nsets,
                                                   base_mul, stride, sign, roots, twiddle);
  count_launches(1);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

int step_n(int N, float2* grid, int nf1, size_t plane, int nplanes, int c0a, int na, int c0b,
           int nb, int L, int nsets, int base_mul, int stride, int sign, const float2* roots,
           int twiddle, cudaStream_t st) {
#define CG_STEP_CALL(n) \
  launch_step<n>(grid, nf1, plane, nplanes, c0a, na, c0b, nb, L, nsets, base_mul, stride, sign, roots, twiddle, st)
  switch (N) {
    case 16: return CG_STEP_CALL(16);
    case 32: return CG_STEP_CALL(32);
    case 64: return CG_STEP_CALL(64);
    case 128: return CG_STEP_CALL(128);
    case 256: return CG_STEP_CALL(256);
    default: return CG_ERR_ARG;
  }
#undef CG_STEP_CALL
}

}  // namespace

bool four_step_supported(int L, int na, int nb) {
  return (L == 1024 || L == 2048 || L == 4096 || L == 8192 || L == 16384) && na % 16 == 0 &&
         nb % 16 == 0;
}

int make_fft_roots(int L, float2* d_roots, cudaStream_t st) {
  std::vector<float2> h(L);
  for (int n = 0; n < L; n++) {
    const double a = 2.0 * kPi * (double)n / (double)L;
    h[n] = make_float2((float)std::cos(a), (float)std::sin(a));
  }
  CG_CUDA(cudaMemcpyAsync(d_roots, h.data(), sizeof(float2) * L, cudaMemcpyHostToDevice, st));
  CG_CUDA(cudaStreamSynchronize(st));
  return CG_OK;
}

int launch_col_fft_four_step(float2* grid, int L, int nf1, size_t plane, int nplanes, int c0a,
                             int na, int c0b, int nb, int sign, const float2* d_roots,
                             cudaStream_t st) {
  if (!four_step_supported(L, na, nb)) return CG_ERR_ARG;
  const int L2 = L / 64;
  // strided sets: 64 rows j1 + L2 j2 (s = j1); blocks: L2 rows L2 k2 + r (s = k2)
  auto sets = [&](int twiddle) {
    return step_n(64, grid, nf1, plane, nplanes, c0a, na, c0b, nb, L, L2, 1, L2, sign, d_roots,
                  twiddle, st);
  };
  auto blocks = [&](int twiddle) {
    return step_n(L2, grid, nf1, plane, nplanes, c0a, na, c0b, nb, L, 64, L2, 1, sign, d_roots,
                  twiddle, st);
  };
  if (sign > 0) {  // inverse: natural in, permuted out
    CG_TRY(sets(1));
    return blocks(0);
  }
  CG_TRY(blocks(1));  // forward: permuted in, natural out
  return sets(0);
}

int launch_row_fft(float2* grid, int L, size_t plane, int nplanes, int r0, int nrows, int sign,
                   const float2* d_tw, cudaStream_t st, int mid0, int mid1, int skip) {
  if (nrows < 2 || nrows % 2) return CG_ERR_ARG;
  if (skip != 0 && !(0 <= mid0 && mid0 <= mid1 && mid1 <= L)) skip = 0;
#define CG_ROW_CALL(l) launch_row<l>(grid, plane, nplanes, r0, nrows, sign, d_tw, st, mid0, mid1, skip)
  switch (L) {
    case 1024: return CG_ROW_CALL(1024);
    case 2048: return CG_ROW_CALL(2048);
    case 4096: return CG_ROW_CALL(4096);
    case 8192: return CG_ROW_CALL(8192);
    default: return CG_ERR_ARG;
  }
#undef CG_ROW_CALL
}

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
                   int c0b, int nb, int sign, const float2* d_tw, cudaStream_t st, int mid0,
                   int mid1, int skip, int b0, int b1) {
  if ((skip & 3) != 0 && !(0 <= mid0 && mid0 <= mid1 && mid1 <= L)) skip &= ~3;
  if ((skip & 12) != 0 && !(0 <= b0 && b0 <= b1 && b1 <= L)) skip &= ~12;
#define CG_COL_CALL(l) \
  launch_l<l>(grid, nf1, plane, nplanes, c0a, na, c0b, nb, sign, d_tw, st, mid0, mid1, skip, b0, b1)
  switch (L) {
    case 1024: return CG_COL_CALL(1024);
    case 2048: return CG_COL_CALL(2048);
    case 4096: return CG_COL_CALL(4096);
    case 8192: return CG_COL_CALL(8192);
    default: return CG_ERR_ARG;
  }
#undef CG_COL_CALL
}

}  // namespace cg
