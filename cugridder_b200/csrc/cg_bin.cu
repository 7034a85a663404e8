// Hive binning: the reference's bin_mapping (conv_interp_invoker.cu:121-224)
// re-designed as a stable LSD radix sort on the same hive-major cell key.
//
// Reference: histogram_3d_sparse (utils.cu:105-132) counts every one of the
// G grid cells with global atomics, thrust scans all G+1 counters
// (common_utils.cu:156-169; 3.8 GB of counters for a 4096^2 FP64 image) and
// mapping_based_gather_3d (utils.cu:457-486) scatters by atomic rank, so the
// order inside a cell is nondeterministic.  Here the key
//   (hx + hy*nhx + hz*nhx*nhy)*64 + (bx%8) + (by%8)*8      (8x8x1 hives)
// is computed from the same FP64 formulas, the rows are sorted stably by it
// (8-bit digits, tile-local ranks from warp match + per-warp histograms, one
// digit-major exclusive scan per pass), and the per-hive offsets -- the
// reference's hive_count -- are read off the sorted keys by binary search.
// Counts, offsets and cell membership equal the reference's; the order inside
// a cell is the original row order (one of the orders the reference can
// produce), so results are deterministic.
#include <algorithm>
#include <cfloat>

#include "cg_coords.cuh"
#include "cg_launch.cuh"

namespace cg {

// ---------------------------------------------------------------- w range
__device__ __forceinline__ unsigned long long ordered_key(double x) {
  unsigned long long b = (unsigned long long)__double_as_longlong(x);
  return (b & 0x8000000000000000ULL) ? ~b : (b | 0x8000000000000000ULL);
}
double decode_ordered(unsigned long long k) {
  unsigned long long b = (k & 0x8000000000000000ULL) ? (k & 0x7FFFFFFFFFFFFFFFULL) : ~k;
  double x;
  memcpy(&x, &b, sizeof(x));
  return x;
}

// min/max of the raw u, v, w columns (utils.cu:43-54 takes min/max of the
// scaled w; scaling by f/c*sign*2pi is monotone, so the host maps the
// extremes) and a flag for non-finite coordinates.  The u and v ranges give
// the band of grid rows / columns the data can touch (FFT pruning).
// mm layout: [u_min, u_max, v_min, v_max, w_min, w_max] as order-preserving
// integer keys, then the non-finite flag.
__global__ void k_wminmax(const double* __restrict__ uvw, int64_t M, unsigned long long* mm,
                          int* bad) {
  double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
  int nf = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < M;
       i += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const double x = uvw[3 * i + a];
      nf |= !isfinite(x);
      lo[a] = fmin(lo[a], x);
      hi[a] = fmax(hi[a], x);
    }
  }
#pragma unroll
  for (int a = 0; a < 3; a++)
    for (int o = 16; o > 0; o >>= 1) {
      lo[a] = fmin(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
      hi[a] = fmax(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
    }
  for (int o = 16; o > 0; o >>= 1) nf |= __shfl_xor_sync(0xffffffffu, nf, o);
  __shared__ double slo[3][32], shi[3][32];
  __shared__ int snf[32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
#pragma unroll
    for (int a = 0; a < 3; a++) {
      slo[a][warp] = lo[a];
      shi[a][warp] = hi[a];
    }
    snf[warp] = nf;
  }
  __syncthreads();
  if (warp == 0) {
    const int nwp = blockDim.x >> 5;
#pragma unroll
    for (int a = 0; a < 3; a++) {
      lo[a] = lane < nwp ? slo[a][lane] : DBL_MAX;
      hi[a] = lane < nwp ? shi[a][lane] : -DBL_MAX;
      for (int o = 16; o > 0; o >>= 1) {
        lo[a] = fmin(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
        hi[a] = fmax(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
      }
    }
    nf = lane < nwp ? snf[lane] : 0;
    for (int o = 16; o > 0; o >>= 1) nf |= __shfl_xor_sync(0xffffffffu, nf, o);
    if (lane == 0) {
#pragma unroll
      for (int a = 0; a < 3; a++) {
        atomicMin(&mm[2 * a], ordered_key(lo[a]));
        atomicMax(&mm[2 * a + 1], ordered_key(hi[a]));
      }
      if (nf) atomicOr(bad, 1);
    }
  }
}

int launch_wminmax(const double* d_uvw, int64_t M, unsigned long long* d_mm, int* d_bad,
                   cudaStream_t st) {
  unsigned long long init[6] = {~0ULL, 0ULL, ~0ULL, 0ULL, ~0ULL, 0ULL};
  CG_CUDA(cudaMemcpyAsync(d_mm, init, sizeof(init), cudaMemcpyHostToDevice, st));
  CG_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(int), st));
  if (M == 0) return CG_OK;
  int64_t blocks = (M + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_wminmax<<<(int)blocks, 256, 0, st>>>(d_uvw, M, d_mm, d_bad);
  count_launches(1);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

// ---------------------------------------------------------------- keys
template <typename K>
__global__ void k_keys(const double* __restrict__ uvw, int64_t M, Geom g, K* __restrict__ keys,
                       int* __restrict__ vals) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < M;
       i += (int64_t)gridDim.x * blockDim.x) {
    double X0, X1, X2, w;
    grid_coords(uvw + 3 * i, g, X0, X1, X2, w);
    int bx = (int)floor(X0), by = (int)floor(X1), bz = (int)floor(X2);
    K h = (K)(bx >> 3) + (K)(by >> 3) * (K)g.nhx + (K)bz * (K)g.nhx * (K)g.nhy;
    keys[i] = h * 64 + (K)((bx & 7) + ((by & 7) << 3));
    vals[i] = (int)i;
  }
}

// ---------------------------------------------------------------- radix sort
constexpr int kRsThreads = 256;
constexpr int kRsItems = 16;
constexpr int kRsTile = kRsThreads * kRsItems;  // 4096 rows per tile

template <typename K>
__global__ void __launch_bounds__(kRsThreads) k_rs_upsweep(const K* __restrict__ keys, int64_t M,
                                                           int shift, int ntiles,
                                                           int* __restrict__ counts) {
  __shared__ int hist[256];
  hist[threadIdx.x] = 0;
  __syncthreads();
  int64_t base = (int64_t)blockIdx.x * kRsTile;
  // all loads first, so they are in flight together
  int dg[kRsItems];
#pragma unroll
  for (int i = 0; i < kRsItems; i++) {
    int64_t idx = base + i * kRsThreads + threadIdx.x;
    dg[i] = idx < M ? (int)((keys[idx] >> shift) & 0xFF) : -1;
  }
#pragma unroll
  for (int i = 0; i < kRsItems; i++)
    if (dg[i] >= 0) atomicAdd(&hist[dg[i]], 1);
  __syncthreads();
  counts[(int64_t)threadIdx.x * ntiles + blockIdx.x] = hist[threadIdx.x];
}

__device__ __forceinline__ int block_excl_scan(int x, int* s_warp, int& total);

// Tile layout: warp w owns rows [w*512, w*512+512) of the tile, item i of
// lane l is row w*512 + i*32 + l; items are ranked in (w, i, l) order, which
// is the row order, so the pass is stable.  The ranked tile is first
// reordered in shared memory by digit, then written out with consecutive
// threads on consecutive positions of each digit's run (coalesced stores).
template <typename K>
__global__ void __launch_bounds__(kRsThreads) k_rs_downsweep(
    const K* __restrict__ keys_in, const int* __restrict__ vals_in, K* __restrict__ keys_out,
    int* __restrict__ vals_out, int64_t M, int shift, int ntiles, const int* __restrict__ offsets) {
  extern __shared__ __align__(16) unsigned char rs_smem[];
  K* skey = reinterpret_cast<K*>(rs_smem);                       // [kRsTile]
  int* sval = reinterpret_cast<int*>(skey + kRsTile);            // [kRsTile]
  int (*whist)[256] = reinterpret_cast<int (*)[256]>(sval + kRsTile);  // [8][256]
  int (*wpref)[256] = whist + 8;                                  // [8][256]
  int* dstart = &wpref[8][0];                                     // [256]
  int* s_warp = dstart + 256;                                     // [33]
  int* soff = s_warp + 36;                                        // [256]
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // this tile's output base of digit threadIdx.x, fetched while the tile ranks
  const int my_off = offsets[(int64_t)threadIdx.x * ntiles + blockIdx.x];
  for (int d = threadIdx.x; d < 8 * 256; d += kRsThreads) (&whist[0][0])[d] = 0;
  __syncthreads();
  K k[kRsItems];
  int v[kRsItems], r[kRsItems], dg[kRsItems];
  const int64_t tile0 = (int64_t)blockIdx.x * kRsTile;
  int64_t base = tile0 + warp * (kRsTile / 8);
  unsigned lt = (1u << lane) - 1u;
  // all loads first, so they are in flight together (the ranking below
  // synchronizes the warp per item)
#pragma unroll
  for (int i = 0; i < kRsItems; i++) {
    int64_t idx = base + i * 32 + lane;
    bool valid = idx < M;
    k[i] = valid ? keys_in[idx] : (K)0;
    v[i] = valid ? vals_in[idx] : 0;
  }
#pragma unroll
  for (int i = 0; i < kRsItems; i++) {
    int64_t idx = base + i * 32 + lane;
    bool valid = idx < M;
    int d = valid ? (int)((k[i] >> shift) & 0xFF) : 256;
    unsigned peers = __match_any_sync(0xffffffffu, d);
    int cur = (d < 256) ? whist[warp][d] : 0;
    __syncwarp();
    if (d < 256 && lane == __ffs(peers) - 1) whist[warp][d] = cur + __popc(peers);
    __syncwarp();
    r[i] = cur + __popc(peers & lt);
    dg[i] = d;
  }
  __syncthreads();
  int total;
  {
    int d = threadIdx.x, run = 0;
#pragma unroll
    for (int w = 0; w < 8; w++) {
      wpref[w][d] = run;
      run += whist[w][d];
    }
    const int ds = block_excl_scan(run, s_warp, total);  // tile-local start of digit d
    dstart[d] = ds;
    soff[d] = my_off - ds;  // output position of tile slot p of digit d: soff[d] + p
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kRsItems; i++) {
    if (dg[i] < 256) {
      const int p = dstart[dg[i]] + wpref[warp][dg[i]] + r[i];
      skey[p] = k[i];
      sval[p] = v[i];
    }
  }
  __syncthreads();
  for (int p = threadIdx.x; p < total; p += kRsThreads) {
    const K key = skey[p];
    const int d = (int)((key >> shift) & 0xFF);
    const int64_t pos = (int64_t)soff[d] + p;
    keys_out[pos] = key;
    vals_out[pos] = sval[p];
  }
}

template <typename K>
constexpr size_t rs_down_smem() {
  return (size_t)kRsTile * (sizeof(K) + 4) + (8 * 256 * 2 + 256 + 36 + 256) * 4;
}

// ---------------------------------------------------------------- scan
// Exclusive scan of int32 counters, three phases over 4096-element chunks.
constexpr int kScanThreads = 1024;
constexpr int kScanChunk = 4096;

__device__ __forceinline__ int block_excl_scan(int x, int* s_warp, int& total) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int inc = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) s_warp[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    int nw = blockDim.x >> 5;
    int t = lane < nw ? s_warp[lane] : 0;
    int ti = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, ti, o);
      if (lane >= o) ti += y;
    }
    s_warp[lane] = ti - t;
    if (lane == 31) s_warp[32] = ti;
  }
  __syncthreads();
  int res = s_warp[warp] + inc - x;
  total = s_warp[32];
  __syncthreads();
  return res;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const int* __restrict__ in, int64_t n,
                                                              int* __restrict__ sums) {
  __shared__ int s[33];
  int64_t base = (int64_t)blockIdx.x * kScanChunk;
  int acc = 0;
  for (int i = threadIdx.x; i < kScanChunk; i += kScanThreads) {
    int64_t idx = base + i;
    if (idx < n) acc += in[idx];
  }
  int total;
  block_excl_scan(acc, s, total);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_top(int* sums, int nb) {
  __shared__ int s[33];
  int carry = 0;
  for (int base = 0; base < nb; base += kScanThreads) {
    int i = base + threadIdx.x;
    int x = i < nb ? sums[i] : 0;
    int total;
    int ex = block_excl_scan(x, s, total);
    if (i < nb) sums[i] = ex + carry;
    carry += total;
  }
}

__global__ void __launch_bounds__(kScanThreads) k_scan_down(const int* __restrict__ in, int64_t n,
                                                            const int* __restrict__ sums,
                                                            int* __restrict__ out) {
  __shared__ int s[33];
  int64_t base = (int64_t)blockIdx.x * kScanChunk + (int64_t)threadIdx.x * 4;
  int x[4];
#pragma unroll
  for (int j = 0; j < 4; j++) x[j] = (base + j < n) ? in[base + j] : 0;
  int t = x[0] + x[1] + x[2] + x[3];
  int total;
  int ex = block_excl_scan(t, s, total) + sums[blockIdx.x];
#pragma unroll
  for (int j = 0; j < 4; j++) {
    if (base + j < n) out[base + j] = ex;
    ex += x[j];
  }
}

static int scan_exclusive(const int* d_in, int64_t n, int* d_out, int* d_sums, cudaStream_t st) {
  int nb = (int)((n + kScanChunk - 1) / kScanChunk);
  k_scan_reduce<<<nb, kScanThreads, 0, st>>>(d_in, n, d_sums);
  k_scan_top<<<1, kScanThreads, 0, st>>>(d_sums, nb);
  k_scan_down<<<nb, kScanThreads, 0, st>>>(d_in, n, d_sums, d_out);
  count_launches(3);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

// ---------------------------------------------------------------- hive offsets
// hive_start[h] = first sorted row whose key >= 64 h, for h = 0..nh, by
// binary search (used when no scan scratch is given).
template <typename K>
__global__ void k_hive_start(const K* __restrict__ skeys, int64_t M, int64_t nh,
                             int* __restrict__ hive_start) {
  for (int64_t h = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; h <= nh;
       h += (int64_t)gridDim.x * blockDim.x) {
    unsigned long long target = (unsigned long long)h * 64ULL;
    int64_t lo = 0, hi = M;
    while (lo < hi) {
      int64_t mid = (lo + hi) >> 1;
      if ((unsigned long long)skeys[mid] < target) lo = mid + 1; else hi = mid;
    }
    hive_start[h] = (int)lo;
  }
}

// rows per hive from the sorted keys: runs of equal hives inside a warp are
// counted with one atomic by their first lane (counts zeroed beforehand)
template <typename K>
__global__ void k_hive_count(const K* __restrict__ skeys, int64_t M, int* __restrict__ counts) {
  const int lane = threadIdx.x & 31;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < M; base += stride) {
    const int64_t s = base + threadIdx.x;
    const long long h = s < M ? (long long)((unsigned long long)skeys[s] >> 6) : -1LL;
    const unsigned peers = __match_any_sync(0xffffffffu, h);
    if (h >= 0 && lane == __ffs(peers) - 1) atomicAdd(&counts[h], __popc(peers));
  }
}

// ---------------------------------------------------------------- driver
static inline size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

size_t bin_workspace_bytes(int64_t M, int key_bytes) {
  int64_t ntiles = (M + kRsTile - 1) / kRsTile;
  if (ntiles < 1) ntiles = 1;
  int64_t ncount = 256 * ntiles;
  int64_t nsums = (ncount + kScanChunk - 1) / kScanChunk;
  return align256((size_t)M * key_bytes) /* keys ping */ + align256((size_t)M * key_bytes) +
         align256((size_t)M * 4) /* vals pong */ + align256((size_t)ncount * 4) * 2 +
         align256((size_t)nsums * 4);
}

int launch_scan_exclusive(const int* d_in, int64_t n, int* d_out, int* d_sums, cudaStream_t st) {
  return scan_exclusive(d_in, n, d_out, d_sums, st);
}

template <typename K>
static int bin_impl(const double* d_uvw, int64_t M, const Geom& g, void* d_ws, int* d_perm,
                    K* d_sorted_keys, int* d_hive_start, cudaStream_t st, int* d_hs_sums) {
  int64_t ntiles = (M + kRsTile - 1) / kRsTile;
  int64_t ncount = 256 * ntiles;
  char* p = (char*)d_ws;
  K* ka = (K*)p; p += align256((size_t)M * sizeof(K));
  K* kb = (K*)p; p += align256((size_t)M * sizeof(K));
  int* vb = (int*)p; p += align256((size_t)M * 4);
  int* counts = (int*)p; p += align256((size_t)ncount * 4);
  int* offs = (int*)p; p += align256((size_t)ncount * 4);
  int* sums = (int*)p;
  int* va = d_perm;  // values ping buffer doubles as the output permutation

  int64_t nh = (int64_t)g.nhx * g.nhy * g.nhz;
  unsigned long long maxkey = (unsigned long long)nh * 64ULL;
  int bits = 0;
  while (bits < 64 && (maxkey >> bits) != 0ULL) bits++;
  int passes = (bits + 7) / 8;

  if (M > 0) {
    int blocks = (int)((M + 255) / 256);
    if (blocks > 148 * 32) blocks = 148 * 32;
    k_keys<K><<<blocks, 256, 0, st>>>(d_uvw, M, g, ka, va);
  count_launches(1);
    CG_CUDA(cudaGetLastError());
    CG_CUDA(cudaFuncSetAttribute(k_rs_downsweep<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)rs_down_smem<K>()));
    K* kin = ka; int* vin = va; K* kout = kb; int* vout = vb;
    for (int ps = 0; ps < passes; ps++) {
      int shift = 8 * ps;
      if (ps == passes - 1) {  // the last pass writes the outputs in place of a copy
        kout = d_sorted_keys;
        if (vin != d_perm) vout = d_perm;
      }
      k_rs_upsweep<K><<<(int)ntiles, kRsThreads, 0, st>>>(kin, M, shift, (int)ntiles, counts);
      count_launches(1);
      CG_TRY(scan_exclusive(counts, ncount, offs, sums, st));
      k_rs_downsweep<K><<<(int)ntiles, kRsThreads, rs_down_smem<K>(), st>>>(
          kin, vin, kout, vout, M, shift, (int)ntiles, offs);
      count_launches(1);
      CG_CUDA(cudaGetLastError());
      K* tk = kin; kin = kout; kout = tk;
      int* tv = vin; vin = vout; vout = tv;
    }
    if (vin != d_perm) CG_CUDA(cudaMemcpyAsync(d_perm, vin, (size_t)M * 4, cudaMemcpyDeviceToDevice, st));
  }
  if (d_hs_sums) {
    // counts per hive, then an in-place exclusive scan: O(M + nh), no search
    CG_CUDA(cudaMemsetAsync(d_hive_start, 0, (size_t)(nh + 1) * 4, st));
    if (M > 0) {
      int cb = (int)std::min<int64_t>((M + 255) / 256, 148 * 16);
      k_hive_count<K><<<cb, 256, 0, st>>>(d_sorted_keys, M, d_hive_start);
      count_launches(1);
      CG_CUDA(cudaGetLastError());
    }
    return scan_exclusive(d_hive_start, nh + 1, d_hive_start, d_hs_sums, st);
  }
  int hb = (int)((nh + 1 + 255) / 256);
  if (hb > 148 * 32) hb = 148 * 32;
  k_hive_start<K><<<hb, 256, 0, st>>>(d_sorted_keys, M, nh, d_hive_start);
  count_launches(1);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

__global__ void k_iota(int* __restrict__ v, int64_t M) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < M;
       i += (int64_t)gridDim.x * blockDim.x)
    v[i] = (int)i;
}

// Stable sort of 32-bit keys (only the low `bits` bits are significant):
// d_perm gets the original index of each sorted key and d_sorted its key.
// d_keys is overwritten; workspace: bin_workspace_bytes(M, 4).
int launch_sort_u32(uint32_t* d_keys, int64_t M, int bits, void* d_ws, size_t ws_bytes,
                    int* d_perm, uint32_t* d_sorted, cudaStream_t st) {
  if (ws_bytes < bin_workspace_bytes(M, 4)) return CG_ERR_ARG;
  if (M == 0) return CG_OK;
  using K = uint32_t;
  const int64_t ntiles = (M + kRsTile - 1) / kRsTile, ncount = 256 * ntiles;
  char* p = (char*)d_ws;
  K* kb = (K*)p; p += align256((size_t)M * 4);
  p += align256((size_t)M * 4);  // (second key buffer of the plan layout, unused here)
  int* vb = (int*)p; p += align256((size_t)M * 4);
  int* counts = (int*)p; p += align256((size_t)ncount * 4);
  int* offs = (int*)p; p += align256((size_t)ncount * 4);
  int* sums = (int*)p;
  const int blocks = (int)std::min<int64_t>((M + 255) / 256, 148 * 32);
  k_iota<<<blocks, 256, 0, st>>>(d_perm, M);
  count_launches(1);
  CG_CUDA(cudaFuncSetAttribute(k_rs_downsweep<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)rs_down_smem<K>()));
  K* kin = d_keys; int* vin = d_perm; K* kout = kb; int* vout = vb;
  const int passes = std::max(1, (bits + 7) / 8);
  for (int ps = 0; ps < passes; ps++) {
    const int shift = 8 * ps;
    k_rs_upsweep<K><<<(int)ntiles, kRsThreads, 0, st>>>(kin, M, shift, (int)ntiles, counts);
    count_launches(1);
    CG_TRY(scan_exclusive(counts, ncount, offs, sums, st));
    k_rs_downsweep<K><<<(int)ntiles, kRsThreads, rs_down_smem<K>(), st>>>(
        kin, vin, kout, vout, M, shift, (int)ntiles, offs);
    count_launches(1);
    CG_CUDA(cudaGetLastError());
    K* tk = kin; kin = kout; kout = tk;
    int* tv = vin; vin = vout; vout = tv;
  }
  if (vin != d_perm) CG_CUDA(cudaMemcpyAsync(d_perm, vin, (size_t)M * 4, cudaMemcpyDeviceToDevice, st));
  CG_CUDA(cudaMemcpyAsync(d_sorted, kin, (size_t)M * 4, cudaMemcpyDeviceToDevice, st));
  return CG_OK;
}

int launch_bin(const double* d_uvw, int64_t M, const Geom& g, int key_bytes, void* d_ws,
               size_t ws_bytes, int* d_perm, void* d_sorted_keys, int* d_hive_start,
               cudaStream_t st, int* d_hs_sums) {
  if (ws_bytes < bin_workspace_bytes(M, key_bytes)) return CG_ERR_ARG;
  if (key_bytes == 4)
    return bin_impl<uint32_t>(d_uvw, M, g, d_ws, d_perm, (uint32_t*)d_sorted_keys, d_hive_start, st,
                              d_hs_sums);
  return bin_impl<unsigned long long>(d_uvw, M, g, d_ws, d_perm, (unsigned long long*)d_sorted_keys,
                                      d_hive_start, st, d_hs_sums);
}

// ---------------------------------------------------------------- sorted stream
// One record per sorted row: cell + fraction split in FP64, then the payload:
//   gridding:   c = vis * wgt * exp(+i o_c w)   (ra_exec.cu:103-111; pre_stage_1 cuft.cu:46-66)
//   degridding: factor = wgt * exp(-i o_c w)    (cura_fw ra_exec.cu:75-93; shift_corr :55-66)
template <typename T, bool kGrid>
__device__ __forceinline__ Rec<T> make_rec(int64_t i, const double* __restrict__ uvw,
                                           const T* __restrict__ vis, const T* __restrict__ wgt,
                                           const Geom& g) {
  double X0, X1, X2, w;
  grid_coords(uvw + 3 * i, g, X0, X1, X2, w);
  double fb0 = floor(X0), fb1 = floor(X1), fb2 = floor(X2);
  Rec<T> r;
  r.f[0] = (T)(X0 - fb0);
  r.f[1] = (T)(X1 - fb1);
  r.f[2] = (T)(X2 - fb2);
  // guard against a fraction rounding up to 1 in the working precision
  const T below1 = sizeof(T) == 4 ? (T)0.99999994f : (T)0.99999999999999989;
  if (r.f[0] >= (T)1) r.f[0] = below1;
  if (r.f[1] >= (T)1) r.f[1] = below1;
  if (r.f[2] >= (T)1) r.f[2] = below1;
  r.bxy = (uint32_t)(int)fb0 | ((uint32_t)(int)fb1 << 16);
  r.bz = (uint32_t)(int)fb2;
  double sn, cs;
  sincos(g.o_center * w * (kGrid ? 1.0 : -1.0), &sn, &cs);
  double wt = wgt ? (double)wgt[i] : 1.0;
  if (kGrid) {
    double cr = (double)vis[2 * i] * wt, ci = (double)vis[2 * i + 1] * wt;
    r.c[0] = (T)(cr * cs - ci * sn);
    r.c[1] = (T)(cr * sn + ci * cs);
  } else {
    r.c[0] = (T)(wt * cs);
    r.c[1] = (T)(wt * sn);
  }
  return r;
}

// records in the original row order (coalesced reads of uvw / vis / wgt)
template <typename T, bool kGrid>
__global__ void k_build_rows(int64_t M, const double* __restrict__ uvw, const T* __restrict__ vis,
                             const T* __restrict__ wgt, Geom g, Rec<T>* __restrict__ tmp) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < M;
       i += (int64_t)gridDim.x * blockDim.x)
    tmp[i] = make_rec<T, kGrid>(i, uvw, vis, wgt, g);
}

// sorted stream: recs[s] = tmp[perm[s]], one aligned record per gather
template <typename T>
__global__ void k_gather_recs(const int* __restrict__ perm, int64_t M, const Rec<T>* __restrict__ tmp,
                              Rec<T>* __restrict__ recs) {
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < M;
       s += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = perm[s];
    if (i < 0 || i >= M) continue;  // never taken for a valid permutation; no wild reads
    recs[s] = tmp[i];
  }
}

// The records are built in row order into d_tmp (M records) and gathered by
// the sort permutation: random 24/8/4-byte reads of uvw/vis/wgt would each
// pull whole DRAM sectors, a 32-byte record gather pulls one.
template <typename T>
int launch_build_stream(const int* d_perm, int64_t M, const double* d_uvw, const T* d_vis,
                        const T* d_wgt, const Geom& g, bool grid_dir, Rec<T>* d_tmp,
                        Rec<T>* d_recs, cudaStream_t st) {
  if (M == 0) return CG_OK;
  int blocks = (int)((M + 255) / 256);
  if (blocks > 148 * 32) blocks = 148 * 32;
  if (grid_dir)
    k_build_rows<T, true><<<blocks, 256, 0, st>>>(M, d_uvw, d_vis, d_wgt, g, d_tmp);
  else
    k_build_rows<T, false><<<blocks, 256, 0, st>>>(M, d_uvw, d_vis, d_wgt, g, d_tmp);
  k_gather_recs<T><<<blocks, 256, 0, st>>>(d_perm, M, d_tmp, d_recs);
  count_launches(2);
  CG_CUDA(cudaGetLastError());
  return CG_OK;
}

template int launch_build_stream<float>(const int*, int64_t, const double*, const float*,
                                        const float*, const Geom&, bool, Rec<float>*, Rec<float>*,
                                        cudaStream_t);
template int launch_build_stream<double>(const int*, int64_t, const double*, const double*,
                                         const double*, const Geom&, bool, Rec<double>*,
                                         Rec<double>*, cudaStream_t);

}  // namespace cg
