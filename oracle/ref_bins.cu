// TEST INFRASTRUCTURE ONLY -- a parity checker, never shipped, linked into the
// product or measured.
//
// Runs the binning stage of the REFERENCE's own FP64 library
// (oracle/_ref/libcurafft_ref.so: the reference sources compiled for sm_100a
// by oracle/ref.mk) on caller data and reports what that library computed:
//
//  - plan->hive_count after cura_prestage (reference src/astro/ra_exec.cu:95-176,
//    which calls bin_mapping, src/fourier/conv_interp_invoker.cu:121-224): the
//    exclusive row offsets of the 8x8x1 hives;
//  - the rows per grid cell, from the reference's own histogram kernel
//    (histogram_3d_sparse_invoker, src/utils.cu:105-132 and 326-331) run once
//    more on the rows bin_mapping has sorted (a histogram does not depend on
//    the order of its rows).  The histogram index is the reference's padded
//    cell key (hx + hy nhx + hz nhx nhy) * 64 + bx % 8 + (by % 8) * 8.
//
// The set-up follows ms2dirty_exec (src/astro/cugridder.cu:276-360) up to its
// execution step: uvw copied and transposed on the device, then
// gridder_setting with the same arguments (method 6, ES kernel, improved
// w-stacking, direction 1).  Only the reference's own functions compute; this
// file moves data and counts nonzero cells.
//
// Built by oracle/ref.mk into oracle/_ref/libref_bins.so; called through ctypes
// by tests/golden/make_golden.py on a GPU.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "cugridder.h"
#include "common_utils.h"
#include "conv_interp_invoker.h"
#include "cuft.h"
#include "utils.h"

// defined in the reference's src/astro/ra_exec.cu:95 (no header declares it)
int cura_prestage(CURAFFT_PLAN *plan, ragridder_plan *gridder_plan);

extern "C" {

// Returns 0 on success; 2 when the reference takes its memory-limited path
// (no bin_mapping), 3 when an output array is too small (sizes still stored).
//   uvw        host [nrow][3] float64 (metres), as ms2dirty_2 takes it
//   nf, nhive  out: the grid (nf1, nf2, nf3) and hive counts of the plan
//   hive_count out: nhive0 * nhive1 * nhive2 + 1 offsets (capacity hive_cap)
//   cell_key, cell_count  out: the nonzero cells in ascending key order and
//              their row counts (capacity cell_cap); *ncells = their number
//   method     out: the gridding method bin_mapping ran (6, or 2 after the
//              reference's fallback for fewer than 3 hives on an axis)
int refbins_ms2dirty(int nrow, int nxdirty, int nydirty, double fov, double freq,
                     const double *uvw, double epsilon, double sigma, int sign, int *nf,
                     int *nhive, int *hive_count, long long hive_cap,
                     unsigned long long *cell_key, int *cell_count, long long cell_cap,
                     long long *ncells, int *method) {
  CURAFFT_PLAN *plan = new CURAFFT_PLAN();
  ragridder_plan *gp = new ragridder_plan();
  memset(plan, 0, sizeof(CURAFFT_PLAN));
  memset(gp, 0, sizeof(ragridder_plan));
  cudaMalloc((void **)&gp->d_uvw, 3 * (size_t)nrow * sizeof(double));
  cudaMemcpy(gp->d_uvw, uvw, 3 * (size_t)nrow * sizeof(double), cudaMemcpyHostToDevice);
  matrix_transpose_invoker(gp->d_uvw, 3, nrow);
  CUCPX *d_vis = nullptr;
  cudaMalloc((void **)&d_vis, (size_t)nrow * sizeof(CUCPX));
  cudaMemset(d_vis, 0, (size_t)nrow * sizeof(CUCPX));
  double *d_u = gp->d_uvw, *d_v = gp->d_uvw + nrow, *d_w = gp->d_uvw + 2 * (size_t)nrow;

  double f = freq;
  visibility pv;
  memset(&pv, 0, sizeof(pv));
  pv.u = (double *)uvw;
  pv.v = (double *)uvw + nrow;
  pv.w = (double *)uvw + 2 * (size_t)nrow;
  pv.frequency = &f;
  pv.pirange = 0;
  pv.sign = sign;
  gridder_setting(nydirty, nxdirty, 6, 0, 1, epsilon, 1, sigma, 0, 1, nrow, 1, fov, &pv, d_u, d_v,
                  d_w, d_vis, plan, gp);
  if (plan->mem_limit) return 2;
  cura_prestage(plan, gp);

  nf[0] = plan->nf1;
  nf[1] = plan->nf2;
  nf[2] = plan->nf3;
  for (int k = 0; k < 3; k++) nhive[k] = (nf[k] - 1) / plan->hivesize[k] + 1;
  *method = plan->opts.gpu_gridder_method;
  const long long nh = (long long)nhive[0] * nhive[1] * nhive[2];
  int status = 0;
  if (hive_cap >= nh + 1)
    cudaMemcpy(hive_count, plan->hive_count, (size_t)(nh + 1) * sizeof(int), cudaMemcpyDeviceToHost);
  else
    status = 3;

  // rows per cell: the reference's histogram kernel over the sorted rows
  const unsigned long long cells = (unsigned long long)nhive[0] * plan->hivesize[0] *
                                   nhive[1] * plan->hivesize[1] * nhive[2] * plan->hivesize[2];
  int *d_histo = nullptr, *d_rank = nullptr;
  cudaMalloc((void **)&d_histo, (cells + 1) * sizeof(int));
  cudaMemset(d_histo, 0, (cells + 1) * sizeof(int));
  cudaMalloc((void **)&d_rank, (size_t)nrow * sizeof(int));
  histogram_3d_sparse_invoker(plan->d_u, plan->d_v, plan->d_w, d_rank, d_histo, nrow, plan->nf1,
                              plan->nf2, plan->nf3, plan->hivesize, nhive, plan->copts.pirange);
  std::vector<int> histo(cells + 1);
  cudaMemcpy(histo.data(), d_histo, (cells + 1) * sizeof(int), cudaMemcpyDeviceToHost);
  long long n = 0;
  for (unsigned long long k = 0; k <= cells; k++) {
    if (!histo[k]) continue;
    if (n < cell_cap) {
      cell_key[n] = k;
      cell_count[n] = histo[k];
    }
    n++;
  }
  *ncells = n;
  if (n > cell_cap) status = 3;

  cudaFree(d_histo);
  cudaFree(d_rank);
  cudaFree(d_vis);  // bin_mapping replaced plan->d_c by its sorted copy
  cudaFree(plan->hive_count);
  cudaFree(plan->d_x);
  curafft_free(plan);
  delete plan;
  delete gp;
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    fprintf(stderr, "refbins: %s\n", cudaGetErrorString(e));
    return 1;
  }
  return status;
}

}  // extern "C"
