// pair_hist.cuh -- the per-thread FP32 pair histogram shared by the planar
// and spherical pair kernels: layout [bin][quantity][thread] in shared
// memory (a warp's read-modify-writes hit 32 distinct banks), folded into FP64
// every ~4096 sources.
#pragma once
#include <cuda_runtime.h>

#include "tpcf_internal.cuh"

namespace tpcf {

template <int QA, int NC>
__device__ __forceinline__ void hist_add(float* hcol, int bin, const float* v) {
  float* h = hcol + bin * (QA * NC);
#pragma unroll
  for (int q = 0; q < QA; ++q) h[q * NC] += v[q];
}

// Fold the FP32 histogram into FP64: the block sums (times the lens factors
// val*w or w) and, when lens_col is set, this thread's per-lens FP64 column
// (zeroed before the launch: only non-zero cells are added).  Then clear this
// thread's column.  Called by all threads.
template <int QA, int BT>
__device__ __forceinline__ void flush_hist(float* hist, double* bsum, const double* fvw, const double* fw,
                                           int nb, double* lens_col, size_t lens_stride) {
  const int tid = threadIdx.x;
  __syncthreads();
  float* hcol = hist + tid;
  if (lens_col) {
    for (int q = 0; q < kQ; ++q) {
      const int qa = (q == QK && QA == 5) ? QW : q;
      for (int b = 0; b < nb; ++b) {
        const float v = hcol[(b * QA + qa) * BT];
        // the column was zeroed before the launch; one writer per column, so
        // the fire-and-forget adds land in program order (deterministic)
        if (v != 0.f) atomicAdd(lens_col + (size_t)(q * nb + b) * lens_stride, (double)v);
      }
    }
  }
  for (int e = tid; e < kQ * nb; e += BT) {
    const int q = e / nb, b = e - q * nb;
    if (q == QK && QA == 5) continue;  // K == w: copied from the w row at item end
    const float* row = hist + (b * QA + q) * BT;
    const double* f = (q == QGT || q == QGX) ? fvw : fw;
    double s = 0.0;
    if (q == QN) {
      for (int l = 0; l < BT; ++l) s += (double)row[(l + tid) & (BT - 1)];
    } else {
      for (int l = 0; l < BT; ++l) {
        const int c = (l + tid) & (BT - 1);
        s = fma((double)row[c], f[c], s);
      }
    }
    bsum[e] += s;
  }
  __syncthreads();
  for (int e = 0; e < nb * QA; ++e) hcol[e * BT] = 0.f;
}

}  // namespace tpcf
