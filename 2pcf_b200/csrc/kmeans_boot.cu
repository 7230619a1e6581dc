// kmeans_boot.cu -- device k-means patches and the batched block bootstrap.
//
// k-means replaces the Lloyd loop of partition_data (src/kmeans.f90:12-263) in
// its Voronoi-block form (equal_size = .false., src/tpcf.f90:1117-1124): the
// fixed-grid initial centroids (src/kmeans.f90:85-112) and initial labels are
// computed exactly as the reference does in FP32; each iteration assigns every
// point to the nearest centroid by the FP32 distance sqrt(dx*dx + dy*dy) (IEEE
// rounding, no contraction, strict '<' from the first centroid), then sets the
// centroids to the weighted means.  The means are summed in 64-bit fixed point
// (x*w*2^s rounded to an integer, s chosen so no sum overflows), so the result
// does not depend on the order of the atomic additions: every run gives the
// same labels.  The loop stops when no label changes, or when the fraction of
// changed labels drops below the tolerance, or after max_iter + 1 passes, as
// in the reference.
//
// The bootstrap replaces the resampling loop of
// survey_marked_point_block_bootstrap (src/tpcf.f90:1166-1191) and
// covariance_matrix (src/utils.f90:745-764), for all tasks at once: each
// resample draws n_draw patch indices with replacement (Philox4x32-10, a
// counter-based generator, so every draw is a pure function of
// (seed, resample, draw)), and g = sum(mult*S_g)/sum(mult*S_K) per task and bin.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "tpcf_b200.h"
#include "tpcf_ctx.h"
#include "philox.cuh"
#include "tpcf_internal.cuh"
#include "tpcf_kernels.h"

namespace {

using namespace tpcf;

constexpr int kMaxK = 4096;

// ------------------------------------------------------------------ k-means --
__global__ void k_km_init_labels(int* labels, long long n, int k) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    // int(real(i-1)/n_data*k + 1) with 1-based i (src/kmeans.f90:106-107), then 0-based
    const float v = __fadd_rn(__fmul_rn(__fdiv_rn((float)i, (float)n), (float)k), 1.0f);
    labels[i] = (int)v - 1;
  }
}

// Assign each point to its nearest centroid; accumulate fixed-point sums of
// x*w, y*w and w per cluster and count the reassignments.
__global__ void k_km_assign(const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ w,
                            long long n, const float2* __restrict__ cen, int k, float min_init, double sp_scale,
                            double sw_scale, int* labels, unsigned long long* acc, unsigned long long* n_re) {
  extern __shared__ unsigned char sm[];
  float2* c = reinterpret_cast<float2*>(sm);
  unsigned long long* a = reinterpret_cast<unsigned long long*>(c + k);
  for (int j = threadIdx.x; j < k; j += blockDim.x) c[j] = cen[j];
  for (int j = threadIdx.x; j < 3 * k; j += blockDim.x) a[j] = 0ull;
  __syncthreads();
  unsigned long long re = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float xi = x[i], yi = y[i];
    float best = min_init;
    int bi = -1;
    for (int j = 0; j < k; ++j) {
      const float dx = __fsub_rn(xi, c[j].x), dy = __fsub_rn(yi, c[j].y);
      const float d = __fsqrt_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)));
      if (d < best) {
        best = d;
        bi = j;
      }
    }
    if (bi != labels[i]) {
      labels[i] = bi;
      ++re;
    }
    if (bi >= 0) {
      const double wi = (double)w[i];
      atomicAdd(&a[3 * bi + 0], (unsigned long long)__double2ll_rn((double)xi * wi * sp_scale));
      atomicAdd(&a[3 * bi + 1], (unsigned long long)__double2ll_rn((double)yi * wi * sp_scale));
      atomicAdd(&a[3 * bi + 2], (unsigned long long)__double2ll_rn(wi * sw_scale));
    }
  }
  __syncthreads();
  for (int j = threadIdx.x; j < 3 * k; j += blockDim.x)
    if (a[j]) atomicAdd(&acc[j], a[j]);
  for (int o = 16; o; o >>= 1) re += __shfl_xor_sync(0xffffffffu, re, o);
  if ((threadIdx.x & 31) == 0 && re) atomicAdd(n_re, re);
}

// Centroids from the fixed-point sums (two's-complement int64), then clear them.
__global__ void k_km_update(unsigned long long* acc, int k, int sp, int sw, float2* cen) {
  for (int j = threadIdx.x; j < k; j += blockDim.x) {
    const double W = ldexp((double)(long long)acc[3 * j + 2], -sw);
    const double cx = ldexp((double)(long long)acc[3 * j + 0], -sp) / W;
    const double cy = ldexp((double)(long long)acc[3 * j + 1], -sp) / W;
    cen[j] = make_float2((float)cx, (float)cy);
    acc[3 * j + 0] = acc[3 * j + 1] = acc[3 * j + 2] = 0ull;
  }
}

// Largest s with n * vmax * 2^s < 2^62, clamped to [0, 60] (shared with the oracle).
int fixed_scale(long long n, double vmax) {
  if (!(vmax > 0)) return 60;
  int e;
  std::frexp((double)n * vmax, &e);
  return std::max(0, std::min(60, 62 - e));
}

// ---------------------------------------------------------------- bootstrap --
// One block per resample: n_draw Philox draws of a patch index in [0, n_patch)
// (counter (d/4, s, 0x2BCF, 0), word d%4, multiply-shift), counted.
__global__ void k_boot_mult(unsigned long long seed, int n_patch, int n_draw, int* mult) {
  extern __shared__ int hist[];
  const int s = blockIdx.x;
  for (int p = threadIdx.x; p < n_patch; p += blockDim.x) hist[p] = 0;
  __syncthreads();
  for (int q = threadIdx.x; q < (n_draw + 3) / 4; q += blockDim.x) {
    uint32_t c[4] = {(uint32_t)q, (uint32_t)s, 0x2BCFu, 0u};
    philox4x32(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    for (int u = 0; u < 4; ++u) {
      const int d = 4 * q + u;
      if (d < n_draw) atomicAdd(&hist[(int)(((unsigned long long)c[u] * (unsigned)n_patch) >> 32)], 1);
    }
  }
  __syncthreads();
  for (int p = threadIdx.x; p < n_patch; p += blockDim.x) mult[(size_t)s * n_patch + p] = hist[p];
}

// g_t, g_x per (resample, task, bin) and weights per (resample, task) from the
// patch sums [n_task][n_patch][6][n_bin] (rows dw, gt, gx, w, K, n).  Sums run
// over patches in index order.
__global__ void k_boot_resample(const double* __restrict__ ps, const int* __restrict__ mult, int n_boot, int n_task,
                                int n_patch, int nb, double* gt, double* gx, double* W) {
  const long long tot = (long long)n_boot * n_task * (nb + 1);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot; i += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(i % (nb + 1));
    const long long st = i / (nb + 1);
    const int t = (int)(st % n_task);
    const int s = (int)(st / n_task);
    const int* m = mult + (size_t)s * n_patch;
    const double* base = ps + (size_t)t * n_patch * 6 * nb;
    if (b < nb) {
      double St = 0, Sx = 0, SK = 0;
      // products rounded before the sum (no FMA), as src/tpcf.f90:1180-1183 evaluates
      for (int p = 0; p < n_patch; ++p) {
        const double mp = (double)m[p];
        const double* r = base + (size_t)p * 6 * nb;
        St = __dadd_rn(St, __dmul_rn(r[1 * nb + b], mp));
        Sx = __dadd_rn(Sx, __dmul_rn(r[2 * nb + b], mp));
        SK = __dadd_rn(SK, __dmul_rn(r[4 * nb + b], mp));
      }
      const size_t o = ((size_t)s * n_task + t) * nb + b;
      gt[o] = SK > 0 ? St / SK : 0.0;
      gx[o] = SK > 0 ? Sx / SK : 0.0;
    } else if (W) {
      double Sw = 0;
      for (int p = 0; p < n_patch; ++p) {
        const double* r = base + (size_t)p * 6 * nb;
        double pw = 0;
        for (int bb = 0; bb < nb; ++bb) pw += r[3 * nb + bb];
        Sw = __dadd_rn(Sw, __dmul_rn(pw, (double)m[p]));
      }
      W[(size_t)s * n_task + t] = Sw;
    }
  }
}

// Unbiased sample covariance of x [n_s][D]: cov[i][j] (src/utils.f90:745-764).
__global__ void k_cov(const double* __restrict__ x, int n_s, int D, double* cov) {
  const int i = blockIdx.y;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j > i || i >= D) return;
  double mi = 0, mj = 0;
  for (int s = 0; s < n_s; ++s) {
    mi += x[(size_t)s * D + i];
    mj += x[(size_t)s * D + j];
  }
  mi /= n_s;
  mj /= n_s;
  double c = 0;
  for (int s = 0; s < n_s; ++s) c = __dadd_rn(c, __dmul_rn(x[(size_t)s * D + i] - mi, x[(size_t)s * D + j] - mj));
  c /= (n_s - 1);
  cov[(size_t)i * D + j] = c;
  cov[(size_t)j * D + i] = c;
}

tpcf_status fail(tpcf_ctx* c, const Failure& f) {
  c->err = f.msg;
  return f.status;
}

}  // namespace

namespace tpcf {
// Unbiased sample covariance [D][D] of n_s samples x [n_s][D] (covariance_matrix,
// src/utils.f90:745-764), FP64.
cudaError_t launch_cov(const double* x, int n_s, int D, double* cov, cudaStream_t st) {
  dim3 grid((unsigned)((D + 127) / 128), (unsigned)D);
  k_cov<<<grid, 128, 0, st>>>(x, n_s, D, cov);
  return cudaGetLastError();
}
}  // namespace tpcf

extern "C" {

tpcf_status tpcf_kmeans(tpcf_ctx* c, const float* x, const float* y, const float* w, int64_t n, int32_t k,
                        int32_t max_iter, float reassign_tol, int32_t* labels_out, float* centroids_out,
                        int32_t* n_iter_out) {
  if (!c || !labels_out || n < 1 || k < 2 || k > kMaxK || max_iter < 0 || !x || !y || !w ||
      n > (1ll << 31) - 2)
    return c ? (c->err = "invalid k-means arguments", TPCF_ERR_INVALID_ARG) : TPCF_ERR_INVALID_ARG;
  try {
    begin_call(c);
    cudaStream_t st = c->stream;
    x = stage(c, x, n);
    y = stage(c, y, n);
    w = stage(c, w, n);
    // box and max |w| (slot 6) of the points
    int* box_ord = (int*)ws_alloc(c, sizeof(int) * 8);
    unsigned long long* cnt = (unsigned long long*)ws_alloc(c, sizeof(unsigned long long));
    int* pr = (int*)ws_alloc(c, sizeof(int) * 2);
    float* boxf = (float*)ws_alloc(c, sizeof(float) * 8);
    counted(c, launch_bbox_init(box_ord, cnt, pr, 1, st), "bbox init");
    counted(c, launch_bbox(x, y, nullptr, nullptr, nullptr, w, n, 0, box_ord, cnt, pr, st), "bbox");
    counted(c, launch_bbox_finish(box_ord, boxf, 8, st), "bbox finish");
    float hb[8];
    unsigned long long hc = 0;
    check(cudaMemcpyAsync(hb, boxf, sizeof(hb), cudaMemcpyDeviceToHost, st), "D2H box");
    check(cudaMemcpyAsync(&hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, st), "D2H count");
    check(cudaStreamSynchronize(st), "sync box");
    if (hc != (unsigned long long)n) throw Failure(TPCF_ERR_INVALID_ARG, "non-finite k-means positions");
    const float xmn = hb[0], ymn = hb[1], xmx = hb[2], ymx = hb[3];
    // fixed-grid initial centroids, src/kmeans.f90:85-104, in FP32 as written
    std::vector<float> cen(2 * k);
    const int n_side = (int)sqrtf((float)k);
    if (xmx - xmn > ymx - ymn) {
      const float dy = (ymx - ymn) / (float)n_side;
      const float dx = (xmx - xmn) * (float)n_side / (float)k;
      for (int j = 1; j <= k; ++j) {
        const int row = (int)((dx / 2.0f + dx * (float)(j - 1)) / (xmx - xmn));
        cen[2 * (j - 1)] = xmn + fmodf(dx / 2.0f + dx * (float)(j - 1), xmx - xmn);
        cen[2 * (j - 1) + 1] = ymn + dy / 2.0f + dy * (float)row;
      }
    } else {
      const float dx = (xmx - xmn) / (float)n_side;
      const float dy = (ymx - ymn) * (float)n_side / (float)k;
      for (int j = 1; j <= k; ++j) {
        const int row = (int)((dy / 2.0f + dy * (float)(j - 1)) / (ymx - ymn));
        cen[2 * (j - 1) + 1] = ymn + fmodf(dy / 2.0f + dy * (float)(j - 1), ymx - ymn);
        cen[2 * (j - 1)] = xmn + dx / 2.0f + dx * (float)row;
      }
    }
    const float diam = sqrtf((xmx - xmn) * (xmx - xmn) + (ymx - ymn) * (ymx - ymn));
    const double amax = std::max(std::max(std::fabs((double)xmn), std::fabs((double)xmx)),
                                 std::max(std::fabs((double)ymn), std::fabs((double)ymx)));
    const double wmax = hb[6];
    const int sp = fixed_scale(n, amax * wmax), sw = fixed_scale(n, wmax);
    int* lab = (int*)ws_alloc(c, sizeof(int) * n);
    float2* dcen = (float2*)ws_alloc(c, sizeof(float2) * k);
    unsigned long long* acc = (unsigned long long*)ws_alloc(c, sizeof(unsigned long long) * (3 * k + 1));
    unsigned long long* n_re = acc + 3 * k;
    check(cudaMemcpyAsync(dcen, cen.data(), sizeof(float2) * k, cudaMemcpyHostToDevice, st), "H2D centroids");
    check(cudaMemsetAsync(acc, 0, sizeof(unsigned long long) * (3 * k + 1), st), "memset acc");
    k_km_init_labels<<<std::min<long long>((n + 255) / 256, 4096), 256, 0, st>>>(lab, n, k);
    counted(c, cudaGetLastError(), "init labels");
    const size_t smem = sizeof(float2) * k + sizeof(unsigned long long) * 3 * k;
    check(cudaFuncSetAttribute(k_km_assign, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "smem attr");
    const int blocks = std::max(1, std::min<int>((int)((n + 255) / 256), c->num_sms * 4));
    int it = 0;
    unsigned long long hre = 0;
    while (it <= max_iter) {
      ++it;
      check(cudaMemsetAsync(n_re, 0, sizeof(unsigned long long), st), "memset n_re");
      k_km_assign<<<blocks, 256, smem, st>>>(x, y, w, n, dcen, k, diam * 10.0f, std::ldexp(1.0, sp),
                                             std::ldexp(1.0, sw), lab, acc, n_re);
      counted(c, cudaGetLastError(), "k-means assign");
      k_km_update<<<1, 256, 0, st>>>(acc, k, sp, sw, dcen);
      counted(c, cudaGetLastError(), "k-means update");
      check(cudaMemcpyAsync(&hre, n_re, sizeof(hre), cudaMemcpyDeviceToHost, st), "D2H n_re");
      check(cudaStreamSynchronize(st), "sync k-means");
      if (hre == 0) break;
      if ((float)hre / (float)n < reassign_tol) break;
    }
    copy_out(c, labels_out, lab, sizeof(int) * n);
    if (centroids_out) copy_out(c, centroids_out, dcen, sizeof(float2) * k);
    check(cudaStreamSynchronize(st), "sync outputs");
    if (n_iter_out) *n_iter_out = it;
    return TPCF_OK;
  } catch (const Failure& f) {
    return fail(c, f);
  }
}

tpcf_status tpcf_bootstrap(tpcf_ctx* c, const double* patch_sums, int32_t n_task, int32_t n_patch, int32_t n_bin,
                           const int32_t* multiplicity, uint64_t seed, int32_t n_boot, double supersampling,
                           double* g_t, double* g_x, double* weights, double* cov_gt, double* cov_gx,
                           int32_t* mult_out) {
  if (!c || !patch_sums || n_task < 1 || n_patch < 1 || n_bin < 1 || n_bin > kMaxBins || n_boot < 2 || !g_t ||
      !g_x || !(supersampling > 0))
    return c ? (c->err = "invalid bootstrap arguments", TPCF_ERR_INVALID_ARG) : TPCF_ERR_INVALID_ARG;
  try {
    begin_call(c);
    cudaStream_t st = c->stream;
    const double* ps = stage(c, patch_sums, (int64_t)n_task * n_patch * 6 * n_bin);
    const int* mult;
    if (multiplicity) {
      mult = stage(c, (const int*)multiplicity, (int64_t)n_boot * n_patch);
    } else {
      // n_block_samples = int(n_blocks_total*supersampling_factor), src/tpcf.f90:1166
      const int n_draw = (int)((float)n_patch * (float)supersampling);
      if (n_draw < 1) throw Failure(TPCF_ERR_INVALID_ARG, "no draws per resample");
      int* m = (int*)ws_alloc(c, sizeof(int) * n_boot * n_patch);
      k_boot_mult<<<n_boot, 256, sizeof(int) * n_patch, st>>>(seed, n_patch, n_draw, m);
      counted(c, cudaGetLastError(), "bootstrap draws");
      mult = m;
    }
    const size_t D = (size_t)n_task * n_bin;
    double* dgt = (double*)ws_alloc(c, sizeof(double) * n_boot * D);
    double* dgx = (double*)ws_alloc(c, sizeof(double) * n_boot * D);
    double* dW = (double*)ws_alloc(c, sizeof(double) * n_boot * n_task);
    const long long tot = (long long)n_boot * n_task * (n_bin + 1);
    k_boot_resample<<<(unsigned)std::min<long long>((tot + 255) / 256, 65535), 256, 0, st>>>(
        ps, mult, n_boot, n_task, n_patch, n_bin, dgt, dgx, dW);
    counted(c, cudaGetLastError(), "bootstrap resample");
    copy_out(c, g_t, dgt, sizeof(double) * n_boot * D);
    copy_out(c, g_x, dgx, sizeof(double) * n_boot * D);
    if (weights) copy_out(c, weights, dW, sizeof(double) * n_boot * n_task);
    if (mult_out) copy_out(c, mult_out, mult, sizeof(int) * n_boot * n_patch);
    for (int q = 0; q < 2; ++q) {
      double* user = q == 0 ? cov_gt : cov_gx;
      if (!user) continue;
      double* dc = (double*)ws_alloc(c, sizeof(double) * D * D);
      dim3 grid((unsigned)((D + 127) / 128), (unsigned)D);
      k_cov<<<grid, 128, 0, st>>>(q == 0 ? dgt : dgx, n_boot, (int)D, dc);
      counted(c, cudaGetLastError(), "covariance");
      copy_out(c, user, dc, sizeof(double) * D * D);
    }
    check(cudaStreamSynchronize(st), "sync bootstrap");
    return TPCF_OK;
  } catch (const Failure& f) {
    return fail(c, f);
  }
}

}  // extern "C"
