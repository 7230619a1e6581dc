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
#include <cub/cub.cuh>

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
                            double sw_scale, int* labels, unsigned long long* acc, unsigned long long* n_re,
                            const int* state) {
  if (state[0]) return;  // converged in an earlier pass of this batch
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
    // the correctly rounded sqrt (as the reference) only where it can win:
    // q > best^2 (1 + 1e-5) gives sqrt(q) > best whatever the roundings
    float tsq = __fmul_rn(min_init, min_init) * 1.00001f;
    for (int j = 0; j < k; ++j) {
      const float dx = __fsub_rn(xi, c[j].x), dy = __fsub_rn(yi, c[j].y);
      const float q = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
      if (q > tsq) continue;
      const float d = __fsqrt_rn(q);
      if (d < best) {
        best = d;
        bi = j;
        tsq = __fmul_rn(best, best) * 1.00001f;
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

// Centroids from the fixed-point sums (two's-complement int64), then clear
// them; then the stopping rule of src/kmeans.f90:118-137 on the device:
// state = {done, passes}; the run stops after a pass with no reassignment, a
// reassigned fraction below tol, or max_iter + 1 passes.  Without state only
// the centroids are updated.
__global__ void k_km_update(unsigned long long* acc, int k, int sp, int sw, float2* cen, unsigned long long* n_re,
                            long long n, float tol, int max_iter, int* state) {
  if (state && state[0]) return;
  for (int j = threadIdx.x; j < k; j += blockDim.x) {
    const double W = ldexp((double)(long long)acc[3 * j + 2], -sw);
    const double cx = ldexp((double)(long long)acc[3 * j + 0], -sp) / W;
    const double cy = ldexp((double)(long long)acc[3 * j + 1], -sp) / W;
    cen[j] = make_float2((float)cx, (float)cy);
    acc[3 * j + 0] = acc[3 * j + 1] = acc[3 * j + 2] = 0ull;
  }
  if (state && threadIdx.x == 0) {
    const int it = ++state[1];
    const unsigned long long re = *n_re;
    *n_re = 0ull;
    if (re == 0ull || (float)re / (float)n < tol || it > max_iter) state[0] = 1;
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


// --------------------------------------------------- equal-weight k-means --
// partition_data with equal_size (src/kmeans.f90:12-262).  From pass 2 on the
// distance to cluster j is scaled by 1 + (W_j / W_mean - 1) * s (:171-177) and
// each point records its second-nearest cluster with the ratio of the two
// distances (:179-191).  The reference moves a point's weight between clusters
// as soon as the point is reassigned (:193-200), so later points see the
// updated weights; here the points are swept in order in chunks of C: the
// points of one chunk see the weights as the previous chunks left them.  One
// resident block runs the sweep (weights in shared memory, integer fixed
// point, so the sweep is exact and deterministic).
__global__ void __launch_bounds__(1024) k_km_sweep_eq(const float* __restrict__ x, const float* __restrict__ y,
                                                      const float* __restrict__ w, long long n, int chunk,
                                                      const float2* __restrict__ cen, long long* wfix, int k,
                                                      float min_init, float wmean, float scaling, int sw,
                                                      int penalty, int candidates, int* labels, int* cand,
                                                      float* memb, unsigned long long* n_re) {
  extern __shared__ unsigned char sm[];
  float2* c = reinterpret_cast<float2*>(sm);
  long long* W = reinterpret_cast<long long*>(c + k);
  float* f = reinterpret_cast<float*>(W + k);
  for (int j = threadIdx.x; j < k; j += blockDim.x) {
    c[j] = cen[j];
    W[j] = wfix[j];
  }
  unsigned long long re = 0;
  // this thread's point of the next chunk, loaded while the current one is
  // assigned (a point's label is written only by its own thread)
  float nx = 0.f, ny = 0.f, nw = 0.f;
  int nl = -1;
  const bool lane_in = (int)threadIdx.x < chunk;
  if (lane_in && (long long)threadIdx.x < n) {
    nx = x[threadIdx.x];
    ny = y[threadIdx.x];
    nw = w[threadIdx.x];
    nl = labels[threadIdx.x];
  }
  for (long long base = 0; base < n; base += chunk) {
    const float xi = nx, yi = ny, wi = nw;
    const int old = nl;
    const long long inext = base + chunk + threadIdx.x;
    if (lane_in && inext < n) {
      nx = x[inext];
      ny = y[inext];
      nw = w[inext];
      nl = labels[inext];
    }
    __syncthreads();
    for (int j = threadIdx.x; j < k; j += blockDim.x) {
      // 1 + (W_j / W_mean - 1) * s in FP32 as written (kmeans.f90:174)
      const float Wj = (float)ldexp((double)W[j], -sw);
      f[j] = penalty ? __fadd_rn(1.0f, __fmul_rn(__fsub_rn(__fdiv_rn(Wj, wmean), 1.0f), scaling)) : 1.0f;
    }
    __syncthreads();
    const long long i = base + threadIdx.x;
    if (threadIdx.x < chunk && i < n) {
      float best = min_init, cm = 0.f;
      int bi = -1, ci = -1;
      // A cluster can change the outcome only if its scaled distance d is
      // below T = max(best, cm * best) (candidates) or best.  The exact d
      // (correctly rounded sqrt, as the reference) is formed only when
      // f^2 (dx^2 + dy^2) <= T^2 (1 + 1e-5): outside that margin d > T for
      // certain, whatever the FP32 roundings, so the labels do not change.
      float tsq = __fmul_rn(min_init, min_init) * 1.00001f;
      for (int j = 0; j < k; ++j) {
        const float dx = __fsub_rn(xi, c[j].x), dy = __fsub_rn(yi, c[j].y);
        const float q = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
        const float fj = f[j];
        if (fj > 0.f && fj * fj * q > tsq) continue;  // (f <= 0 gives d <= 0: always formed)
        const float d = __fmul_rn(fj, __fsqrt_rn(q));
        if (candidates && d > 0.0f) {
          if (d < best) {
            cm = __fdiv_rn(best, d);
            ci = bi;
            best = d;
            bi = j;
          } else if (d < __fmul_rn(cm, best)) {
            cm = __fdiv_rn(d, best);
            ci = j;
          } else {
            continue;
          }
        } else if (d < best) {
          best = d;
          bi = j;
        } else {
          continue;
        }
        const float t = candidates ? fmaxf(best, __fmul_rn(cm, best)) : best;
        tsq = __fmul_rn(t, t) * 1.00001f;
      }
      if (candidates) {
        cand[i] = ci;
        memb[i] = cm;
      }
      if (bi != old) {
        labels[i] = bi;
        ++re;
        const long long wf = __double2ll_rn(ldexp((double)wi, sw));
        if (old >= 0) atomicAdd((unsigned long long*)&W[old], (unsigned long long)(-wf));
        if (bi >= 0) atomicAdd((unsigned long long*)&W[bi], (unsigned long long)wf);
      }
    }
  }
  __syncthreads();
  for (int j = threadIdx.x; j < k; j += blockDim.x) wfix[j] = W[j];
  for (int o = 16; o; o >>= 1) re += __shfl_xor_sync(0xffffffffu, re, o);
  if ((threadIdx.x & 31) == 0 && re) atomicAdd(n_re, re);
}

// Cluster weights from the sums (the sums stay for the centroid update).
__global__ void k_km_weights(unsigned long long* acc, int k, long long* wfix) {
  for (int j = threadIdx.x; j < k; j += blockDim.x) {
    wfix[j] = (long long)acc[3 * j + 2];
    acc[3 * j + 0] = acc[3 * j + 1] = acc[3 * j + 2] = 0ull;
  }
}

// Fixed-point sums of x w, y w and w per cluster for the centroids.
__global__ void k_km_sums(const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ w,
                          const int* __restrict__ labels, long long n, int k, double sp_scale, double sw_scale,
                          unsigned long long* acc) {
  extern __shared__ unsigned long long a[];
  for (int j = threadIdx.x; j < 3 * k; j += blockDim.x) a[j] = 0ull;
  __syncthreads();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int bi = labels[i];
    if (bi < 0) continue;
    const double wi = (double)w[i];
    atomicAdd(&a[3 * bi + 0], (unsigned long long)__double2ll_rn((double)x[i] * wi * sp_scale));
    atomicAdd(&a[3 * bi + 1], (unsigned long long)__double2ll_rn((double)y[i] * wi * sp_scale));
    atomicAdd(&a[3 * bi + 2], (unsigned long long)__double2ll_rn(wi * sw_scale));
  }
  __syncthreads();
  for (int j = threadIdx.x; j < 3 * k; j += blockDim.x)
    if (a[j]) atomicAdd(&acc[j], a[j]);
}



// Random labels for kmeans_compute_random_initial_centroids (kmeans.f90:78):
// Philox counter (i/4, 0xC4, 0x4B4D, 0), word i%4, label by multiply-shift.
__global__ void k_km_random_labels(int* labels, long long n, int k, unsigned long long seed) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < (n + 3) / 4;
       q += (long long)gridDim.x * blockDim.x) {
    uint32_t c[4] = {(uint32_t)q, 0xC4u, 0x4B4Du, 0u};
    philox4x32(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    for (int u = 0; u < 4; ++u) {
      const long long i = 4 * q + u;
      if (i < n) labels[i] = (int)(((unsigned long long)c[u] * (unsigned)k) >> 32);
    }
  }
}

// Post-processing rebalance (postprocess_weights, kmeans.f90:221-262), one
// cluster cj per step, over the points in candidate order (rank r):
// eligible = member of cj whose candidate is a cluster not yet processed.
__global__ void k_pp_flags(const int* __restrict__ order, const int* __restrict__ labels,
                           const int* __restrict__ cand, const int* __restrict__ processed,
                           const float* __restrict__ w, long long n, int cj, double sw_scale, long long* val) {
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x) {
    const int p = order[r];
    const int d = cand[p];
    const bool e = labels[p] == cj && d >= 0 && !processed[d];
    val[r] = e ? __double2ll_rn((double)w[p] * sw_scale) : 0ll;
  }
}
// First eligible rank at which cluster cj's weight, less the weights moved up
// to and including it, is at or below the threshold (all eligible if none).
__global__ void k_pp_stop(const long long* __restrict__ S, const long long* __restrict__ val,
                          const long long* __restrict__ wfix, int cj, long long thr, long long n, long long* rstop) {
  const long long W = wfix[cj];
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x)
    if (val[r] != 0 && W - S[r] <= thr) atomicMin((unsigned long long*)rstop, (unsigned long long)r);
}
__global__ void k_pp_apply(const int* __restrict__ order, const long long* __restrict__ val,
                           const long long* __restrict__ S, const int* __restrict__ cand, const long long* rstop,
                           long long n, int cj, int* labels, long long* wfix) {
  const long long last = min(*rstop, n - 1);
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r <= last; r += (long long)gridDim.x * blockDim.x) {
    if (val[r] == 0) continue;
    const int p = order[r];
    labels[p] = cand[p];
    atomicAdd((unsigned long long*)&wfix[cand[p]], (unsigned long long)val[r]);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd((unsigned long long*)&wfix[cj], (unsigned long long)(-S[last]));
}

}  // namespace

namespace {
__global__ void k_iota(int* v, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    v[i] = (int)i;
}
cudaError_t launch_iota(int* v, long long n, cudaStream_t st) {
  k_iota<<<(unsigned)std::min<long long>((n + 255) / 256, 4096), 256, 0, st>>>(v, n);
  return cudaGetLastError();
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
    Phase ph("tpcf: k-means");
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
    unsigned long long* acc = (unsigned long long*)ws_alloc(c, sizeof(unsigned long long) * (3 * k + 2));
    unsigned long long* n_re = acc + 3 * k;
    int* state = reinterpret_cast<int*>(acc + 3 * k + 1);  // {done, passes}
    check(cudaMemcpyAsync(dcen, cen.data(), sizeof(float2) * k, cudaMemcpyHostToDevice, st), "H2D centroids");
    check(cudaMemsetAsync(acc, 0, sizeof(unsigned long long) * (3 * k + 2), st), "memset acc");
    k_km_init_labels<<<std::min<long long>((n + 255) / 256, 4096), 256, 0, st>>>(lab, n, k);
    counted(c, cudaGetLastError(), "init labels");
    const size_t smem = sizeof(float2) * k + sizeof(unsigned long long) * 3 * k;
    check(cudaFuncSetAttribute(k_km_assign, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "smem attr");
    const int blocks = std::max(1, std::min<int>((int)((n + 255) / 256), c->num_sms * 4));
    // Lloyd passes in batches of kPassBatch with the stopping rule evaluated on
    // the device (k_km_update): one host synchronisation per batch; passes
    // after convergence return at once.
    constexpr int kPassBatch = 8;
    int hstate[2] = {0, 0};
    for (int done_passes = 0; !hstate[0] && done_passes <= max_iter; done_passes += kPassBatch) {
      for (int b = 0; b < kPassBatch; ++b) {
        k_km_assign<<<blocks, 256, smem, st>>>(x, y, w, n, dcen, k, diam * 10.0f, std::ldexp(1.0, sp),
                                               std::ldexp(1.0, sw), lab, acc, n_re, state);
        counted(c, cudaGetLastError(), "k-means assign");
        k_km_update<<<1, 256, 0, st>>>(acc, k, sp, sw, dcen, n_re, n, reassign_tol, max_iter, state);
        counted(c, cudaGetLastError(), "k-means update");
      }
      check(cudaMemcpyAsync(hstate, state, sizeof(hstate), cudaMemcpyDeviceToHost, st), "D2H k-means state");
      check(cudaStreamSynchronize(st), "sync k-means");
    }
    const int it = hstate[1];
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
    Phase ph_nvtx("tpcf: bootstrap");
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

tpcf_status tpcf_kmeans_equal(tpcf_ctx* c, const float* x, const float* y, const float* w, int64_t n, int32_t k,
                              int32_t max_iter, float reassign_tol, float weight_scaling, float weight_tol,
                              int32_t random_init, uint64_t seed, int32_t* labels_out, float* centroids_out,
                              int32_t* n_iter_out, float* max_dev_out) {
  if (!c || !labels_out || n < 1 || k < 2 || k > kMaxK || max_iter < 0 || !x || !y || !w || n > (1ll << 31) - 2 ||
      !(weight_scaling >= 0) || !(weight_tol >= 0) || (random_init && n < k))
    return c ? (c->err = "invalid k-means arguments", TPCF_ERR_INVALID_ARG) : TPCF_ERR_INVALID_ARG;
  try {
    Phase ph_nvtx("tpcf: equal-weight k-means");
    begin_call(c);
    cudaStream_t st = c->stream;
    x = stage(c, x, n);
    y = stage(c, y, n);
    w = stage(c, w, n);
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
    std::vector<float> cen(2 * k);
    int* lab = (int*)ws_alloc(c, sizeof(int) * n);
    if (random_init) {
      // k distinct points drawn by Philox counter (t/4, 0xC3, 0x4B4D, 0), word t%4,
      // index by multiply-shift, repeats redrawn (kmeans.f90:68-76)
      std::vector<long long> chosen;
      std::vector<float> hx(1), hy(1);
      for (uint32_t t = 0; (int)chosen.size() < k; ++t) {
        uint32_t ctr[4] = {t / 4, 0xC3u, 0x4B4Du, 0u};
        philox4x32_host(ctr, (uint32_t)seed, (uint32_t)(seed >> 32));
        const long long idx = (long long)(((uint64_t)ctr[t % 4] * (uint64_t)n) >> 32);
        if (std::find(chosen.begin(), chosen.end(), idx) == chosen.end()) chosen.push_back(idx);
        if (t > 64u * (uint32_t)k + 1024u) throw Failure(TPCF_ERR_INVALID_ARG, "too few distinct points");
      }
      for (int j = 0; j < k; ++j) {
        check(cudaMemcpyAsync(&cen[2 * j], x + chosen[j], sizeof(float), cudaMemcpyDeviceToHost, st), "D2H point");
        check(cudaMemcpyAsync(&cen[2 * j + 1], y + chosen[j], sizeof(float), cudaMemcpyDeviceToHost, st), "D2H point");
      }
      check(cudaStreamSynchronize(st), "sync points");
      k_km_random_labels<<<std::min<long long>((n / 4 + 256) / 256, 4096), 256, 0, st>>>(lab, n, k, seed);
      counted(c, cudaGetLastError(), "random labels");
    } else {
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
      k_km_init_labels<<<std::min<long long>((n + 255) / 256, 4096), 256, 0, st>>>(lab, n, k);
      counted(c, cudaGetLastError(), "init labels");
    }
    const float diam = sqrtf((xmx - xmn) * (xmx - xmn) + (ymx - ymn) * (ymx - ymn));
    const double amax = std::max(std::max(std::fabs((double)xmn), std::fabs((double)xmx)),
                                 std::max(std::fabs((double)ymn), std::fabs((double)ymx)));
    const double wmax = hb[6];
    const int sp = fixed_scale(n, amax * wmax), sw = fixed_scale(n, wmax);
    float2* dcen = (float2*)ws_alloc(c, sizeof(float2) * k);
    unsigned long long* acc = (unsigned long long*)ws_alloc(c, sizeof(unsigned long long) * (3 * k + 1));
    unsigned long long* n_re = acc + 3 * k;
    long long* wfix = (long long*)ws_alloc(c, sizeof(long long) * k);
    int* cand = (int*)ws_alloc(c, sizeof(int) * n);
    float* memb = (float*)ws_alloc(c, sizeof(float) * n);
    check(cudaMemcpyAsync(dcen, cen.data(), sizeof(float2) * k, cudaMemcpyHostToDevice, st), "H2D centroids");
    check(cudaMemsetAsync(acc, 0, sizeof(unsigned long long) * (3 * k + 1), st), "memset acc");
    check(cudaMemsetAsync(cand, 0xff, sizeof(int) * n, st), "memset cand");
    check(cudaMemsetAsync(memb, 0, sizeof(float) * n, st), "memset memb");
    const size_t ssm = sizeof(unsigned long long) * 3 * k;
    const int sblocks = std::max(1, std::min<int>((int)((n + 255) / 256), c->num_sms * 4));
    // initial cluster weights from the initial labels (kmeans.f90:79-81, :108-110)
    k_km_sums<<<sblocks, 256, ssm, st>>>(x, y, w, lab, n, k, std::ldexp(1.0, sp), std::ldexp(1.0, sw), acc);
    counted(c, cudaGetLastError(), "k-means sums");
    k_km_weights<<<1, 256, 0, st>>>(acc, k, wfix);
    counted(c, cudaGetLastError(), "k-means weights");
    std::vector<long long> hw(k);
    check(cudaMemcpyAsync(hw.data(), wfix, sizeof(long long) * k, cudaMemcpyDeviceToHost, st), "D2H weights");
    check(cudaStreamSynchronize(st), "sync weights");
    long long tot = 0;
    for (long long v : hw) tot += v;
    const float wmean = (float)(std::ldexp((double)tot, -sw) / k);  // sum(weights)/k (kmeans.f90:61)
    // sweep chunk: at most 1/2048 of the points, 32..1024
    const int chunk = (int)std::max<long long>(32, std::min<long long>(1024, n / 2048));
    const size_t smem = sizeof(float2) * k + sizeof(long long) * k + sizeof(float) * k;
    check(cudaFuncSetAttribute(k_km_sweep_eq, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "smem attr");
    check(cudaFuncSetAttribute(k_km_sums, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ssm), "smem attr");
    int it = 0;
    unsigned long long hre = 0;
    while (it <= max_iter) {
      ++it;
      check(cudaMemsetAsync(n_re, 0, sizeof(unsigned long long), st), "memset n_re");
      k_km_sweep_eq<<<1, 1024, smem, st>>>(x, y, w, n, chunk, dcen, wfix, k, diam * 10.0f, wmean, weight_scaling,
                                           sw, it > 1 && weight_scaling > 0.f, it > 1, lab, cand, memb, n_re);
      counted(c, cudaGetLastError(), "k-means sweep");
      k_km_sums<<<sblocks, 256, ssm, st>>>(x, y, w, lab, n, k, std::ldexp(1.0, sp), std::ldexp(1.0, sw), acc);
      counted(c, cudaGetLastError(), "k-means sums");
      k_km_update<<<1, 256, 0, st>>>(acc, k, sp, sw, dcen, nullptr, n, 0.f, 0, nullptr);
      counted(c, cudaGetLastError(), "k-means update");
      check(cudaMemcpyAsync(&hre, n_re, sizeof(hre), cudaMemcpyDeviceToHost, st), "D2H n_re");
      check(cudaMemcpyAsync(hw.data(), wfix, sizeof(long long) * k, cudaMemcpyDeviceToHost, st), "D2H weights");
      check(cudaStreamSynchronize(st), "sync k-means");
      if (hre == 0) break;
      if ((float)hre / (float)n < reassign_tol) break;
    }
    auto max_dev = [&]() {
      long long mx = hw[0], mn = hw[0];
      for (long long v : hw) { mx = std::max(mx, v); mn = std::min(mn, v); }
      return (float)(std::ldexp((double)(mx - mn), -sw) / (double)wmean);
    };
    float dev = max_dev();
    if (centroids_out) copy_out(c, centroids_out, dcen, sizeof(float2) * k);  // before the rebalance, as the reference
    if (dev > weight_tol && it > 1) {
      // clusters by weight, heaviest first; points by candidate ratio, ascending
      std::vector<int> corder(k);
      for (int j = 0; j < k; ++j) corder[j] = j;
      std::stable_sort(corder.begin(), corder.end(), [&](int a, int b) { return hw[a] > hw[b]; });
      int* idx0 = (int*)ws_alloc(c, sizeof(int) * n);
      int* order = (int*)ws_alloc(c, sizeof(int) * n);
      float* mk = (float*)ws_alloc(c, sizeof(float) * n);
      counted(c, launch_iota(idx0, n, st), "iota");
      size_t tb = 0;
      check(cub::DeviceRadixSort::SortPairs(nullptr, tb, memb, mk, idx0, order, (int)n, 0, 32, st), "sort size");
      void* tmp = ws_alloc(c, tb);
      check(cub::DeviceRadixSort::SortPairs(tmp, tb, memb, mk, idx0, order, (int)n, 0, 32, st), "sort candidates");
      int* processed = (int*)ws_alloc(c, sizeof(int) * k);
      check(cudaMemsetAsync(processed, 0, sizeof(int) * k, st), "memset processed");
      long long* val = (long long*)ws_alloc(c, sizeof(long long) * n);
      long long* S = (long long*)ws_alloc(c, sizeof(long long) * n);
      long long* rstop = (long long*)ws_alloc(c, sizeof(long long));
      size_t tb2 = 0;
      check(cub::DeviceScan::InclusiveSum(nullptr, tb2, val, S, (int)n, st), "scan size");
      void* tmp2 = ws_alloc(c, tb2);
      const float thr_f = wmean * (1.0f + weight_tol);
      const long long thr = std::llrint(std::ldexp((double)thr_f, sw));
      const unsigned gb = (unsigned)std::min<long long>((n + 255) / 256, c->num_sms * 8);
      const int one = 1;
      for (int j = 0; j < k; ++j) {
        const int cj = corder[j];
        check(cudaMemcpyAsync(processed + cj, &one, sizeof(int), cudaMemcpyHostToDevice, st), "processed");
        k_pp_flags<<<gb, 256, 0, st>>>(order, lab, cand, processed, w, n, cj, std::ldexp(1.0, sw), val);
        counted(c, cudaGetLastError(), "rebalance flags");
        check(cub::DeviceScan::InclusiveSum(tmp2, tb2, val, S, (int)n, st), "scan");
        const long long nn = n;
        check(cudaMemcpyAsync(rstop, &nn, sizeof(long long), cudaMemcpyHostToDevice, st), "rstop");
        k_pp_stop<<<gb, 256, 0, st>>>(S, val, wfix, cj, thr, n, rstop);
        counted(c, cudaGetLastError(), "rebalance stop");
        k_pp_apply<<<gb, 256, 0, st>>>(order, val, S, cand, rstop, n, cj, lab, wfix);
        counted(c, cudaGetLastError(), "rebalance apply");
        check(cudaStreamSynchronize(st), "sync rebalance");  // host staging (one, nn) reused next step
      }
      check(cudaMemcpyAsync(hw.data(), wfix, sizeof(long long) * k, cudaMemcpyDeviceToHost, st), "D2H weights");
      check(cudaStreamSynchronize(st), "sync weights");
      dev = max_dev();
    }
    copy_out(c, labels_out, lab, sizeof(int) * n);
    check(cudaStreamSynchronize(st), "sync outputs");
    if (n_iter_out) *n_iter_out = it;
    if (max_dev_out) *max_dev_out = dev;
    return TPCF_OK;
  } catch (const Failure& f) {
    return fail(c, f);
  }
}

}  // extern "C"
