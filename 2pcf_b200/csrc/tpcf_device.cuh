// tpcf_device.cuh -- device helpers shared by the pair and adjoint kernels:
// bulk-copy/mbarrier wrappers, the cell-row geometry of a work item, the
// canonical binning (FP32 with an FP64 guard band) and the conservative bin
// classification of a bounding box.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "tpcf_internal.cuh"

namespace tpcf {

// ------------------------------------------------- packed FP32 (f32x2) --
// sm_100 executes add/mul/fma on a pair of FP32 values per instruction (each
// half rounded exactly as the scalar operation).
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 dup2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 lo2(float4 v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(float4 v) { return make_float2(v.z, v.w); }
__device__ __forceinline__ float sum2(float2 v) { return v.x + v.y; }

// ------------------------------------------------------------ PTX helpers --
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
// 1-D bulk copy global -> shared, completion signalled on `bar`.  Both
// addresses 16-byte aligned, bytes a multiple of 16 (SrcRec is 32 bytes).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
// Orders this thread's generic-proxy shared-memory writes before later
// async-proxy (bulk copy) accesses of the same bytes.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: returns false after `limit` polls (default 2^22; each poll may
// suspend the thread for a hardware-defined interval), never spins forever.
constexpr uint32_t kWaitPolls = 1u << 22;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t limit = kWaitPolls) {
  for (uint32_t i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// ------------------------------------------------------------ geometry ------
__device__ __forceinline__ int clamp_floor(float v, int lo, int hi) {
  v = floorf(v);
  v = fminf(fmaxf(v, (float)lo), (float)hi);
  return (int)v;
}
// Rows of cells within R of the box.
__device__ __forceinline__ void row_range(const GridDesc& G, float4 box, float R, float m, int& cy0,
                                          int& cy1) {
  cy0 = clamp_floor((box.y - R - m - G.y0) * G.inv_cell, 0, G.ncy - 1);
  cy1 = clamp_floor((box.w + R + m - G.y0) * G.inv_cell, 0, G.ncy - 1);
}
// The contiguous run of sources of row cy whose cells lie within R of the box.
__device__ __forceinline__ int2 row_span(const GridDesc& G, float4 box, float R, float m, int cy) {
  const float ylo = G.y0 + (float)cy * G.cell - m;
  const float yhi = G.y0 + (float)(cy + 1) * G.cell + m;
  const float dyr = fmaxf(0.f, fmaxf(ylo - box.w, box.y - yhi));
  if (dyr > R) return make_int2(0, 0);
  const float rx = sqrtf(fmaxf(R * R - dyr * dyr, 0.f)) + m;
  const int cx0 = clamp_floor((box.x - rx - G.x0) * G.inv_cell, 0, G.ncx - 1);
  const int cx1 = clamp_floor((box.z + rx - G.x0) * G.inv_cell, 0, G.ncx - 1);
  const int base = cy * G.ncx;
  return make_int2(G.cell_start[base + cx0], G.cell_start[base + cx1 + 1]);
}

// Sort key of work item i (items are built in task, then lens-group order,
// and lens groups follow (patch, Hilbert) order): the item's cost in bands of
// 2^(1/8) (about 9%) on top, the item index below.  Sorted descending, the
// costliest items start first (load balance), and inside one band the items
// run in task and space order, so that the warps resident at one time read
// the same rows of one source grid and those stay in L2.
__device__ __forceinline__ unsigned long long item_key(unsigned long long cost, int i) {
  const unsigned band = (unsigned)(__log2f((float)cost) * 8.f);
  return ((unsigned long long)band << 32) | (unsigned)i;
}

// Position of cell (qx, qy) of a 2^bits x 2^bits grid (bits <= 16) along the
// Hilbert curve: the quadrant digit of each level from the top down, with
// the cell's coordinates inside its quadrant turned into the orientation of
// that quadrant's sub-curve.  Runs of consecutive positions are compact
// (no jumps across the grid, unlike Morton order), so groups of 32
// consecutive objects get small bounding boxes.
__device__ __forceinline__ unsigned hilbert_index(unsigned qx, unsigned qy, int bits) {
  unsigned d = 0;
  for (int b = bits - 1; b >= 0; --b) {
    const unsigned s = 1u << b, m = s - 1u;
    const unsigned rx = (qx >> b) & 1u, ry = (qy >> b) & 1u;
    d += s * s * ((3u * rx) ^ ry);
    unsigned x = qx & m, y = qy & m;
    if (ry == 0u) {
      if (rx == 1u) {
        x = m - x;
        y = m - y;
      }
      const unsigned t = x;
      x = y;
      y = t;
    }
    qx = x;
    qy = y;
  }
  return d;
}

// ------------------------------------------------------------ binning -------
// Canonical FP64 bin of the pair (rare path: pairs inside the guard band).
static __device__ __noinline__ int slow_bin(float lx, float ly, float sx, float sy, const double* e2, int nb) {
  const double dx = __dsub_rn((double)lx, (double)sx);
  const double dy = __dsub_rn((double)ly, (double)sy);
  const double d2 = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
  if (!(d2 >= e2[0]) || d2 > e2[nb]) return -1;
  if (d2 == e2[nb]) return nb - 1;
  int lo = 0, hi = nb;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (d2 >= e2[mid]) lo = mid; else hi = mid;
  }
  return lo;
}

struct BinCtx {
  float A, B, eps, one_m_eps;
  float eps_rel;     // relative guard on d2 around one FP32 edge (register paths)
  float lo_g, hi_g;  // generic: fast reject bounds e2f[0]*(1-eps), e2f[nb]*(1+eps)
  int nb;
  const double* e2s;
  const float* e2f;
};

template <bool LOGB>
__device__ __forceinline__ int pair_bin(float d2, float lx, float ly, float sx, float sy, const BinCtx& C) {
  if (LOGB) {
    const float t = fmaf(__log2f(d2), C.A, C.B);
    const float tf = floorf(t);
    const float fr = t - tf;
    int b = __float2int_rz(tf);
    if (fr < C.eps || fr > C.one_m_eps) b = slow_bin(lx, ly, sx, sy, C.e2s, C.nb);
    return b;
  } else {
    if (d2 < C.lo_g || d2 > C.hi_g) return -1;
    int lo = 0, hi = C.nb;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (d2 >= C.e2f[mid]) lo = mid; else hi = mid;
    }
    const float el = C.e2f[lo], eh = C.e2f[lo + 1];
    if (d2 <= el * (1.f + C.eps) || d2 >= eh * (1.f - C.eps)) lo = slow_bin(lx, ly, sx, sy, C.e2s, C.nb);
    return lo;
  }
}

// Largest i in [0, nb] with e2f[i] <= v, or -1 (generic spacings).
__device__ __forceinline__ int edge_index_f32(float v, const float* e2f, int nb) {
  if (v < e2f[0]) return -1;
  int lo = 0, hi = nb + 1;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (v >= e2f[mid]) lo = mid; else hi = mid;
  }
  return lo;
}

template <bool LOGB, bool HAS_Z, bool ZREG = false>
__device__ __forceinline__ int classify(float lx, float ly, const float4 box, const BinCtx& C, int& blo) {
  const float dxl = fmaxf(fmaxf(box.x - lx, lx - box.z), 0.f);
  const float dyl = fmaxf(fmaxf(box.y - ly, ly - box.w), 0.f);
  const float dxh = fmaxf(lx - box.x, box.z - lx);
  const float dyh = fmaxf(ly - box.y, box.w - ly);
  const float dmin2 = fmaf(dyl, dyl, dxl * dxl);
  const float dmax2 = fmaf(dyh, dyh, dxh * dxh);
  int b0, b1;
  if (LOGB) {
    b0 = __float2int_rd(fmaf(__log2f(dmin2), C.A, C.B) - C.eps);
    b1 = __float2int_rd(fmaf(__log2f(dmax2), C.A, C.B) + C.eps);
  } else {
    b0 = edge_index_f32(dmin2 * (1.f - C.eps), C.e2f, C.nb);
    b1 = edge_index_f32(dmax2 * (1.f + C.eps), C.e2f, C.nb);
  }
  if (b1 < 0 || b0 >= C.nb) return 0;
  b0 = max(b0, -1);  // every bin below 0 or from nb up is dropped alike
  b1 = min(b1, C.nb);
  blo = b0;
  if (HAS_Z && !ZREG) return 3;  // z cut: per-pair path unless the register paths apply it
  if (b0 == b1) return 1;
  if (b1 == b0 + 1) return 2;
  return 3;
}

// Class of a box for the planar pair kernel: 0 when no pair can be in range,
// else 1 + the number of bin edges its distance range [dmin, dmax] may cross
// (guard band eps on both ends) for up to two edges, 4 beyond (per-pair
// binning).  blo = the lowest bin, -1 when the range starts below the first
// edge; bins below 0 and from nb up are all dropped, so the range is clamped
// to [-1, nb] first and every edge blo + 1 + e it names is in [0, nb].
template <bool LOGB>
__device__ __forceinline__ int classify_edges(float lx, float ly, const float4 box, const BinCtx& C, int& blo) {
  const float dxl = fmaxf(fmaxf(box.x - lx, lx - box.z), 0.f);
  const float dyl = fmaxf(fmaxf(box.y - ly, ly - box.w), 0.f);
  const float dxh = fmaxf(lx - box.x, box.z - lx);
  const float dyh = fmaxf(ly - box.y, box.w - ly);
  const float dmin2 = fmaf(dyl, dyl, dxl * dxl);
  const float dmax2 = fmaf(dyh, dyh, dxh * dxh);
  int b0, b1;
  if (LOGB) {
    b0 = __float2int_rd(fmaf(__log2f(dmin2), C.A, C.B) - C.eps);
    b1 = __float2int_rd(fmaf(__log2f(dmax2), C.A, C.B) + C.eps);
  } else {
    b0 = edge_index_f32(dmin2 * (1.f - C.eps), C.e2f, C.nb);
    b1 = edge_index_f32(dmax2 * (1.f + C.eps), C.e2f, C.nb);
  }
  if (b1 < 0 || b0 >= C.nb) return 0;
  b0 = max(b0, -1);
  b1 = min(b1, C.nb);
  blo = b0;
  const int e = b1 - b0;
  return e <= 2 ? 1 + e : 4;
}

}  // namespace tpcf
