// adjoint.cu -- gradients of a scalar loss of the shear-scalar correlation
// function with respect to the per-object inputs (no counterpart in the
// reference, which has no gradients).
//
// With xi_t,b = G_b/K_b, xi_x,b = X_b/K_b (src/tpcf.f90:369-376) and
// lambda_b = dL/dxi_t,b, lambdax_b = dL/dxi_x,b:
//   mu_b = lambda_b/K_b, mux_b = lambdax_b/K_b,
//   nu_b = (lambda_b xi_t,b + lambdax_b xi_x,b)/K_b   (0 where K_b <= 0)
// Lens side (from the forward's raw per-lens sums, no pair pass):
//   dL/dval_i = w_i sum_b (mu_b Rt_ib + mux_b Rx_ib)
//   dL/dw_i   = sum_b (val_i (mu_b Rt_ib + mux_b Rx_ib) - nu_b RK_ib)
// Source side (one pass over all pairs, sources as owners): with
//   A1 = sum_i mu c2 v_i w_i, A2 = sum_i mu s2 v_i w_i, B1, B2 likewise with mux,
//   N = sum_i nu w_i  (bin b = b(i,j), c2 = cos 2phi, s2 = sin 2phi)
//   dL/de1_j = w_j (-A1 + B2), dL/de2_j = w_j (-A2 - B1),
//   dL/dw_j  = -e1 A1 - e2 A2 + e1 B2 - e2 B1 - (1 + m_j) N,  dL/dm_j = -w_j N.
// Each pair is binned exactly as in the forward pass (same canonical rule,
// same classification of 32-object sub-chunks), so the gradient is the one of
// the binned estimator.  The pass mirrors k_pairs with the roles swapped:
// lenses are sorted into the cell grid and streamed through shared memory,
// each thread owns one source and accumulates five sums in registers (FP32
// per tile, FP64 across tiles); there is no histogram.  As in k_pairs, the
// one-bin and one-edge sub-chunk paths run on packed FP32 instructions over
// lens tiles rewritten in place into pair-interleaved LensPair blocks.

#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "tpcf_b200.h"
#include "tpcf_ctx.h"
#include "tpcf_device.cuh"
#include "tpcf_internal.cuh"
#include "tpcf_kernels.h"

namespace {

using namespace tpcf;

constexpr int BT = 128;
// Blocks per SM the adjoint kernel is compiled for.  Declaring it gives the
// compiler a register budget (up to 85 per thread) in place of a spilling
// 56-register schedule; 6 blocks of 128 threads still fit every SM.
constexpr int kAdjMinBlocks = 6;

// One (lens catalogue, source catalogue) task of a batched backward pass.
struct AdjTask {
  GridDesc grid;            // grid over the task's lenses
  const SrcRec* lens;       // lens grid records: a = {x, y, val*w, w}, b = {z, 0, 0, 0}
  const float4* s0;         // the task's sources, sorted: {x, y, e1, e2}
  const float4* s1;         // {w, 1+m, z, 0}
  const float4* gbox;       // source group boxes
  int n_src;                // valid sources
  int pad;
  double* dsum;             // [5][n_src] FP64 sums D1, D2, D3, D4, DN of this task (sorted order)
};

struct AdjParams {
  const AdjTask* tasks;
  const int2* items;        // (task, source group) in processing order
  int n_items;
  int nb;
  int* queue_head;
  unsigned* err;
  const double* e2;
  const float* e2f;
  const float4* coef;       // [n_task][nb] {mu, mux, nu, 0}
  float R, margin, binA, binB, eps;
};

struct AdjSmem {
  size_t tiles, e2s, e2f, coef, span0, span1, tpref, subbox, subw, mbar, misc, total;
};
__host__ __device__ inline size_t au(size_t v, size_t a) { return (v + a - 1) / a * a; }
__host__ __device__ inline AdjSmem adj_smem(int nb) {
  AdjSmem s;
  size_t o = 0;
  s.tiles = o; o += 2 * kTile * sizeof(SrcRec);
  s.e2s = o; o += (size_t)(nb + 1) * sizeof(double);
  s.e2f = o; o += (size_t)(nb + 1) * sizeof(float);
  o = au(o, 16);
  s.coef = o; o += (size_t)(nb + 1) * sizeof(float4);
  s.span0 = o; o += kMaxRows * sizeof(int);
  s.span1 = o; o += kMaxRows * sizeof(int);
  s.tpref = o; o += (kMaxRows + 1) * sizeof(int);
  o = au(o, 16);
  s.subbox = o; o += (kTile / 32) * sizeof(float4);
  s.subw = o; o += (kTile / 32) * sizeof(float);
  o = au(o, 8);
  s.mbar = o; o += 2 * sizeof(uint64_t);
  s.misc = o; o += 16;
  s.total = au(o, 128);
  return s;
}

struct Acc {
  float a1, a2, b1, b2, n;
};

// The bin-independent part of a pair's adjoint terms: with F = val_A w_A / d^2
// (vw = val_A w_A), S1 += F (dx^2 - dy^2), S2 += F dx dy, SN += w_A.  Within
// a run of pairs of one bin the bin's coefficients multiply these sums once:
// a1 = k.x S1, a2 = 2 k.x S2, b1 = k.y S1, b2 = 2 k.y S2, n = k.z SN.
template <bool WX>
__device__ __forceinline__ void adj_apply(const float4 k, float S1, float S2, float SN, Acc& A) {
  A.a1 = fmaf(k.x, S1, A.a1);
  A.a2 = fmaf(2.f * k.x, S2, A.a2);
  if (WX) {
    A.b1 = fmaf(k.y, S1, A.b1);
    A.b2 = fmaf(2.f * k.y, S2, A.b2);
  }
  A.n = fmaf(k.z, SN, A.n);
}

// One pair (the source owns the thread, the lens comes from the tile) with
// its bin's coefficients k: the per-pair form, where bins vary pair to pair.
template <bool LOGB, bool WX>
__device__ __forceinline__ void adj_pair(float sx, float sy, const float4 l, const float4 k, Acc& A) {
  const float dx = l.x - sx;  // lens minus source, as in the forward pass
  const float dy = l.y - sy;
  const float dx2 = dx * dx;
  const float d2 = fmaf(dy, dy, dx2);
  float r;
  if (LOGB) {
    const float rs = rsqrtf(d2);
    r = rs * rs;
  } else {
    r = __frcp_rn(d2);
  }
  const float c2 = fmaf(-dy, dy, dx2) * r;
  const float qq = dx * dy;
  const float s2 = (qq + qq) * r;
  const float mv = k.x * l.z;
  A.a1 = fmaf(mv, c2, A.a1);
  A.a2 = fmaf(mv, s2, A.a2);
  if (WX) {
    const float xv = k.y * l.z;
    A.b1 = fmaf(xv, c2, A.b1);
    A.b2 = fmaf(xv, s2, A.b2);
  }
  A.n = fmaf(k.z, l.w, A.n);
}

// Two consecutive lenses (2k, 2k+1) of a 32-lens sub-chunk in shared memory
// with their fields interleaved, so that a 64-bit register pair holds one
// field of both (the operand form of the sm_100 packed FP32 instructions).
// The kernel rewrites each lens tile in place into this form (the same 64
// bytes as the two SrcRec).  vw = val_A w_A, w = w_A.
struct __align__(16) LensPair {
  float4 xy;  // x0 x1 y0 y1
  float4 fw;  // vw0 vw1 w0 w1
  float4 zz;  // z0 z1 0 0
  float4 pad;
};
static_assert(sizeof(LensPair) == 2 * sizeof(SrcRec), "a LensPair rewrites two SrcRec in place");
// Coordinate of the null lens that pads an odd sub-chunk: finite d^2, zero
// weight and value, NaN z (never in front of a source).
constexpr float kNullLens = 1.0e18f;

// Lens j of a sub-chunk in LensPair form: {x, y, vw, w} and z.
__device__ __forceinline__ float4 lens_of(const LensPair* __restrict__ S, int j, float& z) {
  const float* f = reinterpret_cast<const float*>(S + (j >> 1)) + (j & 1);
  z = f[8];
  return make_float4(f[0], f[2], f[4], f[6]);
}

// The terms of the bin-independent sums (S1: F P, S2: F Q, SN: w) for the two
// lenses of one LensPair (packed FP32): F = vw r (times the z mask),
// P = dx^2 - dy^2, Q = dx dy, each half equal to the scalar computation.  w
// gets the z mask too.
template <bool HAS_Z, bool LOGB>
__device__ __forceinline__ void adj_terms2(float2 nsx, float2 nsy, float sz, const LensPair& lp, float2& d2,
                                           float2& F, float2& Pq, float2& Q, float2& w, bool& z0, bool& z1) {
  const float2 dx = add2(lo2(lp.xy), nsx);  // lens minus source, as in the forward pass
  const float2 dy = add2(hi2(lp.xy), nsy);
  const float2 dx2 = mul2(dx, dx);
  d2 = fma2(dy, dy, dx2);
  float2 r;
  if (LOGB) {
    const float2 rs = make_float2(rsqrtf(d2.x), rsqrtf(d2.y));
    r = mul2(rs, rs);
  } else {
    r = make_float2(__frcp_rn(d2.x), __frcp_rn(d2.y));
  }
  F = mul2(lo2(lp.fw), r);
  w = hi2(lp.fw);
  z0 = z1 = true;
  if (HAS_Z) {  // a lens behind the source adds nothing (src/tpcf.f90:322)
    z0 = lp.zz.x <= sz;
    z1 = lp.zz.y <= sz;
    const float2 zm = make_float2(z0 ? 1.f : 0.f, z1 ? 1.f : 0.f);
    F = mul2(F, zm);
    w = mul2(w, zm);
  }
  Pq = fma2(make_float2(-dy.x, -dy.y), dy, dx2);
  Q = mul2(dx, dy);
}

template <bool HAS_Z, bool LOGB, bool WX>
__global__ void __launch_bounds__(BT, kAdjMinBlocks) k_adj(const AdjParams P) {
  constexpr int NW = BT / 32;
  const int nb = P.nb;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  extern __shared__ __align__(128) unsigned char smem[];
  const AdjSmem L = adj_smem(nb);
  SrcRec* tiles = reinterpret_cast<SrcRec*>(smem + L.tiles);
  double* e2s = reinterpret_cast<double*>(smem + L.e2s);
  float* e2f = reinterpret_cast<float*>(smem + L.e2f);
  float4* coef = reinterpret_cast<float4*>(smem + L.coef);
  int* span0 = reinterpret_cast<int*>(smem + L.span0);
  int* span1 = reinterpret_cast<int*>(smem + L.span1);
  int* tpref = reinterpret_cast<int*>(smem + L.tpref);
  float4* subbox = reinterpret_cast<float4*>(smem + L.subbox);
  float* subw = reinterpret_cast<float*>(smem + L.subw);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + L.mbar);
  int* sh_item = reinterpret_cast<int*>(smem + L.misc);
  if (tid == 0) {
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
    mbar_fence_init();
  }
  for (int i = tid; i <= nb; i += BT) {
    e2s[i] = P.e2[i];
    e2f[i] = P.e2f[i];
  }
  __syncthreads();
  BinCtx C;
  C.A = P.binA; C.B = P.binB; C.eps = P.eps; C.one_m_eps = 1.f - P.eps;
  C.nb = nb; C.e2s = e2s; C.e2f = e2f;
  C.eps_rel = 4e-6f;
  C.lo_g = e2f[0] * (1.f - P.eps);
  C.hi_g = e2f[nb] * (1.f + P.eps);
  uint32_t phase = 0u, tcount = 0u;
  bool timed_out = false;

  for (;;) {
    if (tid == 0) *sh_item = atomicAdd(P.queue_head, 1);
    __syncthreads();
    const int item = *sh_item;
    if (item >= P.n_items) break;
    const int2 it = P.items[item];
    const AdjTask& T = P.tasks[it.x];
    const GridDesc G = T.grid;
    // this task's bin coefficients (read after the next barrier)
    for (int i = tid; i <= nb; i += BT)
      coef[i] = i < nb ? P.coef[(size_t)it.x * nb + i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const int g = it.y;
    const int si = g * BT + tid;
    const bool act = si < T.n_src;
    float4 r0 = make_float4(0.f, 0.f, 0.f, 0.f), r1 = r0;
    if (act) {
      r0 = T.s0[si];
      r1 = T.s1[si];
    }
    const float sx = r0.x, sy = r0.y, sz = r1.z;
    const float2 nsx = dup2(-sx), nsy = dup2(-sy);
    double D1 = 0, D2 = 0, D3 = 0, D4 = 0, DN = 0;
    const float4 box = T.gbox[g];
    int cy0, cy1;
    row_range(G, box, P.R, P.margin, cy0, cy1);
    for (int c0 = cy0; c0 <= cy1; c0 += kMaxRows) {
      const int nr = min(kMaxRows, cy1 - c0 + 1);
      __syncthreads();
      for (int r = tid; r < nr; r += BT) {
        const int2 sp = row_span(G, box, P.R, P.margin, c0 + r);
        span0[r] = sp.x;
        span1[r] = sp.y > sp.x ? sp.y : sp.x;
      }
      __syncthreads();
      if (tid == 0) {
        int acc = 0;
        for (int r = 0; r < nr; ++r) {
          tpref[r] = acc;
          acc += (span1[r] - span0[r] + kTile - 1) / kTile;
        }
        tpref[nr] = acc;
      }
      __syncthreads();
      const int ntiles = tpref[nr];
      int rc = 0, ri = 0;
      if (tid == 0 && ntiles > 0) {
        while (tpref[ri + 1] <= 0) ++ri;
        const int s0 = span0[ri];
        const int n0 = min(kTile, span1[ri] - s0);
        const int bb = tcount & 1u;
        mbar_arrive_tx(&mbar[bb], (uint32_t)(n0 * sizeof(SrcRec)));
        bulk_g2s(tiles + bb * kTile, T.lens + s0, (uint32_t)(n0 * sizeof(SrcRec)), &mbar[bb]);
      }
      for (int k = 0; k < ntiles; ++k) {
        if (tid == 0 && k + 1 < ntiles) {
          while (tpref[ri + 1] <= k + 1) ++ri;
          const int s1 = span0[ri] + (k + 1 - tpref[ri]) * kTile;
          const int n1 = min(kTile, span1[ri] - s1);
          const int bb = (tcount + k + 1) & 1u;
          mbar_arrive_tx(&mbar[bb], (uint32_t)(n1 * sizeof(SrcRec)));
          bulk_g2s(tiles + bb * kTile, T.lens + s1, (uint32_t)(n1 * sizeof(SrcRec)), &mbar[bb]);
        }
        while (tpref[rc + 1] <= k) ++rc;
        const int s = span0[rc] + (k - tpref[rc]) * kTile;
        const int n = min(kTile, span1[rc] - s);
        const int bb = (tcount + k) & 1u;
        const bool ok = mbar_wait_bounded(&mbar[bb], (phase >> bb) & 1u);
        phase ^= (1u << bb);
        // not __restrict__: the sub-chunk pass rewrites these bytes in place
        const SrcRec* S = tiles + bb * kTile;
        const int nsub = (n + 31) >> 5;
        if (ok) {
          // One warp per 32-lens sub-chunk: its bounding box and weight sum,
          // and the rewrite of its records into LensPair form (lanes 2k, 2k+1
          // trade halves with one shuffle round; each lane stores only the 32
          // bytes of its own record).  Slots past the tile's end get the null
          // lens.
          for (int sc = warp; sc < nsub; sc += NW) {
            const int j = sc * 32 + lane;
            float4 a = make_float4(kNullLens, kNullLens, 0.f, 0.f);
            float bz = __int_as_float(0x7fc00000);
            float mnx = INFINITY, mny = INFINITY, mxx = -INFINITY, mxy = -INFINITY;
            if (j < n) {
              a = S[j].a;
              bz = S[j].b.x;
              mnx = mxx = a.x;
              mny = mxy = a.y;
            }
            const bool odd = lane & 1;
            // the even lane takes {x, y, vw, w} of its partner, the odd lane z
            const float r0 = __shfl_xor_sync(0xffffffffu, odd ? a.x : bz, 1);
            const float r1 = __shfl_xor_sync(0xffffffffu, a.y, 1);
            const float r2 = __shfl_xor_sync(0xffffffffu, a.z, 1);
            const float r3 = __shfl_xor_sync(0xffffffffu, a.w, 1);
            float4* dst = reinterpret_cast<float4*>(tiles + bb * kTile + j);
            if (!odd) {
              dst[0] = make_float4(a.x, r0, a.y, r1);
              dst[1] = make_float4(a.z, r2, a.w, r3);
            } else {
              dst[0] = make_float4(r0, bz, 0.f, 0.f);
              dst[1] = make_float4(0.f, 0.f, 0.f, 0.f);
            }
            fence_proxy_async_smem();  // before the bulk copy that later refills this buffer
            float sw = a.w;
#pragma unroll
            for (int o = 16; o; o >>= 1) {
              mnx = fminf(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
              mny = fminf(mny, __shfl_xor_sync(0xffffffffu, mny, o));
              mxx = fmaxf(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
              mxy = fmaxf(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
              sw += __shfl_xor_sync(0xffffffffu, sw, o);
            }
            if (lane == 0) {
              subbox[sc] = make_float4(mnx, mny, mxx, mxy);
              subw[sc] = sw;
            }
          }
        }
        if (__syncthreads_or(!ok)) timed_out = true;
        if (!timed_out) {
          Acc A{0.f, 0.f, 0.f, 0.f, 0.f};
          for (int sc = 0; sc < nsub; ++sc) {
            const int base = sc * 32;
            const int cnt = min(32, n - base);
            int blo = 0;
            const int cls = act ? classify<LOGB, HAS_Z, true>(sx, sy, subbox[sc], C, blo) : 0;
            const int m = (int)__reduce_max_sync(0xffffffffu, (unsigned)cls);
            if (m == 0) continue;
            const LensPair* __restrict__ Sc = reinterpret_cast<const LensPair*>(S + base);
            const int np = (cnt + 1) >> 1;
            constexpr bool LI = !HAS_Z;  // the w sum of every source is the sub-chunk's
            // chunk-local sums: a lane with no pair in range discards its
            // (possibly non-finite) arithmetic instead of adding it to A
            Acc Ac{0.f, 0.f, 0.f, 0.f, 0.f};
            if (m == 1) {
              // every pair of this lane is in bin blo (or the lane has none)
              const float4 kc = cls == 1 ? coef[blo] : make_float4(0.f, 0.f, 0.f, 0.f);
              float2 S1 = dup2(0.f), S2 = dup2(0.f), SN = dup2(0.f);
#pragma unroll 4
              for (int q = 0; q < np; ++q) {
                float2 d2, F, Pq, Q, w;
                bool z0, z1;
                adj_terms2<HAS_Z, LOGB>(nsx, nsy, sz, Sc[q], d2, F, Pq, Q, w, z0, z1);
                S1 = fma2(F, Pq, S1);
                S2 = fma2(F, Q, S2);
                if (!LI) SN = add2(SN, w);
              }
              adj_apply<WX>(kc, sum2(S1), sum2(S2), LI ? subw[sc] : sum2(SN), Ac);
            } else if (m == 2) {
              const float4 kl = (cls >= 1 && blo >= 0) ? coef[blo] : make_float4(0.f, 0.f, 0.f, 0.f);
              // a side outside [x_min, x_max] contributes nothing
              const float4 kz = make_float4(0.f, 0.f, 0.f, 0.f);
              const float4 kh = cls == 2 ? (blo + 1 < nb ? coef[blo + 1] : kz) : kl;
              const float E = cls == 2 ? e2f[blo + 1] : 3.0e38f;
              const float gE = cls == 2 ? E * C.eps_rel : 0.f;
              const float2 nE = dup2(-E);
              bool near = false;  // some pair lies within the guard band of E
              float2 T1 = dup2(0.f), T2 = dup2(0.f), TN = dup2(0.f), H1 = dup2(0.f), H2 = dup2(0.f), HN = dup2(0.f);
#pragma unroll 2
              for (int q = 0; q < np; ++q) {
                float2 d2, F, Pq, Q, w;
                bool z0, z1;
                adj_terms2<HAS_Z, LOGB>(nsx, nsy, sz, Sc[q], d2, F, Pq, Q, w, z0, z1);
                const float2 dE = add2(d2, nE);
                near |= fabsf(dE.x) <= gE;
                near |= fabsf(dE.y) <= gE;
                const bool u0 = z0 && d2.x >= E, u1 = z1 && d2.y >= E;
                T1 = fma2(F, Pq, T1);
                T2 = fma2(F, Q, T2);
                if (!LI) TN = add2(TN, w);
                const float2 Fm = make_float2(u0 ? F.x : 0.f, u1 ? F.y : 0.f);
                H1 = fma2(Fm, Pq, H1);
                H2 = fma2(Fm, Q, H2);
                HN = add2(HN, make_float2(u0 ? w.x : 0.f, u1 ? w.y : 0.f));
              }
              const float h1 = sum2(H1), h2 = sum2(H2), hn = sum2(HN);
              const float tn = LI ? subw[sc] : sum2(TN);
              adj_apply<WX>(kl, sum2(T1) - h1, sum2(T2) - h2, tn - hn, Ac);
              adj_apply<WX>(kh, h1, h2, hn, Ac);
              if (near) {  // rare: this lane's sub-chunk again, pair by pair, by the canonical rule
                Ac = Acc{0.f, 0.f, 0.f, 0.f, 0.f};
                for (int j = 0; j < cnt; ++j) {
                  float lz;
                  const float4 l = lens_of(Sc, j, lz);
                  if (HAS_Z && lz > sz) continue;
                  const float dx = l.x - sx, dy = l.y - sy;
                  const float d2 = fmaf(dy, dy, dx * dx);
                  const int b = pair_bin<LOGB>(d2, l.x, l.y, sx, sy, C);
                  if ((unsigned)b >= (unsigned)nb) continue;
                  adj_pair<LOGB, WX>(sx, sy, l, coef[b], Ac);
                }
              }
            } else if (act) {
              for (int j = 0; j < cnt; ++j) {
                float lz;
                const float4 l = lens_of(Sc, j, lz);
                if (HAS_Z && lz > sz) continue;  // lens behind source (src/tpcf.f90:322)
                const float dx = l.x - sx, dy = l.y - sy;
                const float d2 = fmaf(dy, dy, dx * dx);
                const int b = pair_bin<LOGB>(d2, l.x, l.y, sx, sy, C);
                if ((unsigned)b >= (unsigned)nb) continue;
                adj_pair<LOGB, WX>(sx, sy, l, coef[b], Ac);
              }
            }
            if (cls != 0) {
              A.a1 += Ac.a1; A.a2 += Ac.a2; A.b1 += Ac.b1; A.b2 += Ac.b2; A.n += Ac.n;
            }
          }
          D1 += A.a1; D2 += A.a2; D3 += A.b1; D4 += A.b2; DN += A.n;
        }
        __syncthreads();
      }
      tcount += (uint32_t)ntiles;
    }
    if (act) {
      double* d = T.dsum;
      const size_t n = (size_t)T.n_src;
      d[si] = D1;
      d[n + si] = D2;
      d[2 * n + si] = D3;
      d[3 * n + si] = D4;
      d[4 * n + si] = DN;
    }
    __syncthreads();
  }
  if (timed_out && tid == 0) atomicOr(P.err, kErrTimeout);
}

// --------------------------------------------------------------- prep -------
// Lens grid keys (lens validity: finite, w != 0, z >= 0), cell + Hilbert index inside.
__global__ void k_adj_lens_keys(const float* __restrict__ x, const float* __restrict__ y,
                                const float* __restrict__ z, const float* __restrict__ w, long long n, float x0,
                                float y0, float inv_cell, int ncx, int ncy, int mb, unsigned* keys, int* idx) {
  const unsigned ncells = (unsigned)ncx * (unsigned)ncy;
  const int half = mb >> 1;
  const float q = (float)(1u << half);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float xi = x[i], yi = y[i];
    bool v = isfinite(xi) && isfinite(yi) && w[i] != 0.f && !(z && z[i] < 0.f);
    unsigned key = ncells << mb;
    if (v) {
      const float fx = (xi - x0) * inv_cell, fy = (yi - y0) * inv_cell;
      const int cx = clamp_floor(fx, 0, ncx - 1), cy = clamp_floor(fy, 0, ncy - 1);
      key = ((unsigned)cy * (unsigned)ncx + (unsigned)cx) << mb;
      if (half > 0) {
        unsigned qx = (unsigned)clamp_floor((fx - (float)cx) * q, 0, (1 << half) - 1);
        unsigned qy = (unsigned)clamp_floor((fy - (float)cy) * q, 0, (1 << half) - 1);
        key |= hilbert_index(qx, qy, half);
      }
    }
    keys[i] = key;
    idx[i] = (int)i;
  }
}

__global__ void k_adj_lens_gather(const int* __restrict__ idx, int n_valid, const float* __restrict__ x,
                                  const float* __restrict__ y, const float* __restrict__ z,
                                  const float* __restrict__ val, const float* __restrict__ w, SrcRec* rec) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_valid) return;
  const int i = idx[s];
  SrcRec r;
  r.a = make_float4(x[i], y[i], val[i] * w[i], w[i]);
  r.b = make_float4(z ? z[i] : 0.f, 0.f, 0.f, 0.f);
  rec[s] = r;
}

// Source Hilbert keys over the source box (source validity: finite, z >= 0).
__global__ void k_adj_src_keys(const float* __restrict__ x, const float* __restrict__ y,
                               const float* __restrict__ z, long long n, float4 box, unsigned long long* keys,
                               int* idx) {
  const float sxs = 65535.f / fmaxf(box.z - box.x, 1e-30f), sys = 65535.f / fmaxf(box.w - box.y, 1e-30f);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float xi = x[i], yi = y[i];
    const bool v = isfinite(xi) && isfinite(yi) && !(z && z[i] < 0.f);
    unsigned long long key = ~0ull;
    if (v) {
      const unsigned qx = (unsigned)clamp_floor((xi - box.x) * sxs, 0, 65535);
      const unsigned qy = (unsigned)clamp_floor((yi - box.y) * sys, 0, 65535);
      key = hilbert_index(qx, qy, 16);
    }
    keys[i] = key;
    idx[i] = (int)i;
  }
}

__global__ void k_adj_src_gather(const int* __restrict__ idx, int n_valid, const float* __restrict__ x,
                                 const float* __restrict__ y, const float* __restrict__ z,
                                 const float* __restrict__ e1, const float* __restrict__ e2,
                                 const float* __restrict__ w, const float* __restrict__ m, float4* s0, float4* s1,
                                 int* perm) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_valid) return;
  const int i = idx[s];
  s0[s] = make_float4(x[i], y[i], e1[i], e2[i]);
  s1[s] = make_float4(w[i], 1.0f + (m ? m[i] : 0.f), z ? z[i] : 0.f, 0.f);
  perm[s] = i;
}

__global__ void k_adj_groups(int n_groups, int n_valid, int* gstart) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g <= n_groups) gstart[g] = min(g * BT, n_valid);
}

// Lens-side gradient terms of one task from its raw per-lens sums
// [nA][6][nb] (rows dw, gt, gx, w, K, n without lens factors), added to the
// lens catalogue's FP64 accumulators: acc_a += sum_b (mu_b Rt + mux_b Rx),
// acc_k += sum_b nu_b RK.  Tasks are added one launch after another (fixed
// order).
__global__ void k_adj_lens_acc(const double* __restrict__ raw, long long nA, int nb, const double* __restrict__ mu,
                               double* acc_a, double* acc_k) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nA; i += (long long)gridDim.x * blockDim.x) {
    const double* r = raw + (size_t)i * 6 * nb;
    double a = 0, k = 0;
    for (int b = 0; b < nb; ++b) {
      a += mu[b] * r[1 * nb + b] + mu[nb + b] * r[2 * nb + b];
      k += mu[2 * nb + b] * r[4 * nb + b];
    }
    acc_a[i] += a;
    acc_k[i] += k;
  }
}

// dL/dval_i = w_i acc_a, dL/dw_i = val_i acc_a - acc_k.
__global__ void k_adj_lens_finish(const double* __restrict__ acc_a, const double* __restrict__ acc_k,
                                  const float* __restrict__ val, const float* __restrict__ w, long long nA,
                                  float* g_val, float* g_w) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nA; i += (long long)gridDim.x * blockDim.x) {
    if (g_val) g_val[i] = (float)((double)w[i] * acc_a[i]);
    if (g_w) g_w[i] = (float)((double)val[i] * acc_a[i] - acc_k[i]);
  }
}

// Source gradients of one source catalogue from the D sums of the tasks that
// use it (added in task order), in input order:
//   dL/de1 = w (-D1 + D4), dL/de2 = w (-D2 - D3),
//   dL/dw = -e1 D1 - e2 D2 + e1 D4 - e2 D3 - (1 + m) DN, dL/dm = -w DN.
__global__ void k_adj_src_finish(const double* const* __restrict__ dsums, int n_sum, int ns,
                                 const float4* __restrict__ s0, const float4* __restrict__ s1,
                                 const int* __restrict__ perm, float* g_e1, float* g_e2, float* g_w, float* g_m) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  double D[5] = {0, 0, 0, 0, 0};
  for (int t = 0; t < n_sum; ++t)
    for (int q = 0; q < 5; ++q) D[q] += dsums[t][(size_t)q * ns + s];
  const int j = perm[s];
  const float4 a = s0[s], b = s1[s];
  const double w = (double)b.x, e1 = a.z, e2 = a.w;
  if (g_e1) g_e1[j] = (float)(w * (-D[0] + D[3]));
  if (g_e2) g_e2[j] = (float)(w * (-D[1] - D[2]));
  if (g_w) g_w[j] = (float)(-e1 * D[0] - e2 * D[1] + e1 * D[3] - e2 * D[2] - (double)b.y * D[4]);
  if (g_m) g_m[j] = (float)(-w * D[4]);
}

template <bool HAS_Z, bool LOGB, bool WX>
cudaError_t launch_adj_t(const AdjParams& P, int num_sms, cudaStream_t st) {
  const size_t smem = adj_smem(P.nb).total;
  auto kern = k_adj<HAS_Z, LOGB, WX>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, BT, smem);
  if (e != cudaSuccess) return e;
  int grid = std::max(1, std::min(per_sm * num_sms, P.n_items));
  kern<<<grid, BT, smem, st>>>(P);
  return cudaGetLastError();
}

cudaError_t launch_adj(const AdjParams& P, bool has_z, bool logb, bool wx, int num_sms, cudaStream_t st) {
  if (has_z) {
    if (logb) return wx ? launch_adj_t<true, true, true>(P, num_sms, st) : launch_adj_t<true, true, false>(P, num_sms, st);
    return wx ? launch_adj_t<true, false, true>(P, num_sms, st) : launch_adj_t<true, false, false>(P, num_sms, st);
  }
  if (logb) return wx ? launch_adj_t<false, true, true>(P, num_sms, st) : launch_adj_t<false, true, false>(P, num_sms, st);
  return wx ? launch_adj_t<false, false, true>(P, num_sms, st) : launch_adj_t<false, false, false>(P, num_sms, st);
}

template <class T>
std::vector<T> to_host(tpcf_ctx* c, const T* p, size_t n) {
  std::vector<T> h(n);
  check(cudaMemcpyAsync(h.data(), p, sizeof(T) * n, cudaMemcpyDefault, c->stream), "copy to host");
  check(cudaStreamSynchronize(c->stream), "sync");
  return h;
}

struct AdjLensIn {
  int64_t n;
  const float *x, *y, *z, *val, *w;
  float *g_val, *g_w;
};
struct AdjSrcIn {
  int64_t n;
  const float *x, *y, *z, *e1, *e2, *w, *m;
  float *g_e1, *g_e2, *g_w, *g_m;
};
struct AdjTaskIn {
  int lens, src;
  const double *sum_gt, *sum_gx, *sum_K, *lens_raw, *dL_dgt, *dL_dgx;
};

// The backward pass of a batched forward call: every task's source gradients
// in one persistent launch over all (task, source group) work items, with one
// lens grid per lens catalogue and one sorted source set per source catalogue;
// gradients of a catalogue used by several tasks are summed over them in task
// order (FP64).
tpcf_status run_adjoint_batch(tpcf_ctx* c, std::vector<AdjLensIn> lens, std::vector<AdjSrcIn> srcs,
                              const std::vector<AdjTaskIn>& tasks, const tpcf_bins* bins) {
  Phase ph_nvtx("tpcf: adjoint");
  begin_call(c);
  cudaStream_t st = c->stream;
  const int nb = bins->n_bin;
  const int nL = (int)lens.size(), nS = (int)srcs.size(), nT = (int)tasks.size();
  std::vector<double> e(nb + 1), e2(nb + 1);
  tpcf_status bs = canonical_edges(bins, e.data(), e2.data());
  if (bs != TPCF_OK) throw Failure(bs, "invalid binning");
  if (c->opts.spherical) throw Failure(TPCF_ERR_NOT_SUPPORTED, "spherical coordinates are not supported");
  for (const auto& l : lens)
    if (l.n < 0 || l.n > (1ll << 31) - 2 || (l.n > 0 && (!l.x || !l.y || !l.val || !l.w)))
      throw Failure(TPCF_ERR_INVALID_ARG, "lens catalogue size out of range or array missing");
  for (const auto& s : srcs)
    if (s.n < 0 || s.n > (1ll << 31) - 2 || (s.n > 0 && (!s.x || !s.y || !s.e1 || !s.e2 || !s.w)))
      throw Failure(TPCF_ERR_INVALID_ARG, "source catalogue size out of range or array missing");
  for (const auto& t : tasks) {
    if (t.lens < 0 || t.lens >= nL || t.src < 0 || t.src >= nS) throw Failure(TPCF_ERR_INVALID_ARG, "task index out of range");
    const AdjLensIn& l = lens[t.lens];
    if (!t.sum_gt || !t.sum_K || !t.dL_dgt || ((l.g_val || l.g_w) && !t.lens_raw))
      throw Failure(TPCF_ERR_INVALID_ARG, "missing forward sums, lens_raw or dL/dg_t");
  }

  // per-task bin coefficients mu, mux, nu (FP64 on the host)
  bool wx = false;
  std::vector<double> mu((size_t)nT * 3 * nb, 0.0);
  std::vector<float4> coef((size_t)nT * nb);
  for (int t = 0; t < nT; ++t) {
    const AdjTaskIn& T = tasks[t];
    const std::vector<double> hgt = to_host(c, T.sum_gt, nb), hK = to_host(c, T.sum_K, nb),
                              hl = to_host(c, T.dL_dgt, nb);
    std::vector<double> hgx(nb, 0.0), hlx(nb, 0.0);
    if (T.sum_gx) hgx = to_host(c, T.sum_gx, nb);
    if (T.dL_dgx) hlx = to_host(c, T.dL_dgx, nb);
    wx = wx || T.dL_dgx != nullptr;
    double* m = mu.data() + (size_t)t * 3 * nb;
    for (int b = 0; b < nb; ++b) {
      if (hK[b] > 0) {
        m[b] = hl[b] / hK[b];
        m[nb + b] = hlx[b] / hK[b];
        m[2 * nb + b] = (hl[b] * (hgt[b] / hK[b]) + hlx[b] * (hgx[b] / hK[b])) / hK[b];
      }
      coef[(size_t)t * nb + b] = make_float4((float)m[b], (float)m[nb + b], (float)m[2 * nb + b], 0.f);
    }
  }

  for (auto& l : lens) {
    l.x = stage(c, l.x, l.n); l.y = stage(c, l.y, l.n); l.z = stage(c, l.z, l.n);
    l.val = stage(c, l.val, l.n); l.w = stage(c, l.w, l.n);
  }
  for (auto& s : srcs) {
    s.x = stage(c, s.x, s.n); s.y = stage(c, s.y, s.n); s.z = stage(c, s.z, s.n);
    s.e1 = stage(c, s.e1, s.n); s.e2 = stage(c, s.e2, s.n); s.w = stage(c, s.w, s.n); s.m = stage(c, s.m, s.n);
  }
  double* dmu = (double*)ws_alloc(c, sizeof(double) * mu.size());
  check(cudaMemcpyAsync(dmu, mu.data(), sizeof(double) * mu.size(), cudaMemcpyHostToDevice, st), "H2D mu");
  auto dev_or_ws = [&](float* user, int64_t n) -> float* {
    if (!user) return nullptr;
    return is_device_ptr(user) ? user : (float*)ws_alloc(c, sizeof(float) * (size_t)std::max<int64_t>(n, 1));
  };

  // lens-side gradients: FP64 accumulators per lens catalogue, tasks in order
  for (int i = 0; i < nL; ++i) {
    AdjLensIn& l = lens[i];
    if (!(l.g_val || l.g_w) || l.n == 0) continue;
    double* acc = (double*)ws_alloc(c, sizeof(double) * 2 * l.n);
    check(cudaMemsetAsync(acc, 0, sizeof(double) * 2 * l.n, st), "memset lens acc");
    const unsigned gb = (unsigned)std::min<long long>((l.n + 255) / 256, 4096);
    for (int t = 0; t < nT; ++t) {
      if (tasks[t].lens != i) continue;
      const double* raw = stage(c, tasks[t].lens_raw, l.n * 6 * nb);
      k_adj_lens_acc<<<gb, 256, 0, st>>>(raw, l.n, nb, dmu + (size_t)t * 3 * nb, acc, acc + l.n);
      counted(c, cudaGetLastError(), "lens gradient terms");
    }
    float* dv = dev_or_ws(l.g_val, l.n);
    float* dw = dev_or_ws(l.g_w, l.n);
    k_adj_lens_finish<<<gb, 256, 0, st>>>(acc, acc + l.n, l.val, l.w, l.n, dv, dw);
    counted(c, cudaGetLastError(), "lens gradients");
    if (dv && dv != l.g_val) copy_out(c, l.g_val, dv, sizeof(float) * l.n);
    if (dw && dw != l.g_w) copy_out(c, l.g_w, dw, sizeof(float) * l.n);
  }
  bool any_src = false;
  for (const auto& s : srcs) any_src = any_src || ((s.g_e1 || s.g_e2 || s.g_w || s.g_m) && s.n > 0);
  if (!any_src) {
    check(cudaStreamSynchronize(st), "sync");
    return TPCF_OK;
  }

  // boxes and counts: lens catalogues (kind 1), then source catalogues (kind 0)
  const int ncat = nL + nS;
  int* box_ord = (int*)ws_alloc(c, sizeof(int) * 8 * ncat);
  unsigned long long* cnt = (unsigned long long*)ws_alloc(c, sizeof(unsigned long long) * ncat);
  int* pr = (int*)ws_alloc(c, sizeof(int) * 2 * ncat);
  float* boxf = (float*)ws_alloc(c, sizeof(float) * 8 * ncat);
  counted(c, launch_bbox_init(box_ord, cnt, pr, ncat, st), "bbox init");
  for (int i = 0; i < nL; ++i)
    counted(c, launch_bbox(lens[i].x, lens[i].y, lens[i].z, lens[i].w, nullptr, nullptr, lens[i].n, 1,
                           box_ord + 8 * i, cnt + i, pr + 2 * i, st), "bbox lens");
  for (int i = 0; i < nS; ++i)
    counted(c, launch_bbox(srcs[i].x, srcs[i].y, srcs[i].z, nullptr, nullptr, nullptr, srcs[i].n, 0,
                           box_ord + 8 * (nL + i), cnt + nL + i, pr + 2 * (nL + i), st), "bbox src");
  counted(c, launch_bbox_finish(box_ord, boxf, 8 * ncat, st), "bbox finish");
  std::vector<float> hb(8 * ncat);
  std::vector<unsigned long long> hc(ncat);
  check(cudaMemcpyAsync(hb.data(), boxf, sizeof(float) * 8 * ncat, cudaMemcpyDeviceToHost, st), "D2H box");
  check(cudaMemcpyAsync(hc.data(), cnt, sizeof(unsigned long long) * ncat, cudaMemcpyDeviceToHost, st), "D2H count");
  check(cudaStreamSynchronize(st), "sync box");

  // outputs, zero for sources with no pair
  std::vector<float*> o_e1(nS), o_e2(nS), o_w(nS), o_m(nS);
  for (int i = 0; i < nS; ++i) {
    AdjSrcIn& s = srcs[i];
    o_e1[i] = dev_or_ws(s.g_e1, s.n); o_e2[i] = dev_or_ws(s.g_e2, s.n);
    o_w[i] = dev_or_ws(s.g_w, s.n); o_m[i] = dev_or_ws(s.g_m, s.n);
    for (float* p : {o_e1[i], o_e2[i], o_w[i], o_m[i]})
      if (p && s.n > 0) check(cudaMemsetAsync(p, 0, sizeof(float) * s.n, st), "memset grad");
  }
  bool has_z = false;
  for (const auto& t : tasks) {
    const int li = t.lens, si = nL + t.src;
    if (hc[li] > 0 && hc[si] > 0 && hb[8 * li + 5] > hb[8 * si + 4]) has_z = true;
  }
  const bool logb = bins->spacing == TPCF_LOG;
  const double Rd = bins->x_max;
  const float R = (float)(Rd * (1.0 + 1e-6));

  // one lens grid per lens catalogue
  std::vector<GridDesc> lgrid(nL);
  std::vector<SrcRec*> lrec(nL, nullptr);
  double maxcell = 0.0;
  for (int i = 0; i < nL; ++i) {
    const AdjLensIn& l = lens[i];
    const int nl = (int)hc[i];
    GridDesc& g = lgrid[i];
    const float* b = &hb[8 * i];
    const float x0 = nl ? b[0] : 0.f, y0 = nl ? b[1] : 0.f, ex = nl ? b[2] - b[0] : 0.f, ey = nl ? b[3] - b[1] : 0.f;
    double cell = c->opts.cell_size > 0 ? c->opts.cell_size : Rd / 16.0;
    const double span = std::max((double)ex, (double)ey);
    if (!c->opts.use_grid) cell = span * 2.0 + 1.0;
    while ((span / cell + 2.0) * (span / cell + 2.0) > (double)(1 << 24)) cell *= 1.5;
    if (!(cell > 0)) cell = 1.0;
    maxcell = std::max(maxcell, cell);
    const int ncx = std::max(1, (int)std::floor(ex / cell) + 1), ncy = std::max(1, (int)std::floor(ey / cell) + 1);
    const unsigned ncells = (unsigned)ncx * (unsigned)ncy;
    g.x0 = x0; g.y0 = y0; g.cell = (float)cell; g.inv_cell = (float)(1.0 / cell);
    g.ncx = ncx; g.ncy = ncy; g.n_valid = nl;
    int* cs = (int*)ws_alloc(c, sizeof(int) * (ncells + 1));
    lrec[i] = (SrcRec*)ws_alloc(c, sizeof(SrcRec) * std::max(nl, 1));
    if (l.n > 0) {
      unsigned* k0 = (unsigned*)ws_alloc(c, sizeof(unsigned) * l.n);
      unsigned* k1 = (unsigned*)ws_alloc(c, sizeof(unsigned) * l.n);
      int* i0 = (int*)ws_alloc(c, sizeof(int) * l.n);
      int* i1 = (int*)ws_alloc(c, sizeof(int) * l.n);
      int cell_bits = 1;
      while (cell_bits < 32 && (1ull << cell_bits) <= (unsigned long long)ncells) ++cell_bits;
      const int mb = std::min(16, (32 - cell_bits) & ~1);
      k_adj_lens_keys<<<(unsigned)std::min<long long>((l.n + 255) / 256, 4096), 256, 0, st>>>(
          l.x, l.y, l.z, l.w, l.n, x0, y0, g.inv_cell, ncx, ncy, mb, k0, i0);
      counted(c, cudaGetLastError(), "lens keys");
      size_t tb = 0;
      check(sort_pairs_u32(nullptr, tb, k0, k1, i0, i1, (int)l.n, cell_bits + mb, st), "sort size");
      void* tmp = ws_alloc(c, tb);
      check(sort_pairs_u32(tmp, tb, k0, k1, i0, i1, (int)l.n, cell_bits + mb, st), "sort lenses");
      counted(c, launch_cell_start(k1, l.n, ncells, mb, cs, st), "cell start");
      if (nl > 0) {
        k_adj_lens_gather<<<(nl + 255) / 256, 256, 0, st>>>(i1, nl, l.x, l.y, l.z, l.val, l.w, lrec[i]);
        counted(c, cudaGetLastError(), "lens gather");
      }
    } else {
      check(cudaMemsetAsync(cs, 0, sizeof(int) * (ncells + 1), st), "memset cells");
    }
    g.cell_start = cs;
    g.rec = lrec[i];
  }
  // one sorted source set (with groups of BT) per source catalogue
  std::vector<float4*> s0(nS), s1(nS), gbox(nS);
  std::vector<int*> perm(nS), gstart(nS);
  std::vector<int> ngroups(nS, 0);
  for (int i = 0; i < nS; ++i) {
    const AdjSrcIn& s = srcs[i];
    const int ns = (int)hc[nL + i];
    s0[i] = (float4*)ws_alloc(c, sizeof(float4) * std::max(ns, 1));
    s1[i] = (float4*)ws_alloc(c, sizeof(float4) * std::max(ns, 1));
    perm[i] = (int*)ws_alloc(c, sizeof(int) * std::max(ns, 1));
    ngroups[i] = (ns + BT - 1) / BT;
    gstart[i] = (int*)ws_alloc(c, sizeof(int) * (ngroups[i] + 1));
    gbox[i] = (float4*)ws_alloc(c, sizeof(float4) * std::max(ngroups[i], 1));
    if (ns == 0) continue;
    const float* b = &hb[8 * (nL + i)];
    unsigned long long* k0 = (unsigned long long*)ws_alloc(c, sizeof(unsigned long long) * s.n);
    unsigned long long* k1 = (unsigned long long*)ws_alloc(c, sizeof(unsigned long long) * s.n);
    int* i0 = (int*)ws_alloc(c, sizeof(int) * s.n);
    int* i1 = (int*)ws_alloc(c, sizeof(int) * s.n);
    k_adj_src_keys<<<(unsigned)std::min<long long>((s.n + 255) / 256, 4096), 256, 0, st>>>(
        s.x, s.y, s.z, s.n, make_float4(b[0], b[1], b[2], b[3]), k0, i0);
    counted(c, cudaGetLastError(), "source keys");
    size_t tb = 0;
    check(sort_pairs_u64(nullptr, tb, k0, k1, i0, i1, (int)s.n, st), "sort size");
    void* tmp = ws_alloc(c, tb);
    check(sort_pairs_u64(tmp, tb, k0, k1, i0, i1, (int)s.n, st), "sort sources");
    k_adj_src_gather<<<(ns + 255) / 256, 256, 0, st>>>(i1, ns, s.x, s.y, s.z, s.e1, s.e2, s.w, s.m, s0[i], s1[i],
                                                         perm[i]);
    counted(c, cudaGetLastError(), "source gather");
    k_adj_groups<<<(ngroups[i] + 1 + 255) / 256, 256, 0, st>>>(ngroups[i], ns, gstart[i]);
    counted(c, cudaGetLastError(), "groups");
    counted(c, launch_group_box(s0[i], gstart[i], ngroups[i], gbox[i], st), "group box");
  }
  float margin = 0.f;
  for (int i = 0; i < ncat; ++i)
    if (hc[i] > 0)
      margin = std::max(margin, std::fabs(hb[8 * i]) + std::fabs(hb[8 * i + 1]) + std::fabs(hb[8 * i + 2]) +
                                    std::fabs(hb[8 * i + 3]));
  margin = (float)(1e-5 * (margin + Rd) + 1e-4 * maxcell);

  // tasks, their D sums and the work items (task, source group)
  std::vector<AdjTask> at(nT);
  std::vector<double*> dsum(nT, nullptr);
  std::vector<int2> items;
  std::vector<TaskDesc> tdesc(nT);
  for (int t = 0; t < nT; ++t) {
    const int li = tasks[t].lens, si = tasks[t].src;
    const int ns = (int)hc[nL + si];
    dsum[t] = (double*)ws_alloc(c, sizeof(double) * 5 * std::max(ns, 1));
    if (ns > 0) check(cudaMemsetAsync(dsum[t], 0, sizeof(double) * 5 * ns, st), "memset D sums");
    AdjTask& a = at[t];
    a.grid = lgrid[li]; a.lens = lrec[li]; a.s0 = s0[si]; a.s1 = s1[si]; a.gbox = gbox[si]; a.n_src = ns;
    a.dsum = dsum[t];
    // item cost: the source groups play the lens-group role, the lens grid the source grid
    tdesc[t].lens_cat = si; tdesc[t].src_cat = li; tdesc[t].item_base = 0; tdesc[t].lens_acc_off = -1;
    tdesc[t].margin = margin;
    if (hc[li] > 0)
      for (int g = 0; g < ngroups[si]; ++g) items.push_back(make_int2(t, g));
  }
  const int n_items = (int)items.size();
  if (n_items > 0) {
    std::vector<LensDesc> gdesc(nS);
    for (int i = 0; i < nS; ++i) {
      gdesc[i].rec = s0[i]; gdesc[i].group_start = gstart[i]; gdesc[i].group_box = gbox[i];
      gdesc[i].n_valid = (int)hc[nL + i]; gdesc[i].n_groups = ngroups[i];
    }
    AdjTask* d_at = (AdjTask*)ws_alloc(c, sizeof(AdjTask) * nT);
    TaskDesc* d_td = (TaskDesc*)ws_alloc(c, sizeof(TaskDesc) * nT);
    LensDesc* d_gd = (LensDesc*)ws_alloc(c, sizeof(LensDesc) * nS);
    GridDesc* d_lg = (GridDesc*)ws_alloc(c, sizeof(GridDesc) * nL);
    check(cudaMemcpyAsync(d_at, at.data(), sizeof(AdjTask) * nT, cudaMemcpyHostToDevice, st), "H2D tasks");
    check(cudaMemcpyAsync(d_td, tdesc.data(), sizeof(TaskDesc) * nT, cudaMemcpyHostToDevice, st), "H2D");
    check(cudaMemcpyAsync(d_gd, gdesc.data(), sizeof(LensDesc) * nS, cudaMemcpyHostToDevice, st), "H2D");
    check(cudaMemcpyAsync(d_lg, lgrid.data(), sizeof(GridDesc) * nL, cudaMemcpyHostToDevice, st), "H2D");
    int2* items0 = (int2*)ws_alloc(c, sizeof(int2) * n_items);
    int2* d_items = (int2*)ws_alloc(c, sizeof(int2) * n_items);
    check(cudaMemcpyAsync(items0, items.data(), sizeof(int2) * n_items, cudaMemcpyHostToDevice, st), "H2D items");
    // costliest items first (in cost bands, space order inside a band): cost =
    // lenses in the rows of each source group
    unsigned long long* ck0 = (unsigned long long*)ws_alloc(c, sizeof(unsigned long long) * n_items);
    unsigned long long* ck1 = (unsigned long long*)ws_alloc(c, sizeof(unsigned long long) * n_items);
    int* o0 = (int*)ws_alloc(c, sizeof(int) * n_items);
    int* o1 = (int*)ws_alloc(c, sizeof(int) * n_items);
    counted(c, launch_item_cost(items0, n_items, d_td, d_gd, d_lg, R, ck0, o0, st), "item cost");
    size_t tb = 0;
    check(sort_pairs_u64_desc(nullptr, tb, ck0, ck1, o0, o1, n_items, st), "sort size");
    void* tmp = ws_alloc(c, tb);
    check(sort_pairs_u64_desc(tmp, tb, ck0, ck1, o0, o1, n_items, st), "sort items");
    counted(c, launch_permute_items(items0, o1, n_items, 0, 1, d_items, st), "permute items");
    double* de2 = (double*)ws_alloc(c, sizeof(double) * (nb + 1));
    float* de2f = (float*)ws_alloc(c, sizeof(float) * (nb + 1));
    float4* dcoef = (float4*)ws_alloc(c, sizeof(float4) * coef.size());
    int* head = (int*)ws_alloc(c, sizeof(int) * 4);
    std::vector<float> e2f(nb + 1);
    for (int i = 0; i <= nb; ++i) e2f[i] = (float)e2[i];
    check(cudaMemcpyAsync(de2, e2.data(), sizeof(double) * (nb + 1), cudaMemcpyHostToDevice, st), "H2D e2");
    check(cudaMemcpyAsync(de2f, e2f.data(), sizeof(float) * (nb + 1), cudaMemcpyHostToDevice, st), "H2D e2f");
    check(cudaMemcpyAsync(dcoef, coef.data(), sizeof(float4) * coef.size(), cudaMemcpyHostToDevice, st), "H2D coef");
    check(cudaMemsetAsync(head, 0, sizeof(int) * 4, st), "memset head");
    AdjParams P{};
    P.tasks = d_at; P.items = d_items; P.n_items = n_items; P.nb = nb; P.queue_head = head;
    P.err = (unsigned*)(head + 1); P.e2 = de2; P.e2f = de2f; P.coef = dcoef; P.R = R; P.margin = margin;
    if (logb) {
      const double l0 = std::log2(e2[0]), l1 = std::log2(e2[nb]);
      const double A = nb / (l1 - l0);
      P.binA = (float)A;
      P.binB = (float)(-l0 * A);
      P.eps = 1.0f / 32768.0f;
    } else {
      P.eps = 4e-6f;
    }
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    if (c->time_pairs) {
      check(cudaEventCreate(&ev0), "event");
      check(cudaEventCreate(&ev1), "event");
      check(cudaEventRecord(ev0, st), "event record");
    }
    counted(c, launch_adj(P, has_z, logb, wx, c->num_sms, st), "adjoint kernel");
    if (c->time_pairs) {
      check(cudaEventRecord(ev1, st), "event record");
      check(cudaEventSynchronize(ev1), "event sync");
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ev0, ev1);
      c->last_pair_ms = ms;
      cudaEventDestroy(ev0);
      cudaEventDestroy(ev1);
    }
    unsigned herr = 0;
    check(cudaMemcpyAsync(&herr, head + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, st), "D2H err");
    check(cudaStreamSynchronize(st), "sync adjoint");  // also keeps the host descriptors alive until here
    if (herr & kErrTimeout) throw Failure(TPCF_ERR_TIMEOUT, "a bounded device wait timed out in the adjoint kernel");
  }
  // per source catalogue: D sums of its tasks in task order -> gradients
  for (int i = 0; i < nS; ++i) {
    const int ns = (int)hc[nL + i];
    std::vector<const double*> ds;
    for (int t = 0; t < nT; ++t)
      if (tasks[t].src == i && hc[tasks[t].lens] > 0) ds.push_back(dsum[t]);
    if (ns > 0 && !ds.empty()) {
      const double** d_ds = (const double**)ws_alloc(c, sizeof(double*) * ds.size());
      check(cudaMemcpyAsync(d_ds, ds.data(), sizeof(double*) * ds.size(), cudaMemcpyHostToDevice, st), "H2D sums");
      k_adj_src_finish<<<(ns + 255) / 256, 256, 0, st>>>(d_ds, (int)ds.size(), ns, s0[i], s1[i], perm[i], o_e1[i],
                                                         o_e2[i], o_w[i], o_m[i]);
      counted(c, cudaGetLastError(), "source gradients");
      check(cudaStreamSynchronize(st), "sync source gradients");  // ds outlives its copy
    }
    const AdjSrcIn& s = srcs[i];
    if (o_e1[i] && o_e1[i] != s.g_e1) copy_out(c, s.g_e1, o_e1[i], sizeof(float) * s.n);
    if (o_e2[i] && o_e2[i] != s.g_e2) copy_out(c, s.g_e2, o_e2[i], sizeof(float) * s.n);
    if (o_w[i] && o_w[i] != s.g_w) copy_out(c, s.g_w, o_w[i], sizeof(float) * s.n);
    if (o_m[i] && o_m[i] != s.g_m) copy_out(c, s.g_m, o_m[i], sizeof(float) * s.n);
  }
  check(cudaStreamSynchronize(st), "sync outputs");
  return TPCF_OK;
}

}  // namespace

extern "C" tpcf_status tpcf_shear_scalar_adjoint(
    tpcf_ctx* c, const float* xA, const float* yA, const float* zA, const float* valA, const float* wA, int64_t nA,
    const float* xB, const float* yB, const float* zB, const float* e1B, const float* e2B, const float* wB,
    const float* mB, int64_t nB, const tpcf_bins* bins, const double* sum_gt, const double* sum_gx,
    const double* sum_K, const double* lens_raw, const double* dL_dgt, const double* dL_dgx, float* grad_valA,
    float* grad_wA, float* grad_e1B, float* grad_e2B, float* grad_wB, float* grad_mB) {
  if (!c || !bins) return TPCF_ERR_INVALID_ARG;
  try {
    std::vector<AdjLensIn> L{{nA, xA, yA, zA, valA, wA, grad_valA, grad_wA}};
    std::vector<AdjSrcIn> S{{nB, xB, yB, zB, e1B, e2B, wB, mB, grad_e1B, grad_e2B, grad_wB, grad_mB}};
    std::vector<AdjTaskIn> T{{0, 0, sum_gt, sum_gx, sum_K, lens_raw, dL_dgt, dL_dgx}};
    return run_adjoint_batch(c, L, S, T, bins);
  } catch (const Failure& f) {
    c->err = f.msg;
    return f.status;
  }
}

extern "C" tpcf_status tpcf_batch_shear_scalar_adjoint(
    tpcf_ctx* c, int32_t n_lens_cat, const tpcf_lens_catalog* lenses, tpcf_lens_grad* lens_grads,
    int32_t n_src_cat, const tpcf_shear_catalog* sources, tpcf_shear_grad* src_grads, int32_t n_task,
    const int32_t* task_lens, const int32_t* task_src, const tpcf_bins* bins, const tpcf_adjoint_task* task_in) {
  if (!c || !bins || n_lens_cat < 1 || n_src_cat < 1 || n_task < 1 || !lenses || !sources || !task_lens ||
      !task_src || !task_in)
    return TPCF_ERR_INVALID_ARG;
  try {
    std::vector<AdjLensIn> L;
    for (int i = 0; i < n_lens_cat; ++i) {
      const tpcf_lens_catalog& l = lenses[i];
      L.push_back({l.n, l.x, l.y, l.z, l.val, l.w, lens_grads ? lens_grads[i].val : nullptr,
                   lens_grads ? lens_grads[i].w : nullptr});
    }
    std::vector<AdjSrcIn> S;
    for (int i = 0; i < n_src_cat; ++i) {
      const tpcf_shear_catalog& s = sources[i];
      const tpcf_shear_grad* g = src_grads ? &src_grads[i] : nullptr;
      S.push_back({s.n, s.x, s.y, s.z, s.e1, s.e2, s.w, s.m, g ? g->e1 : nullptr, g ? g->e2 : nullptr,
                   g ? g->w : nullptr, g ? g->m : nullptr});
    }
    std::vector<AdjTaskIn> T;
    for (int t = 0; t < n_task; ++t) {
      const tpcf_adjoint_task& a = task_in[t];
      T.push_back({task_lens[t], task_src[t], a.sum_gt, a.sum_gx, a.sum_K, a.lens_raw, a.dL_dgt, a.dL_dgx});
    }
    return run_adjoint_batch(c, L, S, T, bins);
  } catch (const Failure& f) {
    c->err = f.msg;
    return f.status;
  }
}
