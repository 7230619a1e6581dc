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

struct AdjParams {
  const SrcRec* lens;       // lens grid records: a = {x, y, val*w, w}, b = {z, 0, 0, 0}
  GridDesc grid;            // grid over the lenses
  const float4* s0;         // sources sorted: {x, y, e1, e2}
  const float4* s1;         // {w, 1+m, z, 0}
  const int* perm;          // sorted source -> input index
  const float4* gbox;       // source group boxes
  const int2* items;        // (0, group) in processing order
  int n_items;
  int n_src;                // valid sources
  int nb;
  int* queue_head;
  unsigned* err;
  const double* e2;
  const float* e2f;
  const float4* coef;       // [nb] {mu, mux, nu, 0}
  float R, margin, binA, binB, eps;
  float* g_e1;
  float* g_e2;
  float* g_w;
  float* g_m;
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
    coef[i] = i < nb ? P.coef[i] : make_float4(0.f, 0.f, 0.f, 0.f);
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
  const GridDesc& G = P.grid;

  for (;;) {
    if (tid == 0) *sh_item = atomicAdd(P.queue_head, 1);
    __syncthreads();
    const int item = *sh_item;
    if (item >= P.n_items) break;
    const int g = P.items[item].y;
    const int si = g * BT + tid;
    const bool act = si < P.n_src;
    float4 r0 = make_float4(0.f, 0.f, 0.f, 0.f), r1 = r0;
    if (act) {
      r0 = P.s0[si];
      r1 = P.s1[si];
    }
    const float sx = r0.x, sy = r0.y, sz = r1.z;
    const float2 nsx = dup2(-sx), nsy = dup2(-sy);
    double D1 = 0, D2 = 0, D3 = 0, D4 = 0, DN = 0;
    const float4 box = P.gbox[g];
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
        bulk_g2s(tiles + bb * kTile, P.lens + s0, (uint32_t)(n0 * sizeof(SrcRec)), &mbar[bb]);
      }
      for (int k = 0; k < ntiles; ++k) {
        if (tid == 0 && k + 1 < ntiles) {
          while (tpref[ri + 1] <= k + 1) ++ri;
          const int s1 = span0[ri] + (k + 1 - tpref[ri]) * kTile;
          const int n1 = min(kTile, span1[ri] - s1);
          const int bb = (tcount + k + 1) & 1u;
          mbar_arrive_tx(&mbar[bb], (uint32_t)(n1 * sizeof(SrcRec)));
          bulk_g2s(tiles + bb * kTile, P.lens + s1, (uint32_t)(n1 * sizeof(SrcRec)), &mbar[bb]);
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
      const int j = P.perm[si];
      const double w = (double)r1.x;
      const double e1 = r0.z, e2 = r0.w;
      if (P.g_e1) P.g_e1[j] = (float)(w * (-D1 + D4));
      if (P.g_e2) P.g_e2[j] = (float)(w * (-D2 - D3));
      if (P.g_w) P.g_w[j] = (float)(-e1 * D1 - e2 * D2 + e1 * D4 - e2 * D3 - (double)r1.y * DN);
      if (P.g_m) P.g_m[j] = (float)(-w * DN);
    }
    __syncthreads();
  }
  if (timed_out && tid == 0) atomicOr(P.err, kErrTimeout);
}

// --------------------------------------------------------------- prep -------
// Lens grid keys (lens validity: finite, w != 0, z >= 0), cell + Morton inside.
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
        unsigned m = 0;
        for (int b = 0; b < half; ++b) m |= (((qx >> b) & 1u) << (2 * b)) | (((qy >> b) & 1u) << (2 * b + 1));
        key |= m;
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

// Source Morton keys over the source box (source validity: finite, z >= 0).
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
      unsigned m = 0;
      for (int b = 0; b < 16; ++b) m |= (((qx >> b) & 1u) << (2 * b)) | (((qy >> b) & 1u) << (2 * b + 1));
      key = m;
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

__global__ void k_adj_groups(int n_groups, int n_valid, int* gstart, int2* items) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g <= n_groups) gstart[g] = min(g * BT, n_valid);
  if (g < n_groups) items[g] = make_int2(0, g);
}

// Lens-side gradients from the raw per-lens sums [nA][6][nb] (rows dw, gt, gx,
// w, K, n without lens factors).
__global__ void k_adj_lens_grads(const double* __restrict__ raw, const float* __restrict__ val,
                                 const float* __restrict__ w, long long nA, int nb, const double* __restrict__ mu,
                                 float* g_val, float* g_w) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nA; i += (long long)gridDim.x * blockDim.x) {
    const double* r = raw + (size_t)i * 6 * nb;
    double a = 0, k = 0;
    for (int b = 0; b < nb; ++b) {
      a += mu[b] * r[1 * nb + b] + mu[nb + b] * r[2 * nb + b];
      k += mu[2 * nb + b] * r[4 * nb + b];
    }
    if (g_val) g_val[i] = (float)((double)w[i] * a);
    if (g_w) g_w[i] = (float)((double)val[i] * a - k);
  }
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

tpcf_status run_adjoint(tpcf_ctx* c, const float* xA, const float* yA, const float* zA, const float* valA,
                        const float* wA, int64_t nA, const float* xB, const float* yB, const float* zB,
                        const float* e1B, const float* e2B, const float* wB, const float* mB, int64_t nB,
                        const tpcf_bins* bins, const double* sum_gt, const double* sum_gx, const double* sum_K,
                        const double* lens_raw, const double* dL_dgt, const double* dL_dgx, float* g_val,
                        float* g_wA, float* g_e1, float* g_e2, float* g_wB, float* g_m) {
  begin_call(c);
  cudaStream_t st = c->stream;
  const int nb = bins->n_bin;
  std::vector<double> e(nb + 1), e2(nb + 1);
  tpcf_status bs = canonical_edges(bins, e.data(), e2.data());
  if (bs != TPCF_OK) throw Failure(bs, "invalid binning");
  if (c->opts.spherical) throw Failure(TPCF_ERR_NOT_SUPPORTED, "spherical coordinates are not supported");
  if (!sum_gt || !sum_K || !dL_dgt || ((g_val || g_wA) && !lens_raw))
    throw Failure(TPCF_ERR_INVALID_ARG, "missing forward sums, lens_raw or dL/dg_t");
  if (nA < 0 || nB < 0 || nA > (1ll << 31) - 2 || nB > (1ll << 31) - 2)
    throw Failure(TPCF_ERR_INVALID_ARG, "catalogue size out of range");

  // per-bin coefficients mu, mux, nu (FP64 on the host)
  const std::vector<double> hgt = to_host(c, sum_gt, nb), hK = to_host(c, sum_K, nb), hl = to_host(c, dL_dgt, nb);
  std::vector<double> hgx(nb, 0.0), hlx(nb, 0.0);
  if (sum_gx) hgx = to_host(c, sum_gx, nb);
  if (dL_dgx) hlx = to_host(c, dL_dgx, nb);
  const bool wx = dL_dgx != nullptr;
  std::vector<double> mu(3 * nb, 0.0);
  std::vector<float4> coef(nb);
  for (int b = 0; b < nb; ++b) {
    if (hK[b] > 0) {
      mu[b] = hl[b] / hK[b];
      mu[nb + b] = hlx[b] / hK[b];
      mu[2 * nb + b] = (hl[b] * (hgt[b] / hK[b]) + hlx[b] * (hgx[b] / hK[b])) / hK[b];
    }
    coef[b] = make_float4((float)mu[b], (float)mu[nb + b], (float)mu[2 * nb + b], 0.f);
  }

  xA = stage(c, xA, nA); yA = stage(c, yA, nA); zA = stage(c, zA, nA);
  valA = stage(c, valA, nA); wA = stage(c, wA, nA);
  xB = stage(c, xB, nB); yB = stage(c, yB, nB); zB = stage(c, zB, nB);
  e1B = stage(c, e1B, nB); e2B = stage(c, e2B, nB); wB = stage(c, wB, nB); mB = stage(c, mB, nB);

  // lens-side gradients
  double* dmu = (double*)ws_alloc(c, sizeof(double) * 3 * nb);
  check(cudaMemcpyAsync(dmu, mu.data(), sizeof(double) * 3 * nb, cudaMemcpyHostToDevice, st), "H2D mu");
  if ((g_val || g_wA) && nA > 0) {
    const double* raw = stage(c, lens_raw, nA * 6 * nb);
    float* dv = g_val ? (is_device_ptr(g_val) ? g_val : (float*)ws_alloc(c, sizeof(float) * nA)) : nullptr;
    float* dw = g_wA ? (is_device_ptr(g_wA) ? g_wA : (float*)ws_alloc(c, sizeof(float) * nA)) : nullptr;
    k_adj_lens_grads<<<(unsigned)std::min<long long>((nA + 255) / 256, 4096), 256, 0, st>>>(raw, valA, wA, nA, nb,
                                                                                          dmu, dv, dw);
    counted(c, cudaGetLastError(), "lens gradients");
    if (dv && dv != g_val) copy_out(c, g_val, dv, sizeof(float) * nA);
    if (dw && dw != g_wA) copy_out(c, g_wA, dw, sizeof(float) * nA);
  }
  if (!(g_e1 || g_e2 || g_wB || g_m) || nB == 0) {
    check(cudaStreamSynchronize(st), "sync");
    return TPCF_OK;
  }

  // boxes: lens (kind 1) and source (kind 0)
  int* box_ord = (int*)ws_alloc(c, sizeof(int) * 16);
  unsigned long long* cnt = (unsigned long long*)ws_alloc(c, sizeof(unsigned long long) * 2);
  int* pr = (int*)ws_alloc(c, sizeof(int) * 4);
  float* boxf = (float*)ws_alloc(c, sizeof(float) * 16);
  counted(c, launch_bbox_init(box_ord, cnt, pr, 2, st), "bbox init");
  counted(c, launch_bbox(xA, yA, zA, wA, nullptr, nullptr, nA, 1, box_ord, cnt, pr, st), "bbox lens");
  counted(c, launch_bbox(xB, yB, zB, nullptr, nullptr, nullptr, nB, 0, box_ord + 8, cnt + 1, pr + 2, st), "bbox src");
  counted(c, launch_bbox_finish(box_ord, boxf, 16, st), "bbox finish");
  float hb[16];
  unsigned long long hc[2];
  check(cudaMemcpyAsync(hb, boxf, sizeof(hb), cudaMemcpyDeviceToHost, st), "D2H box");
  check(cudaMemcpyAsync(hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, st), "D2H count");
  check(cudaStreamSynchronize(st), "sync box");
  const int nl = (int)hc[0], ns = (int)hc[1];
  // sources with no pair keep gradient 0
  auto zero_out = [&](float* p) {
    if (p) check(cudaMemsetAsync(p, 0, sizeof(float) * nB, st), "memset grad");
  };
  float* out_e1 = g_e1 ? (is_device_ptr(g_e1) ? g_e1 : (float*)ws_alloc(c, sizeof(float) * nB)) : nullptr;
  float* out_e2 = g_e2 ? (is_device_ptr(g_e2) ? g_e2 : (float*)ws_alloc(c, sizeof(float) * nB)) : nullptr;
  float* out_w = g_wB ? (is_device_ptr(g_wB) ? g_wB : (float*)ws_alloc(c, sizeof(float) * nB)) : nullptr;
  float* out_m = g_m ? (is_device_ptr(g_m) ? g_m : (float*)ws_alloc(c, sizeof(float) * nB)) : nullptr;
  zero_out(out_e1); zero_out(out_e2); zero_out(out_w); zero_out(out_m);
  const bool has_z = nl > 0 && ns > 0 && hb[5] > hb[8 + 4];
  const bool logb = bins->spacing == TPCF_LOG;
  const double Rd = bins->x_max;
  const float R = (float)(Rd * (1.0 + 1e-6));

  if (nl > 0 && ns > 0) {
    // grid over the lenses
    GridDesc g{};
    const float x0 = hb[0], y0 = hb[1], ex = hb[2] - hb[0], ey = hb[3] - hb[1];
    double cell = c->opts.cell_size > 0 ? c->opts.cell_size : Rd / 16.0;
    const double span = std::max((double)ex, (double)ey);
    if (!c->opts.use_grid) cell = span * 2.0 + 1.0;
    while ((span / cell + 2.0) * (span / cell + 2.0) > (double)(1 << 24)) cell *= 1.5;
    if (!(cell > 0)) cell = 1.0;
    const int ncx = std::max(1, (int)std::floor(ex / cell) + 1), ncy = std::max(1, (int)std::floor(ey / cell) + 1);
    const unsigned ncells = (unsigned)ncx * (unsigned)ncy;
    g.x0 = x0; g.y0 = y0; g.cell = (float)cell; g.inv_cell = (float)(1.0 / cell);
    g.ncx = ncx; g.ncy = ncy; g.n_valid = nl;
    int* cs = (int*)ws_alloc(c, sizeof(int) * (ncells + 1));
    SrcRec* lrec = (SrcRec*)ws_alloc(c, sizeof(SrcRec) * nl);
    {
      unsigned* k0 = (unsigned*)ws_alloc(c, sizeof(unsigned) * nA);
      unsigned* k1 = (unsigned*)ws_alloc(c, sizeof(unsigned) * nA);
      int* i0 = (int*)ws_alloc(c, sizeof(int) * nA);
      int* i1 = (int*)ws_alloc(c, sizeof(int) * nA);
      int cell_bits = 1;
      while (cell_bits < 32 && (1ull << cell_bits) <= (unsigned long long)ncells) ++cell_bits;
      const int mb = std::min(16, (32 - cell_bits) & ~1);
      k_adj_lens_keys<<<(unsigned)std::min<long long>((nA + 255) / 256, 4096), 256, 0, st>>>(
          xA, yA, zA, wA, nA, x0, y0, g.inv_cell, ncx, ncy, mb, k0, i0);
      counted(c, cudaGetLastError(), "lens keys");
      size_t tb = 0;
      check(sort_pairs_u32(nullptr, tb, k0, k1, i0, i1, (int)nA, cell_bits + mb, st), "sort size");
      void* tmp = ws_alloc(c, tb);
      check(sort_pairs_u32(tmp, tb, k0, k1, i0, i1, (int)nA, cell_bits + mb, st), "sort lenses");
      counted(c, launch_cell_start(k1, nA, ncells, mb, cs, st), "cell start");
      k_adj_lens_gather<<<(nl + 255) / 256, 256, 0, st>>>(i1, nl, xA, yA, zA, valA, wA, lrec);
      counted(c, cudaGetLastError(), "lens gather");
    }
    g.cell_start = cs;
    g.rec = lrec;
    // source groups
    float4* s0 = (float4*)ws_alloc(c, sizeof(float4) * ns);
    float4* s1 = (float4*)ws_alloc(c, sizeof(float4) * ns);
    int* perm = (int*)ws_alloc(c, sizeof(int) * ns);
    {
      unsigned long long* k0 = (unsigned long long*)ws_alloc(c, sizeof(unsigned long long) * nB);
      unsigned long long* k1 = (unsigned long long*)ws_alloc(c, sizeof(unsigned long long) * nB);
      int* i0 = (int*)ws_alloc(c, sizeof(int) * nB);
      int* i1 = (int*)ws_alloc(c, sizeof(int) * nB);
      k_adj_src_keys<<<(unsigned)std::min<long long>((nB + 255) / 256, 4096), 256, 0, st>>>(
          xB, yB, zB, nB, make_float4(hb[8], hb[9], hb[10], hb[11]), k0, i0);
      counted(c, cudaGetLastError(), "source keys");
      size_t tb = 0;
      check(sort_pairs_u64(nullptr, tb, k0, k1, i0, i1, (int)nB, st), "sort size");
      void* tmp = ws_alloc(c, tb);
      check(sort_pairs_u64(tmp, tb, k0, k1, i0, i1, (int)nB, st), "sort sources");
      k_adj_src_gather<<<(ns + 255) / 256, 256, 0, st>>>(i1, ns, xB, yB, zB, e1B, e2B, wB, mB, s0, s1, perm);
      counted(c, cudaGetLastError(), "source gather");
    }
    const int n_groups = (ns + BT - 1) / BT;
    int* gstart = (int*)ws_alloc(c, sizeof(int) * (n_groups + 1));
    int2* items0 = (int2*)ws_alloc(c, sizeof(int2) * n_groups);
    int2* items = (int2*)ws_alloc(c, sizeof(int2) * n_groups);
    float4* gbox = (float4*)ws_alloc(c, sizeof(float4) * n_groups);
    k_adj_groups<<<(n_groups + 1 + 255) / 256, 256, 0, st>>>(n_groups, ns, gstart, items0);
    counted(c, cudaGetLastError(), "groups");
    counted(c, launch_group_box(s0, gstart, n_groups, gbox, st), "group box");
    float margin = 0.f;
    for (int i = 0; i < 2; ++i)
      margin = std::max(margin, std::fabs(hb[8 * i]) + std::fabs(hb[8 * i + 1]) + std::fabs(hb[8 * i + 2]) +
                                    std::fabs(hb[8 * i + 3]));
    margin = (float)(1e-5 * (margin + Rd) + 1e-4 * g.cell);
    // longest items first: cost = lenses in the rows of each group
    {
      TaskDesc td{};
      td.lens_cat = 0; td.src_cat = 0; td.item_base = 0; td.lens_acc_off = -1;
      LensDesc ld{};
      ld.rec = s0; ld.group_start = gstart; ld.group_box = gbox; ld.n_valid = ns; ld.n_groups = n_groups;
      TaskDesc* dt = (TaskDesc*)ws_alloc(c, sizeof(TaskDesc));
      LensDesc* dl = (LensDesc*)ws_alloc(c, sizeof(LensDesc));
      GridDesc* dg = (GridDesc*)ws_alloc(c, sizeof(GridDesc));
      check(cudaMemcpyAsync(dt, &td, sizeof(td), cudaMemcpyHostToDevice, st), "H2D");
      check(cudaMemcpyAsync(dl, &ld, sizeof(ld), cudaMemcpyHostToDevice, st), "H2D");
      check(cudaMemcpyAsync(dg, &g, sizeof(g), cudaMemcpyHostToDevice, st), "H2D");
      unsigned long long* ck0 = (unsigned long long*)ws_alloc(c, sizeof(unsigned long long) * n_groups);
      unsigned long long* ck1 = (unsigned long long*)ws_alloc(c, sizeof(unsigned long long) * n_groups);
      int* o0 = (int*)ws_alloc(c, sizeof(int) * n_groups);
      int* o1 = (int*)ws_alloc(c, sizeof(int) * n_groups);
      counted(c, launch_item_cost(items0, n_groups, dt, dl, dg, R, margin, ck0, o0, st), "item cost");
      size_t tb = 0;
      check(sort_pairs_u64_desc(nullptr, tb, ck0, ck1, o0, o1, n_groups, st), "sort size");
      void* tmp = ws_alloc(c, tb);
      check(sort_pairs_u64_desc(tmp, tb, ck0, ck1, o0, o1, n_groups, st), "sort items");
      counted(c, launch_permute_items(items0, o1, n_groups, 0, 1, items, st), "permute items");
      check(cudaStreamSynchronize(st), "sync items");  // host descriptors above go out of scope
    }
    double* de2 = (double*)ws_alloc(c, sizeof(double) * (nb + 1));
    float* de2f = (float*)ws_alloc(c, sizeof(float) * (nb + 1));
    float4* dcoef = (float4*)ws_alloc(c, sizeof(float4) * nb);
    int* head = (int*)ws_alloc(c, sizeof(int) * 4);
    std::vector<float> e2f(nb + 1);
    for (int i = 0; i <= nb; ++i) e2f[i] = (float)e2[i];
    check(cudaMemcpyAsync(de2, e2.data(), sizeof(double) * (nb + 1), cudaMemcpyHostToDevice, st), "H2D e2");
    check(cudaMemcpyAsync(de2f, e2f.data(), sizeof(float) * (nb + 1), cudaMemcpyHostToDevice, st), "H2D e2f");
    check(cudaMemcpyAsync(dcoef, coef.data(), sizeof(float4) * nb, cudaMemcpyHostToDevice, st), "H2D coef");
    check(cudaMemsetAsync(head, 0, sizeof(int) * 4, st), "memset head");
    AdjParams P{};
    P.lens = lrec; P.grid = g; P.s0 = s0; P.s1 = s1; P.perm = perm; P.gbox = gbox; P.items = items;
    P.n_items = n_groups; P.n_src = ns; P.nb = nb; P.queue_head = head; P.err = (unsigned*)(head + 1);
    P.e2 = de2; P.e2f = de2f; P.coef = dcoef; P.R = R; P.margin = margin;
    if (logb) {
      const double l0 = std::log2(e2[0]), l1 = std::log2(e2[nb]);
      const double A = nb / (l1 - l0);
      P.binA = (float)A;
      P.binB = (float)(-l0 * A);
      P.eps = 1.0f / 32768.0f;
    } else {
      P.eps = 4e-6f;
    }
    P.g_e1 = out_e1; P.g_e2 = out_e2; P.g_w = out_w; P.g_m = out_m;
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
    check(cudaStreamSynchronize(st), "sync adjoint");
    if (herr & kErrTimeout) throw Failure(TPCF_ERR_TIMEOUT, "a bounded device wait timed out in the adjoint kernel");
  }
  if (out_e1 && out_e1 != g_e1) copy_out(c, g_e1, out_e1, sizeof(float) * nB);
  if (out_e2 && out_e2 != g_e2) copy_out(c, g_e2, out_e2, sizeof(float) * nB);
  if (out_w && out_w != g_wB) copy_out(c, g_wB, out_w, sizeof(float) * nB);
  if (out_m && out_m != g_m) copy_out(c, g_m, out_m, sizeof(float) * nB);
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
    return run_adjoint(c, xA, yA, zA, valA, wA, nA, xB, yB, zB, e1B, e2B, wB, mB, nB, bins, sum_gt, sum_gx, sum_K,
                       lens_raw, dL_dgt, dL_dgx, grad_valA, grad_wA, grad_e1B, grad_e2B, grad_wB, grad_mB);
  } catch (const Failure& f) {
    c->err = f.msg;
    return f.status;
  }
}
