// sphere.cu -- pair sums on the sphere: the spherical_coords branch of
// tangential_shear_tpcf / scalar_kappa_tpcf (src/tpcf.f90:297-359, with
// distance_sphere src/utils.f90:512-528 and angles_sphere :618-639).
//
// Positions are FP32 (lambda, phi) in radians.  Each object becomes its unit
// vector u, computed in FP64 by canon_sincos (sph_canon.cuh) and split into
// FP32 hi + lo parts.  For a pair (lens A, source B):
//   chord^2  c^2 = |u_B - u_A|^2, binned against (2 sin(e_i/2))^2 of the FP64
//            angle edges e_i (monotone in the angle, so the same bins);
//   angle    theta = 2 asin(c/2) (the reference's acos of the dot product);
//   position angle at the lens, A = (u_B - u_A).east_A and
//            B = (u_B - u_A).north_A.  These are the numerators of
//            angles_sphere, so cos 2phi = (A^2 - B^2)/(A^2 + B^2) and
//            sin 2phi = 2AB/(A^2 + B^2), the same as 2 cs1^2 - 1, 2 cs1 cs2.
// The pair arithmetic is FP32 on hi + lo differences (relative error ~1e-7
// at any separation).  The FP64 guard band re-bins a pair by the canonical
// rule: u = hi + lo in FP64, c^2 = (dx^2 + dy^2) + dz^2 rounded as written.
// The one-bin and one-edge sub-chunk paths run on packed FP32 instructions
// (two pairs per instruction) over tiles rewritten in place into SrcPairS.
//
// Pruning: a cell grid over (lambda reduced to [0, 2 pi), phi).  The rows of a
// work item are the phi rows within R of the lens box (angular distance
// >= |dphi|).  In each row the cells lie within the lambda reach
// asin(sin R / cos phi*) of the box, phi* being its largest |phi|, taken
// modulo 2 pi as up to three disjoint cell runs.  A pole within reach scans
// the whole row.  The reference aborts near poles and the prime meridian
// (src/kdtree.f90:398-413); here every position is valid.

#include <cstdio>

#include "pair_hist.cuh"
#include "sph_canon.cuh"
#include "tpcf_device.cuh"
#include "tpcf_internal.cuh"
#include "tpcf_kernels.h"

namespace tpcf {

// --------------------------------------------------- canonical unit vector --
// u = (cos phi cos lambda, cos phi sin lambda, sin phi), hi = fl32(u),
// lo = fl32(u - hi).
__device__ __forceinline__ void canon_unit(float lam, float phi, float4& hi, float4& lo) {
  double sl, cl, sp, cp;
  canon_sincos((double)lam, sl, cl);
  canon_sincos((double)phi, sp, cp);
  const double ux = __dmul_rn(cp, cl), uy = __dmul_rn(cp, sl), uz = sp;
  hi = make_float4(__double2float_rn(ux), __double2float_rn(uy), __double2float_rn(uz), 0.f);
  lo = make_float4(__double2float_rn(__dsub_rn(ux, (double)hi.x)), __double2float_rn(__dsub_rn(uy, (double)hi.y)),
                   __double2float_rn(__dsub_rn(uz, (double)hi.z)), 0.f);
}

// Canonical FP64 bin of a pair on the sphere (the guard-band path).
__device__ __forceinline__ int slow_bin_s(float4 ha, float4 la, float4 hb, float4 lb, const double* e2,
                                              int nb) {
  const double dx = __dsub_rn(__dadd_rn((double)hb.x, (double)lb.x), __dadd_rn((double)ha.x, (double)la.x));
  const double dy = __dsub_rn(__dadd_rn((double)hb.y, (double)lb.y), __dadd_rn((double)ha.y, (double)la.y));
  const double dz = __dsub_rn(__dadd_rn((double)hb.z, (double)lb.z), __dadd_rn((double)ha.z, (double)la.z));
  const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
  if (!(d2 >= e2[0]) || d2 > e2[nb]) return -1;
  if (d2 == e2[nb]) return nb - 1;
  int lo = 0, hi = nb;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (d2 >= e2[mid]) lo = mid; else hi = mid;
  }
  return lo;
}

// ------------------------------------------------------------ pair terms ----
// One lens: unit vector hi/lo and its local east/north basis.
struct LensS {
  float4 h, l;
  float ex, ey, nx, ny, nz;
};

__device__ __forceinline__ LensS lens_frame(float4 h, float4 l) {
  LensS L;
  L.h = h;
  L.l = l;
  const double ux = (double)h.x + (double)l.x, uy = (double)h.y + (double)l.y, uz = (double)h.z + (double)l.z;
  const double rho = sqrt(ux * ux + uy * uy);
  if (rho > 0.0) {
    L.ex = (float)(-uy / rho); L.ey = (float)(ux / rho);
    L.nx = (float)(-uz * ux / rho); L.ny = (float)(-uz * uy / rho); L.nz = (float)rho;
  } else {  // exactly on a pole: any tangent basis
    L.ex = 0.f; L.ey = 1.f; L.nx = uz > 0 ? -1.f : 1.f; L.ny = 0.f; L.nz = 0.f;
  }
  return L;
}

// theta = 2 asin(c/2) from c^2 and c.  SMALL (c <= 0.25): the series
// c (1 + c^2/24 + 3 c^4/640 + 5 c^6/7168), truncation < 2e-9 relative.
template <bool SMALL>
__device__ __forceinline__ float chord_theta(float d2, float c) {
  if (SMALL) return c * fmaf(d2, fmaf(d2, fmaf(d2, 6.9754464e-4f, 4.6875e-3f), 4.16666679e-2f), 1.f);
  return 2.f * asinf(fminf(0.5f * c, 1.f));
}
// theta^2 / c^2 by the same series (log-spaced binning in theta^2).
__device__ __forceinline__ float chord_theta2(float d2) {
  const float g = fmaf(d2, fmaf(d2, fmaf(d2, 6.9754464e-4f, 4.6875e-3f), 4.16666679e-2f), 1.f);
  return d2 * g * g;
}

// d2 = c^2, th = theta, r = 1/(A^2+B^2), X = p P + q U, Y = q P - p U with
// P = A^2 - B^2, U = 2AB (shear); scalar: r = 1, X = p, Y = q.
template <int MODE, bool SMALL>
__device__ __forceinline__ void sph_terms(const LensS& L, const float4 a, const float4 b, float& d2, float& th,
                                          float& r, float& X, float& Y) {
  const float dx = (a.x - L.h.x) + (b.x - L.l.x);
  const float dy = (a.y - L.h.y) + (b.y - L.l.y);
  const float dz = (a.z - L.h.z) + (b.z - L.l.z);
  d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
  // series path: binned pairs have d2 > 0; otherwise c = 0 exactly at d2 = 0
  const float c = SMALL ? d2 * rsqrtf(d2) : sqrtf(d2);
  th = chord_theta<SMALL>(d2, c);
  if (MODE == 0) {
    const float A = fmaf(dy, L.ey, dx * L.ex);
    const float B = fmaf(dz, L.nz, fmaf(dy, L.ny, dx * L.nx));
    const float A2 = A * A;
    const float P = fmaf(-B, B, A2);
    const float s = fmaf(B, B, A2);
    const float ab = A * B;
    const float U = ab + ab;
    r = __fdividef(1.f, s);
    X = fmaf(a.w, P, b.w * U);
    Y = fmaf(b.w, P, -(a.w * U));
  } else {
    r = 1.f;
    X = a.w;
    Y = b.w;
  }
}

template <bool LOGB>
__device__ __forceinline__ int pair_bin_s(float d2, const LensS& L, const float4 a, const float4 b,
                                          const BinCtx& C) {
  if (LOGB) {
    const float t = fmaf(__log2f(chord_theta2(d2)), C.A, C.B);
    const float tf = floorf(t);
    const float fr = t - tf;
    int bin = __float2int_rz(tf);
    if (fr < C.eps || fr > C.one_m_eps) bin = slow_bin_s(L.h, L.l, a, b, C.e2s, C.nb);
    return bin;
  } else {
    if (d2 < C.lo_g || d2 > C.hi_g) return -1;
    int lo = 0, hi = C.nb;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (d2 >= C.e2f[mid]) lo = mid; else hi = mid;
    }
    const float el = C.e2f[lo], eh = C.e2f[lo + 1];
    if (d2 <= el * (1.f + C.eps) || d2 >= eh * (1.f - C.eps)) lo = slow_bin_s(L.h, L.l, a, b, C.e2s, C.nb);
    return lo;
  }
}

// Conservative bin class of a 3-D box (min mn, max mx of the chunk's hi parts,
// already widened by the hi/lo split error) for one lens; classes as in the
// planar kernel.
template <bool LOGB, bool HAS_Z>
__device__ __forceinline__ int classify_s(const LensS& L, const float4 mn, const float4 mx, const BinCtx& C,
                                          int& blo) {
  const float dxl = fmaxf(fmaxf(mn.x - L.h.x, L.h.x - mx.x), 0.f);
  const float dyl = fmaxf(fmaxf(mn.y - L.h.y, L.h.y - mx.y), 0.f);
  const float dzl = fmaxf(fmaxf(mn.z - L.h.z, L.h.z - mx.z), 0.f);
  const float dxh = fmaxf(L.h.x - mn.x, mx.x - L.h.x);
  const float dyh = fmaxf(L.h.y - mn.y, mx.y - L.h.y);
  const float dzh = fmaxf(L.h.z - mn.z, mx.z - L.h.z);
  const float dmin2 = fmaf(dzl, dzl, fmaf(dyl, dyl, dxl * dxl));
  const float dmax2 = fmaf(dzh, dzh, fmaf(dyh, dyh, dxh * dxh));
  int b0, b1;
  if (LOGB) {
    b0 = __float2int_rd(fmaf(__log2f(chord_theta2(dmin2)), C.A, C.B) - C.eps);
    b1 = __float2int_rd(fmaf(__log2f(chord_theta2(dmax2)), C.A, C.B) + C.eps);
  } else {
    b0 = edge_index_f32(dmin2 * (1.f - C.eps), C.e2f, C.nb);
    b1 = edge_index_f32(dmax2 * (1.f + C.eps), C.e2f, C.nb);
  }
  if (b1 < 0 || b0 >= C.nb) return 0;
  b0 = max(b0, -1);  // every bin below 0 or from nb up is dropped alike
  b1 = min(b1, C.nb);
  blo = b0;
  if (b0 == b1) return 1;  // a z cut is applied inside the register paths
  if (b1 == b0 + 1) return 2;
  return 3;
}

template <int MODE, bool HAS_M, bool HAS_Z, bool LOGB, bool SMALL, int NC, int QA>
__device__ __forceinline__ void do_pair_s(const LensS& L, float lz, const SrcRecS& s, float* __restrict__ hcol,
                                          const BinCtx& C) {
  if (HAS_Z) {
    if (lz > s.c.z) return;  // src/tpcf.f90:322
  }
  float d2, th, r, X, Y;
  sph_terms<MODE, SMALL>(L, s.a, s.b, d2, th, r, X, Y);
  const int bin = pair_bin_s<LOGB>(d2, L, s.a, s.b, C);
  if ((unsigned)bin >= (unsigned)C.nb) return;
  float* h = hcol + bin * (QA * NC);
  h[QGT * NC] = fmaf(r, X, h[QGT * NC]);
  h[QGX * NC] = fmaf(r, Y, h[QGX * NC]);
  h[QW * NC] += s.c.x;
  h[QDW * NC] = fmaf(th, s.c.x, h[QDW * NC]);
  h[QN * NC] += 1.0f;
  if (MODE == 0 && HAS_M) h[QK * NC] += s.c.y;
}

// Two consecutive sources (2k, 2k+1) of a 32-source sub-chunk in shared
// memory with their fields interleaved, so that a 64-bit register pair holds
// one field of both (the operand form of the sm_100 packed FP32
// instructions).  The kernel rewrites each tile in place into this form (the
// same 96 bytes as the two SrcRecS).  p, q = a.w, b.w of SrcRecS; w, K, z =
// c.x, c.y, c.z.
struct __align__(16) SrcPairS {
  float4 hxy;  // hi.x0 hi.x1 hi.y0 hi.y1
  float4 hzp;  // hi.z0 hi.z1 p0 p1
  float4 lxy;  // lo.x0 lo.x1 lo.y0 lo.y1
  float4 lzq;  // lo.z0 lo.z1 q0 q1
  float4 wk;   // w0 w1 K0 K1
  float4 zz;   // z0 z1 0 0
};
static_assert(sizeof(SrcPairS) == 2 * sizeof(SrcRecS), "a SrcPairS rewrites two SrcRecS in place");

// Source j of a sub-chunk in SrcPairS form, as a SrcRecS.
__device__ __forceinline__ SrcRecS src_of_s(const SrcPairS* __restrict__ S, int j) {
  const float* f = reinterpret_cast<const float*>(S + (j >> 1)) + (j & 1);
  SrcRecS r;
  r.a = make_float4(f[0], f[2], f[4], f[6]);
  r.b = make_float4(f[8], f[10], f[12], f[14]);
  r.c = make_float4(f[16], f[18], f[20], 0.f);
  return r;
}

// One source in both halves of a SrcPairS (the odd last source of a sub-chunk;
// the second half is masked out by the step that takes it).
__device__ __forceinline__ SrcPairS dup_pair_s(const SrcRecS& r) {
  SrcPairS p;
  p.hxy = make_float4(r.a.x, r.a.x, r.a.y, r.a.y);
  p.hzp = make_float4(r.a.z, r.a.z, r.a.w, r.a.w);
  p.lxy = make_float4(r.b.x, r.b.x, r.b.y, r.b.y);
  p.lzq = make_float4(r.b.z, r.b.z, r.b.w, r.b.w);
  p.wk = make_float4(r.c.x, r.c.x, r.c.y, r.c.y);
  p.zz = make_float4(r.c.z, r.c.z, 0.f, 0.f);
  return p;
}

// A lens's constants in packed form: -hi, -lo and the east/north basis.
struct LensS2 {
  float2 nhx, nhy, nhz, nlx, nly, nlz, ex, ey, nx, ny, nz;
};
__device__ __forceinline__ LensS2 lens_pack(const LensS& L) {
  LensS2 P;
  P.nhx = dup2(-L.h.x); P.nhy = dup2(-L.h.y); P.nhz = dup2(-L.h.z);
  P.nlx = dup2(-L.l.x); P.nly = dup2(-L.l.y); P.nlz = dup2(-L.l.z);
  P.ex = dup2(L.ex); P.ey = dup2(L.ey);
  P.nx = dup2(L.nx); P.ny = dup2(L.ny); P.nz = dup2(L.nz);
  return P;
}

// sph_terms for the two sources of one SrcPairS (packed FP32; each half
// equals the scalar computation: a.x - h.x = a.x + (-h.x)).
template <int MODE, bool SMALL>
__device__ __forceinline__ void sph_terms2(const LensS2& L, const SrcPairS& s, float2& d2, float2& th, float2& r,
                                           float2& X, float2& Y) {
  const float2 dx = add2(add2(lo2(s.hxy), L.nhx), add2(lo2(s.lxy), L.nlx));
  const float2 dy = add2(add2(hi2(s.hxy), L.nhy), add2(hi2(s.lxy), L.nly));
  const float2 dz = add2(add2(lo2(s.hzp), L.nhz), add2(lo2(s.lzq), L.nlz));
  d2 = fma2(dz, dz, fma2(dy, dy, mul2(dx, dx)));
  if (SMALL) {
    const float2 c = mul2(d2, make_float2(rsqrtf(d2.x), rsqrtf(d2.y)));
    th = mul2(c, fma2(d2, fma2(d2, fma2(d2, dup2(6.9754464e-4f), dup2(4.6875e-3f)), dup2(4.16666679e-2f)),
                      dup2(1.f)));
  } else {
    th = make_float2(chord_theta<false>(d2.x, sqrtf(d2.x)), chord_theta<false>(d2.y, sqrtf(d2.y)));
  }
  if (MODE == 0) {
    const float2 A = fma2(dy, L.ey, mul2(dx, L.ex));
    const float2 B = fma2(dz, L.nz, fma2(dy, L.ny, mul2(dx, L.nx)));
    const float2 A2 = mul2(A, A);
    const float2 P = fma2(make_float2(-B.x, -B.y), B, A2);
    const float2 sq = fma2(B, B, A2);
    const float2 ab = mul2(A, B);
    const float2 U = add2(ab, ab);
    r = make_float2(__fdividef(1.f, sq.x), __fdividef(1.f, sq.y));
    X = fma2(hi2(s.hzp), P, mul2(hi2(s.lzq), U));
    const float2 pU = mul2(hi2(s.hzp), U);
    Y = fma2(hi2(s.lzq), P, make_float2(-pU.x, -pU.y));
  } else {
    r = dup2(1.f);
    X = hi2(s.hzp);
    Y = hi2(s.lzq);
  }
}

// Register sums of one lens over a sub-chunk: all pairs (s*) and, in the
// one-edge path, the upper side (h*).
struct SphAcc {
  float2 sgt, sgx, sw, sdw, sk, sn, hgt, hgx, hw, hdw, hk, hn, nc;
};
__device__ __forceinline__ void sph_acc_zero(SphAcc& A) {
  A.sgt = A.sgx = A.sw = A.sdw = A.sk = A.sn = dup2(0.f);
  A.hgt = A.hgx = A.hw = A.hdw = A.hk = A.hn = A.nc = dup2(0.f);
}

// The two pairs of one SrcPairS against a lens (TAIL: only the first; the
// second half is a copy, masked out).  With a z cut a pair with z_A > z_B
// (src/tpcf.f90:322) adds nothing.  DUAL also forms the upper-side sums
// (pairs with d2 >= E, the side a 1.0/0.0 mask from one FP32 compare at
// Ehi = E (1 + eps), applied by multiplication) and counts the pairs between
// Elo = E (1 - eps) and Ehi, inside the guard band (A.nc).  Without a z cut
// the w and K sums of all pairs (and, scalar-scalar, the g sums) are the
// sub-chunk's totals, so they are not accumulated here.
template <int MODE, bool HAS_M, bool HAS_Z, bool SMALL, bool DUAL, bool TAIL>
__device__ __forceinline__ void sph_step(const LensS2& L, float lz, const SrcPairS& s, float Elo, float Ehi,
                                         SphAcc& A) {
  constexpr bool LI = !HAS_Z;
  float2 d2, th, r, X, Y;
  sph_terms2<MODE, SMALL>(L, s, d2, th, r, X, Y);
  float2 w = lo2(s.wk), K = hi2(s.wk);
  bool v0 = true, v1 = !TAIL;
  if (HAS_Z) {
    v0 = lz <= s.zz.x;
    v1 = v1 && lz <= s.zz.y;
  }
  const float2 vm = make_float2(v0 ? 1.f : 0.f, v1 ? 1.f : 0.f);
  if (HAS_Z || TAIL) {
    r = mul2(r, vm);
    w = mul2(w, vm);
    if (MODE == 0 && HAS_M) K = mul2(K, vm);
    if (HAS_Z) A.sn = add2(A.sn, vm);
  }
  if (!(LI && MODE == 1)) {
    A.sgt = fma2(r, X, A.sgt);
    A.sgx = fma2(r, Y, A.sgx);
  }
  if (!LI) A.sw = add2(A.sw, w);
  A.sdw = fma2(th, w, A.sdw);
  if (MODE == 0 && HAS_M && !LI) A.sk = add2(A.sk, K);
  if (DUAL) {
    float2 mh = make_float2(d2.x >= Ehi ? 1.f : 0.f, d2.y >= Ehi ? 1.f : 0.f);
    const float2 ml = make_float2(d2.x >= Elo ? 1.f : 0.f, d2.y >= Elo ? 1.f : 0.f);
    if (HAS_Z || TAIL) {
      A.nc = fma2(add2(ml, make_float2(-mh.x, -mh.y)), vm, A.nc);
      mh = mul2(mh, vm);
    } else {
      A.nc = add2(A.nc, add2(ml, make_float2(-mh.x, -mh.y)));
    }
    const float2 rm = mul2(r, mh);  // r, w, K carry the validity mask already
    const float2 wm = mul2(w, mh);
    A.hgt = fma2(rm, X, A.hgt);
    A.hgx = fma2(rm, Y, A.hgx);
    A.hw = add2(A.hw, wm);
    A.hdw = fma2(th, wm, A.hdw);
    A.hn = add2(A.hn, mh);
    if (MODE == 0 && HAS_M) A.hk = fma2(K, mh, A.hk);
  }
}

// Sums over all pairs of a sub-chunk; ss = {sum p, sum q, sum w, sum K}.
template <int MODE, bool HAS_M, bool HAS_Z, int QA>
__device__ __forceinline__ void sph_totals(const SphAcc& A, int cnt, const float4 ss, float* tot) {
  constexpr bool LI = !HAS_Z;
  tot[QGT] = (LI && MODE == 1) ? ss.x : sum2(A.sgt);
  tot[QGX] = (LI && MODE == 1) ? ss.y : sum2(A.sgx);
  tot[QW] = LI ? ss.z : sum2(A.sw);
  tot[QDW] = sum2(A.sdw);
  tot[QN] = HAS_Z ? sum2(A.sn) : (float)cnt;
  if (MODE == 0 && HAS_M) tot[QK] = LI ? ss.w : sum2(A.sk);
}

// Class 1: every pair of the chunk is in bin `blo`.
template <int MODE, bool HAS_M, bool HAS_Z, bool SMALL, int NC, int QA>
__device__ __forceinline__ void chunk_single_s(const SrcPairS* __restrict__ S, int cnt, const LensS2& L, float lz,
                                               int cls, int blo, float* __restrict__ hcol, const float4 ss) {
  SphAcc A;
  sph_acc_zero(A);
  const int np = cnt >> 1;
#pragma unroll 2
  for (int k = 0; k < np; ++k) sph_step<MODE, HAS_M, HAS_Z, SMALL, false, false>(L, lz, S[k], 0.f, 0.f, A);
  if (cnt & 1)
    sph_step<MODE, HAS_M, HAS_Z, SMALL, false, true>(L, lz, dup_pair_s(src_of_s(S, cnt - 1)), 0.f, 0.f, A);
  if (cls != 1) return;
  float acc[QA];
  sph_totals<MODE, HAS_M, HAS_Z, QA>(A, cnt, ss, acc);
  hist_add<QA, NC>(hcol, blo, acc);
}

// Class 2: pairs in bins blo and blo+1 (either may be out of range, then it is
// dropped); the edge between them is e2f[blo+1].
template <int MODE, bool HAS_M, bool HAS_Z, bool SMALL, int NC, int QA>
__device__ __forceinline__ void chunk_dual_s(const SrcPairS* __restrict__ S, int cnt, const LensS& Lf,
                                             const LensS2& L, float lz, int cls, int blo, float* __restrict__ hcol,
                                             const BinCtx& C, const float4 ss) {
  // lanes of class 1 (or 0) keep an edge no pair reaches
  const float E = C.e2f[min(max(blo + 1, 0), C.nb)];
  const float Elo = (cls == 2) ? E * (1.f - C.eps_rel) : 3.0e38f;
  const float Ehi = (cls == 2) ? E * (1.f + C.eps_rel) : 3.0e38f;
  SphAcc A;
  sph_acc_zero(A);
  const int np = cnt >> 1;
#pragma unroll 2
  for (int k = 0; k < np; ++k) sph_step<MODE, HAS_M, HAS_Z, SMALL, true, false>(L, lz, S[k], Elo, Ehi, A);
  if (cnt & 1)
    sph_step<MODE, HAS_M, HAS_Z, SMALL, true, true>(L, lz, dup_pair_s(src_of_s(S, cnt - 1)), Elo, Ehi, A);
  if (cls == 0) return;
  if (sum2(A.nc) != 0.f) {  // rare: a pair inside the guard band; the sub-chunk is binned pair by pair
    for (int j = 0; j < cnt; ++j) do_pair_s<MODE, HAS_M, HAS_Z, SMALL, SMALL, NC, QA>(Lf, lz, src_of_s(S, j), hcol, C);
    return;
  }
  float tot[QA], hi[QA];
  sph_totals<MODE, HAS_M, HAS_Z, QA>(A, cnt, ss, tot);
  hi[QGT] = sum2(A.hgt);
  hi[QGX] = sum2(A.hgx);
  hi[QW] = sum2(A.hw);
  hi[QDW] = sum2(A.hdw);
  hi[QN] = sum2(A.hn);
  if (MODE == 0 && HAS_M) hi[QK] = sum2(A.hk);
  if (cls == 1) {
    hist_add<QA, NC>(hcol, blo, tot);
    return;
  }
  float lo[QA];
#pragma unroll
  for (int q = 0; q < QA; ++q) lo[q] = tot[q] - hi[q];
  if (blo >= 0) hist_add<QA, NC>(hcol, blo, lo);
  if (blo + 1 < C.nb) hist_add<QA, NC>(hcol, blo + 1, hi);
}

// ------------------------------------------------------------ cell runs -----
constexpr float kTwoPiF = 6.28318548f;      // 2 pi rounded up to FP32
constexpr int kRowsS = kMaxRows / 4;        // rows per chunk: 3 runs each fit kMaxRows
#ifndef TPCF_SPH_TILE
#define TPCF_SPH_TILE 160
#endif
// Sources per shared-memory tile (48-byte records): the tile size sets how
// many blocks share an SM next to the FP32 histogram.
constexpr int kTileS = TPCF_SPH_TILE;
static_assert(kTileS % 32 == 0, "tiles hold whole 32-source sub-chunks");
constexpr int kFlushSrcS = 4096;  // FP32 histogram -> FP64 after about this many sources

// Lambda reach of a work item: full = every cell of a row, else the interval
// [box.x - dl, box.z + dl] modulo 2 pi.
__device__ __forceinline__ void sph_reach(const GridDesc& G, float4 box, float R, float m, float& dl, bool& full) {
  const float ps = fmaxf(fabsf(box.y), fabsf(box.w)) + m;
  full = false;
  dl = 0.f;
  if (ps + R >= 1.5707f) { full = true; return; }
  const float sr = sinf(R) / cosf(ps);
  if (!(sr < 0.999f)) { full = true; return; }
  dl = asinf(sr) * 1.0001f + m;
  if ((box.z - box.x) + 2.f * dl + 2.f * G.cell + 4.f * m >= 6.2831f) full = true;
}

// The runs of sorted sources in row cy whose cells may hold a source within R
// of the box; returns how many (0..3).  The shifted intervals are more than
// two cells apart, so no cell appears in two runs.
__device__ __forceinline__ int sph_row_spans(const GridDesc& G, float4 box, float R, float m, int cy, float dl,
                                             bool full, int2* out) {
  const float ylo = G.y0 + (float)cy * G.cell - m;
  const float yhi = G.y0 + (float)(cy + 1) * G.cell + m;
  const float dyr = fmaxf(0.f, fmaxf(ylo - box.w, box.y - yhi));
  if (dyr > R) return 0;
  const int base = cy * G.ncx;
  if (full) {
    out[0] = make_int2(G.cell_start[base], G.cell_start[base + G.ncx]);
    return 1;
  }
  const float a = box.x - dl, b = box.z + dl;
  const float xmax = G.x0 + (float)G.ncx * G.cell;
  int n = 0;
#pragma unroll
  for (int k = -1; k <= 1; ++k) {
    const float s = (float)k * kTwoPiF;
    if (b + s < G.x0 - m || a + s > xmax + m) continue;
    const int cx0 = clamp_floor((a + s - G.x0) * G.inv_cell, 0, G.ncx - 1);
    const int cx1 = clamp_floor((b + s - G.x0) * G.inv_cell, 0, G.ncx - 1);
    out[n++] = make_int2(G.cell_start[base + cx0], G.cell_start[base + cx1 + 1]);
  }
  return n;
}

// ------------------------------------------------------------ the kernel ----
struct SphSmem {
  size_t tiles, hist, bsum, e2s, fvw, fw, e2f, span0, span1, tpref, subbox, subsum, mbar, misc, total;
};
__host__ __device__ inline size_t align_up_s(size_t v, size_t a) { return (v + a - 1) / a * a; }
__host__ __device__ inline SphSmem sph_smem_layout(int nb, int qa, int bt) {
  SphSmem s;
  size_t o = 0;
  s.tiles = o; o += 2 * kTileS * sizeof(SrcRecS);
  s.hist = o;  o += (size_t)nb * qa * bt * sizeof(float);
  o = align_up_s(o, 16);
  s.bsum = o;  o += (size_t)kQ * nb * sizeof(double);
  s.e2s = o;   o += (size_t)(nb + 1) * sizeof(double);
  s.fvw = o;   o += (size_t)bt * sizeof(double);
  s.fw = o;    o += (size_t)bt * sizeof(double);
  s.e2f = o;   o += (size_t)(nb + 1) * sizeof(float);
  o = align_up_s(o, 16);
  s.span0 = o; o += kMaxRows * sizeof(int);
  s.span1 = o; o += kMaxRows * sizeof(int);
  s.tpref = o; o += (kMaxRows + 1) * sizeof(int);
  o = align_up_s(o, 16);
  s.subbox = o; o += 2 * (kTileS / 32) * sizeof(float4);
  s.subsum = o; o += (kTileS / 32) * sizeof(float4);
  s.mbar = o;  o += 2 * sizeof(uint64_t);
  s.misc = o;  o += 16;
  s.total = align_up_s(o, 128);
  return s;
}

// Persistent: each block takes (task, lens group) items from the queue and
// streams the item's source runs through shared memory (bulk copies,
// double-buffered, bounded waits), as the planar kernel does.
template <int MODE, bool HAS_M, bool HAS_Z, bool LOGB, int BT>
// Compiled for 3 blocks per SM (the shared-memory occupancy at 20 bins),
// which gives the compiler a register budget of up to 170 per thread.
__global__ void __launch_bounds__(BT, 3) k_pairs_sph(const PairParams P) {
  constexpr int QA = (MODE == 0 && HAS_M) ? 6 : 5;
  constexpr int NW = BT / 32;
  constexpr bool SMALL = LOGB;  // log spacing on the sphere is only chosen with chord(x_max) <= 0.25
  const int nb = P.nb;
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  extern __shared__ __align__(128) unsigned char smem[];
  const SphSmem Ls = sph_smem_layout(nb, QA, BT);
  SrcRecS* tiles = reinterpret_cast<SrcRecS*>(smem + Ls.tiles);
  float* hist = reinterpret_cast<float*>(smem + Ls.hist);
  double* bsum = reinterpret_cast<double*>(smem + Ls.bsum);
  double* e2s = reinterpret_cast<double*>(smem + Ls.e2s);
  double* fvw = reinterpret_cast<double*>(smem + Ls.fvw);
  double* fw = reinterpret_cast<double*>(smem + Ls.fw);
  float* e2f = reinterpret_cast<float*>(smem + Ls.e2f);
  int* span0 = reinterpret_cast<int*>(smem + Ls.span0);
  int* span1 = reinterpret_cast<int*>(smem + Ls.span1);
  int* tpref = reinterpret_cast<int*>(smem + Ls.tpref);
  float4* subbox = reinterpret_cast<float4*>(smem + Ls.subbox);
  float4* subsum = reinterpret_cast<float4*>(smem + Ls.subsum);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + Ls.mbar);
  int* sh_item = reinterpret_cast<int*>(smem + Ls.misc);

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

  uint32_t phase = 0u;
  uint32_t tcount = 0u;
  bool timed_out = false;
  float* __restrict__ hcol = hist + tid;
  for (int e = 0; e < nb * QA; ++e) hcol[e * BT] = 0.f;

  for (;;) {
    if (tid == 0) *sh_item = atomicAdd(P.queue_head, 1);
    __syncthreads();
    const int item = *sh_item;
    if (item >= P.n_items) break;
    const int2 it = P.items[item];
    const TaskDesc T = P.tasks[it.x];
    const LensDesc LD = P.lenses[T.lens_cat];
    const GridDesc G = P.grids[T.src_cat];
    const int g = it.y;
    const int gs = LD.group_start[g];
    const int nl = LD.group_start[g + 1] - gs;
    const bool act = tid < nl;
    LensS Lf;
    float lz = 0.f;
    double vw = 0.0, w = 0.0;
    double* lens_col = nullptr;
    if (act) {
      const float4 r = LD.rec[gs + tid];
      Lf = lens_frame(LD.pos[2 * (gs + tid)], LD.pos[2 * (gs + tid) + 1]);
      vw = (double)r.z * (double)r.w;
      w = (double)r.w;
      if (HAS_Z) lz = LD.z[gs + tid];
      if (P.lens_acc && T.lens_acc_off >= 0) lens_col = P.lens_acc + T.lens_acc_off + gs + tid;
    } else {
      Lf = lens_frame(make_float4(1.f, 0.f, 0.f, 0.f), make_float4(0.f, 0.f, 0.f, 0.f));
    }
    const LensS2 LP = lens_pack(Lf);
    fvw[tid] = vw;
    fw[tid] = w;
    const size_t lens_stride = (size_t)LD.n_valid;
    for (int e = tid; e < kQ * nb; e += BT) bsum[e] = 0.0;
    int since_flush = 0;
    const float4 box = LD.group_box[g];
    int cy0, cy1;
    row_range(G, box, P.R, T.margin, cy0, cy1);
    float dl;
    bool full;
    sph_reach(G, box, P.R, T.margin, dl, full);

    for (int c0 = cy0; c0 <= cy1; c0 += kRowsS) {
      const int nr = min(kRowsS, cy1 - c0 + 1);
      const int ns = 3 * nr;
      __syncthreads();
      for (int r = tid; r < nr; r += BT) {
        int2 sp[3];
        const int k = sph_row_spans(G, box, P.R, T.margin, c0 + r, dl, full, sp);
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          const int2 v = j < k ? sp[j] : make_int2(0, 0);
          span0[3 * r + j] = v.x;
          span1[3 * r + j] = v.y > v.x ? v.y : v.x;
        }
      }
      __syncthreads();
      if (tid == 0) {
        int acc = 0;
        for (int r = 0; r < ns; ++r) {
          tpref[r] = acc;
          acc += (span1[r] - span0[r] + kTileS - 1) / kTileS;
        }
        tpref[ns] = acc;
      }
      __syncthreads();
      const int ntiles = tpref[ns];
      int rc = 0, ri = 0;
      if (tid == 0 && ntiles > 0) {
        while (tpref[ri + 1] <= 0) ++ri;
        const int s0 = span0[ri];
        const int n0 = min(kTileS, span1[ri] - s0);
        const int bb = tcount & 1u;
        mbar_arrive_tx(&mbar[bb], (uint32_t)(n0 * sizeof(SrcRecS)));
        bulk_g2s(tiles + bb * kTileS, G.recs + s0, (uint32_t)(n0 * sizeof(SrcRecS)), &mbar[bb]);
      }
      for (int k = 0; k < ntiles; ++k) {
        if (tid == 0 && k + 1 < ntiles) {
          while (tpref[ri + 1] <= k + 1) ++ri;
          const int s1 = span0[ri] + (k + 1 - tpref[ri]) * kTileS;
          const int n1 = min(kTileS, span1[ri] - s1);
          const int bb = (tcount + k + 1) & 1u;
          mbar_arrive_tx(&mbar[bb], (uint32_t)(n1 * sizeof(SrcRecS)));
          bulk_g2s(tiles + bb * kTileS, G.recs + s1, (uint32_t)(n1 * sizeof(SrcRecS)), &mbar[bb]);
        }
        while (tpref[rc + 1] <= k) ++rc;
        const int s = span0[rc] + (k - tpref[rc]) * kTileS;
        const int n = min(kTileS, span1[rc] - s);
        const int bb = (tcount + k) & 1u;
        const bool ok = mbar_wait_bounded(&mbar[bb], (phase >> bb) & 1u);
        phase ^= (1u << bb);
        // not __restrict__: the sub-chunk pass rewrites these bytes in place
        const SrcRecS* S = tiles + bb * kTileS;
        const int nsub = (n + 31) >> 5;
        if (ok) {
          // One warp per 32-source sub-chunk: its 3-D box, widened by 2^-23
          // per side (the hi/lo split of both ends moves u_B - u_A by at most
          // 2^-24), its sums of p, q, w, K, and the rewrite of its records
          // into SrcPairS form (lanes 2k, 2k+1 trade halves with one shuffle
          // round; each lane stores only the 48 bytes of its own record).
          for (int sc = warp; sc < nsub; sc += NW) {
            const int j = sc * 32 + lane;
            float mnx = INFINITY, mny = INFINITY, mnz = INFINITY, mxx = -INFINITY, mxy = -INFINITY,
                  mxz = -INFINITY;
            const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
            float4 a = z4, b = z4, c = z4;
            if (j < n) {
              a = S[j].a;
              b = S[j].b;
              c = S[j].c;
              mnx = mxx = a.x;
              mny = mxy = a.y;
              mnz = mxz = a.z;
            }
            const bool odd = lane & 1;
            // even lane keeps {hi.x, hi.y, hi.z, p, lo.x, lo.y} of both, odd lane {lo.z, q, w, K, z}
            const float r0 = __shfl_xor_sync(0xffffffffu, odd ? a.x : b.z, 1);
            const float r1 = __shfl_xor_sync(0xffffffffu, odd ? a.y : b.w, 1);
            const float r2 = __shfl_xor_sync(0xffffffffu, odd ? a.z : c.x, 1);
            const float r3 = __shfl_xor_sync(0xffffffffu, odd ? a.w : c.y, 1);
            const float r4 = __shfl_xor_sync(0xffffffffu, odd ? b.x : c.z, 1);
            const float r5 = __shfl_xor_sync(0xffffffffu, b.y, 1);
            float4* dst = reinterpret_cast<float4*>(tiles + bb * kTileS + j);
            if (!odd) {
              dst[0] = make_float4(a.x, r0, a.y, r1);
              dst[1] = make_float4(a.z, r2, a.w, r3);
              dst[2] = make_float4(b.x, r4, b.y, r5);
            } else {
              dst[0] = make_float4(r0, b.z, r1, b.w);
              dst[1] = make_float4(r2, c.x, r3, c.y);
              dst[2] = make_float4(r4, c.z, 0.f, 0.f);
            }
            fence_proxy_async_smem();  // before the bulk copy that later refills this buffer
            float s0 = a.w, s1 = b.w, s2 = c.x, s3 = c.y;
#pragma unroll
            for (int o = 16; o; o >>= 1) {
              s0 += __shfl_xor_sync(0xffffffffu, s0, o);
              s1 += __shfl_xor_sync(0xffffffffu, s1, o);
              s2 += __shfl_xor_sync(0xffffffffu, s2, o);
              s3 += __shfl_xor_sync(0xffffffffu, s3, o);
            }
            if (lane == 0) subsum[sc] = make_float4(s0, s1, s2, s3);
#pragma unroll
            for (int o = 16; o; o >>= 1) {
              mnx = fminf(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
              mny = fminf(mny, __shfl_xor_sync(0xffffffffu, mny, o));
              mnz = fminf(mnz, __shfl_xor_sync(0xffffffffu, mnz, o));
              mxx = fmaxf(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
              mxy = fmaxf(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
              mxz = fmaxf(mxz, __shfl_xor_sync(0xffffffffu, mxz, o));
            }
            if (lane == 0) {
              const float d = 1.1920929e-7f;
              subbox[2 * sc] = make_float4(mnx - d, mny - d, mnz - d, 0.f);
              subbox[2 * sc + 1] = make_float4(mxx + d, mxy + d, mxz + d, 0.f);
            }
          }
        }
        if (__syncthreads_or(!ok)) timed_out = true;
        if (!timed_out) {
          for (int sc = 0; sc < nsub; ++sc) {
            const int base = sc * 32;
            const int cnt = min(32, n - base);
            int blo = 0;
            const int cls = act ? classify_s<LOGB, HAS_Z>(Lf, subbox[2 * sc], subbox[2 * sc + 1], C, blo) : 0;
            const int m = (int)__reduce_max_sync(0xffffffffu, (unsigned)cls);
            if (m == 0) continue;
            const SrcPairS* __restrict__ Sc = reinterpret_cast<const SrcPairS*>(S + base);
            if (m == 1) {
              chunk_single_s<MODE, HAS_M, HAS_Z, SMALL, BT, QA>(Sc, cnt, LP, lz, cls, blo, hcol, subsum[sc]);
            } else if (m == 2) {
              chunk_dual_s<MODE, HAS_M, HAS_Z, SMALL, BT, QA>(Sc, cnt, Lf, LP, lz, cls, blo, hcol, C, subsum[sc]);
            } else if (act) {
              for (int j = 0; j < cnt; ++j)
                do_pair_s<MODE, HAS_M, HAS_Z, LOGB, SMALL, BT, QA>(Lf, lz, src_of_s(Sc, j), hcol, C);
            }
          }
        }
        since_flush += n;
        if (since_flush >= (P.flush_src > 0 ? P.flush_src : kFlushSrcS)) {
          flush_hist<QA, BT>(hist, bsum, fvw, fw, nb, lens_col, lens_stride);
          since_flush = 0;
        }
        __syncthreads();
      }
      tcount += (uint32_t)ntiles;
    }
    flush_hist<QA, BT>(hist, bsum, fvw, fw, nb, lens_col, lens_stride);
    __syncthreads();
    double* out = P.item_sums + (size_t)(T.item_base + g) * kQ * nb;
    for (int e = tid; e < kQ * nb; e += BT) {
      const int q = e / nb;
      out[e] = (q == QK && QA == 5) ? bsum[e - (QK - QW) * nb] : bsum[e];
    }
    __syncthreads();
  }
  if (timed_out && tid == 0) atomicOr(P.err, kErrTimeout);
}

// ------------------------------------------------------------ prep kernels --
// lambda reduced to [0, 2 pi) (FP32; used only for the cell grid and the
// lens ordering, never in the pair arithmetic).
__global__ void k_wrap_lambda(const float* __restrict__ x, long long n, float* out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float v = x[i];
    float t = v - kTwoPiF * floorf(v * 0.159154937f);
    if (t < 0.f) t += kTwoPiF;
    if (t >= kTwoPiF) t -= kTwoPiF;
    out[i] = t;
  }
}

__global__ void k_src_gather_sph(const int* __restrict__ idx, int n_valid, int mode, const float* __restrict__ lam,
                                 const float* __restrict__ phi, const float* __restrict__ z,
                                 const float* __restrict__ f1, const float* __restrict__ f2,
                                 const float* __restrict__ w, const float* __restrict__ m, SrcRecS* rec) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_valid) return;
  const int i = idx[s];
  const float wi = w[i];
  float4 hi, lo;
  canon_unit(lam[i], phi[i], hi, lo);
  SrcRecS r;
  if (mode == 0) {
    hi.w = -(f1[i] * wi);
    lo.w = -(f2[i] * wi);
    const float mi = m ? m[i] : 0.f;
    r.c = make_float4(wi, wi * (1.0f + mi), z ? z[i] : 0.f, 0.f);
  } else {
    hi.w = f1[i] * wi;
    lo.w = f2[i] * wi;
    r.c = make_float4(wi, wi, 0.f, 0.f);
  }
  r.a = hi;
  r.b = lo;
  rec[s] = r;
}

// Unit vectors (hi, lo) of the sorted lenses; perm[s] = input index.
__global__ void k_lens_pos_sph(const int* __restrict__ perm, int n_valid, const float* __restrict__ lam,
                               const float* __restrict__ phi, float4* pos) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_valid) return;
  const int i = perm[s];
  float4 hi, lo;
  canon_unit(lam[i], phi[i], hi, lo);
  pos[2 * s] = hi;
  pos[2 * s + 1] = lo;
}

// Unit vectors (hi, lo) in input order (tests and diagnostics).
__global__ void k_unit_vectors(const float* __restrict__ lam, const float* __restrict__ phi, long long n,
                               float* hi, float* lo) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    float4 h, l;
    canon_unit(lam[i], phi[i], h, l);
    hi[3 * i] = h.x; hi[3 * i + 1] = h.y; hi[3 * i + 2] = h.z;
    lo[3 * i] = l.x; lo[3 * i + 1] = l.y; lo[3 * i + 2] = l.z;
  }
}

__global__ void k_item_cost_sph(const int2* __restrict__ items, int n_items, const TaskDesc* __restrict__ tasks,
                                const LensDesc* __restrict__ lenses, const GridDesc* __restrict__ grids, float R,
                                unsigned long long* cost, int* order) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_items) return;
  const int2 it = items[i];
  const TaskDesc T = tasks[it.x];
  const LensDesc L = lenses[T.lens_cat];
  const GridDesc G = grids[T.src_cat];
  const float4 box = L.group_box[it.y];
  int cy0, cy1;
  row_range(G, box, R, T.margin, cy0, cy1);
  float dl;
  bool full;
  sph_reach(G, box, R, T.margin, dl, full);
  unsigned long long s = 0;
  for (int cy = cy0; cy <= cy1; ++cy) {
    int2 sp[3];
    const int k = sph_row_spans(G, box, R, T.margin, cy, dl, full, sp);
    for (int j = 0; j < k; ++j)
      if (sp[j].y > sp[j].x) s += (unsigned long long)(sp[j].y - sp[j].x);
  }
  const unsigned long long nl = (unsigned long long)(L.group_start[it.y + 1] - L.group_start[it.y]);
  cost[i] = item_key(s * nl + 1, i);
  order[i] = i;
}

// --------------------------------------------------------- host launchers --
template <int MODE, bool HAS_M, bool HAS_Z, bool LOGB, int BT>
static cudaError_t launch_sph_t(const PairParams& P, int num_sms, cudaStream_t st, int* grid_out) {
  constexpr int QA = (MODE == 0 && HAS_M) ? 6 : 5;
  const size_t smem = sph_smem_layout(P.nb, QA, BT).total;
  auto kern = k_pairs_sph<MODE, HAS_M, HAS_Z, LOGB, BT>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, BT, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  int grid = per_sm * num_sms;
  if (grid > P.n_items) grid = P.n_items;
  if (grid < 1) grid = 1;
  *grid_out = grid;
  kern<<<grid, BT, smem, st>>>(P);
  return cudaGetLastError();
}

template <int MODE, bool HAS_M, bool HAS_Z, bool LOGB>
static cudaError_t launch_sph_bt(const PairParams& P, int bt, int num_sms, cudaStream_t st, int* grid) {
  if (bt == 128) return launch_sph_t<MODE, HAS_M, HAS_Z, LOGB, 128>(P, num_sms, st, grid);
  if (bt == 64) return launch_sph_t<MODE, HAS_M, HAS_Z, LOGB, 64>(P, num_sms, st, grid);
  return launch_sph_t<MODE, HAS_M, HAS_Z, LOGB, 32>(P, num_sms, st, grid);
}

cudaError_t launch_pairs_sph(const PairParams& P, int mode, bool has_m, bool has_z, bool logb, int bt, int num_sms,
                             cudaStream_t st, int* grid) {
  if (mode == 1) {
    return logb ? launch_sph_bt<1, false, false, true>(P, bt, num_sms, st, grid)
                : launch_sph_bt<1, false, false, false>(P, bt, num_sms, st, grid);
  }
  if (has_m) {
    if (has_z) return logb ? launch_sph_bt<0, true, true, true>(P, bt, num_sms, st, grid)
                           : launch_sph_bt<0, true, true, false>(P, bt, num_sms, st, grid);
    return logb ? launch_sph_bt<0, true, false, true>(P, bt, num_sms, st, grid)
                : launch_sph_bt<0, true, false, false>(P, bt, num_sms, st, grid);
  }
  if (has_z) return logb ? launch_sph_bt<0, false, true, true>(P, bt, num_sms, st, grid)
                         : launch_sph_bt<0, false, true, false>(P, bt, num_sms, st, grid);
  return logb ? launch_sph_bt<0, false, false, true>(P, bt, num_sms, st, grid)
              : launch_sph_bt<0, false, false, false>(P, bt, num_sms, st, grid);
}

static inline unsigned gdim_s(long long n, int b) {
  long long g = (n + b - 1) / b;
  if (g < 1) g = 1;
  if (g > 148 * 32) g = 148 * 32;
  return (unsigned)g;
}

cudaError_t launch_wrap_lambda(const float* x, long long n, float* out, cudaStream_t st) {
  if (n > 0) k_wrap_lambda<<<gdim_s(n, 256), 256, 0, st>>>(x, n, out);
  return cudaGetLastError();
}
cudaError_t launch_src_gather_sph(const int* idx, int n_valid, int mode, const float* lam, const float* phi,
                                  const float* z, const float* f1, const float* f2, const float* w, const float* m,
                                  SrcRecS* rec, cudaStream_t st) {
  if (n_valid > 0)
    k_src_gather_sph<<<(n_valid + 255) / 256, 256, 0, st>>>(idx, n_valid, mode, lam, phi, z, f1, f2, w, m, rec);
  return cudaGetLastError();
}
cudaError_t launch_lens_pos_sph(const int* perm, int n_valid, const float* lam, const float* phi, float4* pos,
                                cudaStream_t st) {
  if (n_valid > 0) k_lens_pos_sph<<<(n_valid + 255) / 256, 256, 0, st>>>(perm, n_valid, lam, phi, pos);
  return cudaGetLastError();
}
cudaError_t launch_unit_vectors(const float* lam, const float* phi, long long n, float* hi, float* lo,
                                cudaStream_t st) {
  if (n > 0) k_unit_vectors<<<gdim_s(n, 256), 256, 0, st>>>(lam, phi, n, hi, lo);
  return cudaGetLastError();
}
cudaError_t launch_item_cost_sph(const int2* items, int n_items, const TaskDesc* tasks, const LensDesc* lenses,
                                 const GridDesc* grids, float R, unsigned long long* cost, int* order,
                                 cudaStream_t st) {
  if (n_items > 0)
    k_item_cost_sph<<<(n_items + 127) / 128, 128, 0, st>>>(items, n_items, tasks, lenses, grids, R, cost,
                                                            order);
  return cudaGetLastError();
}

}  // namespace tpcf
