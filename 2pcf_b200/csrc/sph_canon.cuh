// sph_canon.cuh -- the canonical FP64 sine and cosine of the spherical path,
// shared by the device (unit vectors of the objects) and the host (squared
// chord edges (2 sin(e/2))^2 of the bins).
//
// One fixed sequence of IEEE-rounded FP64 operations, never contracted into
// FMAs: Cody-Waite reduction by pi/2 with a three-part split of pi/2 (each
// k * part exact for |k| < 2^20), then Taylor series through r^17 (sine) and
// r^18 (cosine) on |r| <= pi/4 (truncation below 1e-19).  The result does not
// depend on the host's libm or on the compiler, so the oracle reproduces it
// bit for bit.
#pragma once
#include <cmath>
#include <cuda_runtime.h>

namespace tpcf {
namespace sphc {
constexpr double kTwoOverPi = 0.6366197723675814;
constexpr double kPio2_1 = 1.5707963267341256;      // pi/2 to 33 bits
constexpr double kPio2_2 = 6.077100506303966e-11;   // next 33 bits
constexpr double kPio2_3 = 2.0222662487959506e-21;  // remainder
// 1/n!
constexpr double kF3 = 0.16666666666666666, kF5 = 0.008333333333333333, kF7 = 0.0001984126984126984,
                 kF9 = 2.7557319223985893e-06, kF11 = 2.505210838544172e-08, kF13 = 1.6059043836821613e-10,
                 kF15 = 7.647163731819816e-13, kF17 = 2.8114572543455206e-15;
constexpr double kF4 = 0.041666666666666664, kF6 = 0.001388888888888889, kF8 = 2.48015873015873e-05,
                 kF10 = 2.755731922398589e-07, kF12 = 2.08767569878681e-09, kF14 = 1.1470745597729725e-11,
                 kF16 = 4.779477332387385e-14, kF18 = 1.5619206968586225e-16;

__host__ __device__ __forceinline__ double mul(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dmul_rn(a, b);
#else
  return a * b;  // host objects are built with -ffp-contract=off
#endif
}
__host__ __device__ __forceinline__ double add(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dadd_rn(a, b);
#else
  return a + b;
#endif
}
__host__ __device__ __forceinline__ double sub(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dsub_rn(a, b);
#else
  return a - b;
#endif
}
}  // namespace sphc

__host__ __device__ inline void canon_sincos(double x, double& s, double& c) {
  using namespace sphc;
  const double k = rint(mul(x, kTwoOverPi));
  double r = sub(x, mul(k, kPio2_1));
  r = sub(r, mul(k, kPio2_2));
  r = sub(r, mul(k, kPio2_3));
  const double z = mul(r, r);
  double ps = kF17;
  ps = sub(mul(ps, z), kF15);
  ps = add(mul(ps, z), kF13);
  ps = sub(mul(ps, z), kF11);
  ps = add(mul(ps, z), kF9);
  ps = sub(mul(ps, z), kF7);
  ps = add(mul(ps, z), kF5);
  ps = sub(mul(ps, z), kF3);
  const double sr = add(r, mul(mul(r, z), ps));
  double pc = -kF18;
  pc = add(mul(pc, z), kF16);
  pc = sub(mul(pc, z), kF14);
  pc = add(mul(pc, z), kF12);
  pc = sub(mul(pc, z), kF10);
  pc = add(mul(pc, z), kF8);
  pc = sub(mul(pc, z), kF6);
  pc = add(mul(pc, z), kF4);
  const double cr = add(1.0, add(mul(-0.5, z), mul(mul(z, z), pc)));
  switch ((int)((long long)k & 3)) {
    case 0: s = sr; c = cr; break;
    case 1: s = cr; c = -sr; break;
    case 2: s = -sr; c = -cr; break;
    default: s = -cr; c = sr; break;
  }
}

// Squared chord of an FP64 angle: (2 sin(e/2))^2.
__host__ __device__ inline double canon_chord2(double e) {
  double s, c;
  canon_sincos(sphc::mul(e, 0.5), s, c);
  const double ch = sphc::mul(2.0, s);
  return sphc::mul(ch, ch);
}

}  // namespace tpcf
