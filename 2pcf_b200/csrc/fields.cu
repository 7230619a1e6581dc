// fields.cu -- per-field preprocessing of spherical catalogues on the device:
// the rotation of a field away from the poles and the prime meridian that the
// reference's driver applies before a spherical pair count
// (rotate_data_from_poles_and_meridian, src/main.f90:953-1015, with
// rotation_sphere src/utils.f90:483-509 and distance_to_meridian_sphere
// src/utils.f90:579-599).
//
// The element work (min/max, the wrap of longitudes above pi, the median by a
// radix sort, the rotation) runs on the device; the host only takes the
// decisions on the four extremes, in FP32 as the reference does.  The library's
// own spherical kernels need no rotation (they handle poles and the wrap);
// this entry point exists so that a driver ported from the reference produces
// the same rotated coordinates, and with them the same position angles.

#include <cub/cub.cuh>

#include <cmath>
#include <string>
#include <vector>

#include "tpcf_b200.h"
#include "tpcf_ctx.h"
#include "tpcf_internal.cuh"
#include "tpcf_kernels.h"

namespace tpcf {

constexpr float kPiF = 3.14159274f;  // pi as the reference's single-precision parameter (utils.f90:5)

// x > pi  ->  x - 2 pi, in FP32 (src/main.f90:985, :1000).
__global__ void k_wrap_above_pi(float* x, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float v = x[i];
    if (v > kPiF) x[i] = __fsub_rn(v, __fmul_rn(2.0f, kPiF));
  }
}

// rotation_sphere (src/utils.f90:483-509) evaluated in FP64, rounded to FP32.
__global__ void k_rotate_sphere(float* lam, float* phi, long long n, double lam_rot, double phi_rot) {
  const double hp = 1.5707963267948966;
  const double tr = -phi_rot;
  const double ctr = cos(tr), str = sin(tr);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double sigma = (double)lam[i] + lam_rot;
    const double th = hp - (double)phi[i];
    const double cs = cos(sigma), ss = sin(sigma), ct = cos(th), st = sin(th);
    const double x = cs * ctr * st + ct * str;
    const double y = ss * st;
    const double z = -cs * str * st + ct * ctr;
    double lo = atan(y / x);
    if (x < 0.0) lo += 3.141592653589793;
    double po;
    if (z >= 1.0) po = hp;
    else if (z <= -1.0) po = -hp;
    else po = hp - acos(z);
    lam[i] = (float)lo;
    phi[i] = (float)po;
  }
}

static inline unsigned gdim_f(long long n) {
  long long g = (n + 255) / 256;
  if (g < 1) g = 1;
  if (g > 148 * 32) g = 148 * 32;
  return (unsigned)g;
}

}  // namespace tpcf

using namespace tpcf;

namespace {

// min/max of x and y over the finite entries (one sync).
void minmax(tpcf_ctx* c, const float* x, const float* y, long long n, float out[4]) {
  int* box_ord = (int*)ws_alloc(c, sizeof(int) * 8);
  unsigned long long* cnt = (unsigned long long*)ws_alloc(c, sizeof(unsigned long long));
  int* pr = (int*)ws_alloc(c, sizeof(int) * 2);
  float* boxf = (float*)ws_alloc(c, sizeof(float) * 8);
  counted(c, launch_bbox_init(box_ord, cnt, pr, 1, c->stream), "bbox init");
  counted(c, launch_bbox(x, y, nullptr, nullptr, nullptr, nullptr, n, 0, box_ord, cnt, pr, c->stream), "bbox");
  counted(c, launch_bbox_finish(box_ord, boxf, 8, c->stream), "bbox finish");
  float h[8];
  check(cudaMemcpyAsync(h, boxf, sizeof(h), cudaMemcpyDeviceToHost, c->stream), "D2H box");
  check(cudaStreamSynchronize(c->stream), "sync box");
  out[0] = h[0]; out[1] = h[2]; out[2] = h[1]; out[3] = h[3];  // xmin, xmax, ymin, ymax
}

// median (src/utils.f90:712-726): the (n/2+1)-th smallest, averaged with the
// (n/2)-th for even n, in FP32.
float median(tpcf_ctx* c, const float* x, long long n) {
  float* k0 = (float*)ws_alloc(c, sizeof(float) * n);
  size_t tb = 0;
  check(cub::DeviceRadixSort::SortKeys(nullptr, tb, x, k0, (int)n, 0, 32, c->stream), "sort size");
  void* tmp = ws_alloc(c, tb);
  check(cub::DeviceRadixSort::SortKeys(tmp, tb, x, k0, (int)n, 0, 32, c->stream), "sort median");
  float a = 0.f, b = 0.f;
  check(cudaMemcpyAsync(&a, k0 + n / 2, sizeof(float), cudaMemcpyDeviceToHost, c->stream), "D2H median");
  if (n % 2 == 0)
    check(cudaMemcpyAsync(&b, k0 + n / 2 - 1, sizeof(float), cudaMemcpyDeviceToHost, c->stream), "D2H median");
  check(cudaStreamSynchronize(c->stream), "sync median");
  return n % 2 == 0 ? (a + b) / 2.0f : a;
}

// distance_to_meridian_sphere (src/utils.f90:579-599), FP32.
float distance_to_meridian(float lambda1, float phi1, float lambda2) {
  const float sd = std::fabs(std::sin(lambda2 - lambda1) * std::cos(phi1));
  if (std::fabs(lambda2 - lambda1) <= kPiF / 2.0f) return sd >= 1.0f ? kPiF / 2.0f : std::asin(sd);
  return kPiF / 2.0f - std::fabs(phi1);
}

}  // namespace

extern "C" tpcf_status tpcf_rotate_from_poles(tpcf_ctx* c, float* xA, float* yA, int64_t nA, float* xB, float* yB,
                                              int64_t nB, float r_max, int32_t* rotated, float* center) {
  if (!c || !xA || !yA || nA <= 0 || nA > (1ll << 31) - 2 || nB < 0 || (nB > 0 && (!xB || !yB)) || !rotated)
    return TPCF_ERR_INVALID_ARG;
  try {
    begin_call(c);
    cudaStream_t st = c->stream;
    // device copies (in place when the caller passed device memory)
    auto dev = [&](float* p, int64_t n) -> float* {
      if (!p || n <= 0) return nullptr;
      return const_cast<float*>(stage<float>(c, p, n));
    };
    float* dxA = dev(xA, nA);
    float* dyA = dev(yA, nA);
    float* dxB = dev(xB, nB);
    float* dyB = dev(yB, nB);
    float mm[4];
    minmax(c, dxA, dyA, nA, mm);
    bool rot = false;
    if (mm[3] + r_max >= kPiF / 2.0f) rot = true;             // north pole in reach
    else if (mm[2] - r_max <= -kPiF / 2.0f) rot = true;       // south pole in reach
    if (mm[1] - mm[0] > kPiF) {                               // both sides of the prime meridian
      k_wrap_above_pi<<<gdim_f(nA), 256, 0, st>>>(dxA, nA);
      counted(c, cudaGetLastError(), "wrap");
      minmax(c, dxA, dyA, nA, mm);
      rot = true;
    } else if (distance_to_meridian(mm[1], mm[3], 0.0f) <= r_max || distance_to_meridian(mm[0], mm[3], 0.0f) <= r_max ||
               distance_to_meridian(mm[1], mm[2], 0.0f) <= r_max || distance_to_meridian(mm[0], mm[2], 0.0f) <= r_max) {
      rot = true;
    }
    if (dxB) {
      float mb[4];
      minmax(c, dxB, dyB, nB, mb);
      if (mb[1] - mb[0] > kPiF) {
        k_wrap_above_pi<<<gdim_f(nB), 256, 0, st>>>(dxB, nB);
        counted(c, cudaGetLastError(), "wrap");
      }
    }
    float cx = 0.f, cy = 0.f;
    if (rot) {
      cx = median(c, dxA, nA);
      cy = median(c, dyA, nA);
      const double lr = (double)(kPiF - cx), pr = (double)(-cy);
      k_rotate_sphere<<<gdim_f(nA), 256, 0, st>>>(dxA, dyA, nA, lr, pr);
      counted(c, cudaGetLastError(), "rotate");
      if (dxB) {
        k_rotate_sphere<<<gdim_f(nB), 256, 0, st>>>(dxB, dyB, nB, lr, pr);
        counted(c, cudaGetLastError(), "rotate");
      }
    }
    auto back = [&](float* user, float* d, int64_t n) {
      if (d && d != user) copy_out(c, user, d, sizeof(float) * n);
    };
    back(xA, dxA, nA); back(yA, dyA, nA); back(xB, dxB, nB); back(yB, dyB, nB);
    check(cudaStreamSynchronize(st), "sync rotate");
    *rotated = rot ? 1 : 0;
    if (center) { center[0] = cx; center[1] = cy; }
    return TPCF_OK;
  } catch (const Failure& f) {
    c->err = f.msg;
    return f.status;
  }
}
