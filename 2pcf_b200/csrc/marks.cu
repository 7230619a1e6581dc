// marks.cu -- xi from precomputed per-lens marks (calculate_tpcf_from_marks,
// src/main.f90:1017-1139): for each foreground map m and field i,
//   g_t[b] = sum_j xi_E[j][b] val_mj w_mj / sum_j K[j][b] w_mj,
//   g_x[b] = sum_j xi_B[j][b] val_mj w_mj / sum_j K[j][b] w_mj,
//   weights = sum_j mw_j w_mj,
// over the lenses j with mw_j w_mj > 0 (the reference packs the others away,
// :1089-1104), and the fields stacked by summing numerators and K
// (:1127-1135).  The marks were computed once with val = w = 1; each new map
// only re-weights them, so this is a streaming pass over the marks (HBM-bound:
// 12 bytes per lens and bin, plus 8 bytes per lens and map).
//
// One block = 1024 lenses of one field and up to kMapGroup maps (register
// sums per marks row, FP64), per-block partial sums in scratch, then a
// fixed-order reduction over blocks (deterministic).

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "philox.cuh"
#include "tpcf_b200.h"
#include "tpcf_ctx.h"
#include "tpcf_internal.cuh"
#include "tpcf_kernels.h"

namespace tpcf {

constexpr int kMapGroup = 16;     // maps or resamples per pass over the marks

struct MarksField {
  long long n;
  int n_bin;
  int chunk0;               // first block of this field
  long long lens0;          // index of the field's first lens among all fields
  const float* mw;          // marks weight [n]
  const float* xiE;         // [n][n_bin]
  const float* xiB;
  const float* K;
  const float* val;         // maps: [n_map][n]
  const float* w;           // maps: [n_map][n]
};

// Asynchronous copies global -> shared (cp.async) of 4 or 16 bytes; with
// valid == false nothing is read and the destination is zero-filled.
__device__ __forceinline__ void cp_async4(void* dst, const void* src, bool valid) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(
                   static_cast<unsigned>(__cvta_generic_to_shared(dst))),
               "l"(src), "r"(valid ? 4 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(
                   static_cast<unsigned>(__cvta_generic_to_shared(dst))),
               "l"(src), "r"(valid ? 16 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
__device__ __forceinline__ bool al16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Copies `rows` runs of 64 consecutive 4-byte values, run k from src(k) (a
// device pointer to the run's first value), into dst[k * 64 ..], by all
// threads of the block: valid values are the first nt of each run of the
// first live_rows runs, the rest is zero-filled.  16-byte chunks when the
// tile is whole and every run starts on a 16-byte boundary (vec), else 4-byte
// copies.
template <class SrcOf>
__device__ __forceinline__ void stage_runs(void* dst, int rows, int live_rows, int nt, bool vec, SrcOf src, int tid,
                                           int nthr) {
  unsigned char* d = reinterpret_cast<unsigned char*>(dst);
  if (vec) {
    for (int e = tid; e < rows * 16; e += nthr) {
      const int k = e >> 4, c = e & 15;
      const bool v = k < live_rows;
      cp_async16(d + (size_t)(k * 64 + 4 * c) * 4, v ? reinterpret_cast<const unsigned char*>(src(k)) + 16 * c
                                                        : reinterpret_cast<const unsigned char*>(src(0)), v);
    }
  } else {
    for (int e = tid; e < rows * 64; e += nthr) {
      const int k = e >> 6, jj = e & 63;
      const bool v = k < live_rows && jj < nt;
      cp_async4(d + (size_t)e * 4, v ? reinterpret_cast<const unsigned char*>(src(k)) + 4 * jj
                                      : reinterpret_cast<const unsigned char*>(src(0)), v);
    }
  }
}

// Lens factors of resample/map g for lens jj of a tile.  stage() starts the
// copies of the raw inputs of one tile into shared memory (all threads);
// factors() turns the landed raw values into the numerator factor vw and the
// K factor wm (both 0 for a lens that takes no part).
struct MapFactors {  // foreground maps: vw = val w, wm = w
  static constexpr bool kSame = false;  // vw and wm differ: two factor arrays
  int map0;
  static constexpr size_t kRawBytes = sizeof(float) * (2 * kMapGroup + 1) * 64;
  // raw: val [kMapGroup][64], w [kMapGroup][64], marks weight [64]
  __device__ __forceinline__ void stage(const MarksField& F, long long t0, int nt, int n_g, unsigned char* raw,
                                        int tid, int nthr) const {
    float* rv = reinterpret_cast<float*>(raw);
    const bool vec = nt == 64 && al16(F.val) && al16(F.w) && al16(F.mw) && (F.n & 3) == 0 && (t0 & 3) == 0;
    const size_t o = (size_t)map0 * (size_t)F.n + (size_t)t0;
    const float* val = F.val;
    const float* w = F.w;
    const long long n = F.n;
    stage_runs(rv, kMapGroup, n_g, nt, vec, [&](int k) { return val + o + (size_t)k * n; }, tid, nthr);
    stage_runs(rv + kMapGroup * 64, kMapGroup, n_g, nt, vec, [&](int k) { return w + o + (size_t)k * n; }, tid,
               nthr);
    const float* mw = F.mw + t0;
    stage_runs(rv + 2 * kMapGroup * 64, 1, 1, nt, vec, [&](int) { return mw; }, tid, nthr);
  }
  __device__ __forceinline__ void factors(const unsigned char* raw, int g, int jj, double& vw, double& wm) const {
    const float* rv = reinterpret_cast<const float*>(raw);
    wm = (double)rv[kMapGroup * 64 + g * 64 + jj];
    vw = (double)rv[g * 64 + jj] * wm;
    // calculate_tpcf_from_marks drops lenses with marks weight x weight <= 0
    if (!((double)rv[2 * kMapGroup * 64 + jj] * wm > 0.0)) vw = wm = 0.0;
  }
};
struct MultFactors {  // resamples: vw = wm = multiplicity of the lens's unit
  static constexpr bool kSame = true;  // one factor array serves every row
  const int* mult;    // [G][n_units]
  const int* unit;    // unit of each lens (all fields concatenated), or nullptr: the lens itself
  long long n_units;
  static constexpr size_t kRawBytes = sizeof(int) * kMapGroup * 64;
  __device__ __forceinline__ void stage(const MarksField& F, long long t0, int nt, int n_g, unsigned char* raw,
                                        int tid, int nthr) const {
    int* rm = reinterpret_cast<int*>(raw);
    const long long gl0 = F.lens0 + t0;
    if (!unit) {  // each lens its own unit: runs of consecutive multiplicities
      const bool vec = nt == 64 && al16(mult) && (n_units & 3) == 0 && (gl0 & 3) == 0;
      const int* m = mult + gl0;
      const long long nu = n_units;
      stage_runs(rm, kMapGroup, n_g, nt, vec, [&](int k) { return m + (size_t)k * nu; }, tid, nthr);
      return;
    }
    for (int e = tid; e < kMapGroup * 64; e += nthr) {  // gathered through the unit labels
      const int g = e >> 6, jj = e & 63;
      const bool v = g < n_g && jj < nt;
      const size_t o = v ? (size_t)g * (size_t)n_units + (size_t)__ldg(unit + gl0 + jj) : 0;
      cp_async4(rm + e, mult + o, v);
    }
  }
  // the bootstraps take every drawn lens (src/tpcf.f90:601, :917, :1248)
  __device__ __forceinline__ void factors(const unsigned char* raw, int g, int jj, double& vw, double& wm) const {
    const int m = reinterpret_cast<const int*>(raw)[g * 64 + jj];
    wm = m > 0 ? (double)m : 0.0;
    vw = wm;
  }
};

// partial[(blk * n_g + g) * R + r], R = 3 n_bin + 1 (E, B, K rows, weight).
//
// A block is NG lens groups of TG = 32 ceil(R / 32) threads; thread r of a
// group owns row r of the marks (xi_E, xi_B, K of bin r mod n_bin, or the
// marks weight) and keeps the kMapGroup sums of that row in registers.  The
// block takes kMarksLens lenses in tiles of kTileL.  While the block sums one
// tile, the raw inputs of the next tile's lens factors (per map and lens;
// consecutive threads copy consecutive lenses of one map) are already being
// copied into shared memory (cp.async), so no load latency is exposed and no
// register holds them; after a barrier they become the FP64 factors (zero for
// lenses left out) of the next tile.  Group k takes lenses k, k + NG, ...:
// each thread loads its row of the lens (the group's 32-lane loads cover the
// lens's contiguous marks) and adds it times the n_g factors (FP64 FMA, one
// chain per map).  Streaming the marks once per pass with all n_g maps
// applied keeps the pass near the FP64 roofline.  The groups are summed in
// fixed order at the end (deterministic, no atomics).
//
// The factors of one lens are stored as [vw of the 16 maps | 2 pad | wm of
// the 16 maps | 2 pad] (kLensStride doubles): the summing loop reads its
// half as 8 aligned double2, and a warp whose rows read both halves (E/B rows
// and K/weight rows) hits disjoint banks, as do the 32 lanes of one
// conversion store (one map, 32 lenses).
constexpr int kTileL = 64;
constexpr int kLensStride = 2 * (kMapGroup + 2);
constexpr int kWmOffset = kMapGroup + 2;
constexpr int kMarksLens = 1024;  // lenses per block
// Threads per block at most: one group of 3 kMaxBins + 1 = 385 rows fits, and
// two blocks per SM leave 78 registers per thread (the 16 FP64 sums and the
// staged factor pairs in flight without spilling).
constexpr int kMarksThreads = 416;
static_assert(kTileL == 64, "the raw staging areas hold 64 lenses");
// With STAGE the marks of the next tile (xi_E, xi_B, K [kTileL][n_bin] and the
// marks weight [kTileL], as laid out in HBM) are copied into shared memory by
// cp.async together with the factors' raw inputs, into the other of two
// buffers, so the summing loop reads only shared memory and no global load
// latency is exposed; for wide binnings (marks_stage_floats too large) the
// loop loads the marks from HBM itself.
int marks_stage_floats(int n_bin) { return 3 * kTileL * n_bin + kTileL; }
constexpr int kMaxStageFloats = 3 * kTileL * 32 + kTileL;  // n_bin <= 32
template <class Fac, bool STAGE>
__global__ void __launch_bounds__(kMarksThreads, 2) k_marks_partials(const MarksField* __restrict__ fields, int n_field,
                                                            const Fac fac, int n_g, int n_bin, int tg,
                                                            double* __restrict__ partial) {
  extern __shared__ __align__(16) unsigned char sm[];
  constexpr int TF = kTileL * kLensStride;
  const int R = 3 * n_bin + 1;
  const int ng = blockDim.x / tg;
  double* fac_s = reinterpret_cast<double*>(sm);  // [kTileL][kLensStride] factors of every row
  unsigned char* raw = sm + TF * sizeof(double);
  float* mk = reinterpret_cast<float*>(raw + std::max(MapFactors::kRawBytes, MultFactors::kRawBytes));
  const int MS = 3 * kTileL * n_bin + kTileL;  // floats per marks buffer
  const int blk = blockIdx.x;
  int fi = 0;
  while (fi + 1 < n_field && fields[fi + 1].chunk0 <= blk) ++fi;
  const MarksField& F = fields[fi];  // read where used: its pointers need no registers across the loop
  const long long j0 = (long long)(blk - F.chunk0) * kMarksLens;
  const long long j1 = min(F.n, j0 + kMarksLens);
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int grp = tid / tg, r = tid % tg;
  const int q = r / n_bin, bb = r - q * n_bin;  // q = 3: the marks weight row
  const bool live = r < R;
  const double* fsel = (q < 2 || Fac::kSame) ? fac_s : fac_s + kWmOffset;
  // this thread's marks row: in HBM (lens stride rs) or in a staged buffer
  const float* row = q == 0 ? F.xiE + bb : q == 1 ? F.xiB + bb : q == 2 ? F.K + bb : F.mw;
  const long long rs = q < 3 ? n_bin : 1;
  const int srow = q < 3 ? q * kTileL * n_bin + bb : 3 * kTileL * n_bin;

  auto stage_tile = [&](long long t0, int buf) {
    const int nt = (int)min((long long)kTileL, j1 - t0);
    fac.stage(F, t0, nt, n_g, raw, tid, nthr);
    if (STAGE) {
      // the tile's marks as laid out in HBM: [nt][n_bin] of each quantity, the weights
      float* mb = mk + buf * MS;
      const size_t o = (size_t)t0 * n_bin;
      const int nq = nt * n_bin, cap = kTileL * n_bin;
      const bool vec = nt == kTileL && al16(F.xiE + o) && al16(F.xiB + o) && al16(F.K + o);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const float* src = (k == 0 ? F.xiE : k == 1 ? F.xiB : F.K) + o;
        if (vec) {
          for (int e = tid; e < cap / 4; e += nthr) cp_async16(mb + k * cap + 4 * e, src + 4 * e, true);
        } else {
          for (int e = tid; e < cap; e += nthr) cp_async4(mb + k * cap + e, src + (e < nq ? e : 0), e < nq);
        }
      }
      const float* mw = F.mw + t0;
      stage_runs(mb + 3 * cap, 1, 1, nt, nt == kTileL && al16(mw), [&](int) { return mw; }, tid, nthr);
    }
  };
  auto convert_tile = [&]() {
    for (int e = tid; e < kTileL * kMapGroup; e += nthr) {
      const int g = e >> 6, jj = e & 63;
      double vw, wm;
      fac.factors(raw, g, jj, vw, wm);
      fac_s[jj * kLensStride + g] = vw;
      if (!Fac::kSame) fac_s[jj * kLensStride + kWmOffset + g] = wm;
    }
  };

  double acc[kMapGroup];
#pragma unroll
  for (int g = 0; g < kMapGroup; ++g) acc[g] = 0.0;
  if (j0 < j1) stage_tile(j0, 0);
  cp_async_wait_all();
  __syncthreads();
  if (j0 < j1) convert_tile();
  __syncthreads();
  int buf = 0;
  for (long long t0 = j0; t0 < j1; t0 += kTileL) {
    const int nt = (int)min((long long)kTileL, j1 - t0);
    const bool more = t0 + kTileL < j1;
    // the raw area was read before the last barrier, the other marks buffer
    // before the one ahead of it
    if (more) stage_tile(t0 + kTileL, buf ^ 1);
    if (live) {
      const float* base = STAGE ? mk + buf * MS + srow : row + t0 * rs;
#pragma unroll 1
      for (int jj = grp; jj < nt; jj += ng) {
        const double m = STAGE ? (double)base[jj * rs] : (double)__ldg(base + jj * rs);
        const double2* f2 = reinterpret_cast<const double2*>(fsel + jj * kLensStride);
#pragma unroll
        for (int h = 0; h < kMapGroup / 2; ++h) {
          const double2 f = f2[h];
          acc[2 * h] = fma(m, f.x, acc[2 * h]);
          acc[2 * h + 1] = fma(m, f.y, acc[2 * h + 1]);
        }
      }
    }
    cp_async_wait_all();
    __syncthreads();  // the next tile's copies landed; this tile's factors and marks are no longer read
    if (more) {
      convert_tile();
      __syncthreads();
    }
    buf ^= 1;
  }
  // groups 1.. add their sums into group 0's, in group order
  double* red = fac_s;  // [tg][kMapGroup]
  for (int k = 1; k < ng; ++k) {
    __syncthreads();
    if (grp == k) {
#pragma unroll
      for (int g = 0; g < kMapGroup; ++g) red[r * kMapGroup + g] = acc[g];
    }
    __syncthreads();
    if (grp == 0) {
#pragma unroll
      for (int g = 0; g < kMapGroup; ++g) acc[g] += red[r * kMapGroup + g];
    }
  }
  if (grp == 0 && live) {
#pragma unroll
    for (int g = 0; g < kMapGroup; ++g)
      if (g < n_g) partial[((size_t)blk * n_g + g) * R + r] = acc[g];
  }
}

// Threads per lens group (one per marks row, whole warps) and per block: as
// many groups as fit in kMarksThreads.
int marks_group_threads(int n_bin) { return (3 * n_bin + 1 + 31) / 32 * 32; }
int marks_block_threads(int n_bin) {
  const int tg = marks_group_threads(n_bin);
  return (kMarksThreads / tg) * tg;
}
bool marks_stage(int n_bin) { return marks_stage_floats(n_bin) <= kMaxStageFloats; }
size_t marks_smem(int n_bin) {
  size_t fac = sizeof(double) * kTileL * kLensStride + std::max(MapFactors::kRawBytes, MultFactors::kRawBytes);
  if (marks_stage(n_bin)) fac += 2 * sizeof(float) * (size_t)marks_stage_floats(n_bin);
  const size_t red = sizeof(double) * (size_t)marks_group_threads(n_bin) * kMapGroup;
  return std::max(fac, red);
}
// One pass of k_marks_partials over all fields (the staged form when the
// binning is narrow enough).
template <class Fac>
cudaError_t launch_marks_partials(const MarksField* fields, int n_field, int nblk, const Fac& fac, int n_g, int nb,
                                  double* part, cudaStream_t st) {
  const size_t msm = marks_smem(nb);
  const int bt = marks_block_threads(nb), tg = marks_group_threads(nb);
  if (marks_stage(nb)) {
    cudaError_t e = cudaFuncSetAttribute(k_marks_partials<Fac, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)msm);
    if (e != cudaSuccess) return e;
    k_marks_partials<Fac, true><<<nblk, bt, msm, st>>>(fields, n_field, fac, n_g, nb, tg, part);
  } else {
    cudaError_t e = cudaFuncSetAttribute(k_marks_partials<Fac, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)msm);
    if (e != cudaSuccess) return e;
    k_marks_partials<Fac, false><<<nblk, bt, msm, st>>>(fields, n_field, fac, n_g, nb, tg, part);
  }
  return cudaGetLastError();
}

// maps or resamples per pass over the marks
int marks_group(int) { return kMapGroup; }

// Multiplicities of G resamples s0.. over n_units units: n_draw draws each,
// counter (d/4, s, 0x2BCF, 0), word d%4, index by multiply-shift (the stream
// of the patch bootstrap).  mult must be zeroed.
__global__ void k_unit_mult(unsigned long long seed, long long n_units, long long n_draw, int s0, int G,
                            int* mult) {
  const long long nq = (n_draw + 3) / 4;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nq * G;
       t += (long long)gridDim.x * blockDim.x) {
    const int g = (int)(t / nq);
    const long long q = t % nq;
    uint32_t c[4] = {(uint32_t)q, (uint32_t)(s0 + g), 0x2BCFu, 0u};
    philox4x32(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    for (int u = 0; u < 4; ++u) {
      const long long d = 4 * q + u;
      if (d < n_draw) {
        const long long idx = (long long)(((unsigned long long)c[u] * (unsigned long long)n_units) >> 32);
        atomicAdd(&mult[(size_t)g * (size_t)n_units + (size_t)idx], 1);
      }
    }
  }
}

// Field sums: out[(g * n_field + fi) * R + r] = sum over the field's blocks.
// One warp per output: lane l adds blocks l, l + 32, ... of the field, then
// the lanes are combined by a fixed shuffle tree (the same order every run).
__global__ void k_marks_reduce(const double* __restrict__ partial, const MarksField* __restrict__ fields,
                               int n_field, int n_blocks, int n_map_g, int R, double* __restrict__ out) {
  const int t = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (t >= n_map_g * n_field * R) return;  // whole warps
  const int r = t % R, fi = (t / R) % n_field, g = t / (R * n_field);
  const int c0 = fields[fi].chunk0;
  const int c1 = fi + 1 < n_field ? fields[fi + 1].chunk0 : n_blocks;
  double s = 0.0;
  for (int c = c0 + lane; c < c1; c += 32) s += partial[((size_t)c * n_map_g + g) * R + r];
#pragma unroll
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) out[t] = s;
}

// Flags a unit label outside [0, n_units).
__global__ void k_check_units(const int* __restrict__ unit, long long n, long long n_units, int* bad) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    if (unit[i] < 0 || (long long)unit[i] >= n_units) atomicOr(bad, 1);
}

// max |a - b| over n entries, as order-preserving bits of a non-negative float.
__global__ void k_max_absdiff(const float* __restrict__ a, const float* __restrict__ b, long long n, int* out) {
  float m = 0.f;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float d = fabsf(a[i] - b[i]);
    m = fmaxf(m, d != d ? INFINITY : d);
  }
  for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_int(m));
}

}  // namespace tpcf

using namespace tpcf;

extern "C" tpcf_status tpcf_xi_from_marks(tpcf_ctx* c, int32_t n_field, const tpcf_marks_field* marks,
                                          int32_t n_map, const float* const* val, const float* const* w,
                                          const float* const* lens_x, const float* const* lens_y, double* g_t,
                                          double* g_x, double* weights, double* g_t_stacked,
                                          double* g_x_stacked, double* weights_stacked) {
  if (!c || n_field < 1 || !marks || n_map < 1 || !val || !w) return TPCF_ERR_INVALID_ARG;
  const int nb = (int)marks[0].n_bin;
  if (nb < 1 || nb > kMaxBins) return TPCF_ERR_INVALID_ARG;
  for (int i = 0; i < n_field; ++i) {
    const tpcf_marks_field& m = marks[i];
    if (m.n_bin != nb || m.n < 0 || m.n > (1ll << 31) - 2 || !val[i] || !w[i]) return TPCF_ERR_INVALID_ARG;
    if (m.n > 0 && (!m.w || !m.xi_E || !m.xi_B || !m.K)) return TPCF_ERR_INVALID_ARG;
  }
  try {
    Phase ph_nvtx("tpcf: marks");
    begin_call(c);
    cudaStream_t st = c->stream;
    std::vector<MarksField> hf(n_field);
    int nblk = 0;
    for (int i = 0; i < n_field; ++i) {
      const tpcf_marks_field& m = marks[i];
      const int64_t n = m.n;
      MarksField& F = hf[i];
      F.n = n;
      F.n_bin = nb;
      F.chunk0 = nblk;
      F.lens0 = 0;
      nblk += (int)((n + kMarksLens - 1) / kMarksLens);
      F.mw = stage(c, m.w, n);
      F.xiE = stage(c, m.xi_E, n * nb);
      F.xiB = stage(c, m.xi_B, n * nb);
      F.K = stage(c, m.K, n * nb);
      F.val = stage(c, val[i], n * n_map);
      F.w = stage(c, w[i], n * n_map);
      // the lenses must be the ones the marks were computed for (main.f90:1036-1049)
      if (lens_x && lens_y && lens_x[i] && lens_y[i] && n > 0) {
        if (!m.x || !m.y) throw Failure(TPCF_ERR_INVALID_ARG, "marks positions missing for the check");
        const float* a[2] = {stage(c, m.x, n), stage(c, m.y, n)};
        const float* b[2] = {stage(c, lens_x[i], n), stage(c, lens_y[i], n)};
        int* dm = (int*)ws_alloc(c, sizeof(int) * 2);
        check(cudaMemsetAsync(dm, 0, sizeof(int) * 2, st), "memset");
        for (int k = 0; k < 2; ++k) {
          k_max_absdiff<<<(unsigned)std::min<int64_t>((n + 255) / 256, 148 * 8), 256, 0, st>>>(a[k], b[k], n, dm + k);
          counted(c, cudaGetLastError(), "position check");
        }
        int hm[2];
        check(cudaMemcpyAsync(hm, dm, sizeof(hm), cudaMemcpyDeviceToHost, st), "D2H check");
        check(cudaStreamSynchronize(st), "sync check");
        for (int k = 0; k < 2; ++k) {
          float d;
          std::memcpy(&d, &hm[k], 4);
          if (!(d <= 1.0e-5f))
            throw Failure(TPCF_ERR_INVALID_ARG, std::string(k ? "Y" : "X") + "-coordinates of lenses do not match in field " +
                                                    std::to_string(i));
        }
      }
    }
    MarksField* df = (MarksField*)ws_alloc(c, sizeof(MarksField) * n_field);
    check(cudaMemcpyAsync(df, hf.data(), sizeof(MarksField) * n_field, cudaMemcpyHostToDevice, st), "H2D fields");
    const int R = 3 * nb + 1;
    std::vector<double> sums((size_t)n_map * n_field * R, 0.0);
    double* part = (double*)ws_alloc(c, sizeof(double) * (size_t)std::max(nblk, 1) * kMapGroup * R);
    double* dout = (double*)ws_alloc(c, sizeof(double) * (size_t)kMapGroup * n_field * R);
    const int MG = marks_group(nb);
    for (int m0 = 0; m0 < n_map; m0 += MG) {
      const int g = std::min(MG, n_map - m0);
      if (nblk > 0) counted(c, launch_marks_partials(df, n_field, nblk, MapFactors{m0}, g, nb, part, st), "marks partials");
      const int tot = g * n_field * R;
      if (nblk > 0) {
        k_marks_reduce<<<(tot + 7) / 8, 256, 0, st>>>(part, df, n_field, nblk, g, R, dout);
        counted(c, cudaGetLastError(), "marks reduce");
      } else {
        check(cudaMemsetAsync(dout, 0, sizeof(double) * tot, st), "memset");
      }
      check(cudaMemcpyAsync(sums.data() + (size_t)m0 * n_field * R, dout, sizeof(double) * tot,
                            cudaMemcpyDeviceToHost, st), "D2H sums");
    }
    check(cudaStreamSynchronize(st), "sync marks");
    // normalisation (main.f90:1118-1133): plain quotients, as the reference
    for (int m = 0; m < n_map; ++m) {
      std::vector<double> sE(nb, 0.0), sB(nb, 0.0), sK(nb, 0.0);
      double sw = 0.0;
      for (int i = 0; i < n_field; ++i) {
        const double* s = sums.data() + ((size_t)m * n_field + i) * R;
        for (int b = 0; b < nb; ++b) {
          if (g_t) g_t[((size_t)m * n_field + i) * nb + b] = s[b] / s[2 * nb + b];
          if (g_x) g_x[((size_t)m * n_field + i) * nb + b] = s[nb + b] / s[2 * nb + b];
          sE[b] += s[b];
          sB[b] += s[nb + b];
          sK[b] += s[2 * nb + b];
        }
        if (weights) weights[(size_t)m * n_field + i] = s[3 * nb];
        sw += s[3 * nb];
      }
      for (int b = 0; b < nb; ++b) {
        if (g_t_stacked) g_t_stacked[(size_t)m * nb + b] = sE[b] / sK[b];
        if (g_x_stacked) g_x_stacked[(size_t)m * nb + b] = sB[b] / sK[b];
      }
      if (weights_stacked) weights_stacked[m] = sw;
    }
    return TPCF_OK;
  } catch (const Failure& f) {
    c->err = f.msg;
    return f.status;
  }
}

extern "C" tpcf_status tpcf_marks_bootstrap(tpcf_ctx* c, int32_t n_field, const tpcf_marks_field* marks,
                                            const int32_t* unit, int64_t n_units, const int32_t* multiplicity,
                                            uint64_t seed, int32_t n_boot, double supersampling, int32_t k_guard,
                                            double* g_t, double* g_x, double* weights, double* cov_gt,
                                            double* cov_gx) {
  if (!c || n_field < 1 || !marks || n_boot < 1 || !(supersampling > 0)) return TPCF_ERR_INVALID_ARG;
  const int nb = (int)marks[0].n_bin;
  if (nb < 1 || nb > kMaxBins) return TPCF_ERR_INVALID_ARG;
  int64_t n_lens = 0;
  for (int i = 0; i < n_field; ++i) {
    const tpcf_marks_field& m = marks[i];
    if (m.n_bin != nb || m.n < 0 || (m.n > 0 && (!m.w || !m.xi_E || !m.xi_B || !m.K))) return TPCF_ERR_INVALID_ARG;
    n_lens += m.n;
  }
  if (n_lens > (1ll << 31) - 2) return TPCF_ERR_INVALID_ARG;
  if (!unit) n_units = n_lens;
  if (n_units < 1) return TPCF_ERR_INVALID_ARG;
  try {
    Phase ph_nvtx("tpcf: marks bootstrap");
    begin_call(c);
    cudaStream_t st = c->stream;
    std::vector<MarksField> hf(n_field);
    int nblk = 0;
    int64_t off = 0;
    for (int i = 0; i < n_field; ++i) {
      const tpcf_marks_field& m = marks[i];
      MarksField& F = hf[i];
      F.n = m.n;
      F.n_bin = nb;
      F.chunk0 = nblk;
      F.lens0 = off;
      off += m.n;
      nblk += (int)((m.n + kMarksLens - 1) / kMarksLens);
      F.mw = stage(c, m.w, m.n);
      F.xiE = stage(c, m.xi_E, m.n * nb);
      F.xiB = stage(c, m.xi_B, m.n * nb);
      F.K = stage(c, m.K, m.n * nb);
      F.val = F.w = nullptr;
    }
    const int* dunit = unit ? stage(c, (const int*)unit, n_lens) : nullptr;
    if (dunit) {  // labels must lie in [0, n_units): checked on the device before use
      int* bad = (int*)ws_alloc(c, sizeof(int));
      check(cudaMemsetAsync(bad, 0, sizeof(int), st), "memset");
      k_check_units<<<(unsigned)std::min<int64_t>((n_lens + 255) / 256, 148 * 8), 256, 0, st>>>(dunit, n_lens, n_units,
                                                                                                   bad);
      counted(c, cudaGetLastError(), "unit check");
      int hb = 0;
      check(cudaMemcpyAsync(&hb, bad, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H check");
      check(cudaStreamSynchronize(st), "sync check");
      if (hb) throw Failure(TPCF_ERR_INVALID_ARG, "unit label outside [0, n_units)");
    }
    const int* dmult_all = multiplicity ? stage(c, (const int*)multiplicity, (int64_t)n_boot * n_units) : nullptr;
    // n_samples = int(n_objects * supersampling_factor) (src/tpcf.f90:1234, :894)
    const long long n_draw = (long long)((double)n_units * supersampling);
    if (!multiplicity && n_draw < 1) throw Failure(TPCF_ERR_INVALID_ARG, "no draws per resample");
    MarksField* df = (MarksField*)ws_alloc(c, sizeof(MarksField) * n_field);
    check(cudaMemcpyAsync(df, hf.data(), sizeof(MarksField) * n_field, cudaMemcpyHostToDevice, st), "H2D fields");
    const int R = 3 * nb + 1;
    int* mbuf = multiplicity ? nullptr : (int*)ws_alloc(c, sizeof(int) * (size_t)kMapGroup * n_units);
    double* part = (double*)ws_alloc(c, sizeof(double) * (size_t)std::max(nblk, 1) * kMapGroup * R);
    double* dout = (double*)ws_alloc(c, sizeof(double) * (size_t)kMapGroup * n_field * R);
    std::vector<double> sums((size_t)n_boot * n_field * R, 0.0);
    const int MG = marks_group(nb);
    for (int s0 = 0; s0 < n_boot; s0 += MG) {
      const int G = std::min(MG, n_boot - s0);
      const int* mult;
      if (multiplicity) {
        mult = dmult_all + (size_t)s0 * n_units;
      } else {
        check(cudaMemsetAsync(mbuf, 0, sizeof(int) * (size_t)G * n_units, st), "memset mult");
        const long long work = (n_draw + 3) / 4 * G;
        k_unit_mult<<<(unsigned)std::min<long long>((work + 255) / 256, 148 * 16), 256, 0, st>>>(seed, n_units, n_draw,
                                                                                                 s0, G, mbuf);
        counted(c, cudaGetLastError(), "bootstrap draws");
        mult = mbuf;
      }
      if (nblk > 0) {
        counted(c, launch_marks_partials(df, n_field, nblk, MultFactors{mult, dunit, n_units}, G, nb, part, st),
                "bootstrap partials");
        const int tot = G * n_field * R;
        k_marks_reduce<<<(tot + 7) / 8, 256, 0, st>>>(part, df, n_field, nblk, G, R, dout);
        counted(c, cudaGetLastError(), "bootstrap reduce");
        check(cudaMemcpyAsync(sums.data() + (size_t)s0 * n_field * R, dout, sizeof(double) * tot,
                              cudaMemcpyDeviceToHost, st), "D2H sums");
      }
    }
    check(cudaStreamSynchronize(st), "sync bootstrap");
    // all fields together (src/tpcf.f90:1245-1262); K > 0 guard of the point
    // bootstraps, plain quotients for the pair-weighted block bootstrap (:929-930)
    std::vector<double> gt((size_t)n_boot * nb), gx((size_t)n_boot * nb);
    for (int s = 0; s < n_boot; ++s) {
      double W = 0.0;
      for (int b = 0; b < nb; ++b) {
        double E = 0.0, B = 0.0, K = 0.0;
        for (int i = 0; i < n_field; ++i) {
          const double* r = sums.data() + ((size_t)s * n_field + i) * R;
          E += r[b];
          B += r[nb + b];
          K += r[2 * nb + b];
        }
        const bool zero = k_guard && !(K > 0.0);
        gt[(size_t)s * nb + b] = zero ? 0.0 : E / K;
        gx[(size_t)s * nb + b] = zero ? 0.0 : B / K;
      }
      for (int i = 0; i < n_field; ++i) W += sums[((size_t)s * n_field + i) * R + 3 * nb];
      if (weights) weights[s] = W;
    }
    if (g_t) std::memcpy(g_t, gt.data(), sizeof(double) * gt.size());
    if (g_x) std::memcpy(g_x, gx.data(), sizeof(double) * gx.size());
    if ((cov_gt || cov_gx) && n_boot >= 2) {
      double* dg = (double*)ws_alloc(c, sizeof(double) * gt.size());
      double* dc = (double*)ws_alloc(c, sizeof(double) * (size_t)nb * nb);
      for (int q = 0; q < 2; ++q) {
        double* user = q == 0 ? cov_gt : cov_gx;
        if (!user) continue;
        check(cudaMemcpyAsync(dg, (q == 0 ? gt : gx).data(), sizeof(double) * gt.size(), cudaMemcpyHostToDevice, st),
              "H2D g");
        counted(c, launch_cov(dg, n_boot, nb, dc, st), "covariance");
        check(cudaMemcpyAsync(user, dc, sizeof(double) * nb * nb, cudaMemcpyDefault, st), "D2H cov");
        check(cudaStreamSynchronize(st), "sync cov");
      }
    }
    return TPCF_OK;
  } catch (const Failure& f) {
    c->err = f.msg;
    return f.status;
  }
}
