// marks.cu -- xi from precomputed per-lens marks (calculate_tpcf_from_marks,
// src/main.f90:1017-1139): for each foreground map m and field i,
//   g_t[b] = sum_j xi_E[j][b] val_mj w_mj / sum_j K[j][b] w_mj,
//   g_x[b] = sum_j xi_B[j][b] val_mj w_mj / sum_j K[j][b] w_mj,
//   weights = sum_j mw_j w_mj,
// over the lenses j with mw_j w_mj > 0 (the reference packs the others away,
// :1089-1104), and the fields stacked by summing numerators and K
// (:1127-1135).  The marks were computed once with val = w = 1; each new map
// only re-weights them, so this is a streaming pass over the marks: 12 bytes
// per lens and bin plus 8 bytes per lens and map against 2 FP64 FLOP per lens,
// row and map, which puts 16 maps per pass on both the HBM and the FP64
// roofline.
//
// One block = a run of lenses of one field and up to kMapGroup maps
// (register-tiled FP64 sums, rows x maps), per-block partial sums in scratch,
// then a fixed-order reduction over blocks (deterministic).

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "philox.cuh"
#include "tpcf_b200.h"
#include "tpcf_ctx.h"
#include "tpcf_device.cuh"
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

// Raw factor inputs of a tile in shared memory: one row of 64 lenses per map
// or resample, rows kRawStride floats apart (16-byte aligned rows; the
// conversion's warps read 16 maps x 2 lenses, at most two lanes per bank).
constexpr int kRawStride = 68;

// Copies `rows` runs of 64 consecutive 4-byte values, run k from src(k) (a
// device pointer to the run's first value), into dst rows kRawStride values
// apart, by all threads of the block: valid values are the first nt of each
// run of the first live_rows runs, the rest is zero-filled.  16-byte chunks
// when the tile is whole and every run starts on a 16-byte boundary (vec),
// else 4-byte copies.
template <class SrcOf>
__device__ __forceinline__ void stage_runs(void* dst, int rows, int live_rows, int nt, bool vec, SrcOf src, int tid,
                                           int nthr) {
  unsigned char* d = reinterpret_cast<unsigned char*>(dst);
  if (vec) {
    for (int e = tid; e < rows * 16; e += nthr) {
      const int k = e >> 4, c = e & 15;
      const bool v = k < live_rows;
      cp_async16(d + (size_t)(k * kRawStride + 4 * c) * 4,
                 v ? reinterpret_cast<const unsigned char*>(src(k)) + 16 * c
                   : reinterpret_cast<const unsigned char*>(src(0)), v);
    }
  } else {
    for (int e = tid; e < rows * 64; e += nthr) {
      const int k = e >> 6, jj = e & 63;
      const bool v = k < live_rows && jj < nt;
      cp_async4(d + (size_t)(k * kRawStride + jj) * 4,
                v ? reinterpret_cast<const unsigned char*>(src(k)) + 4 * jj
                  : reinterpret_cast<const unsigned char*>(src(0)), v);
    }
  }
}

// Lens factors of resample/map g for lens jj of a tile.  stage() starts the
// copies of the raw inputs of one tile into shared memory (all threads);
// stage_bulk() does the same for a whole, aligned tile (bulk_ok) by
// bulk_bytes() of one-thread bulk copies signalled on an mbarrier (rows past
// n_g are not copied); factors() turns the landed raw values into the
// numerator factor vw and the K factor wm (both 0 for a lens that takes no
// part).
struct MapFactors {  // foreground maps: vw = val w, wm = w
  static constexpr bool kSame = false;  // vw and wm differ: two factor arrays
  int map0;
  static constexpr size_t kRawBytes = sizeof(float) * (2 * kMapGroup + 1) * kRawStride;
  // raw rows: val of the kMapGroup maps, w of the kMapGroup maps, marks weight
  __device__ __forceinline__ void stage(const MarksField& F, long long t0, int nt, int n_g, unsigned char* raw,
                                        int tid, int nthr) const {
    float* rv = reinterpret_cast<float*>(raw);
    const bool vec = nt == 64 && al16(F.val) && al16(F.w) && al16(F.mw) && (F.n & 3) == 0 && (t0 & 3) == 0;
    const size_t o = (size_t)map0 * (size_t)F.n + (size_t)t0;
    const float* val = F.val;
    const float* w = F.w;
    const long long n = F.n;
    stage_runs(rv, kMapGroup, n_g, nt, vec, [&](int k) { return val + o + (size_t)k * n; }, tid, nthr);
    stage_runs(rv + kMapGroup * kRawStride, kMapGroup, n_g, nt, vec, [&](int k) { return w + o + (size_t)k * n; },
               tid, nthr);
    const float* mw = F.mw + t0;
    stage_runs(rv + 2 * kMapGroup * kRawStride, 1, 1, nt, vec, [&](int) { return mw; }, tid, nthr);
  }
  __device__ __forceinline__ bool bulk_ok(const MarksField& F, long long t0, int nt) const {
    return nt == 64 && al16(F.val) && al16(F.w) && al16(F.mw) && (F.n & 3) == 0 && (t0 & 3) == 0;
  }
  __device__ __forceinline__ uint32_t bulk_bytes(int n_g) const { return 256u * (2 * n_g + 1); }
  __device__ __forceinline__ void stage_bulk(const MarksField& F, long long t0, int n_g, unsigned char* raw,
                                             uint64_t* bar) const {
    float* rv = reinterpret_cast<float*>(raw);
    const size_t o = (size_t)map0 * (size_t)F.n + (size_t)t0;
    for (int k = 0; k < n_g; ++k) {
      bulk_g2s(rv + k * kRawStride, F.val + o + (size_t)k * F.n, 256, bar);
      bulk_g2s(rv + (kMapGroup + k) * kRawStride, F.w + o + (size_t)k * F.n, 256, bar);
    }
    bulk_g2s(rv + 2 * kMapGroup * kRawStride, F.mw + t0, 256, bar);
  }
  __device__ __forceinline__ void factors(const unsigned char* raw, int g, int jj, double& vw, double& wm) const {
    const float* rv = reinterpret_cast<const float*>(raw);
    wm = (double)rv[(kMapGroup + g) * kRawStride + jj];
    vw = (double)rv[g * kRawStride + jj] * wm;
    // calculate_tpcf_from_marks drops lenses with marks weight x weight <= 0
    if (!((double)rv[2 * kMapGroup * kRawStride + jj] * wm > 0.0)) vw = wm = 0.0;
  }
};
struct MultFactors {  // resamples: vw = wm = multiplicity of the lens's unit
  static constexpr bool kSame = true;  // one factor array serves every row
  const int* mult;    // [G][n_units]
  const int* unit;    // unit of each lens (all fields concatenated), or nullptr: the lens itself
  long long n_units;
  static constexpr size_t kRawBytes = sizeof(int) * kMapGroup * kRawStride;
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
      cp_async4(rm + g * kRawStride + jj, mult + o, v);
    }
  }
  __device__ __forceinline__ bool bulk_ok(const MarksField& F, long long t0, int nt) const {
    return !unit && nt == 64 && al16(mult) && (n_units & 3) == 0 && ((F.lens0 + t0) & 3) == 0;
  }
  __device__ __forceinline__ uint32_t bulk_bytes(int n_g) const { return 256u * n_g; }
  __device__ __forceinline__ void stage_bulk(const MarksField& F, long long t0, int n_g, unsigned char* raw,
                                             uint64_t* bar) const {
    int* rm = reinterpret_cast<int*>(raw);
    const int* m = mult + F.lens0 + t0;
    for (int k = 0; k < n_g; ++k) bulk_g2s(rm + k * kRawStride, m + (size_t)k * n_units, 256, bar);
  }
  // the bootstraps take every drawn lens (src/tpcf.f90:601, :917, :1248)
  __device__ __forceinline__ void factors(const unsigned char* raw, int g, int jj, double& vw, double& wm) const {
    const int m = reinterpret_cast<const int*>(raw)[g * kRawStride + jj];
    wm = m > 0 ? (double)m : 0.0;
    vw = wm;
  }
};

// partial[(blk * n_g + g) * R + r], R = 3 n_bin + 1 (E, B, K rows, weight):
// a split-K product of the marks [lens][R] with the lens factors [lens][n_g]
// over the block's lenses.  This FP64 FMA form serves wide binnings
// (n_bin > 32, marks read from HBM by the summing loop); narrower ones run on
// the FP64 tensor cores (k_marks_dmma below).
//
// The rows come in quads: four consecutive bins of one quantity (xi_E, xi_B
// or K; the last quad of a quantity padded with zero bins) and one quad for
// the marks weight (the weight and three zeros).  A lens group is tg
// threads, lane 2 quad + half owning rows quad x maps 8 half .. 8 half + 7 as
// 32 FP64 register sums; per lens it loads its quad's marks (four values)
// and its 8 factors (four 16-byte shared-memory loads) and adds the 32
// products (FP64 FMA).
// The block takes `chunk` lenses of one field in tiles of kTileL; while it
// sums one tile the factors' raw inputs of the next are being copied
// (cp.async) into shared memory, and after a barrier they become the FP64
// factors (zero for lenses left out).  Group k takes the tile's lenses k,
// k + NG, ...; the groups are summed in fixed order at the end
// (deterministic, no atomics).
//
// The factors of one lens are stored as [vw of the 16 maps | 2 pad | wm of
// the 16 maps | 2 pad] (kLensStride doubles): the four 16-byte loads of a
// warp touch at most four distinct chunks (vw or wm, half 0 or 1), on
// disjoint banks; in the tensor-core form a B fragment (4 lenses x 8 maps)
// starts its lens rows 72 words = 8 banks apart, so each half-warp's 16
// values fall on 32 distinct banks.
constexpr int kTileL = 64;
constexpr int kLensStride = 2 * (kMapGroup + 2);
constexpr int kWmOffset = kMapGroup + 2;
// Threads per block at most (whole lens groups); two blocks per SM leave 128
// registers per thread for the 32 FP64 sums and the loads in flight.
constexpr int kMarksThreads = 256;
// Blocks the lenses of a call are spread over: two per SM of a 148-SM part,
// one wave.  A constant, so the summation order (and the result) depends
// only on the input.
constexpr int kMarksBlocks = 2 * 148;
static_assert(kTileL == 64, "the raw staging areas hold 64 lenses");
__host__ __device__ inline int marks_quad_bins(int n_bin) { return (n_bin + 3) / 4 * 4; }
// Factors of one tile: raw inputs -> FP64 vw, wm in fac_s, all threads.
// Consecutive lanes take consecutive maps of one lens, so each warp's stores
// fill whole 128-byte rows.
template <class Fac>
__device__ __forceinline__ void convert_factors(const Fac& fac, const unsigned char* raw, double* fac_s, int tid,
                                                int nthr) {
  static_assert(kMapGroup == 16, "maps are the low 4 bits of the element index");
  for (int e = tid; e < kTileL * kMapGroup; e += nthr) {
    const int g = e & 15, jj = e >> 4;
    double vw, wm;
    fac.factors(raw, g, jj, vw, wm);
    fac_s[jj * kLensStride + g] = vw;
    if (!Fac::kSame) fac_s[jj * kLensStride + kWmOffset + g] = wm;
  }
}

template <class Fac>
__global__ void __launch_bounds__(kMarksThreads, 2) k_marks_partials(const MarksField* __restrict__ fields, int n_field,
                                                            const Fac fac, int n_g, int n_bin, int tg,
                                                            long long chunk, double* __restrict__ partial) {
  extern __shared__ __align__(16) unsigned char sm[];
  constexpr int TF = kTileL * kLensStride;
  const int R = 3 * n_bin + 1;
  const int nbp = marks_quad_bins(n_bin), nbq = nbp / 4;
  const int ng = blockDim.x / tg;
  double* fac_s = reinterpret_cast<double*>(sm);  // [kTileL][kLensStride] factors of every row
  unsigned char* raw = sm + TF * sizeof(double);
  const int blk = blockIdx.x;
  int fi = 0;
  while (fi + 1 < n_field && fields[fi + 1].chunk0 <= blk) ++fi;
  const MarksField& F = fields[fi];  // read where used: its pointers need no registers across the loop
  const long long j0 = (long long)(blk - F.chunk0) * chunk;
  const long long j1 = min(F.n, j0 + chunk);
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int grp = tid / tg, l = tid % tg;
  const int quad = l >> 1, half = l & 1;
  const bool live = quad <= 3 * nbq;
  const int k = quad / nbq, c = quad - k * nbq;  // k = 3: the marks weight quad
  const double* fsel = ((k < 2 || Fac::kSame) ? fac_s : fac_s + kWmOffset) + 8 * half;
  // this lane's quad in HBM: bins 4 c .. of quantity k of lens j, or the marks weight
  const float* qrow = k == 0 ? F.xiE : k == 1 ? F.xiB : k == 2 ? F.K : F.mw;

  auto stage_tile = [&](long long t0) { fac.stage(F, t0, (int)min((long long)kTileL, j1 - t0), n_g, raw, tid, nthr); };
  auto convert_tile = [&]() { convert_factors(fac, raw, fac_s, tid, nthr); };

  double acc[4][8];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int g = 0; g < 8; ++g) acc[i][g] = 0.0;
  if (j0 < j1) stage_tile(j0);
  cp_async_wait_all();
  __syncthreads();
  if (j0 < j1) convert_tile();
  __syncthreads();
  for (long long t0 = j0; t0 < j1; t0 += kTileL) {
    const int nt = (int)min((long long)kTileL, j1 - t0);
    const bool more = t0 + kTileL < j1;
    // the raw area was read before the last barrier
    if (more) stage_tile(t0 + kTileL);
    if (live) {
#pragma unroll 1
      for (int jj = grp; jj < nt; jj += ng) {
        double m[4];
        const long long j = t0 + jj;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const bool v = k < 3 ? 4 * c + i < n_bin : i == 0;
          m[i] = v ? (double)__ldg(k < 3 ? qrow + j * n_bin + 4 * c + i : qrow + j) : 0.0;
        }
        const double2* f2 = reinterpret_cast<const double2*>(fsel + jj * kLensStride);
#pragma unroll
        for (int h = 0; h < 4; ++h) {
          const double2 f = f2[h];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            acc[i][2 * h] = fma(m[i], f.x, acc[i][2 * h]);
            acc[i][2 * h + 1] = fma(m[i], f.y, acc[i][2 * h + 1]);
          }
        }
      }
    }
    cp_async_wait_all();
    __syncthreads();  // the next tile's copies landed; this tile's factors are no longer read
    if (more) {
      convert_tile();
      __syncthreads();
    }
  }
  // groups 1.. add their sums into group 0's, in group order
  double* red = reinterpret_cast<double*>(sm);  // [tg][32]
  for (int kk = 1; kk < ng; ++kk) {
    __syncthreads();
    if (grp == kk) {
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int g = 0; g < 8; ++g) red[l * 32 + i * 8 + g] = acc[i][g];
    }
    __syncthreads();
    if (grp == 0) {
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int g = 0; g < 8; ++g) acc[i][g] += red[l * 32 + i * 8 + g];
    }
  }
  if (grp == 0 && live) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int b = 4 * c + i;
      if (k < 3 ? b >= n_bin : i > 0) continue;
      const int r = k < 3 ? k * n_bin + b : 3 * n_bin;
#pragma unroll
      for (int g = 0; g < 8; ++g) {
        const int map = 8 * half + g;
        if (map < n_g) partial[((size_t)blk * n_g + map) * R + r] = acc[i][g];
      }
    }
  }
}

// FP64 tensor-core form for n_bin <= 32 (tcgen05 has no FP64 kind; the FP64
// tensor instruction of sm_100 is mma.sync m8n8k4 .f64: D[8][8] += A[8][4]
// B[4][8], 256 FMA per warp instruction against 32 for a warp FFMA64).
//
// Rows (A's M dimension) are grouped so that no 8-row m-tile mixes the two
// factor kinds: the xi_E, xi_B rows (vw factors) fill the first
// MV = ceil(2 n_bin / 8) m-tiles, the K rows and the marks weight row (wm
// factors) the next ceil((n_bin + 1) / 8); padding rows read a zeroed area.
// Lenses are K (four per step), maps N (two n-tiles of 8).  Warp w owns
// m-tile w for both n-tiles and every lens of the block, so its sums are
// final for the block: no reduction between warps.  Two accumulator sets
// (even and odd lens steps) halve the dependent chain of the tensor
// instructions.
//
// Staging: thread 0 issues bulk copies of a whole tile (the three marks
// blocks [64][n_bin] as laid out in HBM, the marks weights, the factors' raw
// rows) signalled on the buffer's mbarrier; partial or unaligned tiles go by
// per-thread cp.async with zero fill.  Every wait is bounded: a copy that
// does not land sets kErrTimeout in *err and the block stops.
//
// Staged marks: quantity q of lens jj, bin b at q QS + jj n_bin + b
// (QS = 64 n_bin rounded up to 4 floats), the marks weights at 3 QS + jj, and
// 64 zeros at 3 QS + 64 for the padding rows.
__host__ __device__ inline int marks_dense_slot(int n_bin) { return (kTileL * n_bin + 3) / 4 * 4; }
__host__ __device__ inline int marks_dmma_buffer(int n_bin) { return 3 * marks_dense_slot(n_bin) + 2 * kTileL; }
__host__ __device__ inline int marks_vw_tiles(int n_bin) { return (2 * n_bin + 7) / 8; }
__host__ __device__ inline int marks_m_tiles(int n_bin) { return marks_vw_tiles(n_bin) + (n_bin + 1 + 7) / 8; }
constexpr int kDmmaMaxBins = 32;
constexpr int kDmmaMaxThreads = 32 * ((2 * kDmmaMaxBins + 7) / 8 + (kDmmaMaxBins + 1 + 7) / 8);
// Registers per thread at most: two blocks of kDmmaMaxThreads per SM.
constexpr int kDmmaRegs = 65536 / (2 * kDmmaMaxThreads) / 8 * 8;
constexpr size_t kDmmaRawBytes = std::max(MapFactors::kRawBytes, MultFactors::kRawBytes);

__device__ __forceinline__ void dmma_884(double& d0, double& d1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

template <class Fac>
__global__ void __launch_bounds__(kDmmaMaxThreads, 2) k_marks_dmma(const MarksField* __restrict__ fields, int n_field,
                                                              const Fac fac, int n_g, int n_bin, long long chunk,
                                                              double* __restrict__ partial, unsigned* __restrict__ err,
                                                              int skip_tile, unsigned wait_limit) {
  extern __shared__ __align__(16) unsigned char sm[];
  __shared__ __align__(8) uint64_t full[2];
  constexpr int TF = kTileL * kLensStride;
  const int nb = n_bin, R = 3 * nb + 1;
  const int QS = marks_dense_slot(nb), MS = marks_dmma_buffer(nb);
  const int MV = marks_vw_tiles(nb);
  double* fac_s = reinterpret_cast<double*>(sm);  // [kTileL][kLensStride] factors
  unsigned char* raw = sm + TF * sizeof(double);
  float* mk = reinterpret_cast<float*>(raw + kDmmaRawBytes);
  const int blk = blockIdx.x;
  int fi = 0;
  while (fi + 1 < n_field && fields[fi + 1].chunk0 <= blk) ++fi;
  const MarksField& F = fields[fi];
  const long long j0 = (long long)(blk - F.chunk0) * chunk;
  const long long j1 = min(F.n, j0 + chunk);
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int mt = tid >> 5, lane = tid & 31, gq = lane >> 2, tq = lane & 3;
  // this lane's A row (row gq of m-tile mt): output row r (-1: padding), the
  // staged offset of its value for lens 0 and its lens stride
  int r = -1, aoff = 3 * QS + kTileL, astr = 1;
  if (mt < MV) {
    const int rho = mt * 8 + gq;
    if (rho < 2 * nb) {
      const int q = rho / nb, b = rho - q * nb;
      r = rho, aoff = q * QS + b, astr = nb;
    }
  } else {
    const int rho = (mt - MV) * 8 + gq;
    if (rho < nb) {
      r = 2 * nb + rho, aoff = 2 * QS + rho, astr = nb;
    } else if (rho == nb) {
      r = 3 * nb, aoff = 3 * QS, astr = 1;
    }
  }
  // B: lens tq of the step, map gq of the n-tile
  const double* bsel = ((mt < MV || Fac::kSame) ? fac_s : fac_s + kWmOffset) + gq;
  const bool two = n_g > 8;  // the second n-tile holds maps

  // raw rows past n_g, lenses past a partial tile and the zero area are never
  // copied: start from zeros (ordered before the bulk copies by the fence)
  for (int e = tid; e < (int)(kDmmaRawBytes / 4); e += nthr) reinterpret_cast<float*>(raw)[e] = 0.f;
  for (int e = tid; e < 2 * MS; e += nthr) mk[e] = 0.f;
  if (tid == 0) {
    mbar_init(&full[0], 1);
    mbar_init(&full[1], 1);
    mbar_fence_init();
  }
  fence_proxy_async_smem();
  __syncthreads();
  const bool mbulk = (nb & 3) == 0 && al16(F.xiE) && al16(F.xiB) && al16(F.K) && al16(F.mw);
  uint32_t par = 0;  // bit b: parity of buffer b's next mbarrier phase
  // fault injection for tests (tpcf_debug_inject): the bulk copies of each
  // block's tile skip_tile are never issued, so the wait on them runs out
  // after wait_limit polls (both off in every product call)
  const uint32_t polls = wait_limit ? wait_limit : kWaitPolls;

  // starts the copies of tile t0 into buffer b; true when they complete on full[b]
  auto stage_tile = [&](long long t0, int b) -> bool {
    const int nt = (int)min((long long)kTileL, j1 - t0);
    const bool bm = mbulk && nt == kTileL;
    const bool br = fac.bulk_ok(F, t0, nt);
    float* mb = mk + b * MS;
    if ((bm || br) && tid == 0 && (t0 - j0) / kTileL != skip_tile) {
      mbar_arrive_tx(&full[b], (bm ? 4u * (3 * nb + 1) * kTileL : 0u) + (br ? fac.bulk_bytes(n_g) : 0u));
      if (bm) {
        const size_t o = (size_t)t0 * nb;
        bulk_g2s(mb, F.xiE + o, 4u * kTileL * nb, &full[b]);
        bulk_g2s(mb + QS, F.xiB + o, 4u * kTileL * nb, &full[b]);
        bulk_g2s(mb + 2 * QS, F.K + o, 4u * kTileL * nb, &full[b]);
        bulk_g2s(mb + 3 * QS, F.mw + t0, 4u * kTileL, &full[b]);
      }
      if (br) fac.stage_bulk(F, t0, n_g, raw, &full[b]);
    }
    if (!bm) {  // the marks as laid out in HBM, zero past the tile's end
      const size_t o = (size_t)t0 * nb;
      const int nq = nt * nb;
      const bool vec = (nb & 3) == 0 && al16(F.xiE) && al16(F.xiB) && al16(F.K);
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const float* src = (q == 0 ? F.xiE : q == 1 ? F.xiB : F.K) + o;
        float* dst = mb + q * QS;
        if (vec) {
          for (int e = tid; e < kTileL * nb / 4; e += nthr)
            cp_async16(dst + 4 * e, 4 * e < nq ? src + 4 * e : src, 4 * e < nq);
        } else {
          for (int e = tid; e < kTileL * nb; e += nthr) cp_async4(dst + e, e < nq ? src + e : src, e < nq);
        }
      }
      const float* mw = F.mw + t0;
      for (int e = tid; e < kTileL; e += nthr) cp_async4(mb + 3 * QS + e, e < nt ? mw + e : mw, e < nt);
    }
    if (!br) fac.stage(F, t0, nt, n_g, raw, tid, nthr);
    return bm || br;
  };
  // waits for buffer b's copies; false when a bulk copy did not land in time
  int wb = 0;
  uint32_t wpar = 0;
  auto land = [&](int b, bool bulk) -> bool {
    cp_async_wait_all();
    if (!bulk) return true;
    wb = b, wpar = (par >> b) & 1u;
    par ^= 1u << b;
    return mbar_wait_bounded(&full[b], wpar, polls);
  };

  double acc[2][2][2];
#pragma unroll
  for (int p = 0; p < 2; ++p)
#pragma unroll
    for (int n = 0; n < 2; ++n) acc[p][n][0] = acc[p][n][1] = 0.0;
  bool abort = false;
  if (j0 < j1) abort = __syncthreads_or(!land(0, stage_tile(j0, 0)));
  if (!abort) {
    if (j0 < j1) convert_factors(fac, raw, fac_s, tid, nthr);
    __syncthreads();
  }
  int buf = 0;
  for (long long t0 = j0; t0 < j1 && !abort; t0 += kTileL) {
    const bool more = t0 + kTileL < j1;
    // the raw area was read before the last barrier, the other marks buffer
    // before the one ahead of it
    const bool nbulk = more && stage_tile(t0 + kTileL, buf ^ 1);
    const float* ma = mk + buf * MS + aoff + tq * astr;
    const double* bp = bsel + tq * kLensStride;
#pragma unroll 8
    for (int ks = 0; ks < kTileL / 4; ++ks) {
      const double a = (double)ma[4 * ks * astr];
      const double* b = bp + 4 * ks * kLensStride;
      dmma_884(acc[ks & 1][0][0], acc[ks & 1][0][1], a, b[0]);
      if (two) dmma_884(acc[ks & 1][1][0], acc[ks & 1][1][1], a, b[8]);
    }
    // the next tile's copies landed; this tile's factors and marks are no longer read
    if (__syncthreads_or(more && !land(buf ^ 1, nbulk))) {
      abort = true;
      break;
    }
    if (more) {
      convert_factors(fac, raw, fac_s, tid, nthr);
      __syncthreads();
    }
    buf ^= 1;
  }
  if (abort) {  // a copy did not land: flag it, give it one more bounded wait, leave
    if (tid == 0) {
      atomicOr(err, kErrTimeout);
      mbar_wait_bounded(&full[wb], wpar, polls);
    }
    return;
  }
  if (r >= 0) {
#pragma unroll
    for (int n = 0; n < 2; ++n)
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int map = 8 * n + 2 * tq + i;
        if (map < n_g) partial[((size_t)blk * n_g + map) * R + r] = acc[0][n][i] + acc[1][n][i];
      }
  }
}
size_t marks_dmma_smem(int n_bin) {
  return sizeof(double) * kTileL * kLensStride + kDmmaRawBytes + 2 * sizeof(float) * (size_t)marks_dmma_buffer(n_bin);
}

// Threads per lens group (two per row quad, whole warps) and per block: as
// many groups as fit in kMarksThreads.
int marks_group_threads(int n_bin) { return (2 * (3 * marks_quad_bins(n_bin) / 4 + 1) + 31) / 32 * 32; }
int marks_block_threads(int n_bin) {
  const int tg = marks_group_threads(n_bin);
  return std::max(1, kMarksThreads / tg) * tg;
}
size_t marks_smem(int n_bin) {
  const size_t fac = sizeof(double) * kTileL * kLensStride + std::max(MapFactors::kRawBytes, MultFactors::kRawBytes);
  const size_t red = sizeof(double) * (size_t)marks_group_threads(n_bin) * 32;
  return std::max(fac, red);
}
// Blocks of a pass: as many as fit on a 148-SM part at once (by the shared
// memory and threads of the form used for n_bin), so the pass is one wave.
// A function of n_bin only, so the summation order (and the result) depends
// only on the input.
int marks_blocks(int n_bin) {
  if (n_bin > kDmmaMaxBins) return kMarksBlocks;
  const int bt = 32 * marks_m_tiles(n_bin);
  const int per_sm = std::min({2048 / bt, 65536 / (bt * kDmmaRegs), 233472 / ((int)marks_dmma_smem(n_bin) + 1024)});
  return 148 * std::max(1, per_sm);
}
// Lenses per block for n_lens lenses in all: marks_blocks blocks, whole tiles.
long long marks_chunk(long long n_lens, int n_bin) {
  const long long nbk = marks_blocks(n_bin);
  const long long per = (n_lens + nbk - 1) / nbk;
  return std::max<long long>(kTileL, (per + kTileL - 1) / kTileL * kTileL);
}
// One pass of the partial sums over all fields: the FP64 tensor-core form for
// n_bin <= 32, the FP64 FMA form for wider binnings.
template <class Fac>
cudaError_t launch_marks_partials(const MarksField* fields, int n_field, int nblk, long long chunk, const Fac& fac,
                                  int n_g, int nb, double* part, unsigned* err, int skip_tile, unsigned wait_limit,
                                  cudaStream_t st) {
  if (nb <= kDmmaMaxBins) {
    const size_t msm = marks_dmma_smem(nb);
    cudaError_t e = cudaFuncSetAttribute(k_marks_dmma<Fac>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)msm);
    if (e != cudaSuccess) return e;
    k_marks_dmma<Fac><<<nblk, 32 * marks_m_tiles(nb), msm, st>>>(fields, n_field, fac, n_g, nb, chunk, part, err,
                                                                 skip_tile, wait_limit);
    return cudaGetLastError();
  }
  const size_t msm = marks_smem(nb);
  const int bt = marks_block_threads(nb), tg = marks_group_threads(nb);
  cudaError_t e = cudaFuncSetAttribute(k_marks_partials<Fac>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)msm);
  if (e != cudaSuccess) return e;
  k_marks_partials<Fac><<<nblk, bt, msm, st>>>(fields, n_field, fac, n_g, nb, tg, chunk, part);
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

// With timing enabled (tpcf_set_timing), CUDA events on the call's stream
// around every partial-sum launch; total() after the stream has synchronised
// is their summed device time, kept as the call's kernel time.
struct PassTimer {
  tpcf_ctx* c;
  std::vector<cudaEvent_t> ev;
  explicit PassTimer(tpcf_ctx* ctx) : c(ctx) {}
  ~PassTimer() {
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
  }
  void mark(cudaStream_t st) {
    if (!c->time_pairs) return;
    cudaEvent_t e = nullptr;
    check(cudaEventCreate(&e), "event");
    ev.push_back(e);
    check(cudaEventRecord(e, st), "event record");
  }
  void total() {
    if (!c->time_pairs) return;
    double ms = 0.0;
    for (size_t i = 0; i + 1 < ev.size(); i += 2) {
      float t = 0.f;
      check(cudaEventElapsedTime(&t, ev[i], ev[i + 1]), "event time");
      ms += t;
    }
    c->last_pair_ms = ms;
  }
};

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
    int64_t n_all = 0;
    for (int i = 0; i < n_field; ++i) n_all += marks[i].n;
    const long long chunk = marks_chunk(n_all, nb);
    for (int i = 0; i < n_field; ++i) {
      const tpcf_marks_field& m = marks[i];
      const int64_t n = m.n;
      MarksField& F = hf[i];
      F.n = n;
      F.n_bin = nb;
      F.chunk0 = nblk;
      F.lens0 = 0;
      nblk += (int)((n + chunk - 1) / chunk);
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
    // the sums of every pass stay on the device until one copy after the
    // last pass, so the host queues all passes without waiting on any
    double* dout = (double*)ws_alloc(c, sizeof(double) * sums.size());
    unsigned* derr = (unsigned*)ws_alloc(c, sizeof(unsigned));
    check(cudaMemsetAsync(derr, 0, sizeof(unsigned), st), "memset");
    const int MG = marks_group(nb);
    PassTimer timer(c);
    for (int m0 = 0; m0 < n_map; m0 += MG) {
      const int g = std::min(MG, n_map - m0);
      if (nblk > 0) {
        timer.mark(st);
        counted(c, launch_marks_partials(df, n_field, nblk, chunk, MapFactors{m0}, g, nb, part, derr, c->skip_tile,
                                      c->wait_limit, st),
                "marks partials");
        timer.mark(st);
      }
      const int tot = g * n_field * R;
      double* dpass = dout + (size_t)m0 * n_field * R;
      if (nblk > 0) {
        k_marks_reduce<<<(tot + 7) / 8, 256, 0, st>>>(part, df, n_field, nblk, g, R, dpass);
        counted(c, cudaGetLastError(), "marks reduce");
      } else {
        check(cudaMemsetAsync(dpass, 0, sizeof(double) * tot, st), "memset");
      }
    }
    check(cudaMemcpyAsync(sums.data(), dout, sizeof(double) * sums.size(), cudaMemcpyDeviceToHost, st), "D2H sums");
    unsigned herr = 0;
    check(cudaMemcpyAsync(&herr, derr, sizeof(unsigned), cudaMemcpyDeviceToHost, st), "D2H err");
    check(cudaStreamSynchronize(st), "sync marks");
    if (herr & kErrTimeout) throw Failure(TPCF_ERR_TIMEOUT, "a bounded device wait timed out in the marks kernel");
    timer.total();
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
    const long long chunk = marks_chunk(n_lens, nb);
    for (int i = 0; i < n_field; ++i) {
      const tpcf_marks_field& m = marks[i];
      MarksField& F = hf[i];
      F.n = m.n;
      F.n_bin = nb;
      F.chunk0 = nblk;
      F.lens0 = off;
      off += m.n;
      nblk += (int)((m.n + chunk - 1) / chunk);
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
    std::vector<double> sums((size_t)n_boot * n_field * R, 0.0);
    // the sums of every pass stay on the device until one copy after the
    // last pass, so the host queues all passes without waiting on any
    double* dout = (double*)ws_alloc(c, sizeof(double) * sums.size());
    if (nblk == 0) check(cudaMemsetAsync(dout, 0, sizeof(double) * sums.size(), st), "memset");
    unsigned* derr = (unsigned*)ws_alloc(c, sizeof(unsigned));
    check(cudaMemsetAsync(derr, 0, sizeof(unsigned), st), "memset");
    const int MG = marks_group(nb);
    PassTimer timer(c);
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
        timer.mark(st);
        counted(c,
                launch_marks_partials(df, n_field, nblk, chunk, MultFactors{mult, dunit, n_units}, G, nb, part, derr,
                                      c->skip_tile, c->wait_limit, st),
                "bootstrap partials");
        timer.mark(st);
        const int tot = G * n_field * R;
        k_marks_reduce<<<(tot + 7) / 8, 256, 0, st>>>(part, df, n_field, nblk, G, R,
                                                       dout + (size_t)s0 * n_field * R);
        counted(c, cudaGetLastError(), "bootstrap reduce");
      }
    }
    check(cudaMemcpyAsync(sums.data(), dout, sizeof(double) * sums.size(), cudaMemcpyDeviceToHost, st), "D2H sums");
    unsigned herr = 0;
    check(cudaMemcpyAsync(&herr, derr, sizeof(unsigned), cudaMemcpyDeviceToHost, st), "D2H err");
    check(cudaStreamSynchronize(st), "sync bootstrap");
    if (herr & kErrTimeout) throw Failure(TPCF_ERR_TIMEOUT, "a bounded device wait timed out in the marks kernel");
    timer.total();
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
