// capi.cu -- C ABI and host orchestration of libtpcf_b200.
//
// One call = stage inputs -> per-catalogue grid / lens-group build on the
// device -> one persistent pair-kernel launch over every (task, lens group)
// work item -> deterministic per-patch reduction -> outputs.  The reference
// counterparts are cited at each entry point in include/tpcf_b200.h.

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "sph_canon.cuh"
#include "tpcf_b200.h"
#include "tpcf_internal.cuh"
#include "tpcf_kernels.h"
#include "tpcf_ctx.h"

using namespace tpcf;

// ------------------------------------------------------------- ctx helpers --
namespace tpcf {

void* ws_alloc(tpcf_ctx* c, size_t bytes) {
  if (bytes == 0) bytes = 16;
  if (c->fail_alloc >= 0 && c->fail_alloc-- == 0)
    throw Failure(TPCF_ERR_OOM, "device allocation failed (injected by tpcf_debug_inject)");
  if (c->next_slot == c->slots.size()) c->slots.push_back(Slot{nullptr, 0});
  Slot& s = c->slots[c->next_slot++];
  if (s.bytes < bytes) {
    if (s.ptr) {
      cudaError_t e = cudaFree(s.ptr);
      s.ptr = nullptr;
      s.bytes = 0;
      if (e != cudaSuccess) throw Failure(TPCF_ERR_CUDA, std::string("cudaFree: ") + cudaGetErrorString(e));
    }
    size_t want = bytes + bytes / 4 + 256;
    cudaError_t e = cudaMalloc(&s.ptr, want);
    if (e != cudaSuccess) {
      cudaGetLastError();
      s.ptr = nullptr;
      throw Failure(TPCF_ERR_OOM, "device allocation of " + std::to_string(want) + " bytes failed");
    }
    s.bytes = want;
  }
  return s.ptr;
}

bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw Failure(TPCF_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

void counted(tpcf_ctx* c, cudaError_t e, const char* what) {
  check(e, what);
  c->launches += 1;
}

template <class T>
const T* stage(tpcf_ctx* c, const T* p, int64_t n) {
  if (!p || n <= 0) return p;
  if (is_device_ptr(p)) return p;
  T* d = static_cast<T*>(ws_alloc(c, sizeof(T) * (size_t)n));
  check(cudaMemcpyAsync(d, p, sizeof(T) * (size_t)n, cudaMemcpyHostToDevice, c->stream), "H2D input");
  c->h2d_bytes += sizeof(T) * (size_t)n;
  return d;
}
template const float* stage<float>(tpcf_ctx*, const float*, int64_t);
template const int* stage<int>(tpcf_ctx*, const int*, int64_t);
template const double* stage<double>(tpcf_ctx*, const double*, int64_t);

void copy_out(tpcf_ctx* c, void* dst, const void* src, size_t bytes) {
  if (!dst || bytes == 0) return;
  check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, c->stream), "output copy");
}

void begin_call(tpcf_ctx* c) {
  c->next_slot = 0;
  c->h2d_bytes = 0;
  check(cudaSetDevice(c->device), "cudaSetDevice");
}

void vlog(tpcf_ctx* c, const char* fmt, ...) {
  if (!c->opts.verbose) return;
  va_list ap;
  va_start(ap, fmt);
  std::fprintf(stderr, "[tpcf_b200] ");
  std::vfprintf(stderr, fmt, ap);
  std::fprintf(stderr, "\n");
  va_end(ap);
}

// Canonical FP64 edges (same formulas as the oracle's canon::edges).
tpcf_status canonical_edges(const tpcf_bins* b, double* e, double* e2) {
  if (!b) return TPCF_ERR_INVALID_ARG;
  const int n = b->n_bin;
  const double x_min = b->x_min, x_max = b->x_max, p = b->ihs_theta;
  if (n < 1 || n > kMaxBins || !(x_max > x_min) || !std::isfinite(x_max) || !std::isfinite(x_min))
    return TPCF_ERR_INVALID_ARG;
  if (b->spacing == TPCF_LOG && !(x_min > 0)) return TPCF_ERR_INVALID_ARG;
  if (b->spacing == TPCF_SQRT && !(x_min >= 0)) return TPCF_ERR_INVALID_ARG;
  if (b->spacing == TPCF_IHS && !(p > 0)) return TPCF_ERR_INVALID_ARG;
  if (b->spacing < TPCF_LIN || b->spacing > TPCF_SQRT) return TPCF_ERR_INVALID_ARG;
  e[0] = x_min;
  e[n] = x_max;
  if (b->spacing == TPCF_LIN) {
    const double d = (x_max - x_min) / n;
    for (int i = 1; i < n; ++i) e[i] = x_min + i * d;
  } else if (b->spacing == TPCF_LOG) {
    const double l0 = std::log10(x_min), d = (std::log10(x_max) - l0) / n;
    for (int i = 1; i < n; ++i) e[i] = std::pow(10.0, l0 + i * d);
  } else if (b->spacing == TPCF_SQRT) {
    const double s0 = std::sqrt(x_min), d = (std::sqrt(x_max) - s0) / n;
    for (int i = 1; i < n; ++i) {
      const double s = s0 + i * d;
      e[i] = s * s;
    }
  } else {
    const double t0 = std::log(p * x_min + std::sqrt((p * x_min) * (p * x_min) + 1.0)) / p;
    const double t1 = std::log(p * x_max + std::sqrt((p * x_max) * (p * x_max) + 1.0)) / p;
    const double d = (t1 - t0) / n;
    for (int i = 1; i < n; ++i) e[i] = std::sinh(p * (t0 + i * d)) / p;
  }
  for (int i = 0; i <= n; ++i) e2[i] = e[i] * e[i];
  for (int i = 0; i < n; ++i)
    if (!(e2[i + 1] > e2[i])) return TPCF_ERR_INVALID_ARG;
  return TPCF_OK;
}

// Bin centres in FP32 as create_bins computes them (src/utils.f90:202-229).
void bin_centers_f32(const tpcf_bins* b, float* centers) {
  const int n = b->n_bin;
  const float x_min = (float)b->x_min, x_max = (float)b->x_max, p = (float)b->ihs_theta;
  std::vector<float> e(n + 1);
  float bs;
  auto T = [&](float x) { return logf(p * x + sqrtf((p * x) * (p * x) + 1.0f)) / p; };
  if (b->spacing == TPCF_LIN) bs = (x_max - x_min) / (float)n;
  else if (b->spacing == TPCF_LOG) bs = (log10f(x_max) - log10f(x_min)) / (float)n;
  else if (b->spacing == TPCF_IHS) bs = (T(x_max) - T(x_min)) / (float)n;
  else bs = (sqrtf(x_max) - sqrtf(x_min)) / (float)n;
  e[n] = x_max;
  for (int i = 0; i < n; ++i) {
    if (b->spacing == TPCF_LIN) e[i] = x_min + bs * (float)i;
    else if (b->spacing == TPCF_LOG) e[i] = powf(10.0f, log10f(x_min) + bs * (float)i);
    else if (b->spacing == TPCF_IHS) e[i] = sinhf(p * (T(x_min) + bs * (float)i)) / p;
    else {
      const float s = sqrtf(x_min) + bs * (float)i;
      e[i] = s * s;
    }
  }
  for (int i = 0; i < n; ++i) centers[i] = e[i] + (e[i + 1] - e[i]) / 2.0f;
}

}  // namespace tpcf

// ---------------------------------------------------------- batch engine --
namespace {

struct LensIn {
  int64_t n;
  const float *x, *y, *z, *val, *w;
  const int* patch;
};
struct SrcIn {
  int64_t n;
  const float *x, *y, *z, *f1, *f2, *w, *m;
};

struct LensBuilt {
  int n_valid = 0;
  int n_groups = 0;
  float4* rec = nullptr;
  float* zs = nullptr;
  int* perm = nullptr;
  int* group_start = nullptr;
  float4* group_box = nullptr;
  std::vector<int> patch_groups;  // [n_patch_eff + 1], host
  int* d_patch_groups = nullptr;
};

struct SrcBuilt {
  GridDesc g{};
};

// One prepared batch: every device buffer of the call (in the context's
// workspace) and what the launch and the outputs need.  batch_setup builds
// the grids, lens groups and the sorted work items; batch_launch enqueues the
// pair kernel and the per-patch reductions (no host synchronisation, no
// allocation); batch_finish writes the per-lens outputs, waits and forms the
// totals and normalised outputs.
struct Batch {
  int mode = 0;
  bool sph = false, sharded = false, use_patch_any = false, has_m = false, has_z = false, logb = false;
  int nb = 0, n_patch = 0, n_patch_eff = 1, bt = 128, tch = 2, variant = 0, nT = 0;
  std::vector<int> tl;
  std::vector<int64_t> lens_n;  // input size of each lens catalogue
  std::vector<LensBuilt> lb;
  std::vector<TaskDesc> tdesc;
  std::vector<char> want_lens;
  int n_items = 0, grid = 0;
  PairParams P{};
  PairLaunch L{};
  int* head = nullptr;  // [0] queue head, [1] error flags
  double* item_sums = nullptr;
  double* lens_acc = nullptr;
  long long lens_acc_elems = 0;
  std::vector<double*> dpatch;
};

void batch_setup(tpcf_ctx* c, int mode, std::vector<LensIn> lens, std::vector<SrcIn> srcs, const std::vector<int>& tl,
                 const std::vector<int>& ts, const tpcf_bins* bins, int n_patch, const tpcf_result* outs, Batch& B) {
  begin_call(c);
  cudaStream_t st = c->stream;
  const int nb = bins->n_bin;
  std::vector<double> e(nb + 1), e2(nb + 1);
  tpcf_status bs = canonical_edges(bins, e.data(), e2.data());
  if (bs != TPCF_OK) throw Failure(bs, "invalid binning");
  const bool sph = c->opts.spherical != 0;
  if (sph) {  // squared chords (2 sin(e/2))^2: the same bins on the unit sphere
    for (int i = 0; i <= nb; ++i) e2[i] = canon_chord2(e[i]);
    for (int i = 0; i < nb; ++i)
      if (!(e2[i + 1] > e2[i]) || !(e[nb] <= 3.14159265358979)) throw Failure(TPCF_ERR_INVALID_ARG, "invalid binning");
  }
  if (c->opts.shard_count > 1 && (c->opts.shard_index < 0 || c->opts.shard_index >= c->opts.shard_count))
    throw Failure(TPCF_ERR_INVALID_ARG, "shard_index outside [0, shard_count)");
  const bool sharded = c->opts.shard_count > 1;
  const int nL = (int)lens.size(), nS = (int)srcs.size(), nT = (int)tl.size();
  for (int t = 0; t < nT; ++t)
    if (tl[t] < 0 || tl[t] >= nL || ts[t] < 0 || ts[t] >= nS) throw Failure(TPCF_ERR_INVALID_ARG, "task index out of range");
  const bool use_patch_any = n_patch > 0;
  const int n_patch_eff = use_patch_any ? n_patch : 1;
  for (auto& l : lens) {
    if (l.n < 0 || l.n > (1ll << 31) - 2) throw Failure(TPCF_ERR_INVALID_ARG, "lens catalogue size out of range");
    if (l.n > 0 && (!l.x || !l.y || !l.val || !l.w)) throw Failure(TPCF_ERR_INVALID_ARG, "missing lens array");
    if (l.patch && !use_patch_any) throw Failure(TPCF_ERR_INVALID_ARG, "patch labels given with n_patch <= 0");
  }
  for (auto& s : srcs) {
    if (s.n < 0 || s.n > (1ll << 31) - 2) throw Failure(TPCF_ERR_INVALID_ARG, "source catalogue size out of range");
    if (s.n > 0 && (!s.x || !s.y || !s.f1 || !s.f2 || !s.w)) throw Failure(TPCF_ERR_INVALID_ARG, "missing source array");
  }

  // ---- stage inputs
  Phase ph_stage("tpcf: stage inputs + grid build");
  for (auto& l : lens) {
    l.x = stage(c, l.x, l.n); l.y = stage(c, l.y, l.n); l.z = stage(c, l.z, l.n);
    l.val = stage(c, l.val, l.n); l.w = stage(c, l.w, l.n); l.patch = stage(c, l.patch, l.n);
  }
  for (auto& s : srcs) {
    s.x = stage(c, s.x, s.n); s.y = stage(c, s.y, s.n); s.z = stage(c, s.z, s.n);
    s.f1 = stage(c, s.f1, s.n); s.f2 = stage(c, s.f2, s.n); s.w = stage(c, s.w, s.n); s.m = stage(c, s.m, s.n);
  }

  // ---- sphere: keep the input longitudes for the unit vectors; the grid and
  // the lens order use longitudes reduced to [0, 2 pi)
  std::vector<const float*> lamL(nL, nullptr), lamS(nS, nullptr);
  if (sph) {
    for (int i = 0; i < nL; ++i) {
      lamL[i] = lens[i].x;
      if (lens[i].n <= 0) continue;
      float* xr = (float*)ws_alloc(c, sizeof(float) * lens[i].n);
      counted(c, launch_wrap_lambda(lens[i].x, lens[i].n, xr, st), "wrap lambda");
      lens[i].x = xr;
    }
    for (int i = 0; i < nS; ++i) {
      lamS[i] = srcs[i].x;
      if (srcs[i].n <= 0) continue;
      float* xr = (float*)ws_alloc(c, sizeof(float) * srcs[i].n);
      counted(c, launch_wrap_lambda(srcs[i].x, srcs[i].n, xr, st), "wrap lambda");
      srcs[i].x = xr;
    }
  }

  // ---- bounding boxes, z ranges, max |m|, counts, patch ranges (one sync)
  const int ncat = nL + nS;
  int* box_ord = (int*)ws_alloc(c, sizeof(int) * 8 * ncat);
  unsigned long long* cnt = (unsigned long long*)ws_alloc(c, sizeof(unsigned long long) * ncat);
  int* pr = (int*)ws_alloc(c, sizeof(int) * 2 * ncat);
  float* boxf = (float*)ws_alloc(c, sizeof(float) * 8 * ncat);
  counted(c, launch_bbox_init(box_ord, cnt, pr, ncat, st), "bbox init");
  for (int i = 0; i < nL; ++i)
    counted(c, launch_bbox(lens[i].x, lens[i].y, lens[i].z, lens[i].w, lens[i].patch, nullptr, lens[i].n, 1,
                           box_ord + 8 * i, cnt + i, pr + 2 * i, st), "bbox lens");
  for (int i = 0; i < nS; ++i)
    counted(c, launch_bbox(srcs[i].x, srcs[i].y, srcs[i].z, nullptr, nullptr, srcs[i].m, srcs[i].n, 0,
                           box_ord + 8 * (nL + i), cnt + nL + i, pr + 2 * (nL + i), st), "bbox src");
  counted(c, launch_bbox_finish(box_ord, boxf, 8 * ncat, st), "bbox finish");
  std::vector<float> hbox(8 * ncat);
  std::vector<unsigned long long> hcnt(ncat);
  std::vector<int> hpr(2 * ncat);
  check(cudaMemcpyAsync(hbox.data(), boxf, sizeof(float) * 8 * ncat, cudaMemcpyDeviceToHost, st), "D2H box");
  check(cudaMemcpyAsync(hcnt.data(), cnt, sizeof(unsigned long long) * ncat, cudaMemcpyDeviceToHost, st), "D2H count");
  check(cudaMemcpyAsync(hpr.data(), pr, sizeof(int) * 2 * ncat, cudaMemcpyDeviceToHost, st), "D2H prange");
  check(cudaStreamSynchronize(st), "sync bbox");
  for (int i = 0; i < nL; ++i)
    if (lens[i].patch && hcnt[i] > 0 && (hpr[2 * i] < 0 || hpr[2 * i + 1] >= n_patch))
      throw Failure(TPCF_ERR_INVALID_ARG, "patch label outside [0, n_patch)");

  if (sph)
    for (int i = 0; i < ncat; ++i)
      if (hcnt[i] > 0 && (hbox[8 * i + 1] < -1.57079637f || hbox[8 * i + 3] > 1.57079637f))
        throw Failure(TPCF_ERR_INVALID_ARG, "latitude outside [-pi/2, pi/2] (spherical positions are radians)");

  // ---- kernel configuration
  bool has_m = false, has_z = false;
  for (int i = 0; i < nS; ++i)  // K differs from w only where some m != 0
    has_m = has_m || (mode == 0 && srcs[i].m != nullptr && hcnt[nL + i] > 0 && hbox[8 * (nL + i) + 6] != 0.f);
  for (int t = 0; t < nT; ++t) {
    const int li = tl[t], si = ts[t];
    if (mode == 0 && hcnt[li] > 0 && hcnt[nL + si] > 0) {
      const float lz_max = hbox[8 * li + 5], sz_min = hbox[8 * (nL + si) + 4];
      if (lz_max > sz_min) has_z = true;
    }
  }
  // On the sphere log binning maps theta^2 by a series valid for chords <= 0.25.
  const bool logb = bins->spacing == TPCF_LOG && (!sph || e2[nb] <= 0.0625);
  const int qa = has_m ? 6 : 5;
  int bt = 128;
  while (bt > 32 && (size_t)nb * qa * bt * 4 > 100 * 1024) bt /= 2;
  // planar: bt threads per block, each warp one 32-lens group at a time, tiles
  // of tch sub-chunks; sphere: one bt-lens group per block
  int tch = 2;
  if (!sph && c->opts.group_size > 0 && c->opts.group_size <= bt) bt = c->opts.group_size;
  if (!sph && c->opts.tile_chunks == 1) tch = 1;
  const int lens_group = sph ? bt : 32;

  const double Rd = bins->x_max;
  float R = (float)(Rd * (1.0 + 1e-6));

  // ---- source grids
  std::vector<GridDesc> grids(nS);
  for (int i = 0; i < nS; ++i) {
    const SrcIn& s = srcs[i];
    GridDesc& g = grids[i];
    const float* b = &hbox[8 * (nL + i)];
    const int n_valid = (int)hcnt[nL + i];
    float x0 = n_valid ? b[0] : 0.f, y0 = n_valid ? b[1] : 0.f;
    float ex = n_valid ? b[2] - b[0] : 0.f, ey = n_valid ? b[3] - b[1] : 0.f;
    if (sph) {  // longitude cells cover the whole circle
      x0 = 0.f;
      ex = 6.28318548f;
    }
    double cell = c->opts.cell_size > 0 ? c->opts.cell_size : Rd / 16.0;
    const double span = std::max((double)ex, (double)ey);
    if (!c->opts.use_grid) cell = span * 2.0 + 1.0;
    // keep the grid below 2^24 cells
    while ((span / cell + 2.0) * (span / cell + 2.0) > (double)(1 << 24)) cell *= 1.5;
    if (!(cell > 0)) cell = 1.0;
    int ncx = (int)std::floor(ex / cell) + 1, ncy = (int)std::floor(ey / cell) + 1;
    ncx = std::max(1, ncx); ncy = std::max(1, ncy);
    const unsigned ncells = (unsigned)ncx * (unsigned)ncy;
    g.x0 = x0; g.y0 = y0; g.cell = (float)cell; g.inv_cell = (float)(1.0 / cell);
    g.ncx = ncx; g.ncy = ncy; g.n_valid = n_valid;
    int* cs = (int*)ws_alloc(c, sizeof(int) * (ncells + 1));
    const int n_chunks = std::max((n_valid + kChunk - 1) / kChunk, 1);
    SrcPair* pairs = sph ? nullptr : (SrcPair*)ws_alloc(c, sizeof(SrcPair) * (kChunk / 2) * n_chunks);
    ChunkMeta* cmeta = sph ? nullptr : (ChunkMeta*)ws_alloc(c, sizeof(ChunkMeta) * n_chunks);
    SrcRecS* recs = sph ? (SrcRecS*)ws_alloc(c, sizeof(SrcRecS) * std::max(n_valid, 1)) : nullptr;
    if (s.n > 0) {
      unsigned* k0 = (unsigned*)ws_alloc(c, sizeof(unsigned) * s.n);
      unsigned* k1 = (unsigned*)ws_alloc(c, sizeof(unsigned) * s.n);
      int* i0 = (int*)ws_alloc(c, sizeof(int) * s.n);
      int* i1 = (int*)ws_alloc(c, sizeof(int) * s.n);
      int cell_bits = 1;
      while (cell_bits < 32 && (1ull << cell_bits) <= (unsigned long long)ncells) ++cell_bits;
      const int mb = std::min(16, (32 - cell_bits) & ~1);  // within-cell Hilbert bits
      counted(c, launch_src_keys(s.x, s.y, s.z, s.n, x0, y0, g.inv_cell, ncx, ncy, mb, k0, i0, st), "src keys");
      const int end_bit = cell_bits + mb;
      size_t tb = 0;
      check(sort_pairs_u32(nullptr, tb, k0, k1, i0, i1, (int)s.n, end_bit, st), "sort size");
      void* tmp = ws_alloc(c, tb);
      check(sort_pairs_u32(tmp, tb, k0, k1, i0, i1, (int)s.n, end_bit, st), "sort sources");
      counted(c, launch_cell_start(k1, s.n, ncells, mb, cs, st), "cell start");
      if (sph)
        counted(c, launch_src_gather_sph(i1, n_valid, mode, lamS[i], s.y, s.z, s.f1, s.f2, s.w, s.m, recs, st),
                "src gather");
      else
        counted(c, launch_src_pairs(i1, n_valid, mode, s.x, s.y, s.z, s.f1, s.f2, s.w, s.m, pairs, cmeta, st),
                "src gather");
    } else {
      check(cudaMemsetAsync(cs, 0, sizeof(int) * (ncells + 1), st), "memset cells");
    }
    g.cell_start = cs;
    g.rec = nullptr;
    g.recs = recs;
    g.pairs = pairs;
    g.meta = cmeta;
  }
  // FP32 guard on the reach of a task's rows and cells: the rounding scale of
  // the coordinates its two catalogues hold, so that a task's tiles (and its
  // sums, bit for bit) do not depend on the other tasks of a batch
  std::vector<double> extent(ncat, 0.0);
  for (int i = 0; i < ncat; ++i) {
    const float* b = &hbox[8 * i];
    if (hcnt[i] == 0) continue;
    extent[i] = std::fabs(b[0]) + std::fabs(b[1]) + std::fabs(b[2]) + std::fabs(b[3]);
    if (sph) extent[i] = 2.0 * M_PI + M_PI;  // reduced longitudes and latitudes
  }
  auto task_margin = [&](int li, int si) {
    return (float)(1e-5 * (std::max(extent[li], extent[nL + si]) + Rd) + 1e-4 * grids[si].cell);
  };

  // ---- lens catalogues: sort by (patch, Hilbert index), groups of <= lens_group lenses
  std::vector<LensBuilt>& lb = B.lb;
  lb.assign(nL, LensBuilt{});
  std::vector<LensDesc> ldesc(nL);
  for (int i = 0; i < nL; ++i) {
    const LensIn& l = lens[i];
    LensBuilt& LB = lb[i];
    LB.n_valid = (int)hcnt[i];
    const float* b = &hbox[8 * i];
    LB.rec = (float4*)ws_alloc(c, sizeof(float4) * std::max(LB.n_valid, 1));
    LB.zs = mode == 0 ? (float*)ws_alloc(c, sizeof(float) * std::max(LB.n_valid, 1)) : nullptr;
    LB.perm = (int*)ws_alloc(c, sizeof(int) * std::max(LB.n_valid, 1));
    std::vector<int> off(n_patch_eff + 1, 0);
    if (l.n > 0 && LB.n_valid > 0) {
      unsigned long long* k0 = (unsigned long long*)ws_alloc(c, sizeof(unsigned long long) * l.n);
      unsigned long long* k1 = (unsigned long long*)ws_alloc(c, sizeof(unsigned long long) * l.n);
      int* i0 = (int*)ws_alloc(c, sizeof(int) * l.n);
      int* i1 = (int*)ws_alloc(c, sizeof(int) * l.n);
      float4 box = make_float4(b[0], b[1], b[2], b[3]);
      counted(c, launch_lens_keys(l.x, l.y, l.z, l.w, l.patch, l.n, box, k0, i0, st), "lens keys");
      size_t tb = 0;
      check(sort_pairs_u64(nullptr, tb, k0, k1, i0, i1, (int)l.n, st), "sort size");
      void* tmp = ws_alloc(c, tb);
      check(sort_pairs_u64(tmp, tb, k0, k1, i0, i1, (int)l.n, st), "sort lenses");
      counted(c, launch_lens_gather(i1, LB.n_valid, l.x, l.y, l.z, l.val, l.w, LB.rec, LB.zs, LB.perm, st), "lens gather");
      if (l.patch) {
        int* doff = (int*)ws_alloc(c, sizeof(int) * (n_patch_eff + 1));
        counted(c, launch_patch_offsets(k1, LB.n_valid, n_patch_eff, doff, st), "patch offsets");
        check(cudaMemcpyAsync(off.data(), doff, sizeof(int) * (n_patch_eff + 1), cudaMemcpyDeviceToHost, st), "D2H off");
        check(cudaStreamSynchronize(st), "sync offsets");
      } else {
        for (int p = 1; p <= n_patch_eff; ++p) off[p] = LB.n_valid;
      }
    }
    std::vector<int> gstart;
    LB.patch_groups.assign(n_patch_eff + 1, 0);
    for (int p = 0; p < n_patch_eff; ++p) {
      LB.patch_groups[p] = (int)gstart.size();
      for (int s0 = off[p]; s0 < off[p + 1]; s0 += lens_group) gstart.push_back(s0);
    }
    LB.patch_groups[n_patch_eff] = (int)gstart.size();
    LB.n_groups = (int)gstart.size();
    gstart.push_back(LB.n_valid);
    LB.group_start = (int*)ws_alloc(c, sizeof(int) * gstart.size());
    check(cudaMemcpyAsync(LB.group_start, gstart.data(), sizeof(int) * gstart.size(), cudaMemcpyHostToDevice, st), "H2D groups");
    LB.d_patch_groups = (int*)ws_alloc(c, sizeof(int) * (n_patch_eff + 1));
    check(cudaMemcpyAsync(LB.d_patch_groups, LB.patch_groups.data(), sizeof(int) * (n_patch_eff + 1),
                          cudaMemcpyHostToDevice, st), "H2D patch groups");
    float4* pos = nullptr;
    if (sph) {
      pos = (float4*)ws_alloc(c, sizeof(float4) * 2 * std::max(LB.n_valid, 1));
      if (LB.n_valid > 0) counted(c, launch_lens_pos_sph(LB.perm, LB.n_valid, lamL[i], l.y, pos, st), "lens pos");
    }
    LB.group_box = (float4*)ws_alloc(c, sizeof(float4) * std::max(LB.n_groups, 1));
    counted(c, launch_group_box(LB.rec, LB.group_start, LB.n_groups, LB.group_box, st), "group box");
    check(cudaStreamSynchronize(st), "sync groups");  // host vectors above must outlive the async copies
    LensDesc& d = ldesc[i];
    d.rec = LB.rec; d.z = LB.zs; d.group_start = LB.group_start; d.group_box = LB.group_box;
    d.n_valid = LB.n_valid; d.n_groups = LB.n_groups;
    d.pos = pos;
  }

  // ---- tasks and work items
  Phase ph_items("tpcf: work items");
  std::vector<TaskDesc>& tdesc = B.tdesc;
  tdesc.assign(nT, TaskDesc{});
  std::vector<int2> items;
  B.want_lens.assign(nT, 0);
  long long lens_acc_elems = 0;
  for (int t = 0; t < nT; ++t) {
    TaskDesc& d = tdesc[t];
    d.lens_cat = tl[t];
    d.src_cat = ts[t];
    d.margin = task_margin(tl[t], ts[t]);
    d.item_base = (int)items.size();
    for (int g = 0; g < lb[tl[t]].n_groups; ++g) items.push_back(make_int2(t, g));
    const tpcf_result& o = outs[t];
    B.want_lens[t] =
        (o.xi_E_marks || o.xi_B_marks || o.K_marks || o.w_marks || o.marks_weight || o.lens_sums || o.lens_raw) ? 1 : 0;
    d.lens_acc_off = -1;
    if (B.want_lens[t]) {
      d.lens_acc_off = lens_acc_elems;
      lens_acc_elems += (long long)kQ * nb * std::max(lb[tl[t]].n_valid, 1);
    }
  }
  const int n_items = (int)items.size();
  TaskDesc* d_tasks = (TaskDesc*)ws_alloc(c, sizeof(TaskDesc) * std::max(nT, 1));
  LensDesc* d_lens = (LensDesc*)ws_alloc(c, sizeof(LensDesc) * std::max(nL, 1));
  GridDesc* d_grids = (GridDesc*)ws_alloc(c, sizeof(GridDesc) * std::max(nS, 1));
  check(cudaMemcpyAsync(d_tasks, tdesc.data(), sizeof(TaskDesc) * nT, cudaMemcpyHostToDevice, st), "H2D tasks");
  check(cudaMemcpyAsync(d_lens, ldesc.data(), sizeof(LensDesc) * nL, cudaMemcpyHostToDevice, st), "H2D lens desc");
  check(cudaMemcpyAsync(d_grids, grids.data(), sizeof(GridDesc) * nS, cudaMemcpyHostToDevice, st), "H2D grid desc");
  double* item_sums = (double*)ws_alloc(c, sizeof(double) * kQ * nb * std::max(n_items, 1));
  double* lens_acc = lens_acc_elems ? (double*)ws_alloc(c, sizeof(double) * lens_acc_elems) : nullptr;
  int* head = (int*)ws_alloc(c, sizeof(int) * 4);
  unsigned* err = (unsigned*)(head + 1);
  double* d_e2 = (double*)ws_alloc(c, sizeof(double) * (nb + 1));
  float* d_e2f = (float*)ws_alloc(c, sizeof(float) * (nb + 1));
  std::vector<float> e2f(nb + 1);
  for (int i = 0; i <= nb; ++i) e2f[i] = (float)e2[i];
  check(cudaMemcpyAsync(d_e2, e2.data(), sizeof(double) * (nb + 1), cudaMemcpyHostToDevice, st), "H2D edges");
  check(cudaMemcpyAsync(d_e2f, e2f.data(), sizeof(float) * (nb + 1), cudaMemcpyHostToDevice, st), "H2D edges f");

  int2* d_items = (int2*)ws_alloc(c, sizeof(int2) * std::max(n_items, 1));
  int n_run = 0;
  if (n_items > 0) {
    int2* d_items0 = (int2*)ws_alloc(c, sizeof(int2) * n_items);
    check(cudaMemcpyAsync(d_items0, items.data(), sizeof(int2) * n_items, cudaMemcpyHostToDevice, st), "H2D items");
    unsigned long long* ck0 = (unsigned long long*)ws_alloc(c, sizeof(unsigned long long) * n_items);
    unsigned long long* ck1 = (unsigned long long*)ws_alloc(c, sizeof(unsigned long long) * n_items);
    int* o0 = (int*)ws_alloc(c, sizeof(int) * n_items);
    int* o1 = (int*)ws_alloc(c, sizeof(int) * n_items);
    if (sph)
      counted(c, launch_item_cost_sph(d_items0, n_items, d_tasks, d_lens, d_grids, R, ck0, o0, st),
              "item cost");
    else
      counted(c, launch_item_cost(d_items0, n_items, d_tasks, d_lens, d_grids, R, ck0, o0, st), "item cost");
    size_t tb = 0;
    check(sort_pairs_u64_desc(nullptr, tb, ck0, ck1, o0, o1, n_items, st), "sort size");
    void* tmp = ws_alloc(c, tb);
    check(sort_pairs_u64_desc(tmp, tb, ck0, ck1, o0, o1, n_items, st), "sort items");
    const int sc = c->opts.shard_count > 1 ? c->opts.shard_count : 1;
    const int si = sc > 1 ? c->opts.shard_index : 0;
    counted(c, launch_permute_items(d_items0, o1, n_items, si, sc, d_items, st), "permute items");
    n_run = sc > 1 ? (n_items - si + sc - 1) / sc : n_items;
  }
  PairParams& P = B.P;
  P = PairParams{};
  P.tasks = d_tasks; P.lenses = d_lens; P.grids = d_grids; P.items = d_items; P.n_items = n_run;
  P.nb = nb; P.queue_head = head; P.item_sums = item_sums; P.lens_acc = lens_acc; P.err = err;
  P.e2 = d_e2; P.e2f = d_e2f; P.R = R;
  if (logb) {  // t = log2(theta^2) A + B (planar: theta^2 = d2)
    const double l0 = std::log2(e[0] * e[0]), l1 = std::log2(e[nb] * e[nb]);
    const double A = nb / (l1 - l0);
    P.binA = (float)A;
    P.binB = (float)(-l0 * A);
    P.eps = 1.0f / 32768.0f;
  } else {
    P.binA = P.binB = 0.f;
    P.eps = 4e-6f;
  }
  // FP32 histogram folded into FP64 every 4096 sources (each histogram cell
  // then holds at most 128 register sums of 32 pairs): the per-bin sums of
  // the call stay within 1e-6 of sum|terms|.  Per-lens outputs are sums of
  // far fewer terms per cell, so their FP32 partials are folded every 1024
  // sources (at 4096 one lens and bin of the 2 M x 0.5 M clustered
  // workload reached 1.05e-6 of its sum|terms|)
  P.flush_src = lens_acc ? 1024 : 4096;
  P.debug_skip_tile = c->skip_tile + 1;
  P.wait_limit = c->wait_limit;
  const char* var_env = std::getenv("TPCF_PAIR_VARIANT");
  B.variant = var_env ? std::atoi(var_env) : 0;
  if (n_items > 0 && !sph)
    counted(c, prepare_pairs(P, mode, has_m, has_z, logb, bt, tch, B.variant, c->num_sms, &B.L), "pair kernel");

  B.mode = mode; B.sph = sph; B.sharded = sharded; B.use_patch_any = use_patch_any;
  B.has_m = has_m; B.has_z = has_z; B.logb = logb;
  B.nb = nb; B.n_patch = n_patch; B.n_patch_eff = n_patch_eff; B.bt = bt; B.tch = tch; B.nT = nT;
  B.tl = tl;
  B.lens_n.assign(nL, 0);
  for (int i = 0; i < nL; ++i) B.lens_n[i] = lens[i].n;
  B.n_items = n_items;
  B.head = head;
  B.item_sums = item_sums;
  B.lens_acc = lens_acc;
  B.lens_acc_elems = lens_acc_elems;
  B.dpatch.assign(nT, nullptr);
  for (int t = 0; t < nT; ++t) B.dpatch[t] = (double*)ws_alloc(c, sizeof(double) * kQ * nb * n_patch_eff);
}

// The pair kernel and the per-patch reductions of a prepared batch: device
// work only, in stream order (a CUDA graph may record it).  The queue head and
// the error flags are cleared first, so a batch may be launched again.
void batch_launch(tpcf_ctx* c, Batch& B, bool timed) {
  Phase ph("tpcf: pair kernel + patch reduction");
  cudaStream_t st = c->stream;
  const int nb = B.nb;
  check(cudaMemsetAsync(B.head, 0, sizeof(int) * 4, st), "memset head");
  if (B.n_items > 0) {
    if (B.sharded) check(cudaMemsetAsync(B.item_sums, 0, sizeof(double) * kQ * nb * B.n_items, st), "memset items");
    // the kernel adds only the non-zero cells of each per-lens fold
    if (B.lens_acc) check(cudaMemsetAsync(B.lens_acc, 0, sizeof(double) * B.lens_acc_elems, st), "memset lens");
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    if (timed) {
      check(cudaEventCreate(&ev0), "event");
      check(cudaEventCreate(&ev1), "event");
      check(cudaEventRecord(ev0, st), "event record");
    }
    if (B.sph) {
      counted(c, launch_pairs_sph(B.P, B.mode, B.has_m, B.has_z, B.logb, B.bt, c->num_sms, st, &B.grid),
              "pair kernel");
    } else {
      B.grid = B.L.grid;
      counted(c, launch_prepared(B.L, B.P, st), "pair kernel");
    }
    if (timed) {
      check(cudaEventRecord(ev1, st), "event record");
      c->pending_ev0 = ev0;
      c->pending_ev1 = ev1;
    }
  }
  for (int t = 0; t < B.nT; ++t) {
    const LensBuilt& LB = B.lb[B.tl[t]];
    if (B.n_items > 0 && LB.n_groups > 0)
      counted(c, launch_patch_reduce(B.item_sums, B.tdesc[t].item_base, LB.d_patch_groups, B.n_patch_eff, nb,
                                     B.dpatch[t], st), "patch reduce");
    else
      check(cudaMemsetAsync(B.dpatch[t], 0, sizeof(double) * kQ * nb * B.n_patch_eff, st), "memset patch");
  }
}

// Per-lens outputs, the wait for the launch, and the totals and normalised
// outputs of every task (host, fixed order).
void batch_finish(tpcf_ctx* c, Batch& B, const tpcf_bins* bins, tpcf_result* outs) {
  Phase ph_reduce("tpcf: outputs");
  cudaStream_t st = c->stream;
  const int nb = B.nb, nT = B.nT, n_patch_eff = B.n_patch_eff, n_patch = B.n_patch;
  std::vector<std::vector<double>> hpatch(nT);
  for (int t = 0; t < nT; ++t) {
    const LensBuilt& LB = B.lb[B.tl[t]];
    hpatch[t].resize((size_t)kQ * nb * n_patch_eff);
    check(cudaMemcpyAsync(hpatch[t].data(), B.dpatch[t], sizeof(double) * kQ * nb * n_patch_eff,
                          cudaMemcpyDeviceToHost, st), "D2H patch");
    if (B.want_lens[t]) {
      const tpcf_result& o = outs[t];
      const int64_t nA = B.lens_n[B.tl[t]];
      auto dev_out = [&](void* user, size_t bytes) -> void* {
        if (!user) return nullptr;
        void* d = is_device_ptr(user) ? user : ws_alloc(c, bytes);
        check(cudaMemsetAsync(d, 0, bytes, st), "memset lens out");
        return d;
      };
      const size_t mb = sizeof(float) * nb * (size_t)std::max<int64_t>(nA, 0);
      float* xE = (float*)dev_out(o.xi_E_marks, mb);
      float* xB = (float*)dev_out(o.xi_B_marks, mb);
      float* Km = (float*)dev_out(o.K_marks, mb);
      float* wm = (float*)dev_out(o.w_marks, mb);
      float* mw = (float*)dev_out(o.marks_weight, sizeof(float) * std::max<int64_t>(nA, 0));
      double* ls = (double*)dev_out(o.lens_sums, sizeof(double) * 6 * nb * (size_t)std::max<int64_t>(nA, 0));
      double* lr = (double*)dev_out(o.lens_raw, sizeof(double) * 6 * nb * (size_t)std::max<int64_t>(nA, 0));
      const bool marks_all = xE && xB && Km && wm;
      if (!marks_all && (xE || xB || Km || wm))
        throw Failure(TPCF_ERR_INVALID_ARG, "xi_E_marks, xi_B_marks, K_marks and w_marks go together");
      if (LB.n_valid > 0 && B.n_items > 0 && B.lens_acc)
        counted(c, launch_lens_outputs(B.lens_acc + B.tdesc[t].lens_acc_off, LB.rec, LB.perm, LB.n_valid, nb, xE,
                                       xB, Km, wm, mw, ls, lr, st), "lens outputs");
      if (xE && xE != (void*)o.xi_E_marks) copy_out(c, o.xi_E_marks, xE, mb);
      if (xB && xB != (void*)o.xi_B_marks) copy_out(c, o.xi_B_marks, xB, mb);
      if (Km && Km != (void*)o.K_marks) copy_out(c, o.K_marks, Km, mb);
      if (wm && wm != (void*)o.w_marks) copy_out(c, o.w_marks, wm, mb);
      if (mw && mw != (void*)o.marks_weight) copy_out(c, o.marks_weight, mw, sizeof(float) * nA);
      if (ls && ls != (void*)o.lens_sums) copy_out(c, o.lens_sums, ls, sizeof(double) * 6 * nb * nA);
      if (lr && lr != (void*)o.lens_raw) copy_out(c, o.lens_raw, lr, sizeof(double) * 6 * nb * nA);
    }
  }
  unsigned herr = 0;
  check(cudaMemcpyAsync(&herr, B.head + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, st), "D2H err");
  check(cudaStreamSynchronize(st), "sync results");
  if (herr & kErrTimeout) throw Failure(TPCF_ERR_TIMEOUT, "a bounded device wait timed out in the pair kernel");
  if (herr) throw Failure(TPCF_ERR_CUDA, "device error flags " + std::to_string(herr));
  if (c->pending_ev0) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->pending_ev0, c->pending_ev1);
    c->last_pair_ms = ms;
    cudaEventDestroy(c->pending_ev0);
    cudaEventDestroy(c->pending_ev1);
    c->pending_ev0 = c->pending_ev1 = nullptr;
  }

  // ---- totals and normalised outputs (host, fixed order)
  std::vector<float> centers(nb);
  bin_centers_f32(bins, centers.data());
  static const int pub_row[6] = {QDW, QGT, QGX, QW, QK, QN};  // public row order (dw, gt, gx, w, K, n)
  c->last_pairs = 0;
  for (int t = 0; t < nT; ++t) {
    tpcf_result& o = outs[t];
    std::vector<double> tot((size_t)kQ * nb, 0.0);
    for (int p = 0; p < n_patch_eff; ++p)
      for (int q = 0; q < kQ * nb; ++q) tot[q] += hpatch[t][(size_t)p * kQ * nb + q];
    std::vector<double> sdw(nb), sgt(nb), sgx(nb), sw(nb), sK(nb);
    std::vector<int64_t> np(nb);
    std::vector<float> mt(nb), gt(nb), gx(nb), ww(nb);
    for (int b = 0; b < nb; ++b) {
      sdw[b] = tot[QDW * nb + b]; sgt[b] = tot[QGT * nb + b]; sgx[b] = tot[QGX * nb + b];
      sw[b] = tot[QW * nb + b]; sK[b] = tot[QK * nb + b]; np[b] = (int64_t)llround(tot[QN * nb + b]);
      c->last_pairs += np[b];
      mt[b] = (float)(sdw[b] / sw[b]);
      gt[b] = sK[b] > 0 ? (float)(sgt[b] / sK[b]) : 0.f;
      gx[b] = sK[b] > 0 ? (float)(sgx[b] / sK[b]) : 0.f;
      ww[b] = (float)sw[b];
    }
    copy_out(c, o.sum_dw, sdw.data(), sizeof(double) * nb);
    copy_out(c, o.sum_gt, sgt.data(), sizeof(double) * nb);
    copy_out(c, o.sum_gx, sgx.data(), sizeof(double) * nb);
    copy_out(c, o.sum_w, sw.data(), sizeof(double) * nb);
    copy_out(c, o.sum_K, sK.data(), sizeof(double) * nb);
    copy_out(c, o.n_pairs, np.data(), sizeof(int64_t) * nb);
    copy_out(c, o.theta, centers.data(), sizeof(float) * nb);
    if (!B.sharded) {
      copy_out(c, o.mean_theta, mt.data(), sizeof(float) * nb);
      copy_out(c, o.g_t, gt.data(), sizeof(float) * nb);
      copy_out(c, o.g_x, gx.data(), sizeof(float) * nb);
      copy_out(c, o.weights, ww.data(), sizeof(float) * nb);
    }
    if (o.patch_sums && B.use_patch_any) {
      std::vector<double> ps((size_t)n_patch * 6 * nb);
      for (int p = 0; p < n_patch; ++p)
        for (int r = 0; r < 6; ++r)
          for (int b = 0; b < nb; ++b)
            ps[((size_t)p * 6 + r) * nb + b] = hpatch[t][(size_t)p * kQ * nb + pub_row[r] * nb + b];
      copy_out(c, o.patch_sums, ps.data(), sizeof(double) * ps.size());
    }
    check(cudaStreamSynchronize(st), "sync outputs");  // host staging vectors are freed at scope exit
  }
}

// Everything one batched call needs; outs[t] receives task t.
tpcf_status run_batch(tpcf_ctx* c, int mode, std::vector<LensIn> lens, std::vector<SrcIn> srcs,
                      const std::vector<int>& tl, const std::vector<int>& ts, const tpcf_bins* bins, int n_patch,
                      tpcf_result* outs) {
  auto t_start = std::chrono::steady_clock::now();
  Batch B;
  batch_setup(c, mode, std::move(lens), std::move(srcs), tl, ts, bins, n_patch, outs, B);
  batch_launch(c, B, c->time_pairs);
  vlog(c, "mode=%d tasks=%d items=%d grid=%d bt=%d has_m=%d has_z=%d", mode, B.nT, B.n_items, B.grid, B.bt,
       (int)B.has_m, (int)B.has_z);
  batch_finish(c, B, bins, outs);
  c->last_call_ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
  vlog(c, "call %.3f ms, pairs %lld", c->last_call_ms, (long long)c->last_pairs);
  return TPCF_OK;
}

tpcf_status fail(tpcf_ctx* c, const Failure& f) {
  if (c) c->err = f.msg;
  return f.status;
}

}  // namespace

// ============================================================== C ABI ======
extern "C" {

int32_t tpcf_abi_version(void) { return TPCF_ABI_VERSION; }

tpcf_status tpcf_create(tpcf_ctx** out, int32_t device, const tpcf_opts* opts) {
  if (!out) return TPCF_ERR_INVALID_ARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return TPCF_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= n) return TPCF_ERR_INVALID_ARG;
  tpcf_ctx* c = new tpcf_ctx();
  c->device = device;
  if (opts) c->opts = *opts;
  else {
    std::memset(&c->opts, 0, sizeof(c->opts));
    c->opts.use_grid = 1;
  }
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    delete c;
    return TPCF_ERR_CUDA;
  }
  c->stream = c->own_stream;
  cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
  int major = 0;
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device);
  if (major < 10) {
    cudaStreamDestroy(c->own_stream);
    delete c;
    return TPCF_ERR_NO_DEVICE;  // kernels are built for sm_100a only
  }
  *out = c;
  return TPCF_OK;
}

tpcf_status tpcf_destroy(tpcf_ctx* c) {
  if (!c) return TPCF_OK;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  for (auto& s : c->slots)
    if (s.ptr) cudaFree(s.ptr);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  delete c;
  return TPCF_OK;
}

const char* tpcf_last_error(const tpcf_ctx* c) { return c ? c->err.c_str() : "no context"; }

tpcf_status tpcf_set_stream(tpcf_ctx* c, void* s) {
  if (!c) return TPCF_ERR_INVALID_ARG;
  c->stream = s ? (cudaStream_t)s : c->own_stream;
  return TPCF_OK;
}

int64_t tpcf_kernel_launches(const tpcf_ctx* c) { return c ? c->launches : 0; }

tpcf_status tpcf_set_timing(tpcf_ctx* c, int32_t enable) {
  if (!c) return TPCF_ERR_INVALID_ARG;
  c->time_pairs = enable != 0;
  return TPCF_OK;
}

tpcf_status tpcf_set_cell_size(tpcf_ctx* c, double cell_size) {
  if (!c || !(cell_size >= 0) || !std::isfinite(cell_size)) return TPCF_ERR_INVALID_ARG;
  c->opts.cell_size = cell_size;
  return TPCF_OK;
}

tpcf_status tpcf_debug_inject(tpcf_ctx* c, int64_t fail_alloc, int32_t skip_tile, uint32_t wait_polls) {
  if (!c || fail_alloc < -1 || skip_tile < -1) return TPCF_ERR_INVALID_ARG;
  c->fail_alloc = fail_alloc;
  c->skip_tile = skip_tile;
  c->wait_limit = wait_polls;
  return TPCF_OK;
}

tpcf_status tpcf_set_tile_shape(tpcf_ctx* c, int32_t group_size, int32_t tile_chunks) {
  if (!c || (group_size != 0 && group_size != 32 && group_size != 64 && group_size != 128) ||
      (tile_chunks != 0 && tile_chunks != 1 && tile_chunks != 2))
    return TPCF_ERR_INVALID_ARG;
  c->opts.group_size = group_size;
  c->opts.tile_chunks = tile_chunks;
  return TPCF_OK;
}

tpcf_status tpcf_set_spherical(tpcf_ctx* c, int32_t on) {
  if (!c || (on != 0 && on != 1)) return TPCF_ERR_INVALID_ARG;
  c->opts.spherical = on;
  return TPCF_OK;
}

tpcf_status tpcf_chord_edges(const tpcf_bins* bins, double* chord_sq) {
  if (!bins || !chord_sq) return TPCF_ERR_INVALID_ARG;
  std::vector<double> e(kMaxBins + 1), e2(kMaxBins + 1);
  tpcf_status s = canonical_edges(bins, e.data(), e2.data());
  if (s != TPCF_OK) return s;
  if (!(e[bins->n_bin] <= 3.14159265358979)) return TPCF_ERR_INVALID_ARG;
  for (int i = 0; i <= bins->n_bin; ++i) chord_sq[i] = canon_chord2(e[i]);
  return TPCF_OK;
}

tpcf_status tpcf_unit_vectors(tpcf_ctx* c, const float* lam, const float* phi, int64_t n, float* hi, float* lo) {
  if (!c || n < 0 || (n > 0 && (!lam || !phi || !hi || !lo))) return TPCF_ERR_INVALID_ARG;
  try {
    begin_call(c);
    if (n == 0) return TPCF_OK;
    const float* dl = stage(c, lam, n);
    const float* dp = stage(c, phi, n);
    float* dh = is_device_ptr(hi) ? hi : (float*)ws_alloc(c, sizeof(float) * 3 * (size_t)n);
    float* dlo = is_device_ptr(lo) ? lo : (float*)ws_alloc(c, sizeof(float) * 3 * (size_t)n);
    counted(c, launch_unit_vectors(dl, dp, n, dh, dlo, c->stream), "unit vectors");
    if (dh != hi) copy_out(c, hi, dh, sizeof(float) * 3 * (size_t)n);
    if (dlo != lo) copy_out(c, lo, dlo, sizeof(float) * 3 * (size_t)n);
    check(cudaStreamSynchronize(c->stream), "sync unit vectors");
    return TPCF_OK;
  } catch (const Failure& f) {
    return fail(c, f);
  }
}

tpcf_status tpcf_set_shard(tpcf_ctx* c, int32_t index, int32_t count) {
  if (!c || count < 0 || (count > 1 && (index < 0 || index >= count))) return TPCF_ERR_INVALID_ARG;
  c->opts.shard_index = index;
  c->opts.shard_count = count;
  return TPCF_OK;
}

tpcf_status tpcf_measure_fp32_peak(tpcf_ctx* c, double* tflops) {
  if (!c || !tflops) return TPCF_ERR_INVALID_ARG;
  try {
    begin_call(c);
    float* out = (float*)ws_alloc(c, 16);
    const int threads = 256, blocks = c->num_sms * 8, iters = 1 << 16;
    cudaEvent_t e0, e1;
    check(cudaEventCreate(&e0), "event");
    check(cudaEventCreate(&e1), "event");
    counted(c, launch_ffma_peak(out, blocks, threads, 1024, c->stream), "ffma warm-up");
    check(cudaEventRecord(e0, c->stream), "event record");
    counted(c, launch_ffma_peak(out, blocks, threads, iters, c->stream), "ffma peak");
    check(cudaEventRecord(e1, c->stream), "event record");
    check(cudaEventSynchronize(e1), "event sync");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *tflops = 2.0 * 8.0 * (double)iters * threads * blocks / (ms * 1e-3) / 1e12;
    return TPCF_OK;
  } catch (const Failure& f) {
    return fail(c, f);
  }
}

tpcf_status tpcf_measure_fp64_peak(tpcf_ctx* c, double* tflops) {
  if (!c || !tflops) return TPCF_ERR_INVALID_ARG;
  try {
    begin_call(c);
    double* out = (double*)ws_alloc(c, 16);
    const int threads = 256, blocks = c->num_sms * 8, iters = 1 << 14;
    cudaEvent_t e0, e1;
    check(cudaEventCreate(&e0), "event");
    check(cudaEventCreate(&e1), "event");
    counted(c, launch_dfma_peak(out, blocks, threads, 256, c->stream), "dfma warm-up");
    check(cudaEventRecord(e0, c->stream), "event record");
    counted(c, launch_dfma_peak(out, blocks, threads, iters, c->stream), "dfma peak");
    check(cudaEventRecord(e1, c->stream), "event record");
    check(cudaEventSynchronize(e1), "event sync");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *tflops = 2.0 * 8.0 * (double)iters * threads * blocks / (ms * 1e-3) / 1e12;
    return TPCF_OK;
  } catch (const Failure& f) {
    return fail(c, f);
  }
}

tpcf_status tpcf_last_stats(const tpcf_ctx* c, tpcf_stats* s) {
  if (!c || !s) return TPCF_ERR_INVALID_ARG;
  s->pair_kernel_ms = c->time_pairs ? c->last_pair_ms : 0.0;
  s->call_ms = c->last_call_ms;
  s->n_pairs = c->last_pairs;
  s->h2d_bytes = c->h2d_bytes;
  s->kernel_launches = c->launches;
  s->workspace_bytes = 0;
  for (const auto& sl : c->slots) s->workspace_bytes += (int64_t)sl.bytes;
  return TPCF_OK;
}

tpcf_status tpcf_canonical_edges(const tpcf_bins* bins, double* edges, double* edges_sq) {
  if (!bins || !edges || !edges_sq) return TPCF_ERR_INVALID_ARG;
  return canonical_edges(bins, edges, edges_sq);
}

tpcf_status tpcf_bin_centers(const tpcf_bins* bins, float* centers) {
  if (!bins || !centers) return TPCF_ERR_INVALID_ARG;
  std::vector<double> e(kMaxBins + 1), e2(kMaxBins + 1);
  tpcf_status s = canonical_edges(bins, e.data(), e2.data());
  if (s != TPCF_OK) return s;
  bin_centers_f32(bins, centers);
  return TPCF_OK;
}

tpcf_status tpcf_shear_scalar(tpcf_ctx* c, const float* xA, const float* yA, const float* zA, const float* valA,
                              const float* wA, int64_t nA, const float* xB, const float* yB, const float* zB,
                              const float* e1B, const float* e2B, const float* wB, const float* mB, int64_t nB,
                              const tpcf_bins* bins, const int32_t* patchA, int32_t n_patch, tpcf_result* out) {
  if (!c || !bins || !out) return TPCF_ERR_INVALID_ARG;
  try {
    std::vector<LensIn> L{{nA, xA, yA, zA, valA, wA, patchA}};
    std::vector<SrcIn> S{{nB, xB, yB, zB, e1B, e2B, wB, mB}};
    return run_batch(c, 0, L, S, {0}, {0}, bins, n_patch, out);
  } catch (const Failure& f) {
    return fail(c, f);
  }
}

tpcf_status tpcf_scalar_scalar(tpcf_ctx* c, const float* xA, const float* yA, const float* valA, const float* wA,
                               int64_t nA, const float* xB, const float* yB, const float* kE, const float* kB,
                               const float* wB, int64_t nB, const tpcf_bins* bins, const int32_t* patchA,
                               int32_t n_patch, tpcf_result* out) {
  if (!c || !bins || !out) return TPCF_ERR_INVALID_ARG;
  try {
    std::vector<LensIn> L{{nA, xA, yA, nullptr, valA, wA, patchA}};
    std::vector<SrcIn> S{{nB, xB, yB, nullptr, kE, kB, wB, nullptr}};
    return run_batch(c, 1, L, S, {0}, {0}, bins, n_patch, out);
  } catch (const Failure& f) {
    return fail(c, f);
  }
}

tpcf_status tpcf_batch_shear_scalar(tpcf_ctx* c, int32_t n_lens_cat, const tpcf_lens_catalog* lenses,
                                    int32_t n_src_cat, const tpcf_shear_catalog* sources, int32_t n_task,
                                    const int32_t* task_lens, const int32_t* task_src, const tpcf_bins* bins,
                                    int32_t n_patch, tpcf_result* outs) {
  if (!c || !bins || !outs || n_lens_cat < 1 || n_src_cat < 1 || n_task < 1 || !lenses || !sources || !task_lens ||
      !task_src)
    return TPCF_ERR_INVALID_ARG;
  try {
    std::vector<LensIn> L;
    for (int i = 0; i < n_lens_cat; ++i) {
      const tpcf_lens_catalog& l = lenses[i];
      L.push_back({l.n, l.x, l.y, l.z, l.val, l.w, l.patch});
    }
    std::vector<SrcIn> S;
    for (int i = 0; i < n_src_cat; ++i) {
      const tpcf_shear_catalog& s = sources[i];
      S.push_back({s.n, s.x, s.y, s.z, s.e1, s.e2, s.w, s.m});
    }
    std::vector<int> tl(task_lens, task_lens + n_task), ts(task_src, task_src + n_task);
    return run_batch(c, 0, L, S, tl, ts, bins, n_patch, outs);
  } catch (const Failure& f) {
    return fail(c, f);
  }
}

// ------------------------------------------------------------ plans --------
// A prepared batched call: the grids, lens groups and sorted work items of
// one tpcf_batch_shear_scalar call, built once and kept in the plan's own
// workspace, so that the pair kernel and the per-patch reductions can be
// enqueued again (and recorded into a CUDA graph) without host work.
}  // extern "C"

struct tpcf_plan {
  tpcf_ctx* ctx = nullptr;  // the plan's own context; its stream is the caller's
  Batch B;
  tpcf_bins bins{};
  std::vector<tpcf_result> shape;  // which outputs each task has (non-null fields)
  size_t slot_mark = 0;            // workspace slots of the batch; later ones are the outputs' scratch
};

extern "C" {

tpcf_status tpcf_plan_shear_scalar(tpcf_ctx* c, int32_t n_lens_cat, const tpcf_lens_catalog* lenses,
                                   int32_t n_src_cat, const tpcf_shear_catalog* sources, int32_t n_task,
                                   const int32_t* task_lens, const int32_t* task_src, const tpcf_bins* bins,
                                   int32_t n_patch, const tpcf_result* outs, tpcf_plan** plan) {
  if (!c || !bins || !outs || !plan || n_lens_cat < 1 || n_src_cat < 1 || n_task < 1 || !lenses || !sources ||
      !task_lens || !task_src)
    return TPCF_ERR_INVALID_ARG;
  *plan = nullptr;
  if (c->opts.spherical) {
    c->err = "plans are planar";
    return TPCF_ERR_NOT_SUPPORTED;
  }
  tpcf_ctx* pc = nullptr;
  tpcf_status st = tpcf_create(&pc, c->device, &c->opts);
  if (st != TPCF_OK) return st;
  pc->stream = c->stream;
  tpcf_plan* pl = new tpcf_plan();
  pl->ctx = pc;
  pl->bins = *bins;
  pl->shape.assign(outs, outs + n_task);
  try {
    std::vector<LensIn> L;
    for (int i = 0; i < n_lens_cat; ++i) {
      const tpcf_lens_catalog& l = lenses[i];
      L.push_back({l.n, l.x, l.y, l.z, l.val, l.w, l.patch});
    }
    std::vector<SrcIn> S;
    for (int i = 0; i < n_src_cat; ++i) {
      const tpcf_shear_catalog& s = sources[i];
      S.push_back({s.n, s.x, s.y, s.z, s.e1, s.e2, s.w, s.m});
    }
    std::vector<int> tl(task_lens, task_lens + n_task), ts(task_src, task_src + n_task);
    batch_setup(pc, 0, L, S, tl, ts, bins, n_patch, outs, pl->B);
    check(cudaStreamSynchronize(pc->stream), "sync plan");
    pl->slot_mark = pc->next_slot;
  } catch (const Failure& f) {
    c->err = f.msg;
    tpcf_destroy(pc);
    delete pl;
    return f.status;
  }
  *plan = pl;
  return TPCF_OK;
}

tpcf_status tpcf_plan_launch(tpcf_plan* pl) {
  if (!pl) return TPCF_ERR_INVALID_ARG;
  try {
    batch_launch(pl->ctx, pl->B, false);
  } catch (const Failure& f) {
    return fail(pl->ctx, f);
  }
  return TPCF_OK;
}

tpcf_status tpcf_plan_results(tpcf_plan* pl, tpcf_result* outs) {
  if (!pl || !outs) return TPCF_ERR_INVALID_ARG;
  for (int t = 0; t < pl->B.nT; ++t) {  // the per-lens outputs must be the ones the plan was made for
    const tpcf_result& a = pl->shape[t];
    const tpcf_result& b = outs[t];
    if (!a.xi_E_marks != !b.xi_E_marks || !a.xi_B_marks != !b.xi_B_marks || !a.K_marks != !b.K_marks ||
        !a.w_marks != !b.w_marks || !a.marks_weight != !b.marks_weight || !a.lens_sums != !b.lens_sums ||
        !a.lens_raw != !b.lens_raw) {
      pl->ctx->err = "per-lens outputs differ from the plan's";
      return TPCF_ERR_INVALID_ARG;
    }
  }
  try {
    pl->ctx->next_slot = pl->slot_mark;  // the outputs' staging reuses the same slots every time
    batch_finish(pl->ctx, pl->B, &pl->bins, outs);
  } catch (const Failure& f) {
    return fail(pl->ctx, f);
  }
  return TPCF_OK;
}

tpcf_status tpcf_plan_set_stream(tpcf_plan* pl, void* stream) {
  if (!pl) return TPCF_ERR_INVALID_ARG;
  pl->ctx->stream = stream ? (cudaStream_t)stream : pl->ctx->own_stream;
  return TPCF_OK;
}

const char* tpcf_plan_last_error(const tpcf_plan* pl) { return pl ? pl->ctx->err.c_str() : ""; }

tpcf_status tpcf_plan_destroy(tpcf_plan* pl) {
  if (!pl) return TPCF_OK;
  tpcf_destroy(pl->ctx);
  delete pl;
  return TPCF_OK;
}

tpcf_status tpcf_batch_scalar_scalar(tpcf_ctx* c, int32_t n_lens_cat, const tpcf_lens_catalog* lenses,
                                     int32_t n_kappa_cat, const tpcf_kappa_catalog* kappas, int32_t n_task,
                                     const int32_t* task_lens, const int32_t* task_kappa, const tpcf_bins* bins,
                                     int32_t n_patch, tpcf_result* outs) {
  if (!c || !bins || !outs || n_lens_cat < 1 || n_kappa_cat < 1 || n_task < 1 || !lenses || !kappas ||
      !task_lens || !task_kappa)
    return TPCF_ERR_INVALID_ARG;
  try {
    std::vector<LensIn> L;
    for (int i = 0; i < n_lens_cat; ++i) {
      const tpcf_lens_catalog& l = lenses[i];
      L.push_back({l.n, l.x, l.y, nullptr, l.val, l.w, l.patch});
    }
    std::vector<SrcIn> S;
    for (int i = 0; i < n_kappa_cat; ++i) {
      const tpcf_kappa_catalog& k = kappas[i];
      S.push_back({k.n, k.x, k.y, nullptr, k.kE, k.kB, k.w, nullptr});
    }
    std::vector<int> tl(task_lens, task_lens + n_task), ts(task_kappa, task_kappa + n_task);
    return run_batch(c, 1, L, S, tl, ts, bins, n_patch, outs);
  } catch (const Failure& f) {
    return fail(c, f);
  }
}

}  // extern "C"
