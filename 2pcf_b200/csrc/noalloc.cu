// noalloc.cu -- tpcf_shear_scalar_noalloc: the shear-scalar pair sum for callers
// that cannot allocate device memory.
//
// Who needs it: a caller whose device memory belongs to someone else -- a
// framework's caching allocator or a fixed memory pool that owns the GPU's
// memory, where an extra cudaMalloc fails or fragments the pool -- and a
// caller that cannot afford cudaMalloc/cudaFree, which may synchronise the
// whole device, inside a latency-critical loop.  The regular entry points grow
// a per-context device workspace with cudaMalloc; this one uses only the
// static array below.
//
// Scratch: one file-scope device array of kScratchBytes (64 MiB).  Every GPU
// that loads the library holds it until the process exits.  Host code never
// uses the array's name as an address: on the first call on each device (with
// that device current) the address is looked up with cudaGetSymbolAddress and
// cached; that first call must therefore come before any stream capture.
// Every call reuses the same array, whose contents persist between calls:
// everything that must start at zero is cleared at the start of each call, and
// calls that overlap on the GPU (two host threads, or two streams) race on it.
//
// The computation is the one of tpcf_shear_scalar (same grid, same kernels, same
// canonical binning, items reduced in the same order), without patches and
// per-lens outputs.  A call whose buffers do not fit in kScratchBytes fails
// with TPCF_ERR_OVERFLOW before any pair work.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "tpcf_b200.h"
#include "tpcf_ctx.h"
#include "tpcf_internal.cuh"
#include "tpcf_kernels.h"

namespace {

using namespace tpcf;

constexpr size_t kScratchBytes = size_t(64) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_addr_mu;
void* g_addr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (looked up once
// per device; it stays valid as long as the device's primary context does, so
// cudaDeviceReset between calls is not supported).
void* scratch_base(int device) {
  if (device < 0 || device >= kMaxDevices) throw Failure(TPCF_ERR_INVALID_ARG, "device index too large");
  std::lock_guard<std::mutex> lk(g_addr_mu);
  if (!g_addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      throw Failure(TPCF_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    }
    g_addr[device] = p;
  }
  return g_addr[device];
}

// Bump allocator over the static scratch.
struct Carver {
  unsigned char* base;
  size_t used = 0;
  void* take(size_t bytes) {
    const size_t off = (used + 255) & ~size_t(255);
    if (off + bytes > kScratchBytes)
      throw Failure(TPCF_ERR_OVERFLOW, "the call needs more than the " + std::to_string(kScratchBytes >> 20) +
                                           " MiB static scratch (already " + std::to_string(off) +
                                           " bytes, asking " + std::to_string(bytes) + " more); use tpcf_shear_scalar");
    used = off + bytes;
    return base + off;
  }
};

template <class T>
const T* stage_na(tpcf_ctx* c, Carver& cv, const T* p, int64_t n) {
  if (!p || n <= 0) return p;
  if (is_device_ptr(p)) return p;
  T* d = static_cast<T*>(cv.take(sizeof(T) * (size_t)n));
  check(cudaMemcpyAsync(d, p, sizeof(T) * (size_t)n, cudaMemcpyHostToDevice, c->stream), "H2D input");
  return d;
}

__global__ void k_na_groups(int* gstart, int n_groups, int n_valid, int gsz, int2* items, int* patch_groups) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g <= n_groups) gstart[g] = min(g * gsz, n_valid);
  if (g < n_groups) items[g] = make_int2(0, g);
  if (g == 0) {
    patch_groups[0] = 0;
    patch_groups[1] = n_groups;
  }
}

tpcf_status run_noalloc(tpcf_ctx* c, const float* xA, const float* yA, const float* zA, const float* valA,
                        const float* wA, int64_t nA, const float* xB, const float* yB, const float* zB,
                        const float* e1B, const float* e2B, const float* wB, const float* mB, int64_t nB,
                        const tpcf_bins* bins, tpcf_result* o) {
  check(cudaSetDevice(c->device), "cudaSetDevice");
  cudaStream_t st = c->stream;
  const int nb = bins->n_bin;
  double e[kMaxBins + 1], e2[kMaxBins + 1];
  tpcf_status bs = canonical_edges(bins, e, e2);
  if (bs != TPCF_OK) throw Failure(bs, "invalid binning");
  if (c->opts.spherical) throw Failure(TPCF_ERR_NOT_SUPPORTED, "spherical coordinates are not supported");
  if (o->xi_E_marks || o->xi_B_marks || o->K_marks || o->w_marks || o->marks_weight || o->lens_sums ||
      o->patch_sums)
    throw Failure(TPCF_ERR_INVALID_ARG, "per-lens and per-patch outputs are not available without allocation");
  if (nA < 0 || nB < 0 || nA > (1ll << 31) - 2 || nB > (1ll << 31) - 2)
    throw Failure(TPCF_ERR_INVALID_ARG, "catalogue size out of range");
  if ((nA > 0 && (!xA || !yA || !valA || !wA)) || (nB > 0 && (!xB || !yB || !e1B || !e2B || !wB)))
    throw Failure(TPCF_ERR_INVALID_ARG, "missing input array");

  Carver cv{static_cast<unsigned char*>(scratch_base(c->device))};
  xA = stage_na(c, cv, xA, nA); yA = stage_na(c, cv, yA, nA); zA = stage_na(c, cv, zA, nA);
  valA = stage_na(c, cv, valA, nA); wA = stage_na(c, cv, wA, nA);
  xB = stage_na(c, cv, xB, nB); yB = stage_na(c, cv, yB, nB); zB = stage_na(c, cv, zB, nB);
  e1B = stage_na(c, cv, e1B, nB); e2B = stage_na(c, cv, e2B, nB); wB = stage_na(c, cv, wB, nB);
  mB = stage_na(c, cv, mB, nB);

  // bounding boxes (lens catalogue 0, source catalogue 1); cleared by bbox_init
  int* box_ord = (int*)cv.take(sizeof(int) * 16);
  unsigned long long* cnt = (unsigned long long*)cv.take(sizeof(unsigned long long) * 2);
  int* pr = (int*)cv.take(sizeof(int) * 4);
  float* boxf = (float*)cv.take(sizeof(float) * 16);
  counted(c, launch_bbox_init(box_ord, cnt, pr, 2, st), "bbox init");
  counted(c, launch_bbox(xA, yA, zA, wA, nullptr, nullptr, nA, 1, box_ord, cnt, pr, st), "bbox lens");
  counted(c, launch_bbox(xB, yB, zB, nullptr, nullptr, mB, nB, 0, box_ord + 8, cnt + 1, pr + 2, st), "bbox src");
  counted(c, launch_bbox_finish(box_ord, boxf, 16, st), "bbox finish");
  float hbox[16];
  unsigned long long hcnt[2];
  check(cudaMemcpyAsync(hbox, boxf, sizeof(hbox), cudaMemcpyDeviceToHost, st), "D2H box");
  check(cudaMemcpyAsync(hcnt, cnt, sizeof(hcnt), cudaMemcpyDeviceToHost, st), "D2H count");
  check(cudaStreamSynchronize(st), "sync bbox");

  const bool has_m = mB != nullptr && hcnt[1] > 0 && hbox[8 + 6] != 0.f;
  const bool has_z = hcnt[0] > 0 && hcnt[1] > 0 && hbox[5] > hbox[8 + 4];
  const bool logb = bins->spacing == TPCF_LOG;
  const int qa = has_m ? 6 : 5;
  int bt = 128;
  while (bt > 32 && (size_t)nb * qa * bt * 4 > 100 * 1024) bt /= 2;
  const double Rd = bins->x_max;
  const float R = (float)(Rd * (1.0 + 1e-6));

  // source grid, same rule as the regular entry points
  GridDesc g{};
  const int ns_valid = (int)hcnt[1];
  const float* b = hbox + 8;
  const float x0 = ns_valid ? b[0] : 0.f, y0 = ns_valid ? b[1] : 0.f;
  const float ex = ns_valid ? b[2] - b[0] : 0.f, ey = ns_valid ? b[3] - b[1] : 0.f;
  double cell = c->opts.cell_size > 0 ? c->opts.cell_size : Rd / 16.0;
  const double span = std::max((double)ex, (double)ey);
  if (!c->opts.use_grid) cell = span * 2.0 + 1.0;
  while ((span / cell + 2.0) * (span / cell + 2.0) > (double)(1 << 24)) cell *= 1.5;
  // The cell table (4 bytes per cell) may take at most an eighth of the
  // scratch: a small theta_max over a wide field gets coarser cells here than
  // in the regular entry points.  The results do not depend on the cell side.
  while ((span / cell + 2.0) * (span / cell + 2.0) * 4.0 > (double)(kScratchBytes / 8)) cell *= 1.5;
  if (!(cell > 0)) cell = 1.0;
  const int ncx = std::max(1, (int)std::floor(ex / cell) + 1), ncy = std::max(1, (int)std::floor(ey / cell) + 1);
  const unsigned ncells = (unsigned)ncx * (unsigned)ncy;
  g.x0 = x0; g.y0 = y0; g.cell = (float)cell; g.inv_cell = (float)(1.0 / cell);
  g.ncx = ncx; g.ncy = ncy; g.n_valid = ns_valid;
  int* cs = (int*)cv.take(sizeof(int) * (ncells + 1));
  const int n_chunks = std::max((ns_valid + kChunk - 1) / kChunk, 1);
  SrcPair* pairs = (SrcPair*)cv.take(sizeof(SrcPair) * (kChunk / 2) * n_chunks);
  ChunkMeta* cmeta = (ChunkMeta*)cv.take(sizeof(ChunkMeta) * n_chunks);
  if (nB > 0) {
    unsigned* k0 = (unsigned*)cv.take(sizeof(unsigned) * nB);
    unsigned* k1 = (unsigned*)cv.take(sizeof(unsigned) * nB);
    int* i0 = (int*)cv.take(sizeof(int) * nB);
    int* i1 = (int*)cv.take(sizeof(int) * nB);
    int cell_bits = 1;
    while (cell_bits < 32 && (1ull << cell_bits) <= (unsigned long long)ncells) ++cell_bits;
    const int mb = std::min(16, (32 - cell_bits) & ~1);
    const int end_bit = cell_bits + mb;
    size_t tb = 0;
    check(sort_pairs_u32(nullptr, tb, k0, k1, i0, i1, (int)nB, end_bit, st), "sort size");
    void* tmp = cv.take(tb);
    counted(c, launch_src_keys(xB, yB, zB, nB, x0, y0, g.inv_cell, ncx, ncy, mb, k0, i0, st), "src keys");
    check(sort_pairs_u32(tmp, tb, k0, k1, i0, i1, (int)nB, end_bit, st), "sort sources");
    counted(c, launch_cell_start(k1, nB, ncells, mb, cs, st), "cell start");
    counted(c, launch_src_pairs(i1, ns_valid, 0, xB, yB, zB, e1B, e2B, wB, mB, pairs, cmeta, st), "src gather");
  } else {
    check(cudaMemsetAsync(cs, 0, sizeof(int) * (ncells + 1), st), "memset cells");
  }
  g.cell_start = cs;
  g.pairs = pairs;
  g.meta = cmeta;
  float margin = 0.f;
  for (int i = 0; i < 2; ++i)
    if (hcnt[i] > 0)
      margin = std::max(margin, std::fabs(hbox[8 * i]) + std::fabs(hbox[8 * i + 1]) + std::fabs(hbox[8 * i + 2]) +
                                    std::fabs(hbox[8 * i + 3]));
  margin = (float)(1e-5 * (margin + Rd) + 1e-4 * g.cell);

  // lenses: sorted by Hilbert index, groups of 32 (one per warp of the pair kernel; one patch)
  const int nl_valid = (int)hcnt[0];
  float4* lrec = (float4*)cv.take(sizeof(float4) * std::max(nl_valid, 1));
  float* zs = (float*)cv.take(sizeof(float) * std::max(nl_valid, 1));
  int* perm = (int*)cv.take(sizeof(int) * std::max(nl_valid, 1));
  if (nA > 0 && nl_valid > 0) {
    unsigned long long* k0 = (unsigned long long*)cv.take(sizeof(unsigned long long) * nA);
    unsigned long long* k1 = (unsigned long long*)cv.take(sizeof(unsigned long long) * nA);
    int* i0 = (int*)cv.take(sizeof(int) * nA);
    int* i1 = (int*)cv.take(sizeof(int) * nA);
    size_t tb = 0;
    check(sort_pairs_u64(nullptr, tb, k0, k1, i0, i1, (int)nA, st), "sort size");
    void* tmp = cv.take(tb);
    const float4 lbox = make_float4(hbox[0], hbox[1], hbox[2], hbox[3]);
    counted(c, launch_lens_keys(xA, yA, zA, wA, nullptr, nA, lbox, k0, i0, st), "lens keys");
    check(sort_pairs_u64(tmp, tb, k0, k1, i0, i1, (int)nA, st), "sort lenses");
    counted(c, launch_lens_gather(i1, nl_valid, xA, yA, zA, valA, wA, lrec, zs, perm, st), "lens gather");
  }
  constexpr int kGroup = 32;
  const int n_groups = (nl_valid + kGroup - 1) / kGroup;
  int* gstart = (int*)cv.take(sizeof(int) * (n_groups + 1));
  int2* items = (int2*)cv.take(sizeof(int2) * std::max(n_groups, 1));
  int* pgroups = (int*)cv.take(sizeof(int) * 2);
  float4* gbox = (float4*)cv.take(sizeof(float4) * std::max(n_groups, 1));
  double* item_sums = (double*)cv.take(sizeof(double) * kQ * nb * std::max(n_groups, 1));
  double* psum = (double*)cv.take(sizeof(double) * kQ * nb);
  TaskDesc* d_task = (TaskDesc*)cv.take(sizeof(TaskDesc));
  LensDesc* d_lens = (LensDesc*)cv.take(sizeof(LensDesc));
  GridDesc* d_grid = (GridDesc*)cv.take(sizeof(GridDesc));
  double* d_e2 = (double*)cv.take(sizeof(double) * (nb + 1));
  float* d_e2f = (float*)cv.take(sizeof(float) * (nb + 1));
  int* head = (int*)cv.take(sizeof(int) * 4);
  unsigned* err = (unsigned*)(head + 1);

  k_na_groups<<<(n_groups + 1 + 255) / 256, 256, 0, st>>>(gstart, n_groups, nl_valid, kGroup, items, pgroups);
  counted(c, cudaGetLastError(), "groups");
  counted(c, launch_group_box(lrec, gstart, n_groups, gbox, st), "group box");
  TaskDesc td{};
  td.lens_cat = 0; td.src_cat = 0; td.item_base = 0; td.lens_acc_off = -1; td.margin = margin;
  LensDesc ld{};
  ld.rec = lrec; ld.z = zs; ld.group_start = gstart; ld.group_box = gbox; ld.n_valid = nl_valid;
  ld.n_groups = n_groups;
  float e2f[kMaxBins + 1];
  for (int i = 0; i <= nb; ++i) e2f[i] = (float)e2[i];
  check(cudaMemcpyAsync(d_task, &td, sizeof(td), cudaMemcpyHostToDevice, st), "H2D task");
  check(cudaMemcpyAsync(d_lens, &ld, sizeof(ld), cudaMemcpyHostToDevice, st), "H2D lens desc");
  check(cudaMemcpyAsync(d_grid, &g, sizeof(g), cudaMemcpyHostToDevice, st), "H2D grid desc");
  check(cudaMemcpyAsync(d_e2, e2, sizeof(double) * (nb + 1), cudaMemcpyHostToDevice, st), "H2D edges");
  check(cudaMemcpyAsync(d_e2f, e2f, sizeof(float) * (nb + 1), cudaMemcpyHostToDevice, st), "H2D edges f");
  check(cudaMemsetAsync(head, 0, sizeof(int) * 4, st), "clear queue head and error flags");
  if (n_groups > 0) {
    PairParams P{};
    P.tasks = d_task; P.lenses = d_lens; P.grids = d_grid; P.items = items; P.n_items = n_groups;
    P.nb = nb; P.queue_head = head; P.item_sums = item_sums; P.lens_acc = nullptr; P.err = err;
    P.e2 = d_e2; P.e2f = d_e2f; P.R = R;
    if (logb) {
      const double l0 = std::log2(e2[0]), l1 = std::log2(e2[nb]);
      const double A = nb / (l1 - l0);
      P.binA = (float)A;
      P.binB = (float)(-l0 * A);
      P.eps = 1.0f / 32768.0f;
    } else {
      P.binA = P.binB = 0.f;
      P.eps = 4e-6f;
    }
    int grid = 0;
    counted(c, launch_pairs(P, 0, has_m, has_z, logb, bt, 2, 0, c->num_sms, st, &grid), "pair kernel");
    counted(c, launch_patch_reduce(item_sums, 0, pgroups, 1, nb, psum, st), "patch reduce");
  } else {
    check(cudaMemsetAsync(psum, 0, sizeof(double) * kQ * nb, st), "clear sums");
  }
  double hs[kQ * kMaxBins];
  unsigned herr = 0;
  check(cudaMemcpyAsync(hs, psum, sizeof(double) * kQ * nb, cudaMemcpyDeviceToHost, st), "D2H sums");
  check(cudaMemcpyAsync(&herr, err, sizeof(unsigned), cudaMemcpyDeviceToHost, st), "D2H err");
  check(cudaStreamSynchronize(st), "sync results");
  if (herr & kErrTimeout) throw Failure(TPCF_ERR_TIMEOUT, "a bounded device wait timed out in the pair kernel");
  if (herr) throw Failure(TPCF_ERR_CUDA, "device error flags " + std::to_string(herr));

  double sdw[kMaxBins], sgt[kMaxBins], sgx[kMaxBins], sw[kMaxBins], sK[kMaxBins];
  int64_t np[kMaxBins];
  float mt[kMaxBins], gt[kMaxBins], gx[kMaxBins], ww[kMaxBins];
  for (int i = 0; i < nb; ++i) {
    sdw[i] = hs[QDW * nb + i]; sgt[i] = hs[QGT * nb + i]; sgx[i] = hs[QGX * nb + i];
    sw[i] = hs[QW * nb + i]; sK[i] = hs[QK * nb + i]; np[i] = (int64_t)llround(hs[QN * nb + i]);
    mt[i] = (float)(sdw[i] / sw[i]);
    gt[i] = sK[i] > 0 ? (float)(sgt[i] / sK[i]) : 0.f;
    gx[i] = sK[i] > 0 ? (float)(sgx[i] / sK[i]) : 0.f;
    ww[i] = (float)sw[i];
  }
  float centers[kMaxBins];
  tpcf_bin_centers(bins, centers);
  copy_out(c, o->sum_dw, sdw, sizeof(double) * nb);
  copy_out(c, o->sum_gt, sgt, sizeof(double) * nb);
  copy_out(c, o->sum_gx, sgx, sizeof(double) * nb);
  copy_out(c, o->sum_w, sw, sizeof(double) * nb);
  copy_out(c, o->sum_K, sK, sizeof(double) * nb);
  copy_out(c, o->n_pairs, np, sizeof(int64_t) * nb);
  copy_out(c, o->theta, centers, sizeof(float) * nb);
  copy_out(c, o->mean_theta, mt, sizeof(float) * nb);
  copy_out(c, o->g_t, gt, sizeof(float) * nb);
  copy_out(c, o->g_x, gx, sizeof(float) * nb);
  copy_out(c, o->weights, ww, sizeof(float) * nb);
  check(cudaStreamSynchronize(st), "sync outputs");
  return TPCF_OK;
}

}  // namespace

extern "C" tpcf_status tpcf_shear_scalar_noalloc(tpcf_ctx* c, const float* xA, const float* yA, const float* zA,
                                                 const float* valA, const float* wA, int64_t nA, const float* xB,
                                                 const float* yB, const float* zB, const float* e1B,
                                                 const float* e2B, const float* wB, const float* mB, int64_t nB,
                                                 const tpcf_bins* bins, tpcf_result* out) {
  if (!c || !bins || !out) return TPCF_ERR_INVALID_ARG;
  try {
    return run_noalloc(c, xA, yA, zA, valA, wA, nA, xB, yB, zB, e1B, e2B, wB, mB, nB, bins, out);
  } catch (const Failure& f) {
    c->err = f.msg;
    return f.status;
  }
}
