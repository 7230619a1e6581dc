// tpcf_internal.cuh -- device-side data layout shared by the kernels and the
// host orchestration of libtpcf_b200.
//
// Layout in HBM (one call, many catalogues):
//   source catalogue  -> cell grid: records sorted by row-major cell index,
//                        stored as 32-source sub-chunks (SrcPair form, 1 KB)
//                        with one ChunkMeta each, cell_start[ncx*ncy+1]
//   lens catalogue    -> lenses sorted by (patch, Hilbert index); groups of at
//                        most BT consecutive lenses that never straddle a
//                        patch; one bounding box per group
//   work item         -> (task, group): one lens group against every source
//                        row that intersects the group box dilated by theta_max
//   item_sums         -> FP64 [Q][n_bin] per (task, group), summed per patch
//                        by k_patch_reduce in a fixed order (deterministic)
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace tpcf {

constexpr int kMaxBins = 128;
constexpr int kMaxRows = 256;   // cell rows scanned per chunk of one work item
constexpr int kTile = 256;      // sources per shared-memory tile
constexpr int kQ = 6;           // quantities per bin in item/patch/lens sums

// Quantity rows of every FP64 sum array (item, patch, lens and result sums).
enum Quantity { QGT = 0, QGX = 1, QW = 2, QDW = 3, QN = 4, QK = 5 };

// Device error bits, OR-ed into PairParams::err.
enum ErrBits : unsigned {
  kErrTimeout = 1u,   // a bounded mbarrier wait ran out
  kErrRows = 2u,      // more cell rows than the row chunking expects
  kErrBounds = 4u,    // an index check failed (skipped the access)
};

// A source in shared memory / HBM.  Shear: a = {x, y, -e1*w, -e2*w},
// b = {w, (1+m)*w, z, 0}.  Scalar-scalar: a = {x, y, kE*w, kB*w}, b = {w, w, 0, 0}.
struct __align__(16) SrcRec {
  float4 a;
  float4 b;
};

// Two consecutive sources (2k, 2k+1) of a 32-source sub-chunk in shared
// memory with their fields interleaved, so that one 64-bit register pair holds
// a field of both sources: the operand form of the sm_100 packed FP32
// instructions (add/mul/fma .f32x2).  The planar source grid is built in this
// form (the same 64 bytes as the two SrcRec).  p, q, w, K, z are a.z, a.w,
// b.x, b.y, b.z of SrcRec.
struct __align__(16) SrcPair {
  float4 xy;  // x0 x1 y0 y1
  float4 pq;  // p0 p1 q0 q1
  float4 wk;  // w0 w1 K0 K1
  float4 zn;  // z0 z1 0 0
};
static_assert(sizeof(SrcPair) == 2 * sizeof(SrcRec), "a SrcPair rewrites two SrcRec in place");
static_assert(kTile % 32 == 0, "tiles hold whole 32-source sub-chunks");

// Sources per sub-chunk.  A planar source grid stores its cell-sorted records
// as consecutive sub-chunks of 32 (16 SrcPair, 1 KB each; the last one padded
// with null sources), aligned to multiples of 32 in the sorted order, with one
// ChunkMeta per sub-chunk, so that the pair kernel copies them unchanged.
constexpr int kChunk = 32;
struct __align__(16) ChunkMeta {
  float4 box;  // {xmin, ymin, xmax, ymax} of its real sources
  float4 sum;  // {sum p, sum q, sum w, sum K} over its real sources
};

// A source on the sphere: the unit vector u of (lambda, phi) split into FP32
// hi + lo parts (u = hi + lo to ~2^-48), so that u_B - u_A keeps full FP32
// relative precision at small separations.  Shear: a = {hi, -e1*w},
// b = {lo, -e2*w}, c = {w, (1+m)*w, z, 0}; scalar-scalar: a = {hi, kE*w},
// b = {lo, kB*w}, c = {w, w, 0, 0}.
struct __align__(16) SrcRecS {
  float4 a;
  float4 b;
  float4 c;
};

// Cell grid of one source catalogue.  Planar: cells over (x, y).  Sphere:
// cells over (lambda reduced to [0, 2 pi), phi), records in `recs`.
struct GridDesc {
  float x0, y0, cell, inv_cell;
  int ncx, ncy;
  int n_valid;
  int pad;
  const int* cell_start;  // [ncx*ncy + 1]
  const SrcRec* rec;      // [n_valid], sorted by cell (lens grid of the adjoint)
  const SrcRecS* recs;    // [n_valid], sorted by cell (sphere), else nullptr
  const SrcPair* pairs;   // planar sources: [ceil(n_valid/32) * 16] in sub-chunk form
  const ChunkMeta* meta;  // [ceil(n_valid/32)]
};

struct LensDesc {
  const float4* rec;        // {x, y, val, w}, sorted (sphere: x = lambda in [0, 2 pi))
  const float* z;           // sorted z, or nullptr
  const int* group_start;   // [n_groups + 1] into the sorted lenses
  const float4* group_box;  // {xmin, ymin, xmax, ymax}
  int n_valid;
  int n_groups;
  const float4* pos;        // sphere: {hi.xyz, 0}, {lo.xyz, 0} per sorted lens, else nullptr
};

struct TaskDesc {
  int lens_cat;
  int src_cat;
  int item_base;            // row of (task, group 0) in item_sums
  float margin;             // FP32 guard on the reach of this task's rows and cells
  long long lens_acc_off;   // element offset of this task's per-lens sums, -1 = none
};

struct PairParams {
  const TaskDesc* tasks;
  const LensDesc* lenses;
  const GridDesc* grids;
  const int2* items;        // (task, group) in processing order
  int n_items;
  int nb;
  int* queue_head;
  double* item_sums;        // [n_slots][kQ][nb]
  double* lens_acc;         // per-lens FP64 [kQ][nb][n_valid] per task, or nullptr
  unsigned* err;
  const double* e2;         // canonical squared edges [nb+1]
  const float* e2f;         // FP32 squared edges [nb+1] (generic spacing)
  float R;                  // search radius: theta_max with a relative margin
  float binA, binB;         // log spacing: t = lg2(d2)*binA + binB
  float eps;                // guard band half-width in t units (log) or relative (generic)
  int flush_src;            // FP32 histogram -> FP64 after this many sources (0: 4096)
  // Fault injection for tests only (0 in every product call): 1 + the ring
  // index of a source tile whose bulk copy is never issued, so that the waits
  // on it run out (0: none), and the poll limit of the waits (0: kWaitPolls).
  int debug_skip_tile;
  unsigned wait_limit;
};

}  // namespace tpcf
