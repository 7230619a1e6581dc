// tpcf_kernels.h -- host-callable launchers of the device kernels
// (implemented in pairs.cu); used by the C-ABI layer in capi.cu.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>

#include "tpcf_internal.cuh"

namespace tpcf {

size_t pair_smem_bytes(int nb, int qa, int bt, int tch);
// bt = lenses per group (threads per block), tch = 32-source sub-chunks per
// source tile; variant 1 bins every pair one by one (A/B measurement).
cudaError_t launch_pairs(const PairParams& P, int mode, bool has_m, bool has_z, bool logb, int bt, int tch,
                         int variant, int num_sms, cudaStream_t st, int* grid);
// The same in two steps: prepare_pairs picks the kernel instantiation, sets
// its shared-memory attribute and sizes the grid; launch_prepared is one
// cudaLaunchKernel (no other API call, so it may be recorded into a graph).
struct PairLaunch {
  const void* func = nullptr;
  int grid = 0, block = 0;
  size_t smem = 0;
};
cudaError_t prepare_pairs(const PairParams& P, int mode, bool has_m, bool has_z, bool logb, int bt, int tch,
                          int variant, int num_sms, PairLaunch* L);
cudaError_t launch_prepared(const PairLaunch& L, const PairParams& P, cudaStream_t st);

// Spherical pair kernel (sphere.cu); P.grids[*].recs and P.lenses[*].pos set.
cudaError_t launch_pairs_sph(const PairParams& P, int mode, bool has_m, bool has_z, bool logb, int bt, int num_sms,
                             cudaStream_t st, int* grid);
cudaError_t launch_wrap_lambda(const float* x, long long n, float* out, cudaStream_t st);
cudaError_t launch_src_gather_sph(const int* idx, int n_valid, int mode, const float* lam, const float* phi,
                                  const float* z, const float* f1, const float* f2, const float* w, const float* m,
                                  SrcRecS* rec, cudaStream_t st);
cudaError_t launch_lens_pos_sph(const int* perm, int n_valid, const float* lam, const float* phi, float4* pos,
                                cudaStream_t st);
cudaError_t launch_unit_vectors(const float* lam, const float* phi, long long n, float* hi, float* lo,
                                cudaStream_t st);
cudaError_t launch_item_cost_sph(const int2* items, int n_items, const TaskDesc* tasks, const LensDesc* lenses,
                                 const GridDesc* grids, float R, unsigned long long* cost, int* order,
                                 cudaStream_t st);

cudaError_t launch_bbox_init(int* box_ord, unsigned long long* count, int* prange, int n, cudaStream_t st);
// box_ord holds 8 order-preserving ints per catalogue: minx, miny, maxx, maxy,
// minz, maxz, max|m|, unused.
cudaError_t launch_bbox(const float* x, const float* y, const float* z, const float* w, const int* patch,
                        const float* m, long long n, int kind, int* box_ord, unsigned long long* count,
                        int* prange, cudaStream_t st);
cudaError_t launch_bbox_finish(const int* box_ord, float* box, int n, cudaStream_t st);
// mb = bits of the within-cell Hilbert index in the source sort key.
cudaError_t launch_src_keys(const float* x, const float* y, const float* z, long long n, float x0, float y0,
                            float inv_cell, int ncx, int ncy, int mb, unsigned* keys, int* idx, cudaStream_t st);
cudaError_t launch_cell_start(const unsigned* keys, long long n, unsigned ncells, int mb, int* cell_start,
                              cudaStream_t st);
// Planar source grid records in sub-chunk form: pairs [ceil(n_valid/32)*16],
// meta [ceil(n_valid/32)].
cudaError_t launch_src_pairs(const int* idx, int n_valid, int mode, const float* x, const float* y,
                             const float* z, const float* f1, const float* f2, const float* w, const float* m,
                             SrcPair* pairs, ChunkMeta* meta, cudaStream_t st);
cudaError_t launch_lens_keys(const float* x, const float* y, const float* z, const float* w, const int* patch,
                             long long n, float4 box, unsigned long long* keys, int* idx, cudaStream_t st);
cudaError_t launch_lens_gather(const int* idx, int n_valid, const float* x, const float* y, const float* z,
                               const float* val, const float* w, float4* rec, float* zs, int* perm,
                               cudaStream_t st);
cudaError_t launch_patch_offsets(const unsigned long long* keys, int n_valid, int n_patch, int* off,
                                 cudaStream_t st);
cudaError_t launch_group_box(const float4* rec, const int* gstart, int n_groups, float4* box, cudaStream_t st);
cudaError_t launch_item_cost(const int2* items, int n_items, const TaskDesc* tasks, const LensDesc* lenses,
                             const GridDesc* grids, float R, unsigned long long* cost, int* order,
                             cudaStream_t st);
cudaError_t launch_permute_items(const int2* items, const int* order, int n, int index, int count, int2* out,
                                 cudaStream_t st);
cudaError_t launch_ffma_peak(float* out, int blocks, int threads, int iters, cudaStream_t st);
cudaError_t launch_dfma_peak(double* out, int blocks, int threads, int iters, cudaStream_t st);
cudaError_t launch_patch_reduce(const double* item_sums, int item_base, const int* patch_groups, int n_patch,
                                int nb, double* patch_sums, cudaStream_t st);
cudaError_t launch_lens_outputs(const double* acc, const float4* rec, const int* perm, int n_valid, int nb,
                                float* xi_E, float* xi_B, float* K_m, float* w_m, float* marks_weight,
                                double* lens_sums, double* lens_raw, cudaStream_t st);

cudaError_t launch_cov(const double* x, int n_s, int D, double* cov, cudaStream_t st);

cudaError_t sort_pairs_u32(void* tmp, size_t& tmp_bytes, const unsigned* kin, unsigned* kout, const int* vin,
                           int* vout, int n, int end_bit, cudaStream_t st);
cudaError_t sort_pairs_u64(void* tmp, size_t& tmp_bytes, const unsigned long long* kin, unsigned long long* kout,
                           const int* vin, int* vout, int n, cudaStream_t st);
cudaError_t sort_pairs_u64_desc(void* tmp, size_t& tmp_bytes, const unsigned long long* kin,
                                unsigned long long* kout, const int* vin, int* vout, int n, cudaStream_t st);

}  // namespace tpcf
