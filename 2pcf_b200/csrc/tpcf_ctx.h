// tpcf_ctx.h -- the context object behind the opaque tpcf_ctx handle and the
// host helpers shared by the C-ABI translation units.
#pragma once
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cstdint>
#include <string>
#include <vector>

#include "tpcf_b200.h"

namespace tpcf {

// Internal failure carried to the C boundary, where it becomes a status code.
struct Failure {
  tpcf_status status;
  std::string msg;
  Failure(tpcf_status s, std::string m) : status(s), msg(std::move(m)) {}
};

// NVTX range over one phase of a call (grid build, pair kernel, reduction,
// k-means, resampling), visible in Nsight timelines; free when no tool is
// attached.
struct Phase {
  explicit Phase(const char* name) { nvtxRangePushA(name); }
  ~Phase() { nvtxRangePop(); }
  Phase(const Phase&) = delete;
  Phase& operator=(const Phase&) = delete;
};

// Grow-only device buffer.  A call takes slots in a fixed order, so repeated
// calls of the same shape allocate nothing after the first.
struct Slot {
  void* ptr;
  size_t bytes;
};

}  // namespace tpcf

struct tpcf_ctx {
  int device = 0;
  int num_sms = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  tpcf_opts opts{};
  std::string err;
  std::vector<tpcf::Slot> slots;
  size_t next_slot = 0;
  int64_t launches = 0;
  int64_t h2d_bytes = 0;
  // statistics of the last call
  bool time_pairs = false;
  cudaEvent_t pending_ev0 = nullptr, pending_ev1 = nullptr;
  double last_pair_ms = 0.0;
  double last_call_ms = 0.0;
  int64_t last_pairs = 0;
  // fault injection for tests (tpcf_debug_inject): the fail_alloc-th workspace
  // allocation from now fails with TPCF_ERR_OOM (-1: none); pair-kernel tile
  // whose copy is never issued (-1: none) and the poll limit of the waits
  int64_t fail_alloc = -1;
  int32_t skip_tile = -1;
  uint32_t wait_limit = 0;
};

namespace tpcf {
void* ws_alloc(tpcf_ctx* c, size_t bytes);
bool is_device_ptr(const void* p);
void check(cudaError_t e, const char* what);
void counted(tpcf_ctx* c, cudaError_t e, const char* what);
template <class T>
const T* stage(tpcf_ctx* c, const T* p, int64_t n);
void copy_out(tpcf_ctx* c, void* dst, const void* src, size_t bytes);
void begin_call(tpcf_ctx* c);
tpcf_status canonical_edges(const tpcf_bins* b, double* e, double* e2);
}  // namespace tpcf
