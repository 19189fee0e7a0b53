// Host side of merged launches (see launch.cuh): the record of one launch,
// the per-thread recorder a batch installs while it enqueues its members,
// and the table a merged launch reads.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <vector>

namespace msm {

// ---- recording (host) ----
struct LaunchRec {
  enum Kind { kKernel, kClear, kFork, kJoin } kind = kKernel;
  const void *kmulti = nullptr;  // k_multi instantiation (kKernel)
  uint3 grid{1, 1, 1};
  dim3 block{1, 1, 1};
  size_t smem = 0;
  std::vector<char> pack;     // argument bytes
  std::vector<char> uniform;  // the uniform last argument (ParamTab::u), or empty
  // layout of kmulti's parameter (ParamTab): size, member capacity, field
  // offsets and the stride of the packs
  size_t tab_bytes = 0, off_u = 0, off_n = 0, off_first = 0, off_grid = 0, off_packs = 0,
         pack_stride = 0;
  int tab_max = 0;
  int branch = 0;          // 0: the member's main stream, 1: its short-range branch
  void *ptr = nullptr;     // kClear: bytes to zero
  size_t bytes = 0;
};

struct Recorder {
  std::vector<LaunchRec> recs;
  cudaStream_t aux = nullptr;  // the member's short-range branch stream
  bool ok = true;              // false: a launch that cannot be merged was met
};

Recorder *&tls_recorder();

inline int rec_branch(Recorder *r, cudaStream_t s) { return (r->aux && s == r->aux) ? 1 : 0; }

// Marks a launcher whose kernels are not written for merging: recording
// then fails (the batch keeps its per-member graph) and nothing is launched.
inline bool record_unsupported() {
  if (Recorder *r = tls_recorder()) {
    r->ok = false;
    return true;
  }
  return false;
}

// cudaMemsetAsync(ptr, 0, bytes, s), or a record of it
inline cudaError_t clear_async(void *ptr, size_t bytes, cudaStream_t s) {
  if (Recorder *r = tls_recorder()) {
    LaunchRec rec;
    rec.kind = LaunchRec::kClear;
    rec.ptr = ptr;
    rec.bytes = bytes;
    rec.branch = rec_branch(r, s);
    r->recs.push_back(std::move(rec));
    return cudaSuccess;
  }
  return cudaMemsetAsync(ptr, 0, bytes, s);
}

// Sets the dynamic shared memory limit of a recorded launch's k_multi
inline cudaError_t multi_smem_attr(const void *kmulti, size_t bytes) {
  return cudaFuncSetAttribute(kmulti, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

}  // namespace msm
