// Batches: many independent systems (each an FF handle built by FF_build)
// evaluated by ONE CUDA graph launch. No counterpart in the reference, which
// evaluates one system per FF_energy call (code/forcefield0.c:684-780).
//
// Small systems cannot fill 148 SMs on their own: a 500-atom box is 63 pair
// clusters, a few warps per phase. The batch captures every member's launch
// sequence (the same kernels FF_energy_device replays) into one graph, spread
// over K parallel branches (fork and join by events during capture), so the
// hardware scheduler runs kernels of different systems side by side and the
// host pays one launch per step. Members go to branches longest-first onto
// the least-loaded branch (LPT on the atom count). K is given, or picked on
// the first call by timing replays of candidate graphs (the batch autotuner).
// The graph is re-captured, and updated in place where its shape allows, when
// a pointer, a weight or a member's box (FF_rebuild / FF_rebuild_device)
// changes.
#include <algorithm>
#include <cstring>
#include <new>
#include <numeric>
#include <vector>

#include <cuda_runtime.h>

#include "engine.h"
#include "msmpb_b200.h"

struct FFBatch {
  std::vector<FF *> ffs;
  int device = 0;
  int requested = 0;  // branches asked for (0 = tune)
  int branches = 0;   // branches of the current graph
  cudaStream_t cap = nullptr;
  std::vector<cudaStream_t> br;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraphExec_t exec = nullptr;
  // what the current graph was captured with
  std::vector<const void *> key_ptrs;
  std::vector<double> key_w;
  std::vector<long> key_ver;
  int launches = 0;
  int last_error = MSMPB_OK;
};

namespace {

constexpr int kMaxBranches = 64;
constexpr int kW = msm::kMaxLevels + 1;

int fail(FFBatch *b, int code) {
  if (b && code != MSMPB_OK) b->last_error = code;
  return code;
}

struct Inputs {
  const double *const *pos, *const *q, *const *weight;
  double *const *force, *const *phi;
  double *energy;
};

void make_key(const FFBatch *b, const Inputs &in, std::vector<const void *> &ptrs,
              std::vector<double> &w, std::vector<long> &ver) {
  const size_t n = b->ffs.size();
  ptrs.assign(5 * n, nullptr);
  w.assign(kW * n, 1.0);
  ver.resize(n);
  for (size_t i = 0; i < n; ++i) {
    ptrs[5 * i] = in.pos[i];
    ptrs[5 * i + 1] = in.q[i];
    ptrs[5 * i + 2] = in.force ? in.force[i] : nullptr;
    ptrs[5 * i + 3] = in.phi ? in.phi[i] : nullptr;
    ptrs[5 * i + 4] = in.energy ? in.energy + i : nullptr;
    const double *wi = in.weight ? in.weight[i] : nullptr;
    const int L = std::min(b->ffs[i]->maxLevel, msm::kMaxLevels);
    if (wi)
      for (int l = 0; l <= L; ++l) w[kW * i + l] = wi[l];
    ver[i] = msm::engine_version(b->ffs[i]->dev);
  }
}

// Captures every member's evaluation on K branches into *graph.
int capture(FFBatch *b, int K, const Inputs &in, cudaGraph_t *graph) {
  const int n = (int)b->ffs.size();
  *graph = nullptr;
  if (cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
    return MSMPB_ERR_CUDA;
  int st = MSMPB_OK;
  if (cudaEventRecord(b->fork, b->cap) != cudaSuccess) st = MSMPB_ERR_CUDA;
  for (int k = 0; k < K && st == MSMPB_OK; ++k)
    if (cudaStreamWaitEvent(b->br[k], b->fork, 0) != cudaSuccess) st = MSMPB_ERR_CUDA;
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int c) { return b->ffs[a]->N > b->ffs[c]->N; });
  std::vector<double> load(K, 0.0);
  int launches = 0;
  for (int i : order) {
    if (st != MSMPB_OK) break;
    const int k = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    load[k] += b->ffs[i]->N;
    double w[kW];
    const int L = std::min(b->ffs[i]->maxLevel, msm::kMaxLevels);
    for (int l = 0; l <= L; ++l) w[l] = in.weight && in.weight[i] ? in.weight[i][l] : 1.0;
    msm::EvalRequest r{};
    r.pos = in.pos[i];
    r.q = in.q[i];
    r.host = false;
    r.weight = w;
    r.force = in.force ? in.force[i] : nullptr;
    r.phi = in.phi ? in.phi[i] : nullptr;
    r.energy_dev = in.energy ? in.energy + i : nullptr;
    r.stream = b->br[k];
    r.timing = false;
    st = msm::engine_enqueue(b->ffs[i]->dev, r, b->br[k]);
    launches += msm::engine_kernel_launches(b->ffs[i]->dev);
  }
  for (int k = 0; k < K && st == MSMPB_OK; ++k) {
    if (cudaEventRecord(b->join[k], b->br[k]) != cudaSuccess ||
        cudaStreamWaitEvent(b->cap, b->join[k], 0) != cudaSuccess)
      st = MSMPB_ERR_CUDA;
  }
  cudaGraph_t g = nullptr;
  // always end the capture, also after a failure, so the streams stay usable
  const cudaError_t ce = cudaStreamEndCapture(b->cap, &g);
  if (st == MSMPB_OK && ce != cudaSuccess) st = MSMPB_ERR_CUDA;
  if (st != MSMPB_OK) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return st;
  }
  *graph = g;
  b->launches = launches;
  return MSMPB_OK;
}

// Captures on K branches and installs the result as b->exec.
int install(FFBatch *b, int K, const Inputs &in) {
  cudaGraph_t g;
  int st = capture(b, K, in, &g);
  if (st != MSMPB_OK) return st;
  cudaError_t ie = cudaErrorUnknown;
  if (b->exec && b->branches == K) {
    cudaGraphExecUpdateResultInfo info{};
    ie = cudaGraphExecUpdate(b->exec, g, &info);
    if (ie != cudaSuccess) cudaGetLastError();
  }
  if (ie != cudaSuccess) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
    ie = cudaGraphInstantiate(&b->exec, g, 0);
  }
  cudaGraphDestroy(g);
  if (ie != cudaSuccess) {
    b->exec = nullptr;
    cudaGetLastError();
    return MSMPB_ERR_CUDA;
  }
  b->branches = K;
  return MSMPB_OK;
}

int launch(FFBatch *b, cudaStream_t s) {
  for (FF *f : b->ffs) {
    const int st = msm::engine_begin(f->dev, s);
    if (st != MSMPB_OK) return st;
  }
  return cudaGraphLaunch(b->exec, s) == cudaSuccess ? MSMPB_OK : MSMPB_ERR_CUDA;
}

// The batch autotuner: replays a graph per candidate branch count on s and
// keeps the fastest (median of three timed replays after one warm-up).
int tune(FFBatch *b, const Inputs &in, cudaStream_t s) {
  const int n = (int)b->ffs.size();
  std::vector<int> cands;
  for (int K : {4, 8, 16, 32, 64})
    if (K < n) cands.push_back(K);
  cands.push_back(std::min(n, kMaxBranches));
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return MSMPB_ERR_CUDA;
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return MSMPB_ERR_CUDA;
  }
  int best = cands.back(), st = MSMPB_OK;
  float best_ms = 1e30f;
  for (int K : cands) {
    st = install(b, K, in);
    if (st != MSMPB_OK) break;
    float t[3];
    if ((st = launch(b, s)) != MSMPB_OK) break;
    for (int r = 0; r < 3 && st == MSMPB_OK; ++r) {
      cudaEventRecord(e0, s);
      st = launch(b, s);
      cudaEventRecord(e1, s);
      if (cudaEventSynchronize(e1) != cudaSuccess) st = MSMPB_ERR_CUDA;
      cudaEventElapsedTime(&t[r], e0, e1);
    }
    if (st != MSMPB_OK) break;
    std::sort(t, t + 3);
    if (t[1] < best_ms) {
      best_ms = t[1];
      best = K;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st != MSMPB_OK) return st;
  b->requested = best;
  return install(b, best, in);
}

}  // namespace

extern "C" {

FFBatch *FF_batch_new(FF *const *members, int n, int branches, int *status) {
  int dummy;
  int &st = status ? *status : dummy;
  st = MSMPB_ERR_ARGUMENT;
  if (!members || n <= 0 || branches < 0 || branches > kMaxBranches) return nullptr;
  for (int i = 0; i < n; ++i) {
    if (!members[i]) return nullptr;
    if (!members[i]->dev) {  // not built, or no device
      st = MSMPB_ERR_STATE;
      return nullptr;
    }
    for (int j = 0; j < i; ++j)
      if (members[j] == members[i]) return nullptr;  // would race on its buffers
  }
  const int device = msm::engine_device(members[0]->dev);
  for (int i = 1; i < n; ++i)
    if (msm::engine_device(members[i]->dev) != device) return nullptr;
  FFBatch *b = new (std::nothrow) FFBatch;
  if (!b) {
    st = MSMPB_ERR_NOMEM;
    return nullptr;
  }
  b->ffs.assign(members, members + n);
  b->device = device;
  b->requested = branches;
  st = MSMPB_ERR_CUDA;
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess) {
    FF_batch_delete(b);
    return nullptr;
  }
  const int K = std::min(n, kMaxBranches);
  b->br.assign(K, nullptr);
  b->join.assign(K, nullptr);
  for (int k = 0; k < K; ++k)
    if (cudaStreamCreateWithFlags(&b->br[k], cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->join[k], cudaEventDisableTiming) != cudaSuccess) {
      FF_batch_delete(b);
      return nullptr;
    }
  st = MSMPB_OK;
  return b;
}

int FF_batch_energy_device(FFBatch *b, const double *const *position_d,
                           const double *const *charge_d, const double *const *weight,
                           double *const *force_d, double *const *potential_d,
                           double *energy_d, void *stream) {
  if (!b) return MSMPB_ERR_ARGUMENT;
  b->last_error = MSMPB_OK;  // the status of this call
  if (!position_d || !charge_d) return fail(b, MSMPB_ERR_ARGUMENT);
  for (size_t i = 0; i < b->ffs.size(); ++i)
    if (!position_d[i] || !charge_d[i]) return fail(b, MSMPB_ERR_ARGUMENT);
  if (cudaSetDevice(b->device) != cudaSuccess) return fail(b, MSMPB_ERR_CUDA);
  cudaGetLastError();
  const Inputs in{position_d, charge_d, weight, force_d, potential_d, energy_d};
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  std::vector<const void *> ptrs;
  std::vector<double> w;
  std::vector<long> ver;
  make_key(b, in, ptrs, w, ver);
  int st = MSMPB_OK;
  if (b->requested == 0) {
    st = tune(b, in, s);
  } else if (!b->exec || ptrs != b->key_ptrs || w != b->key_w || ver != b->key_ver) {
    st = install(b, std::min<int>(b->requested, (int)b->ffs.size()), in);
  }
  if (st != MSMPB_OK) return fail(b, st);
  b->key_ptrs.swap(ptrs);
  b->key_w.swap(w);
  b->key_ver.swap(ver);
  return fail(b, launch(b, s));
}

int FF_batch_branches(const FFBatch *b) { return b ? b->branches : 0; }

int FF_batch_kernel_launches(const FFBatch *b) { return b ? b->launches : 0; }

int FF_batch_last_error(const FFBatch *b) { return b ? b->last_error : MSMPB_ERR_ARGUMENT; }

void FF_batch_delete(FFBatch *b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  for (cudaEvent_t e : b->join)
    if (e) cudaEventDestroy(e);
  for (cudaStream_t s : b->br)
    if (s) cudaStreamDestroy(s);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->cap) cudaStreamDestroy(b->cap);
  delete b;
}

}  // extern "C"
