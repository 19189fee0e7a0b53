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
// the least-loaded branch (LPT on the atom count).
//
// Merged form (branches = -K, FF_BATCH_MERGED = -1): every member's launch sequence is
// recorded (launch.cuh) instead of launched, and the launches of the same
// kernel across members become ONE launch over a table of the members'
// arguments and block ranges (k_multi): a few tens of graph nodes for any
// number of systems, each phase one GPU-filling launch. The members are dealt
// over K branches of the graph whose merged chains overlap; within a branch
// the sequences are merged per segment
// (binning; the short-range branch, on its own graph branch; the grid
// branch; the combine), greedily taking at each step the kernel that is next
// for the most members. Each member's blocks compute exactly what its own
// launch computes, so results are bit-identical to FF_energy_device.
//
// The form (merged, or K branches) is given, or picked on the first call by
// timing replays of the candidates (the batch autotuner).
// The graph is re-captured, and updated in place where its shape allows, when
// a pointer, a weight or a member's box (FF_rebuild / FF_rebuild_device)
// changes.
#include <algorithm>
#include <cstdio>
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
  int merge_ok = -1;  // merged form: -1 untried, 0 a member cannot be merged, 1 fine
  std::vector<cudaStream_t> mbr;  // merged form: two streams per group
  std::vector<cudaEvent_t> mev;
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

// ---- merged form ----
// One merged launch: the members (index, their record) that run its kernel
struct Merged {
  const msm::LaunchRec *key = nullptr;
  size_t smem = 0;
  long nblocks = 0;
  std::vector<std::pair<int, const msm::LaunchRec *>> members;
};

// Greedy merge of one segment: lists[i] is member i's launch sequence. At
// each step one kernel (same merged kernel, block shape and uniform argument)
// runs for every member whose next launch it is, in groups of at most the
// kernel's table capacity. Preferred are kernels that no other member still
// needs later (so members whose sequences diverge, e.g. a three-pass scan
// against a one-pass one, catch up and merge again), and among those the one
// that is next for the most members.
void merge_segment(const std::vector<std::vector<const msm::LaunchRec *>> &lists,
                   std::vector<Merged> &out) {
  const int n = (int)lists.size();
  std::vector<size_t> cur(n, 0);
  auto same = [](const msm::LaunchRec *a, const msm::LaunchRec *c) {
    return a->kmulti == c->kmulti && a->block.x == c->block.x && a->block.y == c->block.y &&
           a->block.z == c->block.z && a->uniform == c->uniform;
  };
  // ahead: some member whose next launch is another kernel needs k later
  auto ahead = [&](const msm::LaunchRec *k) {
    for (int j = 0; j < n; ++j) {
      if (cur[j] >= lists[j].size() || same(lists[j][cur[j]], k)) continue;
      for (size_t t = cur[j] + 1; t < lists[j].size(); ++t)
        if (same(lists[j][t], k)) return true;
    }
    return false;
  };
  std::vector<const msm::LaunchRec *> seen;  // candidate kernels of this step
  for (;;) {
    const msm::LaunchRec *best = nullptr;
    int best_count = 0;
    bool best_ahead = true;
    seen.clear();
    for (int i = 0; i < n; ++i) {
      if (cur[i] >= lists[i].size()) continue;
      const msm::LaunchRec *k = lists[i][cur[i]];
      if (std::any_of(seen.begin(), seen.end(),
                      [&](const msm::LaunchRec *x) { return same(x, k); }))
        continue;
      seen.push_back(k);
      int count = 0;
      for (int j = 0; j < n; ++j)
        if (cur[j] < lists[j].size() && same(lists[j][cur[j]], k)) ++count;
      const bool a = ahead(k);
      if (!best || (best_ahead && !a) || (a == best_ahead && count > best_count)) {
        best_count = count;
        best = k;
        best_ahead = a;
      }
    }
    if (!best) return;
    Merged m;
    m.key = best;
    for (int i = 0; i < n; ++i) {
      if (cur[i] >= lists[i].size() || !same(lists[i][cur[i]], best)) continue;
      if ((int)m.members.size() == best->tab_max) {
        out.push_back(std::move(m));
        m = Merged{};
        m.key = best;
      }
      const msm::LaunchRec *r = lists[i][cur[i]++];
      m.members.emplace_back(i, r);
      m.smem = std::max(m.smem, r->smem);
      m.nblocks += (long)r->grid.x * r->grid.y * r->grid.z;
    }
    out.push_back(std::move(m));
  }
}

// The kernel parameter of a merged launch (the ParamTab of launch.cuh)
bool param_table(const Merged &m, std::vector<char> &buf) {
  const msm::LaunchRec &k = *m.key;
  buf.assign(k.tab_bytes, 0);
  if (!k.uniform.empty()) std::memcpy(buf.data() + k.off_u, k.uniform.data(), k.uniform.size());
  const int nm = (int)m.members.size();
  std::memcpy(buf.data() + k.off_n, &nm, sizeof(int));
  long acc = 0;
  for (int j = 0; j < nm; ++j) {
    const msm::LaunchRec *r = m.members[j].second;
    const int f = (int)acc;
    std::memcpy(buf.data() + k.off_first + sizeof(int) * j, &f, sizeof(int));
    std::memcpy(buf.data() + k.off_grid + sizeof(uint3) * j, &r->grid, sizeof(uint3));
    std::memcpy(buf.data() + k.off_packs + k.pack_stride * j, r->pack.data(), r->pack.size());
    acc += (long)r->grid.x * r->grid.y * r->grid.z;
  }
  const int f = (int)acc;
  std::memcpy(buf.data() + k.off_first + sizeof(int) * nm, &f, sizeof(int));
  return acc <= 0x7fffffffL;
}

// Records every member, merges the four segments of each of K branches and
// captures the merged launches into *graph. MSMPB_ERR_UNSUPPORTED: a member
// has a launch that cannot be merged (nothing captured).
int capture_merged(FFBatch *b, int K, const Inputs &in, cudaGraph_t *graph) {
  const int n = (int)b->ffs.size();
  *graph = nullptr;
  std::vector<msm::Recorder> recs(n);
  for (int i = 0; i < n; ++i) {
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
    r.timing = false;
    const int st = msm::engine_record(b->ffs[i]->dev, r, recs[i]);
    if (st != MSMPB_OK) return st;
    if (!recs[i].ok) return MSMPB_ERR_UNSUPPORTED;
  }
  if (cudaSetDevice(b->device) != cudaSuccess) return MSMPB_ERR_CUDA;
  // Members over G = K branches of the graph, each branch's members merged:
  // members sorted by order, precision and size, dealt round-robin, so every
  // branch holds a like mix; the branches' latency-bound phases (small FFTs,
  // scans) overlap other branches' compute.
  const int G = std::max(1, std::min(K, n));
  std::vector<int> ord(n), gof(n);
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int c) {
    const FF *x = b->ffs[a], *y = b->ffs[c];
    if (x->orderAcc != y->orderAcc) return x->orderAcc < y->orderAcc;
    if (x->precision != y->precision) return x->precision < y->precision;
    return x->N > y->N;
  });
  for (int t = 0; t < n; ++t) gof[ord[t]] = t % G;
  while ((int)b->mbr.size() < 2 * G) {
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return MSMPB_ERR_CUDA;
    b->mbr.push_back(st);
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return MSMPB_ERR_CUDA;
    b->mev.push_back(ev);
  }
  // segments per group: 0 binning, 1 short-range branch, 2 grid branch, 3 combine
  std::vector<std::vector<Merged>> ms(4 * G);
  for (int g = 0; g < G; ++g) {
    std::vector<std::vector<const msm::LaunchRec *>> seg[4];
    for (int i = 0; i < n; ++i) {
      if (gof[i] != g) continue;
      for (auto &v : seg) v.emplace_back();
      int state = 0;
      for (const msm::LaunchRec &r : recs[i].recs) {
        if (r.kind == msm::LaunchRec::kFork) state = 2;
        else if (r.kind == msm::LaunchRec::kJoin) state = 3;
        else if (r.kind == msm::LaunchRec::kKernel)
          seg[r.branch == 1 ? 1 : state].back().push_back(&r);
        else return MSMPB_ERR_UNSUPPORTED;
      }
    }
    for (int k = 0; k < 4; ++k) merge_segment(seg[k], ms[4 * g + k]);
  }
  // dynamic shared memory limits of the merged kernels
  // (one limit per kernel: the largest of its merged launches)
  std::vector<std::pair<const void *, size_t>> smem_max;
  for (auto &v : ms)
    for (const Merged &m : v) {
      auto it = std::find_if(smem_max.begin(), smem_max.end(),
                             [&](const std::pair<const void *, size_t> &x) {
                               return x.first == m.key->kmulti;
                             });
      if (it == smem_max.end())
        smem_max.emplace_back(m.key->kmulti, m.smem);
      else
        it->second = std::max(it->second, m.smem);
    }
  for (const auto &x : smem_max)
    if (x.second > 48 * 1024) {
      const cudaError_t ae = msm::multi_smem_attr(x.first, x.second);
      if (ae != cudaSuccess) {
        std::fprintf(stderr, "msmpb_b200: merged kernel shared memory %zu: %s\n", x.second,
                     cudaGetErrorString(ae));
        return MSMPB_ERR_CUDA;
      }
    }
  std::vector<char> buf;
  bool fits = true;
  auto launch_one = [&](const Merged &m, cudaStream_t s) {
    if (!param_table(m, buf)) fits = false;
    void *args[] = {buf.data()};
    const cudaError_t le = cudaLaunchKernel(m.key->kmulti, dim3((unsigned)m.nblocks),
                                            m.key->block, args, m.smem, s);
    if (le != cudaSuccess)
      std::fprintf(stderr,
                   "msmpb_b200: merged launch failed (%s): %d members, %ld blocks of %u, "
                   "%zu bytes shared, %zu bytes of parameters\n",
                   cudaGetErrorString(le), (int)m.members.size(), m.nblocks, m.key->block.x,
                   m.smem, m.key->tab_bytes);
    return le;
  };
  if (cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
    return MSMPB_ERR_CUDA;
  cudaError_t e = cudaEventRecord(b->fork, b->cap);
  int launches = 0;
  for (int g = 0; g < G && e == cudaSuccess; ++g) {
    cudaStream_t main = b->mbr[2 * g], side = b->mbr[2 * g + 1];
    cudaEvent_t evf = b->mev[2 * g], evj = b->mev[2 * g + 1];
    e = cudaStreamWaitEvent(main, b->fork, 0);
    for (const Merged &m : ms[4 * g])
      if (e == cudaSuccess) e = launch_one(m, main), ++launches;
    const bool branch = !ms[4 * g + 1].empty();
    if (branch && e == cudaSuccess) {
      e = cudaEventRecord(evf, main);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(side, evf, 0);
      for (const Merged &m : ms[4 * g + 1])
        if (e == cudaSuccess) e = launch_one(m, side), ++launches;
      if (e == cudaSuccess) e = cudaEventRecord(evj, side);
    }
    for (const Merged &m : ms[4 * g + 2])
      if (e == cudaSuccess) e = launch_one(m, main), ++launches;
    if (branch && e == cudaSuccess) e = cudaStreamWaitEvent(main, evj, 0);
    for (const Merged &m : ms[4 * g + 3])
      if (e == cudaSuccess) e = launch_one(m, main), ++launches;
    // the group's end joins the capture stream (reusing its fork event slot)
    if (e == cudaSuccess) e = cudaEventRecord(evf, main);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(b->cap, evf, 0);
  }
  cudaGraph_t g = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(b->cap, &g);
  if (e != cudaSuccess || ce != cudaSuccess || !fits) {
    if (ce != cudaSuccess)
      std::fprintf(stderr, "msmpb_b200: merged capture failed: %s\n", cudaGetErrorString(ce));
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return fits ? MSMPB_ERR_CUDA : MSMPB_ERR_UNSUPPORTED;
  }
  *graph = g;
  b->launches = launches;
  return MSMPB_OK;
}

// Captures on K branches (K < 0: the merged form on -K branches) and installs
// the result as b->exec.
int install(FFBatch *b, int K, const Inputs &in) {
  cudaGraph_t g;
  int st = K < 0 ? capture_merged(b, -K, in, &g) : capture(b, K, in, &g);
  if (K < 0) b->merge_ok = st == MSMPB_ERR_UNSUPPORTED ? 0 : 1;
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
    std::fprintf(stderr, "msmpb_b200: batch graph instantiation failed: %s\n",
                 cudaGetErrorString(ie));
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
  const cudaError_t ge = cudaGraphLaunch(b->exec, s);
  if (ge != cudaSuccess)
    std::fprintf(stderr, "msmpb_b200: batch graph launch failed: %s\n", cudaGetErrorString(ge));
  return ge == cudaSuccess ? MSMPB_OK : MSMPB_ERR_CUDA;
}

// The batch autotuner: replays a graph per candidate branch count on s and
// keeps the fastest (median of three timed replays after one warm-up).
int tune(FFBatch *b, const Inputs &in, cudaStream_t s) {
  const int n = (int)b->ffs.size();
  std::vector<int> cands;
  if (b->merge_ok != 0)
    for (int K : {1, 2, 4})
      if (K == 1 || K < n) cands.push_back(-K);
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
    if (K < 0 && st == MSMPB_ERR_UNSUPPORTED) {
      st = MSMPB_OK;  // a member cannot be merged: branches only
      continue;
    }
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
  if (!members || n <= 0 || branches < -kMaxBranches || branches > kMaxBranches) return nullptr;
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
    const int n = (int)b->ffs.size();
    st = install(b, b->requested < 0 ? -std::min(-b->requested, n) : std::min(b->requested, n), in);
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
  for (cudaEvent_t e : b->mev)
    if (e) cudaEventDestroy(e);
  for (cudaStream_t s : b->mbr)
    if (s) cudaStreamDestroy(s);
  for (cudaStream_t s : b->br)
    if (s) cudaStreamDestroy(s);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->cap) cudaStreamDestroy(b->cap);
  delete b;
}

}  // extern "C"
