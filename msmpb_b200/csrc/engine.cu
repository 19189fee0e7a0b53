// Device plan and the launch sequence of one MSM evaluation
// (code/forcefield1.c:101-235 restated for one B200):
//
//   bin + sort atoms (pair cells, finest-grid cells),   k_prep, scans, k_scatter2,
//   charge sums (per block in k_prep)                    k_sort_cells, k_gather2
//   charge-sum reduction (on the short-range branch)     k_qstats_final
//   cluster build (column counts in k_scatter2)          scan, k_cluster_fill
//   short-range pair sum                                 k_pair_clusters_f32/_f64
//   anterpolation -> q^1                                 k_anterp_tiles, k_anterp_fold
//   restriction q^l -> q^{l+1}, l < L                    k_restrict
//   top level: FFT(q^L) * khat_L -> e^L (FP64)           k_fft_plane/k_fft_xlines
//                                                        or k_fft_lines x5
//   for l = L-1..1: e^l = prolong(e^{l+1}) + w_l K_l q^l  k_prolong, k_pad, stencil
//   interpolation of e^1 -> E, phi_long                  k_grid_dot, k_interpolate
//   per-atom combine, energy reductions (FP64)           k_combine, k_energy_total
//
// Everything after the input copy is captured once into a CUDA graph and
// replayed; the graph is re-captured only when pointers, weights or the box
// change (after a box change it is updated in place where it can be).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "engine.h"
#include "kernels.h"
#include "msmpb_b200.h"

struct FFDevice {
  virtual ~FFDevice() {}
  virtual int update(const msm::Tables &t) = 0;
  // new box with the level stencils computed on the device, in the order of
  // `stream` (no host synchronisation); t holds everything else
  virtual int update_device(const msm::Tables &t, cudaStream_t stream) = 0;
  virtual int evaluate(const msm::EvalRequest &r, double *energy) = 0;
  virtual int adjoint(const msm::AdjointRequest &r) = 0;
  virtual long evaluations() const = 0;
  // the launch sequence of one device-pointer evaluation on s, nothing else
  // (no waits, no host work): for capture into a caller's graph
  virtual int enqueue_into(const msm::EvalRequest &r, cudaStream_t s) = 0;
  // the same launch sequence appended to rec instead of launched (merged
  // batches, launch.cuh)
  virtual int record_into(const msm::EvalRequest &r, msm::Recorder &rec) = 0;
  // an evaluation issued outside this plan (a batch replay) is about to run
  // on s: order it after a pending device rebuild and count it
  virtual int begin(cudaStream_t s) = 0;
  virtual long version() const = 0;  // bumped by every box update
  virtual int device_index() const = 0;
  virtual int sync() = 0;
  virtual int phase_times(double *ms, int n) = 0;
  virtual int launches() = 0;
  virtual int level_times(double *ms, int n) = 0;
};

namespace msm {

// The recorder of merged batch launches installed on this host thread, if any
Recorder *&tls_recorder() {
  static thread_local Recorder *r = nullptr;
  return r;
}

// Zeroes `words` 32-bit words at p (the recordable form of the evaluation's
// cudaMemsetAsync calls, so that a batch can merge them)
__device__ __forceinline__ void clear_words_body(const BlockCtx &ctx, int *p, long words) {
  for (long i = (long)ctx.b.x * blockDim.x + threadIdx.x; i < words;
       i += (long)ctx.g.x * blockDim.x)
    p[i] = 0;
}
struct KClearWords {
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) {
    clear_words_body(c, a...);
  }
};
__global__ void __launch_bounds__(256) k_clear_words(int *p, long words) {
  clear_words_body(hw_ctx(), p, words);
}

// cudaMemsetAsync(p, 0, bytes, s); while a batch records, a clear kernel
// (bytes are whole 32-bit words here)
cudaError_t zero_async(void *p, size_t bytes, cudaStream_t s) {
  if (!tls_recorder()) return cudaMemsetAsync(p, 0, bytes, s);
  const long words = (long)(bytes / 4);
  const int blocks = (int)std::max<long>(1, std::min<long>((words + 255) / 256, 1024));
  launch<KClearWords, 256, 8>(s, k_clear_words, blocks, 256, 0, static_cast<int *>(p), words);
  return cudaSuccess;
}

// Stamps for engine_version (see Plan::version_).
long next_version() {
  static std::atomic<long> counter{0};
  return ++counter;
}
namespace {

#define MSM_CUDA_TRY(expr)                       \
  do {                                           \
    cudaError_t e_ = (expr);                     \
    if (e_ != cudaSuccess) return MSMPB_ERR_CUDA; \
  } while (0)

// One cudaMalloc arena, carved into 256-byte aligned pieces.
struct Arena {
  char *base = nullptr;
  size_t size = 0, used = 0;
  std::vector<std::pair<void **, size_t>> plan;
  template <typename P>
  void want(P **p, size_t bytes) {
    plan.push_back({(void **)p, bytes});
  }
  int commit() {
    size_t total = 0;
    for (auto &e : plan) total += (e.second + 255) / 256 * 256;
    if (cudaMalloc(&base, std::max<size_t>(total, 256)) != cudaSuccess) {
      base = nullptr;
      return MSMPB_ERR_NOMEM;
    }
    size = total;
    for (auto &e : plan) {
      *e.first = base + used;
      used += (e.second + 255) / 256 * 256;
    }
    return MSMPB_OK;
  }
  ~Arena() {
    if (base) cudaFree(base);
  }
};

struct GraphKey {
  const void *pos, *q, *force, *phi, *energy;
  double w[kMaxLevels + 1];
  bool timing;
  bool operator==(const GraphKey &o) const {
    return std::memcmp(this, &o, sizeof(GraphKey)) == 0;
  }
};

template <typename T>
class Plan : public FFDevice {
 public:
  int init(const Tables &t, int device);
  ~Plan() override;
  int update(const Tables &t) override;
  int update_device(const Tables &t, cudaStream_t stream) override;
  int evaluate(const EvalRequest &r, double *energy) override;
  int adjoint(const AdjointRequest &r) override;
  long evaluations() const override { return nevals_; }
  int enqueue_into(const EvalRequest &r, cudaStream_t s) override {
    return enqueue(r, s, r.pos, r.q, r.force, r.phi, r.energy_dev ? r.energy_dev : energy_);
  }
  int record_into(const EvalRequest &r, Recorder &rec) override {
    MSM_CUDA_TRY(cudaSetDevice(device_));
    rec.aux = aux_[0];
    Recorder *prev = tls_recorder();
    tls_recorder() = &rec;
    EvalRequest rr = r;
    rr.timing = false;
    const int st =
        enqueue(rr, stream_, r.pos, r.q, r.force, r.phi, r.energy_dev ? r.energy_dev : energy_);
    tls_recorder() = prev;
    return st;
  }
  int begin(cudaStream_t s) override {
    MSM_CUDA_TRY(cudaSetDevice(device_));
    last_stream_ = s;
    if (rebuild_recorded_) MSM_CUDA_TRY(cudaStreamWaitEvent(s, rebuild_ev_, 0));
    ++nevals_;
    return MSMPB_OK;
  }
  long version() const override { return version_; }
  int device_index() const override { return device_; }
  int sync() override;
  int phase_times(double *ms, int n) override;
  int launches() override { return nlaunch_; }
  // stencil kernel time per level of the last timed evaluation
  int level_times(double *ms, int n) override {
    if (!timed_) return 0;
    cudaStreamSynchronize(stream_);
    int m = 0;
    for (int l = 1; l < L_ && m < n; ++l) {
      float t = 0;
      cudaEventElapsedTime(&t, lev_ev_[l][0], lev_ev_[l][1]);
      ms[m++] = t;
    }
    cudaGetLastError();
    return m;
  }

 private:
  int set_tables(const Tables &t);
  int update_box(const Tables &t, cudaStream_t s, bool stencils_on_device);
  int enqueue_chain(cudaStream_t s, T *const *qg, T *const *eg, const double *w, bool tm,
                    bool fork);
  int tune_levels(size_t pad_cap, size_t part_cap);
  int launch_graph(const EvalRequest &r, cudaStream_t s, const double *pos,
                   const double *q, double *force, double *phi, double *edev);
  PairClusterArgs<T> cluster_args() const;
  int enqueue(const EvalRequest &r, cudaStream_t s, const double *pos,
              const double *q, double *force, double *phi, double *energy);
  // Phase boundary: optional event, and with MSMPB_DEBUG_SYNC=1 (eager
  // launches only) a synchronising check that names the failing phase.
  void mark(cudaStream_t s, int phase, bool timing) {
    if (debug_sync_ && timing) {
      cudaError_t e = cudaStreamSynchronize(s);
      if (e == cudaSuccess) e = cudaGetLastError();
      if (e != cudaSuccess)
        std::fprintf(stderr, "msmpb_b200: CUDA error before phase %d: %s\n",
                     phase, cudaGetErrorString(e));
    }
    if (timing) cudaEventRecord(ev_[phase], s);
  }
  bool debug_sync_ = std::getenv("MSMPB_DEBUG_SYNC") != nullptr;
  // Pair sum: 2 = clusters (default); 1 = one thread per atom, the form for
  // geometries the cluster form does not take, which MSMPB_PAIR=thread
  // selects everywhere
  int pair_variant_ = [] {
    const char *v = std::getenv("MSMPB_PAIR");
    if (v && v[0] == 't') return 1;
    return 2;
  }();
  // Level stencils of symmetric kernels use the folded sweep unless
  // MSMPB_STENCIL=full
  bool fold_enabled_ = [] {
    const char *v = std::getenv("MSMPB_STENCIL");
    return !(v && v[0] == 'f');
  }();
  // Anterpolation: tile scatter (default); the slab-staged gather (the form
  // for grids smaller than the order), which MSMPB_ANTERP=gather selects
  // everywhere
  int anterp_variant_ = [] {
    const char *v = std::getenv("MSMPB_ANTERP");
    if (v && v[0] == 'g') return 2;
    return 0;
  }();

  int device_ = 0;
  cudaStream_t stream_ = nullptr;
  cudaStream_t last_stream_ = nullptr;
  int N_ = 0, L_ = 0, nu_ = 0;
  int grid_[kMaxLevels + 2][3] = {};
  StencilShape sh_[kMaxLevels + 2] = {};
  StencilTile tile_[kMaxLevels + 2] = {};
  bool tune_[kMaxLevels + 2] = {};
  Geometry geom_{};
  PairConsts<T> pc_{};
  SplineConsts<T> sc_{};
  double J_[11] = {};
  double coeff1_ = 0, coeff2_ = 0, gamma0_a0_ = 0;
  int ncp_ = 0, ncg_ = 0, noff_ = 0;
  int ncol_ = 0, maxcl_ = 0, ncoloff_ = 0, K2_ = 0, ozero_ = 0;
  bool ortho_ = false;
  bool clusters_ok_ = false;
  bool self_images_ = false;  // a lattice vector shorter than a0
  int kind_ = kKindMsm;       // kKindPme: one-level PME plan
  double cz_[3] = {};
  int nq_ = 0, ncomb_ = 0, ngrid_ = 0;
  std::vector<CellOffset<T>> offsets_;
  std::vector<ColumnOffset> coloffs_;
  Arena arena_;
  // device buffers
  double *pos_s_ = nullptr, *q_s_ = nullptr, *force_s_ = nullptr,
         *phi_s_ = nullptr;
  int *pcell_ = nullptr, *gcell_ = nullptr, *pcount_ = nullptr,
      *gcount_ = nullptr, *pstart_ = nullptr, *gstart_ = nullptr,
      *pcursor_ = nullptr, *gcursor_ = nullptr, *scan_tmp_ = nullptr;
  int *pperm_ = nullptr, *gperm_ = nullptr, *pinv_ = nullptr,
      *ginv_ = nullptr, *pcs_ = nullptr, *gcs_ = nullptr;
  V4<T> *prel_ = nullptr, *gfrac_ = nullptr, *psorted_ = nullptr,
        *gsorted_ = nullptr, *pout_ = nullptr, *gout_ = nullptr;
  // FP64 cell-relative positions for the close pairs of the mixed form
  V4<double> *prel64_ = nullptr, *psorted64_ = nullptr;
  static constexpr bool kMixed = sizeof(T) == 4;
  T *qg_[kMaxLevels + 2] = {}, *eg_[kMaxLevels + 2] = {};
  T *padded_ = nullptr, *part_ = nullptr, *kh_[kMaxLevels + 2] = {};
  // the levels below the finest in forked evaluations run beside the
  // level-1 stencil: their own padded copy and split partial sums
  T *padded2_ = nullptr, *part2_ = nullptr;
  // forked evaluations: the pair sum and the level-1 stencil on their own
  // streams (graph branches when captured), joined by events
  cudaStream_t aux_[2] = {};
  cudaEvent_t fork_ev_[4] = {};
  T *khf_[kMaxLevels + 2] = {};  // folded taps (symmetric stencils)
  // level stencil taps for the sweep variant in use
  const T *level_taps(int l) const { return sh_[l].sym ? khf_[l] : kh_[l]; }
  void plan_level(int l);
  T *anterp_scratch_ = nullptr;
  int *fold_tab_ = nullptr;
  double *khat_top_ = nullptr;
  double2 *fft_ = nullptr;
  double *qparts_ = nullptr, *short_parts_ = nullptr, *grid_parts_ = nullptr,
         *qstats_ = nullptr, *energy_ = nullptr;
  CellOffset<T> *off_d_ = nullptr;
  // clusters
  ColumnOffset *coloff_d_ = nullptr;
  int *clcount_ = nullptr, *clstart_ = nullptr;
  V4<T> *cpos_ = nullptr;
  V4<double> *cpos64_ = nullptr;
  ClusterInfo *cinfo_ = nullptr;
  UnitBox *cubox_ = nullptr;
  int2 *ulist_ = nullptr, *ulcnt_ = nullptr;  // unit lists (mixed form)
  int *err_d_ = nullptr;
  // graph
  cudaGraphExec_t exec_ = nullptr;
  GraphKey key_{};
  bool have_graph_ = false;
  bool graph_stale_ = false;  // kernel parameters changed (new box)
  long nevals_ = 0;           // forward evaluations so far
  // process-wide unique stamp of the current box tables: a new engine and
  // every box update take the next value, so a replaced engine never
  // matches a stamp recorded for its predecessor
  long version_ = next_version();
  // adjoint buffers (allocated on first use)
  void *adj_mem_ = nullptr;
  V4<T> *fbs_ = nullptr, *dip_ = nullptr, *adj_a_ = nullptr, *adj_b_ = nullptr,
        *adj_g_ = nullptr, *adj_h_ = nullptr, *fslot_ = nullptr;
  T *qg2_[kMaxLevels + 2] = {}, *eg2_[kMaxLevels + 2] = {};
  // recorded after a device-side rebuild; every later evaluation's stream
  // waits for it (the rebuild may run on another stream)
  cudaEvent_t rebuild_ev_ = nullptr;
  bool rebuild_recorded_ = false;
  // omega' rows (x, y, z of each level, stride oms_) and work space of the
  // device stencil computation
  double *om_d_ = nullptr, *stwork_ = nullptr;
  int oms_ = 1;
  cudaEvent_t ev_[kNumPhases + 1] = {};
  cudaEvent_t lev_ev_[kMaxLevels + 2][2] = {};
  bool timed_ = false;
  int nlaunch_ = 0;
};

template <typename T>
Plan<T>::~Plan() {
  if (stream_) cudaStreamSynchronize(stream_);
  if (exec_) cudaGraphExecDestroy(exec_);
  if (rebuild_ev_) cudaEventDestroy(rebuild_ev_);
  if (adj_mem_) cudaFree(adj_mem_);
  for (auto &e : ev_)
    if (e) cudaEventDestroy(e);
  for (auto &pr : lev_ev_)
    for (auto &e : pr)
      if (e) cudaEventDestroy(e);
  for (auto &e : fork_ev_)
    if (e) cudaEventDestroy(e);
  for (auto &a : aux_)
    if (a) {
      cudaStreamSynchronize(a);
      cudaStreamDestroy(a);
    }
  if (stream_) cudaStreamDestroy(stream_);
}

template <typename T>
int Plan<T>::init(const Tables &t, int device) {
  device_ = device;
  MSM_CUDA_TRY(cudaSetDevice(device));
  MSM_CUDA_TRY(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  for (auto &a : aux_) MSM_CUDA_TRY(cudaStreamCreateWithFlags(&a, cudaStreamNonBlocking));
  for (auto &e : fork_ev_) MSM_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  for (auto &e : ev_) MSM_CUDA_TRY(cudaEventCreate(&e));
  for (auto &pr : lev_ev_)
    for (auto &e : pr) MSM_CUDA_TRY(cudaEventCreate(&e));
  const Params &p = t.p;
  N_ = p.N;
  L_ = p.L;
  nu_ = p.nu;
  for (int l = 1; l <= L_; ++l)
    for (int k = 0; k < 3; ++k) grid_[l][k] = t.grid[l][k];
  // pair cells at least a0/2 thick: nc = floor(2 / (a0 |a*|))
  long ncell = 1;
  for (int k = 0; k < 3; ++k) {
    double w = p.a0 * std::sqrt(p.Ai[k][0] * p.Ai[k][0] + p.Ai[k][1] * p.Ai[k][1] +
                                p.Ai[k][2] * p.Ai[k][2]);
    int nc = (int)std::floor(2.0 / w);
    geom_.nc[k] = std::max(1, std::min(nc, 512));
    ncell *= geom_.nc[k];
    geom_.M1[k] = t.grid[1][k];
  }
  ncp_ = (int)ncell;
  ncol_ = geom_.nc[0] * geom_.nc[1];
  maxcl_ = cluster_capacity(N_, ncol_);
  ncg_ = grid_[1][0] * grid_[1][1] * grid_[1][2];
  if (!top_solve_supported(p.top)) return MSMPB_ERR_UNSUPPORTED;
  top_solve_prepare();
  anterpolate_prepare<T>();
  int err = set_tables(t);
  if (err) return err;
  // stencil shapes; scratch for both sweep variants (a rebuild with a new
  // box can make a stencil lose or gain its mirror symmetry)
  size_t pad_max = 1, part_max = 1, pad2_max = 1, part2_max = 1;
  for (int l = 1; l < L_; ++l) {
    StencilShape &s = sh_[l];
    for (int k = 0; k < 3; ++k) {
      s.M[k] = grid_[l][k];
      s.S[k] = t.sten[l][k];
    }
    const bool fp64 = sizeof(T) == 8;
    std::vector<double> kf;
    for (int v = 0; v < 2; ++v) {
      s.sym = v;
      if (v && (s.S[0] % 2 == 0 || s.S[1] % 2 == 0)) continue;
      plan_level(l);
      pad_max = std::max(pad_max, (size_t)s.P[0] * s.P[1] * s.P[2]);
      if (tile_[l].nsplit > 1)
        part_max = std::max(part_max, (size_t)tile_[l].nsplit * s.M[0] * s.M[1] * s.M[2]);
    }
    s.sym = fold_enabled_ && stencil_templated(s) &&
            stencil_fold_taps(t.khat[l].data(), s.S, fp64, kf);
    plan_level(l);
    // levels worth tuning: size the scratch for every candidate tile
    const double gflop = 2e-9 * s.M[0] * s.M[1] * s.M[2] * (double)s.S[0] * s.S[1] * s.S[2];
    tune_[l] = tile_[l].nz > 0 && gflop >= 1.0 && stencil_tuning_enabled();
    if (tune_[l])
      for (const StencilTile &c : stencil_candidates(s, fp64)) {
        int P[3];
        stencil_padded_dims(s, c, fp64, P);
        pad_max = std::max(pad_max, (size_t)P[0] * P[1] * P[2]);
        if (c.nsplit > 1)
          part_max = std::max(part_max, (size_t)c.nsplit * s.M[0] * s.M[1] * s.M[2]);
      }
  }
  // the same bounds over the levels below the finest only (their stencils
  // run beside the level-1 stencil in forked evaluations)
  for (int l = 2; l < L_; ++l) {
    const StencilShape &s = sh_[l];
    const bool fp64 = sizeof(T) == 8;
    std::vector<StencilTile> tiles{tile_[l]};
    StencilShape alt = s;
    for (int v = 0; v < 2; ++v) {  // both sweep variants' default tiles
      alt.sym = v;
      if (v && (s.S[0] % 2 == 0 || s.S[1] % 2 == 0)) continue;
      tiles.push_back(stencil_default_tile(alt, fp64));
    }
    if (tune_[l])
      for (const StencilTile &c : stencil_candidates(s, fp64)) tiles.push_back(c);
    for (const StencilTile &c : tiles) {
      int P[3];
      stencil_padded_dims(s, c, fp64, P);
      if (!stencil_templated(s) || c.nz <= 0)
        for (int k = 0; k < 3; ++k) P[k] = s.M[k] + s.S[k] - 1;
      pad2_max = std::max(pad2_max, (size_t)P[0] * P[1] * P[2]);
      if (c.nsplit > 1)
        part2_max = std::max(part2_max, (size_t)c.nsplit * s.M[0] * s.M[1] * s.M[2]);
    }
  }
  const size_t n = N_;
  nq_ = prep_blocks(N_);
  ncomb_ = combine_blocks(N_);
  ngrid_ = grid_dot_blocks((size_t)ncg_);
  Arena &a = arena_;
  a.want(&pos_s_, 3 * n * sizeof(double));
  a.want(&q_s_, n * sizeof(double));
  a.want(&force_s_, 3 * n * sizeof(double));
  a.want(&phi_s_, n * sizeof(double));
  for (int **b : {&pcell_, &gcell_, &pperm_, &gperm_, &pinv_, &ginv_, &pcs_, &gcs_})
    a.want(b, n * sizeof(int));
  // the four counters consecutive, cleared by one memset per evaluation
  a.want(&pcount_, (ncp_ + 1) * sizeof(int));
  a.want(&pcursor_, (ncp_ + 1) * sizeof(int));
  a.want(&gcount_, (ncg_ + 1) * sizeof(int));
  a.want(&gcursor_, (ncg_ + 1) * sizeof(int));
  a.want(&pstart_, (ncp_ + 1) * sizeof(int));
  a.want(&gstart_, (ncg_ + 1) * sizeof(int));
  a.want(&scan_tmp_, (scan_temp_ints(ncp_) + scan_temp_ints(ncg_)) * sizeof(int));
  for (V4<T> **b : {&prel_, &gfrac_, &psorted_, &gsorted_, &pout_, &gout_})
    a.want(b, n * sizeof(V4<T>));
  if (kMixed) {
    a.want(&prel64_, n * sizeof(V4<double>));
    a.want(&psorted64_, n * sizeof(V4<double>));
  }
  for (int l = 1; l <= L_; ++l) {
    size_t g = (size_t)grid_[l][0] * grid_[l][1] * grid_[l][2];
    a.want(&qg_[l], g * sizeof(T));
    a.want(&eg_[l], g * sizeof(T));
    if (l < L_) {
      a.want(&kh_[l], (size_t)sh_[l].S[0] * sh_[l].S[1] *
                          stencil_tap_pitch(sh_[l].S[2], !kMixed) * sizeof(T));
      a.want(&khf_[l], (size_t)(sh_[l].S[0] / 2 + 1) * (sh_[l].S[1] / 2 + 1) *
                           stencil_tap_pitch(sh_[l].S[2], !kMixed) * sizeof(T));
    }
  }
  a.want(&padded_, pad_max * sizeof(T));
  std::vector<int> fold_tab;
  if (anterp_tiles_supported(grid_[1], nu_)) {
    a.want(&anterp_scratch_, anterp_scratch_elems(grid_[1], nu_) * sizeof(T));
    fold_tab = anterp_fold_table(grid_[1], nu_);
    a.want(&fold_tab_, fold_tab.size() * sizeof(int));
  }
  a.want(&part_, part_max * sizeof(T));
  if (L_ > 2) {
    a.want(&padded2_, std::min(pad2_max, pad_max) * sizeof(T));
    a.want(&part2_, std::min(part2_max, part_max) * sizeof(T));
  }
  size_t ntop = (size_t)grid_[L_][0] * grid_[L_][1] * grid_[L_][2];
  a.want(&khat_top_, ntop * sizeof(double));
  a.want(&fft_, ntop * sizeof(double2));
  a.want(&qparts_, 2 * nq_ * sizeof(double));
  a.want(&short_parts_, ncomb_ * sizeof(double));
  a.want(&grid_parts_, ngrid_ * sizeof(double));
  a.want(&qstats_, 2 * sizeof(double));
  a.want(&energy_, sizeof(double));
  a.want(&off_d_, kMaxNeighbourOffsets * sizeof(CellOffset<T>));
  a.want(&coloff_d_, kMaxColumnOffsets * sizeof(ColumnOffset));
  oms_ = 1;
  size_t stn = 1;
  for (int l = 1; l < L_; ++l) {
    stn = std::max(stn, (size_t)sh_[l].S[0] * sh_[l].S[1] * sh_[l].S[2]);
    for (int k = 0; k < 3; ++k) oms_ = std::max(oms_, (int)t.omegap[l][k].size());
  }
  a.want(&om_d_, (size_t)(L_ + 1) * 3 * oms_ * sizeof(double));
  a.want(&stwork_, 3 * stn * sizeof(double));
  a.want(&clcount_, (ncol_ + 1) * sizeof(int));
  a.want(&clstart_, (ncol_ + 1) * sizeof(int));
  a.want(&cpos_, (size_t)maxcl_ * 8 * sizeof(V4<T>));
  if (kMixed) a.want(&cpos64_, (size_t)maxcl_ * 8 * sizeof(V4<double>));
  a.want(&cinfo_, (size_t)maxcl_ * sizeof(ClusterInfo));
  a.want(&cubox_, (size_t)maxcl_ * 2 * sizeof(UnitBox));

  a.want(&err_d_, sizeof(int));
  if ((err = a.commit())) return err;
  MSM_CUDA_TRY(cudaMemset(err_d_, 0, sizeof(int)));
  if (fold_tab_)
    MSM_CUDA_TRY(cudaMemcpy(fold_tab_, fold_tab.data(), fold_tab.size() * sizeof(int),
                            cudaMemcpyHostToDevice));
  {  // omega' rows depend on the grid sizes only
    std::vector<double> om((size_t)(L_ + 1) * 3 * oms_, 0.);
    for (int l = 1; l < L_; ++l)
      for (int k = 0; k < 3; ++k)
        std::copy(t.omegap[l][k].begin(), t.omegap[l][k].end(),
                  om.begin() + ((size_t)l * 3 + k) * oms_);
    MSM_CUDA_TRY(cudaMemcpy(om_d_, om.data(), om.size() * sizeof(double),
                            cudaMemcpyHostToDevice));
  }
  if ((err = update(t))) return err;
  return tune_levels(pad_max, part_max);
}

// Empirical tile choice for the levels with the most work (see tune.cu)
template <typename T>
int Plan<T>::tune_levels(size_t pad_cap, size_t part_cap) {
  MSM_CUDA_TRY(cudaMemsetAsync(padded_, 0, pad_cap * sizeof(T), stream_));
  const int khz_fp64 = !kMixed;
  for (int l = 1; l < L_; ++l) {
    if (!tune_[l]) continue;
    double ms = 0;
    StencilTile best = stencil_autotune<T>(
        stream_, device_, sh_[l], tile_[l], padded_, pad_cap, level_taps(l),
        stencil_tap_pitch(sh_[l].S[2], khz_fp64), eg_[l], part_, part_cap, &ms);
    if (stencil_prepare<T>(sh_[l], best) < 0) continue;
    tile_[l] = best;
    stencil_padded_dims(sh_[l], best, !kMixed, sh_[l].P);
  }
  MSM_CUDA_TRY(cudaStreamSynchronize(stream_));
  cudaGetLastError();
  return MSMPB_OK;
}

// Default tile, shared-memory attribute and padded dims of level l for the
// sweep variant sh_[l].sym
template <typename T>
void Plan<T>::plan_level(int l) {
  StencilShape &s = sh_[l];
  const bool fp64 = sizeof(T) == 8;
  tile_[l] = stencil_default_tile(s, fp64);
  if (!stencil_templated(s) || stencil_prepare<T>(s, tile_[l]) < 0) {
    tile_[l] = StencilTile();  // reference-form sweep
    s.sym = 0;
    s.P[0] = s.M[0] + s.S[0] - 1;
    s.P[1] = s.M[1] + s.S[1] - 1;
    s.P[2] = s.M[2] + s.S[2] - 1;
  } else {
    stencil_padded_dims(s, tile_[l], fp64, s.P);
  }
}

// Constants that depend only on the parameter set (not on the box)
template <typename T>
int Plan<T>::set_tables(const Tables &t) {
  const Params &p = t.p;
  kind_ = t.kind;
  pc_.nu = t.kind == kKindPme ? 0 : p.nu;  // 0 selects the erfc kernel
  sc_.nu = p.nu;
  const double c_exp = 2. * t.beta / std::sqrt(std::acos(-1.));
  pc_.beta = (T)t.beta;
  pc_.beta2 = (T)(t.beta * t.beta);
  pc_.c_exp = (T)c_exp;
  pc_.betad = t.beta;
  pc_.beta2d = t.beta * t.beta;
  pc_.c_expd = c_exp;
  pc_.a02 = (T)(p.a0 * p.a0);
  pc_.inv_a02 = (T)(1. / (p.a0 * p.a0));
  pc_.inv_a0 = (T)(1. / p.a0);
  pc_.two_inv_a03 = (T)(2. / (p.a0 * p.a0 * p.a0));
  for (int k = 0; k < 16; ++k) pc_.tau[k] = (T)t.tau[k];
  // pairs closer than 2.5 A (bonded and hydrogen-bonded distances) are
  // summed in FP64 in the mixed form
  pc_.close2 = kMixed ? (T)(2.5 * 2.5) : (T)0;
  pc_.a02d = p.a0 * p.a0;
  pc_.inv_a02d = 1. / (p.a0 * p.a0);
  pc_.inv_a0d = 1. / p.a0;
  pc_.two_inv_a03d = 2. / (p.a0 * p.a0 * p.a0);
  for (int k = 0; k < 16; ++k) pc_.taud[k] = t.tau[k];
  for (int k = 0; k < 50; ++k) sc_.Q[k] = (T)t.Q[k];
  for (int k = 0; k < 11; ++k) J_[k] = t.J[k];
  return MSMPB_OK;
}

// Box-dependent state: geometry, neighbour offsets, stencils, constants
template <typename T>
int Plan<T>::update(const Tables &t) {
  // the previous evaluation may still read the tables being replaced
  MSM_CUDA_TRY(cudaSetDevice(device_));
  MSM_CUDA_TRY(cudaStreamSynchronize(stream_));
  if (last_stream_ && last_stream_ != stream_)
    MSM_CUDA_TRY(cudaStreamSynchronize(last_stream_));
  const int st = update_box(t, stream_, false);
  MSM_CUDA_TRY(cudaStreamSynchronize(stream_));
  return st;
}

template <typename T>
int Plan<T>::update_device(const Tables &t, cudaStream_t stream) {
  if (t.kind != kKindMsm) return MSMPB_ERR_UNSUPPORTED;  // MSM level stencils only
  MSM_CUDA_TRY(cudaSetDevice(device_));
  if (!rebuild_ev_)
    MSM_CUDA_TRY(cudaEventCreateWithFlags(&rebuild_ev_, cudaEventDisableTiming));
  const int st = update_box(t, stream, true);
  if (st != MSMPB_OK) return st;
  MSM_CUDA_TRY(cudaEventRecord(rebuild_ev_, stream));
  rebuild_recorded_ = true;
  return MSMPB_OK;
}

// Box-dependent state: geometry, neighbour lists, constants, top multiplier
// and level stencils (from t, or computed on the device), uploaded in the
// order of s.
template <typename T>
int Plan<T>::update_box(const Tables &t, cudaStream_t s, bool stencils_on_device) {
  const Params &p = t.p;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      geom_.A[3 * r + c] = p.A[r][c];
      geom_.Ai[3 * r + c] = p.Ai[r][c];
    }
  coeff1_ = t.coeff1;
  coeff2_ = t.coeff2;
  gamma0_a0_ = t.gamma0 / p.a0;
  // an atom's own periodic images within a0 (the lattice vectors the
  // constant coeff1 sums, code/forcefield0.c:612-636)
  self_images_ = false;
  {
    int lim[3];
    for (int k = 0; k < 3; ++k)
      lim[k] = (int)std::ceil(p.a0 * std::sqrt(p.Ai[k][0] * p.Ai[k][0] + p.Ai[k][1] * p.Ai[k][1] +
                                               p.Ai[k][2] * p.Ai[k][2]) - 1.);
    for (int x = -lim[0]; x <= lim[0] && !self_images_; ++x)
      for (int y = -lim[1]; y <= lim[1] && !self_images_; ++y)
        for (int z = -lim[2]; z <= lim[2] && !self_images_; ++z) {
          if (x == 0 && y == 0 && z == 0) continue;
          double r2 = 0;
          for (int k = 0; k < 3; ++k) {
            const double rk = p.A[k][0] * x + p.A[k][1] * y + p.A[k][2] * z;
            r2 += rk * rk;
          }
          self_images_ = r2 < p.a0 * p.a0;
        }
  }
  // neighbour-cell instances: every offset d with |d_k| <= ceil(a0|a*_k| nc_k)
  bool ortho = true;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c)
      if (r != c && p.A[r][c] != 0.) ortho = false;
  int K[3];
  for (int k = 0; k < 3; ++k) {
    double w = p.a0 * std::sqrt(p.Ai[k][0] * p.Ai[k][0] + p.Ai[k][1] * p.Ai[k][1] +
                                p.Ai[k][2] * p.Ai[k][2]);
    K[k] = (int)std::ceil(w * geom_.nc[k]);
  }
  offsets_.clear();
  for (int dx = -K[0]; dx <= K[0]; ++dx)
    for (int dy = -K[1]; dy <= K[1]; ++dy)
      for (int dz = -K[2]; dz <= K[2]; ++dz) {
        int d[3] = {dx, dy, dz};
        if (ortho) {  // skip cells whose nearest point is beyond a0
          double m2 = 0;
          for (int k = 0; k < 3; ++k) {
            double gap = std::max(0, std::abs(d[k]) - 1) * std::fabs(p.A[k][k]) / geom_.nc[k];
            m2 += gap * gap;
          }
          if (m2 >= p.a0 * p.a0) continue;
        }
        CellOffset<T> o{};
        for (int k = 0; k < 3; ++k) o.d[k] = d[k];
        for (int r = 0; r < 3; ++r) {
          double v = 0;
          for (int c = 0; c < 3; ++c) v += p.A[r][c] * ((double)d[c] / geom_.nc[c]);
          o.shift[r] = (T)v;
          o.shift64[r] = v;
        }
        offsets_.push_back(o);
      }
  if ((int)offsets_.size() > kMaxNeighbourOffsets) return MSMPB_ERR_UNSUPPORTED;
  noff_ = (int)offsets_.size();
  // neighbour columns of the cluster form: (du, dv) with the same bounds
  // (and, for orthorhombic boxes, the same gap pruning in x and y); along
  // the column every cell within K2 of the cluster's cells is a candidate
  coloffs_.clear();
  for (int du = -K[0]; du <= K[0]; ++du)
    for (int dv = -K[1]; dv <= K[1]; ++dv) {
      if (ortho) {
        const double gx = std::max(0, std::abs(du) - 1) * std::fabs(p.A[0][0]) / geom_.nc[0];
        const double gy = std::max(0, std::abs(dv) - 1) * std::fabs(p.A[1][1]) / geom_.nc[1];
        if (gx * gx + gy * gy >= p.a0 * p.a0) continue;
      }
      ColumnOffset c{};
      c.du = du;
      c.dv = dv;
      if (du == 0 && dv == 0) ozero_ = (int)coloffs_.size();
      for (int r = 0; r < 3; ++r)
        c.base[r] = p.A[r][0] * ((double)du / geom_.nc[0]) +
                    p.A[r][1] * ((double)dv / geom_.nc[1]);
      coloffs_.push_back(c);
    }
  ncoloff_ = (int)coloffs_.size();
  ortho_ = ortho;
  K2_ = K[2];
  for (int r = 0; r < 3; ++r) cz_[r] = p.A[r][2] / geom_.nc[2];
  // the close-pair record packs the column index in 23 bits and the image
  // index along the column in 8
  clusters_ok_ = ncoloff_ <= kMaxColumnOffsets && K2_ / geom_.nc[2] + 2 < 120;
  if (clusters_ok_)
    MSM_CUDA_TRY(cudaMemcpyAsync(coloff_d_, coloffs_.data(), ncoloff_ * sizeof(ColumnOffset),
                                 cudaMemcpyHostToDevice, s));
  MSM_CUDA_TRY(cudaMemcpyAsync(off_d_, offsets_.data(), noff_ * sizeof(CellOffset<T>),
                               cudaMemcpyHostToDevice, s));
  if (stencils_on_device) {
    // mirror symmetry in x and y holds for every orthorhombic box
    for (int l = 1; l < L_; ++l) {
      const int sym = fold_enabled_ && ortho && stencil_templated(sh_[l]) &&
                      sh_[l].S[0] % 2 == 1 && sh_[l].S[1] % 2 == 1;
      if (sym != sh_[l].sym) {
        sh_[l].sym = sym;
        plan_level(l);
      }
      LevelStencilArgs la{};
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) la.A[3 * r + c] = p.A[r][c];
      for (int k = 0; k < 3; ++k) {
        la.as[k] = std::sqrt(p.Ai[0][k] * p.Ai[0][k] + p.Ai[1][k] * p.Ai[1][k] +
                             p.Ai[2][k] * p.Ai[2][k]);
        la.g[k] = grid_[l][k];
        la.sd[k] = sh_[l].S[k];
      }
      la.al = p.aCut[l];
      for (int k = 0; k < nu_ && k < 16; ++k) la.tau[k] = t.tau[k];
      la.nu = nu_;
      la.oms = oms_;
      launch_level_stencil<T>(s, la, om_d_ + (size_t)l * 3 * oms_, stwork_, kh_[l],
                              sh_[l].sym ? khf_[l] : nullptr, !kMixed);
    }
  }
  for (int l = 1; l < L_ && !stencils_on_device; ++l) {
    // rows of S2 taps padded to a 16-byte pitch (zeros), z fastest
    const int S0 = sh_[l].S[0], S1 = sh_[l].S[1], S2 = sh_[l].S[2];
    const int sp = stencil_tap_pitch(S2, !kMixed);
    std::vector<T> kh((size_t)S0 * S1 * sp, T(0));
    for (int i = 0; i < S0; ++i)
      for (int j = 0; j < S1; ++j)
        for (int k = 0; k < S2; ++k)
          kh[((size_t)i * S1 + j) * sp + k] = (T)t.khat[l][((size_t)i * S1 + j) * S2 + k];
    MSM_CUDA_TRY(cudaMemcpyAsync(kh_[l], kh.data(), kh.size() * sizeof(T),
                                 cudaMemcpyHostToDevice, s));
    MSM_CUDA_TRY(cudaStreamSynchronize(s));  // kh is a local
    // folded taps when the stencil is mirror-symmetric in x and y
    std::vector<double> kf;
    const int sym = fold_enabled_ && stencil_templated(sh_[l]) &&
                    stencil_fold_taps(t.khat[l].data(), sh_[l].S, !kMixed, kf);
    if (sym != sh_[l].sym) {
      sh_[l].sym = sym;
      plan_level(l);
    }
    if (sh_[l].sym) {
      std::vector<T> kft(kf.size());
      for (size_t n = 0; n < kf.size(); ++n) kft[n] = (T)kf[n];
      MSM_CUDA_TRY(cudaMemcpyAsync(khf_[l], kft.data(), kft.size() * sizeof(T),
                                   cudaMemcpyHostToDevice, s));
      MSM_CUDA_TRY(cudaStreamSynchronize(s));  // kft is a local
    }
  }
  MSM_CUDA_TRY(cudaMemcpyAsync(khat_top_, t.khat[L_].data(),
                               t.khat[L_].size() * sizeof(double),
                               cudaMemcpyHostToDevice, s));
  // geometry and constants are kernel parameters: the next graph launch
  // re-captures and updates the instantiated graph in place
  graph_stale_ = true;
  version_ = next_version();
  return MSMPB_OK;
}

// The grid operator K: q[1] -> e[1] (restriction, top solve, then from the
// coarsest level down, prolongation plus the level stencil). Returns the
// number of kernel launches.
//
// Forked form (fork = true, every evaluation except the eagerly timed one):
// the level-1 stencil depends on q[1] alone, so it runs on its own stream
// (a branch of the captured graph) and stores e[1] = w1 K1 q[1], while the
// restrictions, the top solve and the levels below run on s (with their own
// padded copy and partial sums); s then waits for it and adds the
// prolongation of e[2] into e[1]. The latency-bound small levels hide behind
// the level-1 stencil, and e[1] gets the same two terms (addition commutes).
template <typename T>
int Plan<T>::enqueue_chain(cudaStream_t s, T *const *qg, T *const *eg, const double *w,
                           bool tm, bool fork) {
  int nl = 0;
  fork = fork && L_ > 2 && padded2_ && part2_;
  // a batch recording keeps the forked order of operations (so results match
  // the replayed evaluation bit for bit) as one chain: no events
  const bool rec = tls_recorder() != nullptr;
  if (fork) {
    cudaStream_t b = rec ? s : aux_[1];
    if (!rec) {
      cudaEventRecord(fork_ev_[2], s);
      cudaStreamWaitEvent(b, fork_ev_[2], 0);
    }
    StencilShape st = sh_[1];
    st.store = 1;
    launch_pad<T>(b, st, qg[1], padded_);
    launch_stencil<T>(b, st, tile_[1], padded_, level_taps(1),
                      stencil_tap_pitch(st.S[2], !kMixed), (T)w[1], eg[1], part_);
    if (!rec) cudaEventRecord(fork_ev_[3], b);
    nl += 1 + stencil_launches(st, tile_[1]);
  }
  mark(s, kPhaseRestrict, tm);
  for (int l = 1; l < L_; ++l) {
    launch_restrict<T>(s, grid_[l], qg[l], qg[l + 1], J_, nu_);
    nl += 1;
  }
  mark(s, kPhaseTop, tm);
  launch_top_solve<T>(s, grid_[L_], qg[L_], khat_top_, w[L_], fft_, nullptr, eg[L_]);
  nl += top_solve_launches(grid_[L_]);
  for (int l = L_ - 1; l >= 1; --l) {
    if (fork && l == 1) {
      if (!rec) cudaStreamWaitEvent(s, fork_ev_[3], 0);
      launch_prolong_add<T>(s, grid_[1], eg[2], eg[1], J_, nu_);
      nl += 1;
      break;
    }
    T *pad = fork ? padded2_ : padded_;
    T *part = fork ? part2_ : part_;
    mark(s, kPhaseProlong, tm && l == L_ - 1);
    zero_async(eg[l], (size_t)grid_[l][0] * grid_[l][1] * grid_[l][2] * sizeof(T), s);
    launch_prolong_add<T>(s, grid_[l], eg[l + 1], eg[l], J_, nu_);
    mark(s, kPhaseStencil, tm && l == L_ - 1);
    launch_pad<T>(s, sh_[l], qg[l], pad);
    if (tm) cudaEventRecord(lev_ev_[l][0], s);
    launch_stencil<T>(s, sh_[l], tile_[l], pad, level_taps(l),
                      stencil_tap_pitch(sh_[l].S[2], !kMixed), (T)w[l], eg[l], part);
    if (tm) cudaEventRecord(lev_ev_[l][1], s);
    nl += 2 + stencil_launches(sh_[l], tile_[l]);
  }
  return nl;
}

// Arguments of the cluster pair kernels over this plan's buffers
template <typename T>
PairClusterArgs<T> Plan<T>::cluster_args() const {
  PairClusterArgs<T> ca{};
  ca.maxcl = maxcl_;
  ca.ncol = ncol_;
  ca.nc0 = geom_.nc[0];
  ca.nc1 = geom_.nc[1];
  ca.nc2 = geom_.nc[2];
  ca.K2 = K2_;
  ca.ncoloff = ncoloff_;
  const double rb = std::sqrt((double)pc_.a02) * (1.0 + 1e-4) + 1e-6;
  ca.rbox2 = (float)(rb * rb);
  const double rn = std::sqrt((double)pc_.close2) * (1.0 + 1e-4) + 1e-5;
  ca.rnear2 = (float)(rn * rn);
  ca.ortho = ortho_ ? 1 : 0;
  ca.ozero = ozero_;
  for (int k = 0; k < 3; ++k) ca.cw[k] = (float)(geom_.A[4 * k] / geom_.nc[k]);
  for (int r = 0; r < 3; ++r) ca.cz[r] = cz_[r];
  ca.start = pstart_;
  ca.clstart = clstart_;
  ca.coloff = coloff_d_;
  ca.info = cinfo_;
  ca.ubox = cubox_;
  ca.cpos = cpos_;
  ca.cpos64 = cpos64_;
  ca.out = pout_;
  ca.err = err_d_;
  ca.self_images = self_images_ ? 1 : 0;
  ca.list = ulist_;
  ca.lcnt = ulcnt_;
  ca.lcap = kUnitListCap;
  return ca;
}

template <typename T>
int Plan<T>::enqueue(const EvalRequest &r, cudaStream_t s, const double *pos,
                     const double *q, double *force, double *phi,
                     double *energy) {
  const bool tm = r.timing;
  int nl = 0;
  double w[kMaxLevels + 1];
  for (int l = 0; l <= L_; ++l) w[l] = r.weight ? r.weight[l] : 1.0;
  mark(s, kPhaseBin, tm);
  // the four cell counters are consecutive in the arena: one clear
  zero_async(pcount_,
             reinterpret_cast<char *>(gcursor_ + ncg_ + 1) - reinterpret_cast<char *>(pcount_),
             s);
  launch_prep<T>(s, N_, pos, q, geom_, pcell_, gcell_, pcount_, gcount_, prel_,
                 gfrac_, prel64_, err_d_, qparts_);
  launch_scan2(s, pcount_, pstart_, ncp_, gcount_, gstart_, ncg_, scan_tmp_);
  const bool clusters = pair_variant_ == 2 && clusters_ok_;
  launch_bin_scatter(s, N_, pcell_, pstart_, pcursor_, pperm_, gcell_, gstart_, gcursor_,
                     gperm_, clusters ? ncol_ : 0, geom_.nc[2], clcount_);
  launch_bin_sort<T>(s, ncp_, pstart_, pperm_, prel_, ncg_, gstart_, gperm_);
  launch_bin_gather<T>(s, N_, GatherSide<T>{pperm_, prel_, pcell_, psorted_, pcs_, pinv_},
                       kMixed ? prel64_ : nullptr, kMixed ? psorted64_ : nullptr,
                       GatherSide<T>{gperm_, gfrac_, gcell_, gsorted_, gcs_, ginv_});
  nl += 2 + scan2_launches(ncp_, ncg_) + 3;
  // Forked form (all but the eagerly timed evaluation): after binning the
  // short-range branch (cluster build and pair sum) runs on its own stream
  // beside the grid branch (anterpolation, grid operator, interpolation);
  // the combine waits for both. Captured, the two are branches of one graph.
  // While a batch records, the branch is a pair of markers around the
  // launches on aux_[0] instead of events.
  const bool fork = !tm;
  Recorder *rec = tls_recorder();
  cudaStream_t sp = s;
  if (fork) {
    if (rec) {
      rec->recs.emplace_back();
      rec->recs.back().kind = LaunchRec::kFork;
    } else {
      cudaEventRecord(fork_ev_[0], s);
      cudaStreamWaitEvent(aux_[0], fork_ev_[0], 0);
    }
    sp = aux_[0];
  }
  // the charge sums (one latency-bound CTA, read by the combine only) on the
  // short-range branch, off the serial binning path
  launch_qstats_final(sp, qparts_, nq_, qstats_);
  if (clusters) {  // cluster build (part of the binning phase)
    const V4<double> *src64 =
        kMixed ? psorted64_ : reinterpret_cast<const V4<double> *>(psorted_);
    launch_scan(sp, clcount_, clstart_, ncol_, scan_tmp_);
    launch_cluster_fill<T>(sp, maxcl_, ncol_, geom_.nc[2], pstart_, clstart_, pcs_,
                           src64, cz_, cpos_, cpos64_, cinfo_, cubox_);
  }
  mark(s, kPhasePair, tm);
  if (clusters) {
    const PairClusterArgs<T> ca = cluster_args();
    launch_pair_clusters<T>(sp, ca, pc_);
    nl += scan_launches(ncol_) + 1;
  } else {
    launch_pair<T>(sp, N_, psorted_, psorted64_, pcs_, pstart_, geom_, off_d_,
                   noff_, pc_, pout_);
  }
  nl += 1;
  if (fork && !rec) cudaEventRecord(fork_ev_[1], sp);
  mark(s, kPhaseAnterp, tm);
  launch_anterpolate<T>(s, grid_[1], gsorted_, gcs_, gstart_, sc_, qg_[1],
                        anterp_variant_, err_d_, N_, anterp_scratch_, fold_tab_);
  nl += (anterp_variant_ == 0 && anterp_scratch_) ? 2 : 1;
  nl += enqueue_chain(s, qg_, eg_, w, tm, fork);
  mark(s, kPhaseInterp, tm);
  launch_grid_dot<T>(s, (size_t)ncg_, qg_[1], eg_[1], grid_parts_, ngrid_);
  launch_interpolate<T>(s, N_, grid_[1], gsorted_, gcs_, eg_[1], sc_, geom_, gout_);
  nl += 2;
  if (fork) {
    if (rec) {
      rec->recs.emplace_back();
      rec->recs.back().kind = LaunchRec::kJoin;
    } else {
      cudaStreamWaitEvent(s, fork_ev_[1], 0);
    }
  }
  mark(s, kPhaseCombine, tm);
  CombineArgs ca;
  ca.N = N_;
  ca.w0 = w[0];
  ca.coeff1 = coeff1_;
  ca.coeff2 = coeff2_;
  ca.gamma0_over_a0 = gamma0_a0_;
  ca.q = q;
  ca.qstats = qstats_;
  ca.nqparts = nq_;
  ca.qparts = qparts_;
  ca.force = force;
  ca.phi = phi;
  ca.epart = short_parts_;
  launch_combine<T>(s, ca, pinv_, ginv_, pout_, gout_, ncomb_);
  EnergyArgs ea;
  ea.qparts = qparts_;
  ea.nqparts = nq_;
  ea.short_parts = short_parts_;
  ea.nshort = ncomb_;
  ea.grid_parts = grid_parts_;
  ea.ngrid = ngrid_;
  ea.w0 = w[0];
  ea.coeff1 = coeff1_;
  ea.coeff2 = coeff2_;
  ea.gamma0_over_a0 = gamma0_a0_;
  ea.energy = energy ? energy : energy_;
  ea.qstats = qstats_;
  // PME weighs the grid charges before the solve and dots the weighted
  // charges with the result: its grid energy carries w_1^2
  // (code/pme1.c:86-101); MSM's carries w_L once
  ea.grid_scale = kind_ == kKindPme ? w[1] : 1.0;
  launch_energy_total(s, ea);
  nl += 2;
  mark(s, kNumPhases, tm);
  nlaunch_ = nl;
  cudaError_t ce = cudaGetLastError();
  if (ce != cudaSuccess) {
    std::fprintf(stderr, "msmpb_b200: launch error: %s\n", cudaGetErrorString(ce));
    return MSMPB_ERR_CUDA;
  }
  return MSMPB_OK;
}

template <typename T>
int Plan<T>::evaluate(const EvalRequest &r, double *energy) {
  MSM_CUDA_TRY(cudaSetDevice(device_));
  // Host calls run on the library's stream; device calls are ordered on the
  // caller's stream (0 = the legacy default stream).
  cudaStream_t s = r.host ? stream_ : r.stream;
  last_stream_ = s;
  if (rebuild_recorded_) MSM_CUDA_TRY(cudaStreamWaitEvent(s, rebuild_ev_, 0));
  ++nevals_;
  const double *pos = r.pos, *q = r.q;
  double *force = r.force, *phi = r.phi;
  if (r.host) {
    MSM_CUDA_TRY(cudaMemcpyAsync(pos_s_, r.pos, 3 * (size_t)N_ * sizeof(double),
                                 cudaMemcpyHostToDevice, s));
    MSM_CUDA_TRY(cudaMemcpyAsync(q_s_, r.q, (size_t)N_ * sizeof(double),
                                 cudaMemcpyHostToDevice, s));
    pos = pos_s_;
    q = q_s_;
    force = r.force ? force_s_ : nullptr;
    phi = r.phi ? phi_s_ : nullptr;
  }
  double *edev = r.host ? energy_ : (r.energy_dev ? r.energy_dev : energy_);
  cudaGetLastError();  // never inherit an earlier, unrelated error
  if (r.timing) {
    // Per-phase timing uses events between eager launches (events recorded
    // by graph nodes cannot be timed); untimed calls replay the graph.
    int st = enqueue(r, s, pos, q, force, phi, edev);
    if (st != MSMPB_OK) return st;
  } else {
    int st = launch_graph(r, s, pos, q, force, phi, edev);
    if (st != MSMPB_OK) return st;
  }
  timed_ = r.timing;
  if (r.host) {
    if (r.force)
      MSM_CUDA_TRY(cudaMemcpyAsync(r.force, force_s_, 3 * (size_t)N_ * sizeof(double),
                                   cudaMemcpyDeviceToHost, s));
    if (r.phi)
      MSM_CUDA_TRY(cudaMemcpyAsync(r.phi, phi_s_, (size_t)N_ * sizeof(double),
                                   cudaMemcpyDeviceToHost, s));
    double e = 0, qs[2] = {0, 0};
    MSM_CUDA_TRY(cudaMemcpyAsync(&e, energy_, sizeof(double),
                                 cudaMemcpyDeviceToHost, s));
    if (r.q2)
      MSM_CUDA_TRY(cudaMemcpyAsync(qs, qstats_, 2 * sizeof(double),
                                   cudaMemcpyDeviceToHost, s));
    int st = sync();
    if (energy) *energy = e;
    if (r.q2) *r.q2 = qs[1];
    return st;
  }
  return MSMPB_OK;
}

template <typename T>
int Plan<T>::adjoint(const AdjointRequest &r) {
  MSM_CUDA_TRY(cudaSetDevice(device_));
  // the adjoint's pair Hessian is written for the MSM kernel
  if (kind_ != kKindMsm || !anterp_scratch_ || !fold_tab_) return MSMPB_ERR_UNSUPPORTED;
  if (!r.pos || !r.q || !r.fbar) return MSMPB_ERR_ARGUMENT;
  if (!adj_mem_) {
    // six per-atom records and a second set of level grids
    // (+ the cluster pass's Fbar in slot order and unit lists, mixed form)
    const bool lists = kMixed && clusters_ok_;
    size_t bytes = 6 * (size_t)N_ * sizeof(V4<T>) + 256 * 9 + 8 * (size_t)maxcl_ * sizeof(V4<T>);
    if (lists)
      bytes += (size_t)maxcl_ * (kUnitListCap + 1) * sizeof(int2);
    for (int l = 1; l <= L_; ++l)
      bytes += 2 * ((size_t)grid_[l][0] * grid_[l][1] * grid_[l][2] * sizeof(T) + 256);
    if (cudaMalloc(&adj_mem_, bytes) != cudaSuccess) {
      adj_mem_ = nullptr;
      cudaGetLastError();
      return MSMPB_ERR_NOMEM;
    }
    char *p = static_cast<char *>(adj_mem_);
    auto take = [&](size_t b) {
      char *q = p;
      p += (b + 255) / 256 * 256;
      return q;
    };
    for (V4<T> **b : {&fbs_, &dip_, &adj_a_, &adj_b_, &adj_g_, &adj_h_})
      *b = reinterpret_cast<V4<T> *>(take((size_t)N_ * sizeof(V4<T>)));
    fslot_ = reinterpret_cast<V4<T> *>(take(8 * (size_t)maxcl_ * sizeof(V4<T>)));
    if (lists) {
      ulist_ = reinterpret_cast<int2 *>(take((size_t)maxcl_ * kUnitListCap * sizeof(int2)));
      ulcnt_ = reinterpret_cast<int2 *>(take((size_t)maxcl_ * sizeof(int2)));
    }
    for (int l = 1; l <= L_; ++l) {
      const size_t g = (size_t)grid_[l][0] * grid_[l][1] * grid_[l][2] * sizeof(T);
      qg2_[l] = reinterpret_cast<T *>(take(g));
      eg2_[l] = reinterpret_cast<T *>(take(g));
    }
  }
  cudaStream_t s = r.stream;
  last_stream_ = s;
  if (rebuild_recorded_) MSM_CUDA_TRY(cudaStreamWaitEvent(s, rebuild_ev_, 0));
  double w[kMaxLevels + 1];
  for (int l = 0; l <= L_; ++l) w[l] = r.weight ? r.weight[l] : 1.0;
  cudaGetLastError();
  if (!r.reuse) {  // the forward state this adjoint linearises about
    EvalRequest fr{};
    fr.pos = r.pos;
    fr.q = r.q;
    fr.weight = r.weight;
    const int st = enqueue(fr, s, r.pos, r.q, nullptr, nullptr, energy_);
    if (st != MSMPB_OK) return st;
    ++nevals_;
  }
  launch_adj_gather<T>(s, N_, pperm_, r.fbar, fbs_);
  // the forward just run (or reused) built the clusters of these positions
  if (pair_variant_ == 2 && clusters_ok_ && adj_pair_clusters_supported<T>()) {
    const PairClusterArgs<T> ca = cluster_args();
    if (ca.list) launch_pair_list<T>(s, ca);  // the unit lists of these positions
    launch_adj_pair_clusters<T>(s, ca, pc_, fbs_, fslot_, adj_a_, adj_b_);
  }
  else
    launch_adj_pair<T>(s, N_, psorted_, fbs_, pcs_, pstart_, geom_, off_d_, noff_, pc_,
                       adj_a_, adj_b_);
  launch_adj_dipoles<T>(s, N_, gperm_, r.q, r.fbar, geom_, dip_);
  launch_adj_anterpolate<T>(s, grid_[1], gsorted_, gcs_, gstart_, sc_, dip_, qg2_[1],
                            anterp_scratch_, fold_tab_);
  enqueue_chain(s, qg2_, eg2_, w, false, true);
  launch_adj_interpolate<T>(s, N_, grid_[1], gsorted_, gcs_, gperm_, r.fbar, eg2_[1],
                            eg_[1], sc_, geom_, adj_g_, adj_h_);
  AdjointCombineArgs ca{};
  ca.N = N_;
  ca.w0 = w[0];
  ca.coeff1 = coeff1_;
  ca.coeff2 = coeff2_;
  ca.gamma0_over_a0 = gamma0_a0_;
  ca.q = r.q;
  ca.qstats = qstats_;
  ca.fbar = r.fbar;
  ca.ubar = r.ubar;
  ca.dq = r.dq;
  ca.dr = r.dr;
  launch_adj_combine<T>(s, ca, pinv_, ginv_, pout_, gout_, adj_a_, adj_b_, adj_g_, adj_h_);
  const cudaError_t ce = cudaGetLastError();
  if (ce != cudaSuccess) {
    std::fprintf(stderr, "msmpb_b200: adjoint launch error: %s\n", cudaGetErrorString(ce));
    return MSMPB_ERR_CUDA;
  }
  return MSMPB_OK;
}

template <typename T>
int Plan<T>::launch_graph(const EvalRequest &r, cudaStream_t s,
                          const double *pos, const double *q, double *force,
                          double *phi, double *edev) {
  GraphKey key{};
  key.pos = pos;
  key.q = q;
  key.force = force;
  key.phi = phi;
  key.energy = edev;
  for (int l = 0; l <= L_; ++l) key.w[l] = r.weight ? r.weight[l] : 1.0;
  key.timing = false;
  if (!have_graph_ || !(key == key_) || graph_stale_) {
    // same buffers, new parameters: update the instantiated graph in place
    const bool refresh = have_graph_ && exec_ && key == key_;
    if (exec_ && !refresh) {
      cudaGraphExecDestroy(exec_);
      exec_ = nullptr;
    }
    have_graph_ = false;
    cudaGraph_t g = nullptr;
    // capture on the private stream (the legacy default stream cannot be
    // captured); the graph is then launched on the caller's stream
    MSM_CUDA_TRY(cudaStreamSynchronize(stream_));
    MSM_CUDA_TRY(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    EvalRequest untimed = r;
    untimed.timing = false;
    int st = enqueue(untimed, stream_, pos, q, force, phi, edev);
    cudaError_t ce = cudaStreamEndCapture(stream_, &g);
    if (st != MSMPB_OK || ce != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      return st != MSMPB_OK ? st : MSMPB_ERR_CUDA;
    }
    cudaError_t ie = cudaErrorUnknown;
    if (refresh) {
      cudaGraphExecUpdateResultInfo info{};
      ie = cudaGraphExecUpdate(exec_, g, &info);
      if (ie != cudaSuccess) {  // the launch sequence changed shape
        cudaGetLastError();
        cudaGraphExecDestroy(exec_);
        exec_ = nullptr;
      }
    }
    if (!exec_) ie = cudaGraphInstantiate(&exec_, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
      exec_ = nullptr;
      return MSMPB_ERR_CUDA;
    }
    key_ = key;
    have_graph_ = true;
    graph_stale_ = false;
  }
  MSM_CUDA_TRY(cudaGraphLaunch(exec_, s));
  return MSMPB_OK;
}

template <typename T>
int Plan<T>::sync() {
  MSM_CUDA_TRY(cudaSetDevice(device_));
  MSM_CUDA_TRY(cudaStreamSynchronize(stream_));
  if (last_stream_ != stream_) MSM_CUDA_TRY(cudaStreamSynchronize(last_stream_));
  int flag = 0;
  MSM_CUDA_TRY(cudaMemcpy(&flag, err_d_, sizeof(int), cudaMemcpyDeviceToHost));
  if (flag) {
    cudaMemset(err_d_, 0, sizeof(int));
    return MSMPB_ERR_DEVICE_CHECK;
  }
  return MSMPB_OK;
}

template <typename T>
int Plan<T>::phase_times(double *ms, int n) {
  if (!timed_) return 0;
  cudaStreamSynchronize(stream_);
  int order[kNumPhases + 1];
  for (int k = 0; k <= kNumPhases; ++k) order[k] = k;
  // phases were recorded in pipeline order: bin, pair, anterp, restrict,
  // top, prolong, stencil, interp, combine, end
  int seq[] = {kPhaseBin, kPhasePair, kPhaseAnterp, kPhaseRestrict, kPhaseTop,
               kPhaseProlong, kPhaseStencil, kPhaseInterp, kPhaseCombine,
               kNumPhases};
  double out[kNumPhases + 1] = {};
  const int nseq = sizeof(seq) / sizeof(int);
  for (int i = 0; i + 1 < nseq; ++i) {
    int a = seq[i];
    int b = seq[i + 1];
    if (L_ == 1 && (a == kPhaseProlong || a == kPhaseStencil)) continue;
    if (L_ == 1 && a == kPhaseTop) b = kPhaseInterp;
    float t = 0;
    if (cudaEventElapsedTime(&t, ev_[a], ev_[b]) == cudaSuccess) out[a] = t;
  }
  // prolongation and stencils interleave over levels: the span from the
  // first prolongation to the interpolation is attributed to the stencil
  // phase except for the first level's prolongation
  float tot = 0;
  cudaEventElapsedTime(&tot, ev_[kPhaseBin], ev_[kNumPhases]);
  out[kNumPhases] = tot;
  (void)order;
  cudaGetLastError();
  int m = std::min(n, kNumPhases + 1);
  for (int k = 0; k < m; ++k) ms[k] = out[k];
  return m;
}

}  // namespace

FFDevice *engine_create(const Tables &t, int precision, int device, int *err) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    *err = MSMPB_ERR_NODEVICE;
    return nullptr;
  }
  if (device < 0 || device >= ndev) {
    *err = MSMPB_ERR_ARGUMENT;
    return nullptr;
  }
  FFDevice *d = nullptr;
  int st;
  if (precision == MSMPB_PRECISION_FP64) {
    auto *p = new Plan<double>();
    st = p->init(t, device);
    d = p;
  } else {
    auto *p = new Plan<float>();
    st = p->init(t, device);
    d = p;
  }
  if (st != MSMPB_OK) {
    delete d;
    *err = st;
    return nullptr;
  }
  *err = MSMPB_OK;
  return d;
}

void engine_destroy(FFDevice *d) { delete d; }

int engine_update_tables(FFDevice *d, const Tables &t) { return d->update(t); }
int engine_adjoint(FFDevice *d, const AdjointRequest &r) { return d->adjoint(r); }
int engine_enqueue(FFDevice *d, const EvalRequest &r, cudaStream_t s) {
  return d->enqueue_into(r, s);
}
int engine_record(FFDevice *d, const EvalRequest &r, Recorder &rec) {
  return d->record_into(r, rec);
}
int engine_begin(FFDevice *d, cudaStream_t s) { return d->begin(s); }
long engine_version(FFDevice *d) { return d->version(); }
int engine_device(FFDevice *d) { return d->device_index(); }
long engine_evaluations(FFDevice *d) { return d->evaluations(); }
int engine_update_tables_device(FFDevice *d, const Tables &t, cudaStream_t stream) {
  return d->update_device(t, stream);
}

int engine_evaluate(FFDevice *d, const EvalRequest &r, double *energy) {
  return d->evaluate(r, energy);
}

int engine_sync(FFDevice *d) { return d->sync(); }

int engine_phase_times(FFDevice *d, double *ms, int n) {
  return d->phase_times(ms, n);
}

int engine_kernel_launches(FFDevice *d) { return d->launches(); }

}  // namespace msm

namespace msm {
int engine_level_times(FFDevice *d, double *ms, int n) {
  return d->level_times(ms, n);
}
}  // namespace msm
