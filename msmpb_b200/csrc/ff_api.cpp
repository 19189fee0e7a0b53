// C ABI of the drop-in library: every function of the reference's
// code/forcefield.h:70-112 with its exact signature, plus the extensions of
// msmpb_b200.h. Host-side parameter selection and tables run here (FP64);
// every evaluation runs on the GPU through the engine. There is no CPU
// evaluation path: without a usable device FF_energy returns NaN and records
// MSMPB_ERR_NODEVICE.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <new>

#include "engine.h"
#include "msm_host.h"
#include "msmpb_b200.h"

namespace {

struct HostState {
  msm::Params params;
  msm::Tables tables;
  bool built = false;
};

HostState *host(FF *ff) { return static_cast<HostState *>(ff->host_state); }

void set_error(FF *ff, int code) {
  if (ff && code != MSMPB_OK) ff->last_error = code;
}

// FF_last_error reports the outcome of the latest working call: each of
// them (build, rebuild, evaluation, adjoint, sync) clears it first
void begin_call(FF *ff) {
  if (ff) ff->last_error = MSMPB_OK;
}

bool timing_enabled() {
  static int cached = -1;
  if (cached < 0) {
    const char *v = std::getenv("MSMPB_TIMING");
    cached = (v && v[0] == '0') ? 0 : 1;
  }
  return cached == 1;
}

void free_tables(FF *ff) {
  std::free(ff->aCut);
  std::free(ff->tau);
  std::free(ff->Q);
  std::free(ff->J);
  if (ff->khat) {
    for (int l = 1; l <= ff->maxLevel && l <= msm::kMaxLevels; ++l) std::free(ff->khat[l]);
    std::free(ff->khat);
  }
  if (ff->omegap) {
    for (int l = 1; l <= ff->maxLevel && l <= msm::kMaxLevels; ++l)
      for (int a = 0; a < 3; ++a) std::free(ff->omegap[l][a]);
    std::free(ff->omegap);
  }
  for (int a = 0; a < 3; ++a) {
    std::free(ff->cL[a]);
    ff->cL[a] = nullptr;
  }
  ff->aCut = ff->tau = ff->Q = ff->J = nullptr;
  ff->khat = nullptr;
  ff->omegap = nullptr;
}

double *copy_array(const double *src, size_t n) {
  double *d = static_cast<double *>(std::malloc(sizeof(double) * (n ? n : 1)));
  if (d && n) std::memcpy(d, src, sizeof(double) * n);
  return d;
}

// Mirror the host tables into the reference's FF members
void export_tables(FF *ff, const msm::Tables &t) {
  free_tables(ff);
  const msm::Params &p = t.p;
  const int L = p.L;
  ff->aCut = copy_array(p.aCut, L + 1);
  ff->tau = copy_array(t.tau, p.nu);
  ff->Q = copy_array(t.Q, (p.nu / 2) * p.nu);
  ff->J = copy_array(t.J, p.nu + 1);
  ff->khat = static_cast<double **>(std::calloc(L + 1, sizeof(double *)));
  ff->omegap = static_cast<double *(*)[3]>(std::calloc(L + 1, sizeof(double *[3])));
  for (int l = 1; l <= L; ++l) {
    ff->khat[l] = copy_array(t.khat[l].data(), t.khat[l].size());
    for (int a = 0; a < 3; ++a)
      ff->omegap[l][a] = copy_array(t.omegap[l][a].data(), t.omegap[l][a].size());
  }
  for (int a = 0; a < 3; ++a) ff->cL[a] = copy_array(t.cL[a].data(), t.cL[a].size());
  ff->coeff1 = t.coeff1;
  ff->coeff2 = t.coeff2;
}

void export_params(FF *ff, const msm::Params &p) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      ff->A[i][j] = p.A[i][j];
      ff->Ai[i][j] = p.Ai[i][j];
    }
  ff->detA = p.detA;
  ff->estErr = p.estErr;
  ff->maxLevel = p.L;
  for (int k = 0; k < 3; ++k) ff->topGridDim[k] = p.top[k];
  ff->cutoff = p.a0;
  ff->orderAcc = p.nu;
  ff->relCutoff = p.relCutoff;
  ff->nLim = p.nLim;
}

void make_device(FF *ff) {
  HostState *h = host(ff);
  if (ff->dev) {
    msm::engine_destroy(ff->dev);
    ff->dev = nullptr;
  }
  int err = MSMPB_OK;
  ff->dev = msm::engine_create(h->tables, ff->precision, ff->device, &err);
  if (!ff->dev) {
    set_error(ff, err);
    if (err == MSMPB_ERR_NODEVICE)
      std::fprintf(stderr, "msmpb_b200: no usable CUDA device; FF_energy will "
                           "return NaN\n");
  }
}

double seconds_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

void fill_times(FF *ff) {
  double ms[msm::kNumPhases + 1] = {};
  int n = msm::engine_phase_times(ff->dev, ms, msm::kNumPhases + 1);
  if (n <= 0) return;
  const int L = ff->maxLevel;
  ff->time_nlist = ms[msm::kPhaseBin] * 1e-3;
  ff->time_partcl2partcl = ms[msm::kPhasePair] * 1e-3;
  ff->time_anterpolation = ms[msm::kPhaseAnterp] * 1e-3;
  ff->time_interpolation = (ms[msm::kPhaseInterp] + ms[msm::kPhaseCombine]) * 1e-3;
  for (int l = 0; l < 10; ++l)
    ff->time_grid2grid[l] = ff->time_restriction[l] = ff->time_prolongation[l] =
        ff->time_padding[l] = 0.;
  if (L >= 1 && L < 10) ff->time_grid2grid[L] = ms[msm::kPhaseTop] * 1e-3;
  if (L > 1) {
    ff->time_grid2grid[1] = ms[msm::kPhaseStencil] * 1e-3;
    ff->time_restriction[2] = ms[msm::kPhaseRestrict] * 1e-3;
    ff->time_prolongation[1] = ms[msm::kPhaseProlong] * 1e-3;
  }
}

}  // namespace

extern "C" {

FF *FF_new(int N, double *q) {
  FF *ff = static_cast<FF *>(std::calloc(1, sizeof(FF)));
  if (!ff) return nullptr;
  ff->FFT = true;
  ff->N = N;
  ff->q = q;
  ff->maxLevel = -1;
  ff->orderAcc = -1;
  ff->topGridDim[0] = ff->topGridDim[1] = ff->topGridDim[2] = -1;
  ff->cutoff = -1;
  ff->estErr = -1;
  ff->precision = MSMPB_PRECISION_MIXED;
  const char *pv = std::getenv("MSMPB_PRECISION");
  if (pv && (std::strcmp(pv, "fp64") == 0 || std::strcmp(pv, "FP64") == 0))
    ff->precision = MSMPB_PRECISION_FP64;
  ff->device = 0;
  ff->timing = timing_enabled() ? 1 : 0;
  ff->host_state = new (std::nothrow) HostState();
  if (N <= 0 || !q) ff->last_error = MSMPB_ERR_ARGUMENT;
  return ff;
}

void FF_set_orderAcc(FF *ff, int orderAcc) { ff->orderAcc = orderAcc; }
void FF_set_maxLevel(FF *ff, int maxLevel) { ff->maxLevel = maxLevel; }
void FF_set_topGridDim(FF *ff, int topGridDim[3]) {
  for (int k = 0; k < 3; ++k) ff->topGridDim[k] = topGridDim[k];
}
void FF_set_estErr(FF *ff, double estErr) { ff->estErr = estErr; }
double FF_get_estErr(FF *ff) { return ff->estErr; }
void FF_set_cutoff(FF *ff, double cutoff) { ff->cutoff = cutoff; }
double FF_get_cutoff(FF *ff) { return ff->cutoff; }
// Unlike the reference's -DNO_FFT build (code/forcefield0.c:209-215) this
// never exits: FFT = false only changes the automatic parameter choice
// (code/forcefield0.c:251-307); the top level is always solved by FFT.
void FF_set_FFT(FF *ff, bool FFT) { ff->FFT = FFT; }
int FF_get_orderAcc(FF *ff) { return ff->orderAcc; }
int FF_get_maxLevel(FF *ff) { return ff->maxLevel; }
void FF_get_topGridDim(FF *ff, int topGridDim[3]) {
  for (int k = 0; k < 3; ++k) topGridDim[k] = ff->topGridDim[k];
}
bool FF_get_FFT(FF *ff) { return ff->FFT; }

void FF_build(FF *ff, int N, double (*position)[3], double edges[3][3],
              double margin) {
  begin_call(ff);
  (void)position;
  HostState *h = host(ff);
  if (!h || ff->N <= 0 || !ff->q || !edges || N != ff->N) {
    set_error(ff, MSMPB_ERR_ARGUMENT);
    return;
  }
  ff->ntc = 7;
  ff->tmax = 4;
  ff->margin = margin;
  int err = MSMPB_OK;
  if (!msm::select_params(h->params, ff->N, ff->q, edges, ff->cutoff,
                          ff->orderAcc, ff->maxLevel, ff->topGridDim,
                          ff->estErr, ff->FFT, &err)) {
    set_error(ff, err);
    return;
  }
  export_params(ff, h->params);
  auto t0 = std::chrono::steady_clock::now();
  msm::build_tables(h->tables, h->params);
  double ts = seconds_since(t0);
  for (int l = 0; l < 10; ++l) ff->time_stencil[l] = 0.;
  if (ff->maxLevel < 10) ff->time_stencil[1] = ts;
  export_tables(ff, h->tables);
  h->built = true;
  ff->nlist = nullptr;
  ff->nlist_len = 0;
  ff->nlist_interaction_count = 0;
  make_device(ff);
}

void FF_rebuild(FF *ff, double edges[3][3], double (*position)[3],
                double margin) {
  begin_call(ff);
  (void)position;
  HostState *h = host(ff);
  if (!h || !h->built) {
    set_error(ff, MSMPB_ERR_STATE);
    return;
  }
  ff->margin = margin;
  // new box, same grid sizes, order, cutoff and nLim
  // (code/forcefield0.c:598-680 keeps every FF_build choice)
  msm::Params &p = h->params;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) p.A[i][j] = edges[i][j];
  p.detA = msm::invert3(p.A, p.Ai);
  if (!(p.detA > 0)) {
    set_error(ff, MSMPB_ERR_ARGUMENT);
    return;
  }
  export_params(ff, p);
  msm::build_tables(h->tables, p);
  export_tables(ff, h->tables);
  if (ff->dev) {
    int st = msm::engine_update_tables(ff->dev, h->tables);
    if (st != MSMPB_OK) set_error(ff, st);
  } else {
    make_device(ff);
  }
}

int FF_rebuild_device(FF *ff, double edges[3][3], void *stream) {
  begin_call(ff);
  HostState *h = host(ff);
  if (!h || !h->built) return ff->last_error = MSMPB_ERR_STATE;
  if (!ff->dev) return ff->last_error = MSMPB_ERR_NODEVICE;
  msm::Params p = h->params;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) p.A[i][j] = edges[i][j];
  p.detA = msm::invert3(p.A, p.Ai);
  if (!(p.detA > 0)) return ff->last_error = MSMPB_ERR_ARGUMENT;
  h->params = p;
  export_params(ff, p);
  msm::rebuild_box_tables(h->tables, p);
  export_tables(ff, h->tables);
  int st = msm::engine_update_tables_device(ff->dev, h->tables,
                                            static_cast<cudaStream_t>(stream));
  if (st != MSMPB_OK) ff->last_error = st;
  return st;
}

double FF_energy_potentials(FF *ff, double (*force)[3], double (*position)[3],
                            double *weight, double *potential) {
  begin_call(ff);
  HostState *h = host(ff);
  if (!h || !h->built) {
    set_error(ff, MSMPB_ERR_STATE);
    return NAN;
  }
  if (!ff->dev) {
    set_error(ff, MSMPB_ERR_NODEVICE);
    return NAN;
  }
  if (!position || !ff->q) {
    set_error(ff, MSMPB_ERR_ARGUMENT);
    return NAN;
  }
  msm::EvalRequest r{};
  r.pos = &position[0][0];
  r.q = ff->q;
  r.host = true;
  r.weight = weight;
  r.force = force ? &force[0][0] : nullptr;
  r.phi = potential;
  r.timing = ff->timing != 0;
  double e = NAN, q2 = 0;
  r.q2 = &q2;
  int st = msm::engine_evaluate(ff->dev, r, &e);
  if (st != MSMPB_OK) {
    set_error(ff, st);
    return NAN;
  }
  if (r.timing) fill_times(ff);
  // the reference refreshes the estimate after every evaluation
  // (code/forcefield1.c:233); sum q^2 comes from the device reduction
  ff->errEst = msm::err_model_q2(h->params, q2, ff->orderAcc) /
               std::pow(ff->cutoff, ff->orderAcc);
  return e;
}

double FF_energy(FF *ff, double (*force)[3], double (*position)[3],
                 double *weight) {
  return FF_energy_potentials(ff, force, position, weight, nullptr);
}

int FF_energy_device(FF *ff, const double *position_d, const double *charge_d,
                     const double *weight, double *force_d,
                     double *potential_d, double *energy_d, void *stream) {
  begin_call(ff);
  HostState *h = host(ff);
  if (!h || !h->built) return ff->last_error = MSMPB_ERR_STATE;
  if (!ff->dev) return ff->last_error = MSMPB_ERR_NODEVICE;
  if (!position_d || !charge_d) return ff->last_error = MSMPB_ERR_ARGUMENT;
  msm::EvalRequest r{};
  r.pos = position_d;
  r.q = charge_d;
  r.host = false;
  r.weight = weight;
  r.force = force_d;
  r.phi = potential_d;
  r.energy_dev = energy_d;
  r.stream = static_cast<cudaStream_t>(stream);
  r.timing = ff->timing != 0;
  int st = msm::engine_evaluate(ff->dev, r, nullptr);
  if (st != MSMPB_OK) ff->last_error = st;
  return st;
}

int FF_adjoint_device(FF *ff, const double *position_d, const double *charge_d,
                      const double *weight, const double *force_bar_d, double energy_bar,
                      double *charge_grad_d, double *position_grad_d, int reuse_forward,
                      void *stream) {
  begin_call(ff);
  HostState *h = host(ff);
  if (!h || !h->built) return ff->last_error = MSMPB_ERR_STATE;
  if (!ff->dev) return ff->last_error = MSMPB_ERR_NODEVICE;
  if (!position_d || !charge_d || !force_bar_d) return ff->last_error = MSMPB_ERR_ARGUMENT;
  msm::AdjointRequest r{};
  r.pos = position_d;
  r.q = charge_d;
  r.weight = weight;
  r.fbar = force_bar_d;
  r.ubar = energy_bar;
  r.dq = charge_grad_d;
  r.dr = position_grad_d;
  r.reuse = reuse_forward != 0;
  r.stream = static_cast<cudaStream_t>(stream);
  const int st = msm::engine_adjoint(ff->dev, r);
  if (st != MSMPB_OK) ff->last_error = st;
  return st;
}

long FF_evaluation_count(const FF *ff) {
  return ff->dev ? msm::engine_evaluations(ff->dev) : 0;
}

int FF_sync(FF *ff) {
  begin_call(ff);
  if (!ff->dev) return MSMPB_ERR_NODEVICE;
  int st = msm::engine_sync(ff->dev);
  if (st != MSMPB_OK) ff->last_error = st;
  return st;
}

int FF_phase_times(FF *ff, double *ms, int n) {
  if (!ff->dev) return 0;
  return msm::engine_phase_times(ff->dev, ms, n);
}

int FF_kernel_launches(FF *ff) {
  return ff->dev ? msm::engine_kernel_launches(ff->dev) : 0;
}

int FF_stencil_times(FF *ff, double *ms, int n) {
  return ff->dev ? msm::engine_level_times(ff->dev, ms, n) : 0;
}

void FF_set_timing(FF *ff, int enabled) { ff->timing = enabled ? 1 : 0; }

int FF_last_error(const FF *ff) { return ff ? ff->last_error : MSMPB_ERR_ARGUMENT; }

const char *FF_error_string(int code) {
  switch (code) {
    case MSMPB_OK: return "ok";
    case MSMPB_ERR_ARGUMENT: return "invalid argument";
    case MSMPB_ERR_STATE: return "call order violated";
    case MSMPB_ERR_CUDA: return "CUDA runtime error";
    case MSMPB_ERR_NOMEM: return "out of memory";
    case MSMPB_ERR_NODEVICE: return "no usable CUDA device";
    case MSMPB_ERR_DEVICE_CHECK: return "device-side check failed";
    case MSMPB_ERR_UNSUPPORTED: return "unsupported parameters";
    default: return "unknown error";
  }
}

void FF_set_precision(FF *ff, int precision) {
  if (precision != MSMPB_PRECISION_MIXED && precision != MSMPB_PRECISION_FP64) {
    set_error(ff, MSMPB_ERR_ARGUMENT);
    return;
  }
  if (ff->precision == precision) return;
  ff->precision = precision;
  HostState *h = host(ff);
  if (h && h->built) make_device(ff);
}

int FF_get_precision(const FF *ff) { return ff->precision; }

void FF_set_device(FF *ff, int device) {
  if (ff->device == device) return;
  ff->device = device;
  HostState *h = host(ff);
  if (h && h->built) make_device(ff);
}

void FF_delete(FF *ff) {
  if (!ff) return;
  if (ff->dev) msm::engine_destroy(ff->dev);
  free_tables(ff);
  delete host(ff);
  std::free(ff);
}

double FF_get_deltaF(FF *ff) {
  HostState *h = host(ff);
  if (!h || !h->built) return NAN;
  return msm::delta_f(h->params, ff->q);
}

double _FF_get_errEst(FF *ff, int nu) {
  HostState *h = host(ff);
  if (!h) return NAN;
  msm::Params p = h->params;
  if (!h->built) {  // callable mid-build in the reference; use FF fields
    p.N = ff->N;
    p.L = ff->maxLevel;
    for (int k = 0; k < 3; ++k) p.top[k] = ff->topGridDim[k];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) p.A[i][j] = ff->A[i][j];
    p.detA = ff->detA;
  }
  return msm::err_model(p, ff->q, nu);
}

double FF_get_errEst(FF *ff) {
  return _FF_get_errEst(ff, ff->orderAcc) / std::pow(ff->cutoff, ff->orderAcc);
}

// clock()-based tic/toc stack (code/forcefield1.c:35-56)
double msm4g_tictocmanager(int push) {
  static clock_t stack[100];
  static int top = 0;
  if (push) {
    if (top < 100) stack[top++] = std::clock();
    return 0.0;
  }
  if (top <= 0) return 0.0;
  clock_t now = std::clock();
  return (double)(now - stack[--top]) / CLOCKS_PER_SEC;
}
void msm4g_tic(void) { msm4g_tictocmanager(1); }
double msm4g_toc(void) { return msm4g_tictocmanager(0); }

// In-place inverse; returns |det A| (code/forcefield0.c:709-724)
double invert(Matrix *A) {
  double a[3][3], ai[3][3];
  std::memcpy(a, A, sizeof a);
  double d = msm::invert3(a, ai);
  std::memcpy(A, ai, sizeof ai);
  return d;
}

// Rebuilds ff->omegap and ff->cL from the current parameters
// (code/forcefield0.c:726-767)
void omegap(FF *ff) {
  HostState *h = host(ff);
  if (!h || !h->built) {
    set_error(ff, MSMPB_ERR_STATE);
    return;
  }
  msm::build_omegap_tables(h->tables);
  export_tables(ff, h->tables);
}

Vector prod(Matrix m, Vector v) {
  Vector r = {m.xx * v.x + m.xy * v.y + m.xz * v.z,
              m.yx * v.x + m.yy * v.y + m.yz * v.z,
              m.zx * v.x + m.zy * v.y + m.zz * v.z};
  return r;
}

Vector prodT(Matrix m, Vector v) {
  Vector r = {m.xx * v.x + m.yx * v.y + m.zx * v.z,
              m.xy * v.x + m.yy * v.y + m.zy * v.z,
              m.xz * v.x + m.yz * v.y + m.zz * v.z};
  return r;
}

}  // extern "C"
