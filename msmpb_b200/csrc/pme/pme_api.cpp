// C ABI of the drop-in PME library (msmpb_b200/libpme.so): every function of
// the reference's code/pme.h:45-68 with its exact signature, plus the
// extensions of pme_b200.h. Parameter selection and tables run on the host
// in FP64 (pme_setup.cpp); every evaluation runs on the GPU through the
// engine's one-level plan with the erfc direct-space kernel. There is no CPU
// evaluation path: without a usable device FF_energy returns NaN and
// records MSMPB_ERR_NODEVICE.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <new>

#include "engine.h"
#include "msm_host.h"
#include "pme_b200.h"

namespace {

struct HostState {
  msm::Params params;
  msm::Tables tables;
  double beta = 0, tol = 0;
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

double *copy_array(const double *src, size_t n) {
  double *d = static_cast<double *>(std::malloc(sizeof(double) * (n ? n : 1)));
  if (d && n) std::memcpy(d, src, sizeof(double) * n);
  return d;
}

void free_tables(FF *ff) {
  std::free(ff->Q);
  std::free(ff->khat);
  for (int a = 0; a < 3; ++a) {
    std::free(ff->cL[a]);
    ff->cL[a] = nullptr;
  }
  ff->Q = ff->khat = nullptr;
}

// Mirror the host tables and parameters into the reference's FF members
void export_state(FF *ff, const HostState &h) {
  const msm::Params &p = h.params;
  const msm::Tables &t = h.tables;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      ff->A[i][j] = p.A[i][j];
      ff->Ai[i][j] = p.Ai[i][j];
    }
  ff->detA = p.detA;
  ff->cutoff = p.a0;
  ff->orderAcc = p.nu;
  for (int k = 0; k < 3; ++k) ff->topGridDim[k] = p.top[k];
  ff->tolDir = h.tol;
  ff->beta = h.beta;
  free_tables(ff);
  ff->Q = copy_array(t.Q, (p.nu / 2) * p.nu);
  for (int a = 0; a < 3; ++a) ff->cL[a] = copy_array(t.cL[a].data(), t.cL[a].size());
  ff->khat = copy_array(t.khat[1].data(), t.khat[1].size());
  ff->coeff1 = t.coeff1;
  ff->coeff2 = t.coeff2;
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
      std::fprintf(stderr, "pme_b200: no usable CUDA device; FF_energy will return NaN\n");
  }
}

void fill_times(FF *ff) {
  double ms[msm::kNumPhases + 1] = {};
  if (msm::engine_phase_times(ff->dev, ms, msm::kNumPhases + 1) <= 0) return;
  ff->time_nlist = ms[msm::kPhaseBin] * 1e-3;
  ff->time_partcl2partcl = ms[msm::kPhasePair] * 1e-3;
  ff->time_anterpolation = ms[msm::kPhaseAnterp] * 1e-3;
  ff->time_grid2grid = ms[msm::kPhaseTop] * 1e-3;
  ff->time_interpolation = (ms[msm::kPhaseInterp] + ms[msm::kPhaseCombine]) * 1e-3;
}

bool timing_enabled() {
  const char *v = std::getenv("MSMPB_TIMING");
  return !(v && v[0] == '0');
}

}  // namespace

extern "C" {

FF *FF_new(int N, double *q, double edges[3][3]) {
  FF *ff = static_cast<FF *>(std::calloc(1, sizeof(FF)));
  if (!ff) return nullptr;
  ff->N = N;
  ff->q = q;
  if (edges)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) ff->A[i][j] = edges[i][j];
  ff->precision = MSMPB_PRECISION_MIXED;
  const char *pv = std::getenv("MSMPB_PRECISION");
  if (pv && (std::strcmp(pv, "fp64") == 0 || std::strcmp(pv, "FP64") == 0))
    ff->precision = MSMPB_PRECISION_FP64;
  ff->timing = timing_enabled() ? 1 : 0;
  ff->host_state = new (std::nothrow) HostState();
  if (N <= 0 || !q || !edges) ff->last_error = MSMPB_ERR_ARGUMENT;
  return ff;
}

void FF_set_cutoff(FF *ff, double cutoff) { ff->cutoff = cutoff; }
double FF_get_cutoff(FF *ff) { return ff->cutoff; }
void FF_set_orderAcc(FF *ff, int orderAcc) { ff->orderAcc = orderAcc; }
void FF_set_topGridDim(FF *ff, int topGridDim[3]) {
  for (int k = 0; k < 3; ++k) ff->topGridDim[k] = topGridDim[k];
}
void FF_set_tolDir(FF *ff, double tolDir) { ff->tolDir = tolDir; }
int FF_get_orderAcc(FF *ff) { return ff->orderAcc; }
void FF_get_topGridDim(FF *ff, int topGridDim[3]) {
  for (int k = 0; k < 3; ++k) topGridDim[k] = ff->topGridDim[k];
}
double FF_get_tolDir(FF *ff) { return ff->tolDir; }

void FF_build(FF *ff, double (*position)[3]) {
  begin_call(ff);
  (void)position;  // the pair set is rebuilt on the GPU at every evaluation
  HostState *h = host(ff);
  if (!h || ff->N <= 0 || !ff->q) {
    set_error(ff, MSMPB_ERR_ARGUMENT);
    return;
  }
  msm::pme::Settings s;
  s.cutoff = ff->cutoff;
  s.tolDir = ff->tolDir;
  s.nu = ff->orderAcc;
  for (int k = 0; k < 3; ++k) s.M[k] = ff->topGridDim[k];
  int err = MSMPB_OK;
  if (!msm::pme::select(h->params, &h->beta, &h->tol, ff->N, ff->A, s, &err)) {
    if (err == MSMPB_ERR_UNSUPPORTED)
      std::fprintf(stderr, "pme_b200: default grid dimension unavailable for order %d, "
                           "cutoff %f\n", s.nu > 0 ? s.nu : 6, s.cutoff > 0 ? s.cutoff : 8.);
    set_error(ff, err);
    return;
  }
  auto t0 = std::chrono::steady_clock::now();
  msm::pme::build_tables(h->tables, h->params, h->beta);
  ff->time_stencil =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  export_state(ff, *h);
  h->built = true;
  ff->nlist = nullptr;
  ff->nlist_len = 0;
  ff->nlist_interaction_count = 0;
  make_device(ff);
}

double FF_get_errEst(FF *ff, int N, double *charge) {
  HostState *h = host(ff);
  if (!h || !charge) return NAN;
  msm::Params p = h->params;
  p.N = N;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) p.A[i][j] = ff->A[i][j];
  p.nu = ff->orderAcc;
  p.a0 = ff->cutoff;
  for (int k = 0; k < 3; ++k) p.top[k] = ff->topGridDim[k];
  return msm::pme::err_est(p, charge);
}

void FF_rebuild(FF *ff, double edges[3][3], double (*position)[3]) {
  begin_call(ff);
  (void)position;
  HostState *h = host(ff);
  if (!h || !h->built) {
    set_error(ff, MSMPB_ERR_STATE);
    return;
  }
  msm::Params p = h->params;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) p.A[i][j] = edges[i][j];
  p.detA = msm::invert3(p.A, p.Ai);
  if (!(p.detA > 0)) {
    set_error(ff, MSMPB_ERR_ARGUMENT);
    return;
  }
  h->params = p;
  auto t0 = std::chrono::steady_clock::now();
  msm::pme::build_tables(h->tables, p, h->beta);
  ff->time_stencil =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  export_state(ff, *h);
  if (ff->dev) {
    const int st = msm::engine_update_tables(ff->dev, h->tables);
    if (st != MSMPB_OK) set_error(ff, st);
  } else {
    make_device(ff);
  }
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
  double e = NAN;
  const int st = msm::engine_evaluate(ff->dev, r, &e);
  if (st != MSMPB_OK) {
    set_error(ff, st);
    return NAN;
  }
  if (r.timing) fill_times(ff);
  return e;
}

double FF_energy(FF *ff, double (*force)[3], double (*position)[3], double *weight) {
  return FF_energy_potentials(ff, force, position, weight, nullptr);
}

int FF_energy_device(FF *ff, const double *position_d, const double *charge_d,
                     const double *weight, double *force_d, double *potential_d,
                     double *energy_d, void *stream) {
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
  const int st = msm::engine_evaluate(ff->dev, r, nullptr);
  if (st != MSMPB_OK) ff->last_error = st;
  return st;
}

int FF_sync(FF *ff) {
  begin_call(ff);
  if (!ff->dev) return MSMPB_ERR_NODEVICE;
  const int st = msm::engine_sync(ff->dev);
  if (st != MSMPB_OK) ff->last_error = st;
  return st;
}

int FF_phase_times(FF *ff, double *ms, int n) {
  return ff->dev ? msm::engine_phase_times(ff->dev, ms, n) : 0;
}

int FF_kernel_launches(FF *ff) { return ff->dev ? msm::engine_kernel_launches(ff->dev) : 0; }

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

// clock()-based tic/toc stack (code/pme1.c:24-48)
double msm4g_tictocmanager(int push) {
  static clock_t stack[100];
  static int top = 0;
  if (push) {
    if (top < 100) stack[top++] = std::clock();
    return 0.0;
  }
  if (top <= 0) return 0.0;
  const clock_t now = std::clock();
  return (double)(now - stack[--top]) / CLOCKS_PER_SEC;
}
void msm4g_tic(void) { msm4g_tictocmanager(1); }
double msm4g_toc(void) { return msm4g_tictocmanager(0); }

Vector prod(Matrix m, Vector v) {
  Vector r = {m.xx * v.x + m.xy * v.y + m.xz * v.z, m.yx * v.x + m.yy * v.y + m.yz * v.z,
              m.zx * v.x + m.zy * v.y + m.zz * v.z};
  return r;
}

Vector prodT(Matrix m, Vector v) {
  Vector r = {m.xx * v.x + m.yx * v.y + m.zx * v.z, m.xy * v.x + m.yy * v.y + m.zy * v.z,
              m.xz * v.x + m.yz * v.y + m.zz * v.z};
  return r;
}

}  // extern "C"
