// Device plan for one FF handle: buffers, uploaded tables, the launch
// sequence of one evaluation and its CUDA graph.
#pragma once

#include <cuda_runtime.h>

#include "launch_rec.h"
#include "msm_host.h"

struct FFDevice;

namespace msm {

enum Phase {
  kPhaseBin = 0,
  kPhasePair,
  kPhaseAnterp,
  kPhaseRestrict,
  kPhaseStencil,
  kPhaseTop,
  kPhaseProlong,
  kPhaseInterp,
  kPhaseCombine,
  kNumPhases
};

// Creates the device plan for the tables (allocates everything an
// evaluation needs). Returns nullptr and sets *err on failure.
FFDevice *engine_create(const Tables &t, int precision, int device, int *err);
void engine_destroy(FFDevice *d);

// Re-uploads box-dependent tables after FF_rebuild (same sizes).
int engine_update_tables(FFDevice *d, const Tables &t);
// The same with the level stencils computed on the device, ordered on
// `stream` (t's level stencils are not read).
int engine_update_tables_device(FFDevice *d, const Tables &t, cudaStream_t stream);

struct EvalRequest {
  const double *pos;     // host or device N*3
  const double *q;       // host or device N
  bool host;             // pos/q/force/phi are host pointers
  const double *weight;  // host, L+1 entries or nullptr
  double *force;         // N*3 or nullptr
  double *phi;           // N or nullptr
  double *energy_dev;    // device scalar or nullptr (device mode)
  cudaStream_t stream;   // device mode: caller stream (0 = own stream)
  bool timing;           // record per-phase events
  double *q2;            // host mode, may be null: receives sum q_i^2 (FP64,
                         // reduced on the device)
};

// Runs one evaluation. Host mode synchronises and returns the energy in
// *energy; device mode is asynchronous. Returns an MSMPB_* status.
int engine_evaluate(FFDevice *d, const EvalRequest &r, double *energy);

// Adjoint of one evaluation (see k_adjoint.cu): for the cotangents fbar
// (device, N*3) and ubar, charge and position gradients of
// ubar U + sum fbar . F (device outputs, input order, each may be null).
// reuse: the last evaluation of this plan had these inputs and weights, so
// its retained state is used; otherwise a forward pass runs first.
struct AdjointRequest {
  const double *pos, *q, *weight, *fbar;
  double ubar;
  double *dq, *dr;
  bool reuse;
  cudaStream_t stream;
};
int engine_adjoint(FFDevice *d, const AdjointRequest &r);
// Enqueues one device-pointer evaluation (r.pos, r.q, r.force, r.phi,
// r.energy_dev; r.host false) on s with no waits or host work, for capture
// into a caller's graph; engine_version changes with every box update and
// differs between engines (a rebuilt or re-targeted FF gets a new engine).
// engine_begin, outside any capture, orders such an evaluation about to run
// on s after a pending device rebuild and counts it.
int engine_enqueue(FFDevice *d, const EvalRequest &r, cudaStream_t s);
int engine_begin(FFDevice *d, cudaStream_t s);
// Appends the launches engine_enqueue would issue for r to rec (kernels with
// their arguments, clears as kernels, kFork / kJoin around the short-range
// branch); rec.ok turns false if a launch cannot be merged.
int engine_record(FFDevice *d, const EvalRequest &r, Recorder &rec);
long engine_version(FFDevice *d);
int engine_device(FFDevice *d);
long engine_evaluations(FFDevice *d);

// Waits for outstanding work and returns device-side check flags as status.
int engine_sync(FFDevice *d);

// Phase times of the last timed evaluation (ms), kNumPhases + total.
int engine_phase_times(FFDevice *d, double *ms, int n);
int engine_kernel_launches(FFDevice *d);
// Stencil kernel time per level (1..L-1) of the last timed evaluation
int engine_level_times(FFDevice *d, double *ms, int n);

}  // namespace msm
