/* msmpb_b200.h - extensions of the drop-in MSM API (see forcefield.h).
 *
 * The reference API (code/forcefield.h:70-112) has no status codes, no
 * per-atom potentials, no precision choice and host arrays only. These entry
 * points add them without changing any reference signature.
 */
#ifndef MSMPB_B200_EXT_H
#define MSMPB_B200_EXT_H

#include "forcefield.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes (FF_last_error and int-returning entry points). The
 * reference prints and continues, or exits (code/forcefield0.c:152,
 * :210-213); this library never exits and never traps the GPU. FF_last_error
 * holds the status of the latest working call (FF_build, FF_rebuild,
 * FF_rebuild_device, FF_energy, FF_energy_potentials, FF_energy_device,
 * FF_adjoint_device, FF_sync): each clears it first. Device-side checks of an
 * asynchronous evaluation surface at the next call or at FF_sync. */
#define MSMPB_OK 0
#define MSMPB_ERR_ARGUMENT 1     /* invalid size, pointer or parameter */
#define MSMPB_ERR_STATE 2        /* call order violated (e.g. energy before build) */
#define MSMPB_ERR_CUDA 3         /* a CUDA runtime call failed */
#define MSMPB_ERR_NOMEM 4        /* device or host allocation failed */
#define MSMPB_ERR_NODEVICE 5     /* no usable sm_100 device */
#define MSMPB_ERR_DEVICE_CHECK 6 /* a kernel's own bounds or wait check tripped */
#define MSMPB_ERR_UNSUPPORTED 7  /* parameter outside what the kernels support */

/* Arithmetic of the evaluation. MIXED: pair sum, grid transfers, stencils and
 * interpolation in FP32 with compensated per-atom accumulation; top-level FFT,
 * energy reductions and charge-neutrality terms in FP64. FP64: everything in
 * FP64 (the plain FP64 GPU form). */
#define MSMPB_PRECISION_MIXED 0
#define MSMPB_PRECISION_FP64 1

int FF_last_error(const FF *ff);
const char *FF_error_string(int code);

/* Precision and device: may be called before FF_build or between
 * evaluations (the device plan is rebuilt). */
void FF_set_precision(FF *ff, int precision);
int FF_get_precision(const FF *ff);
void FF_set_device(FF *ff, int device);

/* FF_energy plus per-atom potentials phi_i = dU/dq_i (N doubles, may be
 * NULL). Same host-array conventions as FF_energy. */
double FF_energy_potentials(FF *ff, double (*force)[3], double (*position)[3],
                            double *weight, double *potential);

/* Device-resident evaluation, asynchronous and ordered on `stream` (a
 * cudaStream_t; NULL = the legacy default stream). The launch sequence is
 * captured once on a private stream and replayed as a CUDA graph on `stream`
 * (timing off), or launched eagerly on `stream` with per-phase events
 * (timing on). position_d: N*3 doubles; charge_d: N doubles;
 * weight: host array of maxLevel+1 doubles or NULL; force_d (N*3),
 * potential_d (N) and energy_d (1) are device outputs, each may be NULL.
 * Returns MSMPB_OK or an error code; kernel-side checks are reported by the
 * next call or by FF_sync. */
int FF_energy_device(FF *ff, const double *position_d, const double *charge_d,
                     const double *weight, double *force_d,
                     double *potential_d, double *energy_d, void *stream);

/* Waits for the library's stream and reports device-side check failures. */
int FF_sync(FF *ff);

/* Adjoint of an evaluation (no counterpart in the reference, which computes
 * no derivatives beyond forces): for a force cotangent Fbar (device, N*3)
 * and an energy cotangent Ubar, the gradients of
 *   L = Ubar U + sum_i Fbar_i . F_i
 * with respect to the charges (charge_grad_d, N) and the positions
 * (position_grad_d, N*3), device outputs in input order, either may be
 * NULL; same inputs, weights and stream conventions as FF_energy_device.
 * The transposed operator chain runs on the GPU: the short-range pair
 * Hessian, anterpolation of the dipoles q_i Fbar_i with derivative
 * B-splines, the same grid operator, interpolation with first and second
 * derivative B-splines. reuse_forward != 0 promises that the last
 * evaluation of this handle (FF_evaluation_count) had these inputs and
 * weights and reuses its grids and per-atom results; otherwise a forward
 * pass runs first. Finest grids smaller than the B-spline order along an
 * axis return MSMPB_ERR_UNSUPPORTED. */
int FF_adjoint_device(FF *ff, const double *position_d, const double *charge_d,
                      const double *weight, const double *force_bar_d, double energy_bar,
                      double *charge_grad_d, double *position_grad_d, int reuse_forward,
                      void *stream);

/* Forward evaluations run by this handle so far (any entry point). */
long FF_evaluation_count(const FF *ff);

/* FF_rebuild (code/forcefield0.c:598-680: new box, every build-time choice
 * kept) with the level stencils computed on the GPU, ordered on `stream`
 * (a cudaStream_t; NULL = the legacy default stream) with no host
 * synchronisation: for box changes every step (constant-pressure MD). The
 * box-dependent constants and the top-level multiplier are recomputed on
 * the host (microseconds). The host copies of the level stencils
 * (ff->khat[1..maxLevel-1]) keep the previous box's values; FF_rebuild
 * refreshes them. Pair lists are rebuilt at every evaluation, so no
 * positions are needed. Returns MSMPB_OK or an error code. */
int FF_rebuild_device(FF *ff, double edges[3][3], void *stream);

/* Batches: many independent systems evaluated by one CUDA graph launch. No
 * counterpart in the reference (one system per FF_energy call,
 * code/forcefield0.c:684-780).
 *
 * Each member is an FF handle after FF_build, on one device, each handle at
 * most once; the handles may differ in N, box, order, levels and precision.
 * The batch captures every member's evaluation (the launch sequence of
 * FF_energy_device) into one graph over `branches` parallel branches, so
 * kernels of different systems run side by side on the GPU; members are
 * placed longest-first on the least-loaded branch. branches = -K
 * (FF_BATCH_MERGED = -1) instead merges the members' launches: the members
 * are dealt over K branches, and on each branch every kernel of the
 * evaluation runs as ONE launch over all its members that need it (a table
 * of the members' arguments and block ranges passed as the kernel's
 * parameter), a few tens of graph nodes per branch whatever the member count
 * (FF_batch_energy_device returns MSMPB_ERR_UNSUPPORTED if a member's
 * evaluation has a launch that cannot be merged). branches = 0 lets the
 * first FF_batch_energy_device call pick the form by timing replays of
 * candidate graphs (merged on 1, 2 and 4 branches; 4, 8, 16, 32, 64 and
 * min(n, 64) branches of per-member launches); that call synchronises
 * `stream`. At most 64 branches either way. Returns NULL with *status set (may be
 * NULL) on an invalid list (NULL or repeated handle, mixed devices:
 * MSMPB_ERR_ARGUMENT; a handle not built: MSMPB_ERR_STATE) or a CUDA
 * failure. The handles must outlive the batch and must not be evaluated
 * while a batch replay that holds them runs. */
typedef struct FFBatch FFBatch;
#define FF_BATCH_MERGED (-1)
FFBatch *FF_batch_new(FF *const *members, int n, int branches, int *status);

/* Evaluates every member, asynchronously on `stream` (a cudaStream_t; NULL
 * = the legacy default stream). Arrays of n device pointers, in member
 * order, with FF_energy_device's per-system meaning: position_d[i] (N_i*3
 * doubles), charge_d[i] (N_i); weight (host, may be NULL, as may an entry:
 * maxLevel_i+1 doubles each), force_d and potential_d (may be NULL, as may an
 * entry); energy_d: n doubles on the device (may be NULL). The graph is
 * captured on the first call and again when a pointer, a weight or a
 * member's box (FF_rebuild, FF_rebuild_device) changes; otherwise a call is
 * one graph launch. Device-side checks are reported by FF_sync of a member.
 * Returns MSMPB_OK or an error code (also kept for FF_batch_last_error). */
int FF_batch_energy_device(FFBatch *batch, const double *const *position_d,
                           const double *const *charge_d, const double *const *weight,
                           double *const *force_d, double *const *potential_d,
                           double *energy_d, void *stream);

/* Branches of the current graph (after tuning: the chosen count; -K for
 * the merged form on K branches), kernel nodes it launches, the status
 * of the latest FF_batch_energy_device call; and release. */
int FF_batch_branches(const FFBatch *batch);
int FF_batch_kernel_launches(const FFBatch *batch);
int FF_batch_last_error(const FFBatch *batch);
void FF_batch_delete(FFBatch *batch);

/* Milliseconds of each phase of the last evaluation, measured with CUDA
 * events on the evaluation stream (also copied into the reference's time_*
 * fields in seconds). Order: bin, pair, anterpolation, restriction,
 * stencils (all levels), top solve, prolongation, interpolation, combine,
 * total. Returns the number of entries written (<= n). */
int FF_phase_times(FF *ff, double *ms, int n);

/* Number of kernel launches one evaluation issues (for accounting). */
int FF_kernel_launches(FF *ff);

/* Per-level direct-stencil kernel time (ms) of the last evaluation run with
 * timing on, levels 1..maxLevel-1. Returns the number of entries written. */
int FF_stencil_times(FF *ff, double *ms, int n);

/* Timing on (default; MSMPB_TIMING=0 in the environment turns it off):
 * host-API evaluations launch eagerly with per-phase events and fill the
 * time_* members. Off: the evaluation replays a captured CUDA graph. */
void FF_set_timing(FF *ff, int enabled);

/* Measured FP32 FMA throughput of `device` in TFLOP/s: a pure-FFMA kernel
 * on every SM for about `milliseconds` (the FP32-pipe roofline peak). */
double msmpb_measure_fp32_tflops(int device, int milliseconds);

/* Size of the fixed scratch array of msmpb_level_stencil_noalloc (per device). */
#define MSMPB_NOALLOC_SCRATCH_BYTES (16u << 20)

/* One periodic level stencil that allocates no memory. No counterpart in the
 * reference, which allocates its work arrays in FF_build.
 *
 * For callers that cannot let a library allocate device memory: MD engines
 * and frameworks that own all of it through their own pool allocator (a
 * cudaMalloc behind the pool escapes its budget, and cudaMalloc / cudaFree
 * may synchronise the whole device in the middle of their step). Computes,
 * in FP64, asynchronously on `stream` (a cudaStream_t; NULL = the legacy
 * default stream) of the current device,
 *   e[x] += weight * sum_{d in [0,S)^3} k[d] * q[(x + d - S/2) mod M]
 * (S/2 rounded down per axis) for x in [0,M)^3: the direct stencil of one
 * level of FF_energy_device. q (charge_grid_d) and e (potential_grid_d) are
 * M0*M1*M2 doubles, k (stencil_d) S0*S1*S2 doubles, all row-major with the
 * last index fastest, on the current device; 1 <= S[a] <= M[a]. e is added
 * to, so clear it for a plain result.
 *
 * Scratch (tap copy, padded grid, partial sums) lives in one array of
 * MSMPB_NOALLOC_SCRATCH_BYTES compiled into the library. The tap copy and
 * the padded grid, about S0*S1*S2 + (M0+S0+3)(M1+S1+15)(M2+S2+5) doubles,
 * must fit in it (a 96^3 grid with a 25^3 stencil fits); larger sizes
 * return MSMPB_ERR_UNSUPPORTED and launch nothing. Nothing in the array has
 * to start at zero: every call rewrites what it reads.
 *
 * The first call on a device looks up the array's address there
 * (cudaGetSymbolAddress, which may load the library's GPU code); make it
 * before any stream capture. The address is kept until the process exits:
 * do not reset the device (cudaDeviceReset or a primary-context reset)
 * between calls. All calls on a device share the array: calls
 * whose GPU work overlaps race, so order them on one stream or with events.
 * Returns MSMPB_OK, MSMPB_ERR_ARGUMENT, MSMPB_ERR_UNSUPPORTED, or
 * MSMPB_ERR_NODEVICE / MSMPB_ERR_CUDA when a CUDA call fails. */
int msmpb_level_stencil_noalloc(const int M[3], const int S[3],
                                const double *charge_grid_d,
                                const double *stencil_d, double weight,
                                double *potential_grid_d, void *stream);

#ifdef __cplusplus
}
#endif
#endif
