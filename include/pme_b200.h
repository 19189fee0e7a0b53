/* pme_b200.h - extensions of the drop-in PME API (see pme.h), exported by
 * msmpb_b200/libpme.so with the same names and meanings as the MSM
 * library's extensions (msmpb_b200.h). The reference PME (code/pme.h) has
 * no status codes, no potentials, no precision choice and host arrays only.
 */
#ifndef MSMPB_B200_PME_EXT_H
#define MSMPB_B200_PME_EXT_H

#include "pme.h"

#ifdef __cplusplus
extern "C" {
#endif

#define MSMPB_OK 0
#define MSMPB_ERR_ARGUMENT 1
#define MSMPB_ERR_STATE 2
#define MSMPB_ERR_CUDA 3
#define MSMPB_ERR_NOMEM 4
#define MSMPB_ERR_NODEVICE 5
#define MSMPB_ERR_DEVICE_CHECK 6
#define MSMPB_ERR_UNSUPPORTED 7

/* MIXED: direct-space sum (erfc kernel), charge assignment and
 * interpolation in FP32 with compensated per-atom sums, close pairs in FP64;
 * FFT, multiplier, energy sums and constant terms in FP64. FP64: all FP64. */
/* FF_last_error: the status of the latest working call (FF_build,
 * FF_rebuild, FF_energy, FF_energy_potentials, FF_energy_device, FF_sync),
 * each of which clears it first. */

#define MSMPB_PRECISION_MIXED 0
#define MSMPB_PRECISION_FP64 1

int FF_last_error(const FF *ff);
const char *FF_error_string(int code);
void FF_set_precision(FF *ff, int precision);
int FF_get_precision(const FF *ff);
void FF_set_device(FF *ff, int device);
void FF_set_timing(FF *ff, int enabled);

/* FF_energy plus per-atom potentials (N doubles, may be NULL): the direct
 * and grid potentials at each atom, each weighted once as the forces are
 * (with unit weights, phi_i = dU/dq_i). */
double FF_energy_potentials(FF *ff, double (*force)[3], double (*position)[3],
                            double *weight, double *potential);

/* Device-resident evaluation on `stream` (a cudaStream_t), same conventions
 * as the MSM library's FF_energy_device; weight: NULL or 2 host doubles. */
int FF_energy_device(FF *ff, const double *position_d, const double *charge_d,
                     const double *weight, double *force_d, double *potential_d,
                     double *energy_d, void *stream);
int FF_sync(FF *ff);
/* per-phase milliseconds of the last timed evaluation (bin, pair,
 * anterpolation, restriction, stencil, top, prolongation, interpolation,
 * combine, total) and kernel launches per evaluation */
int FF_phase_times(FF *ff, double *ms, int n);
int FF_kernel_launches(FF *ff);

#ifdef __cplusplus
}
#endif
#endif
