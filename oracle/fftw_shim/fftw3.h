/* Minimal FFTW3-compatible declarations (test infrastructure only).
 *
 * The reference MSM library includes "fftw3.h" unconditionally
 * (code/forcefield.h:3) and uses exactly five FFTW symbols:
 *   fftw_malloc / fftw_plan_dft_3d            code/forcefield0.c:454-458
 *   fftw_execute                              code/forcefield1.c:519,524
 *   fftw_destroy_plan / fftw_free             code/forcefield0.c:700-702
 * FFTW itself is not installed in this image, so oracle/fftw_shim/fft_shim.c
 * provides a project-written FP64 mixed-radix FFT behind the same names.
 * Convention follows FFTW: FORWARD uses exp(-2*pi*i*jk/n), no normalisation.
 */
#ifndef MSMPB_ORACLE_FFTW3_SHIM_H
#define MSMPB_ORACLE_FFTW3_SHIM_H
#include <complex.h>

typedef double _Complex fftw_complex;
typedef struct msm_shim_plan *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in,
                           fftw_complex *out, int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
void *fftw_malloc(unsigned long n);
void fftw_free(void *p);

/* Direct entry used by the oracle restatement: in-place 3-D c2c transform of
 * an n0 x n1 x n2 row-major array (last index fastest). */
void msm_shim_fft3d(fftw_complex *a, int n0, int n1, int n2, int sign);

#endif
