/* pme.h - drop-in replacement for the reference's smooth-PME comparator API
 * (hkayabilisim/msmpb code/pme.h), evaluated on one NVIDIA B200 by
 * msmpb_b200/libpme.so.
 *
 * Source- and binary-compatible with the reference driver code/pme.c:
 *  - every function code/pme.h:45-68 declares keeps its exact C signature;
 *  - struct FF keeps every member of code/pme.h:16-44 in order, with the same
 *    types and offsets (the driver reads ff->beta, ff->detA, the time_*
 *    members and nlist_len / nlist_interaction_count). The three FFTW members
 *    become same-size opaque pointers, so no fftw3.h is needed. Device state
 *    is appended at the end; FF objects are only ever allocated by FF_new.
 *  - struct O / extern o (code/pme.h:9-13) stay declared because the driver
 *    defines o; this library never reads it.
 * The MSM library (forcefield.h, libmsmpb.so) exports the same FF_* names
 * for its own method, so a program links one of the two.
 * Extensions (precision, potentials, device pointers, error codes) are
 * declared in pme_b200.h.
 */
#ifndef MSMPB_B200_PME_H
#define MSMPB_B200_PME_H

#include <stdbool.h>
#include <time.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct Vector {double x, y, z;} Vector;
typedef struct Matrix {double xx, xy, xz, yx, yy, yz, zx, zy, zz;} Matrix;
typedef struct Triple {int x, y, z;} Triple;

/* code/pme.h:9-13 */
struct O {
  char *test;
  clock_t time;
};
extern struct O o;

struct FFDevice; /* device-side plan and buffers (opaque) */

/* code/pme.h:16-44 */
typedef struct FF {
  int N;
  double *q;                  /* caller-owned charges, re-read every FF_energy */
  double A[3][3], Ai[3][3];   /* box (columns = edge vectors) and inverse */
  double detA;
  double cutoff;
  int orderAcc;
  int topGridDim[3];
  int *nlist;                 /* always NULL: the pair set is rebuilt on the
                                 GPU inside every FF_energy */
  int nlist_len;
  int nlist_interaction_count;
  double tolDir;
  void *fftw_in;              /* reference: fftw_complex*; unused */
  void *forward, *backward;   /* reference: fftw_plan; unused */
  double beta;
  double *Q;
  double *cL[3];
  double *khat;
  double coeff1, coeff2;
  double time_partcl2partcl;
  double time_nlist;
  double time_grid2grid;
  double time_stencil;
  double time_anterpolation;
  double time_interpolation;
  /* ---- appended by this implementation ---- */
  struct FFDevice *dev;
  void *host_state;           /* host-side tables (opaque) */
  int last_error;
  int precision;
  int device;
  int timing;                 /* fill time_* from per-phase CUDA events */
} FF;

FF *FF_new(int N, double *q, double edges[3][3]);
void FF_set_cutoff(FF *ff, double cutoff);
double FF_get_cutoff(FF *ff);
void FF_set_orderAcc(FF *ff, int orderAcc);
void FF_set_topGridDim(FF *ff, int topGridDim[3]);
void FF_set_tolDir(FF *ff, double tolDir);
/* Never exits: where the reference prints "default grid dimension
 * unavailable" and calls exit(1) (code/pme0.c:230-242) this records
 * MSMPB_ERR_UNSUPPORTED (FF_last_error) and FF_energy returns NaN. */
void FF_build(FF *ff, double (*position)[3]);
int FF_get_orderAcc(FF *ff);
void FF_get_topGridDim(FF *ff, int topGridDim[3]);
double FF_get_tolDir(FF *ff);
double FF_get_errEst(FF *ff, int N, double *charge);
/* New box, same parameters. The Fourier multiplier is recomputed from zero
 * (the reference adds the new one onto the old, code/pme0.c:408 with
 * :500, which is only right right after FF_build). */
void FF_rebuild(FF *ff, double edges[3][3], double (*position)[3]);
double FF_energy(FF *ff, double (*force)[3], double (*position)[3], double *weight);
  /* if weights == NULL, unit weights are assumed; otherwise weight[0]
     scales the direct part and weight[1] the grid charges (code/pme1.c:57-92) */
void FF_delete(FF *ff);

double msm4g_tictocmanager(int push);
void msm4g_tic();
double msm4g_toc();

Vector prod(Matrix m, Vector v);
Vector prodT(Matrix m, Vector v);

#ifdef __cplusplus
}
#endif
#endif
