/* forcefield.h - drop-in replacement for the reference MSM C API
 * (hkayabilisim/msmpb code/forcefield.h), evaluated on one NVIDIA B200.
 *
 * Source- and binary-compatible with the reference drivers (code/msmpb.c,
 * code/example.c):
 *  - every function the reference exports keeps its exact C signature;
 *  - struct FF keeps every member, in the same order and with the same types
 *    and offsets, so drivers that read members directly (code/msmpb.c:187-273:
 *    time_*, ntc, tmax, nlist_len, nlist_interaction_count, detA) still work.
 *    The three FFTW members (code/forcefield.h:40-41) become same-size opaque
 *    pointers, so no fftw3.h is needed. Device state is appended at the end;
 *    FF objects are only ever allocated by FF_new.
 *  - struct O / extern o (code/forcefield.h:9-19) stay declared because the
 *    drivers define o; this library never reads it.
 * Extensions (precision, potentials, device pointers, error codes, batches)
 * are declared in msmpb_b200.h.
 */
#ifndef MSMPB_B200_FORCEFIELD_H
#define MSMPB_B200_FORCEFIELD_H

#include <stdbool.h>
#include <time.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct Vector {double x, y, z;} Vector;
typedef struct Matrix {double xx, xy, xz, yx, yy, yz, zx, zy, zz;} Matrix;
typedef struct Triple {int x, y, z;} Triple;

/* code/forcefield.h:9-19: optional-output hook defined by the drivers */
struct O {
  char *test;
  double *khatLp1;
  double **kappa;
  double e_const;
  double *e;
  bool recX;
  clock_t time;
  int level;
};
extern struct O o;

struct FFDevice; /* device-side plan and buffers (opaque) */

/* code/forcefield.h:22-69 */
typedef struct FF {
  int N;
  double *q;                  /* caller-owned charges, re-read every FF_energy */
  double A[3][3], Ai[3][3];   /* box (columns = edge vectors) and inverse */
  double detA;
  double relCutoff;
  double errEst;
  double errEstMoore;
  int ntc;
  int tmax;
  double estErr;
  int orderAcc;
  int maxLevel;
  int topGridDim[3];
  int *nlist;                 /* always NULL: the pair list is rebuilt on the
                                 GPU inside every FF_energy */
  int nlist_len;
  int nlist_interaction_count;
  bool FFT;
  void *fftw_in;              /* reference: fftw_complex*; unused */
  void *forward, *backward;   /* reference: fftw_plan; unused */
  double *tau;
  double *dsigma;
  double **sigmad;
  double *Q;
  double *J;
  double *(*omegap)[3];
  int nLim;
  double *aCut;
  double cutoff;
  double *cL[3];
  double **khat;
  double coeff1, coeff2;
  double time_partcl2partcl;
  double time_nlist;
  double time_grid2grid[10];
  double time_stencil[10];
  double time_anterpolation;
  double time_interpolation;
  double time_restriction[10];
  double time_prolongation[10];
  double time_padding[10];
  /* ---- appended by this implementation ---- */
  struct FFDevice *dev;
  void *host_state;           /* host-side tables (opaque) */
  int last_error;
  int precision;
  int device;
  int timing;                 /* fill time_* from per-phase CUDA events */
  double margin;
} FF;

FF *FF_new(int N, double *q);
double FF_get_cutoff(FF *ff);
void FF_set_cutoff(FF *ff, double cutoff);
void FF_set_orderAcc(FF *ff, int orderAcc);
void FF_set_maxLevel(FF *ff, int maxLevel);
void FF_set_topGridDim(FF *ff, int topGridDim[3]);
void FF_set_FFT(FF *ff, bool FFT);
void FF_build(FF *ff, int N, double (*position)[3], double edges[3][3],
              double margin);
int FF_get_orderAcc(FF *ff);
int FF_get_maxLevel(FF *ff);
void FF_get_topGridDim(FF *ff, int topGridDim[3]);
bool FF_get_FFT(FF *ff);
double FF_get_errEst(FF *ff);
double FF_get_estErr(FF *ff);
void FF_set_estErr(FF *ff, double estErr);
void FF_rebuild(FF *ff, double edges[3][3], double (*position)[3],
                double margin);
double FF_energy(FF *ff, double (*force)[3], double (*position)[3],
                 double *weight);
void FF_delete(FF *ff);
double FF_get_deltaF(FF *ff);

double msm4g_tictocmanager(int push);
void msm4g_tic(void);
double msm4g_toc(void);

double invert(Matrix *A);
void omegap(FF *ff);

Vector prod(Matrix m, Vector v);
Vector prodT(Matrix m, Vector v);

double _FF_get_errEst(FF *ff, int nu);

#ifdef __cplusplus
}
#endif

#ifndef __cplusplus
/* code/forcefield.h:99-107 (GNU statement expressions) */
#define max(a,b) \
({ __typeof__ (a) _a = (a); \
  __typeof__ (b) _b = (b); \
  _a > _b ? _a : _b; })

#define min(a,b) \
({ __typeof__ (a) _a = (a); \
  __typeof__ (b) _b = (b); \
  _a > _b ? _b : _a; })
#endif

#endif
