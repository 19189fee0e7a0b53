/* FP64 CPU restatement of the reference MSM evaluation path.
 *
 * TEST INFRASTRUCTURE ONLY: this is the checker the CUDA library is compared
 * against. Nothing in the product library links, loads or calls it; only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg do.
 *
 * Parity pin: tests/test_oracle_pin.py checks this restatement against the
 * reference's own outputs (oracle/_ref, built by oracle/build_ref.py from the
 * reference sources plus two documented index patches) and against the
 * reference's golden fixtures (data/*.pot, data/*.acc, results/*.json values
 * committed under tests/golden/).
 */
#ifndef MSM_ORACLE_H
#define MSM_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

#define MSMO_MAXL 12

typedef struct msmo msmo;

/* Parameter selection mirrors FF_new, the FF_set_ setters and FF_build
 * (code/forcefield0.c:166-367); -1 means "auto" for every argument.
 * edges: row-major 3x3, columns are the box vectors (forcefield0.c:275).
 * q: charges (length N), used by the error model. fft: 1 unless the caller
 * emulates FF_set_FFT(false). Returns NULL on invalid input. */
msmo *msmo_create(int N, const double *q, const double *edges, double cutoff,
                  int nu, int maxLevel, const int *topGridDim, double estErr,
                  int fft);
void msmo_destroy(msmo *o);

/* selected parameters */
void msmo_params(const msmo *o, double *cutoff, int *nu, int *maxLevel,
                 int *topGridDim, int *nLim, double *detA);
/* error model (code/forcefield0.c:521-587) */
double msmo_errEst(const msmo *o, const double *q);
double msmo_deltaF(const msmo *o, const double *q);

/* setup tables, for checking the product's host setup */
void msmo_coeffs(const msmo *o, double *coeff1, double *coeff2);
/* level l stencil (l < maxLevel: sd^3 real-space stencil; l == maxLevel:
 * M_L^3 Fourier multiplier). dims[3] receives its shape. */
const double *msmo_khat(const msmo *o, int l, int *dims);
const double *msmo_omegap(const msmo *o, int l, int axis, int *len);
const double *msmo_cL(const msmo *o, int axis);

/* One evaluation (FF_energy, code/forcefield1.c:101-235, with the two index
 * fixes): returns the energy; force (N x 3) is overwritten; phi (N, may be
 * NULL) receives per-atom potentials dU/dq_i. weight: NULL or maxLevel+1
 * level weights (linear-in-weight semantics, see msm_oracle.c). */
double msmo_energy(const msmo *o, const double *q, const double *pos,
                   const double *weight, double *force, double *phi);

/* Instrumented pieces (same conventions as msmo_energy) */
double msmo_short_range(const msmo *o, const double *q, const double *pos,
                        double *force, double *phi);
/* grid charges at the finest level (M_1^3, unpadded, z fastest) */
void msmo_anterpolate(const msmo *o, const double *q, const double *pos,
                      double *grid);
/* finest-level potential grid e^1 from finest-level charges q^1 */
void msmo_grid_chain(const msmo *o, const double *q1, const double *weight,
                     double *e1);
void msmo_restrict(const msmo *o, int l, const double *ql, double *qlp1);
void msmo_prolong_add(const msmo *o, int l, const double *elp1, double *el);
void msmo_stencil_add(const msmo *o, int l, const double *ql, double *el);
void msmo_top_solve(const msmo *o, const double *qL, double *eL);
void msmo_interpolate(const msmo *o, const double *pos, const double *e1,
                      double *efield, double *phi_long);
int msmo_grid_dims(const msmo *o, int l, int *dims);
long msmo_pair_count(const msmo *o, const double *pos);

#ifdef __cplusplus
}
#endif
#endif
