/* FP64 CPU restatement of the reference smooth-PME evaluation (the
 * comparator of hkayabilisim/msmpb: code/pme0.c, code/pme1.c, code/pme.h).
 *
 * TEST INFRASTRUCTURE ONLY: the checker the CUDA PME library (libpme.so) is
 * compared against. Nothing in the product links, loads or calls it.
 *
 * Parity pin: tests/test_pme.py checks this restatement against the
 * reference PME built from its own sources (oracle/_ref/libpme_ref.so, by
 * oracle/build_ref.py) and against fixtures made from that build
 * (tests/golden/pme_*.npz, tests/golden/make_golden_pme.py).
 */
#ifndef PME_ORACLE_H
#define PME_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct pmeo pmeo;

/* FF_new + FF_set_* + FF_build of code/pme0.c:164-322. edges: row-major
 * 3x3 (the reference's A, box vectors as columns). cutoff, nu, tolDir <= 0
 * and M == NULL (or M[0] <= 0) mean the reference defaults (8 A, 6, 1e-5,
 * grid from its spacing table). Returns NULL where the reference exits
 * (no default grid for this order or cutoff). */
pmeo *pmeo_create(int N, const double *edges, double cutoff, int nu, const int *M,
                  double tolDir);
void pmeo_destroy(pmeo *o);
/* FF_rebuild (code/pme0.c:365-412): new box, same parameters; the Fourier
 * multiplier is recomputed from zero */
void pmeo_rebuild(pmeo *o, const double *edges);

void pmeo_params(const pmeo *o, double *cutoff, int *nu, int *M, double *tolDir,
                 double *beta, double *detA);
void pmeo_coeffs(const pmeo *o, double *coeff1, double *coeff2);
const double *pmeo_khat(const pmeo *o);         /* M0*M1*M2, z fastest */
const double *pmeo_cL(const pmeo *o, int axis); /* M_axis/2 + 1 entries */
/* FF_get_errEst (code/pme0.c:333-361) */
double pmeo_errEst(const pmeo *o, const double *q);

/* FF_energy (code/pme1.c:50-118): returns U; force (N*3) overwritten; phi
 * (may be NULL) receives per-atom potentials (pair and grid, each weighted
 * once, as the forces are). weight: NULL or 2 entries. */
double pmeo_energy(const pmeo *o, const double *q, const double *pos, const double *weight,
                   double *force, double *phi);
/* the direct-space part alone (pair energy, forces, potentials) */
double pmeo_short_range(const pmeo *o, const double *q, const double *pos, double *force,
                        double *phi);

#ifdef __cplusplus
}
#endif
#endif
