/* FP64 CPU restatement of the reference smooth-PME path (hkayabilisim/msmpb
 * code/pme0.c, code/pme1.c). TEST INFRASTRUCTURE ONLY: see pme_oracle.h.
 *
 * Written from the method, not from the reference's code: the Ewald splitting
 * parameter from erfc(beta a0)/a0 = tolDir by Newton's method; the
 * direct-space sum of erfc(beta r)/r over all pairs and periodic images
 * within a0; order-nu B-spline charge assignment to an M0 x M1 x M2 grid;
 * the reciprocal part as a Fourier multiplier (Gaussian-screened 1/k^2 with
 * the B-spline deconvolution factors); interpolation with derivative
 * B-splines. Tables whose values must match the reference (the default grid
 * spacings, the error-model constants) carry the reference's line numbers.
 */
#include "pme_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "fftw_shim/fftw3.h"

static const double PI = 3.14159265358979323846264338327950288;

struct pmeo {
  int N;
  double A[3][3], Ai[3][3], detA;
  double a0, tol, beta;
  int nu, M[3];
  double Q[5 * 10];
  double *cL[3];
  double *khat;
  double coeff1, coeff2;
};

static int wrap(int i, int n) {
  int r = i % n;
  return r < 0 ? r + n : r;
}

/* inverse by the adjugate; returns |det| */
static double inverse3(const double a[3][3], double ai[3][3]) {
  double adj[3][3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      adj[i][j] = a[(j + 1) % 3][(i + 1) % 3] * a[(j + 2) % 3][(i + 2) % 3] -
                  a[(j + 2) % 3][(i + 1) % 3] * a[(j + 1) % 3][(i + 2) % 3];
  double det = a[0][0] * adj[0][0] + a[0][1] * adj[1][0] + a[0][2] * adj[2][0];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) ai[i][j] = adj[i][j] / det;
  return fabs(det);
}

static double row_norm(const double m[3][3], int r) {
  return sqrt(m[r][0] * m[r][0] + m[r][1] * m[r][1] + m[r][2] * m[r][2]);
}
static double col_norm(const double m[3][3], int c) {
  return sqrt(m[0][c] * m[0][c] + m[1][c] * m[1][c] + m[2][c] * m[2][c]);
}

/* root b of erfc(b) = c by Newton from b = 0, stopping when the residual
 * stops decreasing (code/pme0.c:207-222) */
static double erfc_root(double c) {
  double b = 0., res = erfc(b) - c, prev = 2. * res;
  while (fabs(res) < fabs(prev)) {
    b += res / (2. / sqrt(PI) * exp(-b * b));
    prev = res;
    res = erfc(b) - c;
  }
  return b;
}

static long long binom(int n, int k) {
  if (k < 0 || k > n) return 0;
  long long r = 1;
  for (int i = 1; i <= k; i++) r = r * (n - k + i) / i;
  return r;
}

/* Q[j*nu+k] = coefficient of t^k in the cardinal B-spline Q_nu(j+t),
 * j < nu/2, from Q_nu(x) = 1/(nu-1)! sum_i (-1)^i C(nu,i) (x-i)_+^(nu-1) */
static void build_Q(pmeo *o) {
  const int nu = o->nu;
  double fact = 1;
  for (int i = 2; i < nu; i++) fact *= i;
  for (int j = 0; j < nu / 2; j++)
    for (int k = 0; k < nu; k++) {
      long long s = 0;
      for (int i = 0; i <= j; i++) {
        long long p = 1;
        for (int e = 0; e < nu - 1 - k; e++) p *= (j - i);
        s += ((i & 1) ? -1 : 1) * binom(nu, i) * p;
      }
      o->Q[j * nu + k] = (double)(binom(nu - 1, k) * s) / fact;
    }
}

/* Q_nu(i + t), 0 <= i < nu, with d/dt in *d (may be NULL) */
static double bspline(const pmeo *o, int i, double t, double *d) {
  const int nu = o->nu;
  double sign = 1.;
  if (i >= nu / 2) {
    i = nu - 1 - i;
    t = 1. - t;
    sign = -1.;
  }
  const double *c = o->Q + i * nu;
  double v = c[nu - 1], dv = 0.;
  for (int k = nu - 2; k >= 0; k--) {
    dv = v + t * dv;
    v = c[k] + t * v;
  }
  if (d) *d = sign * dv;
  return v;
}

/* B-spline deconvolution factors c_a(k) = |sum_n Q_nu(nu/2 + n) e^{2 pi i k n / M}|^-2
 * for k = 0..M/2 (code/pme0.c:444-471) */
static void build_cL(pmeo *o) {
  const int nu = o->nu, h = nu / 2;
  double phi[8];
  for (int n = 0; n < h; n++) phi[n] = bspline(o, h + n, 0., NULL);  /* Q_nu(h + n) */
  for (int a = 0; a < 3; a++) {
    const int M = o->M[a];
    free(o->cL[a]);
    o->cL[a] = malloc(sizeof(double) * (M / 2 + 1));
    for (int k = 0; k <= M / 2; k++) {
      double s = phi[0];
      for (int n = 1; n < h; n++) s += 2. * phi[n] * cos(2. * PI * k * n / M);
      o->cL[a][k] = 1. / (s * s);
    }
  }
}

/* box-dependent constants and the Fourier multiplier (code/pme0.c:365-412,
 * :473-503) */
static void build_box(pmeo *o) {
  o->detA = inverse3(o->A, o->Ai);
  const double a0 = o->a0, beta = o->beta;
  /* coeff1: the atom's own images within a0 and its self term */
  const double as[3] = {col_norm(o->Ai, 0), col_norm(o->Ai, 1), col_norm(o->Ai, 2)};
  int lim[3];
  for (int k = 0; k < 3; k++) lim[k] = (int)ceil(a0 * as[k] - 1.);
  double c1 = 0.;
  for (int x = -lim[0]; x <= lim[0]; x++)
    for (int y = -lim[1]; y <= lim[1]; y++)
      for (int z = -lim[2]; z <= lim[2]; z++) {
        double r2 = 0.;
        for (int k = 0; k < 3; k++) {
          double rk = o->A[k][0] * x + o->A[k][1] * y + o->A[k][2] * z;
          r2 += rk * rk;
        }
        if (r2 >= a0 * a0) continue;
        if (r2 != 0.)
          c1 += erfc(beta * sqrt(r2)) / sqrt(r2);
        else
          c1 -= 2. * beta / sqrt(PI);
      }
  o->coeff1 = c1;
  o->coeff2 = PI / (beta * beta * o->detA);
  /* multiplier at wavevector K = Ai^T k, k centred */
  const int *M = o->M;
  const long n = (long)M[0] * M[1] * M[2];
  free(o->khat);
  o->khat = calloc(n, sizeof(double));
  for (int i = 0; i < M[0]; i++)
    for (int j = 0; j < M[1]; j++)
      for (int l = 0; l < M[2]; l++) {
        const int k[3] = {wrap(i + M[0] / 2, M[0]) - M[0] / 2, wrap(j + M[1] / 2, M[1]) - M[1] / 2,
                          wrap(l + M[2] / 2, M[2]) - M[2] / 2};
        double K2 = 0.;
        for (int a = 0; a < 3; a++) {
          double Ka = o->Ai[0][a] * k[0] + o->Ai[1][a] * k[1] + o->Ai[2][a] * k[2];
          K2 += Ka * Ka;
        }
        if (K2 == 0.) continue;
        const double c = o->cL[0][abs(k[0])] * o->cL[1][abs(k[1])] * o->cL[2][abs(k[2])];
        o->khat[((long)i * M[1] + j) * M[2] + l] =
            exp(-PI * PI * K2 / (beta * beta)) / (PI * o->detA * K2) * c * (double)n;
      }
}

pmeo *pmeo_create(int N, const double *edges, double cutoff, int nu, const int *M,
                  double tolDir) {
  if (N <= 0 || !edges) return NULL;
  pmeo *o = calloc(1, sizeof(pmeo));
  o->N = N;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) o->A[i][j] = edges[3 * i + j];
  o->detA = inverse3(o->A, o->Ai);
  o->a0 = cutoff > 0 ? cutoff : 8.;
  o->nu = nu > 0 ? nu : 6;
  o->tol = tolDir > 0 ? tolDir : 1e-5;
  o->beta = erfc_root(o->tol * o->a0) / o->a0;
  if (M && M[0] > 0) {
    for (int k = 0; k < 3; k++) o->M[k] = M[k];
  } else {
    /* default spacing h_ref(order, cutoff) for tolDir_ref = 1e-5 h* (code/pme0.c:224-260) */
    static const double href[2][9] = {{0.70, 0.77, 0.83, 0.91, 1.00, 1.11, 1.21, 1.33, 1.48},
                                      {1.05, 1.18, 1.29, 1.43, 1.54, 1.67, 1.82, 2.00, 2.22}};
    const int i = (o->nu - 4) / 2, j = (int)round((o->a0 - 6.) / 0.5);
    if (i < 0 || i > 1 || j < 0 || j > 8) {  /* the reference prints and exits */
      free(o);
      return NULL;
    }
    const double hstar = pow(o->detA / N, 1. / 3.);
    const double tol_ref = 1e-5 * hstar;
    const double beta_ref = erfc_root(tol_ref * o->a0 / hstar) / o->a0;
    const double h = pow(o->tol / tol_ref, 1. / o->nu) * (beta_ref / o->beta) * href[i][j];
    for (int k = 0; k < 3; k++) o->M[k] = (int)ceil(row_norm(o->A, k) / h);
  }
  build_Q(o);
  build_cL(o);
  build_box(o);
  return o;
}

void pmeo_rebuild(pmeo *o, const double *edges) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) o->A[i][j] = edges[3 * i + j];
  build_box(o);
}

void pmeo_destroy(pmeo *o) {
  if (!o) return;
  for (int a = 0; a < 3; a++) free(o->cL[a]);
  free(o->khat);
  free(o);
}

void pmeo_params(const pmeo *o, double *cutoff, int *nu, int *M, double *tolDir,
                 double *beta, double *detA) {
  if (cutoff) *cutoff = o->a0;
  if (nu) *nu = o->nu;
  if (M)
    for (int k = 0; k < 3; k++) M[k] = o->M[k];
  if (tolDir) *tolDir = o->tol;
  if (beta) *beta = o->beta;
  if (detA) *detA = o->detA;
}

void pmeo_coeffs(const pmeo *o, double *c1, double *c2) {
  *c1 = o->coeff1;
  *c2 = o->coeff2;
}
const double *pmeo_khat(const pmeo *o) { return o->khat; }
const double *pmeo_cL(const pmeo *o, int a) { return o->cL[a]; }

/* error model constants per order 4, 6, 8, 10 (code/pme0.c:339-345) */
double pmeo_errEst(const pmeo *o, const double *q) {
  if (o->nu > 10) return NAN;
  static const double Mc[4] = {9., 825., 130095., 34096545.};
  static const double cbar[4] = {1. / 6., 1. / 30., 1. / 140., 1. / 630.};
  static const double kc[4] = {0.39189561, 0.150829428, 0.049632967, 0.013520855};
  const int id = (o->nu - 4) / 2;
  const double C = 4. / 3. * Mc[id] * cbar[id] * kc[id];
  double Ai[3][3];
  const double det = inverse3(o->A, Ai);
  double hmin = INFINITY;
  for (int k = 0; k < 3; k++) hmin = fmin(hmin, 1. / (row_norm(Ai, k) * o->M[k]));
  double Q2 = 0.;
  for (int i = 0; i < o->N; i++) Q2 += q[i] * q[i];
  return Q2 * C * pow(hmin, o->nu - 2) /
         (pow(det, 1. / 3.) * sqrt((double)o->N) * pow(o->a0, o->nu - 1));
}

/* gather form: every (i, j != i, image) within a0; the atom's own images
 * are in coeff1 */
double pmeo_short_range(const pmeo *o, const double *q, const double *pos, double *force,
                        double *phi) {
  const int N = o->N;
  const double a02 = o->a0 * o->a0, beta = o->beta, cexp = 2. * beta / sqrt(PI);
  int lim[3];
  for (int k = 0; k < 3; k++) lim[k] = (int)ceil(o->a0 * col_norm(o->Ai, k) - 0.5);
  double e = 0.;
  for (int i = 0; i < N; i++) {
    double f[3] = {0, 0, 0}, p = 0.;
    for (int j = 0; j < N; j++) {
      if (j == i) continue;
      double d[3], s[3];
      for (int k = 0; k < 3; k++) d[k] = pos[3 * j + k] - pos[3 * i + k];
      for (int k = 0; k < 3; k++)
        s[k] = floor(o->Ai[k][0] * d[0] + o->Ai[k][1] * d[1] + o->Ai[k][2] * d[2] + 0.5);
      for (int k = 0; k < 3; k++)
        d[k] -= o->A[k][0] * s[0] + o->A[k][1] * s[1] + o->A[k][2] * s[2];
      for (int x = -lim[0]; x <= lim[0]; x++)
        for (int y = -lim[1]; y <= lim[1]; y++)
          for (int z = -lim[2]; z <= lim[2]; z++) {
            double r[3], r2 = 0.;
            for (int k = 0; k < 3; k++) {
              r[k] = d[k] + o->A[k][0] * x + o->A[k][1] * y + o->A[k][2] * z;
              r2 += r[k] * r[k];
            }
            if (r2 >= a02) continue;
            const double rr = sqrt(r2), v = erfc(beta * rr) / rr;
            const double g = -(v + cexp * exp(-beta * beta * r2)) / r2;
            p += q[j] * v;
            for (int k = 0; k < 3; k++) f[k] += q[j] * g * r[k];
          }
    }
    if (force)
      for (int k = 0; k < 3; k++) force[3 * i + k] = q[i] * f[k];
    if (phi) phi[i] = p;
    e += 0.5 * q[i] * p;
  }
  return e;
}

double pmeo_energy(const pmeo *o, const double *q, const double *pos, const double *weight,
                   double *force, double *phi) {
  const int N = o->N, nu = o->nu, *M = o->M;
  const double w0 = weight ? weight[0] : 1., w1 = weight ? weight[1] : 1.;
  double qs = 0., q2 = 0.;
  for (int i = 0; i < N; i++) {
    qs += q[i];
    q2 += q[i] * q[i];
  }
  double *ps = phi ? malloc(sizeof(double) * N) : NULL;
  double U = w0 * (0.5 * q2 * o->coeff1 - 0.5 * qs * qs * o->coeff2);
  U += w0 * pmeo_short_range(o, q, pos, force, ps);
  for (int i = 0; i < 3 * N; i++) force[i] *= w0;
  /* charge assignment: q_grid[(m - n) mod M] += q Q(n + nu/2, t) per axis */
  const long ng = (long)M[0] * M[1] * M[2];
  double complex *g = calloc(ng, sizeof(double complex));
  double *qg = calloc(ng, sizeof(double));
  for (int i = 0; i < N; i++) {
    int m[3];
    double t[3];
    for (int k = 0; k < 3; k++) {
      double s = o->Ai[k][0] * pos[3 * i] + o->Ai[k][1] * pos[3 * i + 1] +
                 o->Ai[k][2] * pos[3 * i + 2];
      s -= floor(s);
      t[k] = M[k] * s;
      m[k] = (int)floor(t[k]);
      t[k] -= m[k];
    }
    for (int a = -nu / 2; a < nu / 2; a++) {
      const double wa = bspline(o, a + nu / 2, t[0], NULL);
      for (int b = -nu / 2; b < nu / 2; b++) {
        const double wb = wa * bspline(o, b + nu / 2, t[1], NULL);
        for (int c = -nu / 2; c < nu / 2; c++) {
          const long idx = ((long)wrap(m[0] - a, M[0]) * M[1] + wrap(m[1] - b, M[1])) * M[2] +
                           wrap(m[2] - c, M[2]);
          qg[idx] += q[i] * wb * bspline(o, c + nu / 2, t[2], NULL);
        }
      }
    }
  }
  /* e = K (w1 q): FFT, multiply, inverse FFT over M^3 */
  for (long k = 0; k < ng; k++) g[k] = w1 * qg[k];
  msm_shim_fft3d(g, M[0], M[1], M[2], FFTW_FORWARD);
  for (long k = 0; k < ng; k++) g[k] *= o->khat[k];
  msm_shim_fft3d(g, M[0], M[1], M[2], FFTW_BACKWARD);
  double ug = 0.;
  for (long k = 0; k < ng; k++) ug += w1 * qg[k] * creal(g[k]) / (double)ng;
  U += 0.5 * ug;
  /* field and potential at the atoms, derivative B-splines */
  for (int i = 0; i < N; i++) {
    int m[3];
    double t[3];
    for (int k = 0; k < 3; k++) {
      const double s = o->Ai[k][0] * pos[3 * i] + o->Ai[k][1] * pos[3 * i + 1] +
                       o->Ai[k][2] * pos[3 * i + 2];
      t[k] = M[k] * s;
      m[k] = (int)floor(t[k]);
      t[k] -= m[k];
    }
    double gu[3] = {0, 0, 0}, pv = 0.;
    for (int a = -nu / 2; a < nu / 2; a++) {
      double da, va = bspline(o, a + nu / 2, t[0], &da);
      for (int b = -nu / 2; b < nu / 2; b++) {
        double db, vb = bspline(o, b + nu / 2, t[1], &db);
        for (int c = -nu / 2; c < nu / 2; c++) {
          double dc, vc = bspline(o, c + nu / 2, t[2], &dc);
          const long idx = ((long)wrap(m[0] - a, M[0]) * M[1] + wrap(m[1] - b, M[1])) * M[2] +
                           wrap(m[2] - c, M[2]);
          const double e = creal(g[idx]) / (double)ng;
          gu[0] += da * vb * vc * e;
          gu[1] += va * db * vc * e;
          gu[2] += va * vb * dc * e;
          pv += va * vb * vc * e;
        }
      }
    }
    for (int k = 0; k < 3; k++) gu[k] *= M[k];
    for (int k = 0; k < 3; k++) {
      const double E = -(o->Ai[0][k] * gu[0] + o->Ai[1][k] * gu[1] + o->Ai[2][k] * gu[2]);
      force[3 * i + k] += q[i] * E;
    }
    if (phi) phi[i] = w0 * (q[i] * o->coeff1 - qs * o->coeff2 + ps[i]) + pv;
  }
  free(ps);
  free(g);
  free(qg);
  return U;
}
