/* FP64 CPU restatement of the reference MSM path (hkayabilisim/msmpb).
 *
 * TEST INFRASTRUCTURE ONLY - the oracle the CUDA library is checked against.
 * It is never linked into or called by the product library.
 *
 * Every function cites the reference code it restates (paths are relative to
 * the reference project). Grids are stored unpadded with periodic index
 * arithmetic instead of the reference's halo copies; the arithmetic per grid
 * point is the same. Two index bugs of the shipped reference are fixed here:
 *   - the L=1 grid-energy read of q[1] (code/forcefield1.c:195-204);
 *   - the unpadded top-level read in FFTg2g at L>1 (code/forcefield1.c:504-514).
 * The short-range sum enumerates every (pair, lattice image) with r < a0
 * through a periodic cell grid. For the orthorhombic boxes of every reference
 * fixture this is exactly the reference's neighbour-list + image-window sum
 * (code/forcefield0.c:21-164, code/forcefield1.c:240-321).
 */
#include "msm_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "fftw_shim/fftw3.h"

struct msmo {
  int N;
  double A[3][3], Ai[3][3], detA;
  double estErr;
  int nu, L, M[3], fft;
  double a0;
  double aCut[MSMO_MAXL + 2];
  double relCutoff;
  int nLim;
  double tau[16];
  double Q[5 * 10];
  double J[11];
  int gd[MSMO_MAXL + 2][3];
  int sd[MSMO_MAXL + 2][3];
  double *omegap[MSMO_MAXL + 2][3];
  int opD[MSMO_MAXL + 2][3];
  double *cL[3];
  double *khat[MSMO_MAXL + 2];
  double coeff1, coeff2;
};

static const double PI = 3.14159265358979323846264338327950288;

/* ---- small helpers ------------------------------------------------------ */

static double horner(const double *c, int n, double s) {
  double v = c[n - 1];
  for (int k = n - 2; k >= 0; k--) v = c[k] + s * v;
  return v;
}

static int wrap(int i, int n) {
  int r = i % n;
  return r < 0 ? r + n : r;
}

/* 3x3 inverse via the adjugate; returns |det| (code/forcefield0.c:709-724) */
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

/* ---- parameter selection (code/forcefield0.c:219-348, :553-587) -------- */

/* next integer >= m whose prime factors are all in {2,3,5,7}
 * (code/forcefield0.c:219-245) */
static int smooth7(int m) {
  for (;; m++) {
    int r = m;
    for (int f = 2; f <= 7 && r > 1; f++)
      while (r % f == 0) r /= f;
    if (r == 1 || m <= 1) return m;
  }
}

/* auto top-grid size (code/forcefield0.c:247-269); row norms of A */
static void auto_grid(const msmo *o, int L, int out[3]) {
  double eta = 1.0;
  if (o->fft) eta = (L >= 2) ? 0.83 : 5.7;
  double a[3] = {row_norm(o->A, 0), row_norm(o->A, 1), row_norm(o->A, 2)};
  double g = pow(a[0] * a[1] * a[2], -1. / 3.);
  for (int k = 0; k < 3; k++)
    out[k] = (int)ceil(pow(2., 1. - L) * pow(eta * o->N, 1. / 3.) * a[k] * g);
}

/* error-model numerator (code/forcefield0.c:553-582) */
static double err_model(const msmo *o, const double *q, int nu) {
  int L = o->L, N = o->N;
  int M1[3] = {o->M[0], o->M[1], o->M[2]};
  for (int i = 1; i < L; i++)
    for (int k = 0; k < 3; k++) M1[k] *= 2;
  double Q2 = 0;
  for (int i = 0; i < N; i++) Q2 += q[i] * q[i];
  double Fref = (Q2 / (double)N) / pow(o->detA / (double)N, 5. / 6.);
  double h1 = fmax(fmax(row_norm(o->A, 0) / M1[0], row_norm(o->A, 1) / M1[1]),
                   row_norm(o->A, 2) / M1[2]);
  double dF = Q2 * (1 - pow(4.0, -L)) * pow(h1, nu - 1) *
              pow(o->detA, -1. / 3.) * pow(N, -2.0 / 3.0);
  return dF / Fref;
}

double msmo_errEst(const msmo *o, const double *q) {
  return err_model(o, q, o->nu) / pow(o->a0, o->nu);
}

/* code/forcefield0.c:521-551 (fitted constants C_{nu-1}) */
double msmo_deltaF(const msmo *o, const double *q) {
  static const double C[4] = {0.825169, 5.16701, 73.6508, 1977.23};
  int L = o->L, N = o->N, nu = o->nu;
  int M1[3] = {o->M[0], o->M[1], o->M[2]};
  for (int i = 1; i < L; i++)
    for (int k = 0; k < 3; k++) M1[k] *= 2;
  double Q2 = 0;
  for (int i = 0; i < N; i++) Q2 += q[i] * q[i];
  double h1 = fmax(fmax(row_norm(o->A, 0) / M1[0], row_norm(o->A, 1) / M1[1]),
                   row_norm(o->A, 2) / M1[2]);
  return C[(nu - 4) / 2] * Q2 * (1 - pow(4.0, -L)) * pow(h1, nu - 1) *
         pow(o->detA, -1. / 3.) * pow(N, -2.0 / 3.0) / pow(o->a0, nu);
}

/* ---- coefficient tables (code/forcefield0.c:369-416) -------------------- */

static long long binom(int n, int k) {
  if (k < 0 || k > n) return 0;
  long long r = 1;
  for (int i = 1; i <= k; i++) r = r * (n - k + i) / i;
  return r;
}

/* Softening polynomial: Taylor coefficients of (1+s)^(-1/2) */
static void build_tau(msmo *o) {
  o->tau[0] = 1.;
  for (int i = 1; i < o->nu; i++)
    o->tau[i] = -(1. - 0.5 / (double)i) * o->tau[i - 1];
}

/* B-spline pieces: Q[j*nu+k] = coefficient of t^k in Q_nu(j+t), j < nu/2,
 * from the truncated-power form
 * Q_nu(x) = 1/(nu-1)! sum_i (-1)^i C(nu,i) (x-i)_+^(nu-1). */
static void build_Q(msmo *o) {
  int nu = o->nu;
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

/* Q_nu(i + t) for 0 <= i < nu, 0 <= t <= 1 (code/forcefield1.c:609-622);
 * d (may be NULL) receives d/dt (code/forcefield1.c:624-637) */
static double bspline(const msmo *o, int i, double t, double *d) {
  int nu = o->nu;
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

/* two-scale stencil J[n+nu/2] = 2^(1-nu) C(nu, n+nu/2) */
static void build_J(msmo *o) {
  for (int n = 0; n <= o->nu; n++)
    o->J[n] = (double)binom(o->nu, n) * pow(2., 1 - o->nu);
}

/* ---- quasi-interpolation (code/forcefield0.c:726-767) ------------------- */
static void build_omegap(msmo *o) {
  int nu = o->nu, h = nu / 2;
  double Phi[8] = {0};
  for (int n = 1; n < h; n++) Phi[n] = o->Q[(h - n) * nu];
  for (int k = 0; k < nu; k++) Phi[0] += o->Q[(h - 1) * nu + k];
  int M[3] = {o->M[0], o->M[1], o->M[2]};
  int opLim = 2 * o->nLim;
  for (int l = o->L; l >= 1; l--) {
    for (int a = 0; a < 3; a++) {
      int Ma = M[a];
      double *c = malloc(sizeof(double) * Ma);
      for (int k = 0; k < Ma; k++) {
        double th = 2. * PI * (double)k / (double)Ma;
        double v = Phi[0];
        for (int n = 1; n < h; n++) v += 2. * Phi[n] * cos((double)n * th);
        c[k] = 1. / (v * v);
      }
      int opD = (Ma / 2 > opLim) ? opLim + 1 : Ma / 2 + 1;
      double *om = calloc(opD, sizeof(double));
      for (int m = 0; m < opD; m++) {
        double v = c[0];
        for (int k = 1; k <= (Ma - 1) / 2; k++)
          v += 2. * c[k] * cos(2. * PI * (double)(k * m) / (double)Ma);
        if (Ma % 2 == 0) v += c[Ma / 2] * cos(PI * (double)m);
        om[m] = v / (double)Ma;
      }
      o->omegap[l][a] = om;
      o->opD[l][a] = opD;
      if (l == o->L)
        o->cL[a] = c;
      else
        free(c);
    }
    for (int a = 0; a < 3; a++) M[a] *= 2;
  }
}

/* ---- level-l real-space stencils (code/forcefield0.c:965-1081) ---------- */

/* kappa_l(A s): image sum of g_{a_l/2} - g_{a_l} (code/forcefield0.c:1041) */
static double kappa_l(const msmo *o, int l, const double s[3],
                      const double as[3]) {
  int nu = o->nu;
  double al = o->aCut[l], acc = 0.;
  double lo[3], hi[3];
  for (int k = 0; k < 3; k++) {
    lo[k] = floor(s[k] - al * as[k] + 1.);
    hi[k] = ceil(s[k] + al * as[k] - 1.);
  }
  for (double px = lo[0]; px <= hi[0]; px++)
    for (double py = lo[1]; py <= hi[1]; py++)
      for (double pz = lo[2]; pz <= hi[2]; pz++) {
        double x = s[0] - px, y = s[1] - py, z = s[2] - pz;
        double rx = o->A[0][0] * x + o->A[0][1] * y + o->A[0][2] * z;
        double ry = o->A[1][0] * x + o->A[1][1] * y + o->A[1][2] * z;
        double rz = o->A[2][0] * x + o->A[2][1] * y + o->A[2][2] * z;
        double rho = sqrt(rx * rx + ry * ry + rz * rz) / al;
        if (rho >= 1.) continue;
        double g1 = horner(o->tau, nu, rho * rho - 1.) / al;
        double r2 = 2. * rho;
        double g2 = (r2 >= 1.) ? 1. / r2 : horner(o->tau, nu, r2 * r2 - 1.);
        g2 *= 2. / al;
        acc += g2 - g1;
      }
  return acc;
}

/* periodic offset in [-n/2, n - n/2) as in code/forcefield0.c:1002 */
static int centred(int d, int n) { return wrap(d + n / 2, n) - n / 2; }

static void build_level_stencil(msmo *o, int l, const double as[3]) {
  const int *gd = o->gd[l], *sd = o->sd[l];
  int kx = sd[0], ky = sd[1], kz = sd[2];
  double *kap = malloc(sizeof(double) * kx * ky * kz);
  for (int i = 0; i < kx; i++)
    for (int j = 0; j < ky; j++)
      for (int k = 0; k < kz; k++) {
        double s[3] = {(double)(i - kx / 2) / gd[0], (double)(j - ky / 2) / gd[1],
                       (double)(k - kz / 2) / gd[2]};
        kap[(i * ky + j) * kz + k] = kappa_l(o, l, s, as);
      }
  double *const *op = o->omegap[l];
  double *F = calloc((size_t)kx * ky * kz, sizeof(double));
  double *G = calloc((size_t)kx * ky * kz, sizeof(double));
  double *kh = o->khat[l];
  /* z pass */
  for (int i = 0; i < kx; i++)
    for (int j = 0; j < ky; j++)
      for (int k1 = 0; k1 < kz; k1++) {
        double acc = 0.;
        for (int k0 = 0; k0 < kz; k0++)
          acc += op[2][abs(centred(k0 - k1, gd[2]))] * kap[(i * ky + j) * kz + k0];
        F[(i * ky + j) * kz + k1] = acc;
      }
  /* y pass */
  for (int i = 0; i < kx; i++)
    for (int j1 = 0; j1 < ky; j1++)
      for (int k = 0; k < kz; k++) {
        double acc = 0.;
        for (int j0 = 0; j0 < ky; j0++)
          acc += op[1][abs(centred(j0 - j1, gd[1]))] * F[(i * ky + j0) * kz + k];
        G[(i * ky + j1) * kz + k] = acc;
      }
  /* x pass */
  for (int i1 = 0; i1 < kx; i1++)
    for (int j = 0; j < ky; j++)
      for (int k = 0; k < kz; k++) {
        double acc = 0.;
        for (int i0 = 0; i0 < kx; i0++)
          acc += op[0][abs(centred(i0 - i1, gd[0]))] * G[(i0 * ky + j) * kz + k];
        kh[(i1 * ky + j) * kz + k] = acc;
      }
  free(kap);
  free(F);
  free(G);
}

/* ---- top-level Fourier multiplier (code/forcefield0.c:769-896) ---------- */

/* Numerator polynomials of the spherical Bessel function j_{nu-1}:
 * t^(nu-1) j_{nu-1}(t) = S(t^2) sin(t)/t - C(t^2) cos(t), from the Rayleigh
 * expansion (Abramowitz & Stegun 10.1.8). S[k], C[k] multiply t^(2k). */
static void bessel_numerators(int nu, double S[8], double C[8]) {
  int n = nu - 1, m = (n - 1) / 2; /* n odd */
  double sg = (m & 1) ? -1. : 1.;
  for (int k = 0; k < 8; k++) S[k] = C[k] = 0.;
  for (int k = 0; 2 * k <= n; k++) { /* cos-part: t^(n-1-2k) */
    long double v = 1.L;
    for (int i = n - 2 * k + 1; i <= n + 2 * k; i++) v *= i;
    for (int i = 2; i <= 2 * k; i++) v /= i;
    v /= powl(2.L, 2 * k);
    C[(n - 1 - 2 * k) / 2] = sg * ((k & 1) ? -1. : 1.) * (double)v;
  }
  for (int k = 0; 2 * k + 1 <= n; k++) { /* sin-part: t^(n-2k-1) */
    long double v = 1.L;
    for (int i = n - 2 * k; i <= n + 2 * k + 1; i++) v *= i;
    for (int i = 2; i <= 2 * k + 1; i++) v /= i;
    v /= powl(2.L, 2 * k + 1);
    S[(n - 2 * k - 1) / 2] = sg * ((k & 1) ? -1. : 1.) * (double)v;
  }
}

/* psi(|k|): Fourier transform of the top-level kernel */
static double top_psi(const msmo *o, double k2, const double S[8],
                      const double C[8], const double tc[7]) {
  if (k2 == 0) return 0.;
  int nu = o->nu;
  double aL = o->aCut[o->L];
  double t = PI * sqrt(k2) * aL, t2 = t * t, v;
  if (t <= 4 * PI / 4.0) { /* Taylor branch, ntc = 7 terms, tmax = 4 */
    double acc = 0., tp = 1.;
    for (int i = 0; i < 7; i++) {
      acc += tp / tc[i];
      tp *= t2;
    }
    v = acc / t2;
  } else {
    double s = 0., c = 0., tp = 1.;
    for (int k = 0; k < nu / 2; k++) {
      s += S[k] * tp;
      c += C[k] * tp;
      tp *= t2;
    }
    v = (s * (sin(t) / t) - c * cos(t)) / pow(t, 2.0 * nu);
  }
  double dfact = 1.;
  for (int i = 1; i <= 2 * nu - 1; i += 2) dfact *= i;
  return v * (dfact * PI * aL * aL / o->detA);
}

static void build_top(msmo *o) {
  int nu = o->nu;
  double S[8], C[8], tc[7];
  bessel_numerators(nu, S, C);
  /* Taylor series of j_{nu-1}(t)/t^(nu-1): 1/tc_i with tc_0 = (2nu-1)!!,
   * tc_i = -2i(2nu-1+2i) tc_{i-1}; exact integers then one rounding */
  __int128 t = 1;
  for (int i = 1; i <= 2 * nu - 1; i += 2) t *= i;
  tc[0] = (double)t;
  for (int i = 1; i < 7; i++) {
    t = -t * (2 * i) * (2 * nu - 1 + 2 * i);
    tc[i] = (double)t;
  }
  const int *g = o->M;
  double *kh = o->khat[o->L];
  for (int x = 0; x < g[0]; x++) {
    int cx = x < (g[0] + 1) / 2 ? x : x - g[0];
    for (int y = 0; y < g[1]; y++) {
      int cy = y < (g[1] + 1) / 2 ? y : y - g[1];
      for (int z = 0; z < g[2]; z++) {
        int cz = z < (g[2] + 1) / 2 ? z : z - g[2];
        double ax = o->Ai[0][0] * cx + o->Ai[1][0] * cy + o->Ai[2][0] * cz;
        double ay = o->Ai[0][1] * cx + o->Ai[1][1] * cy + o->Ai[2][1] * cz;
        double az = o->Ai[0][2] * cx + o->Ai[1][2] * cy + o->Ai[2][2] * cz;
        double psi = top_psi(o, ax * ax + ay * ay + az * az, S, C, tc);
        double w = o->cL[0][x] * o->cL[1][y] * o->cL[2][z];
        kh[(x * g[1] + y) * g[2] + z] = psi * w * g[0] * g[1] * g[2];
      }
    }
  }
}

/* ---- constant terms (code/forcefield0.c:612-643) ------------------------ */
static void build_coeffs(msmo *o, const double as[3]) {
  int nu = o->nu;
  double a0 = o->aCut[0];
  double lim[3];
  for (int k = 0; k < 3; k++) lim[k] = ceil(a0 * as[k] - 1.);
  double c1 = 0.;
  for (double x = -lim[0]; x <= lim[0]; x++)
    for (double y = -lim[1]; y <= lim[1]; y++)
      for (double z = -lim[2]; z <= lim[2]; z++) {
        if (x * x + y * y + z * z == 0) continue;
        double rx = o->A[0][0] * x + o->A[0][1] * y + o->A[0][2] * z;
        double ry = o->A[1][0] * x + o->A[1][1] * y + o->A[1][2] * z;
        double rz = o->A[2][0] * x + o->A[2][1] * y + o->A[2][2] * z;
        double r2 = rx * rx + ry * ry + rz * rz;
        if (r2 >= a0 * a0) continue;
        if (r2 != 0.) c1 += 1. / sqrt(r2);
        c1 -= horner(o->tau, nu, r2 / (a0 * a0) - 1.) / a0;
      }
  o->coeff1 = c1;
  double aL = o->aCut[o->L];
  o->coeff2 = PI * aL * aL / ((4 * nu + 2) * o->detA);
}

/* ---- construction (code/forcefield0.c:271-367, :598-680) ---------------- */
msmo *msmo_create(int N, const double *q, const double *edges, double cutoff,
                  int nu, int maxLevel, const int *topGridDim, double estErr,
                  int fft) {
  if (N <= 0 || !q || !edges) return NULL;
  msmo *o = calloc(1, sizeof(msmo));
  o->N = N;
  o->fft = fft ? 1 : 0;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) o->A[i][j] = edges[3 * i + j];
  o->detA = inverse3(o->A, o->Ai);
  o->estErr = (estErr == -1) ? 0.001 : estErr;
  o->L = (maxLevel == -1) ? 1 : maxLevel;
  int haveM = topGridDim && topGridDim[0] != -1;
  if (haveM)
    for (int k = 0; k < 3; k++) o->M[k] = topGridDim[k];
  if (!o->fft && !haveM) { /* code/forcefield0.c:292-307 */
    int l = 1, Mest[3];
    for (;;) {
      auto_grid(o, l, Mest);
      if (Mest[0] * Mest[1] * Mest[2] <= sqrt(N)) break;
      l++;
    }
    o->L = l;
    for (int k = 0; k < 3; k++) o->M[k] = Mest[k];
  }
  if (o->fft && !haveM) auto_grid(o, o->L, o->M);
  if (o->fft)
    for (int k = 0; k < 3; k++) o->M[k] = smooth7(o->M[k]);
  if (o->L < 1 || o->L > MSMO_MAXL) {
    free(o);
    return NULL;
  }
  o->nu = nu;
  if (cutoff == -1) {
    if (nu == -1) {
      double best = INFINITY;
      for (int t = 4; t <= 10; t += 2) {
        o->nu = t;
        double c = pow(err_model(o, q, t) / o->estErr, 1. / t);
        if (c < best) best = c;
      }
      o->nu = -1;
      cutoff = best;
    } else {
      cutoff = pow(err_model(o, q, nu) / o->estErr, 1. / nu);
    }
  }
  if (nu == -1) {
    double best = INFINITY;
    int bnu = 4;
    for (int t = 4; t <= 10; t += 2) {
      double e = err_model(o, q, t) / pow(cutoff, t);
      if (e < best) {
        best = e;
        bnu = t;
      }
    }
    nu = bnu;
  }
  if (nu < 4 || nu > 10 || (nu & 1)) {
    free(o);
    return NULL;
  }
  o->nu = nu;
  o->a0 = cutoff;
  o->aCut[0] = cutoff;
  for (int l = 1; l <= o->L; l++) o->aCut[l] = 2.0 * o->aCut[l - 1];
  int nbar = 0;
  for (int k = 0; k < 3; k++) {
    int v = (int)ceil(o->aCut[o->L] * o->M[k] * row_norm(o->Ai, k));
    if (v > nbar) nbar = v;
  }
  o->relCutoff = nbar;
  o->nLim = (int)ceil(o->relCutoff - 1.);
  build_tau(o);
  build_Q(o);
  build_J(o);
  for (int k = 0; k < 3; k++) o->gd[o->L][k] = o->M[k];
  for (int l = o->L - 1; l >= 1; l--)
    for (int k = 0; k < 3; k++) o->gd[l][k] = 2 * o->gd[l + 1][k];
  int dmax = 2 * o->nLim + 1;
  for (int l = 1; l < o->L; l++)
    for (int k = 0; k < 3; k++)
      o->sd[l][k] = dmax < o->gd[l][k] ? dmax : o->gd[l][k];
  for (int k = 0; k < 3; k++) o->sd[o->L][k] = o->M[k];
  build_omegap(o);
  /* FF_rebuild uses column norms of Ai (code/forcefield0.c:618-620) */
  double as[3] = {col_norm(o->Ai, 0), col_norm(o->Ai, 1), col_norm(o->Ai, 2)};
  build_coeffs(o, as);
  for (int l = 1; l <= o->L; l++)
    o->khat[l] = calloc((size_t)o->sd[l][0] * o->sd[l][1] * o->sd[l][2],
                        sizeof(double));
  build_top(o);
  for (int l = o->L - 1; l >= 1; l--) build_level_stencil(o, l, as);
  return o;
}

void msmo_destroy(msmo *o) {
  if (!o) return;
  for (int l = 1; l <= o->L; l++) {
    free(o->khat[l]);
    for (int a = 0; a < 3; a++) free(o->omegap[l][a]);
  }
  for (int a = 0; a < 3; a++) free(o->cL[a]);
  free(o);
}

void msmo_params(const msmo *o, double *cutoff, int *nu, int *maxLevel,
                 int *topGridDim, int *nLim, double *detA) {
  if (cutoff) *cutoff = o->a0;
  if (nu) *nu = o->nu;
  if (maxLevel) *maxLevel = o->L;
  if (topGridDim)
    for (int k = 0; k < 3; k++) topGridDim[k] = o->M[k];
  if (nLim) *nLim = o->nLim;
  if (detA) *detA = o->detA;
}

void msmo_coeffs(const msmo *o, double *c1, double *c2) {
  *c1 = o->coeff1;
  *c2 = o->coeff2;
}

const double *msmo_khat(const msmo *o, int l, int *dims) {
  if (l < 1 || l > o->L) return NULL;
  for (int k = 0; k < 3; k++) dims[k] = o->sd[l][k];
  return o->khat[l];
}

const double *msmo_omegap(const msmo *o, int l, int a, int *len) {
  if (l < 1 || l > o->L || a < 0 || a > 2) return NULL;
  *len = o->opD[l][a];
  return o->omegap[l][a];
}

const double *msmo_cL(const msmo *o, int a) { return o->cL[a]; }

int msmo_grid_dims(const msmo *o, int l, int *dims) {
  if (l < 1 || l > o->L) return -1;
  for (int k = 0; k < 3; k++) dims[k] = o->gd[l][k];
  return 0;
}

/* ---- short-range part (code/forcefield1.c:240-321) ---------------------- */

/* Every (j != i, lattice image n) with |r_j + A n - r_i| < a0, found through a
 * periodic cell grid whose slabs are at least a0 thick. Returns
 * sum_i q_i phi_i / 2 and fills per-atom force and potential. */
static double short_range(const msmo *o, const double *q, const double *pos,
                          double *force, double *phi, long *npairs) {
  int N = o->N, nu = o->nu;
  double a0 = o->aCut[0], a02 = a0 * a0, a03 = a0 * a0 * a0;
  int nc[3], K[3];
  for (int k = 0; k < 3; k++) {
    double w = a0 * row_norm(o->Ai, k);
    nc[k] = (int)floor(1.0 / w);
    if (nc[k] < 1) nc[k] = 1;
    K[k] = (int)ceil(w * nc[k]);
  }
  int ncell = nc[0] * nc[1] * nc[2];
  int *head = malloc(sizeof(int) * ncell), *next = malloc(sizeof(int) * N);
  int (*cell)[3] = malloc(sizeof(int[3]) * N);
  int (*wrapn)[3] = malloc(sizeof(int[3]) * N);
  for (int c = 0; c < ncell; c++) head[c] = -1;
  for (int i = N - 1; i >= 0; i--) {
    const double *r = pos + 3 * i;
    int ci[3];
    for (int k = 0; k < 3; k++) {
      double s = o->Ai[k][0] * r[0] + o->Ai[k][1] * r[1] + o->Ai[k][2] * r[2];
      double f = floor(s);
      wrapn[i][k] = (int)f;
      ci[k] = (int)((s - f) * nc[k]);
      if (ci[k] >= nc[k]) ci[k] = nc[k] - 1;
      cell[i][k] = ci[k];
    }
    int c = (ci[0] * nc[1] + ci[1]) * nc[2] + ci[2];
    next[i] = head[c];
    head[c] = i;
  }
  double esum = 0.;
  long cnt = 0;
  for (int i = 0; i < N; i++) {
    const double *ri = pos + 3 * i;
    double fx = 0, fy = 0, fz = 0, ph = 0;
    for (int dx = -K[0]; dx <= K[0]; dx++)
      for (int dy = -K[1]; dy <= K[1]; dy++)
        for (int dz = -K[2]; dz <= K[2]; dz++) {
          int u[3] = {cell[i][0] + dx, cell[i][1] + dy, cell[i][2] + dz};
          int cw[3], img[3];
          for (int k = 0; k < 3; k++) {
            cw[k] = wrap(u[k], nc[k]);
            img[k] = (u[k] - cw[k]) / nc[k];
          }
          int c = (cw[0] * nc[1] + cw[1]) * nc[2] + cw[2];
          for (int j = head[c]; j >= 0; j = next[j]) {
            if (j == i) continue;
            const double *rj = pos + 3 * j;
            double n[3];
            for (int k = 0; k < 3; k++)
              n[k] = (double)(img[k] - wrapn[j][k] + wrapn[i][k]);
            double rx = rj[0] - ri[0] + o->A[0][0] * n[0] + o->A[0][1] * n[1] + o->A[0][2] * n[2];
            double ry = rj[1] - ri[1] + o->A[1][0] * n[0] + o->A[1][1] * n[1] + o->A[1][2] * n[2];
            double rz = rj[2] - ri[2] + o->A[2][0] * n[0] + o->A[2][1] * n[1] + o->A[2][2] * n[2];
            double r2 = rx * rx + ry * ry + rz * rz;
            if (r2 >= a02) continue;
            cnt++;
            double s = r2 / a02 - 1.;
            double ts = o->tau[nu - 1], t1 = 0.;
            for (int k = nu - 2; k >= 0; k--) {
              t1 = ts + s * t1;
              ts = o->tau[k] + s * ts;
            }
            double rinv = 1. / sqrt(r2);
            ph += q[j] * (rinv - ts / a0);
            double cf = q[j] * (-rinv * rinv * rinv - 2. * t1 / a03);
            fx += cf * rx;
            fy += cf * ry;
            fz += cf * rz;
          }
        }
    if (force) {
      force[3 * i] = q[i] * fx;
      force[3 * i + 1] = q[i] * fy;
      force[3 * i + 2] = q[i] * fz;
    }
    if (phi) phi[i] = ph;
    esum += q[i] * ph;
  }
  free(head);
  free(next);
  free(cell);
  free(wrapn);
  if (npairs) *npairs = cnt / 2;
  return 0.5 * esum;
}

double msmo_short_range(const msmo *o, const double *q, const double *pos,
                        double *force, double *phi) {
  return short_range(o, q, pos, force, phi, NULL);
}

long msmo_pair_count(const msmo *o, const double *pos) {
  double *q = malloc(sizeof(double) * o->N);
  for (int i = 0; i < o->N; i++) q[i] = 1.;
  long n = 0;
  short_range(o, q, pos, NULL, NULL, &n);
  free(q);
  return n;
}

/* ---- grid transfers ---------------------------------------------------- */

/* charges -> finest grid (code/forcefield1.c:324-398) */
void msmo_anterpolate(const msmo *o, const double *q, const double *pos,
                      double *grid) {
  int nu = o->nu, h = nu / 2;
  const int *g = o->gd[1];
  memset(grid, 0, sizeof(double) * g[0] * g[1] * g[2]);
  double w[3][10];
  for (int i = 0; i < o->N; i++) {
    const double *r = pos + 3 * i;
    int m[3];
    for (int k = 0; k < 3; k++) {
      double s = o->Ai[k][0] * r[0] + o->Ai[k][1] * r[1] + o->Ai[k][2] * r[2];
      s = s - floor(s);
      double u = (double)g[k] * s, f = floor(u);
      m[k] = (int)f;
      for (int n = -h; n < h; n++) w[k][n + h] = bspline(o, n + h, u - f, NULL);
    }
    for (int nx = -h; nx < h; nx++) {
      int gx = wrap(m[0] - nx, g[0]);
      for (int ny = -h; ny < h; ny++) {
        int gy = wrap(m[1] - ny, g[1]);
        double wxy = q[i] * w[0][nx + h] * w[1][ny + h];
        for (int nz = -h; nz < h; nz++) {
          int gz = wrap(m[2] - nz, g[2]);
          grid[(gx * g[1] + gy) * g[2] + gz] += wxy * w[2][nz + h];
        }
      }
    }
  }
}

/* q^{l+1}_m = sum_n J_n q^l_{2m+n} (code/forcefield1.c:401-477) */
void msmo_restrict(const msmo *o, int l, const double *ql, double *out) {
  const int *gf = o->gd[l], *gc = o->gd[l + 1];
  int h = o->nu / 2;
  for (int x = 0; x < gc[0]; x++)
    for (int y = 0; y < gc[1]; y++)
      for (int z = 0; z < gc[2]; z++) {
        double acc = 0.;
        for (int nx = -h; nx <= h; nx++) {
          int fx = wrap(2 * x + nx, gf[0]);
          for (int ny = -h; ny <= h; ny++) {
            int fy = wrap(2 * y + ny, gf[1]);
            double jxy = o->J[nx + h] * o->J[ny + h];
            for (int nz = -h; nz <= h; nz++) {
              int fz = wrap(2 * z + nz, gf[2]);
              acc += jxy * o->J[nz + h] * ql[(fx * gf[1] + fy) * gf[2] + fz];
            }
          }
        }
        out[(x * gc[1] + y) * gc[2] + z] = acc;
      }
}

/* e^l_{2m+n} += J_n e^{l+1}_m (code/forcefield1.c:530-567) */
void msmo_prolong_add(const msmo *o, int l, const double *ec, double *ef) {
  const int *gf = o->gd[l], *gc = o->gd[l + 1];
  int h = o->nu / 2;
  for (int x = 0; x < gc[0]; x++)
    for (int y = 0; y < gc[1]; y++)
      for (int z = 0; z < gc[2]; z++) {
        double v = ec[(x * gc[1] + y) * gc[2] + z];
        for (int nx = -h; nx <= h; nx++) {
          int fx = wrap(2 * x + nx, gf[0]);
          for (int ny = -h; ny <= h; ny++) {
            int fy = wrap(2 * y + ny, gf[1]);
            double jxy = o->J[nx + h] * o->J[ny + h] * v;
            for (int nz = -h; nz <= h; nz++) {
              int fz = wrap(2 * z + nz, gf[2]);
              ef[(fx * gf[1] + fy) * gf[2] + fz] += jxy * o->J[nz + h];
            }
          }
        }
      }
}

/* e^l_x += sum_d khat_l[d] q^l_{x+d}, d in [-sd/2, (sd-1)/2]^3
 * (code/forcefield0.c:898-931 over the halo of code/forcefield1.c:58-99) */
void msmo_stencil_add(const msmo *o, int l, const double *ql, double *el) {
  const int *g = o->gd[l], *s = o->sd[l];
  const double *kh = o->khat[l];
  for (int x = 0; x < g[0]; x++)
    for (int y = 0; y < g[1]; y++)
      for (int z = 0; z < g[2]; z++) {
        double acc = 0.;
        for (int i = 0; i < s[0]; i++) {
          int qx = wrap(x + i - s[0] / 2, g[0]);
          for (int j = 0; j < s[1]; j++) {
            int qy = wrap(y + j - s[1] / 2, g[1]);
            const double *krow = kh + (i * s[1] + j) * s[2];
            const double *qrow = ql + (qx * g[1] + qy) * g[2];
            for (int k = 0; k < s[2]; k++)
              acc += krow[k] * qrow[wrap(z + k - s[2] / 2, g[2])];
          }
        }
        el[(x * g[1] + y) * g[2] + z] += acc;
      }
}

/* e^L = IFFT(khat_L * FFT(q^L)) / M^3 (code/forcefield1.c:499-528) */
void msmo_top_solve(const msmo *o, const double *qL, double *eL) {
  const int *g = o->M;
  long n = (long)g[0] * g[1] * g[2];
  double complex *a = malloc(sizeof(double complex) * n);
  for (long i = 0; i < n; i++) a[i] = qL[i];
  msm_shim_fft3d(a, g[0], g[1], g[2], FFTW_FORWARD);
  for (long i = 0; i < n; i++) a[i] *= o->khat[o->L][i];
  msm_shim_fft3d(a, g[0], g[1], g[2], FFTW_BACKWARD);
  for (long i = 0; i < n; i++) eL[i] = creal(a[i]) / (double)n;
  free(a);
}

static long gsize(const msmo *o, int l) {
  return (long)o->gd[l][0] * o->gd[l][1] * o->gd[l][2];
}

/* Level chain of FF_energy (code/forcefield1.c:157-192). Weighted levels
 * scale each level's operator linearly: e^1 = sum_l w_l P^(l-1) K_l R^(l-1) q^1.
 * (The reference scales q[l] in place over only the first M_l^3 entries of
 * a padded array, code/forcefield1.c:169,184, so it defines no usable
 * non-unit weight semantics; unit weights agree exactly.) */
void msmo_grid_chain(const msmo *o, const double *q1, const double *weight,
                     double *e1) {
  int L = o->L;
  double *qs[MSMO_MAXL + 2] = {0}, *es[MSMO_MAXL + 2] = {0};
  qs[1] = (double *)q1;
  for (int l = 1; l < L; l++) {
    qs[l + 1] = malloc(sizeof(double) * gsize(o, l + 1));
    msmo_restrict(o, l, qs[l], qs[l + 1]);
  }
  double wL = weight ? weight[L] : 1.;
  double *qw = malloc(sizeof(double) * gsize(o, L));
  for (long i = 0; i < gsize(o, L); i++) qw[i] = wL * qs[L][i];
  es[L] = (L == 1) ? e1 : malloc(sizeof(double) * gsize(o, L));
  msmo_top_solve(o, qw, es[L]);
  free(qw);
  for (int l = L - 1; l >= 1; l--) {
    es[l] = (l == 1) ? e1 : malloc(sizeof(double) * gsize(o, l));
    memset(es[l], 0, sizeof(double) * gsize(o, l));
    msmo_prolong_add(o, l, es[l + 1], es[l]);
    double wl = weight ? weight[l] : 1.;
    double *tmp = calloc(gsize(o, l), sizeof(double));
    msmo_stencil_add(o, l, qs[l], tmp);
    for (long i = 0; i < gsize(o, l); i++) es[l][i] += wl * tmp[i];
    free(tmp);
    free(es[l + 1]);
    es[l + 1] = NULL;
  }
  for (int l = 2; l <= L; l++) free(qs[l]);
}

/* field and potential at the atoms (code/forcefield1.c:570-607) */
void msmo_interpolate(const msmo *o, const double *pos, const double *e1,
                      double *efield, double *phi_long) {
  int nu = o->nu, h = nu / 2;
  const int *g = o->gd[1];
  double w[3][10], d[3][10];
  for (int i = 0; i < o->N; i++) {
    const double *r = pos + 3 * i;
    int m[3];
    for (int k = 0; k < 3; k++) {
      double s = o->Ai[k][0] * r[0] + o->Ai[k][1] * r[1] + o->Ai[k][2] * r[2];
      double u = (double)g[k] * s, f = floor(u);
      m[k] = (int)f;
      for (int n = -h; n < h; n++)
        w[k][n + h] = bspline(o, n + h, u - f, &d[k][n + h]);
    }
    double ex = 0, ey = 0, ez = 0, ph = 0;
    for (int nx = -h; nx < h; nx++) {
      int gx = wrap(m[0] - nx, g[0]);
      for (int ny = -h; ny < h; ny++) {
        int gy = wrap(m[1] - ny, g[1]);
        for (int nz = -h; nz < h; nz++) {
          int gz = wrap(m[2] - nz, g[2]);
          double e = e1[(gx * g[1] + gy) * g[2] + gz];
          double wx = w[0][nx + h], wy = w[1][ny + h], wz = w[2][nz + h];
          ex -= d[0][nx + h] * wy * wz * e;
          ey -= wx * d[1][ny + h] * wz * e;
          ez -= wx * wy * d[2][nz + h] * e;
          ph += wx * wy * wz * e;
        }
      }
    }
    ex *= g[0];
    ey *= g[1];
    ez *= g[2];
    if (efield) { /* E = Ai^T E_grid */
      efield[3 * i] = o->Ai[0][0] * ex + o->Ai[1][0] * ey + o->Ai[2][0] * ez;
      efield[3 * i + 1] = o->Ai[0][1] * ex + o->Ai[1][1] * ey + o->Ai[2][1] * ez;
      efield[3 * i + 2] = o->Ai[0][2] * ex + o->Ai[1][2] * ey + o->Ai[2][2] * ez;
    }
    if (phi_long) phi_long[i] = ph;
  }
}

/* ---- full evaluation (code/forcefield1.c:101-235) ----------------------- */
double msmo_energy(const msmo *o, const double *q, const double *pos,
                   const double *weight, double *force, double *phi) {
  int N = o->N, nu = o->nu;
  double w0 = weight ? weight[0] : 1.;
  double qsum = 0., q2sum = 0.;
  for (int i = 0; i < N; i++) {
    qsum += q[i];
    q2sum += q[i] * q[i];
  }
  double gam0 = horner(o->tau, nu, -1.);
  double a0 = o->aCut[0];
  double u_const = 0.5 * q2sum * o->coeff1 - 0.5 * qsum * qsum * o->coeff2 -
                   0.5 * q2sum * gam0 / a0;
  double *phis = malloc(sizeof(double) * N);
  double u_short = short_range(o, q, pos, force, phis, NULL);
  long ng = gsize(o, 1);
  double *q1 = malloc(sizeof(double) * ng), *e1 = malloc(sizeof(double) * ng);
  msmo_anterpolate(o, q, pos, q1);
  msmo_grid_chain(o, q1, weight, e1);
  double ug = 0.;
  for (long i = 0; i < ng; i++) ug += q1[i] * e1[i];
  double *ef = malloc(sizeof(double) * 3 * N), *phil = malloc(sizeof(double) * N);
  msmo_interpolate(o, pos, e1, ef, phil);
  for (int i = 0; i < N; i++) {
    if (force)
      for (int k = 0; k < 3; k++)
        force[3 * i + k] = w0 * force[3 * i + k] + q[i] * ef[3 * i + k];
    if (phi)
      phi[i] = w0 * (q[i] * o->coeff1 - qsum * o->coeff2 - q[i] * gam0 / a0 +
                     phis[i]) +
               phil[i];
  }
  free(phis);
  free(q1);
  free(e1);
  free(ef);
  free(phil);
  return w0 * (u_const + u_short) + 0.5 * ug;
}
