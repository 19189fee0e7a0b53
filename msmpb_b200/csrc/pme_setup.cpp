// Host-side FP64 setup of the smooth-PME comparator (code/pme0.c): the
// Ewald splitting parameter, the default grid, the B-spline deconvolution
// factors, the Fourier multiplier of the reciprocal part and the constant
// energy terms. The evaluation itself is the engine's one-level plan with
// the erfc kernel (Tables::kind = kKindPme).
#include <cmath>

#include "msm_host.h"
#include "msmpb_b200.h"

namespace msm {
namespace pme {
namespace {

constexpr double kPi = 3.14159265358979323846264338327950288;

double row_norm(const double m[3][3], int r) {
  return std::sqrt(m[r][0] * m[r][0] + m[r][1] * m[r][1] + m[r][2] * m[r][2]);
}
double col_norm(const double m[3][3], int c) {
  return std::sqrt(m[0][c] * m[0][c] + m[1][c] * m[1][c] + m[2][c] * m[2][c]);
}

// b with erfc(b) = c: Newton from 0 while the residual shrinks
// (code/pme0.c:207-222)
double erfc_root(double c) {
  double b = 0., res = std::erfc(b) - c, prev = 2. * res;
  while (std::fabs(res) < std::fabs(prev)) {
    b += res / (2. / std::sqrt(kPi) * std::exp(-b * b));
    prev = res;
    res = std::erfc(b) - c;
  }
  return b;
}

// Q_nu(i + t) from the pieces (mirror image for i >= nu/2)
double bspline_at(const double *Q, int nu, int i, double t) {
  if (i >= nu / 2) {
    i = nu - 1 - i;
    t = 1. - t;
  }
  const double *c = Q + i * nu;
  double v = c[nu - 1];
  for (int k = nu - 2; k >= 0; --k) v = c[k] + t * v;
  return v;
}

// c_a(k) = |sum_n Q_nu(nu/2 + n) e^{2 pi i k n / M_a}|^-2, k = 0..M_a/2
// (code/pme0.c:444-471)
void make_cL(Tables &t) {
  const int nu = t.p.nu, h = nu / 2;
  double phi[8];
  for (int n = 0; n < h; ++n) phi[n] = bspline_at(t.Q, nu, h + n, 0.);
  for (int a = 0; a < 3; ++a) {
    const int M = t.p.top[a];
    t.cL[a].assign(M / 2 + 1, 0.);
    for (int k = 0; k <= M / 2; ++k) {
      double s = phi[0];
      for (int n = 1; n < h; ++n) s += 2. * phi[n] * std::cos(2. * kPi * k * n / M);
      t.cL[a][k] = 1. / (s * s);
    }
  }
}

// coeff1: the atom's own images within a0 plus its self term; coeff2 the
// neutralising-background term (code/pme0.c:377-399)
void make_constants(Tables &t, double beta) {
  const Params &p = t.p;
  int lim[3];
  for (int k = 0; k < 3; ++k) lim[k] = (int)std::ceil(p.a0 * col_norm(p.Ai, k) - 1.);
  double c1 = 0.;
  for (int x = -lim[0]; x <= lim[0]; ++x)
    for (int y = -lim[1]; y <= lim[1]; ++y)
      for (int z = -lim[2]; z <= lim[2]; ++z) {
        double r2 = 0.;
        for (int k = 0; k < 3; ++k) {
          const double rk = p.A[k][0] * x + p.A[k][1] * y + p.A[k][2] * z;
          r2 += rk * rk;
        }
        if (r2 >= p.a0 * p.a0) continue;
        if (r2 != 0.)
          c1 += std::erfc(beta * std::sqrt(r2)) / std::sqrt(r2);
        else
          c1 -= 2. * beta / std::sqrt(kPi);
      }
  t.coeff1 = c1;
  t.coeff2 = kPi / (beta * beta * p.detA);
  t.gamma0 = 0.;
}

// Fourier multiplier exp(-pi^2 K^2 / beta^2) / (pi detA K^2) c_x c_y c_z M^3
// at K = Ai^T k, k the centred index; zero at K = 0 (code/pme0.c:473-503).
// Computed from zero at every call.
void make_multiplier(Tables &t, double beta) {
  const Params &p = t.p;
  const int *M = p.top;
  const size_t n = (size_t)M[0] * M[1] * M[2];
  std::vector<double> &kh = t.khat[1];
  kh.assign(n, 0.);
  for (int i = 0; i < M[0]; ++i)
    for (int j = 0; j < M[1]; ++j)
      for (int l = 0; l < M[2]; ++l) {
        const int k[3] = {(i + M[0] / 2) % M[0] - M[0] / 2, (j + M[1] / 2) % M[1] - M[1] / 2,
                          (l + M[2] / 2) % M[2] - M[2] / 2};
        double K2 = 0.;
        for (int a = 0; a < 3; ++a) {
          const double Ka = p.Ai[0][a] * k[0] + p.Ai[1][a] * k[1] + p.Ai[2][a] * k[2];
          K2 += Ka * Ka;
        }
        if (K2 == 0.) continue;
        const double c = t.cL[0][std::abs(k[0])] * t.cL[1][std::abs(k[1])] *
                         t.cL[2][std::abs(k[2])];
        kh[((size_t)i * M[1] + j) * M[2] + l] =
            std::exp(-kPi * kPi * K2 / (beta * beta)) / (kPi * p.detA * K2) * c * (double)n;
      }
}

}  // namespace

bool select(Params &p, double *beta, double *tolDir, int N, const double edges[3][3],
            const Settings &s, int *err) {
  p = Params{};
  p.N = N;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) p.A[i][j] = edges[i][j];
  p.detA = invert3(p.A, p.Ai);
  if (N <= 0 || !(p.detA > 0)) {
    *err = MSMPB_ERR_ARGUMENT;
    return false;
  }
  p.a0 = s.cutoff > 0 ? s.cutoff : 8.;
  p.nu = s.nu > 0 ? s.nu : 6;
  *tolDir = s.tolDir > 0 ? s.tolDir : 1e-5;
  if (p.nu < 4 || p.nu > 10 || p.nu % 2) {
    *err = MSMPB_ERR_UNSUPPORTED;
    return false;
  }
  *beta = erfc_root(*tolDir * p.a0) / p.a0;
  if (s.M[0] > 0) {
    for (int k = 0; k < 3; ++k) p.top[k] = s.M[k];
  } else {
    // default spacing for tolDir_ref = 1e-5 h*, orders 4 and 6, cutoffs
    // 6..10 A in steps of 0.5 (code/pme0.c:224-260)
    static const double href[2][9] = {{0.70, 0.77, 0.83, 0.91, 1.00, 1.11, 1.21, 1.33, 1.48},
                                      {1.05, 1.18, 1.29, 1.43, 1.54, 1.67, 1.82, 2.00, 2.22}};
    const int i = (p.nu - 4) / 2, j = (int)std::lround((p.a0 - 6.) / 0.5);
    if (i > 1 || j < 0 || j > 8) {
      *err = MSMPB_ERR_UNSUPPORTED;
      return false;
    }
    const double hstar = std::pow(p.detA / N, 1. / 3.);
    const double tol_ref = 1e-5 * hstar;
    const double beta_ref = erfc_root(tol_ref * p.a0 / hstar) / p.a0;
    const double h = std::pow(*tolDir / tol_ref, 1. / p.nu) * (beta_ref / *beta) * href[i][j];
    for (int k = 0; k < 3; ++k) p.top[k] = (int)std::ceil(row_norm(p.A, k) / h);
  }
  for (int k = 0; k < 3; ++k)
    if (p.top[k] < 1) {
      *err = MSMPB_ERR_ARGUMENT;
      return false;
    }
  p.L = 1;
  p.aCut[0] = p.a0;
  p.aCut[1] = 2. * p.a0;
  p.fft = true;
  return true;
}

void build_tables(Tables &t, const Params &p, double beta) {
  t.kind = kKindPme;
  t.beta = beta;
  t.p = p;
  bspline_pieces(p.nu, t.Q);
  for (int k = 0; k < 3; ++k) t.grid[1][k] = p.top[k];
  make_cL(t);
  make_constants(t, beta);
  make_multiplier(t, beta);
}

double err_est(const Params &p, const double *q) {
  if (p.nu > 10) return NAN;
  static const double Mc[4] = {9., 825., 130095., 34096545.};
  static const double cbar[4] = {1. / 6., 1. / 30., 1. / 140., 1. / 630.};
  static const double kc[4] = {0.39189561, 0.150829428, 0.049632967, 0.013520855};
  const int id = (p.nu - 4) / 2;
  const double C = 4. / 3. * Mc[id] * cbar[id] * kc[id];
  double Ai[3][3];
  const double det = invert3(p.A, Ai);
  double hmin = INFINITY;
  for (int k = 0; k < 3; ++k) hmin = std::fmin(hmin, 1. / (row_norm(Ai, k) * p.top[k]));
  double Q2 = 0.;
  for (int i = 0; i < p.N; ++i) Q2 += q[i] * q[i];
  return Q2 * C * std::pow(hmin, p.nu - 2) /
         (std::pow(det, 1. / 3.) * std::sqrt((double)p.N) * std::pow(p.a0, p.nu - 1));
}

}  // namespace pme
}  // namespace msm
