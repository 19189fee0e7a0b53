// Host-side FP64 setup: parameter selection, softening and B-spline tables,
// quasi-interpolation weights, per-level real-space stencils and the
// top-level Fourier multiplier. Runs once per FF_build / FF_rebuild; its
// outputs are uploaded to the device (FP32 or FP64) by the engine.
#include <algorithm>
#include <cmath>
#include <cstdint>

#include "msm_host.h"
#include "msmpb_b200.h"

namespace msm {
namespace {

constexpr double kPi = 3.14159265358979323846264338327950288;

double norm_row(const double m[3][3], int r) {
  return std::sqrt(m[r][0] * m[r][0] + m[r][1] * m[r][1] + m[r][2] * m[r][2]);
}
double norm_col(const double m[3][3], int c) {
  return std::sqrt(m[0][c] * m[0][c] + m[1][c] * m[1][c] + m[2][c] * m[2][c]);
}

// polynomial sum_k c[k] s^k, evaluated from the top coefficient down
double poly(const double *c, int n, double s) {
  double v = c[n - 1];
  for (int k = n - 2; k >= 0; --k) v = c[k] + s * v;
  return v;
}

// Smallest m' >= m with no prime factor above 7 (code/forcefield0.c:219-245)
int fft_friendly(int m) {
  for (;; ++m) {
    int r = m;
    for (int f : {2, 3, 5, 7})
      while (r > 1 && r % f == 0) r /= f;
    if (r <= 1) return m;
  }
}

// Auto grid size for level count L (code/forcefield0.c:247-269)
void auto_top_grid(const Params &p, int L, int out[3]) {
  double eta = p.fft ? (L >= 2 ? 0.83 : 5.7) : 1.0;
  double a[3] = {norm_row(p.A, 0), norm_row(p.A, 1), norm_row(p.A, 2)};
  double vol = std::pow(a[0] * a[1] * a[2], -1. / 3.);
  double base = std::pow(2., 1. - L) * std::pow(eta * p.N, 1. / 3.);
  for (int k = 0; k < 3; ++k) out[k] = (int)std::ceil(base * a[k] * vol);
}

int64_t choose(int n, int k) {
  if (k < 0 || k > n) return 0;
  int64_t r = 1;
  for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
  return r;
}

// offset d reduced to the centred range [-n/2, n - n/2)
int centred_offset(int d, int n) {
  int r = (d + n / 2) % n;
  if (r < 0) r += n;
  return r - n / 2;
}

}  // namespace

void bspline_pieces(int nu, double *Q) {
  double fact = 1;
  for (int i = 2; i < nu; ++i) fact *= i;
  for (int j = 0; j < nu / 2; ++j)
    for (int k = 0; k < nu; ++k) {
      int64_t s = 0;
      for (int i = 0; i <= j; ++i) {
        int64_t pw = 1;
        for (int e = 0; e < nu - 1 - k; ++e) pw *= (j - i);
        s += ((i & 1) ? -1 : 1) * choose(nu, i) * pw;
      }
      Q[j * nu + k] = (double)(choose(nu - 1, k) * s) / fact;
    }
}

double invert3(const double a[3][3], double ai[3][3]) {
  double c[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      c[i][j] = a[(j + 1) % 3][(i + 1) % 3] * a[(j + 2) % 3][(i + 2) % 3] -
                a[(j + 2) % 3][(i + 1) % 3] * a[(j + 1) % 3][(i + 2) % 3];
  double det = a[0][0] * c[0][0] + a[0][1] * c[1][0] + a[0][2] * c[2][0];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) ai[i][j] = c[i][j] / det;
  return std::fabs(det);
}

double err_model(const Params &p, const double *q, int nu) {
  double Q2 = 0;
  for (int i = 0; i < p.N; ++i) Q2 += q[i] * q[i];
  return err_model_q2(p, Q2, nu);
}

double err_model_q2(const Params &p, double Q2, int nu) {
  int M1[3] = {p.top[0], p.top[1], p.top[2]};
  for (int l = 1; l < p.L; ++l)
    for (int &m : M1) m *= 2;
  double Fref = (Q2 / (double)p.N) / std::pow(p.detA / (double)p.N, 5. / 6.);
  double h1 = std::max({norm_row(p.A, 0) / M1[0], norm_row(p.A, 1) / M1[1],
                        norm_row(p.A, 2) / M1[2]});
  double dF = Q2 * (1 - std::pow(4.0, -p.L)) * std::pow(h1, nu - 1) *
              std::pow(p.detA, -1. / 3.) * std::pow(p.N, -2.0 / 3.0);
  return dF / Fref;
}

double delta_f(const Params &p, const double *q) {
  // fitted constants C_{nu-1} of the force-error estimate
  // (code/forcefield0.c:531)
  static const double C[4] = {0.825169, 5.16701, 73.6508, 1977.23};
  int M1[3] = {p.top[0], p.top[1], p.top[2]};
  for (int l = 1; l < p.L; ++l)
    for (int &m : M1) m *= 2;
  double Q2 = 0;
  for (int i = 0; i < p.N; ++i) Q2 += q[i] * q[i];
  double h1 = std::max({norm_row(p.A, 0) / M1[0], norm_row(p.A, 1) / M1[1],
                        norm_row(p.A, 2) / M1[2]});
  return C[(p.nu - 4) / 2] * Q2 * (1 - std::pow(4.0, -p.L)) *
         std::pow(h1, p.nu - 1) * std::pow(p.detA, -1. / 3.) *
         std::pow(p.N, -2.0 / 3.0) / std::pow(p.a0, p.nu);
}

bool select_params(Params &p, int N, const double *q, const double edges[3][3],
                   double cutoff, int nu, int L, const int top[3],
                   double estErr, bool fft, int *err) {
  *err = MSMPB_OK;
  p = Params();
  p.N = N;
  p.fft = fft;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) p.A[i][j] = edges[i][j];
  p.detA = invert3(p.A, p.Ai);
  if (!(p.detA > 0) || !std::isfinite(p.detA)) {
    *err = MSMPB_ERR_ARGUMENT;
    return false;
  }
  p.estErr = (estErr == -1) ? 0.001 : estErr;
  p.L = (L == -1) ? 1 : L;
  bool have_top = top[0] != -1;
  if (have_top)
    for (int k = 0; k < 3; ++k) p.top[k] = top[k];
  if (!fft && !have_top) {  // code/forcefield0.c:292-307
    int l = 1, m[3];
    for (; l <= kMaxLevels; ++l) {
      auto_top_grid(p, l, m);
      if (m[0] * m[1] * m[2] <= std::sqrt((double)N)) break;
    }
    p.L = l;
    for (int k = 0; k < 3; ++k) p.top[k] = m[k];
  }
  if (fft && !have_top) auto_top_grid(p, p.L, p.top);
  if (fft)
    for (int &m : p.top) m = fft_friendly(m);
  if (p.L < 1 || p.L > kMaxLevels || p.top[0] < 1 || p.top[1] < 1 ||
      p.top[2] < 1) {
    *err = MSMPB_ERR_UNSUPPORTED;
    return false;
  }
  if (cutoff == -1) {  // code/forcefield0.c:320-334
    if (nu == -1) {
      double best = INFINITY;
      for (int t = 4; t <= 10; t += 2)
        best = std::min(best, std::pow(err_model(p, q, t) / p.estErr, 1. / t));
      cutoff = best;
    } else {
      cutoff = std::pow(err_model(p, q, nu) / p.estErr, 1. / nu);
    }
  }
  if (nu == -1) {  // code/forcefield0.c:337-348
    double best = INFINITY;
    nu = 4;
    for (int t = 4; t <= 10; t += 2) {
      double e = err_model(p, q, t) / std::pow(cutoff, t);
      if (e < best) {
        best = e;
        nu = t;
      }
    }
  }
  if (nu < 4 || nu > 10 || (nu & 1)) {
    *err = MSMPB_ERR_UNSUPPORTED;
    return false;
  }
  if (!(cutoff > 0) || !std::isfinite(cutoff)) {
    *err = MSMPB_ERR_ARGUMENT;
    return false;
  }
  p.nu = nu;
  p.a0 = cutoff;
  p.aCut[0] = cutoff;
  for (int l = 1; l <= p.L; ++l) p.aCut[l] = 2.0 * p.aCut[l - 1];
  int nbar = 0;  // code/forcefield0.c:360-367 (row norms of Ai)
  for (int k = 0; k < 3; ++k)
    nbar = std::max(nbar, (int)std::ceil(p.aCut[p.L] * p.top[k] * norm_row(p.Ai, k)));
  p.relCutoff = nbar;
  p.nLim = (int)std::ceil(p.relCutoff - 1.);
  return true;
}

namespace {

// tau_k: Taylor coefficients of (1+s)^(-1/2) (code/forcefield0.c:369-373)
void make_tau(Tables &t) {
  t.tau[0] = 1.;
  for (int i = 1; i < t.p.nu; ++i) t.tau[i] = -(1. - 0.5 / i) * t.tau[i - 1];
  t.gamma0 = poly(t.tau, t.p.nu, -1.);
}

// B-spline pieces from the truncated-power representation
//   Q_nu(x) = 1/(nu-1)! * sum_i (-1)^i C(nu,i) (x-i)_+^(nu-1)
// (same table as code/forcefield0.c:375-406, derived in closed form)
void make_bspline(Tables &t) {
  const int nu = t.p.nu;
  bspline_pieces(nu, t.Q);
  for (int n = 0; n <= nu; ++n) t.J[n] = (double)choose(nu, n) * std::pow(2., 1 - nu);
}

// omega'_m and c_L (code/forcefield0.c:726-767)
void make_omegap(Tables &t) {
  const Params &p = t.p;
  const int nu = p.nu, h = nu / 2;
  double phi[8] = {};  // centred B-spline at the integers 0..h-1
  for (int n = 1; n < h; ++n) phi[n] = t.Q[(h - n) * nu];
  for (int k = 0; k < nu; ++k) phi[0] += t.Q[(h - 1) * nu + k];
  const int oplim = 2 * p.nLim;
  for (int l = p.L; l >= 1; --l)
    for (int a = 0; a < 3; ++a) {
      const int m = t.grid[l][a];
      std::vector<double> c(m);
      for (int k = 0; k < m; ++k) {
        double th = 2. * kPi * k / m, v = phi[0];
        for (int n = 1; n < h; ++n) v += 2. * phi[n] * std::cos(n * th);
        c[k] = 1. / (v * v);
      }
      int len = (m / 2 > oplim) ? oplim + 1 : m / 2 + 1;
      std::vector<double> om(len);
      for (int j = 0; j < len; ++j) {
        double v = c[0];
        for (int k = 1; k <= (m - 1) / 2; ++k)
          v += 2. * c[k] * std::cos(2. * kPi * (double)(k * j) / m);
        if (m % 2 == 0) v += c[m / 2] * std::cos(kPi * j);
        om[j] = v / m;
      }
      t.omegap[l][a] = std::move(om);
      if (l == p.L) t.cL[a] = std::move(c);
    }
}

// constant energy terms (code/forcefield0.c:612-643)
void make_constants(Tables &t, const double as[3]) {
  const Params &p = t.p;
  const double a0 = p.a0;
  int lim[3];
  for (int k = 0; k < 3; ++k) lim[k] = (int)std::ceil(a0 * as[k] - 1.);
  double c1 = 0.;
  for (int x = -lim[0]; x <= lim[0]; ++x)
    for (int y = -lim[1]; y <= lim[1]; ++y)
      for (int z = -lim[2]; z <= lim[2]; ++z) {
        if (x == 0 && y == 0 && z == 0) continue;
        double r[3];
        for (int k = 0; k < 3; ++k) r[k] = p.A[k][0] * x + p.A[k][1] * y + p.A[k][2] * z;
        double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
        if (r2 >= a0 * a0) continue;
        if (r2 != 0.) c1 += 1. / std::sqrt(r2);
        c1 -= poly(t.tau, p.nu, r2 / (a0 * a0) - 1.) / a0;
      }
  t.coeff1 = c1;
  t.coeff2 = kPi * p.aCut[p.L] * p.aCut[p.L] / ((4 * p.nu + 2) * p.detA);
}

// level-l kernel kappa_l(A s) = sum over images of g_{a_l/2} - g_{a_l}
// (code/forcefield0.c:1041-1081)
double kappa(const Tables &t, int l, const double s[3], const double as[3]) {
  const Params &p = t.p;
  const double al = p.aCut[l];
  double lo[3], hi[3];
  for (int k = 0; k < 3; ++k) {
    lo[k] = std::floor(s[k] - al * as[k] + 1.);
    hi[k] = std::ceil(s[k] + al * as[k] - 1.);
  }
  double acc = 0.;
  for (double px = lo[0]; px <= hi[0]; ++px)
    for (double py = lo[1]; py <= hi[1]; ++py)
      for (double pz = lo[2]; pz <= hi[2]; ++pz) {
        const double d[3] = {s[0] - px, s[1] - py, s[2] - pz};
        double r2 = 0;
        for (int k = 0; k < 3; ++k) {
          double rk = p.A[k][0] * d[0] + p.A[k][1] * d[1] + p.A[k][2] * d[2];
          r2 += rk * rk;
        }
        double rho = std::sqrt(r2) / al;
        if (rho >= 1.) continue;
        double g1 = poly(t.tau, p.nu, rho * rho - 1.) / al;
        double rho2 = 2. * rho;
        double g2 = rho2 >= 1. ? 1. / rho2 : poly(t.tau, p.nu, rho2 * rho2 - 1.);
        acc += g2 * (2. / al) - g1;
      }
  return acc;
}

// khat_l = omega' (x) omega' (x) omega' applied to kappa_l samples
// (code/forcefield0.c:965-1039)
void make_level_stencil(Tables &t, int l, const double as[3]) {
  const int *g = t.grid[l], *sd = t.sten[l];
  const int nx = sd[0], ny = sd[1], nz = sd[2];
  const size_t n = (size_t)nx * ny * nz;
  std::vector<double> kap(n), f(n), h(n);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        double s[3] = {(double)(i - nx / 2) / g[0], (double)(j - ny / 2) / g[1],
                       (double)(k - nz / 2) / g[2]};
        kap[((size_t)i * ny + j) * nz + k] = kappa(t, l, s, as);
      }
  const auto &ox = t.omegap[l][0], &oy = t.omegap[l][1], &oz = t.omegap[l][2];
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k1 = 0; k1 < nz; ++k1) {
        double acc = 0;
        for (int k0 = 0; k0 < nz; ++k0)
          acc += oz[std::abs(centred_offset(k0 - k1, g[2]))] * kap[((size_t)i * ny + j) * nz + k0];
        f[((size_t)i * ny + j) * nz + k1] = acc;
      }
  for (int i = 0; i < nx; ++i)
    for (int j1 = 0; j1 < ny; ++j1)
      for (int k = 0; k < nz; ++k) {
        double acc = 0;
        for (int j0 = 0; j0 < ny; ++j0)
          acc += oy[std::abs(centred_offset(j0 - j1, g[1]))] * f[((size_t)i * ny + j0) * nz + k];
        h[((size_t)i * ny + j1) * nz + k] = acc;
      }
  std::vector<double> &kh = t.khat[l];
  kh.assign(n, 0.);
  for (int i1 = 0; i1 < nx; ++i1)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        double acc = 0;
        for (int i0 = 0; i0 < nx; ++i0)
          acc += ox[std::abs(centred_offset(i0 - i1, g[0]))] * h[((size_t)i0 * ny + j) * nz + k];
        kh[((size_t)i1 * ny + j) * nz + k] = acc;
      }
}

// Top level: psi(k) = (2nu-1)!! pi aL^2/detA * j_{nu-1}(t)/t^(nu+1),
// t = pi |A^-T k| aL, times c_L(kx) c_L(ky) c_L(kz) M^3
// (code/forcefield0.c:769-896). For t <= pi the Taylor series of
// j_{nu-1}(t)/t^(nu-1) (7 terms) is used; above it the closed form with the
// Rayleigh numerator polynomials (Abramowitz & Stegun 10.1.8).
void make_top(Tables &t) {
  const Params &p = t.p;
  const int nu = p.nu, n = nu - 1, m = (n - 1) / 2;
  double S[8] = {}, Cc[8] = {};
  const double sg = (m & 1) ? -1. : 1.;
  for (int k = 0; 2 * k <= n; ++k) {
    long double v = 1.L;
    for (int i = n - 2 * k + 1; i <= n + 2 * k; ++i) v *= i;
    for (int i = 2; i <= 2 * k; ++i) v /= i;
    v /= std::pow(2.L, 2 * k);
    Cc[(n - 1 - 2 * k) / 2] = sg * ((k & 1) ? -1. : 1.) * (double)v;
  }
  for (int k = 0; 2 * k + 1 <= n; ++k) {
    long double v = 1.L;
    for (int i = n - 2 * k; i <= n + 2 * k + 1; ++i) v *= i;
    for (int i = 2; i <= 2 * k + 1; ++i) v /= i;
    v /= std::pow(2.L, 2 * k + 1);
    S[(n - 2 * k - 1) / 2] = sg * ((k & 1) ? -1. : 1.) * (double)v;
  }
  double tc[7];
  __int128 tv = 1;
  for (int i = 1; i <= 2 * nu - 1; i += 2) tv *= i;
  tc[0] = (double)tv;
  for (int i = 1; i < 7; ++i) {
    tv = -tv * (2 * i) * (2 * nu - 1 + 2 * i);
    tc[i] = (double)tv;
  }
  double dfact = 1;
  for (int i = 1; i <= 2 * nu - 1; i += 2) dfact *= i;
  const double aL = p.aCut[p.L];
  const double scale = dfact * kPi * aL * aL / p.detA;
  const int *g = p.top;
  std::vector<double> &kh = t.khat[p.L];
  kh.assign((size_t)g[0] * g[1] * g[2], 0.);
  for (int x = 0; x < g[0]; ++x)
    for (int y = 0; y < g[1]; ++y)
      for (int z = 0; z < g[2]; ++z) {
        int c[3] = {x < (g[0] + 1) / 2 ? x : x - g[0], y < (g[1] + 1) / 2 ? y : y - g[1],
                    z < (g[2] + 1) / 2 ? z : z - g[2]};
        double k2 = 0;
        for (int a = 0; a < 3; ++a) {
          double ka = p.Ai[0][a] * c[0] + p.Ai[1][a] * c[1] + p.Ai[2][a] * c[2];
          k2 += ka * ka;
        }
        double psi = 0;
        if (k2 != 0) {
          double tt = kPi * std::sqrt(k2) * aL, t2 = tt * tt;
          if (tt <= kPi) {
            double acc = 0, tp = 1;
            for (int i = 0; i < 7; ++i) {
              acc += tp / tc[i];
              tp *= t2;
            }
            psi = acc / t2;
          } else {
            double sp = 0, cp = 0, tp = 1;
            for (int k = 0; k < nu / 2; ++k) {
              sp += S[k] * tp;
              cp += Cc[k] * tp;
              tp *= t2;
            }
            psi = (sp * (std::sin(tt) / tt) - cp * std::cos(tt)) / std::pow(tt, 2.0 * nu);
          }
          psi *= scale;
        }
        kh[((size_t)x * g[1] + y) * g[2] + z] =
            psi * t.cL[0][x] * t.cL[1][y] * t.cL[2][z] * g[0] * g[1] * g[2];
      }
}

}  // namespace

void build_omegap_tables(Tables &t) { make_omegap(t); }

void build_tables(Tables &t, const Params &p) {
  t = Tables();
  t.p = p;
  make_tau(t);
  make_bspline(t);
  for (int k = 0; k < 3; ++k) t.grid[p.L][k] = p.top[k];
  for (int l = p.L - 1; l >= 1; --l)
    for (int k = 0; k < 3; ++k) t.grid[l][k] = 2 * t.grid[l + 1][k];
  const int dmax = 2 * p.nLim + 1;
  for (int l = 1; l < p.L; ++l)
    for (int k = 0; k < 3; ++k) t.sten[l][k] = std::min(dmax, t.grid[l][k]);
  for (int k = 0; k < 3; ++k) t.sten[p.L][k] = p.top[k];
  make_omegap(t);
  // FF_rebuild takes column norms of Ai (code/forcefield0.c:618-620)
  const double as[3] = {norm_col(p.Ai, 0), norm_col(p.Ai, 1), norm_col(p.Ai, 2)};
  make_constants(t, as);
  make_top(t);
  for (int l = p.L - 1; l >= 1; --l) make_level_stencil(t, l, as);
}

void rebuild_box_tables(Tables &t, const Params &p) {
  t.p = p;
  const double as[3] = {norm_col(p.Ai, 0), norm_col(p.Ai, 1), norm_col(p.Ai, 2)};
  make_constants(t, as);
  make_top(t);
}

}  // namespace msm
