// Host-side (FP64) setup of the MSM evaluation: parameters, coefficient
// tables and per-level stencils that the device kernels consume.
#pragma once

#include <vector>

namespace msm {

constexpr int kMaxLevels = 10;  // FF's time_* arrays hold 10 levels

struct Params {
  int N = 0;
  double A[3][3] = {}, Ai[3][3] = {}, detA = 0;
  double estErr = 1e-3;
  int nu = 0, L = 0;
  int top[3] = {0, 0, 0};
  double a0 = 0;
  double aCut[kMaxLevels + 2] = {};
  double relCutoff = 0;
  int nLim = 0;
  bool fft = true;
};

// Method of a table set: B-spline MSM, or smooth PME (code/pme0.c, pme1.c),
// which the engine evaluates as a one-level plan with the direct-space
// kernel erfc(beta r)/r and the PME influence function as top multiplier.
constexpr int kKindMsm = 0, kKindPme = 1;

struct Tables {
  int kind = kKindMsm;
  double beta = 0;           // PME Ewald splitting parameter
  Params p;
  double tau[16] = {};       // softening polynomial, degree nu-1
  double Q[5 * 10] = {};     // B-spline pieces: Q[j*nu+k] = [t^k] Q_nu(j+t)
  double J[11] = {};         // two-scale stencil J[n + nu/2]
  double gamma0 = 0;         // tau(-1) = gamma(0)
  double coeff1 = 0, coeff2 = 0;
  int grid[kMaxLevels + 2][3] = {};   // level-l grid dims
  int sten[kMaxLevels + 2][3] = {};   // level-l stencil dims (l < L)
  std::vector<double> omegap[kMaxLevels + 2][3];
  std::vector<double> cL[3];
  std::vector<double> khat[kMaxLevels + 2];  // l<L: stencil; L: multiplier
};

// Matrix helpers (reference code/forcefield0.c:709-724)
double invert3(const double a[3][3], double ai[3][3]);

// B-spline pieces Q[j*nu+k] = [t^k] Q_nu(j+t), j < nu/2
void bspline_pieces(int nu, double *Q);

// Smooth-PME comparator (code/pme0.c, code/pme1.c): host setup of a
// one-level table set (kind kKindPme) for the engine.
namespace pme {
struct Settings {  // the FF_set_* values; <= 0 means the reference default
  double cutoff = 0, tolDir = 0;
  int nu = 0;
  int M[3] = {0, 0, 0};
};
// Parameters as FF_build (code/pme0.c:192-260): defaults, beta from
// erfc(beta a0)/a0 = tolDir, grid from the spacing table. Returns false (and
// MSMPB_ERR_UNSUPPORTED in *err) where the reference prints and exits: no
// default grid for this order or cutoff.
bool select(Params &p, double *beta, double *tolDir, int N, const double edges[3][3],
            const Settings &s, int *err);
// Every table of a parameter set (code/pme0.c:262-322, :365-412, :444-503)
void build_tables(Tables &t, const Params &p, double beta);
// FF_get_errEst (code/pme0.c:333-361)
double err_est(const Params &p, const double *q);
}  // namespace pme

// Parameter selection exactly as FF_build (code/forcefield0.c:271-367).
// Arguments use the reference's -1 = auto convention. Returns false when the
// parameters are unusable (error code in *err).
bool select_params(Params &p, int N, const double *q, const double edges[3][3],
                   double cutoff, int nu, int L, const int top[3],
                   double estErr, bool fft, int *err);

// Error model (code/forcefield0.c:521-587)
double err_model(const Params &p, const double *q, int nu);
// the same from a precomputed sum of q_i^2
double err_model_q2(const Params &p, double Q2, int nu);
double delta_f(const Params &p, const double *q);

// Quasi-interpolation weights omega'_l and c_L only (code/forcefield0.c:726-767);
// needs t.p, t.Q and t.grid.
void build_omegap_tables(Tables &t);

// All tables for a parameter set (code/forcefield0.c:369-467, :598-675).
void build_tables(Tables &t, const Params &p);
// New box, same grid sizes and order: refreshes the box-dependent constants
// and the top-level multiplier; the level stencils t.khat[1..L-1] are left
// as they are (the device computes its own).
void rebuild_box_tables(Tables &t, const Params &p);

}  // namespace msm
