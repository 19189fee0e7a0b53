// Adjoint of the evaluation (no counterpart in the reference, which has no
// derivatives beyond forces). For L = Ubar U + sum_m Fbar_m . F_m at the
// current positions and charges, with p_m = q_m Fbar_m, F_m = q_m E_m:
//   dL/dq_k = Ubar phi_k + Fbar_k . E_k - psi_k,
//       psi_k = sum_j p_j . grad v(r_j - r_k) + B_k . (K d),  d = sum_m p_m . grad B_m
//   dL/dr_k = -Ubar F_k + q_k sum_j q_j H(r_kj) (Fbar_j - Fbar_k)
//             - q_k [ (grad grad (B_k . e1)) Fbar_k + grad (B_k . K d) ]
// with v the softened short-range kernel, H its Hessian, B_k the B-spline
// weights of atom k on the finest grid, e1 = K q1 the forward's finest-grid
// potential and K the grid operator (restriction, level stencils, top solve,
// prolongation). The dipole grid d runs through the same K as the charges.
// Here: the short-range terms (one thread per atom over the neighbour-cell
// list), the dipoles in grid units, and the final combine in FP64.
#include "kernels.h"

namespace msm {
namespace {

constexpr int kThreads = 128;

inline int blocks_for(long n) { return (int)std::max<long>(1, (n + kThreads - 1) / kThreads); }

// Fbar in pair-cell order: fbs[k] = (Fbar of atom pperm[k], 0)
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_adj_gather(int N, const int *__restrict__ perm, const double *__restrict__ fbar,
             V4<T> *__restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  const int i = perm[k];
  V4<T> v;
  v.x = (T)fbar[3 * i];
  v.y = (T)fbar[3 * i + 1];
  v.z = (T)fbar[3 * i + 2];
  v.w = T(0);
  out[k] = v;
}

// dipoles p_i = q_i Fbar_i in grid units, p^_a = M_a (A^-1 p)_a, grid-cell order
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_adj_dipoles(int N, const int *__restrict__ perm, const double *__restrict__ q,
              const double *__restrict__ fbar, Geometry g, V4<T> *__restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  const int i = perm[k];
  const double p[3] = {q[i] * fbar[3 * i], q[i] * fbar[3 * i + 1], q[i] * fbar[3 * i + 2]};
  double d[3];
  for (int a = 0; a < 3; ++a)
    d[a] = g.M1[a] * (g.Ai[3 * a] * p[0] + g.Ai[3 * a + 1] * p[1] + g.Ai[3 * a + 2] * p[2]);
  V4<T> v;
  v.x = (T)d[0];
  v.y = (T)d[1];
  v.z = (T)d[2];
  v.w = T(0);
  out[k] = v;
}

// Short-range part, per atom k (pair-cell order), d = r_j - r_k:
//   E_k = sum_j q_j g1 d,  psi_k = sum_j g1 (p_j . d),
//   h_k = sum_j q_j [g1 (Fbar_j - Fbar_k) + g2 d (d . (Fbar_j - Fbar_k))]
// with grad v = g1 d, H = g1 I + g2 d d^T,
//   g1 = -1/r^3 - (2/a0^3) tau'(s),  g2 = 3/r^5 - (4/a0^5) tau''(s),
//   s = r^2/a0^2 - 1. out_a = (E, psi), out_b = (h, 0). Partial sums per
// neighbour cell in T, accumulated in FP64.
template <typename T, int NU>
__global__ void __launch_bounds__(kThreads)
k_adj_pair(int N, const V4<T> *__restrict__ ps, const V4<T> *__restrict__ fbs,
           const int *__restrict__ pcs, const int *__restrict__ start, int nc0, int nc1,
           int nc2, const CellOffset<T> *__restrict__ off, int noff, PairConsts<T> pc,
           V4<T> *__restrict__ out_a, V4<T> *__restrict__ out_b) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  const V4<T> ai = ps[k];
  const V4<T> fk = fbs[k];
  const int c = pcs[k];
  const int cz = c % nc2, cy = (c / nc2) % nc1, cx = c / (nc1 * nc2);
  const T c2 = T(2) * pc.two_inv_a03 * pc.inv_a02;  // 4/a0^5
  double ex = 0, ey = 0, ez = 0, ps_ = 0, hx = 0, hy = 0, hz = 0;
  for (int o = 0; o < noff; ++o) {
    const CellOffset<T> co = off[o];
    const int ux = pwrap(cx + co.d[0], nc0), uy = pwrap(cy + co.d[1], nc1),
              uz = pwrap(cz + co.d[2], nc2);
    const int cw = (ux * nc1 + uy) * nc2 + uz;
    const int b = start[cw], e = start[cw + 1];
    const T sx = co.shift[0] - ai.x, sy = co.shift[1] - ai.y, sz = co.shift[2] - ai.z;
    T pex = 0, pey = 0, pez = 0, pp = 0, phx = 0, phy = 0, phz = 0;
    for (int j = b; j < e; ++j) {
      const V4<T> aj = ps[j];
      const T dx = aj.x + sx, dy = aj.y + sy, dz = aj.z + sz;
      const T r2 = dx * dx + dy * dy + dz * dz;
      if (r2 < pc.a02 && j != k) {  // never the atom itself, at any image
        const T s = r2 * pc.inv_a02 - T(1);
        T p0 = pc.tau[NU - 1], p1 = T(0), p2 = T(0);
#pragma unroll
        for (int m = NU - 2; m >= 0; --m) {
          p2 = p1 + s * p2;
          p1 = p0 + s * p1;
          p0 = pc.tau[m] + s * p0;
        }
        // p1 = tau'(s), 2 p2 = tau''(s)
        const T rinv = rsqrt_t<T>(r2);
        const T rinv2 = rinv * rinv, rinv3 = rinv2 * rinv;
        const T g1 = -rinv3 - p1 * pc.two_inv_a03;
        const T g2 = T(3) * rinv3 * rinv2 - T(2) * p2 * c2;
        const V4<T> fj = fbs[j];
        const T qj = aj.w;
        pex += qj * g1 * dx;
        pey += qj * g1 * dy;
        pez += qj * g1 * dz;
        pp += qj * g1 * (fj.x * dx + fj.y * dy + fj.z * dz);
        const T Dx = fj.x - fk.x, Dy = fj.y - fk.y, Dz = fj.z - fk.z;
        const T dd = g2 * (dx * Dx + dy * Dy + dz * Dz);
        phx += qj * (g1 * Dx + dd * dx);
        phy += qj * (g1 * Dy + dd * dy);
        phz += qj * (g1 * Dz + dd * dz);
      }
    }
    ex += pex;
    ey += pey;
    ez += pez;
    ps_ += pp;
    hx += phx;
    hy += phy;
    hz += phz;
  }
  V4<T> a, bb;
  a.x = (T)ex;
  a.y = (T)ey;
  a.z = (T)ez;
  a.w = (T)ps_;
  bb.x = (T)hx;
  bb.y = (T)hy;
  bb.z = (T)hz;
  bb.w = T(0);
  out_a[k] = a;
  out_b[k] = bb;
}

template <typename T>
__global__ void __launch_bounds__(kThreads)
k_adj_combine(AdjointCombineArgs a, const int *__restrict__ pinv, const int *__restrict__ ginv,
              const V4<T> *__restrict__ pout, const V4<T> *__restrict__ gout,
              const V4<T> *__restrict__ adj_a, const V4<T> *__restrict__ adj_b,
              const V4<T> *__restrict__ adj_g, const V4<T> *__restrict__ adj_h) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.N) return;
  const double qi = a.q[i], Q = a.qstats[0];
  const V4<T> ps = pout[pinv[i]], gs = gout[ginv[i]];
  const V4<T> A = adj_a[pinv[i]], B = adj_b[pinv[i]];
  const V4<T> G = adj_g[ginv[i]], H = adj_h[ginv[i]];
  const double phi = a.w0 * (qi * a.coeff1 - Q * a.coeff2 - qi * a.gamma0_over_a0 +
                             (double)ps.w) + (double)gs.w;
  const double E[3] = {a.w0 * (double)A.x + (double)gs.x, a.w0 * (double)A.y + (double)gs.y,
                       a.w0 * (double)A.z + (double)gs.z};
  const double F[3] = {a.w0 * (double)ps.x + qi * (double)gs.x,
                       a.w0 * (double)ps.y + qi * (double)gs.y,
                       a.w0 * (double)ps.z + qi * (double)gs.z};
  const double fb[3] = {a.fbar[3 * i], a.fbar[3 * i + 1], a.fbar[3 * i + 2]};
  if (a.dq)
    a.dq[i] = a.ubar * phi + (fb[0] * E[0] + fb[1] * E[1] + fb[2] * E[2]) -
              (a.w0 * (double)A.w + (double)G.w);
  if (a.dr) {
    const double h[3] = {(double)B.x, (double)B.y, (double)B.z};
    const double g[3] = {(double)G.x + (double)H.x, (double)G.y + (double)H.y,
                         (double)G.z + (double)H.z};
    for (int c = 0; c < 3; ++c) a.dr[3 * i + c] = -a.ubar * F[c] + qi * (a.w0 * h[c] - g[c]);
  }
}

}  // namespace

template <typename T>
void launch_adj_gather(cudaStream_t s, int N, const int *perm, const double *fbar, V4<T> *out) {
  k_adj_gather<T><<<blocks_for(N), kThreads, 0, s>>>(N, perm, fbar, out);
}

template <typename T>
void launch_adj_dipoles(cudaStream_t s, int N, const int *perm, const double *q,
                        const double *fbar, const Geometry &g, V4<T> *out) {
  k_adj_dipoles<T><<<blocks_for(N), kThreads, 0, s>>>(N, perm, q, fbar, g, out);
}

template <typename T>
void launch_adj_pair(cudaStream_t s, int N, const V4<T> *ps, const V4<T> *fbs, const int *pcs,
                     const int *start, const Geometry &g, const CellOffset<T> *off, int noff,
                     const PairConsts<T> &pc, V4<T> *out_a, V4<T> *out_b) {
#define MSM_ADJ_PAIR(NUV)                                                              \
  k_adj_pair<T, NUV><<<blocks_for(N), kThreads, 0, s>>>(N, ps, fbs, pcs, start, g.nc[0], \
                                                        g.nc[1], g.nc[2], off, noff, pc, \
                                                        out_a, out_b)
  switch (pc.nu) {
    case 4: MSM_ADJ_PAIR(4); break;
    case 6: MSM_ADJ_PAIR(6); break;
    case 8: MSM_ADJ_PAIR(8); break;
    default: MSM_ADJ_PAIR(10); break;
  }
#undef MSM_ADJ_PAIR
}

template <typename T>
void launch_adj_combine(cudaStream_t s, const AdjointCombineArgs &a, const int *pinv,
                        const int *ginv, const V4<T> *pout, const V4<T> *gout,
                        const V4<T> *adj_a, const V4<T> *adj_b, const V4<T> *adj_g,
                        const V4<T> *adj_h) {
  k_adj_combine<T><<<blocks_for(a.N), kThreads, 0, s>>>(a, pinv, ginv, pout, gout, adj_a,
                                                         adj_b, adj_g, adj_h);
}

#define MSM_INST_ADJ(T)                                                                    \
  template void launch_adj_gather<T>(cudaStream_t, int, const int *, const double *,      \
                                     V4<T> *);                                             \
  template void launch_adj_dipoles<T>(cudaStream_t, int, const int *, const double *,     \
                                      const double *, const Geometry &, V4<T> *);          \
  template void launch_adj_pair<T>(cudaStream_t, int, const V4<T> *, const V4<T> *,       \
                                   const int *, const int *, const Geometry &,             \
                                   const CellOffset<T> *, int, const PairConsts<T> &,      \
                                   V4<T> *, V4<T> *);                                      \
  template void launch_adj_combine<T>(cudaStream_t, const AdjointCombineArgs &,           \
                                      const int *, const int *, const V4<T> *,             \
                                      const V4<T> *, const V4<T> *, const V4<T> *,         \
                                      const V4<T> *, const V4<T> *);
MSM_INST_ADJ(float)
MSM_INST_ADJ(double)

}  // namespace msm
