// Level stencils on the GPU for a new box (the device form of
// make_level_stencil in setup.cpp, code/forcefield0.c:965-1081): grid sizes,
// order and cutoff are kept, so only the taps change. Everything in FP64, in
// stream order, no host synchronisation:
//   kappa_l(s) = sum over images of g_{a_l/2} - g_{a_l} at the stencil
//   offsets s = (i - S0/2) / M0, ...;  then khat_l = omega'_x (x) omega'_y
//   (x) omega'_z applied to kappa_l (three separable passes, z, y, x);
// then the taps are packed into the sweep layouts (padded rows; folded rows
// for mirror-symmetric stencils).
#include "kernels.h"

namespace msm {
namespace {

constexpr int kThreads = 256;

inline int blocks_for(long n) { return (int)std::max<long>(1, (n + kThreads - 1) / kThreads); }

// offset d reduced to the centred range [-n/2, n - n/2)
__device__ __forceinline__ int centred(int d, int n) {
  int r = (d + n / 2) % n;
  if (r < 0) r += n;
  return r - n / 2;
}

__device__ __forceinline__ double dpoly(const double *c, int n, double s) {
  double v = c[n - 1];
  for (int k = n - 2; k >= 0; --k) v = c[k] + s * v;
  return v;
}

__global__ void __launch_bounds__(kThreads) k_kappa(LevelStencilArgs a, double *__restrict__ kap) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int n1 = a.sd[1], n2 = a.sd[2];
  if (idx >= (long)a.sd[0] * n1 * n2) return;
  const int k = idx % n2, j = (idx / n2) % n1, i = idx / ((long)n1 * n2);
  const double s[3] = {(double)(i - a.sd[0] / 2) / a.g[0], (double)(j - n1 / 2) / a.g[1],
                       (double)(k - n2 / 2) / a.g[2]};
  double lo[3], hi[3];
  for (int q = 0; q < 3; ++q) {
    lo[q] = floor(s[q] - a.al * a.as[q] + 1.);
    hi[q] = ceil(s[q] + a.al * a.as[q] - 1.);
  }
  double acc = 0.;
  for (double px = lo[0]; px <= hi[0]; ++px)
    for (double py = lo[1]; py <= hi[1]; ++py)
      for (double pz = lo[2]; pz <= hi[2]; ++pz) {
        const double d[3] = {s[0] - px, s[1] - py, s[2] - pz};
        double r2 = 0;
        for (int q = 0; q < 3; ++q) {
          const double rq = a.A[3 * q] * d[0] + a.A[3 * q + 1] * d[1] + a.A[3 * q + 2] * d[2];
          r2 += rq * rq;
        }
        const double rho = sqrt(r2) / a.al;
        if (rho >= 1.) continue;
        const double g1 = dpoly(a.tau, a.nu, rho * rho - 1.) / a.al;
        const double rho2 = 2. * rho;
        const double g2 = rho2 >= 1. ? 1. / rho2 : dpoly(a.tau, a.nu, rho2 * rho2 - 1.);
        acc += g2 * (2. / a.al) - g1;
      }
  kap[idx] = acc;
}

// out = omega' applied along axis ax (grid size g on that axis)
__global__ void __launch_bounds__(kThreads)
k_omega_axis(int n0, int n1, int n2, int ax, int g, const double *__restrict__ om,
             const double *__restrict__ in, double *__restrict__ out) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)n0 * n1 * n2) return;
  const int k = idx % n2, j = (idx / n2) % n1, i = idx / ((long)n1 * n2);
  const int len = ax == 0 ? n0 : (ax == 1 ? n1 : n2);
  const int pos = ax == 0 ? i : (ax == 1 ? j : k);
  const long stride = ax == 0 ? (long)n1 * n2 : (ax == 1 ? n2 : 1);
  const long base = idx - pos * stride;
  double acc = 0;
  for (int q = 0; q < len; ++q) acc += om[abs(centred(q - pos, g))] * in[base + q * stride];
  out[idx] = acc;
}

// padded rows (zeros past S2) and, when kf is given, the folded rows
// kf[i][c1-d][k] = mean of kh[c0+-i][c1+-d][k] (i <= c0, d <= c1)
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_pack_taps(int S0, int S1, int S2, int SP, const double *__restrict__ kh, T *__restrict__ kp,
            T *__restrict__ kf) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)S0 * S1 * SP) return;
  const int k = idx % SP, j = (idx / SP) % S1, i = idx / ((long)S1 * SP);
  auto at = [&](int a, int b) { return kh[((long)a * S1 + b) * S2 + k]; };
  kp[idx] = k < S2 ? (T)at(i, j) : T(0);
  const int c0 = S0 / 2, c1 = S1 / 2;
  if (kf && i <= c0 && j <= c1) {
    const int d = j;
    T v = T(0);
    if (k < S2)
      v = (T)(0.25 * (at(c0 + i, c1 + d) + at(c0 - i, c1 + d) + at(c0 + i, c1 - d) +
                      at(c0 - i, c1 - d)));
    kf[((long)i * (c1 + 1) + (c1 - d)) * SP + k] = v;
  }
}

}  // namespace

template <typename T>
void launch_level_stencil(cudaStream_t s, const LevelStencilArgs &a, const double *om,
                          double *work, T *kp, T *kf, bool fp64) {
  const long n = (long)a.sd[0] * a.sd[1] * a.sd[2];
  const int OMS = a.oms;
  double *kap = work, *f = work + n, *h = work + 2 * n;
  k_kappa<<<blocks_for(n), kThreads, 0, s>>>(a, kap);
  k_omega_axis<<<blocks_for(n), kThreads, 0, s>>>(a.sd[0], a.sd[1], a.sd[2], 2, a.g[2],
                                                  om + 2 * OMS, kap, f);
  k_omega_axis<<<blocks_for(n), kThreads, 0, s>>>(a.sd[0], a.sd[1], a.sd[2], 1, a.g[1],
                                                  om + OMS, f, h);
  k_omega_axis<<<blocks_for(n), kThreads, 0, s>>>(a.sd[0], a.sd[1], a.sd[2], 0, a.g[0], om,
                                                  h, kap);
  const int SP = stencil_tap_pitch(a.sd[2], fp64);
  const long np = (long)a.sd[0] * a.sd[1] * SP;
  k_pack_taps<T><<<blocks_for(np), kThreads, 0, s>>>(a.sd[0], a.sd[1], a.sd[2], SP, kap, kp,
                                                     kf);
}

template void launch_level_stencil<float>(cudaStream_t, const LevelStencilArgs &,
                                          const double *, double *, float *, float *, bool);
template void launch_level_stencil<double>(cudaStream_t, const LevelStencilArgs &,
                                           const double *, double *, double *, double *,
                                           bool);

}  // namespace msm
