// Radial pair functions of the short-range sums: V(r) and f(r) = V'(r) / r,
// so that the pair adds q_j V to the potential of i and q_j f (r_j - r_i) to
// its field.
//
//  NU = 4..10  MSM softened kernel (code/forcefield1.c:290-305):
//              V = 1/r - tau(r^2/a0^2 - 1)/a0,  f = -1/r^3 - 2 tau'(s)/a0^3
//  NU = 0      PME direct-space kernel (code/pme1.c:165-170):
//              V = erfc(beta r)/r,  f = -(V + 2 beta/sqrt(pi) exp(-beta^2 r^2)) / r^2
#pragma once

#include "kernels.h"

namespace msm {

template <typename T> __device__ __forceinline__ T erfc_t(T x);
template <> __device__ __forceinline__ float erfc_t<float>(float x) { return erfcf(x); }
template <> __device__ __forceinline__ double erfc_t<double>(double x) { return erfc(x); }
template <typename T> __device__ __forceinline__ T exp_t(T x);
template <> __device__ __forceinline__ float exp_t<float>(float x) { return expf(x); }
template <> __device__ __forceinline__ double exp_t<double>(double x) { return exp(x); }

// In the evaluation precision T
template <typename T, int NU>
__device__ __forceinline__ void pair_radial(const PairConsts<T> &pc, T r2, T &v, T &f) {
  if constexpr (NU == 0) {
    const T rinv = rsqrt_t<T>(r2);
    v = erfc_t<T>(pc.beta * (r2 * rinv)) * rinv;
    f = -(v + pc.c_exp * exp_t<T>(-pc.beta2 * r2)) * (rinv * rinv);
  } else {
    const T s = r2 * pc.inv_a02 - T(1);
    T ts = pc.tau[NU - 1], t1 = T(0);
#pragma unroll
    for (int m = NU - 2; m >= 0; --m) {
      t1 = ts + s * t1;
      ts = pc.tau[m] + s * ts;
    }
    const T rinv = rsqrt_t<T>(r2);
    v = rinv - ts * pc.inv_a0;
    f = -rinv * rinv * rinv - t1 * pc.two_inv_a03;
  }
}

// In FP64 from the FP64 copies of the constants (close pairs of the mixed
// form, where the displacement is formed in FP64)
template <int NU, typename T>
__device__ __forceinline__ void pair_radial64(const PairConsts<T> &pc, double d2, double &v,
                                              double &f) {
  if constexpr (NU == 0) {
    const double rinv = 1.0 / sqrt(d2);
    v = erfc(pc.betad * (d2 * rinv)) * rinv;
    f = -(v + pc.c_expd * exp(-pc.beta2d * d2)) * (rinv * rinv);
  } else {
    const double sd = d2 * pc.inv_a02d - 1.0;
    double ts = pc.taud[NU - 1], t1 = 0.0;
#pragma unroll
    for (int m = NU - 2; m >= 0; --m) {
      t1 = ts + sd * t1;
      ts = pc.taud[m] + sd * ts;
    }
    const double rinv = 1.0 / sqrt(d2);
    v = rinv - ts * pc.inv_a0d;
    f = -rinv * rinv * rinv - t1 * pc.two_inv_a03d;
  }
}

// PME kernel on two pairs at once in packed FP32 (the mixed form's tile
// loop): erfc(z), z = beta r >= 0, by the Chebyshev-fitted form of Numerical
// Recipes (Press et al., 2nd ed., sec. 6.2, "erfcc"; fractional error below
// 1.2e-7 for all z >= 0),
//   erfc(z) = t exp(-z^2) exp(P(t)),  t = 1 / (1 + z/2),
// so that exp(-z^2), which the force term needs as well, is computed once.
// Returns V = erfc(z)/r and f = -(V + 2 beta/sqrt(pi) exp(-z^2)) / r^2.
__device__ __forceinline__ void pme_radial2(const PairConsts<float> &pc, float2 r2,
                                            float2 &v, float2 &f) {
  const float2 rinv = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
  const float2 z = __fmul2_rn(__fmul2_rn(r2, rinv), make_float2(pc.beta, pc.beta));
  const float2 d = __ffma2_rn(z, make_float2(0.5f, 0.5f), make_float2(1.f, 1.f));
  const float2 t = make_float2(__fdividef(1.f, d.x), __fdividef(1.f, d.y));
  constexpr float c[10] = {-1.26551223f, 1.00002368f, 0.37409196f, 0.09678418f,
                           -0.18628806f, 0.27886807f, -1.13520398f, 1.48851587f,
                           -0.82215223f, 0.17087277f};
  float2 p = make_float2(c[9], c[9]);
#pragma unroll
  for (int k = 8; k >= 0; --k) p = __ffma2_rn(p, t, make_float2(c[k], c[k]));
  const float2 mz2 = __fmul2_rn(r2, make_float2(-pc.beta2, -pc.beta2));
  const float2 ez2 = make_float2(__expf(mz2.x), __expf(mz2.y));
  const float2 g = make_float2(__expf(p.x), __expf(p.y));
  v = __fmul2_rn(__fmul2_rn(__fmul2_rn(t, ez2), g), rinv);
  const float2 s = __ffma2_rn(make_float2(pc.c_exp, pc.c_exp), ez2, v);
  f = __fmul2_rn(s, __fmul2_rn(rinv, make_float2(-rinv.x, -rinv.y)));
}

}  // namespace msm
