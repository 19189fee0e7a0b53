// Per-level grid-to-grid direct stencil (code/forcefield0.c:898-931):
//   e^l_x += w_l * sum_{d in [0,S)^3} khat_l[d] q^l_{x + d - S/2}  (periodic)
// The periodic wrap is materialised once per level as a padded copy
// P[a][b][c] = q[(a - S0/2) mod M0][(b - S1/2) mod M1][(c - S2/2) mod M2]
// (the reference pads the same way, code/forcefield1.c:58-99), so the sweep
// itself reads a dense box with no index arithmetic modulo M.
#include <algorithm>

#include "kernels.h"

namespace msm {
namespace {

constexpr int kThreads = 256;

template <typename T>
__global__ void __launch_bounds__(kThreads)
k_pad(StencilShape sh, const T *__restrict__ q, T *__restrict__ p) {
  long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long n = (long)sh.P[0] * sh.P[1] * sh.P[2];
  if (idx >= n) return;
  const int c = idx % sh.P[2], b = (idx / sh.P[2]) % sh.P[1],
            a = idx / ((long)sh.P[1] * sh.P[2]);
  const int x = pwrap(a - sh.S[0] / 2, sh.M[0]);
  const int y = pwrap(b - sh.S[1] / 2, sh.M[1]);
  const int z = pwrap(c - sh.S[2] / 2, sh.M[2]);
  p[idx] = q[((long)x * sh.M[1] + y) * sh.M[2] + z];
}

// Reference-form sweep: one output per thread, all loops at run time.
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_stencil_simple(StencilShape sh, const T *__restrict__ p,
                 const T *__restrict__ kh, T w, T *__restrict__ e) {
  long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long n = (long)sh.M[0] * sh.M[1] * sh.M[2];
  if (idx >= n) return;
  const int z = idx % sh.M[2], y = (idx / sh.M[2]) % sh.M[1],
            x = idx / ((long)sh.M[1] * sh.M[2]);
  Acc<T> acc;
  acc.zero();
  for (int i = 0; i < sh.S[0]; ++i) {
    T pl = 0;
    for (int j = 0; j < sh.S[1]; ++j) {
      const T *row = p + ((long)(x + i) * sh.P[1] + (y + j)) * sh.P[2] + z;
      const T *kr = kh + ((long)i * sh.S[1] + j) * sh.S[2];
      T r = 0;
      for (int k = 0; k < sh.S[2]; ++k) r += kr[k] * row[k];
      pl += r;
    }
    acc.add(pl);
  }
  e[idx] += w * acc.value();
}

inline int blocks_for(long n) {
  return (int)std::max<long>(1, (n + kThreads - 1) / kThreads);
}

}  // namespace

int stencil_padded_z(int Mz, int Sz) {
  int pz = Mz + Sz - 1;
  return (pz + 3) / 4 * 4;  // 16-byte rows for FP32 tiles
}

template <typename T>
void launch_pad(cudaStream_t s, const StencilShape &sh, const T *q, T *p) {
  long n = (long)sh.P[0] * sh.P[1] * sh.P[2];
  k_pad<T><<<blocks_for(n), kThreads, 0, s>>>(sh, q, p);
}

template <typename T>
void launch_stencil(cudaStream_t s, const StencilShape &sh, const T *p,
                    const T *kh, T w, T *e, int variant) {
  (void)variant;
  long n = (long)sh.M[0] * sh.M[1] * sh.M[2];
  k_stencil_simple<T><<<blocks_for(n), kThreads, 0, s>>>(sh, p, kh, w, e);
}

template void launch_pad<float>(cudaStream_t, const StencilShape &,
                                const float *, float *);
template void launch_pad<double>(cudaStream_t, const StencilShape &,
                                 const double *, double *);
template void launch_stencil<float>(cudaStream_t, const StencilShape &,
                                    const float *, const float *, float,
                                    float *, int);
template void launch_stencil<double>(cudaStream_t, const StencilShape &,
                                     const double *, const double *, double,
                                     double *, int);

}  // namespace msm
