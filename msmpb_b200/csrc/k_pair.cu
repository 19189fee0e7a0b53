// Short-range softened pair sum (code/forcefield1.c:240-321 over the
// neighbour list of code/forcefield0.c:21-164), rebuilt on the GPU each call.
//
// Atoms are sorted by pair cell (cells at least a0/2 thick). Each atom i
// sweeps a host-built list of neighbour-cell instances: a cell offset d and
// the Cartesian offset of that cell's origin relative to i's home-cell origin,
// periodic image included. Positions are stored relative to their own cell
// origin, so r_j - r_i = (rel_j + shift_d) - rel_i is formed from small
// numbers and stays accurate in FP32. Every (j != i, image) with r < a0 is
// summed, each unordered pair once from each side (gather form: no atomics,
// per-atom potential and force fall out directly).
//
// V(r) = 1/r - tau(r^2/a0^2 - 1)/a0,  F_i = q_i q_j (-1/r^3 - 2 tau'(s)/a0^3) r.
//
// Mixed form: FP32 arithmetic with compensated (Kahan) accumulation across
// neighbour cells, except pairs closer than sqrt(close2) (2.5 A): their
// displacement is formed from FP64 cell-relative positions and FP64 cell
// offsets and the pair is summed in FP64. Those pairs carry the largest
// forces, and an FP32 coordinate rounds by up to 2.4e-7 A, which is a
// relative error of 2.4e-7 on a 1 A bond; everywhere else the FP32 result
// is within rounding of the FP64 one.
#include "kernels.h"
#include "pair_fn.cuh"

namespace msm {
namespace {

constexpr int kPairThreads = 128;

template <typename T, int NU, bool COMPENSATE, bool CLOSE>
__device__ __forceinline__ void pair_body(const BlockCtx &ctx, int N, const V4<T> *__restrict__ ps, const V4<double> *__restrict__ ps64,
       const int *__restrict__ pcs, const int *__restrict__ start, int nc0,
       int nc1, int nc2, const CellOffset<T> *__restrict__ off, int noff,
       PairConsts<T> pc, V4<T> *__restrict__ out) {
  int k = ctx.b.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  const V4<T> ai = ps[k];
  V4<double> ai64;
  if (CLOSE) ai64 = ps64[k];
  double cfx = 0., cfy = 0., cfz = 0., cph = 0.;  // close pairs (FP64)
  // close pairs found during the sweep, evaluated in FP64 after it
  constexpr int kCloseList = 12;
  int close_j[CLOSE ? kCloseList : 1], close_o[CLOSE ? kCloseList : 1];
  int nclose = 0;
  const int c = pcs[k];
  const int cz = c % nc2, cy = (c / nc2) % nc1, cx = c / (nc1 * nc2);
  Acc<T> fx, fy, fz, ph;
  fx.zero();
  fy.zero();
  fz.zero();
  ph.zero();
  for (int o = 0; o < noff; ++o) {
    const CellOffset<T> co = off[o];
    const int ux = pwrap(cx + co.d[0], nc0), uy = pwrap(cy + co.d[1], nc1),
              uz = pwrap(cz + co.d[2], nc2);
    const int cw = (ux * nc1 + uy) * nc2 + uz;
    const int b = start[cw], e = start[cw + 1];
    const T sx = co.shift[0] - ai.x, sy = co.shift[1] - ai.y,
            sz = co.shift[2] - ai.z;
    T px = 0, py = 0, pz = 0, pp = 0;
    for (int j = b; j < e; ++j) {
      const V4<T> aj = ps[j];
      const T dx = aj.x + sx, dy = aj.y + sy, dz = aj.z + sz;
      const T r2 = dx * dx + dy * dy + dz * dz;
      // the atom itself is skipped at every image: the reference pairs no
      // atom with itself and sums its own images in the constant coeff1
      if (r2 < pc.a02 && j != k) {
        if (CLOSE && r2 < pc.close2 && nclose < kCloseList) {
          close_j[nclose] = j;
          close_o[nclose] = o;
          ++nclose;
          continue;
        }
        if (CLOSE && r2 < pc.close2) {  // list full: evaluate now
          const V4<double> aj = ps64[j];
          const double ex = (aj.x + co.shift64[0]) - ai64.x;
          const double ey = (aj.y + co.shift64[1]) - ai64.y;
          const double ez = (aj.z + co.shift64[2]) - ai64.z;
          const double d2 = ex * ex + ey * ey + ez * ez;
          double v, f;
          pair_radial64<NU>(pc, d2, v, f);
          cph += aj.w * v;
          const double cf = aj.w * f;
          cfx += cf * ex;
          cfy += cf * ey;
          cfz += cf * ez;
          continue;
        }
        T v, f;
        pair_radial<T, NU>(pc, r2, v, f);
        pp += aj.w * v;
        const T cf = aj.w * f;
        px += cf * dx;
        py += cf * dy;
        pz += cf * dz;
      }
    }
    if (COMPENSATE) {
      fx.add(px);
      fy.add(py);
      fz.add(pz);
      ph.add(pp);
    } else {
      fx.s += px;
      fy.s += py;
      fz.s += pz;
      ph.s += pp;
    }
  }
  if constexpr (CLOSE) {
    for (int t = 0; t < nclose; ++t) {
      const int j = close_j[t];
      const CellOffset<T> &co = off[close_o[t]];
      const V4<double> aj = ps64[j];
      const double ex = (aj.x + co.shift64[0]) - ai64.x;
      const double ey = (aj.y + co.shift64[1]) - ai64.y;
      const double ez = (aj.z + co.shift64[2]) - ai64.z;
      const double d2 = ex * ex + ey * ey + ez * ez;
      double v, f;
      pair_radial64<NU>(pc, d2, v, f);
      cph += aj.w * v;
      const double cf = aj.w * f;
      cfx += cf * ex;
      cfy += cf * ey;
      cfz += cf * ez;
    }
  }
  V4<T> r;
  if (CLOSE) {
    const double qi = ai64.w;
    r.x = (T)(qi * ((double)fx.value() + cfx));
    r.y = (T)(qi * ((double)fy.value() + cfy));
    r.z = (T)(qi * ((double)fz.value() + cfz));
    r.w = (T)((double)ph.value() + cph);
  } else {
    r.x = ai.w * fx.value();
    r.y = ai.w * fy.value();
    r.z = ai.w * fz.value();
    r.w = ph.value();
  }
  out[k] = r;
}
template <typename T, int NU, bool COMPENSATE, bool CLOSE>
struct KPair {
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { pair_body<T, NU, COMPENSATE, CLOSE>(c, a...); }
};
template <typename T, int NU, bool COMPENSATE, bool CLOSE>
__global__ void __launch_bounds__(kPairThreads)
k_pair(int N, const V4<T> *__restrict__ ps, const V4<double> *__restrict__ ps64,
       const int *__restrict__ pcs, const int *__restrict__ start, int nc0,
       int nc1, int nc2, const CellOffset<T> *__restrict__ off, int noff,
       PairConsts<T> pc, V4<T> *__restrict__ out) {
  pair_body<T, NU, COMPENSATE, CLOSE>(hw_ctx(), N, ps, ps64, pcs, start, nc0, nc1, nc2, off, noff, pc, out);
}

template <typename T, int NU>
void launch_nu(cudaStream_t s, int N, const V4<T> *ps, const V4<double> *ps64,
               const int *pcs, const int *start, const Geometry &g,
               const CellOffset<T> *off, int noff, const PairConsts<T> &pc,
               V4<T> *out) {
  int blocks = (N + kPairThreads - 1) / kPairThreads;
  if (blocks < 1) blocks = 1;
  constexpr bool kMixed = sizeof(T) == 4;
  launch<KPair<T, NU, kMixed, kMixed>, kPairThreads, sizeof(T) == 4 ? 6 : 8>(s, k_pair<T, NU, kMixed, kMixed>, blocks, kPairThreads, 0, N, ps, ps64, pcs, start, g.nc[0], g.nc[1], g.nc[2], off, noff, pc, out);
}

}  // namespace

template <typename T>
void launch_pair(cudaStream_t s, int N, const V4<T> *ps, const V4<double> *ps64,
                 const int *pcs, const int *start, const Geometry &g,
                 const CellOffset<T> *off, int noff, const PairConsts<T> &pc,
                 V4<T> *out) {
  switch (pc.nu) {
    case 0: launch_nu<T, 0>(s, N, ps, ps64, pcs, start, g, off, noff, pc, out); break;
    case 4: launch_nu<T, 4>(s, N, ps, ps64, pcs, start, g, off, noff, pc, out); break;
    case 6: launch_nu<T, 6>(s, N, ps, ps64, pcs, start, g, off, noff, pc, out); break;
    case 8: launch_nu<T, 8>(s, N, ps, ps64, pcs, start, g, off, noff, pc, out); break;
    default: launch_nu<T, 10>(s, N, ps, ps64, pcs, start, g, off, noff, pc, out); break;
  }
}

template void launch_pair<float>(cudaStream_t, int, const V4<float> *,
                                 const V4<double> *, const int *, const int *,
                                 const Geometry &, const CellOffset<float> *, int,
                                 const PairConsts<float> &, V4<float> *);
template void launch_pair<double>(cudaStream_t, int, const V4<double> *,
                                  const V4<double> *, const int *, const int *,
                                  const Geometry &, const CellOffset<double> *, int,
                                  const PairConsts<double> &, V4<double> *);

}  // namespace msm
