// Grid transfer kernels between atoms and the finest grid, and between
// levels. Grids are unpadded, periodic, x-major with z fastest.
//
// B-spline convention (code/forcefield1.c:348-368, :609-622): an atom at grid
// coordinate u = M s, m = floor(u), t = u - m contributes
// q * Q_nu(n + nu/2 + t) to grid point m - n for n in [-nu/2, nu/2), per axis.
#include <algorithm>

#include <mutex>

#include "kernels.h"

namespace msm {
namespace {

constexpr int kThreads = 256;

// Q_nu(i + t) for 0 <= i < nu (piece reflection of code/forcefield1.c:612)
template <typename T, int NU>
__device__ __forceinline__ T bspline(const SplineConsts<T> &sc, int i, T t) {
  if (i >= NU / 2) {
    i = NU - 1 - i;
    t = T(1) - t;
  }
  const T *c = sc.Q + i * NU;
  T v = c[NU - 1];
#pragma unroll
  for (int k = NU - 2; k >= 0; --k) v = c[k] + t * v;
  return v;
}

// value and d/dt (code/forcefield1.c:624-637)
template <typename T, int NU>
__device__ __forceinline__ T bspline_d(const SplineConsts<T> &sc, int i, T t,
                                       T &d) {
  T sign = T(1);
  if (i >= NU / 2) {
    i = NU - 1 - i;
    t = T(1) - t;
    sign = T(-1);
  }
  const T *c = sc.Q + i * NU;
  T v = c[NU - 1], dv = T(0);
#pragma unroll
  for (int k = NU - 2; k >= 0; --k) {
    dv = v + t * dv;
    v = c[k] + t * v;
  }
  d = sign * dv;
  return v;
}

// value, d/dt and d^2/dt^2
template <typename T, int NU>
__device__ __forceinline__ T bspline_d2(const SplineConsts<T> &sc, int i, T t, T &d1, T &d2) {
  T sign = T(1);
  if (i >= NU / 2) {
    i = NU - 1 - i;
    t = T(1) - t;
    sign = T(-1);
  }
  const T *c = sc.Q + i * NU;
  T v = c[NU - 1], dv = T(0), ddv = T(0);
#pragma unroll
  for (int k = NU - 2; k >= 0; --k) {
    ddv = dv + t * ddv;
    dv = v + t * dv;
    v = c[k] + t * v;
  }
  d1 = sign * dv;
  d2 = T(2) * ddv;
  return v;
}


// Anterpolation as a slab-staged gather (the fast path).
//
// A CTA owns BX x BY x BZ grid points; thread (tz, ty) accumulates the BX
// points (x0+xo, y0+ty, z0+tz) in registers. The atoms that can reach the
// block lie in the halo cells x0-nu/2 .. x0+BX+nu/2-2 (same in y, z). The
// halo is streamed one x-slab hx at a time: the slab's cells are counted
// and scanned, their atoms (contiguous per cell in cell-sorted order) are
// staged in shared memory with their B-spline weights (q folded into the x
// weights), then every thread adds, for its nu halo rows hy = ty + b and nu
// halo z-cells hz = tz + c, the contributions q wx[hx-xo] wy[b] wz[c].
// Every grid point is written by one thread, atoms are visited in a fixed
// order: no atomics, deterministic sums. Slabs whose atoms exceed the
// staging capacity are processed in row chunks.
template <typename T, int NU, int BX>
__device__ __forceinline__ void anterpolate_slab_body(const BlockCtx &ctx, int M0, int M1, int M2, const V4<T> *__restrict__ atoms,
                   const int *__restrict__ start, SplineConsts<T> sc, int cap,
                   T *__restrict__ grid, int *err) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int BZ = blockDim.x, BY = blockDim.y;
  const int tz = threadIdx.x, ty = threadIdx.y;
  const int tid = ty * BZ + tz, nth = BZ * BY;
  const int EY = BY + NU - 1, EZ = BZ + NU - 1, ncell = EY * EZ;
  const int x0 = ctx.b.z * BX, y0 = ctx.b.y * BY, z0 = ctx.b.x * BZ;
  // shared layout: pre[ncell+1] | hz[cap] | wx[NU][cap] | wy[NU][cap] | wz[NU][cap]
  int *pre = reinterpret_cast<int *>(smem_raw);
  int *shz = pre + ((ncell + 1 + 3) & ~3);
  T *wbase = reinterpret_cast<T *>(shz + ((cap + 3) & ~3));
  T *swx = wbase, *swy = wbase + NU * cap, *swz = wbase + 2 * NU * cap;
  __shared__ int warp_tot[16];

  T acc[BX];
#pragma unroll
  for (int a = 0; a < BX; ++a) acc[a] = T(0);

  for (int hx = 0; hx < BX + NU - 1; ++hx) {
    const int mx = pwrap(x0 - NU / 2 + hx, M0);
    // 1) per-cell counts of this slab, exclusive scan into pre[]
    const int per = (ncell + nth - 1) / nth;
    const int k0 = tid * per;
    int local = 0;
    for (int k = k0; k < min(k0 + per, ncell); ++k) {
      const int hy = k / EZ, hz = k - hy * EZ;
      const int my = pwrap(y0 - NU / 2 + hy, M1), mz = pwrap(z0 - NU / 2 + hz, M2);
      const long c = ((long)mx * M1 + my) * M2 + mz;
      const int n = start[c + 1] - start[c];
      pre[k] = n;
      local += n;
    }
    // block exclusive scan of the per-thread totals; the last warp may be
    // partial (small tiles), so the shuffle mask covers only its lanes
    const int lane = tid & 31, warp = tid >> 5;
    const int wsize = min(32, nth - warp * 32);
    const unsigned mask = wsize == 32 ? 0xffffffffu : ((1u << wsize) - 1u);
    int incl = local;
    for (int o = 1; o < 32; o <<= 1) {
      int v = __shfl_up_sync(mask, incl, o);
      if (lane >= o) incl += v;
    }
    if (lane == wsize - 1) warp_tot[warp] = incl;
    __syncthreads();
    int wbefore = 0, total = 0;
    for (int w = 0; w < (nth + 31) / 32; ++w) {
      if (w < warp) wbefore += warp_tot[w];
      total += warp_tot[w];
    }
    int run = wbefore + incl - local;
    for (int k = k0; k < min(k0 + per, ncell); ++k) {
      const int n = pre[k];
      pre[k] = run;
      run += n;
    }
    if (tid == 0) pre[ncell] = total;
    __syncthreads();
    // 2) stage in row chunks that fit the capacity
    int r0 = 0;
    while (r0 < EY) {
      int r1 = r0 + 1;
      while (r1 < EY && pre[(r1 + 1) * EZ] - pre[r0 * EZ] <= cap) ++r1;
      const int lo = pre[r0 * EZ];
      int hi = pre[r1 * EZ];
      if (hi - lo > cap) {  // one row alone exceeds the capacity
        flag_error(err, kCheckOverflow);
        hi = lo;
      }
      for (int k = r0 * EZ + tid; k < r1 * EZ && hi > lo; k += nth) {
        const int hy = k / EZ, hz = k - hy * EZ;
        const int my = pwrap(y0 - NU / 2 + hy, M1), mz = pwrap(z0 - NU / 2 + hz, M2);
        const long c = ((long)mx * M1 + my) * M2 + mz;
        const int b = start[c];
        const int n = start[c + 1] - b;
        const int slot0 = pre[k] - lo;
        if (slot0 < 0 || slot0 + n > hi - lo) {  // self-check, never expected
          flag_error(err, kCheckIndex);
          continue;
        }
        for (int u = 0; u < n; ++u) {
          const V4<T> at = atoms[b + u];
          const int s = slot0 + u;
          shz[s] = hz;
#pragma unroll
          for (int i = 0; i < NU; ++i) {
            swx[i * cap + s] = at.w * bspline<T, NU>(sc, i, at.x);
            swy[i * cap + s] = bspline<T, NU>(sc, i, at.y);
            swz[i * cap + s] = bspline<T, NU>(sc, i, at.z);
          }
        }
      }
      __syncthreads();
      // 3) accumulate from the staged rows
      for (int bb = 0; bb < NU; ++bb) {
        const int hy = ty + bb;
        if (hy < r0 || hy >= r1 || hi == lo) continue;
        const int s0 = max(0, pre[hy * EZ + tz] - lo);
        const int s1 = min(hi - lo, pre[hy * EZ + tz + NU] - lo);
        for (int s = s0; s < s1; ++s) {
          const int c = shz[s] - tz;
          if ((unsigned)c >= (unsigned)NU) continue;  // never taken
          const T wyz = swy[bb * cap + s] * swz[c * cap + s];
#pragma unroll
          for (int xo = 0; xo < BX; ++xo) {
            const int a = hx - xo;
            if (a >= 0 && a < NU) acc[xo] = fma(wyz, swx[a * cap + s], acc[xo]);
          }
        }
      }
      __syncthreads();
      r0 = r1;
    }
  }
  const int y = y0 + ty, z = z0 + tz;
  if (y >= M1 || z >= M2) return;
#pragma unroll
  for (int xo = 0; xo < BX; ++xo) {
    const int x = x0 + xo;
    if (x < M0) grid[((long)x * M1 + y) * M2 + z] = acc[xo];
  }
}
template <typename T, int NU, int BX>
struct KAnterpolateSlab {
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { anterpolate_slab_body<T, NU, BX>(c, a...); }
};
template <typename T, int NU, int BX>
__global__ void __launch_bounds__(512)
k_anterpolate_slab(int M0, int M1, int M2, const V4<T> *__restrict__ atoms,
                   const int *__restrict__ start, SplineConsts<T> sc, int cap,
                   T *__restrict__ grid, int *err) {
  anterpolate_slab_body<T, NU, BX>(hw_ctx(), M0, M1, M2, atoms, start, sc, cap, grid, err);
}

// Anterpolation as a tile scatter (the default).
//
// One warp per tile of kAT^3 grid cells. The tile's own atoms (cell-sorted,
// so one contiguous run per (x, y) cell row; 64 runs concatenated by a warp
// scan) are taken 32 at a time: each lane computes one atom's 3 nu B-spline
// weights (q folded into the x weights). The atoms are then added one after
// another into a shared accumulator covering every grid point the tile's
// atoms reach, (kAT + nu - 1)^3 points. The nu^3 contributions of one atom
// go to distinct points: lane l takes the (y, z) weight pairs l, l + 32, ...
// and loops over the nu x weights (compile-time offsets), and the pairs left
// over after the last full pass are spread one contribution per lane. One
// warp and a fixed atom order make every sum deterministic without atomics.
// The accumulator is written to the tile's scratch block; k_anterp_fold then
// adds, for each grid point, the (at most 8) blocks that cover it in a fixed
// order.
constexpr int kAT = 8;

template <int NU>
struct TileGeom {
  static constexpr int E = kAT + NU - 1;  // accumulator edge
  static constexpr int E3 = E * E * E;
  static constexpr int NP = NU * NU;      // (y, z) weight pairs
  static constexpr int FP = NP / 32;      // passes with a pair on every lane
  static constexpr int RC = (NP % 32) * NU;  // contributions of the other pairs
  static constexpr int RR = (RC + 31) / 32;  // their rounds, one per lane
  static constexpr int NW = 3 * NU + 2;   // weight row (even: vector loads)
};

// DIP: dipoles instead of charges (the adjoint's dipole grid,
// d_g = sum_i p_i . grad B_i(g)): dip[k] holds the atom's dipole in grid
// units, p^_a = M_a (A^-1 p)_a, and a contribution is
// p^x Q'x Qy Qz + p^y Qx Q'y Qz + p^z Qx Qy Q'z. Weight row: P = p^x Q'x, Qx,
// Qy, Qz, p^y Q'y, p^z Q'z (nu each).
template <typename T, int NU, bool DIP>
__device__ __forceinline__ void anterp_tiles_body(const BlockCtx &ctx, int M0, int M1, int M2, int nt1, int nt2, const V4<T> *__restrict__ atoms,
               const int *__restrict__ cell, const int *__restrict__ start,
               SplineConsts<T> sc, T *__restrict__ scratch, const V4<T> *__restrict__ dip) {
  using G = TileGeom<NU>;
  constexpr int E = G::E, NW = DIP ? 6 * NU + 2 : G::NW;
  // offsets of the y and z weights in the row
  constexpr int OY = DIP ? 2 * NU : NU, OZ = DIP ? 3 * NU : 2 * NU;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *acc = reinterpret_cast<T *>(smem_raw);  // G::E3 values
  __shared__ __align__(16) T w[32 * NW];
  __shared__ int base[32];
  __shared__ int rowbeg[64], rowoff[64];
  const int lane = threadIdx.x;
  const int tile = ctx.b.x;
  const int tz = tile % nt2, ty = (tile / nt2) % nt1, tx = tile / (nt2 * nt1);
  const int X0 = tx * kAT, Y0 = ty * kAT, Z0 = tz * kAT;
  const int nx = min(kAT, M0 - X0), ny = min(kAT, M1 - Y0), nz = min(kAT, M2 - Z0);
  for (int i = lane; i < G::E3; i += 32) acc[i] = T(0);
  // this lane's pairs of the full passes, and its leftover contributions
  int poff[G::FP > 0 ? G::FP : 1], pwb[G::FP > 0 ? G::FP : 1], pwc[G::FP > 0 ? G::FP : 1];
#pragma unroll
  for (int f = 0; f < G::FP; ++f) {
    const int pr = f * 32 + lane, b = pr / NU, c = pr % NU;
    poff[f] = b * E + c;
    pwb[f] = OY + b;
    pwc[f] = OZ + c;
  }
  int roff[G::RR > 0 ? G::RR : 1], ra[G::RR > 0 ? G::RR : 1], rb[G::RR > 0 ? G::RR : 1],
      rc[G::RR > 0 ? G::RR : 1];
#pragma unroll
  for (int r = 0; r < G::RR; ++r) {
    const int ci = r * 32 + lane;
    roff[r] = -1;
    ra[r] = rb[r] = rc[r] = 0;
    if (ci < G::RC) {
      const int pr = G::FP * 32 + ci / NU, a = ci % NU, b = pr / NU, c = pr % NU;
      roff[r] = a * E * E + b * E + c;
      ra[r] = a;
      rb[r] = OY + b;
      rc[r] = OZ + c;
    }
  }
  // the 64 cell rows of the tile
  int cnt[2], beg[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int rr = lane + 32 * h, x = rr / kAT, y = rr % kAT;
    cnt[h] = 0;
    beg[h] = 0;
    if (x < nx && y < ny) {
      const long c0 = ((long)(X0 + x) * M1 + (Y0 + y)) * M2 + Z0;
      beg[h] = start[c0];
      cnt[h] = start[c0 + nz] - beg[h];
    }
  }
  int incl0 = cnt[0], incl1 = cnt[1];
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int y0 = __shfl_up_sync(0xffffffffu, incl0, d);
    const int y1 = __shfl_up_sync(0xffffffffu, incl1, d);
    if (lane >= d) {
      incl0 += y0;
      incl1 += y1;
    }
  }
  const int tot0 = __shfl_sync(0xffffffffu, incl0, 31);
  const int total = tot0 + __shfl_sync(0xffffffffu, incl1, 31);
  rowbeg[lane] = beg[0];
  rowbeg[lane + 32] = beg[1];
  rowoff[lane] = incl0 - cnt[0];
  rowoff[lane + 32] = tot0 + incl1 - cnt[1];
  __syncwarp();

  for (int k0 = 0; k0 < total; k0 += 32) {
    const int k = k0 + lane;
    const int n = min(32, total - k0);
    if (k < total) {
      int r = 0;  // last row starting at or before k
#pragma unroll
      for (int step = 32; step; step >>= 1)
        if (r + step < 64 && rowoff[r + step] <= k) r += step;
      const int g = rowbeg[r] + (k - rowoff[r]);
      const V4<T> at = atoms[g];
      const int x = r / kAT, y = r % kAT;
      const long c0 = ((long)(X0 + x) * M1 + (Y0 + y)) * M2 + Z0;
      const int z = (int)(cell[g] - c0);  // the row's cells are c0 .. c0 + nz - 1
      base[lane] = (x + NU - 1) * E * E + (y + NU - 1) * E + (z + NU - 1);
      T *wl = w + lane * NW;
      if constexpr (DIP) {
        const V4<T> dp = dip[g];
#pragma unroll
        for (int i = 0; i < NU; ++i) {
          T d;
          wl[NU + i] = bspline_d<T, NU>(sc, i, at.x, d);
          wl[i] = dp.x * d;
          wl[OY + i] = bspline_d<T, NU>(sc, i, at.y, d);
          wl[4 * NU + i] = dp.y * d;
          wl[OZ + i] = bspline_d<T, NU>(sc, i, at.z, d);
          wl[5 * NU + i] = dp.z * d;
        }
      } else {
#pragma unroll
        for (int i = 0; i < NU; ++i) {
          wl[i] = at.w * bspline<T, NU>(sc, i, at.x);
          wl[NU + i] = bspline<T, NU>(sc, i, at.y);
          wl[2 * NU + i] = bspline<T, NU>(sc, i, at.z);
        }
      }
    }
    __syncwarp();
    for (int j = 0; j < n; ++j) {
      const int bj = base[j];
      const T *wj = w + j * NW;
      T wa[NU];
#pragma unroll
      for (int a = 0; a < NU; a += 2) {
        if constexpr (sizeof(T) == 4) {
          const float2 v = *reinterpret_cast<const float2 *>(wj + a);
          wa[a] = v.x;
          wa[a + 1] = v.y;
        } else {
          const double2 v = *reinterpret_cast<const double2 *>(wj + a);
          wa[a] = v.x;
          wa[a + 1] = v.y;
        }
      }
      T wx[DIP ? NU : 1];
      if constexpr (DIP) {
#pragma unroll
        for (int a = 0; a < NU; ++a) wx[a] = wj[NU + a];
      }
#pragma unroll
      for (int f = 0; f < G::FP; ++f) {
        const T wyz = wj[pwb[f]] * wj[pwc[f]];
        T *ap = acc + (bj - poff[f]);
        if constexpr (DIP) {
          // pwb - OY = b, pwc - OZ = c
          const T u = wj[pwc[f]] * wj[4 * NU + pwb[f] - OY] +
                      wj[pwb[f]] * wj[5 * NU + pwc[f] - OZ];
#pragma unroll
          for (int a = 0; a < NU; ++a)
            ap[-a * E * E] = fma(wyz, wa[a], fma(u, wx[a], ap[-a * E * E]));
        } else {
#pragma unroll
          for (int a = 0; a < NU; ++a) ap[-a * E * E] = fma(wyz, wa[a], ap[-a * E * E]);
        }
      }
#pragma unroll
      for (int r = 0; r < G::RR; ++r) {
        if (roff[r] >= 0) {
          T *ap = acc + (bj - roff[r]);
          if constexpr (DIP) {
            const T wyz = wj[rb[r]] * wj[rc[r]];
            const T u = wj[rc[r]] * wj[4 * NU + rb[r] - OY] + wj[rb[r]] * wj[5 * NU + rc[r] - OZ];
            *ap = fma(wyz, wj[ra[r]], fma(u, wj[NU + ra[r]], *ap));
          } else {
            *ap = fma(wj[rb[r]] * wj[rc[r]], wj[ra[r]], *ap);
          }
        }
      }
      __syncwarp();
    }
  }
  __syncwarp();
  T *out = scratch + (long)tile * G::E3;
  for (int i = lane; i < G::E3; i += 32) out[i] = acc[i];
}
template <typename T, int NU, bool DIP>
struct KAnterpTiles {
  static constexpr int kUniformArg = 8;  // SplineConsts
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { anterp_tiles_body<T, NU, DIP>(c, a...); }
};
template <typename T, int NU, bool DIP>
__global__ void __launch_bounds__(32)
k_anterp_tiles(int M0, int M1, int M2, int nt1, int nt2, const V4<T> *__restrict__ atoms,
               const int *__restrict__ cell, const int *__restrict__ start,
               SplineConsts<T> sc, T *__restrict__ scratch, const V4<T> *__restrict__ dip) {
  anterp_tiles_body<T, NU, DIP>(hw_ctx(), M0, M1, M2, nt1, nt2, atoms, cell, start, sc, scratch, dip);
}

// grid[p] = sum over the tiles covering p of their block value at p, in a
// fixed order. tab (host-built, anterp_fold_table): per axis and point, the
// count (<= 4) and the (tile, local index) covers packed as tile << 8 | local.
template <typename T, int NU>
__device__ __forceinline__ void anterp_fold_body(const BlockCtx &ctx, int M0, int M1, int M2, int nt1, int nt2, const int *__restrict__ tab,
              const T *__restrict__ scratch, T *__restrict__ grid) {
  using G = TileGeom<NU>;
  const long idx = (long)ctx.b.x * blockDim.x + threadIdx.x;
  if (idx >= (long)M0 * M1 * M2) return;
  const int p2 = idx % M2, p1 = (idx / M2) % M1, p0 = idx / ((long)M1 * M2);
  const int *t0 = tab + 5 * p0, *t1 = tab + 5 * (M0 + p1), *t2 = tab + 5 * (M0 + M1 + p2);
  const int n0 = t0[0], n1 = t1[0], n2 = t2[0];
  T s = T(0);
  for (int a = 0; a < n0; ++a) {
    const int e0 = t0[1 + a];
    for (int b = 0; b < n1; ++b) {
      const int e1 = t1[1 + b];
      const long tl = (long)(e0 >> 8) * nt1 + (e1 >> 8);
      const int l01 = ((e0 & 255) * G::E + (e1 & 255)) * G::E;
      for (int c = 0; c < n2; ++c) {
        const int e2 = t2[1 + c];
        s += scratch[(tl * nt2 + (e2 >> 8)) * G::E3 + l01 + (e2 & 255)];
      }
    }
  }
  grid[idx] = s;
}
template <typename T, int NU>
struct KAnterpFold {
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { anterp_fold_body<T, NU>(c, a...); }
};
template <typename T, int NU>
__global__ void __launch_bounds__(kThreads)
k_anterp_fold(int M0, int M1, int M2, int nt1, int nt2, const int *__restrict__ tab,
              const T *__restrict__ scratch, T *__restrict__ grid) {
  anterp_fold_body<T, NU>(hw_ctx(), M0, M1, M2, nt1, nt2, tab, scratch, grid);
}

// Field and potential at each atom (code/forcefield1.c:570-607), separable:
// z sums first, then y, then x. Output E in Cartesian components
// (E = A^-T (M * grad_u)) and phi_long.
template <typename T, int NU>
__device__ __forceinline__ void interpolate_body(const BlockCtx &ctx, int N, int M0, int M1, int M2, const V4<T> *__restrict__ atoms,
              const int *__restrict__ cell, const T *__restrict__ grid,
              SplineConsts<T> sc, Geometry g, V4<T> *__restrict__ out) {
  int k = ctx.b.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  const V4<T> at = atoms[k];
  const int c = cell[k];
  const int mz = c % M2, my = (c / M2) % M1, mx = c / (M1 * M2);
  T wx[NU], dx[NU], wy[NU], dy[NU], wz[NU], dz[NU];
#pragma unroll
  for (int i = 0; i < NU; ++i) {
    wx[i] = bspline_d<T, NU>(sc, i, at.x, dx[i]);
    wy[i] = bspline_d<T, NU>(sc, i, at.y, dy[i]);
    wz[i] = bspline_d<T, NU>(sc, i, at.z, dz[i]);
  }
  int zi[NU];
#pragma unroll
  for (int i = 0; i < NU; ++i) zi[i] = pwrap(mz - (i - NU / 2), M2);
  // The sums run over e - e_c, e_c the potential at the atom's own grid
  // point: the derivative weights sum to zero and the value weights to one,
  // so the results are unchanged in exact arithmetic, while the rounded
  // products are of differences (about h |E|) rather than of potentials,
  // which are much larger than h |E|.
  const T ec = grid[((long)mx * M1 + my) * M2 + mz];
  T phi = 0, ex = 0, ey = 0, ez = 0;
  for (int a = 0; a < NU; ++a) {
    const int gx = pwrap(mx - (a - NU / 2), M0);
    T t00 = 0, t10 = 0, t01 = 0;
    for (int b = 0; b < NU; ++b) {
      const int gy = pwrap(my - (b - NU / 2), M1);
      const T *row = grid + ((long)gx * M1 + gy) * M2;
      T s0 = 0, s1 = 0;
      if constexpr (sizeof(T) == 4) {
        // the value and derivative sums as one packed FP32 multiply-add per
        // grid value (each half rounded as the scalar one)
        float2 s = make_float2(0.f, 0.f);
#pragma unroll
        for (int i = 0; i < NU; ++i) {
          const float e = row[zi[i]] - ec;
          s = __ffma2_rn(make_float2(wz[i], dz[i]), make_float2(e, e), s);
        }
        s0 = s.x;
        s1 = s.y;
      } else {
#pragma unroll
        for (int i = 0; i < NU; ++i) {
          const T e = row[zi[i]] - ec;
          s0 += wz[i] * e;
          s1 += dz[i] * e;
        }
      }
      t00 += wy[b] * s0;
      t10 += dy[b] * s0;
      t01 += wy[b] * s1;
    }
    phi += wx[a] * t00;
    ex -= dx[a] * t00;
    ey -= wx[a] * t10;
    ez -= wx[a] * t01;
  }
  const double gxv = (double)ex * M0, gyv = (double)ey * M1, gzv = (double)ez * M2;
  V4<T> r;
  r.x = (T)(g.Ai[0] * gxv + g.Ai[3] * gyv + g.Ai[6] * gzv);
  r.y = (T)(g.Ai[1] * gxv + g.Ai[4] * gyv + g.Ai[7] * gzv);
  r.z = (T)(g.Ai[2] * gxv + g.Ai[5] * gyv + g.Ai[8] * gzv);
  r.w = phi + ec;
  out[k] = r;
}
template <typename T, int NU>
struct KInterpolate {
  static constexpr int kUniformArg = 7;  // SplineConsts
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { interpolate_body<T, NU>(c, a...); }
};
template <typename T, int NU>
__global__ void __launch_bounds__(kThreads)
k_interpolate(int N, int M0, int M1, int M2, const V4<T> *__restrict__ atoms,
              const int *__restrict__ cell, const T *__restrict__ grid,
              SplineConsts<T> sc, Geometry g, V4<T> *__restrict__ out) {
  interpolate_body<T, NU>(hw_ctx(), N, M0, M1, M2, atoms, cell, grid, sc, g, out);
}

// Adjoint interpolation, per atom (grid-sorted order): the value psi and
// the Cartesian gradient G of the interpolated dipole potential ed, and the
// Hessian of the interpolated charge potential e1 applied to the force
// cotangent: Hess F^ = A^-T D H_u D A^-1 F^ (D = diag(M), H_u the second
// derivatives in grid units, from second-derivative B-splines). All sums run
// about the home grid value (derivative weights sum to zero).
// out_g = (G, psi), out_h = (Hess F^, 0).
template <typename T, int NU>
__global__ void __launch_bounds__(kThreads)
k_adj_interp(int N, int M0, int M1, int M2, const V4<T> *__restrict__ atoms,
             const int *__restrict__ cell, const int *__restrict__ gperm,
             const double *__restrict__ fbar, const T *__restrict__ ed,
             const T *__restrict__ e1, SplineConsts<T> sc, Geometry g,
             V4<T> *__restrict__ out_g, V4<T> *__restrict__ out_h) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  const V4<T> at = atoms[k];
  const int c = cell[k];
  const int mz = c % M2, my = (c / M2) % M1, mx = c / (M1 * M2);
  T wx[NU], dx[NU], hx[NU], wy[NU], dy[NU], hy[NU], wz[NU], dz[NU], hz[NU];
#pragma unroll
  for (int i = 0; i < NU; ++i) {
    wx[i] = bspline_d2<T, NU>(sc, i, at.x, dx[i], hx[i]);
    wy[i] = bspline_d2<T, NU>(sc, i, at.y, dy[i], hy[i]);
    wz[i] = bspline_d2<T, NU>(sc, i, at.z, dz[i], hz[i]);
  }
  int zi[NU];
#pragma unroll
  for (int i = 0; i < NU; ++i) zi[i] = pwrap(mz - (i - NU / 2), M2);
  const long home = ((long)mx * M1 + my) * M2 + mz;
  const T cd = ed[home], c1 = e1[home];
  T p = 0, gx = 0, gy = 0, gz = 0;                       // ed: value, grad_u
  T hxx = 0, hyy = 0, hzz = 0, hxy = 0, hxz = 0, hyz = 0;  // e1: H_u
  for (int a = 0; a < NU; ++a) {
    const int ix = pwrap(mx - (a - NU / 2), M0);
    T t00 = 0, t10 = 0, t01 = 0;                 // ed
    T u00 = 0, u10 = 0, u01 = 0, u20 = 0, u11 = 0, u02 = 0;  // e1
    for (int b = 0; b < NU; ++b) {
      const int iy = pwrap(my - (b - NU / 2), M1);
      const long row = ((long)ix * M1 + iy) * M2;
      T s0 = 0, s1 = 0, r0 = 0, r1 = 0, r2 = 0;
#pragma unroll
      for (int i = 0; i < NU; ++i) {
        const T vd = ed[row + zi[i]] - cd, v1 = e1[row + zi[i]] - c1;
        s0 += wz[i] * vd;
        s1 += dz[i] * vd;
        r0 += wz[i] * v1;
        r1 += dz[i] * v1;
        r2 += hz[i] * v1;
      }
      t00 += wy[b] * s0;
      t10 += dy[b] * s0;
      t01 += wy[b] * s1;
      u00 += wy[b] * r0;
      u10 += dy[b] * r0;
      u01 += wy[b] * r1;
      u20 += hy[b] * r0;
      u11 += dy[b] * r1;
      u02 += wy[b] * r2;
    }
    p += wx[a] * t00;
    gx += dx[a] * t00;
    gy += wx[a] * t10;
    gz += wx[a] * t01;
    hxx += hx[a] * u00;
    hyy += wx[a] * u20;
    hzz += wx[a] * u02;
    hxy += dx[a] * u10;
    hxz += dx[a] * u01;
    hyz += wx[a] * u11;
  }
  // grid-unit derivatives to Cartesian
  const double Mv[3] = {(double)M0, (double)M1, (double)M2};
  const double gu[3] = {(double)gx * Mv[0], (double)gy * Mv[1], (double)gz * Mv[2]};
  const int i = gperm[k];
  const double fb[3] = {fbar[3 * i], fbar[3 * i + 1], fbar[3 * i + 2]};
  double v[3];  // D A^-1 F^
  for (int q = 0; q < 3; ++q)
    v[q] = Mv[q] * (g.Ai[3 * q] * fb[0] + g.Ai[3 * q + 1] * fb[1] + g.Ai[3 * q + 2] * fb[2]);
  const double H[3][3] = {{hxx, hxy, hxz}, {hxy, hyy, hyz}, {hxz, hyz, hzz}};
  double hv[3];  // D H_u v
  for (int q = 0; q < 3; ++q) hv[q] = Mv[q] * (H[q][0] * v[0] + H[q][1] * v[1] + H[q][2] * v[2]);
  V4<T> og, oh;
  og.x = (T)(g.Ai[0] * gu[0] + g.Ai[3] * gu[1] + g.Ai[6] * gu[2]);
  og.y = (T)(g.Ai[1] * gu[0] + g.Ai[4] * gu[1] + g.Ai[7] * gu[2]);
  og.z = (T)(g.Ai[2] * gu[0] + g.Ai[5] * gu[1] + g.Ai[8] * gu[2]);
  og.w = p + cd;
  oh.x = (T)(g.Ai[0] * hv[0] + g.Ai[3] * hv[1] + g.Ai[6] * hv[2]);
  oh.y = (T)(g.Ai[1] * hv[0] + g.Ai[4] * hv[1] + g.Ai[7] * hv[2]);
  oh.z = (T)(g.Ai[2] * hv[0] + g.Ai[5] * hv[1] + g.Ai[8] * hv[2]);
  oh.w = T(0);
  out_g[k] = og;
  out_h[k] = oh;
}

struct TwoScale {
  double J[11];
};

// Restriction and prolongation as separable per-axis two-scale sums: a CTA
// stages its tile plus the B-spline halo in shared memory (periodic wrap
// applied once, at the load) and contracts z, then y, then x there, so a
// point costs 3 (nu + 1) multiply-adds instead of (nu + 1)^3 (restriction)
// or about (nu / 2 + 1)^3 (prolongation) wrapped loads.
constexpr int kSepThreads = 256;

// Restriction tile: CX x CY x CZ coarse points (z fastest)
template <typename T>
struct RestrictTile {
  static constexpr int CX = 4, CY = 8, CZ = sizeof(T) == 4 ? 16 : 8;
};
template <typename T, int NU>
struct RestrictGeom {
  using Tl = RestrictTile<T>;
  static constexpr int RX = 2 * Tl::CX + NU - 1, RY = 2 * Tl::CY + NU - 1,
                       RZ = 2 * Tl::CZ + NU - 1;
  // fine region, then the z-contracted region (RX x RY x CZ); the y pass
  // writes RX x CY x CZ over the start of the fine region
  static constexpr int SMEM = (RX * RY * RZ + RX * RY * Tl::CZ) * (int)sizeof(T);
};

// q^{l+1}_m = sum_n J_n q^l_{2m+n}, n in [-nu/2, nu/2]^3
// (code/forcefield1.c:401-477)
template <typename T, int NU>
__device__ __forceinline__ void restrict_body(const BlockCtx &ctx, int F0, int F1, int F2, const T *__restrict__ fine,
           T *__restrict__ coarse, TwoScale js) {
  using Tl = RestrictTile<T>;
  using G = RestrictGeom<T, NU>;
  constexpr int CX = Tl::CX, CY = Tl::CY, CZ = Tl::CZ, RX = G::RX, RY = G::RY, RZ = G::RZ;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *reg = reinterpret_cast<T *>(smem_raw);
  T *t1 = reg + RX * RY * RZ;
  T *t2 = reg;
  const int C0 = F0 / 2, C1 = F1 / 2, C2 = F2 / 2;
  const int nbz = (C2 + CZ - 1) / CZ, nby = (C1 + CY - 1) / CY;
  const int bz = ctx.b.x % nbz, by = (ctx.b.x / nbz) % nby, bx = ctx.b.x / (nbz * nby);
  const int x0 = bx * CX, y0 = by * CY, z0 = bz * CZ;
  __shared__ int wrap[RX + RY + RZ];  // periodic indices of the region's planes, rows, columns
  T J[NU + 1];
#pragma unroll
  for (int i = 0; i <= NU; ++i) J[i] = (T)js.J[i];
  for (int i = threadIdx.x; i < RX + RY + RZ; i += kSepThreads)
    wrap[i] = i < RX        ? pwrap(2 * x0 - NU / 2 + i, F0) * F1
              : i < RX + RY ? pwrap(2 * y0 - NU / 2 + i - RX, F1)
                            : pwrap(2 * z0 - NU / 2 + i - RX - RY, F2);
  __syncthreads();
#pragma unroll 4
  for (int t = threadIdx.x; t < RX * RY * RZ; t += kSepThreads) {
    const int rz = t % RZ, ry = (t / RZ) % RY, rx = t / (RZ * RY);
    reg[t] = fine[(long)(wrap[rx] + wrap[RX + ry]) * F2 + wrap[RX + RY + rz]];
  }
  __syncthreads();
  for (int t = threadIdx.x; t < RX * RY * CZ; t += kSepThreads) {
    const int cz = t % CZ, r = t / CZ;  // r = rx * RY + ry
    const T *row = reg + r * RZ + 2 * cz;
    T acc = 0;
#pragma unroll
    for (int c = 0; c <= NU; ++c) acc += J[c] * row[c];
    t1[t] = acc;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < RX * CY * CZ; t += kSepThreads) {
    const int cz = t % CZ, cy = (t / CZ) % CY, rx = t / (CZ * CY);
    const T *col = t1 + (rx * RY + 2 * cy) * CZ + cz;
    T acc = 0;
#pragma unroll
    for (int b = 0; b <= NU; ++b) acc += J[b] * col[b * CZ];
    t2[t] = acc;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < CX * CY * CZ; t += kSepThreads) {
    const int cz = t % CZ, cy = (t / CZ) % CY, cx = t / (CZ * CY);
    const int x = x0 + cx, y = y0 + cy, z = z0 + cz;
    if (x >= C0 || y >= C1 || z >= C2) continue;
    const T *col = t2 + ((2 * cx) * CY + cy) * CZ + cz;
    T acc = 0;
#pragma unroll
    for (int a = 0; a <= NU; ++a) acc += J[a] * col[a * CY * CZ];
    coarse[((long)x * C1 + y) * C2 + z] = acc;
  }
}
template <typename T, int NU>
struct KRestrict {
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { restrict_body<T, NU>(c, a...); }
};
template <typename T, int NU>
__global__ void __launch_bounds__(kSepThreads)
k_restrict(int F0, int F1, int F2, const T *__restrict__ fine,
           T *__restrict__ coarse, TwoScale js) {
  restrict_body<T, NU>(hw_ctx(), F0, F1, F2, fine, coarse, js);
}

// Prolongation tile: FX x FY x FZ fine points; the coarse region along an
// axis covers every m with |x - 2m| <= nu/2 for x in the tile
constexpr int kPX = 8, kPY = 8, kPZ = 32;
template <int NU>
struct ProlongGeom {
  // tile starts are even, so m runs over [x0/2 - ceil(nu/4), (x0 + F - 1 + nu/2)/2]
  static constexpr int lo = (NU / 2 + 1) / 2;
  static constexpr int RX = (kPX - 1 + NU / 2) / 2 + lo + 1, RY = (kPY - 1 + NU / 2) / 2 + lo + 1,
                       RZ = (kPZ - 1 + NU / 2) / 2 + lo + 1;
  static constexpr int N_REG = RX * RY * RZ, N_T1 = RX * RY * kPZ, N_T2 = RX * kPY * kPZ;
};

// Taps of fine index x: n = x - 2m in [-nu/2, nu/2] with the parity of
// x + nu/2, i.e. n = -nu/2 + p + 2k, p = (x + nu/2) & 1, k = 0.. (nu/2 - p);
// weights picked by compile-time k so J stays in registers.
template <int NU>
__device__ __forceinline__ bool tap_live(int x, int k) {
  return k < NU / 2 || ((x + NU / 2) & 1) == 0;
}
template <typename T, int NU>
__device__ __forceinline__ T tap_weight(const T (&J)[NU + 1], int x, int k) {
  const int p = (x + NU / 2) & 1;
  return (p && 2 * k + 1 <= NU) ? J[2 * k + 1 <= NU ? 2 * k + 1 : NU] : J[2 * k];
}
// coarse index m = (x - n) / 2 (x - n is even)
template <int NU>
__device__ __forceinline__ int tap_coarse(int x, int k) {
  return (x + NU / 2 - ((x + NU / 2) & 1) - 2 * k) >> 1;
}

// e^l_x += sum over (m, n) with 2m + n = x (mod M) of J_n e^{l+1}_m
// (transpose of the restriction; code/forcefield1.c:530-567)
template <typename T, int NU>
__device__ __forceinline__ void prolong_body(const BlockCtx &ctx, int F0, int F1, int F2, const T *__restrict__ coarse,
          T *__restrict__ fine, TwoScale js) {
  using G = ProlongGeom<NU>;
  constexpr int RX = G::RX, RY = G::RY, RZ = G::RZ, lo = G::lo;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *reg = reinterpret_cast<T *>(smem_raw);
  T *t1 = reg + G::N_REG;
  T *t2 = t1 + G::N_T1;
  const int C0 = F0 / 2, C1 = F1 / 2, C2 = F2 / 2;
  const int nbz = (F2 + kPZ - 1) / kPZ, nby = (F1 + kPY - 1) / kPY;
  const int bz = ctx.b.x % nbz, by = (ctx.b.x / nbz) % nby, bx = ctx.b.x / (nbz * nby);
  const int x0 = bx * kPX, y0 = by * kPY, z0 = bz * kPZ;
  // coarse region origin along each axis
  const int mx0 = x0 / 2 - lo, my0 = y0 / 2 - lo, mz0 = z0 / 2 - lo;
  __shared__ int wrap[RX + RY + RZ];
  T J[NU + 1];
#pragma unroll
  for (int i = 0; i <= NU; ++i) J[i] = (T)js.J[i];
  for (int i = threadIdx.x; i < RX + RY + RZ; i += kSepThreads)
    wrap[i] = i < RX        ? pwrap(mx0 + i, C0) * C1
              : i < RX + RY ? pwrap(my0 + i - RX, C1)
                            : pwrap(mz0 + i - RX - RY, C2);
  __syncthreads();
#pragma unroll 4
  for (int t = threadIdx.x; t < G::N_REG; t += kSepThreads) {
    const int rz = t % RZ, ry = (t / RZ) % RY, rx = t / (RZ * RY);
    reg[t] = coarse[(long)(wrap[rx] + wrap[RX + ry]) * C2 + wrap[RX + RY + rz]];
  }
  __syncthreads();
  // z: t1[rx][ry][fz] = sum_n J_n reg[rx][ry][(z - n)/2 - mz0], n = z (mod 2)
  for (int t = threadIdx.x; t < G::N_T1; t += kSepThreads) {
    const int fz = t % kPZ, r = t / kPZ;
    const int z = z0 + fz;
    const T *row = reg + r * RZ - mz0;
    T acc = 0;
#pragma unroll
    for (int k = 0; k <= NU / 2; ++k)
      if (tap_live<NU>(z, k)) acc += tap_weight<T, NU>(J, z, k) * row[tap_coarse<NU>(z, k)];
    t1[t] = acc;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < G::N_T2; t += kSepThreads) {
    const int fz = t % kPZ, fy = (t / kPZ) % kPY, rx = t / (kPZ * kPY);
    const int y = y0 + fy;
    const T *col = t1 + rx * RY * kPZ + fz;
    T acc = 0;
#pragma unroll
    for (int k = 0; k <= NU / 2; ++k)
      if (tap_live<NU>(y, k))
        acc += tap_weight<T, NU>(J, y, k) * col[(tap_coarse<NU>(y, k) - my0) * kPZ];
    t2[t] = acc;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < kPX * kPY * kPZ; t += kSepThreads) {
    const int fz = t % kPZ, fy = (t / kPZ) % kPY, fx = t / (kPZ * kPY);
    const int x = x0 + fx, y = y0 + fy, z = z0 + fz;
    if (x >= F0 || y >= F1 || z >= F2) continue;
    const T *col = t2 + fy * kPZ + fz;
    T acc = 0;
#pragma unroll
    for (int k = 0; k <= NU / 2; ++k)
      if (tap_live<NU>(x, k))
        acc += tap_weight<T, NU>(J, x, k) * col[(tap_coarse<NU>(x, k) - mx0) * kPY * kPZ];
    fine[((long)x * F1 + y) * F2 + z] += acc;
  }
}
template <typename T, int NU>
struct KProlong {
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { prolong_body<T, NU>(c, a...); }
};
template <typename T, int NU>
__global__ void __launch_bounds__(kSepThreads)
k_prolong(int F0, int F1, int F2, const T *__restrict__ coarse,
          T *__restrict__ fine, TwoScale js) {
  prolong_body<T, NU>(hw_ctx(), F0, F1, F2, coarse, fine, js);
}

template <typename T, int NU>
constexpr int prolong_smem() {
  return (ProlongGeom<NU>::N_REG + ProlongGeom<NU>::N_T1 + ProlongGeom<NU>::N_T2) *
         (int)sizeof(T);
}

template <typename T>
__device__ __forceinline__ void grid_dot_body(const BlockCtx &ctx, long n, const T *__restrict__ a, const T *__restrict__ b,
           double *partials) {
  __shared__ double sh[kThreads];
  double acc = 0.;
  for (long i = (long)ctx.b.x * kThreads + threadIdx.x; i < n;
       i += (long)ctx.g.x * kThreads)
    acc += (double)a[i] * (double)b[i];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int w = kThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[ctx.b.x] = sh[0];
}
template <typename T>
struct KGridDot {
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { grid_dot_body<T>(c, a...); }
};
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_grid_dot(long n, const T *__restrict__ a, const T *__restrict__ b,
           double *partials) {
  grid_dot_body<T>(hw_ctx(), n, a, b, partials);
}

inline int blocks_for(long n) {
  return (int)std::max<long>(1, (n + kThreads - 1) / kThreads);
}

// Blocks per SM the merged launches of these kernels are compiled for: the
// plain kernels' own occupancy at their register counts (their arguments then
// stay in the constant bank rather than in registers)
template <typename T, int NU>
constexpr int interp_multi_blocks() {
  return sizeof(T) == 4 ? (NU <= 6 ? 3 : NU == 8 ? 2 : 1) : (NU <= 6 ? 2 : 1);
}

#define MSM_NU_SWITCH(nu, CALL)     \
  switch (nu) {                     \
    case 4: { constexpr int NU = 4; CALL; } break;  \
    case 6: { constexpr int NU = 6; CALL; } break;  \
    case 8: { constexpr int NU = 8; CALL; } break;  \
    default: { constexpr int NU = 10; CALL; } break; \
  }
#define MSM_NU_SWITCH_ALL(CALL)                 \
  { constexpr int NU = 4; CALL; }               \
  { constexpr int NU = 6; CALL; }               \
  { constexpr int NU = 8; CALL; }               \
  { constexpr int NU = 10; CALL; }

constexpr int kAnterpBX = 4;
constexpr int kAnterpSmemBudget = 96 * 1024;

struct AnterpTile {
  int bz, by, cap;
  size_t smem;
};

// z extent: the candidate (<= 64) that wastes the fewest points; y fills
// up to 512 threads (at most 8 rows); staging capacity fills the budget.
template <typename T>
AnterpTile anterp_tile(const int M[3], int nu, long natoms) {
  AnterpTile t{};
  int best = 32;
  double best_waste = 1e30;
  for (int bz : {64, 48, 32, 56, 40, 24, 16}) {
    int b = std::min(bz, M[2]);
    double waste = (double)((M[2] + b - 1) / b * b) / M[2] + (b < 32 ? 0.05 : 0.0);
    if (waste < best_waste - 1e-9) {
      best_waste = waste;
      best = b;
    }
  }
  t.bz = best;
  t.by = std::max(1, std::min(std::min(8, M[1]), 512 / t.bz));
  const int ncell = (t.by + nu - 1) * (t.bz + nu - 1);
  const size_t fixed = 4 * (size_t)((ncell + 1 + 3) & ~3);
  // capacity: twice the expected atoms of one halo slab (at least 256),
  // at most the budget; denser slabs are staged in row chunks
  const double per_cell = (double)natoms / ((double)M[0] * M[1] * M[2]);
  const int want = (int)(2.0 * per_cell * ncell) + 64;
  int cap = (int)((kAnterpSmemBudget - fixed - 64) / (3 * nu * sizeof(T) + 4));
  cap = std::min(cap, std::max(256, want));
  cap &= ~3;
  t.cap = std::max(4, cap);
  t.smem = fixed + 4 * (size_t)t.cap + 3 * (size_t)nu * t.cap * sizeof(T);
  return t;
}

}  // namespace

size_t anterp_scratch_elems(const int M[3], int nu) {
  const size_t nt = (size_t)((M[0] + kAT - 1) / kAT) * ((M[1] + kAT - 1) / kAT) *
                    ((M[2] + kAT - 1) / kAT);
  const size_t e = kAT + nu - 1;
  return nt * e * e * e;
}

bool anterp_tiles_supported(const int M[3], int nu) {
  return M[0] >= nu && M[1] >= nu && M[2] >= nu;
}

// Tile j of an axis covers the points j kAT - nu/2 + 1 + l (mod M), l in
// [0, n_j + nu - 1), n_j = min(kAT, M - j kAT). With M >= nu a point has at
// most 4 covers per axis.
std::vector<int> anterp_fold_table(const int M[3], int nu) {
  std::vector<int> tab(5 * (size_t)(M[0] + M[1] + M[2]), 0);
  size_t o = 0;
  for (int ax = 0; ax < 3; ++ax) {
    const int nt = (M[ax] + kAT - 1) / kAT;
    for (int p = 0; p < M[ax]; ++p, o += 5) {
      int n = 0;
      for (int j = 0; j < nt; ++j) {
        const int nj = std::min(kAT, M[ax] - j * kAT);
        const int lo = j * kAT - nu / 2 + 1;
        for (int l = ((p - lo) % M[ax] + M[ax]) % M[ax]; l < nj + nu - 1; l += M[ax])
          if (n < 4) tab[o + 1 + n++] = (j << 8) | l;
      }
      tab[o] = n;
    }
  }
  return tab;
}

template <typename T>
void launch_anterpolate(cudaStream_t s, const int M[3], const V4<T> *atoms,
                        const int *cell_sorted, const int *cell_start,
                        const SplineConsts<T> &sc, T *grid, int variant, int *err,
                        long natoms, T *scratch, const int *fold_tab) {
  if (variant == 0 && scratch && fold_tab && anterp_tiles_supported(M, sc.nu)) {
    const int nt0 = (M[0] + kAT - 1) / kAT, nt1 = (M[1] + kAT - 1) / kAT,
              nt2 = (M[2] + kAT - 1) / kAT;
    const int ntiles = nt0 * nt1 * nt2;
    const long n = (long)M[0] * M[1] * M[2];
    MSM_NU_SWITCH(sc.nu, (launch<KAnterpTiles<T, NU, false>, 32, 1>(s, k_anterp_tiles<T, NU, false>, ntiles, 32, TileGeom<NU>::E3 * sizeof(T), M[0], M[1], M[2], nt1, nt2, atoms, cell_sorted, cell_start,
                             sc, scratch, nullptr)));
    MSM_NU_SWITCH(sc.nu, (launch<KAnterpFold<T, NU>, kThreads, 8>(s, k_anterp_fold<T, NU>, blocks_for(n), kThreads, 0, M[0], M[1], M[2], nt1, nt2, fold_tab, scratch, grid)));
    return;
  }
  const AnterpTile t = anterp_tile<T>(M, sc.nu, natoms);
  dim3 block(t.bz, t.by);
  dim3 g((M[2] + t.bz - 1) / t.bz, (M[1] + t.by - 1) / t.by,
         (M[0] + kAnterpBX - 1) / kAnterpBX);
  MSM_NU_SWITCH(sc.nu, (launch<KAnterpolateSlab<T, NU, kAnterpBX>, 512, 1>(s, k_anterpolate_slab<T, NU, kAnterpBX>, g, block, t.smem, M[0], M[1], M[2], atoms, cell_start, sc, t.cap, grid, err)));
}

template <typename T>
void anterpolate_prepare() {
  static std::mutex mu;
  static bool done[kMaxDevices];
  const int dev = device_slot();
  std::lock_guard<std::mutex> lock(mu);
  if (dev >= 0 && done[dev]) return;
  MSM_NU_SWITCH_ALL(cudaFuncSetAttribute(k_anterpolate_slab<T, NU, kAnterpBX>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kAnterpSmemBudget));
  MSM_NU_SWITCH_ALL(cudaFuncSetAttribute(k_anterp_tiles<T, NU, false>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(TileGeom<NU>::E3 * sizeof(T))));
  MSM_NU_SWITCH_ALL(cudaFuncSetAttribute(k_anterp_tiles<T, NU, true>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(TileGeom<NU>::E3 * sizeof(T))));
  MSM_NU_SWITCH_ALL(cudaFuncSetAttribute(k_restrict<T, NU>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         RestrictGeom<T, NU>::SMEM));
  MSM_NU_SWITCH_ALL(cudaFuncSetAttribute(k_prolong<T, NU>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (prolong_smem<T, NU>())));
  if (dev >= 0) done[dev] = true;
}

template <typename T>
void launch_adj_anterpolate(cudaStream_t s, const int M[3], const V4<T> *atoms,
                            const int *cell_sorted, const int *cell_start,
                            const SplineConsts<T> &sc, const V4<T> *dip, T *grid,
                            T *scratch, const int *fold_tab) {
  const int nt0 = (M[0] + kAT - 1) / kAT, nt1 = (M[1] + kAT - 1) / kAT,
            nt2 = (M[2] + kAT - 1) / kAT;
  const long n = (long)M[0] * M[1] * M[2];
  MSM_NU_SWITCH(sc.nu, (launch<KAnterpTiles<T, NU, true>, 32, 1>(s, k_anterp_tiles<T, NU, true>, nt0 * nt1 * nt2, 32, TileGeom<NU>::E3 * sizeof(T), M[0], M[1], M[2], nt1, nt2, atoms, cell_sorted, cell_start, sc,
                           scratch, dip)));
  MSM_NU_SWITCH(sc.nu, (launch<KAnterpFold<T, NU>, kThreads, 8>(s, k_anterp_fold<T, NU>, blocks_for(n), kThreads, 0, M[0], M[1], M[2], nt1, nt2, fold_tab, scratch, grid)));
}

template <typename T>
void launch_adj_interpolate(cudaStream_t s, int N, const int M[3], const V4<T> *atoms,
                            const int *cell_sorted, const int *gperm, const double *fbar,
                            const T *ed, const T *e1, const SplineConsts<T> &sc,
                            const Geometry &g, V4<T> *out_g, V4<T> *out_h) {
  MSM_NU_SWITCH(sc.nu, (k_adj_interp<T, NU><<<blocks_for(N), kThreads, 0, s>>>(
                           N, M[0], M[1], M[2], atoms, cell_sorted, gperm, fbar, ed, e1, sc,
                           g, out_g, out_h)));
}

template <typename T>
void launch_interpolate(cudaStream_t s, int N, const int M[3],
                        const V4<T> *atoms, const int *cell_sorted,
                        const T *grid, const SplineConsts<T> &sc,
                        const Geometry &g, V4<T> *out) {
  MSM_NU_SWITCH(sc.nu, (launch<KInterpolate<T, NU>, kThreads, interp_multi_blocks<T, NU>()>(s, k_interpolate<T, NU>, blocks_for(N), kThreads, 0, N, M[0], M[1], M[2], atoms, cell_sorted, grid, sc, g, out)));
}

template <typename T>
void launch_restrict(cudaStream_t s, const int Mf[3], const T *fine,
                     T *coarse, const double *J, int nu) {
  TwoScale js;
  for (int i = 0; i <= nu; ++i) js.J[i] = J[i];
  using Tl = RestrictTile<T>;
  const int C0 = Mf[0] / 2, C1 = Mf[1] / 2, C2 = Mf[2] / 2;
  const int blocks = ((C0 + Tl::CX - 1) / Tl::CX) * ((C1 + Tl::CY - 1) / Tl::CY) *
                     ((C2 + Tl::CZ - 1) / Tl::CZ);
  MSM_NU_SWITCH(nu, (launch<KRestrict<T, NU>, kSepThreads, 1>(s, k_restrict<T, NU>, blocks, kSepThreads, RestrictGeom<T, NU>::SMEM, Mf[0], Mf[1], Mf[2], fine, coarse, js)));
}

template <typename T>
void launch_prolong_add(cudaStream_t s, const int Mf[3], const T *coarse,
                        T *fine, const double *J, int nu) {
  TwoScale js;
  for (int i = 0; i <= nu; ++i) js.J[i] = J[i];
  const int blocks = ((Mf[0] + kPX - 1) / kPX) * ((Mf[1] + kPY - 1) / kPY) *
                     ((Mf[2] + kPZ - 1) / kPZ);
  MSM_NU_SWITCH(nu, (launch<KProlong<T, NU>, kSepThreads, 1>(s, k_prolong<T, NU>, blocks, kSepThreads, prolong_smem<T, NU>(), Mf[0], Mf[1], Mf[2], coarse, fine, js)));
}

int grid_dot_blocks(size_t n) {
  return (int)std::min<long>(1024, std::max<long>(1, ((long)n + kThreads - 1) / kThreads));
}

template <typename T>
void launch_grid_dot(cudaStream_t s, size_t n, const T *a, const T *b,
                     double *partials, int nparts) {
  launch<KGridDot<T>, kThreads, 8>(s, k_grid_dot<T>, nparts, kThreads, 0, (long)n, a, b, partials);
}

#define MSM_INST_GRID(T)                                                       \
  template void launch_anterpolate<T>(cudaStream_t, const int *,              \
                                      const V4<T> *, const int *, const int *,\
                                      const SplineConsts<T> &, T *, int,      \
                                      int *, long, T *, const int *);         \
  template void anterpolate_prepare<T>();                                     \
  template void launch_adj_anterpolate<T>(cudaStream_t, const int *, const V4<T> *,  \
                                          const int *, const int *,                 \
                                          const SplineConsts<T> &, const V4<T> *, T *, \
                                          T *, const int *);                        \
  template void launch_adj_interpolate<T>(cudaStream_t, int, const int *,           \
                                          const V4<T> *, const int *, const int *,  \
                                          const double *, const T *, const T *,     \
                                          const SplineConsts<T> &, const Geometry &, \
                                          V4<T> *, V4<T> *);                        \
  template void launch_interpolate<T>(cudaStream_t, int, const int *,         \
                                      const V4<T> *, const int *, const T *,  \
                                      const SplineConsts<T> &,                \
                                      const Geometry &, V4<T> *);             \
  template void launch_restrict<T>(cudaStream_t, const int *, const T *, T *, \
                                   const double *, int);                      \
  template void launch_prolong_add<T>(cudaStream_t, const int *, const T *,   \
                                      T *, const double *, int);              \
  template void launch_grid_dot<T>(cudaStream_t, size_t, const T *,           \
                                   const T *, double *, int);
MSM_INST_GRID(float)
MSM_INST_GRID(double)

}  // namespace msm
