// Short-range pair sum over atom clusters (the same sum as k_pair.cu:
// code/forcefield1.c:240-321 over the pairs of code/forcefield0.c:21-164).
//
// Layout. Pair cells are columns (cx, cy) of cells cz, z fastest, and every
// cell is sorted along z, so each column is one z-ordered run of atoms. A
// cluster is 8 consecutive atoms of a column; its atoms are stored relative
// to the origin of the cell of its first atom (FP32 in the mixed form, plus
// an FP64 copy for close pairs), padded with far-away, uncharged dummies. A
// unit is half a cluster (4 atoms) with its own bounding box.
//
// Sweep. One warp per i-cluster; lane = ii + 8 jq holds i-atom ii and
// j-atom jq of the current unit (an 8 x 4 pair tile per step). For every
// neighbour column (host list) and periodic image along the column, the
// candidate units are those of the clusters whose cells lie within K2 cells
// of the i-cluster's cells; they are tested 32 at a time, one per lane, box
// against box, the passing ones queued in shared memory with their FP32
// image shift, and the tiles of the queue evaluated by the whole warp. Every
// atom pair within the cutoff is summed once from each side (gather form:
// no atomics, fixed order, deterministic); per-column partial sums are added
// with compensation in the mixed form, and pairs closer than sqrt(close2)
// are queued per lane and summed in FP64 after the sweep.
#include <cstdlib>

#include "kernels.h"
#include "pair_fn.cuh"

namespace msm {
namespace {

constexpr int kWarps = 4;  // i-clusters per CTA
constexpr int kCloseCap = 8;
constexpr float kFar = 1e15f;

template <typename T> struct V3 { T x, y, z; };

// Bounding box test with a relative margin that covers the FP32 rounding of
// boxes and shifts (the exact per-pair test follows).
__device__ __forceinline__ bool box_near(const float4 &ic, const float4 &ih,
                                         const float4 &jc, const float4 &jh,
                                         float sx, float sy, float sz, float r2) {
  const float gx = fmaxf(fabsf(jc.x + sx - ic.x) - ih.x - jh.x, 0.f);
  const float gy = fmaxf(fabsf(jc.y + sy - ic.y) - ih.y - jh.y, 0.f);
  const float gz = fmaxf(fabsf(jc.z + sz - ic.z) - ih.z - jh.z, 0.f);
  return gx * gx + gy * gy + gz * gz < r2;
}

__device__ __forceinline__ int floor_div(int a, int n) {
  return a >= 0 ? a / n : -((-a + n - 1) / n);
}

// ---- cluster build: 8 threads per cluster ----
template <typename T>
__device__ __forceinline__ void cluster_fill_body(const BlockCtx &ctx, int maxcl, int ncol, int nc2, const int *__restrict__ start,
               const int *__restrict__ clstart, const int *__restrict__ pcs,
               const V4<double> *__restrict__ src64, double cz0, double cz1,
               double cz2, V4<T> *__restrict__ cpos, V4<double> *__restrict__ cpos64,
               ClusterInfo *__restrict__ info, UnitBox *__restrict__ ubox) {
  const long s = (long)ctx.b.x * blockDim.x + threadIdx.x;
  const int u = (int)(s >> 3), l = (int)(s & 7);
  const int total = clstart[ncol];
  const bool valid = u < maxcl && u < total;
  float lo[3] = {3e38f, 3e38f, 3e38f}, hi[3] = {-3e38f, -3e38f, -3e38f};
  int n = 0, a0 = 0, czf = 0, col = 0;
  if (valid) {
    int a = 0, b = ncol;  // last column with clstart[col] <= u
    while (b - a > 1) {
      const int m = (a + b) >> 1;
      if (clstart[m] <= u) a = m; else b = m;
    }
    col = a;
    const int cs = start[col * nc2], ce = start[(col + 1) * nc2];
    a0 = cs + 8 * (u - clstart[col]);
    n = min(8, ce - a0);
    czf = pcs[a0] % nc2;
    V4<T> p;
    if (l < n) {
      const V4<double> r = src64[a0 + l];
      const double dz = (double)(pcs[a0 + l] % nc2 - czf);
      V4<double> c;
      c.x = r.x + dz * cz0;
      c.y = r.y + dz * cz1;
      c.z = r.z + dz * cz2;
      c.w = r.w;
      p.x = (T)c.x;
      p.y = (T)c.y;
      p.z = (T)c.z;
      p.w = (T)c.w;
      if (cpos64) cpos64[s] = c;
      lo[0] = hi[0] = (float)p.x;
      lo[1] = hi[1] = (float)p.y;
      lo[2] = hi[2] = (float)p.z;
    } else {
      p.x = p.y = p.z = (T)kFar;
      p.w = T(0);
      if (cpos64) cpos64[s] = V4<double>{(double)kFar, (double)kFar, (double)kFar, 0.};
    }
    cpos[s] = p;
  }
  // half boxes (4 lanes), then the whole cluster (8 lanes)
  float hlo[3], hhi[3];
  for (int k = 0; k < 3; ++k) {
    for (int o = 1; o < 4; o <<= 1) {
      lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
      hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
    }
    hlo[k] = lo[k];
    hhi[k] = hi[k];
    lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], 4));
    hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], 4));
  }
  if (!valid) return;
  if ((l & 3) == 0) {
    UnitBox b;
    if (l < n) {
      b.c = make_float4(0.5f * (hlo[0] + hhi[0]), 0.5f * (hlo[1] + hhi[1]),
                        0.5f * (hlo[2] + hhi[2]), __int_as_float(czf));
      b.h = make_float4(0.5f * (hhi[0] - hlo[0]), 0.5f * (hhi[1] - hlo[1]),
                        0.5f * (hhi[2] - hlo[2]), 0.f);
    } else {  // empty unit: never near anything
      b.c = make_float4(kFar, kFar, kFar, __int_as_float(czf));
      b.h = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    ubox[2 * u + (l >> 2)] = b;
  }
  if (l == 0) {
    ClusterInfo ci;
    ci.first = a0;
    ci.n = n;
    ci.col = col;
    ci.czf = czf;
    ci.czl = pcs[a0 + n - 1] % nc2;
    ci.pad[0] = ci.pad[1] = ci.pad[2] = 0;
    ci.c = make_float4(0.5f * (lo[0] + hi[0]), 0.5f * (lo[1] + hi[1]),
                       0.5f * (lo[2] + hi[2]), 0.f);
    ci.h = make_float4(0.5f * (hi[0] - lo[0]), 0.5f * (hi[1] - lo[1]),
                       0.5f * (hi[2] - lo[2]), 0.f);
    info[u] = ci;
  }
}
template <typename T>
struct KClusterFill {
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { cluster_fill_body<T>(c, a...); }
};
template <typename T>
__global__ void __launch_bounds__(256)
k_cluster_fill(int maxcl, int ncol, int nc2, const int *__restrict__ start,
               const int *__restrict__ clstart, const int *__restrict__ pcs,
               const V4<double> *__restrict__ src64, double cz0, double cz1,
               double cz2, V4<T> *__restrict__ cpos, V4<double> *__restrict__ cpos64,
               ClusterInfo *__restrict__ info, UnitBox *__restrict__ ubox) {
  cluster_fill_body<T>(hw_ctx(), maxcl, ncol, nc2, start, clstart, pcs, src64, cz0, cz1, cz2, cpos, cpos64, info, ubox);
}

template <typename T, int NU>
__device__ __forceinline__ void pair_terms(const PairConsts<T> &pc, T r2, T qj,
                                           T &pot, T &fs) {
  T v, f;
  pair_radial<T, NU>(pc, r2, v, f);
  pot = qj * v;
  fs = qj * f;
}

// One pair in FP64 from FP64 cluster-frame positions and the FP64 shift of
// the j cluster's frame (close pairs of the mixed form).
template <int NU>
__device__ __forceinline__ void close_pair64(const PairConsts<float> &pc,
                                             const V4<double> &ai, const V4<double> &aj,
                                             double sx, double sy, double sz,
                                             double &fx, double &fy, double &fz,
                                             double &p) {
  const double ex = (aj.x + sx) - ai.x;
  const double ey = (aj.y + sy) - ai.y;
  const double ez = (aj.z + sz) - ai.z;
  const double d2 = ex * ex + ey * ey + ez * ez;
  double v, f;
  pair_radial64<NU>(pc, d2, v, f);
  p += aj.w * v;
  const double cf = aj.w * f;
  fx += cf * ex;
  fy += cf * ey;
  fz += cf * ez;
}

// One 8 x 4 tile: lane (ii, jq) takes pair (i-atom ii, j-atom jq of the
// queued unit, already shifted into the i-cluster's frame). Close pairs
// (mixed form) are recorded for the FP64 pass while the lane's record has
// room, else summed here in FP32. The atom itself is never a pair: the
// reference sums an atom's own periodic images in the constant coeff1
// (code/forcefield0.c:612-636). SELF: the box has a lattice vector shorter
// than a0, so the atom's images can reach the tile and every pair checks
// its slot; otherwise only the zero-shift atom (r2 == 0) can be itself.
template <typename T, int NU, bool MIXED, bool SELF>
__device__ __forceinline__ void tile(const PairConsts<T> &pc, const V4<T> &ai,
                                     const V4<T> &aj, const int *qunit, int e, int jq,
                                     int islot, const int *qcode, int2 *closeq,
                                     int &nclose, T &px, T &py, T &pz, T &pp) {
  const T dx = aj.x - ai.x, dy = aj.y - ai.y, dz = aj.z - ai.z;
  const T r2 = dx * dx + dy * dy + dz * dz;
  if (r2 < pc.a02) {
    if ((SELF || r2 == T(0)) && qunit[e] * 4 + jq == islot) return;
    if constexpr (MIXED) {
      if (r2 < pc.close2 && nclose < kCloseCap) {
        closeq[nclose++] = make_int2(qunit[e] * 4 + jq, qcode[e]);
        return;
      }
    }
    T pot, fs;
    pair_terms<T, NU>(pc, r2, aj.w, pot, fs);
    pp += pot;
    px += fs * dx;
    py += fs * dy;
    pz += fs * dz;
  }
}

// The two packed pairs' potential and force terms: rr the squared
// distances (replaced by a02 where the pair is masked), qj the j charges
// (zero where masked).
template <int NU>
__device__ __forceinline__ void tile2_sum(const PairConsts<float> &pc, const float2 &rr,
                                          const float2 &qj, const float2 &dx, const float2 &dy,
                                          const float2 &dz, float2 &px, float2 &py, float2 &pz,
                                          float2 &pp) {
  if constexpr (NU == 0) {  // PME kernel, packed (pair_fn.cuh)
    float2 v, f;
    pme_radial2(pc, rr, v, f);
    const float2 fs = __fmul2_rn(qj, f);
    pp = __ffma2_rn(qj, v, pp);
    px = __ffma2_rn(fs, dx, px);
    py = __ffma2_rn(fs, dy, py);
    pz = __ffma2_rn(fs, dz, pz);
  } else {
    const float2 s =
        __ffma2_rn(rr, make_float2(pc.inv_a02, pc.inv_a02), make_float2(-1.f, -1.f));
    float2 ts = make_float2(pc.tau[NU - 1], pc.tau[NU - 1]), t1 = make_float2(0.f, 0.f);
#pragma unroll
    for (int m = NU - 2; m >= 0; --m) {
      t1 = __ffma2_rn(s, t1, ts);
      ts = __ffma2_rn(s, ts, make_float2(pc.tau[m], pc.tau[m]));
    }
    const float2 rinv = make_float2(rsqrtf(rr.x), rsqrtf(rr.y));
    const float2 pot =
        __fmul2_rn(qj, __ffma2_rn(ts, make_float2(-pc.inv_a0, -pc.inv_a0), rinv));
    const float2 rinv3 = __fmul2_rn(__fmul2_rn(rinv, rinv), rinv);
    const float2 fs = __fmul2_rn(
        make_float2(-qj.x, -qj.y),
        __ffma2_rn(t1, make_float2(pc.two_inv_a03, pc.two_inv_a03), rinv3));
    pp = __fadd2_rn(pp, pot);
    px = __ffma2_rn(fs, dx, px);
    py = __ffma2_rn(fs, dy, py);
    pz = __ffma2_rn(fs, dz, pz);
  }
}

// Two tiles at once in the mixed form (queue entries e, e+1 on the two
// halves of packed FP32 registers: fma.rn.f32x2 and friends do two FP32
// operations per instruction, each rounded as the scalar one). X = (x_e,
// x_e+1, y_e, y_e+1), Y = (z_e, z_e+1, q_e, q_e+1). Pairs beyond the cutoff
// contribute exactly zero (their charge is masked, their r^2 replaced by a
// safe value); close pairs and the atom itself go the scalar way.
template <int NU, bool SELF>
__device__ __forceinline__ void tile2(const PairConsts<float> &pc, const V4<float> &ai,
                                      const float4 &X, const float4 &Y, const int *qunit,
                                      int e, int jq, int islot, const int *qcode,
                                      int2 *closeq, int &nclose, float2 &px, float2 &py,
                                      float2 &pz, float2 &pp) {
  const float2 nx = make_float2(-ai.x, -ai.x), ny = make_float2(-ai.y, -ai.y),
               nz = make_float2(-ai.z, -ai.z);
  const float2 dx = __fadd2_rn(make_float2(X.x, X.y), nx);
  const float2 dy = __fadd2_rn(make_float2(X.z, X.w), ny);
  const float2 dz = __fadd2_rn(make_float2(Y.x, Y.y), nz);
  float2 r2 = __fmul2_rn(dx, dx);
  r2 = __ffma2_rn(dy, dy, r2);
  r2 = __ffma2_rn(dz, dz, r2);
  // Warp-uniform fast path (about four steps in five on water): no lane
  // holds a close pair (nor the atom itself, r2 = 0 < close2), so every
  // pair is either summed here or beyond the cutoff, and out-of-range pairs
  // are masked without per-lane branches (the same values as below).
  if (!SELF && !__any_sync(0xffffffffu, fminf(r2.x, r2.y) < pc.close2)) {
    const float2 rr = make_float2(fminf(r2.x, pc.a02), fminf(r2.y, pc.a02));
    const float2 qj = make_float2(r2.x < pc.a02 ? Y.z : 0.f, r2.y < pc.a02 ? Y.w : 0.f);
    tile2_sum<NU>(pc, rr, qj, dx, dy, dz, px, py, pz, pp);
    return;
  }
  bool h0 = r2.x < pc.a02, h1 = r2.y < pc.a02;
  if constexpr (SELF) {
    if (h0 && qunit[e] * 4 + jq == islot) h0 = false;
    if (h1 && qunit[e + 1] * 4 + jq == islot) h1 = false;
  }
  if (!(h0 || h1)) return;
  // the atom itself is skipped; close pairs are recorded for the FP64 pass
  // while there is room (else they stay here, in FP32)
  auto consumed = [&](int ee, float r) {
    const int jslot = qunit[ee] * 4 + jq;
    if (r == 0.f && jslot == islot) return true;
    if (nclose < kCloseCap) {
      closeq[nclose++] = make_int2(jslot, qcode[ee]);
      return true;
    }
    return false;
  };
  if (h0 && r2.x < pc.close2 && consumed(e, r2.x)) h0 = false;
  if (h1 && r2.y < pc.close2 && consumed(e + 1, r2.y)) h1 = false;
  if (!(h0 || h1)) return;
  const float2 rr = make_float2(h0 ? r2.x : pc.a02, h1 ? r2.y : pc.a02);
  const float2 qj = make_float2(h0 ? Y.z : 0.f, h1 ? Y.w : 0.f);
  tile2_sum<NU>(pc, rr, qj, dx, dy, dz, px, py, pz, pp);
}

template <typename T, int NU, bool MIXED, bool SELF>
__device__ __forceinline__ void pair_clusters(const BlockCtx &ctx, const PairClusterArgs<T> &a,
                                              const PairConsts<T> &pc) {
  // passing units of the current batch: their 4 atoms shifted into the
  // i-cluster's frame, the unit index and the (column, image) code
  // (mixed form: entries interleaved in pairs, at qpk[w][e/2][8 jq ..] =
  // x_e, x_e+1, y_e, y_e+1, z_e, z_e+1, q_e, q_e+1; each pair's block padded to
  // 36 words so that the per-slot writes of one warp spread over the banks)
  constexpr int kPk = 36;
  __shared__ V4<T> qatoms[MIXED ? 1 : kWarps][MIXED ? 1 : 32][4];
  __shared__ __align__(16) float qpk[MIXED ? kWarps : 1][16][kPk];
  __shared__ int qunit[kWarps][32], qcode[kWarps][32];
  __shared__ int item_off[kWarps][32], item_u0[kWarps][32], item_code[kWarps][32];
  __shared__ int2 closeq[MIXED ? kWarps : 1][MIXED ? 32 * kCloseCap : 1];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int u = ctx.b.x * kWarps + warp;
  if (u >= a.maxcl || u >= a.clstart[a.ncol]) return;  // whole warp
  const ClusterInfo ci = a.info[u];
  const int ii = lane & 7, jq = lane >> 3;
  const int islot = u * 8 + ii;
  V4<T> ai = a.cpos[islot];
  if (ii >= ci.n) ai.x = ai.y = ai.z = -(T)kFar;
  const int cx = ci.col / a.nc1, cy = ci.col - cx * a.nc1;
  const unsigned lt = (1u << lane) - 1u;
  // cells along the column within K2 of the cluster's cells, split at the
  // periodic boundary into segments k (image k of the column)
  const int lo = ci.czf - a.K2, hi = ci.czl + a.K2;
  const int klo = floor_div(lo, a.nc2);
  const int nseg = floor_div(hi, a.nc2) - klo + 1;
  const int nitems = a.ncoloff * nseg;
  Acc<T> fx, fy, fz, ph;
  fx.zero();
  fy.zero();
  fz.zero();
  ph.zero();
  int nclose = 0;
  int2 *myclose = MIXED ? &closeq[MIXED ? warp : 0][lane * kCloseCap] : nullptr;
  double cfx = 0., cfy = 0., cfz = 0., cph = 0.;

  for (int i0 = 0; i0 < nitems; i0 += 32) {
    // Phase A: one (column, segment) item per lane -> its run of units
    int nun = 0, uu0 = 0, code = 0;
    const int it = i0 + lane;
    if (it < nitems) {
      const int o = nseg == 1 ? it : it / nseg;
      const int k = klo + (it - o * nseg);
      const int2 d = *reinterpret_cast<const int2 *>(&a.coloff[o].du);
      int x = cx + d.x, y = cy + d.y;
      while (x < 0) x += a.nc0;
      while (x >= a.nc0) x -= a.nc0;
      while (y < 0) y += a.nc1;
      while (y >= a.nc1) y -= a.nc1;
      const int col = x * a.nc1 + y;
      const int cb = col * a.nc2;
      const int c0 = max(lo, k * a.nc2) - k * a.nc2;
      const int c1 = min(hi, k * a.nc2 + a.nc2 - 1) - k * a.nc2;
      const int A = a.start[cb + c0], B = a.start[cb + c1 + 1];
      const int cs = a.start[cb], clb = a.clstart[col];
      if (A < B) {
        const int u0 = clb + ((A - cs) >> 3), u1 = clb + ((B - 1 - cs) >> 3);
        nun = 2 * (u1 - u0 + 1);
        uu0 = 2 * u0;
      }
      code = (o << 8) | (k + 128);
    }
    int incl = nun;
#pragma unroll
    for (int dd = 1; dd < 32; dd <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, dd);
      if (lane >= dd) incl += y;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    item_off[warp][lane] = incl - nun;
    item_u0[warp][lane] = uu0;
    item_code[warp][lane] = code;
    __syncwarp();
    // Phase B: the concatenated units, 32 at a time, box-tested per lane
    for (int b0 = 0; b0 < total; b0 += 32) {
      const int c = b0 + lane;
      bool pass = false;
      int ecode = 0, eunit = 0;
      T esx = 0, esy = 0, esz = 0;
      if (c < total) {
        int j = 0;  // last item starting at or before c
#pragma unroll
        for (int step = 16; step; step >>= 1)
          if (item_off[warp][j + step] <= c) j += step;
        const int unit = item_u0[warp][j] + (c - item_off[warp][j]);
        ecode = item_code[warp][j];
        const int o = ecode >> 8, k = (ecode & 255) - 128;
        const UnitBox ub = a.ubox[unit];
        const int dzc = __float_as_int(ub.c.w) + k * a.nc2 - ci.czf;
        const ColumnOffset &co = a.coloff[o];
        const double sx = co.base[0] + dzc * a.cz[0];
        const double sy = co.base[1] + dzc * a.cz[1];
        const double sz = co.base[2] + dzc * a.cz[2];
        pass = box_near(ci.c, ci.h, ub.c, ub.h, (float)sx, (float)sy, (float)sz, a.rbox2);
        eunit = unit;
        esx = (T)sx;
        esy = (T)sy;
        esz = (T)sz;
      }
      const unsigned m = __ballot_sync(0xffffffffu, pass);
      if (pass) {
        const int slot = __popc(m & lt);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          V4<T> v = a.cpos[eunit * 4 + q];
          v.x += esx;
          v.y += esy;
          v.z += esz;
          if constexpr (MIXED) {
            float *d = &qpk[warp][slot >> 1][8 * q + (slot & 1)];
            d[0] = v.x;
            d[2] = v.y;
            d[4] = v.z;
            d[6] = v.w;
          } else {
            qatoms[warp][slot][q] = v;
          }
        }
        qunit[warp][slot] = eunit;
        qcode[warp][slot] = ecode;
      }
      __syncwarp();
      const int nq = __popc(m);
      T px = 0, py = 0, pz = 0, pp = 0;
      const int *qu = qunit[warp], *qc = qcode[warp];
      int e = 0;
      if constexpr (MIXED) {
        float2 px2 = make_float2(0.f, 0.f), py2 = px2, pz2 = px2, pp2 = px2;
        for (; e + 2 <= nq; e += 2) {
          const float4 X = *reinterpret_cast<const float4 *>(&qpk[warp][e >> 1][8 * jq]);
          const float4 Y = *reinterpret_cast<const float4 *>(&qpk[warp][e >> 1][8 * jq + 4]);
          tile2<NU, SELF>(pc, ai, X, Y, qu, e, jq, islot, qc, myclose, nclose, px2, py2, pz2,
                          pp2);
        }
        px = px2.x + px2.y;
        py = py2.x + py2.y;
        pz = pz2.x + pz2.y;
        pp = pp2.x + pp2.y;
        if (e < nq) {  // the last, unpaired entry (even index: first half)
          const float *d = &qpk[warp][e >> 1][8 * jq];
          V4<T> aj;
          aj.x = d[0];
          aj.y = d[2];
          aj.z = d[4];
          aj.w = d[6];
          tile<T, NU, MIXED, SELF>(pc, ai, aj, qu, e, jq, islot, qc, myclose, nclose, px, py, pz,
                             pp);
        }
      } else {
        for (; e + 2 <= nq; e += 2) {
          const V4<T> a0 = qatoms[warp][e][jq], a1 = qatoms[warp][e + 1][jq];
          tile<T, NU, MIXED, SELF>(pc, ai, a0, qu, e, jq, islot, qc, myclose, nclose, px, py, pz,
                             pp);
          tile<T, NU, MIXED, SELF>(pc, ai, a1, qu, e + 1, jq, islot, qc, myclose, nclose, px, py,
                             pz, pp);
        }
        if (e < nq)
          tile<T, NU, MIXED, SELF>(pc, ai, qatoms[warp][e][jq], qu, e, jq, islot, qc, myclose,
                             nclose, px, py, pz, pp);
      }
      __syncwarp();
      if (MIXED) {
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
    __syncwarp();
  }
  if constexpr (MIXED) {
    // close pairs in FP64
    const V4<double> ai64 = a.cpos64[islot];
    for (int t = 0; t < nclose; ++t) {
      const int2 c = myclose[t];
      const int jslot = c.x, o = c.y >> 8, k = (c.y & 255) - 128;
      const ColumnOffset &co = a.coloff[o];
      const int dzc = a.info[jslot >> 3].czf + k * a.nc2 - ci.czf;
      close_pair64<NU>(pc, ai64, a.cpos64[jslot], co.base[0] + dzc * a.cz[0],
                       co.base[1] + dzc * a.cz[1], co.base[2] + dzc * a.cz[2], cfx,
                       cfy, cfz, cph);
    }
  }
  // the four j lanes of each i atom, in a fixed order
  T rx = fx.value(), ry = fy.value(), rz = fz.value(), rp = ph.value();
#pragma unroll
  for (int o = 8; o < 32; o <<= 1) {
    rx += __shfl_xor_sync(0xffffffffu, rx, o);
    ry += __shfl_xor_sync(0xffffffffu, ry, o);
    rz += __shfl_xor_sync(0xffffffffu, rz, o);
    rp += __shfl_xor_sync(0xffffffffu, rp, o);
    if constexpr (MIXED) {
      cfx += __shfl_xor_sync(0xffffffffu, cfx, o);
      cfy += __shfl_xor_sync(0xffffffffu, cfy, o);
      cfz += __shfl_xor_sync(0xffffffffu, cfz, o);
      cph += __shfl_xor_sync(0xffffffffu, cph, o);
    }
  }
  if (jq != 0 || ii >= ci.n) return;
  V4<T> r;
  if constexpr (MIXED) {
    const double qi = a.cpos64[islot].w;
    r.x = (T)(qi * ((double)rx + cfx));
    r.y = (T)(qi * ((double)ry + cfy));
    r.z = (T)(qi * ((double)rz + cfz));
    r.w = (T)((double)rp + cph);
  } else {
    r.x = ai.w * rx;
    r.y = ai.w * ry;
    r.z = ai.w * rz;
    r.w = rp;
  }
  a.out[ci.first + ii] = r;
}

// ---- lanes over j atoms, the 8 i atoms in registers ----
//
// One warp per i-cluster as above, but lane = one j atom at a time and every
// lane holds all 8 i atoms: a j atom costs one shared-memory load for 8 pairs
// (in the mixed form evaluated two at a time in packed FP32: 4 independent
// pair groups per j for the pipelines to overlap). Candidates are single
// atoms: each (column, image) item's run of atoms (for orthorhombic boxes
// only the cells that the cutoff sphere around the i-cluster box reaches
// through the column's xy gap) is box-tested atom by atom against the
// i-cluster's box, and passing atoms are queued in one of two rings: far ones
// (farther than the close distance from the box: no pair of theirs can be
// close or the atom itself) go the lean way; near ones are checked pair by
// pair for the atom itself (skipped) and, in the mixed form, for close pairs
// (recorded per lane, summed in FP64 after the sweep). Gather form: every
// pair is summed once from each side; the lanes' partial sums are combined
// by a fixed butterfly, so the result does not depend on timing.
constexpr int kRing = 64;        // entries per queue ring (a warp adds <= 32 at a time)

// One warp's (column, image) items of the current Phase A batch
struct JlItems {
  int off[32], s0[32], a0[32], code[32];
  double shift[32][3];
};

// Item `it` of i-cluster ci's candidates: the column offset o = it / nseg
// and periodic image k along the column; its run of sorted atoms [A, A + nat)
// (the cells along the column within K2 of the cluster's cells, for
// orthorhombic boxes only those the cutoff sphere around the cluster's box
// reaches through the column's xy gap), the cluster slot s0 of its first
// atom, its code (o << 8 | k + 128) and the FP64 shift of a j cluster frame
// at cell 0 of the column into the i-cluster's frame.
template <typename T>
__device__ __forceinline__ void jl_item(const PairClusterArgs<T> &a, const ClusterInfo &ci,
                                        int cx, int cy, int lo, int hi, int klo, int nseg,
                                        int it, int &A, int &nat, int &s0, int &code,
                                        double &shx, double &shy, double &shz) {
  const int o = nseg == 1 ? it : it / nseg;
  const int k = klo + (it - o * nseg);
  const ColumnOffset &co = a.coloff[o];
  int x = cx + co.du, y = cy + co.dv;
  while (x < 0) x += a.nc0;
  while (x >= a.nc0) x -= a.nc0;
  while (y < 0) y += a.nc1;
  while (y >= a.nc1) y -= a.nc1;
  int wlo = lo, whi = hi;
  if (a.ortho) {
    // the column's slab in the i frame: x in [bx, bx + cw0), y likewise
    const float bx = (float)co.base[0], by = (float)co.base[1];
    const float gx =
        fmaxf(fmaxf(bx - (ci.c.x + ci.h.x), (ci.c.x - ci.h.x) - (bx + a.cw[0])), 0.f);
    const float gy =
        fmaxf(fmaxf(by - (ci.c.y + ci.h.y), (ci.c.y - ci.h.y) - (by + a.cw[1])), 0.f);
    const float rem = a.rbox2 - gx * gx - gy * gy;
    if (rem <= 0.f) {
      whi = wlo - 1;
    } else {
      const float hw = sqrtf(rem) + 1e-3f;
      wlo = max(wlo, ci.czf + (int)floorf((ci.c.z - ci.h.z - hw) / a.cw[2]));
      whi = min(whi, ci.czf + (int)floorf((ci.c.z + ci.h.z + hw) / a.cw[2]));
    }
  }
  const int col = x * a.nc1 + y;
  const int cb = col * a.nc2;
  const int c0 = max(wlo, k * a.nc2) - k * a.nc2;
  const int c1 = min(whi, k * a.nc2 + a.nc2 - 1) - k * a.nc2;
  nat = 0;
  s0 = 0;
  A = 0;
  if (c0 <= c1) {
    A = a.start[cb + c0];
    const int B = a.start[cb + c1 + 1];
    if (A < B) {
      nat = B - A;
      s0 = 8 * a.clstart[col] + (A - a.start[cb]);
    }
  }
  code = (o << 8) | (k + 128);
  const double dz = (double)(k * a.nc2 - ci.czf);
  shx = co.base[0] + dz * a.cz[0];
  shy = co.base[1] + dz * a.cz[1];
  shz = co.base[2] + dz * a.cz[2];
}

// The candidate j atoms of i-cluster u for one warp. Phase A: the (column,
// periodic image) items, 32 at a time, one per lane: each item's run of
// sorted atoms (the cells along the column within K2 of the cluster's cells,
// for orthorhombic boxes only those the cutoff sphere around the cluster's
// box reaches through the column's xy gap). Phase B: the concatenated runs,
// 32 atoms at a time, one per lane: the atom is shifted into the i-cluster's
// frame and tested against its box. `batch(pass, near, J, jslot, jcode,
// selfk, sorted)` is called by the whole warp once per batch: pass, the
// atom is within the cutoff (plus margin) of the box; near, within the close
// distance of it, or it is an atom of the cluster itself (selfk = its slot
// in the cluster, else -1); J the shifted position and charge; jslot the
// atom's cluster slot, jcode its item's (column offset << 8 | image + 128),
// sorted its index in pair-cell order.
template <typename T, bool SELF, typename Batch>
__device__ __forceinline__ void jl_sweep(const PairClusterArgs<T> &a, const ClusterInfo &ci,
                                         int u, int lane, JlItems &it_sh, Batch &&batch) {
  const int cx = ci.col / a.nc1, cy = ci.col - cx * a.nc1;
  const int lo = ci.czf - a.K2, hi = ci.czl + a.K2;
  const int klo = floor_div(lo, a.nc2);
  const int nseg = floor_div(hi, a.nc2) - klo + 1;
  const int nitems = a.ncoloff * nseg;
  for (int i0 = 0; i0 < nitems; i0 += 32) {
    int nat = 0, s0 = 0, A = 0, code = 0;
    double shx = 0., shy = 0., shz = 0.;
    const int it = i0 + lane;
    if (it < nitems)
      jl_item(a, ci, cx, cy, lo, hi, klo, nseg, it, A, nat, s0, code, shx, shy, shz);
    int incl = nat;
#pragma unroll
    for (int dd = 1; dd < 32; dd <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, dd);
      if (lane >= dd) incl += y;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    it_sh.off[lane] = incl - nat;
    it_sh.s0[lane] = s0;
    it_sh.a0[lane] = A;
    it_sh.code[lane] = code;
    it_sh.shift[lane][0] = shx;
    it_sh.shift[lane][1] = shy;
    it_sh.shift[lane][2] = shz;
    __syncwarp();
    for (int b0 = 0; b0 < total; b0 += 32) {
      const int c = b0 + lane;
      bool pass = false, near = false;
      V4<T> J{};
      int jslot = 0, jcode = 0, selfk = -1, sorted = 0;
      if (c < total) {
        int j = 0;  // last item starting at or before c
#pragma unroll
        for (int step = 16; step; step >>= 1)
          if (it_sh.off[j + step] <= c) j += step;
        jslot = it_sh.s0[j] + (c - it_sh.off[j]);
        sorted = it_sh.a0[j] + (c - it_sh.off[j]);
        jcode = it_sh.code[j];
        J = a.cpos[jslot];
        const int jc = jslot >> 3;
        const double czj = (double)__float_as_int(a.ubox[2 * jc].c.w);
        J.x += (T)(it_sh.shift[j][0] + czj * a.cz[0]);
        J.y += (T)(it_sh.shift[j][1] + czj * a.cz[1]);
        J.z += (T)(it_sh.shift[j][2] + czj * a.cz[2]);
        const float gx = fmaxf(fabsf((float)J.x - ci.c.x) - ci.h.x, 0.f);
        const float gy = fmaxf(fabsf((float)J.y - ci.c.y) - ci.h.y, 0.f);
        const float gz = fmaxf(fabsf((float)J.z - ci.c.z) - ci.h.z, 0.f);
        const float g2 = gx * gx + gy * gy + gz * gz;
        pass = g2 < a.rbox2;
        near = g2 < a.rnear2;
        if (jc == u && (SELF || ((jcode >> 8) == a.ozero && (jcode & 255) == 128))) {
          selfk = jslot & 7;
          near = true;
        }
      }
      batch(pass, near, J, jslot, jcode, selfk, sorted);
    }
  }
}

// ---- unit lists: the candidate search of the pair kernels, ahead of them ----
//
// One warp per i-cluster, few registers (many warps per SM hide the
// latencies of the search): the items of jl_item, their atom runs widened to
// whole units (half clusters, 4 slots; the widening adds atoms of the same
// column and image outside the window, i.e. beyond the cutoff, and dummy
// slots, all of which the pair kernels' cutoff test rejects), and every unit
// box-tested against the i-cluster's box, 32 at a time. Passing units are
// written as {unit, code} in a fixed order (item, then unit): far ones from
// the front of the cluster's region, near ones (box within the close
// distance, or a unit of the cluster itself) from the back.
struct ListItems {
  int off[32], u0[32], code[32];
  double shift[32][3];
};

template <typename T>
__global__ void __launch_bounds__(kWarps * 32)
k_pair_list(PairClusterArgs<T> a) {
  __shared__ ListItems sh[kWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int u = blockIdx.x * kWarps + warp;
  if (u >= a.maxcl || u >= a.clstart[a.ncol]) return;  // whole warp
  const ClusterInfo ci = a.info[u];
  const unsigned lt = (1u << lane) - 1u;
  int2 *reg = a.list + (size_t)u * a.lcap;
  int nf = 0, nn = 0;
  const int cx = ci.col / a.nc1, cy = ci.col - cx * a.nc1;
  const int lo = ci.czf - a.K2, hi = ci.czl + a.K2;
  const int klo = floor_div(lo, a.nc2);
  const int nseg = floor_div(hi, a.nc2) - klo + 1;
  const int nitems = a.ncoloff * nseg;
  ListItems &it_sh = sh[warp];
  for (int i0 = 0; i0 < nitems; i0 += 32) {
    int A = 0, nat = 0, s0 = 0, code = 0, nun = 0, u0 = 0;
    double shx = 0., shy = 0., shz = 0.;
    const int it = i0 + lane;
    if (it < nitems) {
      jl_item(a, ci, cx, cy, lo, hi, klo, nseg, it, A, nat, s0, code, shx, shy, shz);
      if (nat > 0) {
        u0 = s0 >> 2;
        nun = ((s0 + nat - 1) >> 2) - u0 + 1;
      }
    }
    int incl = nun;
#pragma unroll
    for (int dd = 1; dd < 32; dd <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, dd);
      if (lane >= dd) incl += y;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    it_sh.off[lane] = incl - nun;
    it_sh.u0[lane] = u0;
    it_sh.code[lane] = code;
    it_sh.shift[lane][0] = shx;
    it_sh.shift[lane][1] = shy;
    it_sh.shift[lane][2] = shz;
    __syncwarp();
    for (int b0 = 0; b0 < total; b0 += 32) {
      const int c = b0 + lane;
      bool pass = false, near = false;
      int unit = 0, ucode = 0;
      if (c < total) {
        int j = 0;  // last item starting at or before c
#pragma unroll
        for (int step = 16; step; step >>= 1)
          if (it_sh.off[j + step] <= c) j += step;
        unit = it_sh.u0[j] + (c - it_sh.off[j]);
        const UnitBox ub = a.ubox[unit];
        // entry: item code (18 bits) and the first cell of the unit's cluster
        ucode = it_sh.code[j] | (__float_as_int(ub.c.w) << 18);
        const double czj = (double)__float_as_int(ub.c.w);
        const float sx = (float)(it_sh.shift[j][0] + czj * a.cz[0]);
        const float sy = (float)(it_sh.shift[j][1] + czj * a.cz[1]);
        const float sz = (float)(it_sh.shift[j][2] + czj * a.cz[2]);
        pass = box_near(ci.c, ci.h, ub.c, ub.h, sx, sy, sz, a.rbox2);
        near = box_near(ci.c, ci.h, ub.c, ub.h, sx, sy, sz, a.rnear2) || (unit >> 1) == u;
        if (pass && !near) {
          // far unit: which of its 4 atoms are within the cutoff of the box
          unsigned m4 = 0;
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const V4<T> at = a.cpos[4 * unit + q];
            const float gx = fmaxf(fabsf((float)at.x + sx - ci.c.x) - ci.h.x, 0.f);
            const float gy = fmaxf(fabsf((float)at.y + sy - ci.c.y) - ci.h.y, 0.f);
            const float gz = fmaxf(fabsf((float)at.z + sz - ci.c.z) - ci.h.z, 0.f);
            if (gx * gx + gy * gy + gz * gz < a.rbox2) m4 |= 1u << q;
          }
          ucode |= (int)(m4 << 27);
          pass = m4 != 0;
        }
      }
      const unsigned mf = __ballot_sync(0xffffffffu, pass && !near);
      const unsigned mn = __ballot_sync(0xffffffffu, pass && near);
      if (pass && !near) {
        const int e = nf + __popc(mf & lt);
        if (e < a.lcap) reg[e] = make_int2(unit, ucode);
      }
      if (pass && near) {
        const int e = nn + __popc(mn & lt);
        if (e < a.lcap) reg[a.lcap - 1 - e] = make_int2(unit, ucode);
      }
      nf += __popc(mf);
      nn += __popc(mn);
    }
    __syncwarp();
  }
  if (lane == 0) a.lcnt[u] = make_int2(nf, nn);
}

// lanes' 32 partial sums -> lane l holds the total of value l (fixed order)
template <typename T>
__device__ __forceinline__ T butterfly32(T (&v)[32], int lane) {
#pragma unroll
  for (int sft = 16; sft >= 1; sft >>= 1) {
    const bool up = (lane & sft) != 0;
#pragma unroll
    for (int k = 0; k < sft; ++k) {
      const T send = up ? v[k] : v[k + sft];
      const T keep = up ? v[k + sft] : v[k];
      v[k] = keep + __shfl_xor_sync(0xffffffffu, send, sft);
    }
  }
  return v[0];
}

// The far atoms of a cluster's unit list, 32 per step: the entries' atom
// masks are compacted into a per-warp ring of atom slots (32 entries at a
// time, in list order, each batch of entries loaded one refill ahead), and
// each step's atom loads are issued before the previous step's pairs. `load(slot)` fetches an atom's data, `use(data,
// y, valid)` evaluates it (every lane, every step; invalid lanes carry none).
constexpr int kAtomRing = 256;
template <typename Data, typename Load, typename Use>
__device__ __forceinline__ void far_atoms(const int2 *reg, int nf, int lane, int *rslot,
                                          int *ry, Load &&load, Use &&use) {
  unsigned head = 0, tail = 0;
  int next_e = 0;
  // the next 32 entries, loaded one refill ahead (the lists live in DRAM)
  int2 en_n = lane < nf ? reg[lane] : make_int2(0, 0);
  auto produce = [&]() {
    const int e = next_e + lane;
    const int2 en = en_n;
    en_n = e + 32 < nf ? reg[e + 32] : make_int2(0, 0);
    const unsigned m4 = e < nf ? ((unsigned)en.y >> 27) & 15u : 0u;
    int incl = __popc(m4);
#pragma unroll
    for (int dd = 1; dd < 32; dd <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, dd);
      if (lane >= dd) incl += y;
    }
    const int tot = __shfl_sync(0xffffffffu, incl, 31);
    int at = tail + incl - __popc(m4);
    for (unsigned m = m4; m; m &= m - 1) {
      const int q = __ffs(m) - 1;
      rslot[at & (kAtomRing - 1)] = 4 * en.x + q;
      ry[at & (kAtomRing - 1)] = en.y;
      ++at;
    }
    tail += tot;
    next_e += 32;
    __syncwarp();
  };
  while (tail - head < 64 && next_e < nf) produce();
  unsigned idx = head + lane;
  bool v1 = idx < tail;
  int y1 = v1 ? ry[idx & (kAtomRing - 1)] : 0;
  Data d1 = load(v1 ? rslot[idx & (kAtomRing - 1)] : -1);
  while (head < tail) {
    const bool v = v1;
    const int y = y1;
    const Data d = d1;
    head = min(head + 32, tail);
    while (tail - head < 64 && next_e < nf) produce();
    idx = head + lane;
    v1 = idx < tail;
    y1 = v1 ? ry[idx & (kAtomRing - 1)] : 0;
    d1 = load(v1 ? rslot[idx & (kAtomRing - 1)] : -1);
    use(d, y, v);
  }
}

// A list atom (cluster-frame position `raw`) shifted into the frame of the
// i-cluster ci by the FP64 shift of its cluster's frame (entry y: item code
// and the cluster's first cell), rounded once.
template <typename T>
__device__ __forceinline__ V4<T> list_shifted(const PairClusterArgs<T> &a, const ClusterInfo &ci,
                                              V4<T> raw, int y) {
  const int o = (y >> 8) & 1023, k = (y & 255) - 128;
  const ColumnOffset &co = a.coloff[o];
  const int dzc = ((y >> 18) & 511) + k * a.nc2 - ci.czf;
  raw.x += (T)(co.base[0] + dzc * a.cz[0]);
  raw.y += (T)(co.base[1] + dzc * a.cz[1]);
  raw.z += (T)(co.base[2] + dzc * a.cz[2]);
  return raw;
}

// ---- adjoint short-range pass on the same sweep (mixed form) ----
// Per atom k, d = r_j - r_k (the short-range terms of dL/dq_k and dL/dr_k,
// as k_adjoint.cu's k_adj_pair computes them):
//   E_k = sum_j q_j g1 d,  psi_k = sum_j q_j g1 (Fbar_j . d),
//   h_k = sum_j q_j [g1 (Fbar_j - Fbar_k) + g2 d (d . (Fbar_j - Fbar_k))],
//   g1 = -1/r^3 - (2/a0^3) tau'(s),  g2 = 3/r^5 - (4/a0^5) tau''(s).
// Lanes over j atoms with the 8 i atoms (position and Fbar) in registers,
// packed FP32 as in the forward; the atom itself skipped at every image
// that reaches it (entries of the i-cluster take the checked path).
template <int NU>
struct AdjLane {
  float2 nix[4], niy[4], niz[4], nfx[4], nfy[4], nfz[4];  // -position, -Fbar
  float2 ex[4], ey[4], ez[4], ps[4], hx[4], hy[4], hz[4];
  template <bool SELFCHECK>
  __device__ __forceinline__ void pairs(const PairConsts<float> &pc, const V4<float> &J,
                                        const V4<float> &F, int selfk) {
    const float2 jx = make_float2(J.x, J.x), jy = make_float2(J.y, J.y),
                 jz = make_float2(J.z, J.z);
    const float2 Fx = make_float2(F.x, F.x), Fy = make_float2(F.y, F.y),
                 Fz = make_float2(F.z, F.z);
    const float c2 = 2.f * pc.two_inv_a03 * pc.inv_a02;  // 4 / a0^5
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      const float2 dx = __fadd2_rn(jx, nix[p]);
      const float2 dy = __fadd2_rn(jy, niy[p]);
      const float2 dz = __fadd2_rn(jz, niz[p]);
      float2 r2 = __fmul2_rn(dx, dx);
      r2 = __ffma2_rn(dy, dy, r2);
      r2 = __ffma2_rn(dz, dz, r2);
      bool h0 = r2.x < pc.a02, h1 = r2.y < pc.a02;
      if constexpr (SELFCHECK) {
        if (selfk == 2 * p) h0 = false;
        if (selfk == 2 * p + 1) h1 = false;
      }
      const float2 rr = make_float2(h0 ? r2.x : pc.a02, h1 ? r2.y : pc.a02);
      const float2 qj = make_float2(h0 ? J.w : 0.f, h1 ? J.w : 0.f);
      const float2 s = __ffma2_rn(rr, make_float2(pc.inv_a02, pc.inv_a02),
                                  make_float2(-1.f, -1.f));
      // tau'(s) and tau''(s)/2 by independent Horner chains
      float2 p1 = make_float2((NU - 1) * pc.tau[NU - 1], (NU - 1) * pc.tau[NU - 1]);
      const float h2 = 0.5f * (NU - 1) * (NU - 2) * pc.tau[NU - 1];
      float2 p2 = make_float2(h2, h2);
#pragma unroll
      for (int m = NU - 2; m >= 1; --m) {
        p1 = __ffma2_rn(s, p1, make_float2(m * pc.tau[m], m * pc.tau[m]));
        if (m >= 2) {
          const float cm = 0.5f * m * (m - 1) * pc.tau[m];
          p2 = __ffma2_rn(s, p2, make_float2(cm, cm));
        }
      }
      const float2 rinv = make_float2(rsqrtf(rr.x), rsqrtf(rr.y));
      const float2 rinv2 = __fmul2_rn(rinv, rinv);
      const float2 rinv3 = __fmul2_rn(rinv2, rinv);
      // g1 = -(rinv3 + p1 2/a0^3); g2 = 3 rinv3 rinv2 - 2 p2 (4/a0^5)
      const float2 g1 = __fmul2_rn(
          __ffma2_rn(p1, make_float2(pc.two_inv_a03, pc.two_inv_a03), rinv3),
          make_float2(-1.f, -1.f));
      const float2 g2 = __ffma2_rn(p2, make_float2(-2.f * c2, -2.f * c2),
                                   __fmul2_rn(__fmul2_rn(rinv3, rinv2), make_float2(3.f, 3.f)));
      const float2 w1 = __fmul2_rn(qj, g1);
      ex[p] = __ffma2_rn(w1, dx, ex[p]);
      ey[p] = __ffma2_rn(w1, dy, ey[p]);
      ez[p] = __ffma2_rn(w1, dz, ez[p]);
      float2 fd = __fmul2_rn(Fx, dx);
      fd = __ffma2_rn(Fy, dy, fd);
      fd = __ffma2_rn(Fz, dz, fd);
      ps[p] = __ffma2_rn(w1, fd, ps[p]);
      const float2 Dx = __fadd2_rn(Fx, nfx[p]), Dy = __fadd2_rn(Fy, nfy[p]),
                   Dz = __fadd2_rn(Fz, nfz[p]);
      float2 dD = __fmul2_rn(dx, Dx);
      dD = __ffma2_rn(dy, Dy, dD);
      dD = __ffma2_rn(dz, Dz, dD);
      const float2 w2 = __fmul2_rn(__fmul2_rn(qj, g2), dD);
      hx[p] = __ffma2_rn(w2, dx, __ffma2_rn(w1, Dx, hx[p]));
      hy[p] = __ffma2_rn(w2, dy, __ffma2_rn(w1, Dy, hy[p]));
      hz[p] = __ffma2_rn(w2, dz, __ffma2_rn(w1, Dz, hz[p]));
    }
  }
};

// Fbar in cluster-slot order (zero for the dummy slots): one thread per slot
__global__ void __launch_bounds__(256)
k_slot_gather(int maxcl, const int *__restrict__ ncl, const ClusterInfo *__restrict__ info,
              const V4<float> *__restrict__ fbs, V4<float> *__restrict__ fslot) {
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= 8L * maxcl) return;
  const int c = (int)(s >> 3), i = (int)(s & 7);
  V4<float> f{0.f, 0.f, 0.f, 0.f};
  if (c < *ncl) {
    const ClusterInfo &ci = info[c];
    if (i < ci.n) f = fbs[ci.first + i];
  }
  fslot[s] = f;
}

struct AdjWarpBufs {
  int rslot[256], ry[256];
  V4<float> far[kRing][2], self[kRing][2];
};
struct AdjShared {
  JlItems items[kWarps];
  AdjWarpBufs w[kWarps];
};

template <int NU, bool SELF>
__global__ void __launch_bounds__(kWarps * 32)
k_adj_pair_jl(PairClusterArgs<float> a, PairConsts<float> pc, const V4<float> *__restrict__ fbs,
              const V4<float> *__restrict__ fslot, V4<float> *__restrict__ out_a,
              V4<float> *__restrict__ out_b) {
  __shared__ AdjShared sh;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int u = blockIdx.x * kWarps + warp;
  if (u >= a.maxcl || u >= a.clstart[a.ncol]) return;  // whole warp
  const ClusterInfo ci = a.info[u];
  const unsigned lt = (1u << lane) - 1u;
  AdjLane<NU> L;
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    V4<float> a0 = a.cpos[u * 8 + 2 * p], a1 = a.cpos[u * 8 + 2 * p + 1];
    V4<float> f0{0.f, 0.f, 0.f, 0.f}, f1 = f0;
    if (2 * p < ci.n) f0 = fbs[ci.first + 2 * p];
    else a0.x = a0.y = a0.z = -kFar;
    if (2 * p + 1 < ci.n) f1 = fbs[ci.first + 2 * p + 1];
    else a1.x = a1.y = a1.z = -kFar;
    L.nix[p] = make_float2(-a0.x, -a1.x);
    L.niy[p] = make_float2(-a0.y, -a1.y);
    L.niz[p] = make_float2(-a0.z, -a1.z);
    L.nfx[p] = make_float2(-f0.x, -f1.x);
    L.nfy[p] = make_float2(-f0.y, -f1.y);
    L.nfz[p] = make_float2(-f0.z, -f1.z);
    L.ex[p] = L.ey[p] = L.ez[p] = L.ps[p] = L.hx[p] = L.hy[p] = L.hz[p] =
        make_float2(0.f, 0.f);
  }
  unsigned fhead = 0, ftail = 0, shead = 0, stail = 0;
  const V4<float> dummy{kFar, kFar, kFar, 0.f};
  auto far_step = [&](int cnt) {
    const int e = (fhead + lane) & (kRing - 1);
    V4<float> J = sh.w[warp].far[e][0], F = sh.w[warp].far[e][1];
    if (lane >= cnt) {  // no entry: zero charge and Fbar (stale slots may hold anything)
      J = dummy;
      F = V4<float>{0.f, 0.f, 0.f, 0.f};
    }
    L.template pairs<false>(pc, J, F, -1);
    fhead += cnt;
  };
  auto self_step = [&](int cnt) {
    const int e = (shead + lane) & (kRing - 1);
    V4<float> J = sh.w[warp].self[e][0], F = sh.w[warp].self[e][1];
    if (lane >= cnt) {
      J = dummy;
      F = V4<float>{0.f, 0.f, 0.f, __int_as_float(-1)};
    }
    L.template pairs<true>(pc, J, F, __float_as_int(F.w));
    shead += cnt;
  };
  bool sweep = true;
  if (a.list) {  // the cluster's unit list (k_pair_list)
    const int2 cnt = a.lcnt[u];
    if (cnt.x + cnt.y <= a.lcap) {
      sweep = false;
      const int2 *reg = a.list + (size_t)u * a.lcap;
      struct AtomF {
        V4<float> raw, F;
      };
      far_atoms<AtomF>(
          reg, cnt.x, lane, sh.w[warp].rslot, sh.w[warp].ry,
          [&](int slot) {
            AtomF d{dummy, V4<float>{0.f, 0.f, 0.f, 0.f}};
            if (slot >= 0) {
              d.raw = a.cpos[slot];
              d.F = fslot[slot];
            }
            return d;
          },
          [&](const AtomF &d, int y, bool v) {
            const V4<float> J = v ? list_shifted(a, ci, d.raw, y) : dummy;
            L.template pairs<false>(pc, J, d.F, -1);
          });
      const int n = cnt.y;
      auto entry = [&](int e) { return e < n ? reg[a.lcap - 1 - e] : make_int2(-1, 0); };
      int2 en1 = entry(lane >> 2), en2 = entry(8 + (lane >> 2));
      V4<float> raw1 = en1.x >= 0 ? a.cpos[4 * en1.x + (lane & 3)] : dummy;
      V4<float> f1 = en1.x >= 0 ? fslot[4 * en1.x + (lane & 3)] : V4<float>{0.f, 0.f, 0.f, 0.f};
      for (int e0 = 0; e0 < n; e0 += 8) {
        const int2 en = en1;
        const V4<float> raw = raw1, F = f1;
        en1 = en2;
        raw1 = en1.x >= 0 ? a.cpos[4 * en1.x + (lane & 3)] : dummy;
        f1 = en1.x >= 0 ? fslot[4 * en1.x + (lane & 3)] : V4<float>{0.f, 0.f, 0.f, 0.f};
        en2 = entry(e0 + 16 + (lane >> 2));
        const V4<float> J = en.x >= 0 ? list_shifted(a, ci, raw, en.y) : dummy;
        const int jslot = 4 * en.x + (lane & 3), jcode = en.y & 0x3ffff;
        int selfk = -1;
        if (en.x >= 0 && (jslot >> 3) == u &&
            (SELF || ((jcode >> 8) == a.ozero && (jcode & 255) == 128)))
          selfk = jslot & 7;
        L.template pairs<true>(pc, J, F, selfk);
      }
    }
  }
  if (sweep) {
  jl_sweep<float, SELF>(a, ci, u, lane, sh.items[warp],
                        [&](bool pass, bool, const V4<float> &J, int, int, int selfk,
                            int sorted) {
    V4<float> F{0.f, 0.f, 0.f, 0.f};
    if (pass) F = fbs[sorted];
    F.w = __int_as_float(selfk);
    const bool own = selfk >= 0;
    const unsigned mf = __ballot_sync(0xffffffffu, pass && !own);
    const unsigned ms = __ballot_sync(0xffffffffu, pass && own);
    if (pass && !own) {
      const int e = (ftail + __popc(mf & lt)) & (kRing - 1);
      sh.w[warp].far[e][0] = J;
      sh.w[warp].far[e][1] = F;
    }
    if (pass && own) {
      const int e = (stail + __popc(ms & lt)) & (kRing - 1);
      sh.w[warp].self[e][0] = J;
      sh.w[warp].self[e][1] = F;
    }
    ftail += __popc(mf);
    stail += __popc(ms);
    __syncwarp();
    if (ftail - fhead >= 32) far_step(32);
    if (stail - shead >= 32) self_step(32);
    __syncwarp();
  });
  if (ftail != fhead) far_step((int)(ftail - fhead));
  if (stail != shead) self_step((int)(stail - shead));
  }

  const int i = lane & 7, c = lane >> 3;
  float v[32];
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    v[2 * p] = L.ex[p].x;
    v[2 * p + 1] = L.ex[p].y;
    v[8 + 2 * p] = L.ey[p].x;
    v[8 + 2 * p + 1] = L.ey[p].y;
    v[16 + 2 * p] = L.ez[p].x;
    v[16 + 2 * p + 1] = L.ez[p].y;
    v[24 + 2 * p] = L.ps[p].x;
    v[24 + 2 * p + 1] = L.ps[p].y;
  }
  const float ra = butterfly32(v, lane);
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    v[2 * p] = L.hx[p].x;
    v[2 * p + 1] = L.hx[p].y;
    v[8 + 2 * p] = L.hy[p].x;
    v[8 + 2 * p + 1] = L.hy[p].y;
    v[16 + 2 * p] = L.hz[p].x;
    v[16 + 2 * p + 1] = L.hz[p].y;
    v[24 + 2 * p] = 0.f;
    v[24 + 2 * p + 1] = 0.f;
  }
  const float rb = butterfly32(v, lane);
  if (i >= ci.n) return;
  reinterpret_cast<float *>(&out_a[ci.first + i])[c] = ra;
  reinterpret_cast<float *>(&out_b[ci.first + i])[c] = rb;
}

// One kernel per precision, for the register budget: FP32 targets 7 CTAs per
// SM (72 registers; unhinted, the fast path of tile2 takes 80 and 6 CTAs, as
// fast within noise), FP64 8 CTAs per SM (64 registers, a few spilled words,
// faster than its unhinted 72). Both measured on the 1M-atom water box.
template <int NU, bool SELF>
__device__ __forceinline__ void pair_clusters_f32_body(const BlockCtx &ctx, PairClusterArgs<float> a, PairConsts<float> pc) {
  pair_clusters<float, NU, true, SELF>(ctx, a, pc);
}
template <int NU, bool SELF>
struct KPairClustersF32 {
  static constexpr int kUniformArg = 1;  // PairConsts
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { pair_clusters_f32_body<NU, SELF>(c, a...); }
};
template <int NU, bool SELF>
__global__ void __launch_bounds__(kWarps * 32, 7)
k_pair_clusters_f32(PairClusterArgs<float> a, PairConsts<float> pc) {
  pair_clusters_f32_body<NU, SELF>(hw_ctx(), a, pc);
}

template <int NU, bool SELF>
__device__ __forceinline__ void pair_clusters_f64_body(const BlockCtx &ctx, PairClusterArgs<double> a, PairConsts<double> pc) {
  pair_clusters<double, NU, false, SELF>(ctx, a, pc);
}
template <int NU, bool SELF>
struct KPairClustersF64 {
  static constexpr int kUniformArg = 1;  // PairConsts
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { pair_clusters_f64_body<NU, SELF>(c, a...); }
};
template <int NU, bool SELF>
__global__ void __launch_bounds__(kWarps * 32, 8)
k_pair_clusters_f64(PairClusterArgs<double> a, PairConsts<double> pc) {
  pair_clusters_f64_body<NU, SELF>(hw_ctx(), a, pc);
}

template <typename T, int NU>
void launch_nu(cudaStream_t s, const PairClusterArgs<T> &a, const PairConsts<T> &pc) {
  const int blocks = std::max(1, (a.maxcl + kWarps - 1) / kWarps);
  if constexpr (sizeof(T) == 4) {
    if (a.self_images)
      launch<KPairClustersF32<NU, true>, kWarps * 32, 7>(s, k_pair_clusters_f32<NU, true>, blocks, kWarps * 32, 0, a, pc);
    else
      launch<KPairClustersF32<NU, false>, kWarps * 32, 7>(s, k_pair_clusters_f32<NU, false>, blocks, kWarps * 32, 0, a, pc);
  } else {
    if (a.self_images)
      launch<KPairClustersF64<NU, true>, kWarps * 32, 8>(s, k_pair_clusters_f64<NU, true>, blocks, kWarps * 32, 0, a, pc);
    else
      launch<KPairClustersF64<NU, false>, kWarps * 32, 8>(s, k_pair_clusters_f64<NU, false>, blocks, kWarps * 32, 0, a, pc);
  }
}

}  // namespace

int cluster_capacity(int N, int ncol) { return N / 8 + ncol + 1; }

template <typename T>
void launch_cluster_fill(cudaStream_t s, int maxcl, int ncol, int nc2,
                         const int *start, const int *clstart, const int *pcs,
                         const V4<double> *src64, const double cz[3], V4<T> *cpos,
                         V4<double> *cpos64, ClusterInfo *info, UnitBox *ubox) {
  const long threads = 8L * maxcl;
  const int blocks = (int)std::max<long>(1, (threads + 255) / 256);
  launch<KClusterFill<T>, 256, 5>(s, k_cluster_fill<T>, blocks, 256, 0, maxcl, ncol, nc2, start, clstart, pcs, src64,
                                           cz[0], cz[1], cz[2], cpos, cpos64, info, ubox);
}

template <typename T>
void launch_pair_list(cudaStream_t s, const PairClusterArgs<T> &a) {
  const int blocks = std::max(1, (a.maxcl + kWarps - 1) / kWarps);
  k_pair_list<T><<<blocks, kWarps * 32, 0, s>>>(a);
}

template <typename T>
bool adj_pair_clusters_supported() { return sizeof(T) == 4; }

template <typename T>
void launch_adj_pair_clusters(cudaStream_t s, const PairClusterArgs<T> &a,
                              const PairConsts<T> &pc, const V4<T> *fbs, V4<T> *fslot,
                              V4<T> *out_a, V4<T> *out_b) {
  if constexpr (sizeof(T) == 4) {
    const long slots = 8L * a.maxcl;
    k_slot_gather<<<(int)std::max<long>(1, (slots + 255) / 256), 256, 0, s>>>(
        a.maxcl, a.clstart + a.ncol, a.info, fbs, fslot);
    const int blocks = std::max(1, (a.maxcl + kWarps - 1) / kWarps);
#define MSM_ADJ_JL(NUV)                                                                 \
  if (a.self_images)                                                                    \
    k_adj_pair_jl<NUV, true><<<blocks, kWarps * 32, 0, s>>>(a, pc, fbs, fslot, out_a, out_b);  \
  else                                                                                  \
    k_adj_pair_jl<NUV, false><<<blocks, kWarps * 32, 0, s>>>(a, pc, fbs, fslot, out_a, out_b)
    switch (pc.nu) {
      case 4: MSM_ADJ_JL(4); break;
      case 6: MSM_ADJ_JL(6); break;
      case 8: MSM_ADJ_JL(8); break;
      default: MSM_ADJ_JL(10); break;
    }
#undef MSM_ADJ_JL
  }
}

template <typename T>
void launch_pair_clusters(cudaStream_t s, const PairClusterArgs<T> &a,
                          const PairConsts<T> &pc) {
  switch (pc.nu) {
    case 0: launch_nu<T, 0>(s, a, pc); break;
    case 4: launch_nu<T, 4>(s, a, pc); break;
    case 6: launch_nu<T, 6>(s, a, pc); break;
    case 8: launch_nu<T, 8>(s, a, pc); break;
    default: launch_nu<T, 10>(s, a, pc); break;
  }
}

template void launch_cluster_fill<float>(cudaStream_t, int, int, int, const int *,
                                         const int *, const int *, const V4<double> *,
                                         const double *, V4<float> *, V4<double> *,
                                         ClusterInfo *, UnitBox *);
template void launch_cluster_fill<double>(cudaStream_t, int, int, int, const int *,
                                          const int *, const int *, const V4<double> *,
                                          const double *, V4<double> *, V4<double> *,
                                          ClusterInfo *, UnitBox *);
template void launch_pair_clusters<float>(cudaStream_t, const PairClusterArgs<float> &,
                                          const PairConsts<float> &);
template void launch_pair_list<float>(cudaStream_t, const PairClusterArgs<float> &);
template void launch_pair_list<double>(cudaStream_t, const PairClusterArgs<double> &);
template bool adj_pair_clusters_supported<float>();
template bool adj_pair_clusters_supported<double>();
template void launch_adj_pair_clusters<float>(cudaStream_t, const PairClusterArgs<float> &,
                                              const PairConsts<float> &, const V4<float> *,
                                              V4<float> *, V4<float> *, V4<float> *);
template void launch_adj_pair_clusters<double>(cudaStream_t, const PairClusterArgs<double> &,
                                               const PairConsts<double> &, const V4<double> *,
                                               V4<double> *, V4<double> *, V4<double> *);
template void launch_pair_clusters<double>(cudaStream_t, const PairClusterArgs<double> &,
                                           const PairConsts<double> &);

}  // namespace msm
