// Atom-side kernels: fractional coordinates and binning, a deterministic
// counting sort by cell (scan + scatter + per-cell ordering by atom index),
// gathers into cell order, the final per-atom combine and the energy sums.
#include <algorithm>

#include "kernels.h"

namespace msm {
namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ double matvec_row(const double *m, int r,
                                             double x, double y, double z) {
  return m[3 * r] * x + m[3 * r + 1] * y + m[3 * r + 2] * z;
}

// Per atom: s = A^-1 r wrapped to [0,1); pair cell; finest-grid cell m and
// offset t = M s - m (code/forcefield1.c:350-357); position relative to the
// pair cell's origin. Counts atoms per cell.
template <typename T>
__device__ __forceinline__ void prep_body(const BlockCtx &ctx, int N, const double *__restrict__ pos, const double *__restrict__ q,
       Geometry g, int *__restrict__ pcell, int *__restrict__ gcell,
       int *__restrict__ pcount, int *__restrict__ gcount,
       V4<T> *__restrict__ prel, V4<T> *__restrict__ gfrac,
       V4<double> *__restrict__ prel64, int *err, double *__restrict__ qparts) {
  int i = ctx.b.x * blockDim.x + threadIdx.x;
  // this block's sums of q and q^2 (FP64, fixed order), one pair per block
  {
    double a = 0., b = 0.;
    if (i < N) {
      a = q[i];
      b = a * a;
    }
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_down_sync(0xffffffffu, a, o);
      b += __shfl_down_sync(0xffffffffu, b, o);
    }
    __shared__ double wa[kThreads / 32], wb[kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
      wa[warp] = a;
      wb[warp] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double sa = 0., sb = 0.;
      for (int w = 0; w < kThreads / 32; ++w) {
        sa += wa[w];
        sb += wb[w];
      }
      qparts[2 * ctx.b.x] = sa;
      qparts[2 * ctx.b.x + 1] = sb;
    }
  }
  if (i >= N) return;
  double r0 = pos[3 * i], r1 = pos[3 * i + 1], r2 = pos[3 * i + 2];
  double qi = q[i];
  double s[3];
  bool ok = isfinite(qi);
  for (int k = 0; k < 3; ++k) {
    s[k] = matvec_row(g.Ai, k, r0, r1, r2);
    ok = ok && isfinite(s[k]);
  }
  if (!ok) {
    flag_error(err, kCheckNonFinite);
    s[0] = s[1] = s[2] = 0.;
  }
  int c[3], m[3];
  double t[3], frac[3];
  for (int k = 0; k < 3; ++k) {
    double sk = s[k] - floor(s[k]);
    c[k] = min((int)(sk * g.nc[k]), g.nc[k] - 1);
    frac[k] = sk - (double)c[k] / g.nc[k];
    double u = sk * g.M1[k];
    double fu = floor(u);
    t[k] = u - fu;
    int mk = (int)fu;
    m[k] = mk >= g.M1[k] ? mk - g.M1[k] : mk;
  }
  int pc = (c[0] * g.nc[1] + c[1]) * g.nc[2] + c[2];
  int gc = (m[0] * g.M1[1] + m[1]) * g.M1[2] + m[2];
  pcell[i] = pc;
  gcell[i] = gc;
  atomicAdd(pcount + pc, 1);
  atomicAdd(gcount + gc, 1);
  const double rx = matvec_row(g.A, 0, frac[0], frac[1], frac[2]);
  const double ry = matvec_row(g.A, 1, frac[0], frac[1], frac[2]);
  const double rz = matvec_row(g.A, 2, frac[0], frac[1], frac[2]);
  V4<T> a;
  a.x = (T)rx;
  a.y = (T)ry;
  a.z = (T)rz;
  a.w = (T)qi;
  prel[i] = a;
  if (prel64) {
    V4<double> a64;
    a64.x = rx;
    a64.y = ry;
    a64.z = rz;
    a64.w = qi;
    prel64[i] = a64;
  }
  V4<T> b;
  b.x = (T)t[0];
  b.y = (T)t[1];
  b.z = (T)t[2];
  b.w = (T)qi;
  gfrac[i] = b;
}
template <typename T>
struct KPrep {
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { prep_body<T>(c, a...); }
};
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_prep(int N, const double *__restrict__ pos, const double *__restrict__ q,
       Geometry g, int *__restrict__ pcell, int *__restrict__ gcell,
       int *__restrict__ pcount, int *__restrict__ gcount,
       V4<T> *__restrict__ prel, V4<T> *__restrict__ gfrac,
       V4<double> *__restrict__ prel64, int *err, double *__restrict__ qparts) {
  prep_body<T>(hw_ctx(), N, pos, q, g, pcell, gcell, pcount, gcount, prel, gfrac, prel64, err, qparts);
}

// ---- exclusive scan (three phases) ----
constexpr int kScanThreads = 512;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ int block_exclusive_scan(int v, int *sh, int *total) {
  // warp-shuffle scan then warp totals
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = (lane < kScanThreads / 32) ? sh[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < kScanThreads / 32) sh[lane] = w;
  }
  __syncthreads();
  int before = (warp > 0 ? sh[warp - 1] : 0) + x - v;
  if (total) *total = sh[kScanThreads / 32 - 1];
  __syncthreads();
  return before;
}

__device__ __forceinline__ void scan_reduce_body(const BlockCtx &ctx, const int *__restrict__ in, int n, int *__restrict__ bsum) {
  __shared__ int sh[32];
  int base = ctx.b.x * kScanTile;
  int v = 0;
  for (int k = 0; k < kScanItems; ++k) {
    int idx = base + threadIdx.x * kScanItems + k;
    if (idx < n) v += in[idx];
  }
  int total;
  block_exclusive_scan(v, sh, &total);
  if (threadIdx.x == 0) bsum[ctx.b.x] = total;
}
struct KScanReduce {
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { scan_reduce_body(c, a...); }
};
__global__ void __launch_bounds__(kScanThreads)
k_scan_reduce(const int *__restrict__ in, int n, int *__restrict__ bsum) {
  scan_reduce_body(hw_ctx(), in, n, bsum);
}

__device__ __forceinline__ void scan_top_body(const BlockCtx &ctx, int *bsum, int nb) {
  __shared__ int sh[32];
  int carry = 0;
  for (int base = 0; base < nb; base += kScanThreads) {
    int idx = base + threadIdx.x;
    int v = idx < nb ? bsum[idx] : 0;
    int total;
    int ex = block_exclusive_scan(v, sh, &total);
    if (idx < nb) bsum[idx] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0) bsum[nb] = carry;
}
struct KScanTop {
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { scan_top_body(c, a...); }
};
__global__ void __launch_bounds__(kScanThreads)
k_scan_top(int *bsum, int nb) {
  scan_top_body(hw_ctx(), bsum, nb);
}

// Short arrays (small systems, column counts): one block walks the tiles in
// order with a running carry, one launch instead of three.
constexpr int kScanSingleMax = 4 * kScanTile;

__device__ __forceinline__ void scan_single_body(const BlockCtx &ctx, const int *__restrict__ in, int n, int *__restrict__ out) {
  __shared__ int sh[32];
  int carry = 0;
  for (int base = 0; base < n; base += kScanTile) {
    int vals[kScanItems];
    int v = 0;
    for (int k = 0; k < kScanItems; ++k) {
      const int idx = base + threadIdx.x * kScanItems + k;
      vals[k] = idx < n ? in[idx] : 0;
      v += vals[k];
    }
    int total;
    int ex = block_exclusive_scan(v, sh, &total) + carry;
    for (int k = 0; k < kScanItems; ++k) {
      const int idx = base + threadIdx.x * kScanItems + k;
      if (idx < n) out[idx] = ex;
      ex += vals[k];
    }
    carry += total;
  }
  if (threadIdx.x == 0) out[n] = carry;
}
struct KScanSingle {
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { scan_single_body(c, a...); }
};
__global__ void __launch_bounds__(kScanThreads)
k_scan_single(const int *__restrict__ in, int n, int *__restrict__ out) {
  scan_single_body(hw_ctx(), in, n, out);
}

__device__ __forceinline__ void scan_apply_body(const BlockCtx &ctx, const int *__restrict__ in, int n, const int *__restrict__ bsum,
             int nb, int *__restrict__ out) {
  __shared__ int sh[32];
  int base = ctx.b.x * kScanTile;
  int vals[kScanItems];
  int v = 0;
  for (int k = 0; k < kScanItems; ++k) {
    int idx = base + threadIdx.x * kScanItems + k;
    vals[k] = idx < n ? in[idx] : 0;
    v += vals[k];
  }
  int ex = block_exclusive_scan(v, sh, nullptr) + bsum[ctx.b.x];
  for (int k = 0; k < kScanItems; ++k) {
    int idx = base + threadIdx.x * kScanItems + k;
    if (idx < n) out[idx] = ex;
    ex += vals[k];
  }
  if (ctx.b.x == 0 && threadIdx.x == 0) out[n] = bsum[nb];
}
struct KScanApply {
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { scan_apply_body(c, a...); }
};
__global__ void __launch_bounds__(kScanThreads)
k_scan_apply(const int *__restrict__ in, int n, const int *__restrict__ bsum,
             int nb, int *__restrict__ out) {
  scan_apply_body(hw_ctx(), in, n, bsum, nb, out);
}

// Both scans of the binning (pair-cell counts, grid-cell counts) in the
// same launches: the blocks of one launch take the first array's tiles,
// then the second's (each block computes what its launch for one array
// would). Integer sums, so the result does not depend on the split.
struct ScanArray {
  const int *in;
  int n;
  int *out;
  int *tmp;  // block sums (nb + 1)
  int nb;    // blocks of the three-pass scan
};
__device__ __forceinline__ BlockCtx second(const BlockCtx &ctx, int nb0) {
  BlockCtx c = ctx;
  c.b.x -= nb0;
  return c;
}
__device__ __forceinline__ void scan_reduce2_body(const BlockCtx &ctx, ScanArray a, ScanArray b) {
  if ((int)ctx.b.x < a.nb) scan_reduce_body(ctx, a.in, a.n, a.tmp);
  else scan_reduce_body(second(ctx, a.nb), b.in, b.n, b.tmp);
}
struct KScanReduce2 {
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { scan_reduce2_body(c, a...); }
};
__global__ void __launch_bounds__(kScanThreads) k_scan_reduce2(ScanArray a, ScanArray b) {
  scan_reduce2_body(hw_ctx(), a, b);
}
__device__ __forceinline__ void scan_top2_body(const BlockCtx &ctx, ScanArray a, ScanArray b) {
  if (ctx.b.x == 0) scan_top_body(ctx, a.tmp, a.nb);
  else scan_top_body(second(ctx, 1), b.tmp, b.nb);
}
struct KScanTop2 {
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { scan_top2_body(c, a...); }
};
__global__ void __launch_bounds__(kScanThreads) k_scan_top2(ScanArray a, ScanArray b) {
  scan_top2_body(hw_ctx(), a, b);
}
__device__ __forceinline__ void scan_apply2_body(const BlockCtx &ctx, ScanArray a, ScanArray b) {
  if ((int)ctx.b.x < a.nb) scan_apply_body(ctx, a.in, a.n, a.tmp, a.nb, a.out);
  else scan_apply_body(second(ctx, a.nb), b.in, b.n, b.tmp, b.nb, b.out);
}
struct KScanApply2 {
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { scan_apply2_body(c, a...); }
};
__global__ void __launch_bounds__(kScanThreads) k_scan_apply2(ScanArray a, ScanArray b) {
  scan_apply2_body(hw_ctx(), a, b);
}
__device__ __forceinline__ void scan_single2_body(const BlockCtx &ctx, ScanArray a, ScanArray b) {
  if (ctx.b.x == 0) scan_single_body(ctx, a.in, a.n, a.out);
  else scan_single_body(second(ctx, 1), b.in, b.n, b.out);
}
struct KScanSingle2 {
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { scan_single2_body(c, a...); }
};
__global__ void __launch_bounds__(kScanThreads) k_scan_single2(ScanArray a, ScanArray b) {
  scan_single2_body(hw_ctx(), a, b);
}

// Both cell scatters of the binning in one launch: threads [0, N) place the
// atoms into pair cells, threads [N, 2N) into grid cells, and threads
// [2N, 2N + ncol) count each pair-cell column's clusters of 8 atoms (for the
// cluster pair sum; ncol = 0 when it is not used).
struct ScatterSide {
  const int *cell, *start;
  int *cursor, *perm;
};

__device__ __forceinline__ void scatter2_body(const BlockCtx &ctx, int N, ScatterSide p, ScatterSide g, int ncol, int nc2, int *__restrict__ clcount) {
  int i = ctx.b.x * blockDim.x + threadIdx.x;
  if (i >= 2 * N) {
    const int c = i - 2 * N;
    if (c < ncol) clcount[c] = (p.start[(c + 1) * nc2] - p.start[c * nc2] + 7) >> 3;
    return;
  }
  const ScatterSide &d = i < N ? p : g;
  if (i >= N) i -= N;
  const int c = d.cell[i];
  const int slot = d.start[c] + atomicAdd(d.cursor + c, 1);
  d.perm[slot] = i;
}
struct KScatter2 {
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { scatter2_body(c, a...); }
};
__global__ void __launch_bounds__(kThreads)
k_scatter2(int N, ScatterSide p, ScatterSide g, int ncol, int nc2, int *__restrict__ clcount) {
  scatter2_body(hw_ctx(), N, p, g, ncol, nc2, clcount);
}

// Orders one grid cell's atoms by atom index, which makes every later
// floating-point sum independent of the scatter's arrival order.
__device__ void sort_cell_by_index(int b, int e, int *__restrict__ perm) {
  for (int k = b + 1; k < e; ++k) {
    int v = perm[k];
    int j = k - 1;
    while (j >= b && perm[j] > v) {
      perm[j + 1] = perm[j];
      --j;
    }
    perm[j + 1] = v;
  }
}

// Orders one pair cell's atoms along z (key[atom].z, the position relative
// to the cell origin), ties by atom index: every column of cells becomes one
// z-ordered run, and the order depends only on the input.
template <typename T>
__device__ void sort_cell_by_z(int b, int e, int *__restrict__ perm,
                               const V4<T> *__restrict__ key) {
  constexpr int kCap = 32;
  if (e - b <= kCap) {
    // rank sort: all loads independent, each atom's place = the number of
    // atoms before it in (z, index) order; the same order as below
    const int n = e - b;
    int id[kCap];
    T kz[kCap];
    for (int i = 0; i < n; ++i) id[i] = perm[b + i];
    for (int i = 0; i < n; ++i) kz[i] = key[id[i]].z;
    for (int i = 0; i < n; ++i) {
      int r = 0;
      for (int j = 0; j < n; ++j)
        r += (kz[j] < kz[i] || (kz[j] == kz[i] && id[j] < id[i])) ? 1 : 0;
      perm[b + r] = id[i];
    }
    return;
  }
  for (int k = b + 1; k < e; ++k) {
    const int v = perm[k];
    const T kv = key[v].z;
    int j = k - 1;
    while (j >= b) {
      const int pj = perm[j];
      const T kj = key[pj].z;
      if (kj < kv || (kj == kv && pj < v)) break;
      perm[j + 1] = pj;
      --j;
    }
    perm[j + 1] = v;
  }
}

// Both per-cell sorts in one launch: a warp per pair cell for threads
// [0, 32 ncp) (along z, ties by atom index), then a thread per grid cell (by
// atom index). In a pair cell of up to 32 atoms lane l holds atom l's key and
// its place is the number of atoms before it in (z, index) order, counted
// from the other lanes' keys by shuffles (the same order as sort_cell_by_z,
// which lane 0 runs for larger cells). blockDim.x is a multiple of 32, so a
// warp never straddles two cells or the two parts.
template <typename T>
__device__ __forceinline__ void sort_cells_body(const BlockCtx &ctx, int ncp, const int *__restrict__ pstart, int *__restrict__ pperm,
             const V4<T> *__restrict__ key, int ncg, const int *__restrict__ gstart,
             int *__restrict__ gperm) {
  const long t = (long)ctx.b.x * blockDim.x + threadIdx.x;
  const long np = 32L * ncp;
  if (t < np) {
    const int c = (int)(t >> 5), lane = threadIdx.x & 31;
    const int b = pstart[c], e = pstart[c + 1], n = e - b;
    if (n <= 32) {
      int id = 0;
      T z = T(0);
      if (lane < n) {
        id = pperm[b + lane];
        z = key[id].z;
      }
      int r = 0;
      for (int j = 0; j < n; ++j) {
        const T zj = __shfl_sync(0xffffffffu, z, j);
        const int ij = __shfl_sync(0xffffffffu, id, j);
        r += (zj < z || (zj == z && ij < id)) ? 1 : 0;
      }
      __syncwarp();  // every lane has read its slot before any lane writes
      if (lane < n) pperm[b + r] = id;
    } else if (lane == 0) {
      sort_cell_by_z<T>(b, e, pperm, key);
    }
    return;
  }
  const long g = t - np;
  if (g < ncg) sort_cell_by_index(gstart[g], gstart[g + 1], gperm);
}
template <typename T>
struct KSortCells {
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { sort_cells_body<T>(c, a...); }
};
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_sort_cells(int ncp, const int *__restrict__ pstart, int *__restrict__ pperm,
             const V4<T> *__restrict__ key, int ncg, const int *__restrict__ gstart,
             int *__restrict__ gperm) {
  sort_cells_body<T>(hw_ctx(), ncp, pstart, pperm, key, ncg, gstart, gperm);
}

// Both gathers into sorted order in one launch (and the FP64 copy of the
// pair-cell records in the mixed form): slot k takes atom perm[k].
template <typename T>
__device__ __forceinline__ void gather2_body(const BlockCtx &ctx, int N, GatherSide<T> p, const V4<double> *__restrict__ src64,
          V4<double> *__restrict__ dst64, GatherSide<T> g) {
  const int k = ctx.b.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  int i = p.perm[k];
  p.dst[k] = p.src[i];
  p.cell_sorted[k] = p.cell[i];
  p.inv[i] = k;
  if (dst64) dst64[k] = src64[i];
  i = g.perm[k];
  g.dst[k] = g.src[i];
  g.cell_sorted[k] = g.cell[i];
  g.inv[i] = k;
}
template <typename T>
struct KGather2 {
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { gather2_body<T>(c, a...); }
};
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_gather2(int N, GatherSide<T> p, const V4<double> *__restrict__ src64,
          V4<double> *__restrict__ dst64, GatherSide<T> g) {
  gather2_body<T>(hw_ctx(), N, p, src64, dst64, g);
}


// Per atom in input order: F_i = w0 F_short + q_i E_i and
// phi_i = w0 (q_i c1 - Q c2 - q_i gamma0/a0 + phi_short) + phi_long.
template <typename T>
__device__ __forceinline__ void combine_body(const BlockCtx &ctx, CombineArgs a, const int *__restrict__ pinv,
          const int *__restrict__ ginv, const V4<T> *__restrict__ pout,
          const V4<T> *__restrict__ gout) {
  __shared__ double red[kThreads];
  const double qsum = a.qstats[0];  // reduced by k_qstats_final
  double e = 0.;
  int i = ctx.b.x * blockDim.x + threadIdx.x;
  if (i < a.N) {
    double qi = a.q[i];
    V4<T> ps = pout[pinv[i]];
    V4<T> gs = gout[ginv[i]];
    if (a.force) {
      a.force[3 * i] = a.w0 * (double)ps.x + qi * (double)gs.x;
      a.force[3 * i + 1] = a.w0 * (double)ps.y + qi * (double)gs.y;
      a.force[3 * i + 2] = a.w0 * (double)ps.z + qi * (double)gs.z;
    }
    if (a.phi)
      a.phi[i] = a.w0 * (qi * a.coeff1 - qsum * a.coeff2 -
                         qi * a.gamma0_over_a0 + (double)ps.w) +
                 (double)gs.w;
    e = 0.5 * a.w0 * qi * (double)ps.w;
  }
  red[threadIdx.x] = e;
  __syncthreads();
  for (int w = kThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) a.epart[ctx.b.x] = red[0];
}
template <typename T>
struct KCombine {
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { combine_body<T>(c, a...); }
};
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_combine(CombineArgs a, const int *__restrict__ pinv,
          const int *__restrict__ ginv, const V4<T> *__restrict__ pout,
          const V4<T> *__restrict__ gout) {
  combine_body<T>(hw_ctx(), a, pinv, ginv, pout, gout);
}

__device__ double block_sum(const double *v, int n, double *sh) {
  double acc = 0.;
  for (int k = threadIdx.x; k < n; k += blockDim.x) acc += v[k];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  double r = sh[0];
  __syncthreads();
  return r;
}

__device__ __forceinline__ void qstats_final_body(const BlockCtx &ctx, const double *qparts, int n,
                                                           double *qstats) {
  __shared__ double sh[kThreads];
  double a = 0., b = 0.;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    a += qparts[2 * k];
    b += qparts[2 * k + 1];
  }
  sh[threadIdx.x] = a;
  __syncthreads();
  for (int w = kThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  double qs = sh[0];
  __syncthreads();
  sh[threadIdx.x] = b;
  __syncthreads();
  for (int w = kThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    qstats[0] = qs;
    qstats[1] = sh[0];
  }
}
struct KQstatsFinal {
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { qstats_final_body(c, a...); }
};
__global__ void __launch_bounds__(kThreads)
k_qstats_final(const double *qparts, int n,
                                                           double *qstats) {
  qstats_final_body(hw_ctx(), qparts, n, qstats);
}

// U = w0 (Q2 c1/2 - Q^2 c2/2 - Q2 gamma0/(2 a0)) + w0 sum q phi_s / 2
//     + q^1 . e^1 / 2      (code/forcefield1.c:114-137, :195-219)
__device__ __forceinline__ void energy_total_body(const BlockCtx &ctx, EnergyArgs a) {
  __shared__ double sh[kThreads];
  double qs = a.qstats[0], q2 = a.qstats[1];
  double us = block_sum(a.short_parts, a.nshort, sh);
  double ug = block_sum(a.grid_parts, a.ngrid, sh);
  if (threadIdx.x == 0) {
    double uc = 0.5 * q2 * a.coeff1 - 0.5 * qs * qs * a.coeff2 -
                0.5 * q2 * a.gamma0_over_a0;
    a.energy[0] = a.w0 * uc + us + 0.5 * a.grid_scale * ug;
  }
}
struct KEnergyTotal {
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { energy_total_body(c, a...); }
};
__global__ void __launch_bounds__(kThreads)
k_energy_total(EnergyArgs a) {
  energy_total_body(hw_ctx(), a);
}

inline int blocks_for(long n, int threads) {
  return (int)std::max<long>(1, (n + threads - 1) / threads);
}

}  // namespace

template <typename T>
void launch_prep(cudaStream_t s, int N, const double *pos, const double *q,
                 const Geometry &g, int *pcell, int *gcell, int *pcount,
                 int *gcount, V4<T> *prel, V4<T> *gfrac, V4<double> *prel64,
                 int *err, double *qparts) {
  launch<KPrep<T>, kThreads, 6>(s, k_prep<T>, blocks_for(N, kThreads), kThreads, 0, N, pos, q, g, pcell, gcell, pcount, gcount, prel, gfrac, prel64, err, qparts);
}

int prep_blocks(int N) { return (int)blocks_for(N, kThreads); }

void launch_qstats_final(cudaStream_t s, const double *qparts, int nqparts,
                         double *qstats) {
  launch<KQstatsFinal, kThreads, 1>(s, k_qstats_final, 1, kThreads, 0, qparts, nqparts, qstats);
}

size_t scan_temp_ints(int n) { return (size_t)(n / kScanTile + 2); }

int scan_launches(int n) { return n <= kScanSingleMax ? 1 : 3; }

void launch_scan(cudaStream_t s, const int *in, int *out, int n, int *tmp) {
  if (n <= kScanSingleMax) {
    launch<KScanSingle, kScanThreads, 4>(s, k_scan_single, 1, kScanThreads, 0, in, n, out);
    return;
  }
  int nb = std::max(1, (n + kScanTile - 1) / kScanTile);
  launch<KScanReduce, kScanThreads, 4>(s, k_scan_reduce, nb, kScanThreads, 0, in, n, tmp);
  launch<KScanTop, kScanThreads, 4>(s, k_scan_top, 1, kScanThreads, 0, tmp, nb);
  launch<KScanApply, kScanThreads, 4>(s, k_scan_apply, nb, kScanThreads, 0, in, n, tmp, nb, out);
}

int scan2_launches(int n0, int n1) {
  return (n0 <= kScanSingleMax && n1 <= kScanSingleMax) ? 1 : 3;
}

void launch_scan2(cudaStream_t s, const int *in0, int *out0, int n0, const int *in1, int *out1,
                  int n1, int *tmp) {
  ScanArray a{in0, n0, out0, tmp, std::max(1, (n0 + kScanTile - 1) / kScanTile)};
  ScanArray b{in1, n1, out1, tmp + a.nb + 1, std::max(1, (n1 + kScanTile - 1) / kScanTile)};
  if (scan2_launches(n0, n1) == 1) {
    launch<KScanSingle2, kScanThreads, 4>(s, k_scan_single2, 2, kScanThreads, 0, a, b);
    return;
  }
  launch<KScanReduce2, kScanThreads, 4>(s, k_scan_reduce2, a.nb + b.nb, kScanThreads, 0, a, b);
  launch<KScanTop2, kScanThreads, 4>(s, k_scan_top2, 2, kScanThreads, 0, a, b);
  launch<KScanApply2, kScanThreads, 4>(s, k_scan_apply2, a.nb + b.nb, kScanThreads, 0, a, b);
}

void launch_bin_scatter(cudaStream_t s, int N, const int *pcell, const int *pstart,
                        int *pcursor, int *pperm, const int *gcell, const int *gstart,
                        int *gcursor, int *gperm, int ncol, int nc2, int *clcount) {
  launch<KScatter2, kThreads, 8>(s, k_scatter2, blocks_for(2L * N + ncol, kThreads), kThreads, 0, N, ScatterSide{pcell, pstart, pcursor, pperm}, ScatterSide{gcell, gstart, gcursor, gperm},
      ncol, nc2, clcount);
}

template <typename T>
void launch_bin_sort(cudaStream_t s, int ncp, const int *pstart, int *pperm, const V4<T> *key,
                     int ncg, const int *gstart, int *gperm) {
  launch<KSortCells<T>, kThreads, 8>(s, k_sort_cells<T>, blocks_for(32L * ncp + ncg, kThreads), kThreads, 0, ncp, pstart, pperm, key, ncg, gstart, gperm);
}

template <typename T>
void launch_bin_gather(cudaStream_t s, int N, const GatherSide<T> &p,
                       const V4<double> *src64, V4<double> *dst64, const GatherSide<T> &g) {
  launch<KGather2<T>, kThreads, 8>(s, k_gather2<T>, blocks_for(N, kThreads), kThreads, 0, N, p, src64, dst64, g);
}

int combine_blocks(int N) { return blocks_for(N, kThreads); }

template <typename T>
void launch_combine(cudaStream_t s, const CombineArgs &a, const int *pinv,
                    const int *ginv, const V4<T> *pout, const V4<T> *gout,
                    int nblocks) {
  launch<KCombine<T>, kThreads, 8>(s, k_combine<T>, nblocks, kThreads, 0, a, pinv, ginv, pout, gout);
}

void launch_energy_total(cudaStream_t s, const EnergyArgs &a) {
  launch<KEnergyTotal, kThreads, 1>(s, k_energy_total, 1, kThreads, 0, a);
}

#define MSM_INST_ATOMS(T)                                                     \
  template void launch_prep<T>(cudaStream_t, int, const double *,            \
                               const double *, const Geometry &, int *,      \
                               int *, int *, int *, V4<T> *, V4<T> *,         \
                               V4<double> *, int *, double *);                \
  template void launch_bin_gather<T>(cudaStream_t, int, const GatherSide<T> &,  \
                                     const V4<double> *, V4<double> *,           \
                                     const GatherSide<T> &);                     \
  template void launch_combine<T>(cudaStream_t, const CombineArgs &,         \
                                  const int *, const int *, const V4<T> *,    \
                                  const V4<T> *, int);                        \
  template void launch_bin_sort<T>(cudaStream_t, int, const int *, int *,      \
                                    const V4<T> *, int, const int *, int *);
MSM_INST_ATOMS(float)
MSM_INST_ATOMS(double)

}  // namespace msm
