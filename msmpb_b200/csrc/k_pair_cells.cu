// Short-range pair sum, cell-staged form with compacted hits (the fast path).
//
// One CTA per home cell. The CTA first enumerates the candidate atoms of all
// neighbour-cell instances of its cell (the host-built offset list: cell
// offset d and the Cartesian shift of that cell's origin relative to the home
// cell's origin, periodic image included) and stages them in shared memory
// with the shift applied, so a candidate's position is relative to the home
// cell origin, like the home atoms'. Each warp then takes home atoms in turn;
// for one home atom i the 32 lanes test 32 candidates at a time, and the
// in-cutoff ones are appended to a warp queue (ballot + prefix popcount).
// Whenever 32 hits are queued, every lane evaluates one: no lane idles on an
// out-of-range candidate. Per-lane partial sums are reduced across the warp
// once per home atom and added to the home atom's shared accumulator; all
// orders are fixed, so results are deterministic.
//
// Mixed form: FP32 except pairs closer than sqrt(close2), which go to a
// small per-warp side queue and are summed in FP64 from FP64 cell-relative
// positions and FP64 shifts once the home atom's sweep ends (see k_pair.cu
// for why: their forces are the largest and the most sensitive to position
// rounding).
#include "kernels.h"
#include "pair_fn.cuh"

namespace msm {
namespace {

constexpr int kThreads = 128;   // 4 warps
constexpr int kWarps = kThreads / 32;
// staged candidates per batch: 24 KB of positions in either precision
template <typename T>
__host__ __device__ constexpr int cand_cap() { return 1536 * 4 / (int)sizeof(T); }
constexpr int kHomeCap = 64;    // home atoms per group
constexpr int kCloseCap = 64;   // close pairs per home atom (then FP32)


template <typename T, int NU>
__device__ __forceinline__ void pair_terms(const PairConsts<T> &pc, T dx, T dy,
                                           T dz, T r2, T qj, T &fx, T &fy,
                                           T &fz, T &ph) {
  T v, f;
  pair_radial<T, NU>(pc, r2, v, f);
  ph += qj * v;
  const T cf = qj * f;
  fx += cf * dx;
  fy += cf * dy;
  fz += cf * dz;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <typename T, int NU, bool CLOSE>
__global__ void __launch_bounds__(kThreads)
k_pair_cells(const V4<T> *__restrict__ ps, const V4<double> *__restrict__ ps64,
             const int *__restrict__ start, int nc0, int nc1, int nc2,
             const CellOffset<T> *__restrict__ off, int noff, PairConsts<T> pc,
             V4<T> *__restrict__ out) {
  constexpr int kCandCap = cand_cap<T>();
  __shared__ V4<T> cpos[kCandCap];
  __shared__ int cid[kCandCap];              // candidate atom index
  __shared__ unsigned short coff[kCandCap];  // its neighbour-cell instance
  __shared__ int ostart[kMaxNeighbourOffsets / 8 + 1];
  __shared__ int qbuf[kWarps][64];
  __shared__ int cbuf[kWarps][kCloseCap];
  __shared__ T hacc[kHomeCap][4];
  __shared__ double hacc64[CLOSE ? kHomeCap : 1][4];
  __shared__ int wtot[kWarps];

  const int c = blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int cz = c % nc2, cy = (c / nc2) % nc1, cx = c / (nc1 * nc2);
  const int hb = start[c], he = start[c + 1];
  if (hb == he) return;  // empty home cell (uniform)
  const unsigned lt = (1u << lane) - 1u;

  // candidate counts per offset, exclusive scan (noff <= ostart capacity)
  const int per = (noff + kThreads - 1) / kThreads;
  int local = 0;
  for (int o = tid * per; o < min(noff, tid * per + per); ++o) {
    const int ux = pwrap(cx + off[o].d[0], nc0), uy = pwrap(cy + off[o].d[1], nc1),
              uz = pwrap(cz + off[o].d[2], nc2);
    const int cw = (ux * nc1 + uy) * nc2 + uz;
    const int n = start[cw + 1] - start[cw];
    ostart[o] = n;
    local += n;
  }
  int incl = local;
  for (int o = 1; o < 32; o <<= 1) {
    int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) wtot[warp] = incl;
  __syncthreads();
  int before = 0, total = 0;
  for (int w = 0; w < kWarps; ++w) {
    if (w < warp) before += wtot[w];
    total += wtot[w];
  }
  {
    int run = before + incl - local;
    for (int o = tid * per; o < min(noff, tid * per + per); ++o) {
      const int n = ostart[o];
      ostart[o] = run;
      run += n;
    }
  }
  if (tid == 0) ostart[noff] = total;
  __syncthreads();

  for (int g0 = hb; g0 < he; g0 += kHomeCap) {
    const int ng = min(kHomeCap, he - g0);
    for (int t = tid; t < ng * 4; t += kThreads) {
      (&hacc[0][0])[t] = T(0);
      if constexpr (CLOSE) (&hacc64[0][0])[t] = 0.0;
    }
    for (int base = 0; base < total; base += kCandCap) {
      const int nb = min(kCandCap, total - base);
      __syncthreads();
      // stage candidates [base, base+nb): position relative to the home
      // cell origin, atom index and neighbour-cell instance
      for (int k = tid; k < nb; k += kThreads) {
        const int gk = base + k;
        int lo = 0, hi = noff - 1;  // last offset with ostart <= gk
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (ostart[mid] <= gk) lo = mid; else hi = mid - 1;
        }
        const CellOffset<T> &co = off[lo];
        const int ux = pwrap(cx + co.d[0], nc0), uy = pwrap(cy + co.d[1], nc1),
                  uz = pwrap(cz + co.d[2], nc2);
        const int j = start[(ux * nc1 + uy) * nc2 + uz] + (gk - ostart[lo]);
        V4<T> a = ps[j];
        a.x += co.shift[0];
        a.y += co.shift[1];
        a.z += co.shift[2];
        cpos[k] = a;
        cid[k] = j;
        coff[k] = (unsigned short)lo;
      }
      __syncthreads();
      for (int h = warp; h < ng; h += kWarps) {
        const int i = g0 + h;
        const V4<T> ri = ps[i];
        T fx = 0, fy = 0, fz = 0, ph = 0;
        int qn = 0, cn = 0;
        for (int k0 = 0; k0 < nb; k0 += 32) {
          const int k = k0 + lane;
          bool hit = false, close = false;
          if (k < nb) {
            const V4<T> a = cpos[k];
            const T dx = a.x - ri.x, dy = a.y - ri.y, dz = a.z - ri.z;
            const T r2 = dx * dx + dy * dy + dz * dz;
            hit = r2 < pc.a02 && cid[k] != i;
            if (CLOSE) {
              close = hit && r2 < pc.close2;
              hit = hit && !close;
            }
          }
          if constexpr (CLOSE) {
            // close pairs beyond the side queue's capacity stay in FP32
            const unsigned cm = __ballot_sync(0xffffffffu, close);
            if (close) {
              const int slot = cn + __popc(cm & lt);
              if (slot < kCloseCap)
                cbuf[warp][slot] = k;
              else {
                close = false;
                hit = true;
              }
            }
            cn = min(kCloseCap, cn + __popc(cm));
          }
          const unsigned m = __ballot_sync(0xffffffffu, hit);
          if (hit) qbuf[warp][qn + __popc(m & lt)] = k;
          qn += __popc(m);
          __syncwarp();
          if (qn >= 32) {  // one full batch: every lane evaluates a hit
            const int q = qbuf[warp][lane];
            const V4<T> a = cpos[q];
            const T dx = a.x - ri.x, dy = a.y - ri.y, dz = a.z - ri.z;
            pair_terms<T, NU>(pc, dx, dy, dz, dx * dx + dy * dy + dz * dz, a.w,
                              fx, fy, fz, ph);
            __syncwarp();
            if (lane < qn - 32) qbuf[warp][lane] = qbuf[warp][lane + 32];
            qn -= 32;
            __syncwarp();
          }
        }
        if (lane < qn) {  // the last partial batch
          const int q = qbuf[warp][lane];
          const V4<T> a = cpos[q];
          const T dx = a.x - ri.x, dy = a.y - ri.y, dz = a.z - ri.z;
          pair_terms<T, NU>(pc, dx, dy, dz, dx * dx + dy * dy + dz * dz, a.w, fx,
                            fy, fz, ph);
        }
        double cfx = 0., cfy = 0., cfz = 0., cph = 0.;
        if (CLOSE && cn > 0) {
          const V4<double> ri64 = ps64[i];
          for (int t = lane; t < cn; t += 32) {
            const int k = cbuf[warp][t];
            const int j = cid[k], o = coff[k];
            const V4<double> aj = ps64[j];
            const double ex = (aj.x + off[o].shift64[0]) - ri64.x;
            const double ey = (aj.y + off[o].shift64[1]) - ri64.y;
            const double ez = (aj.z + off[o].shift64[2]) - ri64.z;
            const double d2 = ex * ex + ey * ey + ez * ez;
            double v, f;
            pair_radial64<NU>(pc, d2, v, f);
            cph += aj.w * v;
            const double cf = aj.w * f;
            cfx += cf * ex;
            cfy += cf * ey;
            cfz += cf * ez;
          }
          cfx = warp_sum(cfx);
          cfy = warp_sum(cfy);
          cfz = warp_sum(cfz);
          cph = warp_sum(cph);
        }
        fx = warp_sum(fx);
        fy = warp_sum(fy);
        fz = warp_sum(fz);
        ph = warp_sum(ph);
        if (lane == 0) {
          hacc[h][0] += fx;
          hacc[h][1] += fy;
          hacc[h][2] += fz;
          hacc[h][3] += ph;
          if constexpr (CLOSE) {
            hacc64[h][0] += cfx;
            hacc64[h][1] += cfy;
            hacc64[h][2] += cfz;
            hacc64[h][3] += cph;
          }
        }
      }
    }
    __syncthreads();
    for (int h = tid; h < ng; h += kThreads) {
      const int i = g0 + h;
      V4<T> r;
      if constexpr (CLOSE) {
        const double qi = ps64[i].w;
        r.x = (T)(qi * ((double)hacc[h][0] + hacc64[h][0]));
        r.y = (T)(qi * ((double)hacc[h][1] + hacc64[h][1]));
        r.z = (T)(qi * ((double)hacc[h][2] + hacc64[h][2]));
        r.w = (T)((double)hacc[h][3] + hacc64[h][3]);
      } else {
        const T qi = ps[i].w;
        r.x = qi * hacc[h][0];
        r.y = qi * hacc[h][1];
        r.z = qi * hacc[h][2];
        r.w = hacc[h][3];
      }
      out[i] = r;
    }
    __syncthreads();
  }
}

template <typename T, int NU>
void launch_nu(cudaStream_t s, int ncell, const V4<T> *ps, const V4<double> *ps64,
               const int *start, const Geometry &g, const CellOffset<T> *off,
               int noff, const PairConsts<T> &pc, V4<T> *out, int *err) {
  constexpr bool kMixed = sizeof(T) == 4;
  (void)err;
  k_pair_cells<T, NU, kMixed><<<ncell, kThreads, 0, s>>>(
      ps, ps64, start, g.nc[0], g.nc[1], g.nc[2], off, noff, pc, out);
}

}  // namespace

bool pair_cells_supported(int noff, long natoms) {
  return noff <= kMaxNeighbourOffsets / 8 && natoms < (1L << 31);
}

template <typename T>
void launch_pair_cells(cudaStream_t s, int ncell, const V4<T> *ps,
                       const V4<double> *ps64, const int *start,
                       const Geometry &g, const CellOffset<T> *off, int noff,
                       const PairConsts<T> &pc, V4<T> *out, int *err) {
  switch (pc.nu) {
    case 0: launch_nu<T, 0>(s, ncell, ps, ps64, start, g, off, noff, pc, out, err); break;
    case 4: launch_nu<T, 4>(s, ncell, ps, ps64, start, g, off, noff, pc, out, err); break;
    case 6: launch_nu<T, 6>(s, ncell, ps, ps64, start, g, off, noff, pc, out, err); break;
    case 8: launch_nu<T, 8>(s, ncell, ps, ps64, start, g, off, noff, pc, out, err); break;
    default: launch_nu<T, 10>(s, ncell, ps, ps64, start, g, off, noff, pc, out, err); break;
  }
}

template void launch_pair_cells<float>(cudaStream_t, int, const V4<float> *,
                                       const V4<double> *, const int *,
                                       const Geometry &, const CellOffset<float> *,
                                       int, const PairConsts<float> &,
                                       V4<float> *, int *);
template void launch_pair_cells<double>(cudaStream_t, int, const V4<double> *,
                                        const V4<double> *, const int *,
                                        const Geometry &, const CellOffset<double> *,
                                        int, const PairConsts<double> &,
                                        V4<double> *, int *);

}  // namespace msm
