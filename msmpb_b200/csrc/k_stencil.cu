// Per-level grid-to-grid direct stencil (code/forcefield0.c:898-931):
//   e^l_x += w_l * sum_{d in [0,S)^3} khat_l[d] q^l_{x + d - S/2}  (periodic)
// The periodic wrap is materialised once per level as a padded copy
// P[a][b][c] = q[(a - S0/2) mod M0][(b - S1/2) mod M1][(c - S2/2) mod M2]
// (the reference pads the same way, code/forcefield1.c:58-99), so the sweep
// reads dense boxes with no modular index arithmetic.
//
// Tiled sweep (FP32 CUDA cores; a single-channel stencil is not a GEMM):
//  - a CTA owns TX x TY x (NZ*R) outputs; thread (tz, ty) keeps TX*R
//    accumulators in registers (R consecutive z outputs for each of TX
//    x-planes);
//  - input x-planes stream through a double-buffered shared-memory slice
//    ((TY+S1-1) x (NZ*R+S2-1)) filled with cp.async 16-byte copies while
//    the previous plane is consumed; plane p feeds output planes x0+xo with
//    tap plane i = p - x0 - xo;
//  - per (plane, tap row j) a thread loads one input row segment of
//    R+S2-1 values into registers once and reuses it for all TX output
//    planes; the S2 taps of row (i, j) are uniform across the CTA (L1
//    broadcast). The z extent S2 is a template parameter so the R x S2
//    FMA block is fully unrolled with register-resident operands.
#include <algorithm>
#include <cmath>
#include <mutex>

#include "kernels.h"

namespace msm {
namespace {

constexpr int kThreads = 256;
constexpr int kMaxTemplatedS = 33;

inline int blocks_for(long n) {
  return (int)std::max<long>(1, (n + kThreads - 1) / kThreads);
}

// Row pitch of a shared slice: the nz R + S - 1 values a row needs, in whole
// 16-byte units, padded so that the 16-byte row reads are free of bank
// conflicts. Thread (tz, ty) = tid (tz fastest) reads unit ty p + tz R/V (+v)
// of the slice; a 16-byte load is served 8 lanes at a time, one wavefront
// when their units fall in 8 different 16-byte bank groups (unit mod 8). The
// smallest pitch p that gives that for the CTA's first 128 threads is taken
// (else the one with the fewest conflicts).
inline int slice_pitch(int nz, int R, int S, int V) {
  const int base = (nz * R + S - 1 + V - 1) / V;
  const int step = R / V;
  int best = base, best_c = 1 << 30;
  for (int p = base; p < base + 8; ++p) {
    int conflicts = 0;
    for (int g = 0; g < 128; g += 8) {
      int used = 0;
      for (int l = g; l < g + 8; ++l) {
        const int bank = ((l / nz) * p + (l % nz) * step) & 7;
        if (used & (1 << bank)) ++conflicts;
        used |= 1 << bank;
      }
    }
    if (conflicts < best_c) {
      best_c = conflicts;
      best = p;
      if (!conflicts) break;
    }
  }
  return best * V;
}

// Padded copy: P[a][b][c] = q[wrap(a - S0/2)][wrap(b - S1/2)][wrap(c - S2/2)]
// over the padded dimensions. One padded row (a, b) per warp, lanes along it
// (kThreads / 32 rows per CTA).
template <typename T>
__device__ __forceinline__ void pad_body(const BlockCtx &ctx, StencilShape sh, const T *__restrict__ q, T *__restrict__ p) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long row = (long)ctx.b.x * (blockDim.x >> 5) + warp;
  if (row >= (long)sh.P[0] * sh.P[1]) return;
  const int a = (int)(row / sh.P[1]), b = (int)(row - (long)a * sh.P[1]);
  const int x = pwrap(a - sh.S[0] / 2, sh.M[0]);
  const int y = pwrap(b - sh.S[1] / 2, sh.M[1]);
  const T *src = q + ((long)x * sh.M[1] + y) * sh.M[2];
  T *dst = p + row * sh.P[2];
  const int h = sh.S[2] / 2, M2 = sh.M[2];
  for (int c = lane; c < sh.P[2]; c += 32) {
    int z = c - h;
    if (z < 0 || z >= M2) z = pwrap(z, M2);
    dst[c] = src[z];
  }
}
template <typename T>
struct KPad {
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { pad_body<T>(c, a...); }
};
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_pad(StencilShape sh, const T *__restrict__ q, T *__restrict__ p) {
  pad_body<T>(hw_ctx(), sh, q, p);
}

// Reference-form sweep: one output per thread, all loops at run time.
// Used for stencil widths beyond the templated range.
template <typename T>
__device__ __forceinline__ void stencil_simple_body(const BlockCtx &ctx, StencilShape sh, const T *__restrict__ p,
                 const T *__restrict__ kh, int khz, T w, T *__restrict__ e) {
  long idx = (long)ctx.b.x * blockDim.x + threadIdx.x;
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
      const T *kr = kh + ((long)i * sh.S[1] + j) * khz;
      T r = 0;
      for (int k = 0; k < sh.S[2]; ++k) r += kr[k] * row[k];
      pl += r;
    }
    acc.add(pl);
  }
  e[idx] = (sh.store ? T(0) : e[idx]) + w * acc.value();
}
template <typename T>
struct KStencilSimple {
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { stencil_simple_body<T>(c, a...); }
};
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_stencil_simple(StencilShape sh, const T *__restrict__ p,
                 const T *__restrict__ kh, int khz, T w, T *__restrict__ e) {
  stencil_simple_body<T>(hw_ctx(), sh, p, kh, khz, w, e);
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::);
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// Copies input plane `plane` of the tile into the shared slice: H rows of
// the WC values the sweep reads (WC <= the row pitch W; the pitch's padding
// columns are never read, and copying them could run past the padded grid).
template <typename T>
__device__ __forceinline__ void stage_plane(const T *__restrict__ P,
                                            const StencilShape &sh, int plane,
                                            int y0, int z0, int H, int W, int WC,
                                            T *slice) {
  constexpr int V = 16 / sizeof(T);
  const int wv = WC / V;
  const int nthreads = blockDim.x * blockDim.y;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const T *src = P + ((long)plane * sh.P[1] + y0) * sh.P[2] + z0;
  for (int t = tid; t < H * wv; t += nthreads) {
    const int row = t / wv, c = t - row * wv;
    cp_async16(slice + row * W + c * V, src + (long)row * sh.P[2] + c * V);
  }
}

// Copies one tap plane (S1 rows of SP, contiguous in global) to shared memory.
template <typename T>
__device__ __forceinline__ void stage_taps(const T *__restrict__ kh, int plane,
                                           int n, T *dst) {
  constexpr int V = 16 / sizeof(T);
  const int nthreads = blockDim.x * blockDim.y;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const T *src = kh + (long)plane * n;
  for (int t = tid; t < n / V; t += nthreads) cp_async16(dst + t * V, src + t * V);
}

// Split over tap planes: CTA z-index = x-tile + ntx * chunk index; chunk k
// sums tap planes i in [k*chunk, min(S0, (k+1)*chunk)). With one chunk the
// result is added to e directly; otherwise each chunk stores its partial sum
// in part[k] and k_split_reduce adds them in fixed order (deterministic).
//
// Taps: kh holds S0 x S1 rows of SP (S rounded up to 16 bytes, zero padded).
// The tap planes in use live in a shared ring of TX+1 planes: step pi uses
// planes i_lo+pi-TX+1 .. i_lo+pi and prefetches plane i_lo+pi+1 into the one
// free slot, together with the next input plane.
template <typename T, int S, int R, int TX>
__device__ __forceinline__ void stencil_tiled_body(const BlockCtx &ctx, StencilShape sh, const T *__restrict__ P,
                const T *__restrict__ kh, T w, T *__restrict__ e,
                int ntx, int chunk, T *__restrict__ part, int W) {
  constexpr int V = 16 / sizeof(T);
  constexpr int SP = (S + V - 1) / V * V;        // tap row pitch
  constexpr int RL = R + S - 1;                  // row values per thread
  constexpr int RLV = (RL + V - 1) / V * V;      // rounded to 16-byte loads
  constexpr int NRING = TX + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *smem = reinterpret_cast<T *>(smem_raw);
  const int NZ = blockDim.x, TY = blockDim.y;
  const int tz = threadIdx.x, ty = threadIdx.y;
  const int S0 = sh.S[0], S1 = sh.S[1];
  const int xt = ctx.b.z % ntx, kc = ctx.b.z / ntx;
  const int i_lo = kc * chunk, i_hi = min(S0, i_lo + chunk);
  const int z0 = ctx.b.x * NZ * R, y0 = ctx.b.y * TY, x0 = xt * TX;
  const int H = TY + S1 - 1;
  const int WC = (NZ - 1) * R + RLV;  // values a row's threads read
  const int slice_elems = H * W + V;  // +V: tail reads of the last row
  const int tap_elems = S1 * SP;
  T *buf0 = smem, *buf1 = smem + slice_elems;
  T *ring = smem + 2 * slice_elems;

  T acc[TX][R];
#pragma unroll
  for (int a = 0; a < TX; ++a)
#pragma unroll
    for (int r = 0; r < R; ++r) acc[a][r] = T(0);

  const int nplanes = TX + (i_hi - i_lo) - 1;
  const int p0 = x0 + i_lo;  // first input plane
  stage_plane(P, sh, p0, y0, z0, H, W, WC, buf0);
  stage_taps(kh, i_lo, tap_elems, ring + (i_lo % NRING) * tap_elems);
  cp_async_commit();
  for (int pi = 0; pi < nplanes; ++pi) {
    if (pi + 1 < nplanes) {
      stage_plane(P, sh, p0 + pi + 1, y0, z0, H, W, WC, (pi & 1) ? buf0 : buf1);
      const int inext = i_lo + pi + 1;
      if (inext < i_hi)
        stage_taps(kh, inext, tap_elems, ring + (inext % NRING) * tap_elems);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const T *slice = (pi & 1) ? buf1 : buf0;
    for (int j = 0; j < S1; ++j) {
      const T *rp = slice + (ty + j) * W + tz * R;
      T row[RLV];
#pragma unroll
      for (int v = 0; v < RLV; v += V) {
        if constexpr (sizeof(T) == 4) {
          const float4 q4 = *reinterpret_cast<const float4 *>(rp + v);
          row[v] = (T)q4.x;
          row[v + 1] = (T)q4.y;
          row[v + 2] = (T)q4.z;
          row[v + 3] = (T)q4.w;
        } else {
          const double2 q2 = *reinterpret_cast<const double2 *>(rp + v);
          row[v] = (T)q2.x;
          row[v + 1] = (T)q2.y;
        }
      }
#pragma unroll
      for (int xo = 0; xo < TX; ++xo) {
        const int i = i_lo + pi - xo;
        if (i < i_lo || i >= i_hi) continue;  // uniform across the CTA
        const T *kp = ring + (i % NRING) * tap_elems + j * SP;
#pragma unroll
        for (int kk = 0; kk < SP; kk += V) {
          T t[V];
          if constexpr (sizeof(T) == 4) {
            const float4 t4 = *reinterpret_cast<const float4 *>(kp + kk);
            t[0] = (T)t4.x;
            t[1] = (T)t4.y;
            t[2] = (T)t4.z;
            t[3] = (T)t4.w;
          } else {
            const double2 t2 = *reinterpret_cast<const double2 *>(kp + kk);
            t[0] = (T)t2.x;
            t[1] = (T)t2.y;
          }
#pragma unroll
          for (int u = 0; u < V; ++u) {
            if (kk + u < S) {
#pragma unroll
              for (int r = 0; r < R; ++r)
                acc[xo][r] = fma(t[u], row[r + kk + u], acc[xo][r]);
            }
          }
        }
      }
    }
    __syncthreads();
  }
  const int y = y0 + ty;
  if (y >= sh.M[1]) return;
  const long mtot = (long)sh.M[0] * sh.M[1] * sh.M[2];
#pragma unroll
  for (int xo = 0; xo < TX; ++xo) {
    const int x = x0 + xo;
    if (x >= sh.M[0]) continue;
    const long row0 = ((long)x * sh.M[1] + y) * sh.M[2];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int z = z0 + tz * R + r;
      if (z >= sh.M[2]) continue;
      if (part)
        part[kc * mtot + row0 + z] = acc[xo][r];
      else
        e[row0 + z] = (sh.store ? T(0) : e[row0 + z]) + w * acc[xo][r];
    }
  }
}
template <typename T, int S, int R, int TX>
struct KStencilTiled {
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { stencil_tiled_body<T, S, R, TX>(c, a...); }
};
template <typename T, int S, int R, int TX>
__global__ void __launch_bounds__(kThreads)
k_stencil_tiled(StencilShape sh, const T *__restrict__ P,
                const T *__restrict__ kh, T w, T *__restrict__ e,
                int ntx, int chunk, T *__restrict__ part, int W) {
  stencil_tiled_body<T, S, R, TX>(hw_ctx(), sh, P, kh, w, e, ntx, chunk, part, W);
}

// Folded sweep for stencils that are mirror-symmetric in x and y (every
// orthorhombic box; S0, S1 odd, centres c0 = S0/2, c1 = S1/2):
//   e[x,y,z] = sum_{i<=c0, j<=c1, k} kf[i][j][k] * F_ij[y][z+k],
//   F_i = P[x+c0+i] + P[x+c0-i] (i > 0; P[x+c0] for i = 0),
//   F_ij[y] = F_i[y+j] + F_i[y+S1-1-j] (j < c1; F_i[y+c1] for j = c1),
// with kf[i][j] the tap shared by the (up to) four mirror images. That is
// (c0+1)(c1+1)S2 multiply-adds per output instead of S0 S1 S2, plus the
// plane and row sums. A CTA owns one output plane x and a TY x (NZ R) tile
// of it; for each i the two input planes stream into shared slices
// (cp.async; the next pair's copies overlap this pair's sweep), are summed in
// shared memory, and every thread forms its folded rows in registers. Split over i: chunk k takes
// i in [k chunk, min(c0+1, (k+1) chunk)), partial sums as in k_stencil_tiled.
// kf: (c0+1) x (c1+1) rows of SP taps (zero padded).
template <typename T, int S, int R>
__device__ __forceinline__ void stencil_fold_body(const BlockCtx &ctx, StencilShape sh, const T *__restrict__ P, const T *__restrict__ kf,
               T w, T *__restrict__ e, int chunk, T *__restrict__ part, int W) {
  constexpr int V = 16 / sizeof(T);
  constexpr int SP = (S + V - 1) / V * V;
  constexpr int RL = R + S - 1;
  constexpr int RLV = (RL + V - 1) / V * V;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *smem = reinterpret_cast<T *>(smem_raw);
  const int NZ = blockDim.x, TY = blockDim.y;
  const int tz = threadIdx.x, ty = threadIdx.y;
  const int nth = NZ * TY, tid = ty * NZ + tz;
  const int S1 = sh.S[1], c0 = sh.S[0] / 2, c1 = S1 / 2;
  const int x = ctx.b.z % sh.M[0], kc = ctx.b.z / sh.M[0];
  const int i_lo = kc * chunk, i_hi = min(c0 + 1, i_lo + chunk);
  const int z0 = ctx.b.x * NZ * R, y0 = ctx.b.y * TY;
  const int H = TY + S1 - 1;
  const int WC = (NZ - 1) * R + RLV;  // values a row's threads read
  const int slice = H * W + V;
  const int tap_elems = (c1 + 1) * SP;
  // shared layout: A slices of stages 0 and 1, one B slice, tap blocks of
  // stages 0 and 1. Step i: wait for its planes, add B into A (B is then
  // free), start the copies of step i+1, and sweep while they land.
  T *Bsl = smem + 2 * slice;

  T acc[R];
#pragma unroll
  for (int r = 0; r < R; ++r) acc[r] = T(0);
  auto stage = [&](int i, int s) {
    stage_plane(P, sh, x + c0 + i, y0, z0, H, W, WC, smem + s * slice);
    if (i > 0) stage_plane(P, sh, x + c0 - i, y0, z0, H, W, WC, Bsl);
    stage_taps(kf + (long)i * tap_elems, 0, tap_elems, smem + 3 * slice + s * tap_elems);
  };
  if (i_lo < i_hi) {
    stage(i_lo, 0);
    cp_async_commit();
  }
  for (int i = i_lo; i < i_hi; ++i) {
    const int s = (i - i_lo) & 1;
    cp_async_wait<0>();
    __syncthreads();
    T *As = smem + s * slice;
    const T *Ks = smem + 3 * slice + s * tap_elems;
    if (i > 0) {  // F_i = A + B, in place
      for (int t = tid; t < H * W / V; t += nth) {
        if constexpr (sizeof(T) == 4) {  // packed adds: the same roundings
          const float4 a = reinterpret_cast<float4 *>(As)[t];
          const float4 b = reinterpret_cast<const float4 *>(Bsl)[t];
          const float2 lo = __fadd2_rn(make_float2(a.x, a.y), make_float2(b.x, b.y));
          const float2 hi = __fadd2_rn(make_float2(a.z, a.w), make_float2(b.z, b.w));
          reinterpret_cast<float4 *>(As)[t] = make_float4(lo.x, lo.y, hi.x, hi.y);
        } else {
          double2 a = reinterpret_cast<double2 *>(As)[t];
          const double2 b = reinterpret_cast<const double2 *>(Bsl)[t];
          a.x += b.x;
          a.y += b.y;
          reinterpret_cast<double2 *>(As)[t] = a;
        }
      }
    }
    __syncthreads();  // B consumed; the other stage's buffers are free
    if (i + 1 < i_hi) {
      stage(i + 1, s ^ 1);
      cp_async_commit();
    }
    const T *F = As;
    for (int j = 0; j <= c1; ++j) {
      const T *r1 = F + (ty + j) * W + tz * R;
      const T *r2 = F + (ty + S1 - 1 - j) * W + tz * R;
      T row[RLV];
#pragma unroll
      for (int v = 0; v < RLV; v += V) {
        if constexpr (sizeof(T) == 4) {
          const float4 a = *reinterpret_cast<const float4 *>(r1 + v);
          row[v] = a.x;
          row[v + 1] = a.y;
          row[v + 2] = a.z;
          row[v + 3] = a.w;
        } else {
          const double2 a = *reinterpret_cast<const double2 *>(r1 + v);
          row[v] = a.x;
          row[v + 1] = a.y;
        }
      }
      if (j < c1) {
#pragma unroll
        for (int v = 0; v < RLV; v += V) {
          if constexpr (sizeof(T) == 4) {  // packed adds: the same roundings
            const float4 b = *reinterpret_cast<const float4 *>(r2 + v);
            const float2 lo =
                __fadd2_rn(make_float2(row[v], row[v + 1]), make_float2(b.x, b.y));
            const float2 hi =
                __fadd2_rn(make_float2(row[v + 2], row[v + 3]), make_float2(b.z, b.w));
            row[v] = lo.x;
            row[v + 1] = lo.y;
            row[v + 2] = hi.x;
            row[v + 3] = hi.y;
          } else {
            const double2 b = *reinterpret_cast<const double2 *>(r2 + v);
            row[v] += b.x;
            row[v + 1] += b.y;
          }
        }
      }
      const T *kp = Ks + j * SP;
#pragma unroll
      for (int kk = 0; kk < SP; kk += V) {
        T t[V];
        if constexpr (sizeof(T) == 4) {
          const float4 t4 = *reinterpret_cast<const float4 *>(kp + kk);
          t[0] = t4.x;
          t[1] = t4.y;
          t[2] = t4.z;
          t[3] = t4.w;
        } else {
          const double2 t2 = *reinterpret_cast<const double2 *>(kp + kk);
          t[0] = t2.x;
          t[1] = t2.y;
        }
#pragma unroll
        for (int u = 0; u < V; ++u) {
          if (kk + u < S) {
#pragma unroll
            for (int r = 0; r < R; ++r) acc[r] = fma(t[u], row[r + kk + u], acc[r]);
          }
        }
      }
    }
  }
  const int y = y0 + ty;
  if (y >= sh.M[1]) return;
  const long mtot = (long)sh.M[0] * sh.M[1] * sh.M[2];
  const long row0 = ((long)x * sh.M[1] + y) * sh.M[2];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int z = z0 + tz * R + r;
    if (z >= sh.M[2]) continue;
    if (part)
      part[kc * mtot + row0 + z] = acc[r];
    else
      e[row0 + z] = (sh.store ? T(0) : e[row0 + z]) + w * acc[r];
  }
}
template <typename T, int S, int R>
struct KStencilFold {
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { stencil_fold_body<T, S, R>(c, a...); }
};
template <typename T, int S, int R>
__global__ void __launch_bounds__(kThreads)
k_stencil_fold(StencilShape sh, const T *__restrict__ P, const T *__restrict__ kf,
               T w, T *__restrict__ e, int chunk, T *__restrict__ part, int W) {
  stencil_fold_body<T, S, R>(hw_ctx(), sh, P, kf, w, e, chunk, part, W);
}

// e (+)= w * sum_k part[k], chunks added in index order
template <typename T>
__device__ __forceinline__ void split_reduce_body(const BlockCtx &ctx, long n, int nsplit, const T *__restrict__ part, T w,
               T *__restrict__ e, int store) {
  long idx = (long)ctx.b.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  T s = part[idx];
  for (int k = 1; k < nsplit; ++k) s += part[k * n + idx];
  e[idx] = (store ? T(0) : e[idx]) + w * s;
}
template <typename T>
struct KSplitReduce {
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { split_reduce_body<T>(c, a...); }
};
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_split_reduce(long n, int nsplit, const T *__restrict__ part, T w,
               T *__restrict__ e, int store) {
  split_reduce_body<T>(hw_ctx(), n, nsplit, part, w, e, store);
}

// R: z outputs per thread; RALT: the folded sweep's alternative for widths
// of at least kMinSAlt taps (more outputs per loaded row: the folded sweep
// reads two rows per tap row, and shared-memory bandwidth, not the FMA pipe,
// bounds it at the default R)
template <typename T> struct TileDefaults;
template <> struct TileDefaults<float> { static constexpr int R = 8, TX = 4, RALT = 12; };
template <> struct TileDefaults<double> { static constexpr int R = 4, TX = 4, RALT = 8; };
constexpr int kMinSAlt = 9;

int tile_r_of(const StencilTile &tl, bool fp64) {
  const int d = fp64 ? TileDefaults<double>::R : TileDefaults<float>::R;
  return tl.r > 0 ? tl.r : d;
}

// shared memory of the folded sweep: two A slices, one B slice, two tap blocks
template <typename T>
size_t fold_smem_bytes(const StencilShape &sh, const StencilTile &tl) {
  const int R = tile_r_of(tl, sizeof(T) == 8);
  constexpr int V = 16 / sizeof(T);
  const int H = tl.ty + sh.S[1] - 1;
  const int W = slice_pitch(tl.nz, R, sh.S[2], V);
  const int SP = stencil_tap_pitch(sh.S[2], sizeof(T) == 8);
  return (3 * (size_t)(H * W + V) + 2 * (size_t)(sh.S[1] / 2 + 1) * SP) * sizeof(T);
}

template <typename T, int S>
void launch_tiled(cudaStream_t s, const StencilShape &sh, const StencilTile &tl,
                  const T *p, const T *kh, int khz, T w, T *e, T *part) {
  constexpr int R = TileDefaults<T>::R, TX = TileDefaults<T>::TX;
  constexpr int V = 16 / sizeof(T);
  const int H = tl.ty + sh.S[1] - 1;
  const int W = slice_pitch(tl.nz, R, S, V);
  const size_t smem = (2 * (size_t)(H * W + V) +
                       (size_t)(TX + 1) * sh.S[1] * stencil_tap_pitch(S, sizeof(T) == 8)) *
                      sizeof(T);
  const int ntx = (sh.M[0] + TX - 1) / TX;
  const int nsplit = std::max(1, tl.nsplit);
  const int chunk = (sh.S[0] + nsplit - 1) / nsplit;
  dim3 block(tl.nz, tl.ty);
  dim3 grid((sh.M[2] + tl.nz * R - 1) / (tl.nz * R), (sh.M[1] + tl.ty - 1) / tl.ty,
            ntx * nsplit);
  (void)khz;  // the tiled kernel reads rows of the padded pitch
  launch<KStencilTiled<T, S, R, TX>, kThreads, sizeof(T) == 4 ? 2 : 1>(s, k_stencil_tiled<T, S, R, TX>, grid, block, smem, sh, p, kh, w, e, ntx, chunk, nsplit > 1 ? part : nullptr, W);
  if (nsplit > 1) {
    const long n = (long)sh.M[0] * sh.M[1] * sh.M[2];
    launch<KSplitReduce<T>, kThreads, 8>(s, k_split_reduce<T>, blocks_for(n), kThreads, 0, n, nsplit, part, w, e, sh.store);
  }
}

template <typename T, int S, int R>
void launch_fold_r(cudaStream_t s, const StencilShape &sh, const StencilTile &tl,
                   const T *p, const T *kf, T w, T *e, T *part) {
  constexpr int V = 16 / sizeof(T);
  const int nI = sh.S[0] / 2 + 1;
  const int nsplit = std::max(1, tl.nsplit);
  const int chunk = (nI + nsplit - 1) / nsplit;
  dim3 block(tl.nz, tl.ty);
  dim3 grid((sh.M[2] + tl.nz * R - 1) / (tl.nz * R), (sh.M[1] + tl.ty - 1) / tl.ty,
            sh.M[0] * nsplit);
  launch<KStencilFold<T, S, R>, kThreads, sizeof(T) == 4 ? 3 : 2>(s, k_stencil_fold<T, S, R>, grid, block, fold_smem_bytes<T>(sh, tl), sh, p, kf, w, e, chunk, nsplit > 1 ? part : nullptr, slice_pitch(tl.nz, R, S, V));
  if (nsplit > 1) {
    const long n = (long)sh.M[0] * sh.M[1] * sh.M[2];
    launch<KSplitReduce<T>, kThreads, 8>(s, k_split_reduce<T>, blocks_for(n), kThreads, 0, n, nsplit, part, w, e, sh.store);
  }
}

template <typename T, int S>
void launch_fold(cudaStream_t s, const StencilShape &sh, const StencilTile &tl,
                 const T *p, const T *kf, T w, T *e, T *part) {
  if constexpr (S >= kMinSAlt) {
    if (tile_r_of(tl, sizeof(T) == 8) == TileDefaults<T>::RALT) {
      launch_fold_r<T, S, TileDefaults<T>::RALT>(s, sh, tl, p, kf, w, e, part);
      return;
    }
  }
  launch_fold_r<T, S, TileDefaults<T>::R>(s, sh, tl, p, kf, w, e, part);
}

// Levels (and plans) that share an instantiation need the largest request:
// the attribute is per kernel function and per device, so it is only ever
// raised, and the level granted is kept per device.
// fold: 0 tiled sweep, 1 folded sweep at the default R, 2 at the alternative
template <typename T, int S>
void set_smem_attr(int bytes, int fold) {
  constexpr int R = TileDefaults<T>::R, TX = TileDefaults<T>::TX;
  static std::mutex mu;
  static int current[kMaxDevices][3];
  const int dev = device_slot();
  std::lock_guard<std::mutex> lock(mu);
  if (dev >= 0 && bytes <= std::max(current[dev][fold], 48 * 1024)) return;
  cudaError_t err = cudaErrorInvalidValue;
  if (fold == 0) {
    err = cudaFuncSetAttribute(k_stencil_tiled<T, S, R, TX>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  } else if (fold == 1) {
    err = cudaFuncSetAttribute(k_stencil_fold<T, S, R>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  } else if constexpr (S >= kMinSAlt) {
    err = cudaFuncSetAttribute(k_stencil_fold<T, S, TileDefaults<T>::RALT>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  }
  if (err == cudaSuccess && dev >= 0) current[dev][fold] = bytes;
}

#define MSM_S_CASES(X) \
  X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) \
  X(15) X(16) X(17) X(18) X(19) X(20) X(21) X(22) X(23) X(24) X(25) X(26)    \
  X(27) X(28) X(29) X(30) X(31) X(32) X(33)

}  // namespace

int stencil_tile_r(const StencilTile &tile, bool fp64) { return tile_r_of(tile, fp64); }

int stencil_alt_r(const StencilShape &sh, bool fp64) {
  if (!sh.sym || sh.S[2] < kMinSAlt || sh.S[2] > kMaxTemplatedS) return 0;
  return fp64 ? TileDefaults<double>::RALT : TileDefaults<float>::RALT;
}

StencilTile stencil_default_tile(const StencilShape &sh, bool fp64) {
  const int R = fp64 ? TileDefaults<double>::R : TileDefaults<float>::R;
  const int TX = sh.sym ? 1 : (fp64 ? TileDefaults<double>::TX : TileDefaults<float>::TX);
  StencilTile t;
  t.tx = TX;
  // Tile shape: least padding waste, then least shared-memory traffic per
  // output (halo ratio), with at least two warps per CTA where possible.
  double best = 1e30;
  for (int nz = 1; nz <= 16; ++nz)
    for (int ty : {16, 12, 8, 6, 4, 2, 1}) {
      const int th = nz * ty;
      if (th > kThreads || (ty > sh.M[1] && ty > 1)) continue;
      const int span = nz * R;
      if (span > sh.M[2] + R - 1 && nz > 1) continue;
      const double wz = (double)((sh.M[2] + span - 1) / span * span) / sh.M[2];
      const double wy = (double)((sh.M[1] + ty - 1) / ty * ty) / sh.M[1];
      const double halo = (double)(ty + sh.S[1] - 1) * (span + sh.S[2] - 1) / (ty * span);
      const double score = wz * wy * (1.0 + 0.03 * halo) + (th < 64 ? 0.25 : 0.0);
      if (score < best - 1e-12) {
        best = score;
        t.nz = nz;
        t.ty = ty;
      }
    }
  // Split the tap planes over CTAs until the grid fills the GPU (about four
  // CTAs per SM); every chunk keeps at least one plane.
  const long tiles = (long)((sh.M[2] + t.nz * R - 1) / (t.nz * R)) *
                     ((sh.M[1] + t.ty - 1) / t.ty) * ((sh.M[0] + TX - 1) / TX);
  const int nI = sh.sym ? sh.S[0] / 2 + 1 : sh.S[0];  // tap planes to split
  int ns = (int)std::min<long>(nI, std::max<long>(1, (148L * 4 + tiles - 1) / tiles));
  const int chunk = (nI + ns - 1) / ns;
  t.nsplit = (nI + chunk - 1) / chunk;
  return t;
}

int stencil_tap_pitch(int S2, bool fp64) {
  const int V = fp64 ? 2 : 4;
  return (S2 + V - 1) / V * V;
}

bool stencil_templated(const StencilShape &sh) {
  return sh.S[2] >= 1 && sh.S[2] <= kMaxTemplatedS;
}

void stencil_padded_dims(const StencilShape &sh, const StencilTile &tl,
                         bool fp64, int P[3]) {
  const int R = tile_r_of(tl, fp64);
  const int V = fp64 ? 2 : 4;
  const int span = tl.nz * R;
  const int mz = (sh.M[2] + span - 1) / span * span;
  const int my = (sh.M[1] + tl.ty - 1) / tl.ty * tl.ty;
  const int mx = (sh.M[0] + tl.tx - 1) / tl.tx * tl.tx;
  P[0] = mx + sh.S[0] - 1;
  P[1] = my + sh.S[1] - 1;
  // rows of the last z tile reach z0 + W (+V: 16-byte tail reads)
  P[2] = ((mz + sh.S[2] - 1 + V - 1) / V) * V + 2 * V;
}

template <typename T>
int stencil_prepare(const StencilShape &sh, const StencilTile &tl) {
  if (!stencil_templated(sh)) return 0;
  const int R = tile_r_of(tl, sizeof(T) == 8);
  if (R != TileDefaults<T>::R && R != stencil_alt_r(sh, sizeof(T) == 8)) return -1;
  constexpr int V = 16 / sizeof(T);
  const int H = tl.ty + sh.S[1] - 1;
  const int W = slice_pitch(tl.nz, R, sh.S[2], V);
  const int bytes =
      sh.sym ? (int)fold_smem_bytes<T>(sh, tl)
             : (2 * (H * W + V) +
                (tl.tx + 1) * sh.S[1] * stencil_tap_pitch(sh.S[2], sizeof(T) == 8)) *
                   (int)sizeof(T);
  if (bytes > 200 * 1024) return -1;
  switch (sh.S[2]) {
#define X(SS) \
  case SS:                                                                         \
    set_smem_attr<T, SS>(bytes, !sh.sym ? 0 : (R == TileDefaults<T>::R ? 1 : 2)); \
    break;
    MSM_S_CASES(X)
#undef X
  }
  return 0;
}

bool stencil_fold_taps(const double *kh, const int S[3], bool fp64,
                       std::vector<double> &kf) {
  kf.clear();
  if (S[0] % 2 == 0 || S[1] % 2 == 0) return false;
  const int S0 = S[0], S1 = S[1], S2 = S[2], c0 = S0 / 2, c1 = S1 / 2;
  auto at = [&](int i, int j, int k) { return kh[((size_t)i * S1 + j) * S2 + k]; };
  double amax = 0;
  for (size_t n = 0; n < (size_t)S0 * S1 * S2; ++n) amax = std::max(amax, std::fabs(kh[n]));
  const double tol = 1e-12 * amax;
  for (int i = 0; i < S0; ++i)
    for (int j = 0; j < S1; ++j)
      for (int k = 0; k < S2; ++k)
        if (std::fabs(at(i, j, k) - at(S0 - 1 - i, j, k)) > tol ||
            std::fabs(at(i, j, k) - at(i, S1 - 1 - j, k)) > tol)
          return false;
  const int SP = stencil_tap_pitch(S2, fp64);
  kf.assign((size_t)(c0 + 1) * (c1 + 1) * SP, 0.0);
  for (int i = 0; i <= c0; ++i)
    for (int j = 0; j <= c1; ++j)
      for (int k = 0; k < S2; ++k) {
        const double v = at(c0 + i, c1 + j, k) + at(c0 - i, c1 + j, k) +
                         at(c0 + i, c1 - j, k) + at(c0 - i, c1 - j, k);
        // row j of the folded block pairs rows j and S1-1-j: tap index c1 - j'
        kf[((size_t)i * (c1 + 1) + (c1 - j)) * SP + k] = 0.25 * v;
      }
  return true;
}

template <typename T>
void launch_pad(cudaStream_t s, const StencilShape &sh, const T *q, T *p) {
  const long rows = (long)sh.P[0] * sh.P[1];
  const int per = kThreads / 32;
  launch<KPad<T>, kThreads, 8>(s, k_pad<T>, dim3((unsigned)((rows + per - 1) / per)), kThreads, 0,
                               sh, q, p);
}

template <typename T>
void launch_stencil(cudaStream_t s, const StencilShape &sh, const StencilTile &tl,
                    const T *p, const T *kh, int khz, T w, T *e, T *part) {
  if (!stencil_templated(sh) || tl.nz <= 0) {
    long n = (long)sh.M[0] * sh.M[1] * sh.M[2];
    launch<KStencilSimple<T>, kThreads, 1>(s, k_stencil_simple<T>, blocks_for(n), kThreads, 0, sh, p, kh, khz, w, e);
    return;
  }
  switch (sh.S[2]) {
#define X(SS)                                                      \
  case SS:                                                         \
    if (sh.sym)                                                    \
      launch_fold<T, SS>(s, sh, tl, p, kh, w, e, part);            \
    else                                                           \
      launch_tiled<T, SS>(s, sh, tl, p, kh, khz, w, e, part);      \
    break;
    MSM_S_CASES(X)
#undef X
  }
}

// kernels one launch_stencil issues: the sweep, plus the reduction of the
// split tap-plane partial sums when the tile splits them
int stencil_launches(const StencilShape &sh, const StencilTile &tl) {
  if (!stencil_templated(sh) || tl.nz <= 0) return 1;
  return tl.nsplit > 1 ? 2 : 1;
}

template void launch_pad<float>(cudaStream_t, const StencilShape &,
                                const float *, float *);
template void launch_pad<double>(cudaStream_t, const StencilShape &,
                                 const double *, double *);
template void launch_stencil<float>(cudaStream_t, const StencilShape &,
                                    const StencilTile &, const float *,
                                    const float *, int, float, float *, float *);
template void launch_stencil<double>(cudaStream_t, const StencilShape &,
                                     const StencilTile &, const double *,
                                     const double *, int, double, double *,
                                     double *);
template int stencil_prepare<float>(const StencilShape &, const StencilTile &);
template int stencil_prepare<double>(const StencilShape &, const StencilTile &);

}  // namespace msm
