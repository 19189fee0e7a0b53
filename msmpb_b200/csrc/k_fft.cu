// Top-level periodic solve (code/forcefield1.c:499-528):
//   e^L = IFFT( w_L * khat_L .* FFT(q^L) ) / (M0 M1 M2)
// as a hand-written FP64 mixed-radix Stockham FFT (self-sorting, ping-pong
// buffers in shared memory). Radices 4, 2, 3, 5, 7 cover the 7-smooth sizes
// the reference selects (code/forcefield0.c:219-245); any other prime factor
// runs as a direct length-p DFT stage. Grids whose y-z plane fits in shared
// memory take three launches (plane forward, x-lines with the khat multiply,
// plane inverse; below); larger ones five line passes, each CTA staging a
// batch of lines along one axis, the middle pass running forward x, the khat
// multiply and inverse x in one launch.
#include <algorithm>

#include "kernels.h"

namespace msm {
namespace {

constexpr int kThreads = 256;
constexpr int kMaxFactors = 24;
constexpr int kMaxRadix = 64;

struct FftLines {
  int n;        // line length
  int nlines;   // number of lines
  int inner;    // element stride of a line (product of the faster dims)
  int lpb;      // lines per block
  int nf;       // number of radix stages
  int radix[kMaxFactors];
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// exp(sign * 2 pi i * num / den), argument reduced exactly
__device__ __forceinline__ double2 twiddle(int sign, long num, long den) {
  long r = num % den;
  double s, c;
  sincospi(2.0 * (double)r / (double)den, &s, &c);
  return make_double2(c, sign * s);
}

// One radix stage over every line held in shared memory
__device__ void stockham_stage(const FftLines &f, int R, int Ns, int sign,
                               const double2 *src, double2 *dst) {
  const int n = f.n, m = n / R;
  double2 v[kMaxRadix], y[kMaxRadix];
  for (int t = threadIdx.x; t < f.lpb * m; t += blockDim.x) {
    const int line = t / m, j = t % m;
    const double2 *s = src + line * n;
    double2 *d = dst + line * n;
    const int k = j % Ns;
    for (int r = 0; r < R; ++r) {
      double2 a = s[j + r * m];
      v[r] = r == 0 ? a : cmul(a, twiddle(sign, (long)k * r, (long)Ns * R));
    }
    if (R == 2) {
      y[0] = make_double2(v[0].x + v[1].x, v[0].y + v[1].y);
      y[1] = make_double2(v[0].x - v[1].x, v[0].y - v[1].y);
    } else if (R == 4) {
      double2 a0 = make_double2(v[0].x + v[2].x, v[0].y + v[2].y);
      double2 a1 = make_double2(v[0].x - v[2].x, v[0].y - v[2].y);
      double2 b0 = make_double2(v[1].x + v[3].x, v[1].y + v[3].y);
      double2 b1 = make_double2(v[1].x - v[3].x, v[1].y - v[3].y);
      // multiply b1 by sign * i
      double2 b1i = make_double2(-sign * b1.y, sign * b1.x);
      y[0] = make_double2(a0.x + b0.x, a0.y + b0.y);
      y[2] = make_double2(a0.x - b0.x, a0.y - b0.y);
      y[1] = make_double2(a1.x + b1i.x, a1.y + b1i.y);
      y[3] = make_double2(a1.x - b1i.x, a1.y - b1i.y);
    } else {
      for (int q = 0; q < R; ++q) {
        double2 acc = v[0];
        for (int r = 1; r < R; ++r) {
          double2 w = twiddle(sign, (long)r * q, R);
          double2 p = cmul(v[r], w);
          acc.x += p.x;
          acc.y += p.y;
        }
        y[q] = acc;
      }
    }
    const int base = (j / Ns) * Ns * R + k;
    for (int r = 0; r < R; ++r) d[base + r * Ns] = y[r];
  }
}

// Runs the stages of one direction; returns the buffer holding the result.
__device__ double2 *run_stages(const FftLines &f, int sign, double2 *a,
                               double2 *b) {
  int Ns = 1;
  for (int s = 0; s < f.nf; ++s) {
    const int R = f.radix[s];
    stockham_stage(f, R, Ns, sign, a, b);
    __syncthreads();
    double2 *t = a;
    a = b;
    b = t;
    Ns *= R;
  }
  return a;
}

__device__ __forceinline__ long line_elem(const FftLines &f, int gline, int e) {
  return (long)(gline / f.inner) * ((long)f.n * f.inner) + gline % f.inner +
         (long)e * f.inner;
}

// mode 0: complex in -> forward -> complex out
// mode 1: real T in -> forward -> complex out
// mode 2: complex in -> forward, * (w khat), inverse -> complex out
// mode 3: complex in -> inverse -> real T out (scaled)
// mode 4: complex in -> inverse -> complex out
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_fft_pass(FftLines f, int mode, const T *__restrict__ rin,
           const double2 *in, double2 *out, const double *__restrict__ khat,
           double w, T *__restrict__ rout, double scale) {
  extern __shared__ double2 smem[];
  double2 *a = smem, *b = smem + f.lpb * f.n;
  const int line0 = blockIdx.x * f.lpb;
  for (int t = threadIdx.x; t < f.lpb * f.n; t += blockDim.x) {
    const int line = t / f.n, e = t % f.n, g = line0 + line;
    double2 v = make_double2(0., 0.);
    if (g < f.nlines) {
      const long gi = line_elem(f, g, e);
      v = (mode == 1) ? make_double2((double)rin[gi], 0.) : in[gi];
    }
    a[t] = v;
  }
  __syncthreads();
  const int sign = (mode >= 3) ? +1 : -1;
  double2 *res = run_stages(f, sign, a, b);
  if (mode == 2) {
    for (int t = threadIdx.x; t < f.lpb * f.n; t += blockDim.x) {
      const int line = t / f.n, e = t % f.n, g = line0 + line;
      if (g < f.nlines) {
        const double kv = w * khat[line_elem(f, g, e)];
        res[t].x *= kv;
        res[t].y *= kv;
      }
    }
    __syncthreads();
    double2 *other = (res == a) ? b : a;
    res = run_stages(f, +1, res, other);
  }
  for (int t = threadIdx.x; t < f.lpb * f.n; t += blockDim.x) {
    const int line = t / f.n, e = t % f.n, g = line0 + line;
    if (g >= f.nlines) continue;
    const long gi = line_elem(f, g, e);
    if (mode == 3)
      rout[gi] = (T)(res[t].x * scale);
    else
      out[gi] = res[t];
  }
}

FftLines make_lines(int n, int nlines, int inner) {
  FftLines f{};
  f.n = n;
  f.nlines = nlines;
  f.inner = inner;
  int r = n;
  while (r % 4 == 0 && f.nf < kMaxFactors) { f.radix[f.nf++] = 4; r /= 4; }
  for (int p : {2, 3, 5, 7})
    while (r % p == 0 && f.nf < kMaxFactors) { f.radix[f.nf++] = p; r /= p; }
  for (int p = 11; r > 1 && f.nf < kMaxFactors; p += 2)
    while (r % p == 0 && f.nf < kMaxFactors) { f.radix[f.nf++] = p; r /= p; }
  int lpb = std::max(1, 1024 / std::max(1, n));
  f.lpb = std::min(lpb, nlines);
  return f;
}

template <typename T>
void run_pass(cudaStream_t s, const FftLines &f, int mode, const T *rin,
              const double2 *in, double2 *out, const double *khat, double w,
              T *rout, double scale) {
  size_t smem = 2 * (size_t)f.lpb * f.n * sizeof(double2);
  int blocks = (f.nlines + f.lpb - 1) / f.lpb;
  k_fft_pass<T><<<blocks, kThreads, smem, s>>>(f, mode, rin, in, out, khat, w,
                                               rout, scale);
}

// ---------------------------------------------------------------------------
// Small and medium grids (the y-z plane fits in shared memory): three
// launches instead of five. k_fft_plane transforms one x-plane along z and y
// (forward, from the real grid) or along y and z (inverse, to the real grid,
// scaled); k_fft_xlines runs forward x, the khat multiply and inverse x on 32
// adjacent x-lines per CTA (adjacent in memory, so every load and store is
// coalesced). Twiddles come from a table of the n-th roots of unity per axis
// built in shared memory at kernel start (one sincospi per entry, not per
// butterfly), and the butterflies of radix 2, 3, 4, 5, 7 are unrolled with
// their operands in registers.

struct FftAxis {
  int n, nf;
  int radix[kMaxFactors];
};

FftAxis make_axis(int n) {
  FftLines l = make_lines(n, 1, 1);
  FftAxis a{};
  a.n = n;
  a.nf = l.nf;
  for (int i = 0; i < l.nf; ++i) a.radix[i] = l.radix[i];
  return a;
}

// W[j] = exp(-2 pi i j / n), j < n
__device__ void root_table(int n, double2 *W) {
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    double s, c;
    sincospi(2.0 * (double)j / (double)n, &s, &c);
    W[j] = make_double2(c, -s);
  }
}

// exp(sign 2 pi i j / n) from the forward table
__device__ __forceinline__ double2 root(const double2 *W, int j, int sign) {
  const double2 w = W[j];
  return sign < 0 ? w : make_double2(w.x, -w.y);
}

template <int R>
__device__ __forceinline__ void butterfly(double2 (&v)[R], double2 (&y)[R],
                                          const double2 *W, int n, int sign) {
  if (R == 2) {
    y[0] = make_double2(v[0].x + v[1].x, v[0].y + v[1].y);
    y[1] = make_double2(v[0].x - v[1].x, v[0].y - v[1].y);
  } else if (R == 4) {
    const double2 a0 = make_double2(v[0].x + v[2].x, v[0].y + v[2].y);
    const double2 a1 = make_double2(v[0].x - v[2].x, v[0].y - v[2].y);
    const double2 b0 = make_double2(v[1].x + v[3].x, v[1].y + v[3].y);
    const double2 b1 = make_double2(v[1].x - v[3].x, v[1].y - v[3].y);
    const double2 b1i = make_double2(-sign * b1.y, sign * b1.x);  // sign * i * b1
    y[0] = make_double2(a0.x + b0.x, a0.y + b0.y);
    y[2] = make_double2(a0.x - b0.x, a0.y - b0.y);
    y[1] = make_double2(a1.x + b1i.x, a1.y + b1i.y);
    y[3] = make_double2(a1.x - b1i.x, a1.y - b1i.y);
  } else {  // direct DFT of odd prime length
    const int step = n / R;
#pragma unroll
    for (int q = 0; q < R; ++q) {
      double2 acc = v[0];
#pragma unroll
      for (int r = 1; r < R; ++r) {
        const double2 p = cmul(v[r], root(W, ((r * q) % R) * step, sign));
        acc.x += p.x;
        acc.y += p.y;
      }
      y[q] = acc;
    }
  }
}

// One Stockham stage of radix R on nl lines held in shared memory; element e
// of line l sits at l * ls + e * es in src and dst. line_fast: consecutive
// threads take consecutive lines (lines adjacent in memory), else
// consecutive butterflies of one line.
template <int R>
__device__ void stage_r(int n, int Ns, int nl, int ls, int es, bool line_fast, int sign,
                        const double2 *W, const double2 *src, double2 *dst) {
  const int m = n / R, ts = n / (Ns * R);
  for (int t = threadIdx.x; t < nl * m; t += blockDim.x) {
    const int line = line_fast ? t % nl : t / m;
    const int j = line_fast ? t / nl : t % m;
    const int k = j % Ns;
    const double2 *s = src + line * ls;
    double2 v[R], y[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const double2 a = s[(j + r * m) * es];
      v[r] = r == 0 ? a : cmul(a, root(W, (k * r * ts) % n, sign));
    }
    butterfly<R>(v, y, W, n, sign);
    double2 *d = dst + line * ls;
    const int base = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) d[(base + r * Ns) * es] = y[r];
  }
}

// Radix stage of any other prime length (operands in local memory)
__device__ void stage_generic(int R, int n, int Ns, int nl, int ls, int es, bool line_fast,
                              int sign, const double2 *W, const double2 *src,
                              double2 *dst) {
  const int m = n / R, ts = n / (Ns * R), step = n / R;
  double2 v[kMaxRadix];
  for (int t = threadIdx.x; t < nl * m; t += blockDim.x) {
    const int line = line_fast ? t % nl : t / m;
    const int j = line_fast ? t / nl : t % m;
    const int k = j % Ns;
    const double2 *s = src + line * ls;
    for (int r = 0; r < R; ++r) {
      const double2 a = s[(j + r * m) * es];
      v[r] = r == 0 ? a : cmul(a, root(W, (k * r * ts) % n, sign));
    }
    double2 *d = dst + line * ls;
    const int base = (j / Ns) * Ns * R + k;
    for (int q = 0; q < R; ++q) {
      double2 acc = v[0];
      for (int r = 1; r < R; ++r) {
        const double2 p = cmul(v[r], root(W, ((r * q) % R) * step, sign));
        acc.x += p.x;
        acc.y += p.y;
      }
      d[(base + q * Ns) * es] = acc;
    }
  }
}

// All stages of one axis; returns the buffer that holds the result.
__device__ double2 *axis_fft(const FftAxis &ax, int nl, int ls, int es, bool line_fast,
                             int sign, const double2 *W, double2 *a, double2 *b) {
  int Ns = 1;
  for (int s = 0; s < ax.nf; ++s) {
    const int R = ax.radix[s];
    switch (R) {
      case 2: stage_r<2>(ax.n, Ns, nl, ls, es, line_fast, sign, W, a, b); break;
      case 3: stage_r<3>(ax.n, Ns, nl, ls, es, line_fast, sign, W, a, b); break;
      case 4: stage_r<4>(ax.n, Ns, nl, ls, es, line_fast, sign, W, a, b); break;
      case 5: stage_r<5>(ax.n, Ns, nl, ls, es, line_fast, sign, W, a, b); break;
      case 7: stage_r<7>(ax.n, Ns, nl, ls, es, line_fast, sign, W, a, b); break;
      default: stage_generic(R, ax.n, Ns, nl, ls, es, line_fast, sign, W, a, b);
    }
    __syncthreads();
    double2 *t = a;
    a = b;
    b = t;
    Ns *= R;
  }
  return a;
}

constexpr int kPlaneThreads = 256;
constexpr int kXLines = 32;
constexpr size_t kPlaneSmemMax = 200 * 1024;

// smem row pitch of a plane: odd, so z-lines and y-lines are both
// conflict-free for 16-byte elements
__host__ __device__ __forceinline__ int plane_pitch(int M2) { return M2 | 1; }

size_t plane_smem(const int M[3]) {
  return (2 * (size_t)M[1] * plane_pitch(M[2]) + M[1] + M[2]) * sizeof(double2);
}
size_t xlines_smem(int M0) { return (2 * (size_t)kXLines * M0 + M0) * sizeof(double2); }

// inverse = 0: real q (this plane) -> forward z, forward y -> complex buf
// inverse = 1: complex buf -> inverse y, inverse z -> real e (scaled)
template <typename T>
__global__ void __launch_bounds__(kPlaneThreads)
k_fft_plane(FftAxis ay, FftAxis az, int inverse, const T *__restrict__ rin, double2 *buf,
            T *__restrict__ rout, double scale) {
  extern __shared__ double2 smem[];
  const int M1 = ay.n, M2 = az.n, P = plane_pitch(M2);
  double2 *a = smem, *b = smem + M1 * P, *Wy = smem + 2 * M1 * P, *Wz = Wy + M1;
  root_table(M1, Wy);
  root_table(M2, Wz);
  const long base = (long)blockIdx.x * M1 * M2;
  for (int t = threadIdx.x; t < M1 * M2; t += blockDim.x) {
    const int y = t / M2, z = t % M2;
    a[y * P + z] = inverse ? buf[base + t] : make_double2((double)rin[base + t], 0.);
  }
  __syncthreads();
  double2 *res;
  if (!inverse) {
    res = axis_fft(az, M1, P, 1, false, -1, Wz, a, b);  // z-lines: rows
    double2 *o = res == a ? b : a;
    res = axis_fft(ay, M2, 1, P, true, -1, Wy, res, o);  // y-lines: columns
  } else {
    res = axis_fft(ay, M2, 1, P, true, +1, Wy, a, b);
    double2 *o = res == a ? b : a;
    res = axis_fft(az, M1, P, 1, false, +1, Wz, res, o);
  }
  for (int t = threadIdx.x; t < M1 * M2; t += blockDim.x) {
    const int y = t / M2, z = t % M2;
    const double2 v = res[y * P + z];
    if (inverse)
      rout[base + t] = (T)(v.x * scale);
    else
      buf[base + t] = v;
  }
}

// Forward x, times w * khat, inverse x on kXLines adjacent x-lines
__global__ void __launch_bounds__(kPlaneThreads)
k_fft_xlines(FftAxis ax, int nlines, const double *__restrict__ khat, double w, double2 *buf) {
  extern __shared__ double2 smem[];
  const int n = ax.n, L = kXLines;
  double2 *a = smem, *b = smem + L * n, *W = smem + 2 * L * n;
  root_table(n, W);
  const int line0 = blockIdx.x * L;
  for (int t = threadIdx.x; t < L * n; t += blockDim.x) {
    const int l = t % L, e = t / L, g = line0 + l;
    a[e * L + l] = g < nlines ? buf[(long)e * nlines + g] : make_double2(0., 0.);
  }
  __syncthreads();
  double2 *res = axis_fft(ax, L, 1, L, true, -1, W, a, b);
  for (int t = threadIdx.x; t < L * n; t += blockDim.x) {
    const int l = t % L, e = t / L, g = line0 + l;
    const double kv = g < nlines ? w * khat[(long)e * nlines + g] : 0.;
    res[t].x *= kv;
    res[t].y *= kv;
  }
  __syncthreads();
  double2 *o = res == a ? b : a;
  res = axis_fft(ax, L, 1, L, true, +1, W, res, o);
  for (int t = threadIdx.x; t < L * n; t += blockDim.x) {
    const int l = t % L, e = t / L, g = line0 + l;
    if (g < nlines) buf[(long)e * nlines + g] = res[e * L + l];
  }
}

bool plane_path(const int M[3]) {
  return plane_smem(M) <= kPlaneSmemMax && xlines_smem(M[0]) <= kPlaneSmemMax;
}

}  // namespace

// One-time kernel attribute: lines up to 4096 points need 128 KB of
// shared memory (two buffers of one line). Called outside stream capture.
void top_solve_prepare() {
  static bool done = false;
  if (done) return;
  const int bytes = 2 * 4096 * (int)sizeof(double2);
  cudaFuncSetAttribute(k_fft_pass<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  cudaFuncSetAttribute(k_fft_pass<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  cudaFuncSetAttribute(k_fft_plane<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)kPlaneSmemMax);
  cudaFuncSetAttribute(k_fft_plane<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)kPlaneSmemMax);
  cudaFuncSetAttribute(k_fft_xlines, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)kPlaneSmemMax);
  done = true;
}

// largest supported line length (radix factors <= kMaxRadix, smem <= 128 KB)
bool top_solve_supported(const int M[3]) {
  for (int k = 0; k < 3; ++k) {
    if (M[k] < 1 || M[k] > 4096) return false;
    int r = M[k];
    for (int p = 2; p <= kMaxRadix && r > 1; ++p)
      while (r % p == 0) r /= p;
    if (r != 1) return false;
  }
  return true;
}

int top_solve_launches(const int M[3]) { return plane_path(M) ? 3 : 5; }

template <typename T>
void launch_top_solve(cudaStream_t s, const int M[3], const T *q,
                      const double *khat, double weight, double2 *buf0,
                      double2 *buf1, T *e) {
  (void)buf1;
  const int M0 = M[0], M1 = M[1], M2 = M[2];
  const double scale = 1.0 / ((double)M0 * M1 * M2);
  if (plane_path(M)) {
    const FftAxis ax = make_axis(M0), ay = make_axis(M1), az = make_axis(M2);
    const size_t ps = plane_smem(M), xs = xlines_smem(M0);
    const int nl = M1 * M2;
    k_fft_plane<T><<<M0, kPlaneThreads, ps, s>>>(ay, az, 0, q, buf0, nullptr, 0.);
    k_fft_xlines<<<(nl + kXLines - 1) / kXLines, kPlaneThreads, xs, s>>>(ax, nl, khat, weight,
                                                                         buf0);
    k_fft_plane<T><<<M0, kPlaneThreads, ps, s>>>(ay, az, 1, nullptr, buf0, e, scale);
    return;
  }
  FftLines fz = make_lines(M2, M0 * M1, 1);
  FftLines fy = make_lines(M1, M0 * M2, M2);
  FftLines fx = make_lines(M0, M1 * M2, M1 * M2);
  run_pass<T>(s, fz, 1, q, nullptr, buf0, nullptr, 0., nullptr, 0.);
  run_pass<T>(s, fy, 0, nullptr, buf0, buf0, nullptr, 0., nullptr, 0.);
  run_pass<T>(s, fx, 2, nullptr, buf0, buf0, khat, weight, nullptr, 0.);
  FftLines iy = fy;
  run_pass<T>(s, iy, 4, nullptr, buf0, buf0, nullptr, 0., nullptr, 0.);
  run_pass<T>(s, fz, 3, nullptr, buf0, nullptr, nullptr, 0., e, scale);
}

template void launch_top_solve<float>(cudaStream_t, const int *, const float *,
                                      const double *, double, double2 *,
                                      double2 *, float *);
template void launch_top_solve<double>(cudaStream_t, const int *,
                                       const double *, const double *, double,
                                       double2 *, double2 *, double *);

}  // namespace msm
