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

#include <mutex>

#include "kernels.h"

namespace msm {
namespace {

constexpr int kMaxFactors = 24;
constexpr int kMaxRadix = 64;

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
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

// radix 4 first, then 2, 3, 5, 7, then any other prime
FftAxis make_axis(int n) {
  FftAxis a{};
  a.n = n;
  int r = n;
  while (r % 4 == 0 && a.nf < kMaxFactors) { a.radix[a.nf++] = 4; r /= 4; }
  for (int p : {2, 3, 5, 7})
    while (r % p == 0 && a.nf < kMaxFactors) { a.radix[a.nf++] = p; r /= p; }
  for (int p = 11; r > 1 && a.nf < kMaxFactors; p += 2)
    while (r % p == 0 && a.nf < kMaxFactors) { a.radix[a.nf++] = p; r /= p; }
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

// sign * i * b
__device__ __forceinline__ double2 times_i(double2 b, int sign) {
  return make_double2(-sign * b.y, sign * b.x);
}

template <int R>
__device__ __forceinline__ void butterfly(double2 (&v)[R], double2 (&y)[R],
                                          const double2 *W, int n, int sign) {
  if constexpr (R == 3) {
    // y_q = sum_r v_r w^(r q), w = exp(sign 2 pi i / 3) = -1/2 + sign i sqrt(3)/2
    constexpr double kS3 = 0.86602540378443864676;  // sqrt(3) / 2
    const double2 t = make_double2(v[1].x + v[2].x, v[1].y + v[2].y);
    const double2 d = make_double2(kS3 * (v[1].x - v[2].x), kS3 * (v[1].y - v[2].y));
    const double2 a = make_double2(v[0].x - 0.5 * t.x, v[0].y - 0.5 * t.y);
    const double2 b = times_i(d, sign);
    y[0] = make_double2(v[0].x + t.x, v[0].y + t.y);
    y[1] = make_double2(a.x + b.x, a.y + b.y);
    y[2] = make_double2(a.x - b.x, a.y - b.y);
  } else if constexpr (R == 5) {
    // w^k = cos(2 pi k / 5) + sign i sin(2 pi k / 5); pairs k, 5 - k share the
    // cosine and differ in the sign of the sine
    constexpr double kC1 = 0.30901699437494742410;   // cos(2 pi / 5) = (sqrt 5 - 1) / 4
    constexpr double kC2 = -0.80901699437494742410;  // cos(4 pi / 5) = -(sqrt 5 + 1) / 4
    constexpr double kS1 = 0.95105651629515357212;   // sin(2 pi / 5)
    constexpr double kS2 = 0.58778525229247312917;   // sin(4 pi / 5)
    const double2 t1 = make_double2(v[1].x + v[4].x, v[1].y + v[4].y);
    const double2 t2 = make_double2(v[2].x + v[3].x, v[2].y + v[3].y);
    const double2 t3 = make_double2(v[1].x - v[4].x, v[1].y - v[4].y);
    const double2 t4 = make_double2(v[2].x - v[3].x, v[2].y - v[3].y);
    const double2 a1 = make_double2(v[0].x + kC1 * t1.x + kC2 * t2.x, v[0].y + kC1 * t1.y + kC2 * t2.y);
    const double2 a2 = make_double2(v[0].x + kC2 * t1.x + kC1 * t2.x, v[0].y + kC2 * t1.y + kC1 * t2.y);
    const double2 b1 = times_i(make_double2(kS1 * t3.x + kS2 * t4.x, kS1 * t3.y + kS2 * t4.y), sign);
    const double2 b2 = times_i(make_double2(kS2 * t3.x - kS1 * t4.x, kS2 * t3.y - kS1 * t4.y), sign);
    y[0] = make_double2(v[0].x + t1.x + t2.x, v[0].y + t1.y + t2.y);
    y[1] = make_double2(a1.x + b1.x, a1.y + b1.y);
    y[4] = make_double2(a1.x - b1.x, a1.y - b1.y);
    y[2] = make_double2(a2.x + b2.x, a2.y + b2.y);
    y[3] = make_double2(a2.x - b2.x, a2.y - b2.y);
  } else if constexpr (R == 2) {
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

// q = n / d and r = n % d for 0 <= n < 2^24 and d >= 1, from rd = the
// correctly rounded single-precision 1/d: the product n rd is within one of
// n / d, so one correction step either way makes it exact (checked for every
// d < 4097 and a sample up to 2^16 against integer division)
struct DivD {
  int d;
  float rd;
};
__device__ __forceinline__ DivD divisor(int d) { return DivD{d, __frcp_rn((float)d)}; }
__device__ __forceinline__ int divmod(int n, const DivD &D, int &r) {
  int q = __float2int_rz(__int2float_rn(n) * D.rd);
  r = n - q * D.d;
  if (r < 0) {
    --q;
    r += D.d;
  } else if (r >= D.d) {
    ++q;
    r -= D.d;
  }
  return q;
}

// One Stockham stage of radix R on nl lines held in shared memory; element e
// of line l sits at l * ls + e * es in src and dst. line_fast: consecutive
// threads take consecutive lines (lines adjacent in memory), else
// consecutive butterflies of one line.
template <int R>
__device__ void stage_r(int n, int Ns, int nl, int ls, int es, bool line_fast, int sign,
                        const double2 *W, const double2 *src, double2 *dst) {
  const int m = n / R, ts = n / (Ns * R);
  const DivD dl = divisor(line_fast ? nl : m), dn = divisor(Ns);
  for (int t = threadIdx.x; t < nl * m; t += blockDim.x) {
    int rem;
    const int quo = divmod(t, dl, rem);
    const int line = line_fast ? rem : quo;
    const int j = line_fast ? quo : rem;
    int k;
    const int jq = divmod(j, dn, k);
    const double2 *s = src + line * ls;
    double2 v[R], y[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const double2 a = s[(j + r * m) * es];
      // k r ts < Ns R ts = n: no wrap
      v[r] = r == 0 ? a : cmul(a, root(W, k * r * ts, sign));
    }
    butterfly<R>(v, y, W, n, sign);
    double2 *d = dst + line * ls;
    const int base = jq * Ns * R + k;
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
__device__ __forceinline__ void fft_plane_body(const BlockCtx &ctx, FftAxis ay, FftAxis az, int inverse, const T *__restrict__ rin, double2 *buf,
            T *__restrict__ rout, double scale) {
  extern __shared__ double2 smem[];
  const int M1 = ay.n, M2 = az.n, P = plane_pitch(M2);
  double2 *a = smem, *b = smem + M1 * P, *Wy = smem + 2 * M1 * P, *Wz = Wy + M1;
  root_table(M1, Wy);
  root_table(M2, Wz);
  const long base = (long)ctx.b.x * M1 * M2;
  const DivD d2 = divisor(M2);
#pragma unroll 4
  for (int t = threadIdx.x; t < M1 * M2; t += blockDim.x) {
    int z;
    const int y = divmod(t, d2, z);
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
    int z;
    const int y = divmod(t, d2, z);
    const double2 v = res[y * P + z];
    if (inverse)
      rout[base + t] = (T)(v.x * scale);
    else
      buf[base + t] = v;
  }
}
template <typename T>
struct KFftPlane {
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { fft_plane_body<T>(c, a...); }
};
template <typename T>
__global__ void __launch_bounds__(kPlaneThreads)
k_fft_plane(FftAxis ay, FftAxis az, int inverse, const T *__restrict__ rin, double2 *buf,
            T *__restrict__ rout, double scale) {
  fft_plane_body<T>(hw_ctx(), ay, az, inverse, rin, buf, rout, scale);
}

// Forward x, times w * khat, inverse x on kXLines adjacent x-lines
__device__ __forceinline__ void fft_xlines_body(const BlockCtx &ctx, FftAxis ax, int nlines, const double *__restrict__ khat, double w, double2 *buf) {
  extern __shared__ double2 smem[];
  const int n = ax.n, L = kXLines;
  double2 *a = smem, *b = smem + L * n, *W = smem + 2 * L * n;
  root_table(n, W);
  const int line0 = ctx.b.x * L;
#pragma unroll 4
  for (int t = threadIdx.x; t < L * n; t += blockDim.x) {
    const int l = t % L, e = t / L, g = line0 + l;
    a[e * L + l] = g < nlines ? buf[(long)e * nlines + g] : make_double2(0., 0.);
  }
  __syncthreads();
  double2 *res = axis_fft(ax, L, 1, L, true, -1, W, a, b);
#pragma unroll 4
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
struct KFftXlines {
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { fft_xlines_body(c, a...); }
};
__global__ void __launch_bounds__(kPlaneThreads)
k_fft_xlines(FftAxis ax, int nlines, const double *__restrict__ khat, double w, double2 *buf) {
  fft_xlines_body(hw_ctx(), ax, nlines, khat, w, buf);
}

// Larger grids: one launch per axis pass. A CTA transforms L lines of
// length n along one axis (element e of line g at base(g) + e * inner, with
// base(g) = (g / inner) n inner + g % inner). Lines g, g+1 are adjacent in
// memory when inner > 1, so threads take consecutive lines; rows (inner ==
// 1) are read along the row and transposed into shared memory through a
// pitch of L + 1. Modes: 0 forward, 1 real T in then forward, 2 forward,
// times w khat, inverse, 3 inverse then real T out (scaled), 4 inverse.
constexpr int kLineSmemMax = 200 * 1024;

struct LineShape {
  int L, LP;  // lines per CTA, shared-memory pitch between elements
};

// The most lines (<= 32) that keep three CTAs on an SM (<= 72 KB each),
// else the most that fit at all
LineShape line_shape(int n, int inner) {
  for (size_t cap : {(size_t)72 * 1024, (size_t)kLineSmemMax})
    for (int L = 32; L > 1; L >>= 1) {
      const int LP = inner == 1 ? L + 1 : L;
      if ((2 * (size_t)LP * n + n) * sizeof(double2) <= cap) return {L, LP};
    }
  return {1, 1};
}

size_t line_smem(int n, const LineShape &ls) {
  return (2 * (size_t)ls.LP * n + n) * sizeof(double2);
}

template <typename T>
__device__ __forceinline__ void fft_lines_body(const BlockCtx &ctx, FftAxis ax, int nlines, int inner, LineShape ls, int mode, const T *__restrict__ rin,
            double2 *buf, const double *__restrict__ khat, double w, T *__restrict__ rout,
            double scale) {
  extern __shared__ double2 smem[];
  const int n = ax.n, L = ls.L, LP = ls.LP;
  double2 *a = smem, *b = smem + LP * n, *W = smem + 2 * LP * n;
  root_table(n, W);
  const int line0 = ctx.b.x * L;
  const bool rows = inner == 1;
  auto gaddr = [&](int g, int e) -> long {
    return (long)(g / inner) * ((long)n * inner) + g % inner + (long)e * inner;
  };
  for (int t = threadIdx.x; t < L * n; t += blockDim.x) {
    const int l = rows ? t / n : t % L, e = rows ? t % n : t / L, g = line0 + l;
    double2 v = make_double2(0., 0.);
    if (g < nlines) {
      const long gi = gaddr(g, e);
      v = mode == 1 ? make_double2((double)rin[gi], 0.) : buf[gi];
    }
    a[e * LP + l] = v;
  }
  __syncthreads();
  double2 *res = axis_fft(ax, L, 1, LP, true, mode >= 3 ? +1 : -1, W, a, b);
  if (mode == 2) {
    for (int t = threadIdx.x; t < L * n; t += blockDim.x) {
      const int l = rows ? t / n : t % L, e = rows ? t % n : t / L, g = line0 + l;
      const double kv = g < nlines ? w * khat[gaddr(g, e)] : 0.;
      double2 &v = res[e * LP + l];
      v.x *= kv;
      v.y *= kv;
    }
    __syncthreads();
    double2 *o = res == a ? b : a;
    res = axis_fft(ax, L, 1, LP, true, +1, W, res, o);
  }
  for (int t = threadIdx.x; t < L * n; t += blockDim.x) {
    const int l = rows ? t / n : t % L, e = rows ? t % n : t / L, g = line0 + l;
    if (g >= nlines) continue;
    const long gi = gaddr(g, e);
    const double2 v = res[e * LP + l];
    if (mode == 3)
      rout[gi] = (T)(v.x * scale);
    else
      buf[gi] = v;
  }
}
template <typename T>
struct KFftLines {
  template <typename... A>
  static __device__ __forceinline__ void run(const BlockCtx &c, const A &...a) { fft_lines_body<T>(c, a...); }
};
template <typename T>
__global__ void __launch_bounds__(kPlaneThreads)
k_fft_lines(FftAxis ax, int nlines, int inner, LineShape ls, int mode, const T *__restrict__ rin,
            double2 *buf, const double *__restrict__ khat, double w, T *__restrict__ rout,
            double scale) {
  fft_lines_body<T>(hw_ctx(), ax, nlines, inner, ls, mode, rin, buf, khat, w, rout, scale);
}

template <typename T>
void line_pass(cudaStream_t s, int n, int nlines, int inner, int mode, const T *rin,
               double2 *buf, const double *khat, double w, T *rout, double scale) {
  const FftAxis ax = make_axis(n);
  const LineShape ls = line_shape(n, inner);
  const int blocks = (nlines + ls.L - 1) / ls.L;
  launch<KFftLines<T>, kPlaneThreads, 2>(s, k_fft_lines<T>, blocks, kPlaneThreads, line_smem(n, ls), ax, nlines, inner, ls, mode, rin,
                                                                buf, khat, w, rout, scale);
}

bool plane_path(const int M[3]) {
  return plane_smem(M) <= kPlaneSmemMax && xlines_smem(M[0]) <= kPlaneSmemMax;
}

}  // namespace

// One-time kernel attributes, per device (a line of up to 4096 points with
// its twiddle table needs 192 KB of shared memory). Called outside stream
// capture.
void top_solve_prepare() {
  static std::mutex mu;
  static bool done[kMaxDevices];
  const int dev = device_slot();
  std::lock_guard<std::mutex> lock(mu);
  if (dev >= 0 && done[dev]) return;
  cudaFuncSetAttribute(k_fft_lines<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       kLineSmemMax);
  cudaFuncSetAttribute(k_fft_lines<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       kLineSmemMax);
  cudaFuncSetAttribute(k_fft_plane<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)kPlaneSmemMax);
  cudaFuncSetAttribute(k_fft_plane<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)kPlaneSmemMax);
  cudaFuncSetAttribute(k_fft_xlines, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)kPlaneSmemMax);
  if (dev >= 0) done[dev] = true;
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
    launch<KFftPlane<T>, kPlaneThreads, 2>(s, k_fft_plane<T>, M0, kPlaneThreads, ps, ay, az, 0, q, buf0, nullptr, 0.);
    launch<KFftXlines, kPlaneThreads, 2>(s, k_fft_xlines, (nl + kXLines - 1) / kXLines, kPlaneThreads, xs, ax, nl, khat, weight,
                                                                         buf0);
    launch<KFftPlane<T>, kPlaneThreads, 2>(s, k_fft_plane<T>, M0, kPlaneThreads, ps, ay, az, 1, nullptr, buf0, e, scale);
    return;
  }
  line_pass<T>(s, M2, M0 * M1, 1, 1, q, buf0, nullptr, 0., nullptr, 0.);
  line_pass<T>(s, M1, M0 * M2, M2, 0, nullptr, buf0, nullptr, 0., nullptr, 0.);
  line_pass<T>(s, M0, M1 * M2, M1 * M2, 2, nullptr, buf0, khat, weight, nullptr, 0.);
  line_pass<T>(s, M1, M0 * M2, M2, 4, nullptr, buf0, nullptr, 0., nullptr, 0.);
  line_pass<T>(s, M2, M0 * M1, 1, 3, nullptr, buf0, nullptr, 0., e, scale);
}

template void launch_top_solve<float>(cudaStream_t, const int *, const float *,
                                      const double *, double, double2 *,
                                      double2 *, float *);
template void launch_top_solve<double>(cudaStream_t, const int *,
                                       const double *, const double *, double,
                                       double2 *, double2 *, double *);

}  // namespace msm
