// Device-side building blocks shared by the MSM kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace msm {

// 4-wide record (x, y, z, w) in the evaluation precision T.
template <typename T>
struct alignas(4 * sizeof(T)) V4 {
  T x, y, z, w;
};

// Periodic index reduction into [0, n)
__host__ __device__ __forceinline__ int pwrap(int i, int n) {
  int r = i % n;
  return r < 0 ? r + n : r;
}

// Compensated (Kahan/TwoSum-style) accumulator. With T = double the
// compensation is skipped: FP64 sums are the plain-FP64 reference form.
template <typename T>
struct Acc {
  T s, c;
  __device__ __forceinline__ void zero() { s = T(0); c = T(0); }
  __device__ __forceinline__ void add(T v) {
    T y = v - c;
    T t = s + y;
    c = (t - s) - y;
    s = t;
  }
  __device__ __forceinline__ T value() const { return s; }
};
template <>
struct Acc<double> {
  double s;
  __device__ __forceinline__ void zero() { s = 0.; }
  __device__ __forceinline__ void add(double v) { s += v; }
  __device__ __forceinline__ double value() const { return s; }
};

template <typename T> __device__ __forceinline__ T rsqrt_t(T x);
template <> __device__ __forceinline__ float rsqrt_t<float>(float x) { return rsqrtf(x); }
template <> __device__ __forceinline__ double rsqrt_t<double>(double x) { return rsqrt(x); }

// cudaFuncSetAttribute acts on the device current at the call, so one-time
// kernel set-ups are tracked per device ordinal (ordinals beyond the table
// are set up on every call).
constexpr int kMaxDevices = 64;
inline int device_slot() {
  int d = -1;
  return (cudaGetDevice(&d) == cudaSuccess && d >= 0 && d < kMaxDevices) ? d : -1;
}

// Device error flag bits (read back by the host after each evaluation)
enum DeviceCheck : int {
  kCheckOk = 0,
  kCheckIndex = 1,      // a computed index fell outside its buffer
  kCheckOverflow = 2,   // a per-tile capacity was exceeded
  kCheckNonFinite = 4,  // non-finite position or charge
};

__device__ __forceinline__ void flag_error(int *flag, int bit) {
  if (flag) atomicOr(flag, bit);
}

}  // namespace msm
