// Level stencil that allocates no memory: msmpb_level_stencil_noalloc.
//
// Some callers cannot let a library allocate device memory: MD engines and
// frameworks that own every byte through their own pool allocator (a
// cudaMalloc behind the pool's back escapes its budget, and cudaMalloc /
// cudaFree may synchronise the whole device in the middle of their step).
// This entry point runs the same padded copy and tiled stencil kernels as the
// level stencils of FF_energy_device, with their scratch (tap copy, padded
// charge grid, tap-plane partial sums) in one fixed array compiled into the
// library instead of buffers allocated by FF_build.
//
// Set-up: the first call on a device (the device current at that call) looks
// up the array's device address with cudaGetSymbolAddress, which can load
// this library's GPU code onto the device; make that first call before any
// stream capture. The first call for each stencil width S[2] on a device also
// raises that kernel's shared-memory limit there (cudaFuncSetAttribute). The
// address is kept for the life of the process: do not reset the device
// (cudaDeviceReset, or a reset of its primary context) between calls, since
// later calls would write through the stale address.
//
// Sharing: every call on a device uses the same array, which keeps the last
// call's contents. Nothing in it has to start at zero: each call clears the
// tap copy and then overwrites it, and overwrites every element of the padded
// grid and of the partial sums it reads. Calls whose GPU work overlaps (other
// streams, other host threads without ordering) race on the array; order
// them on one stream or with events.
#include <mutex>

#include "kernels.h"
#include "msmpb_b200.h"

// The scratch array (one copy per device, in the library's device image)
static __device__ __align__(256) double
    g_noalloc_scratch[MSMPB_NOALLOC_SCRATCH_BYTES / sizeof(double)];

namespace {

constexpr int kMaxDevices = 64;
constexpr size_t kWords = MSMPB_NOALLOC_SCRATCH_BYTES / sizeof(double);
constexpr size_t kAlignWords = 256 / sizeof(double);

std::mutex g_mu;
double *g_scratch[kMaxDevices] = {};

size_t align_words(size_t n) { return (n + kAlignWords - 1) / kAlignWords * kAlignWords; }

// Device address of the scratch array on the current device (looked up once
// per device).
int scratch_address(double **out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return MSMPB_ERR_NODEVICE;
  if (dev < 0 || dev >= kMaxDevices) return MSMPB_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch[dev]) {
    double *p = nullptr;
    if (cudaGetSymbolAddress((void **)&p, g_noalloc_scratch) != cudaSuccess || !p)
      return MSMPB_ERR_CUDA;
    g_scratch[dev] = p;
  }
  *out = g_scratch[dev];
  return MSMPB_OK;
}

}  // namespace

extern "C" int msmpb_level_stencil_noalloc(const int M[3], const int S[3],
                                           const double *charge_grid_d,
                                           const double *stencil_d, double weight,
                                           double *potential_grid_d, void *stream) {
  if (!M || !S || !charge_grid_d || !stencil_d || !potential_grid_d)
    return MSMPB_ERR_ARGUMENT;
  msm::StencilShape sh{};
  for (int a = 0; a < 3; ++a) {
    if (M[a] < 1 || S[a] < 1 || S[a] > M[a]) return MSMPB_ERR_ARGUMENT;
    sh.M[a] = M[a];
    sh.S[a] = S[a];
  }
  (void)cudaGetLastError();  // report only this call's launch errors
  double *scratch = nullptr;
  if (int st = scratch_address(&scratch)) return st;

  // Tiled kernel where the width is templated and its shared-memory request
  // fits, else the one-output-per-thread kernel (nz = 0).
  msm::StencilTile tile;
  bool tiled = msm::stencil_templated(sh);
  if (tiled) {
    tile = msm::stencil_default_tile(sh, true);
    tiled = msm::stencil_prepare<double>(sh, tile) == 0;
  }
  if (tiled) {
    msm::stencil_padded_dims(sh, tile, true, sh.P);
  } else {
    tile = msm::StencilTile{};
    for (int a = 0; a < 3; ++a) sh.P[a] = sh.M[a] + sh.S[a] - 1;
  }
  const int pitch = tiled ? msm::stencil_tap_pitch(S[2], true) : S[2];
  const size_t tap_words = align_words((size_t)S[0] * S[1] * pitch);
  const size_t pad_words = align_words((size_t)sh.P[0] * sh.P[1] * sh.P[2]);
  if (tap_words > kWords || pad_words > kWords - tap_words) return MSMPB_ERR_UNSUPPORTED;

  // The partial sums of the tap-plane split take what is left; fewer chunks
  // when it is short (one chunk needs none).
  const size_t mtot = (size_t)M[0] * M[1] * M[2];
  if (tiled && tile.nsplit > 1) {
    const size_t fit = (kWords - tap_words - pad_words) / mtot;
    if (fit < 2) {
      tile.nsplit = 1;
    } else if ((size_t)tile.nsplit > fit) {
      const int chunk = (S[0] + (int)fit - 1) / (int)fit;
      tile.nsplit = (S[0] + chunk - 1) / chunk;
    }
  }
  double *taps = scratch;
  double *padded = scratch + tap_words;
  double *part = padded + pad_words;

  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(taps, 0, tap_words * sizeof(double), s) != cudaSuccess ||
      cudaMemcpy2DAsync(taps, pitch * sizeof(double), stencil_d, S[2] * sizeof(double),
                        S[2] * sizeof(double), (size_t)S[0] * S[1],
                        cudaMemcpyDeviceToDevice, s) != cudaSuccess)
    return MSMPB_ERR_CUDA;
  msm::launch_pad<double>(s, sh, charge_grid_d, padded);
  msm::launch_stencil<double>(s, sh, tile, padded, taps, pitch, weight,
                              potential_grid_d, part);
  return cudaGetLastError() == cudaSuccess ? MSMPB_OK : MSMPB_ERR_CUDA;
}
