// Tile autotuner for the level stencils.
//
// For a level with enough work (>= 1 GFLOP per launch) the plan times a set
// of candidate tiles (CTA thread shape and tap-plane split) on the level's
// own buffers and keeps the fastest; smaller levels use the model-based
// default (stencil_default_tile). Results are cached in a text file, one
// line per (format, device, precision, grid, stencil):
//   <format>|<device name>|<fp32|fp64>|M0,M1,M2|S0,S1,S2|<folded|full> nz ty nsplit r ms
// at $MSMPB_TUNE_CACHE, else $HOME/.cache/msmpb_b200/stencil_tiles.txt. A
// cached tile is used only after the same checks as a freshly timed one
// (shape limits, buffer capacities, stencil_prepare); a line that fails them
// (another library version, a hand-edited file) is ignored and the level is
// tuned again. MSMPB_TUNE=0 disables tuning (default tiles only).
#include <sys/stat.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "kernels.h"

namespace msm {
namespace {

std::mutex g_cache_mu;

// Bumped whenever the candidate set or the meaning of a tile changes, so
// that lines written by another version never match.
constexpr const char *kCacheFormat = "st3";

std::string cache_path() {
  const char *p = std::getenv("MSMPB_TUNE_CACHE");
  if (p && *p) return p;
  const char *home = std::getenv("HOME");
  if (!home) return "";
  std::string dir = std::string(home) + "/.cache";
  mkdir(dir.c_str(), 0755);
  dir += "/msmpb_b200";
  mkdir(dir.c_str(), 0755);
  return dir + "/stencil_tiles.txt";
}

std::string cache_key(const StencilShape &sh, bool fp64, int device) {
  cudaDeviceProp prop{};
  cudaGetDeviceProperties(&prop, device);
  char buf[512];
  std::snprintf(buf, sizeof buf, "%s|%s|%s|%d,%d,%d|%d,%d,%d|%s", kCacheFormat,
                prop.name, fp64 ? "fp64" : "fp32", sh.M[0], sh.M[1], sh.M[2], sh.S[0],
                sh.S[1], sh.S[2], sh.sym ? "folded" : "full");
  for (char *c = buf; *c; ++c)
    if (*c == ' ') *c = '_';
  return buf;
}

bool cache_lookup(const std::string &key, StencilTile &t) {
  std::lock_guard<std::mutex> lock(g_cache_mu);
  const std::string path = cache_path();
  if (path.empty()) return false;
  FILE *f = std::fopen(path.c_str(), "r");
  if (!f) return false;
  char line[1024];
  bool found = false;
  while (std::fgets(line, sizeof line, f)) {
    char k[600];
    int nz, ty, ns, r;
    double ms;
    if (std::sscanf(line, "%599s %d %d %d %d %lf", k, &nz, &ty, &ns, &r, &ms) == 6 &&
        key == k) {
      t.nz = nz;
      t.ty = ty;
      t.nsplit = ns;
      t.r = r;
      found = true;  // the last entry wins
    }
  }
  std::fclose(f);
  return found;
}

void cache_store(const std::string &key, const StencilTile &t, double ms) {
  std::lock_guard<std::mutex> lock(g_cache_mu);
  const std::string path = cache_path();
  if (path.empty()) return;
  FILE *f = std::fopen(path.c_str(), "a");
  if (!f) return;
  std::fprintf(f, "%s %d %d %d %d %.5f\n", key.c_str(), t.nz, t.ty, t.nsplit, t.r, ms);
  std::fclose(f);
}

}  // namespace

bool stencil_tuning_enabled() {
  const char *v = std::getenv("MSMPB_TUNE");
  return !(v && v[0] == '0');
}

std::vector<StencilTile> stencil_candidates(const StencilShape &sh, bool fp64) {
  std::vector<StencilTile> out;
  const StencilTile d = stencil_default_tile(sh, fp64);
  out.push_back(d);
  // the precision's default z outputs per thread, and for folded sweeps of
  // wide stencils the alternative
  const int alt = stencil_alt_r(sh, fp64);
  for (int r : {0, alt}) {
    const int R = r ? r : stencil_tile_r(d, fp64);
    for (int nz : {d.nz, 2, 3, 4, 6, 8, 9, 12})
      for (int ty : {4, 8, 12, 16, 24, 32, 36, 48})
        for (int ns : {1, 2, d.nsplit, 2 * d.nsplit}) {
          StencilTile t = d;
          t.nz = nz;
          t.ty = ty;
          t.r = r;
          if (nz * ty > 256 || nz * ty < 32 || ty > sh.M[1]) continue;
          if (nz * R > sh.M[2] + R - 1 && nz > 1) continue;
          const int nI = sh.sym ? sh.S[0] / 2 + 1 : sh.S[0];
          const int chunk = (nI + std::max(1, ns) - 1) / std::max(1, ns);
          t.nsplit = (nI + chunk - 1) / chunk;
          bool dup = false;
          for (auto &u : out)
            dup |= (u.nz == t.nz && u.ty == t.ty && u.nsplit == t.nsplit && u.r == t.r);
          if (!dup) out.push_back(t);
        }
    if (!alt) break;
  }
  return out;
}

// Whether a tile can run on a level: its shape within the kernels' limits,
// its padded grid and split-K partial sums within the buffers the plan
// allocated, and its kernel's shared memory granted (stencil_prepare). Both
// cached and freshly timed tiles pass through here.
template <typename T>
bool tile_usable(const StencilShape &sh0, const StencilTile &t, size_t padded_cap,
                 size_t part_cap) {
  if (t.nz <= 0 || t.ty <= 0 || t.nz * t.ty > 256 || t.nsplit < 1 || t.tx <= 0) return false;
  const int nI = sh0.sym ? sh0.S[0] / 2 + 1 : sh0.S[0];
  if (t.nsplit > nI) return false;
  StencilShape sh = sh0;
  stencil_padded_dims(sh, t, sizeof(T) == 8, sh.P);
  if (sh.P[0] <= 0 || sh.P[1] <= 0 || sh.P[2] <= 0) return false;
  if ((size_t)sh.P[0] * sh.P[1] * sh.P[2] > padded_cap) return false;
  const size_t mtot = (size_t)sh0.M[0] * sh0.M[1] * sh0.M[2];
  if (t.nsplit > 1 && (size_t)t.nsplit * mtot > part_cap) return false;
  return stencil_prepare<T>(sh, t) >= 0;
}

template <typename T>
StencilTile stencil_autotune(cudaStream_t s, int device, const StencilShape &sh0,
                             const StencilTile &fallback, const T *padded,
                             size_t padded_cap, const T *kh, int khz, T *e,
                             T *part, size_t part_cap, double *best_ms) {
  const bool fp64 = sizeof(T) == 8;
  const std::string key = cache_key(sh0, fp64, device);
  StencilTile cached;
  if (cache_lookup(key, cached)) {
    cached.tx = fallback.tx;
    if (tile_usable<T>(sh0, cached, padded_cap, part_cap)) {
      if (best_ms) *best_ms = -1.0;
      return cached;
    }
  }
  StencilTile best = fallback;
  double best_t = 1e30;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (StencilTile t : stencil_candidates(sh0, fp64)) {
    t.tx = fallback.tx;
    if (!tile_usable<T>(sh0, t, padded_cap, part_cap)) continue;
    StencilShape sh = sh0;
    stencil_padded_dims(sh, t, fp64, sh.P);
    float ms[3];
    bool ok = true;
    launch_stencil<T>(s, sh, t, padded, kh, khz, T(0), e, part);  // warm-up
    for (int r = 0; r < 3 && ok; ++r) {
      cudaEventRecord(e0, s);
      launch_stencil<T>(s, sh, t, padded, kh, khz, T(0), e, part);
      cudaEventRecord(e1, s);
      ok = cudaEventSynchronize(e1) == cudaSuccess &&
           cudaEventElapsedTime(&ms[r], e0, e1) == cudaSuccess;
    }
    if (!ok || cudaGetLastError() != cudaSuccess) continue;
    std::sort(ms, ms + 3);
    if (ms[1] < best_t) {
      best_t = ms[1];
      best = t;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (best_t < 1e30) cache_store(key, best, best_t);
  if (best_ms) *best_ms = best_t;
  return best;
}

template StencilTile stencil_autotune<float>(cudaStream_t, int, const StencilShape &,
                                             const StencilTile &, const float *, size_t,
                                             const float *, int, float *, float *,
                                             size_t, double *);
template StencilTile stencil_autotune<double>(cudaStream_t, int, const StencilShape &,
                                              const StencilTile &, const double *, size_t,
                                              const double *, int, double *, double *,
                                              size_t, double *);

}  // namespace msm
