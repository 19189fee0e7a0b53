// Kernel launches that can be merged across independent systems.
//
// A kernel whose launches may be merged is written as a body struct K with
//   static __device__ void run(const BlockCtx &c, A... args)
// that reads its block index and grid size from c instead of blockIdx and
// gridDim, plus a plain __global__ wrapper (the kernel name profiles show)
// that calls K::run(hw_ctx(), args...). Launchers go through launch<K, ...>:
// normally a plain launch of the wrapper; while a Recorder is installed on
// the calling host thread, the launch (its kernel, grid, block, dynamic
// shared memory and arguments by value) is appended to the recorder instead.
//
// A batch records every member's evaluation, then replaces the k-th launches
// of the same body (same block shape) across members by ONE launch of
// k_multi<K, ...> whose kernel parameter is a table of the members' arguments
// and block ranges: block b of the merged grid belongs to the member whose
// block range holds it, and runs K::run with that member's arguments and its
// own block index and grid size, so each member computes exactly what its own
// launch computes.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstring>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

#include "launch_rec.h"

namespace msm {

struct BlockCtx {
  uint3 b;  // block index
  uint3 g;  // grid size
};

__device__ __forceinline__ BlockCtx hw_ctx() {
  return BlockCtx{blockIdx, make_uint3(gridDim.x, gridDim.y, gridDim.z)};
}

// Arguments of one launch, by value, in declaration order
template <typename... A>
struct Pack {};
template <typename H, typename... R>
struct Pack<H, R...> {
  H h;
  Pack<R...> r;
};

template <typename... A>
inline void fill_pack(Pack<A...> &, A...) {}
template <typename H, typename... R>
inline void fill_pack(Pack<H, R...> &p, H h, R... r) {
  p.h = h;
  fill_pack<R...>(p.r, r...);
}

template <class K, typename... Done>
__device__ __forceinline__ void invoke(const BlockCtx &c, const Pack<> &, const Done &...d) {
  K::run(c, d...);
}
template <class K, typename H, typename... R, typename... Done>
__device__ __forceinline__ void invoke(const BlockCtx &c, const Pack<H, R...> &p,
                                       const Done &...d) {
  invoke<K>(c, p.r, d..., p.h);
}

// Table of one merged launch, passed BY VALUE as the kernel's parameter (the
// constant bank, as the plain launch's arguments): member m owns merged
// blocks [first[m], first[m + 1]), its grid has grid[m] blocks (x fastest)
// and its arguments are packs[m]. U: the uniform argument of bodies that
// declare kUniformArg (otherwise unused). A merged launch holds at most
// NMAX members; larger groups are split over several launches.
constexpr size_t kParamBudget = 32000;  // kernel parameters: at most 32,764 bytes
template <typename P, typename U>
constexpr int tab_members() {
  return (int)((kParamBudget - sizeof(U) - 64) / (sizeof(P) + sizeof(int) + sizeof(uint3)));
}
template <typename P, typename U, int NMAX>
struct ParamTab {
  U u;
  int n;
  int first[NMAX + 1];
  uint3 grid[NMAX];
  P packs[NMAX];
};
struct NoUniform {};

// Bodies with an argument that is a table of constants shared by many
// members (the pair kernels' PairConsts, the B-spline pieces of a given
// order) declare `static constexpr int kUniformArg = <its index>`: their
// merged launches group members whose argument has the same bytes and pass
// it once (ParamTab::u, read at fixed offsets like a plain kernel argument)
// instead of once per member.
template <class K, typename = void>
struct uniform_arg : std::integral_constant<int, -1> {};
template <class K>
struct uniform_arg<K, std::void_t<decltype(K::kUniformArg)>>
    : std::integral_constant<int, K::kUniformArg> {};

template <class K, typename... A>
struct MultiTypes {
  static constexpr int kUI = uniform_arg<K>::value;
  static constexpr bool kU = kUI >= 0;
  using U = typename std::conditional_t<kU, std::tuple_element<(kU ? kUI : 0), std::tuple<A...>>,
                                        std::common_type<NoUniform>>::type;
  using P = Pack<A...>;
  static constexpr int kN = tab_members<P, U>();
  using Tab = ParamTab<P, U, kN>;
  static_assert(kN >= 1 && sizeof(Tab) <= kParamBudget, "merged launch table too large");
};

// K::run with the pack's arguments, argument UI replaced by u
template <class K, int UI, int I, typename U, typename... Done>
__device__ __forceinline__ void invoke_u(const BlockCtx &c, const U &, const Pack<> &,
                                         const Done &...d) {
  K::run(c, d...);
}
template <class K, int UI, int I, typename U, typename H, typename... R, typename... Done>
__device__ __forceinline__ void invoke_u(const BlockCtx &c, const U &u, const Pack<H, R...> &p,
                                         const Done &...d) {
  if constexpr (I == UI)
    invoke_u<K, UI, I + 1, U>(c, u, p.r, d..., u);
  else
    invoke_u<K, UI, I + 1, U>(c, u, p.r, d..., p.h);
}

template <class K, int MAXT, int MINB, typename... A>
__global__ void __launch_bounds__(MAXT, MINB)
k_multi(const __grid_constant__ typename MultiTypes<K, A...>::Tab t) {
  const int bid = (int)blockIdx.x;
  int lo = 0, hi = t.n;  // last member with first[m] <= bid
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (t.first[mid] <= bid) lo = mid; else hi = mid;
  }
  const uint3 g = t.grid[lo];
  const int local = bid - t.first[lo];
  BlockCtx c;
  c.g = g;
  c.b.x = local % g.x;
  c.b.y = (local / g.x) % g.y;
  c.b.z = local / (g.x * g.y);
  using MT = MultiTypes<K, A...>;
  if constexpr (MT::kU)
    invoke_u<K, MT::kUI, 0, typename MT::U>(c, t.u, t.packs[lo]);
  else
    invoke<K>(c, t.packs[lo]);
}

// Launch of body K through its plain wrapper k1, or a record of it.
template <class K, int MAXT, int MINB, typename... A, typename... B>
inline void launch(cudaStream_t s, void (*k1)(A...), dim3 g, dim3 b, size_t smem, B &&...args) {
  static_assert(sizeof...(A) == sizeof...(B), "argument count");
  if (Recorder *r = tls_recorder()) {
    LaunchRec rec;
    rec.kind = LaunchRec::kKernel;
    using MT = MultiTypes<K, A...>;
    using Tab = typename MT::Tab;
    rec.kmulti = reinterpret_cast<const void *>(&k_multi<K, MAXT, MINB, A...>);
    rec.tab_bytes = sizeof(Tab);
    rec.tab_max = MT::kN;
    rec.off_n = offsetof(Tab, n);
    rec.off_first = offsetof(Tab, first);
    rec.off_grid = offsetof(Tab, grid);
    rec.off_packs = offsetof(Tab, packs);
    rec.pack_stride = sizeof(typename MT::P);
    if constexpr (MT::kU) {
      using U = typename MT::U;
      const U u = static_cast<U>(std::get<MT::kUI>(std::forward_as_tuple(args...)));
      rec.uniform.resize(sizeof(U));
      std::memcpy(rec.uniform.data(), &u, sizeof(U));
      rec.off_u = offsetof(Tab, u);
    }
    rec.grid = make_uint3(g.x, g.y, g.z);
    rec.block = b;
    rec.smem = smem;
    Pack<A...> p{};
    fill_pack<A...>(p, static_cast<A>(args)...);
    static_assert(std::is_trivially_copyable<Pack<A...>>::value, "pack must be plain data");
    rec.pack.resize(sizeof(p));
    std::memcpy(rec.pack.data(), &p, sizeof(p));
    rec.branch = rec_branch(r, s);
    r->recs.push_back(std::move(rec));
    return;
  }
  k1<<<g, b, smem, s>>>(static_cast<A>(args)...);
}

}  // namespace msm
