// Instantiation of part 0 of the quartet-class kernel table (see
// dgf_jk_inst.cuh): the cooperative, warp-team and warp-per-quartet kernels,
// and the digestion kernel of stored integrals.
#pragma once

#include "dgf_jk_inst.cuh"
#include "dgf_jk_team.cuh"
#include "dgf_jk_warp.cuh"
#include "dgf_jk_stored.cuh"

namespace dgf {
namespace jkinst {

template <int LA, int LB, int LC, int LD, int WT>
void launch_team(const JKArgs &a, int grid, int block, size_t smem, cudaStream_t s) {
  jk_team_kernel<LA, LB, LC, LD, WT><<<grid, block, smem, s>>>(a);
}

// Classes with the warp-per-quartet kernel: L >= 4 whose per-warp shared
// memory fits one warp in 100 KB (every class up to (fd|fd), not (ff|..)
// pairs with L >= 11).  Below L = 6 it is a candidate of the autotuner next
// to the thread kernels.
template <int LA, int LB, int LC, int LD>
constexpr bool warp_eligible() {
  if constexpr (LA + LB + LC + LD < 4) {
    return false;
  } else {
    return wq::Shape<LA, LB, LC, LD, double>::smem(1) <= 100 * 1024;
  }
}

template <int LA, int LB, int LC, int LD, typename T, bool MMA>
void launch_warp(const JKArgs &a, int grid, int block, size_t smem, cudaStream_t s) {
  jk_warp_kernel<LA, LB, LC, LD, T, MMA><<<grid, block, smem, s>>>(a);
}

template <int LA, int LB, int LC, int LD, typename T, bool MMA = false>
ClassKernel warp_entry() {
  using W = wq::Shape<LA, LB, LC, LD, T>;
  return ClassKernel{&launch_warp<LA, LB, LC, LD, T, MMA>, 32 * W::WPB, W::smem(W::WPB), 1, W::WPB,
                     MMA ? kKindWarpMma : kKindWarp};
}

template <int LA, int LB, int LC, int LD, typename T, bool MMA = false>
cudaError_t prepare_warp() {
  using W = wq::Shape<LA, LB, LC, LD, T>;
  return cudaFuncSetAttribute(jk_warp_kernel<LA, LB, LC, LD, T, MMA>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)W::smem(W::WPB));
}

template <int LA, int LB, int LC, int LD>
void launch_stored_thread(const JKArgs &a, int grid, int block, size_t smem, cudaStream_t s) {
  jk_stored_thread_kernel<LA, LB, LC, LD><<<grid, block, smem, s>>>(a);
}
template <int LA, int LB, int LC, int LD>
void launch_stored_warp(const JKArgs &a, int grid, int block, size_t smem, cudaStream_t s) {
  jk_stored_warp_kernel<LA, LB, LC, LD><<<grid, block, smem, s>>>(a);
}
template <int LA, int LB, int LC, int LD>
constexpr bool stored_by_thread() {
  return ncart(LA) * ncart(LB) * ncart(LC) * ncart(LD) <= kStoredThreadMax;
}

template <int X, int Y>
cudaError_t prepare_team() {
  constexpr int LA = cls_la(X), LB = cls_lb(X), LC = cls_la(Y), LD = cls_lb(Y);
  using TS = TeamShape<LA, LB, LC, LD>;
  cudaError_t e = cudaFuncSetAttribute(jk_team_kernel<LA, LB, LC, LD, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)TS::smem());
  if constexpr (TS::kWarpTeams > 0)
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(jk_team_kernel<LA, LB, LC, LD, TS::kWarpTeams>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TS::smem_w(TS::kWarpTeams));
  if constexpr (warp_eligible<LA, LB, LC, LD>()) {
    if (e == cudaSuccess) e = prepare_warp<LA, LB, LC, LD, double>();
    if (e == cudaSuccess) e = prepare_warp<LA, LB, LC, LD, float>();
    if constexpr (wq::Shape<LA, LB, LC, LD, double>::MMA_OK)
      if (e == cudaSuccess) e = prepare_warp<LA, LB, LC, LD, double, true>();
  }
  if constexpr (!stored_by_thread<LA, LB, LC, LD>()) {
    using SS = StoredShape<LA, LB, LC, LD>;
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(jk_stored_warp_kernel<LA, LB, LC, LD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)SS::smem(SS::WPB));
  }
  return e;
}

template <int X, int Y>
void fill_team() {
  constexpr int LA = cls_la(X), LB = cls_lb(X), LC = cls_la(Y), LD = cls_lb(Y);
  using S = TeamShape<LA, LB, LC, LD>;
  JKEntry &e = g_jk_table[X][Y];
  e.prepare[0] = &prepare_team<X, Y>;
  constexpr int work = S::NAB * S::NCD;
  constexpr int block = work >= 512 ? 128 : work >= 64 ? 64 : 32;
  e.team = ClassKernel{&launch_team<LA, LB, LC, LD, 0>, block, S::smem(), 1, 1, kKindTeam};
  if constexpr (S::kWarpTeams > 0)
    e.wteam = ClassKernel{&launch_team<LA, LB, LC, LD, S::kWarpTeams>, 32 * S::kWarpTeams,
                          S::smem_w(S::kWarpTeams), 1, S::kWarpTeams, kKindWarpTeam};
  if constexpr (warp_eligible<LA, LB, LC, LD>()) {
    e.warp[0] = warp_entry<LA, LB, LC, LD, double>();
    e.warp[1] = warp_entry<LA, LB, LC, LD, float>();
    e.warp_mp = wq::Shape<LA, LB, LC, LD, double>::MP && wq::Shape<LA, LB, LC, LD, float>::MP;
    if constexpr (wq::Shape<LA, LB, LC, LD, double>::MMA_OK) e.warp_mma = warp_entry<LA, LB, LC, LD, double, true>();
  }
  if constexpr (stored_by_thread<LA, LB, LC, LD>()) {
    e.stored = ClassKernel{&launch_stored_thread<LA, LB, LC, LD>, kThreadBlock, 0, 1, kThreadBlock, kKindThread};
  } else {
    using SS = StoredShape<LA, LB, LC, LD>;
    e.stored = ClassKernel{&launch_stored_warp<LA, LB, LC, LD>, 32 * SS::WPB, SS::smem(SS::WPB), 1, SS::WPB, kKindWarp};
  }
}

}  // namespace jkinst
}  // namespace dgf

// Static initialiser filling part 0 of entry (X, Y).
#define DGF_JK_TEAM_CLASS(X, Y)                                                               \
  namespace dgf {                                                                             \
  namespace {                                                                                 \
  struct TeamInit_##X##_##Y {                                                                 \
    TeamInit_##X##_##Y() { jkinst::fill_team<X, Y>(); }                                       \
  } g_team_init_##X##_##Y;                                                                    \
  }                                                                                           \
  }
