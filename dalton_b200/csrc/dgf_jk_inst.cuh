// Instantiation helpers of the quartet-class kernel table: one translation
// unit per class pair (generated by the build, see DGF_JK_CLASS) fills its
// entry, so the classes compile in parallel.
#pragma once

#include <type_traits>
#include <utility>

#include "dgf_jk_thread.cuh"
#include "dgf_jk_warp.cuh"

namespace dgf {

struct JKEntry {
  ClassKernel team;
  ClassKernel wteam;                     // one quartet per warp (light quartets), when it fits
  ClassKernel thr[2][kThreadVariants];   // [precision 0 = FP64, 1 = FP32][variant]
  ClassKernel thr1[2][kThreadVariants];  // same, for kets of one primitive pair each
  ClassKernel warp[2];                   // warp-per-quartet kernel [FP64, FP32] (single primitive pairs)
  cudaError_t (*prepare[3])();           // one per generated part (see DGF_JK_CLASS)
};

extern JKEntry g_jk_table[kNumPairClass][kNumPairClass];

namespace jkinst {

constexpr int cls_la(int X) { return X == 0 ? 0 : X <= 2 ? 1 : X <= 5 ? 2 : 3; }
constexpr int cls_lb(int X) { return X - cls_la(X) * (cls_la(X) + 1) / 2; }

constexpr bool thread_eligible(int LA, int LB, int LC, int LD) {
  const int L = LA + LB + LC + LD;
  if (LA == 3) return LB == 0 && LC == 0 && LD == 0;  // (fs|ss)
  return L <= 5;
}

// Classes with f shells up to L = 5 get the thread kernel in its
// single-ket-primitive form only (every pair of a Dunning basis in the
// working basis has one primitive pair), first chunk variant; their other
// plan entries keep the team kernel.
constexpr bool k1_only_eligible(int LA, int LB, int LC, int LD) {
  return !thread_eligible(LA, LB, LC, LD) && LA + LB + LC + LD <= 5;
}

constexpr int cdiv(int a, int b) { return (a + b - 1) / b; }
constexpr int cmin(int a, int b) { return a < b ? a : b; }
// A-chunk count keeping at most `target` accumulators per thread.
constexpr int chunks_for(int LA, int LB, int LC, int LD, int target) {
  return cmin(ncart(LA), cdiv(ncart(LA) * ncart(LB) * ncart(LC) * ncart(LD), target));
}

template <int LA, int LB, int LC, int LD, int WT>
void launch_team(const JKArgs &a, int grid, int block, size_t smem, cudaStream_t s) {
  jk_team_kernel<LA, LB, LC, LD, WT><<<grid, block, smem, s>>>(a);
}

template <int LA, int LB, int LC, int LD, typename T, int CA, int K1>
void launch_thread(const JKArgs &a, int grid, int block, size_t smem, cudaStream_t s) {
  jk_thread_kernel<LA, LB, LC, LD, T, CA, K1><<<dim3(grid, CA), block, smem, s>>>(a);
}

// Classes with the warp-per-quartet kernel: L >= 6 with at most 36 Cartesian
// components on each side (pairs up to (dd) and (fp)).
constexpr bool warp_eligible(int LA, int LB, int LC, int LD) {
  return LA + LB + LC + LD >= 6 && ncart(LA) * ncart(LB) <= 36 && ncart(LC) * ncart(LD) <= 36;
}

template <int LA, int LB, int LC, int LD, typename T>
void launch_warp(const JKArgs &a, int grid, int block, size_t smem, cudaStream_t s) {
  jk_warp_kernel<LA, LB, LC, LD, T><<<grid, block, smem, s>>>(a);
}

template <int LA, int LB, int LC, int LD, typename T>
ClassKernel warp_entry() {
  using W = wq::Shape<LA, LB, LC, LD, T>;
  return ClassKernel{&launch_warp<LA, LB, LC, LD, T>, 32 * W::WPB, W::smem(W::WPB), 1, W::WPB, kKindWarp, nullptr};
}

template <int LA, int LB, int LC, int LD, typename T>
cudaError_t prepare_warp() {
  using W = wq::Shape<LA, LB, LC, LD, T>;
  return cudaFuncSetAttribute(jk_warp_kernel<LA, LB, LC, LD, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)W::smem(W::WPB));
}

template <int LA, int LB, int LC, int LD, typename T, int CA, int K1>
int occ_thread(size_t smem) {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, jk_thread_kernel<LA, LB, LC, LD, T, CA, K1>, kThreadBlock,
                                                    smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

// Thread-kernel chunk counts of a class: FP64 / FP32, first and second variant.
template <int LA, int LB, int LC, int LD>
struct ThreadCfg {
  static constexpr int c64 = chunks_for(LA, LB, LC, LD, 27), c64b = cmin(ncart(LA), 2 * c64);
  static constexpr int c32 = chunks_for(LA, LB, LC, LD, 54), c32b = cmin(ncart(LA), 2 * c32);
};

// The thread kernels keep ~10 KB of shared memory per block (Boys and
// spherical tables, bra Hermite tables): ask for a small shared-memory
// carveout so that the rest of the unified L1 caches the density rows and
// pair records their quartets gather.
constexpr int kThreadCarveoutPercent = 25;

template <int LA, int LB, int LC, int LD, typename T, int CA, int K1>
cudaError_t carve_one() {
  cudaError_t e = cudaFuncSetAttribute(jk_thread_kernel<LA, LB, LC, LD, T, CA, K1>,
                                       cudaFuncAttributePreferredSharedMemoryCarveout, kThreadCarveoutPercent);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(jk_thread_kernel<LA, LB, LC, LD, T, CA, K1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kTileMaxBytes);
  return e;
}

template <int LA, int LB, int LC, int LD, typename T, int CA>
cudaError_t carve_thread() {
  cudaError_t e = carve_one<LA, LB, LC, LD, T, CA, 0>();
  if (e == cudaSuccess) e = carve_one<LA, LB, LC, LD, T, CA, 1>();
  return e;
}

// The entry of class pair (X, Y) is filled by three generated translation
// units (parts), so that the heaviest classes compile in parallel: part 0
// the cooperative, warp-team and warp-per-quartet kernels, part 1 the FP64
// thread kernels, part 2 the FP32 thread kernels.  Each part sets only its
// own fields of the (zero-initialised) table entry and its own prepare hook.
template <int LA, int LB, int LC, int LD, int P>
cudaError_t prepare_part() {
  using TS = TeamShape<LA, LB, LC, LD>;
  cudaError_t e = cudaSuccess;
  if constexpr (P == 0) {
    e = cudaFuncSetAttribute(jk_team_kernel<LA, LB, LC, LD, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)TS::smem());
    if constexpr (TS::kWarpTeams > 0)
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(jk_team_kernel<LA, LB, LC, LD, TS::kWarpTeams>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TS::smem_w(TS::kWarpTeams));
    if constexpr (warp_eligible(LA, LB, LC, LD)) {
      if (e == cudaSuccess) e = prepare_warp<LA, LB, LC, LD, double>();
      if (e == cudaSuccess) e = prepare_warp<LA, LB, LC, LD, float>();
    }
  } else {
    using T = std::conditional_t<P == 1, double, float>;
    using C = ThreadCfg<LA, LB, LC, LD>;
    constexpr int ca = P == 1 ? C::c64 : C::c32, cb = P == 1 ? C::c64b : C::c32b;
    if constexpr (thread_eligible(LA, LB, LC, LD)) {
      e = carve_thread<LA, LB, LC, LD, T, ca>();
      if constexpr (cb != ca)
        if (e == cudaSuccess) e = carve_thread<LA, LB, LC, LD, T, cb>();
    } else if constexpr (k1_only_eligible(LA, LB, LC, LD)) {
      e = carve_one<LA, LB, LC, LD, T, ca, 1>();
    }
  }
  return e;
}

template <int LA, int LB, int LC, int LD, typename T, int CA, int K1 = 0>
ClassKernel thread_entry() {
  return ClassKernel{&launch_thread<LA, LB, LC, LD, T, CA, K1>, kThreadBlock, 0, CA, kThreadBlock, kKindThread,
                     &occ_thread<LA, LB, LC, LD, T, CA, K1>};
}

template <int X, int Y, int P>
void fill_part() {
  constexpr int LA = cls_la(X), LB = cls_lb(X), LC = cls_la(Y), LD = cls_lb(Y);
  using S = TeamShape<LA, LB, LC, LD>;
  JKEntry &e = g_jk_table[X][Y];
  e.prepare[P] = &prepare_part<LA, LB, LC, LD, P>;
  if constexpr (P == 0) {
    constexpr int work = S::NAB * S::NCD;
    constexpr int block = work >= 512 ? 128 : work >= 64 ? 64 : 32;
    e.team = ClassKernel{&launch_team<LA, LB, LC, LD, 0>, block, S::smem(), 1, 1, kKindTeam, nullptr};
    if constexpr (S::kWarpTeams > 0)
      e.wteam = ClassKernel{&launch_team<LA, LB, LC, LD, S::kWarpTeams>, 32 * S::kWarpTeams,
                            S::smem_w(S::kWarpTeams), 1, S::kWarpTeams, kKindWarpTeam, nullptr};
    if constexpr (warp_eligible(LA, LB, LC, LD)) {
      e.warp[0] = warp_entry<LA, LB, LC, LD, double>();
      e.warp[1] = warp_entry<LA, LB, LC, LD, float>();
    }
  } else {
    using T = std::conditional_t<P == 1, double, float>;
    constexpr int p = P - 1;
    using C = ThreadCfg<LA, LB, LC, LD>;
    constexpr int ca = P == 1 ? C::c64 : C::c32, cb = P == 1 ? C::c64b : C::c32b;
    if constexpr (thread_eligible(LA, LB, LC, LD)) {
      e.thr[p][0] = thread_entry<LA, LB, LC, LD, T, ca>();
      if constexpr (cb != ca) e.thr[p][1] = thread_entry<LA, LB, LC, LD, T, cb>();
      e.thr1[p][0] = thread_entry<LA, LB, LC, LD, T, ca, 1>();
      if constexpr (cb != ca) e.thr1[p][1] = thread_entry<LA, LB, LC, LD, T, cb, 1>();
    } else if constexpr (k1_only_eligible(LA, LB, LC, LD)) {
      e.thr1[p][0] = thread_entry<LA, LB, LC, LD, T, ca, 1>();
    }
  }
}


}  // namespace jkinst
}  // namespace dgf

// Defines the static initialiser that fills part P of entry (X, Y) of the
// table; the build compiles one translation unit per class pair and part, so
// the classes compile in parallel.
#define DGF_JK_CLASS(X, Y, P)                                                                 \
  namespace dgf {                                                                             \
  namespace {                                                                                 \
  struct ClassInit_##X##_##Y##_##P {                                                          \
    ClassInit_##X##_##Y##_##P() { jkinst::fill_part<X, Y, P>(); }                             \
  } g_class_init_##X##_##Y##_##P;                                                             \
  }                                                                                           \
  }
