// Instantiation helpers of the quartet-class kernel table: one translation
// unit per class pair (generated by the build, see DGF_JK_CLASS) fills its
// entry, so the classes compile in parallel.
#pragma once

#include <utility>

#include "dgf_jk_thread.cuh"

namespace dgf {

struct JKEntry {
  ClassKernel team;
  ClassKernel wteam;                     // one quartet per warp (light quartets), when it fits
  ClassKernel thr[2][kThreadVariants];   // [precision 0 = FP64, 1 = FP32][variant]
  ClassKernel thr1[2][kThreadVariants];  // same, for kets of one primitive pair each
  cudaError_t (*prepare)();
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
  return cudaFuncSetAttribute(jk_thread_kernel<LA, LB, LC, LD, T, CA, K1>,
                              cudaFuncAttributePreferredSharedMemoryCarveout, kThreadCarveoutPercent);
}

template <int LA, int LB, int LC, int LD, typename T, int CA>
cudaError_t carve_thread() {
  cudaError_t e = carve_one<LA, LB, LC, LD, T, CA, 0>();
  if (e == cudaSuccess) e = carve_one<LA, LB, LC, LD, T, CA, 1>();
  return e;
}

template <int LA, int LB, int LC, int LD>
cudaError_t prepare_class() {
  using TS = TeamShape<LA, LB, LC, LD>;
  cudaError_t e = cudaFuncSetAttribute(jk_team_kernel<LA, LB, LC, LD, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)TS::smem());
  if constexpr (TS::kWarpTeams > 0)
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(jk_team_kernel<LA, LB, LC, LD, TS::kWarpTeams>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TS::smem_w(TS::kWarpTeams));
  if constexpr (thread_eligible(LA, LB, LC, LD)) {
    using C = ThreadCfg<LA, LB, LC, LD>;
    if (e == cudaSuccess) e = carve_thread<LA, LB, LC, LD, double, C::c64>();
    if (e == cudaSuccess) e = carve_thread<LA, LB, LC, LD, float, C::c32>();
    if constexpr (C::c64b != C::c64)
      if (e == cudaSuccess) e = carve_thread<LA, LB, LC, LD, double, C::c64b>();
    if constexpr (C::c32b != C::c32)
      if (e == cudaSuccess) e = carve_thread<LA, LB, LC, LD, float, C::c32b>();
  } else if constexpr (k1_only_eligible(LA, LB, LC, LD)) {
    using C = ThreadCfg<LA, LB, LC, LD>;
    if (e == cudaSuccess) e = carve_one<LA, LB, LC, LD, double, C::c64, 1>();
    if (e == cudaSuccess) e = carve_one<LA, LB, LC, LD, float, C::c32, 1>();
  }
  return e;
}

template <int LA, int LB, int LC, int LD, typename T, int CA, int K1 = 0>
ClassKernel thread_entry() {
  return ClassKernel{&launch_thread<LA, LB, LC, LD, T, CA, K1>, kThreadBlock, 0, CA, kThreadBlock};
}

template <int X, int Y>
void fill_one() {
  constexpr int LA = cls_la(X), LB = cls_lb(X), LC = cls_la(Y), LD = cls_lb(Y);
  using S = TeamShape<LA, LB, LC, LD>;
  constexpr int work = S::NAB * S::NCD;
  constexpr int block = work >= 512 ? 128 : work >= 64 ? 64 : 32;
  JKEntry &e = g_jk_table[X][Y];
  e.team = ClassKernel{&launch_team<LA, LB, LC, LD, 0>, block, S::smem(), 1, 1};
  if constexpr (S::kWarpTeams > 0)
    e.wteam = ClassKernel{&launch_team<LA, LB, LC, LD, S::kWarpTeams>, 32 * S::kWarpTeams,
                          S::smem_w(S::kWarpTeams), 1, S::kWarpTeams};
  else
    e.wteam = ClassKernel{nullptr, 0, 0, 0, 0};
  e.prepare = &prepare_class<LA, LB, LC, LD>;
  for (int p = 0; p < 2; ++p)
    for (int v = 0; v < kThreadVariants; ++v) e.thr[p][v] = e.thr1[p][v] = ClassKernel{nullptr, 0, 0, 0, 0};
  if constexpr (thread_eligible(LA, LB, LC, LD)) {
    using C = ThreadCfg<LA, LB, LC, LD>;
    constexpr int c64 = C::c64, c64b = C::c64b, c32 = C::c32, c32b = C::c32b;
    e.thr[0][0] = thread_entry<LA, LB, LC, LD, double, c64>();
    e.thr[1][0] = thread_entry<LA, LB, LC, LD, float, c32>();
    if constexpr (c64b != c64) e.thr[0][1] = thread_entry<LA, LB, LC, LD, double, c64b>();
    if constexpr (c32b != c32) e.thr[1][1] = thread_entry<LA, LB, LC, LD, float, c32b>();
    e.thr1[0][0] = thread_entry<LA, LB, LC, LD, double, c64, 1>();
    e.thr1[1][0] = thread_entry<LA, LB, LC, LD, float, c32, 1>();
    if constexpr (c64b != c64) e.thr1[0][1] = thread_entry<LA, LB, LC, LD, double, c64b, 1>();
    if constexpr (c32b != c32) e.thr1[1][1] = thread_entry<LA, LB, LC, LD, float, c32b, 1>();
  } else if constexpr (k1_only_eligible(LA, LB, LC, LD)) {
    using C = ThreadCfg<LA, LB, LC, LD>;
    e.thr1[0][0] = thread_entry<LA, LB, LC, LD, double, C::c64, 1>();
    e.thr1[1][0] = thread_entry<LA, LB, LC, LD, float, C::c32, 1>();
  }
}


}  // namespace jkinst
}  // namespace dgf

// Defines the static initialiser that fills entry (X, Y) of the table; the
// build compiles one translation unit per class pair, so the classes compile
// in parallel.
#define DGF_JK_CLASS(X, Y)                                                                    \
  namespace dgf {                                                                             \
  namespace {                                                                                 \
  struct ClassInit_##X##_##Y {                                                                \
    ClassInit_##X##_##Y() { jkinst::fill_one<X, Y>(); }                                       \
  } g_class_init_##X##_##Y;                                                                   \
  }                                                                                           \
  }
