// Instantiation of parts 1 (FP64) and 2 (FP32) of the quartet-class kernel
// table (see dgf_jk_inst.cuh): the thread-per-quartet kernels.
#pragma once

#include <type_traits>

#include "dgf_jk_inst.cuh"
#include "dgf_jk_thread.cuh"

namespace dgf {
namespace jkinst {

template <int LA, int LB, int LC, int LD, typename T, int CA, int K1>
void launch_thread(const JKArgs &a, int grid, int block, size_t smem, cudaStream_t s) {
  jk_thread_kernel<LA, LB, LC, LD, T, CA, K1><<<dim3(grid, CA), block, smem, s>>>(a);
}

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

template <int X, int Y, int P>
cudaError_t prepare_thread() {
  constexpr int LA = cls_la(X), LB = cls_lb(X), LC = cls_la(Y), LD = cls_lb(Y);
  using T = std::conditional_t<P == 1, double, float>;
  using C = ThreadCfg<LA, LB, LC, LD>;
  constexpr int ca = P == 1 ? C::c64 : C::c32, cb = P == 1 ? C::c64b : C::c32b;
  cudaError_t e = cudaSuccess;
  if constexpr (thread_eligible(LA, LB, LC, LD)) {
    e = carve_thread<LA, LB, LC, LD, T, ca>();
    if constexpr (cb != ca)
      if (e == cudaSuccess) e = carve_thread<LA, LB, LC, LD, T, cb>();
  } else if constexpr (k1_only_eligible(LA, LB, LC, LD)) {
    e = carve_one<LA, LB, LC, LD, T, ca, 1>();
  }
  return e;
}

template <int LA, int LB, int LC, int LD, typename T, int CA, int K1 = 0>
ClassKernel thread_entry() {
  return ClassKernel{&launch_thread<LA, LB, LC, LD, T, CA, K1>, kThreadBlock, 0, CA, kThreadBlock, kKindThread};
}

template <int X, int Y, int P>
void fill_thread() {
  constexpr int LA = cls_la(X), LB = cls_lb(X), LC = cls_la(Y), LD = cls_lb(Y);
  JKEntry &e = g_jk_table[X][Y];
  e.prepare[P] = &prepare_thread<X, Y, P>;
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

}  // namespace jkinst
}  // namespace dgf

// Static initialiser filling part P (1: FP64, 2: FP32) of entry (X, Y).
#define DGF_JK_THREAD_CLASS(X, Y, P)                                                          \
  namespace dgf {                                                                             \
  namespace {                                                                                 \
  struct ThreadInit_##X##_##Y##_##P {                                                         \
    ThreadInit_##X##_##Y##_##P() { jkinst::fill_thread<X, Y, P>(); }                          \
  } g_thread_init_##X##_##Y##_##P;                                                            \
  }                                                                                           \
  }
