// Quartet-class kernel table of libdgfock: for every (bra class, ket class)
// of angular momenta up to f, the cooperative team kernel and, for the low
// classes, the register-resident thread kernel in FP64 and FP32.
#include <utility>

#include "dgf_jk_thread.cuh"

namespace dgf {
namespace {

constexpr int cls_la(int X) { return X == 0 ? 0 : X <= 2 ? 1 : X <= 5 ? 2 : 3; }
constexpr int cls_lb(int X) { return X - cls_la(X) * (cls_la(X) + 1) / 2; }

// Classes small enough for one thread to hold the whole quartet in registers.
constexpr bool thread_eligible(int LA, int LB, int LC, int LD) {
  return ncart(LA) * ncart(LB) * ncart(LC) * ncart(LD) <= 27 && LA + LB + LC + LD <= 4;
}

template <int LA, int LB, int LC, int LD>
void launch_team(const JKArgs &a, int grid, int block, size_t smem, cudaStream_t s) {
  jk_team_kernel<LA, LB, LC, LD><<<grid, block, smem, s>>>(a);
}

template <int LA, int LB, int LC, int LD, typename T>
void launch_thread(const JKArgs &a, int grid, int block, size_t smem, cudaStream_t s) {
  jk_thread_kernel<LA, LB, LC, LD, T><<<grid, block, smem, s>>>(a);
}

template <int LA, int LB, int LC, int LD>
cudaError_t prepare_team() {
  return cudaFuncSetAttribute(jk_team_kernel<LA, LB, LC, LD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)TeamShape<LA, LB, LC, LD>::smem());
}

struct Entry {
  ClassKernel team, thr64, thr32;
  cudaError_t (*prepare)();
};

Entry g_tab[kNumPairClass][kNumPairClass];

template <int X, int Y>
void fill_one() {
  constexpr int LA = cls_la(X), LB = cls_lb(X), LC = cls_la(Y), LD = cls_lb(Y);
  using S = TeamShape<LA, LB, LC, LD>;
  constexpr int work = S::NAB * S::NCD;
  constexpr int block = work >= 512 ? 128 : work >= 64 ? 64 : 32;
  Entry &e = g_tab[X][Y];
  e.team = ClassKernel{&launch_team<LA, LB, LC, LD>, block, S::smem()};
  e.prepare = &prepare_team<LA, LB, LC, LD>;
  if constexpr (thread_eligible(LA, LB, LC, LD)) {
    e.thr64 = ClassKernel{&launch_thread<LA, LB, LC, LD, double>, 128, 0};
    e.thr32 = ClassKernel{&launch_thread<LA, LB, LC, LD, float>, 128, 0};
  } else {
    e.thr64 = ClassKernel{nullptr, 0, 0};
    e.thr32 = ClassKernel{nullptr, 0, 0};
  }
}

template <int X, int... Ys>
void fill_row(std::integer_sequence<int, Ys...>) {
  (fill_one<X, Ys>(), ...);
}

template <int... Xs>
void fill_all(std::integer_sequence<int, Xs...>) {
  (fill_row<Xs>(std::make_integer_sequence<int, Xs + 1>{}), ...);
}

struct Init {
  Init() { fill_all(std::make_integer_sequence<int, kNumPairClass>{}); }
} g_init;

}  // namespace

// precision: 0 = FP64 (thread kernel when the class has one, else team),
// 1 = FP32 thread kernel (launch == nullptr when the class has none),
// 2 = FP64 team kernel.
const ClassKernel &jk_kernel(int X, int Y, int precision) {
  const Entry &e = g_tab[X][Y];
  if (precision == 1) return e.thr32;
  if (precision == 2) return e.team;
  return e.thr64.launch ? e.thr64 : e.team;
}

cudaError_t jk_prepare_all() {
  for (int X = 0; X < kNumPairClass; ++X)
    for (int Y = 0; Y <= X; ++Y) {
      cudaError_t e = g_tab[X][Y].prepare();
      if (e != cudaSuccess) return e;
    }
  return cudaSuccess;
}

}  // namespace dgf
