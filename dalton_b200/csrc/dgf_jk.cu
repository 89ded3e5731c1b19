// Quartet-class kernel table of libdgfock: one instantiation of the J/K
// quartet kernel per (bra class, ket class) of angular momenta up to f.
#include <utility>

#include "dgf_jk_team.cuh"

namespace dgf {
namespace {

constexpr int cls_la(int X) { return X == 0 ? 0 : X <= 2 ? 1 : X <= 5 ? 2 : 3; }
constexpr int cls_lb(int X) { return X - cls_la(X) * (cls_la(X) + 1) / 2; }

template <int LA, int LB, int LC, int LD>
void launch_team(const JKArgs &a, int grid, int block, size_t smem, cudaStream_t s) {
  jk_team_kernel<LA, LB, LC, LD><<<grid, block, smem, s>>>(a);
}

template <int LA, int LB, int LC, int LD>
cudaError_t prepare_team() {
  return cudaFuncSetAttribute(jk_team_kernel<LA, LB, LC, LD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)TeamShape<LA, LB, LC, LD>::smem());
}

struct Entry {
  ClassKernel k;
  cudaError_t (*prepare)();
};

Entry g_team[kNumPairClass][kNumPairClass];

template <int X, int Y>
void fill_one() {
  constexpr int LA = cls_la(X), LB = cls_lb(X), LC = cls_la(Y), LD = cls_lb(Y);
  using S = TeamShape<LA, LB, LC, LD>;
  constexpr int work = S::NAB * S::NCD;
  constexpr int block = work >= 512 ? 128 : work >= 64 ? 64 : 32;
  g_team[X][Y].k = ClassKernel{&launch_team<LA, LB, LC, LD>, block, S::smem()};
  g_team[X][Y].prepare = &prepare_team<LA, LB, LC, LD>;
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

const ClassKernel &jk_kernel(int X, int Y, int precision) {
  (void)precision;
  return g_team[X][Y].k;
}

cudaError_t jk_prepare_all() {
  for (int X = 0; X < kNumPairClass; ++X)
    for (int Y = 0; Y <= X; ++Y) {
      cudaError_t e = g_team[X][Y].prepare();
      if (e != cudaSuccess) return e;
    }
  return cudaSuccess;
}

}  // namespace dgf
