// The quartet-class kernel table of libdgfock and what its instantiation
// units share.  The entry of class pair (X, Y) is filled by three generated
// translation units (parts) so that the heaviest classes compile in
// parallel and a change to one kernel family rebuilds only its units:
// part 0 the cooperative, warp-team and warp-per-quartet kernels
// (dgf_jk_inst_team.cuh), parts 1 and 2 the FP64 and FP32 thread kernels
// (dgf_jk_inst_thread.cuh).  Each part sets only its own fields of the
// (zero-initialised) entry and its own prepare hook.
#pragma once

#include "dgf_internal.h"

namespace dgf {

struct JKEntry {
  ClassKernel team;
  ClassKernel wteam;                     // one quartet per warp (light quartets), when it fits
  ClassKernel thr[2][kThreadVariants];   // [precision 0 = FP64, 1 = FP32][variant]
  ClassKernel thr1[2][kThreadVariants];  // same, for kets of one primitive pair each
  ClassKernel warp[2];                   // warp-per-quartet kernel [FP64, FP32]
  bool warp_mp;                          // the warp kernel loops over primitive pairs (else one per side only)
  ClassKernel warp_mma;                  // warp-per-quartet kernel with DMMA transforms (FP64, any pairs)
  ClassKernel stored;                    // digestion of stored integral blocks (conventional form)
  cudaError_t (*prepare[3])();           // one per generated part
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

// Thread-kernel chunk counts of a class: FP64 / FP32, first and second variant.
template <int LA, int LB, int LC, int LD>
struct ThreadCfg {
  static constexpr int c64 = chunks_for(LA, LB, LC, LD, 27), c64b = cmin(ncart(LA), 2 * c64);
  static constexpr int c32 = chunks_for(LA, LB, LC, LD, 54), c32b = cmin(ncart(LA), 2 * c32);
};

}  // namespace jkinst
}  // namespace dgf
