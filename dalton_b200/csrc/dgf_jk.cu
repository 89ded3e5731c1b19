// Quartet-class kernel table of libdgfock: for every (bra class, ket class)
// of angular momenta up to f, the cooperative team kernel, the
// warp-per-quartet kernel (L >= 4, FP64 and FP32) and, for the classes up to
// L = 5, register-resident thread kernels in FP64 and FP32, each in two
// A-chunk variants (the per-class tuning space).  The entries are filled by
// generated translation units (dgf_jk_inst.cuh).
#include "dgf_jk_inst.cuh"

namespace dgf {

JKEntry g_jk_table[kNumPairClass][kNumPairClass];

namespace {
const ClassKernel kNone{nullptr, 0, 0, 0, 0, 0};
}

// variant: -4 = warp-per-quartet kernel with FP64 tensor-core (DMMA)
// transforms (any pairs), -3 = warp-per-quartet kernel (for launches whose pairs have one
// primitive pair each, or any launch of a class whose warp kernel loops over
// primitives), -2 = warp-team kernel, -1 = team kernel, 0.. = thread-kernel
// variant; precision 0 = FP64, 1 = FP32.
// Returns a kernel with launch == nullptr when absent.
const ClassKernel &jk_kernel_variant(int X, int Y, int precision, int variant, bool ket1, bool bra1) {
  const JKEntry &e = g_jk_table[X][Y];
  const int p = precision ? 1 : 0;
  if (variant == -4) return precision == 0 ? e.warp_mma : kNone;
  if (variant == -3) return ((ket1 && bra1) || e.warp_mp) ? e.warp[p] : kNone;
  if (variant == -2) return precision == 0 ? e.wteam : kNone;
  if (variant < 0) return precision == 0 ? e.team : kNone;
  if (variant >= kThreadVariants) return kNone;
  if (ket1 && e.thr1[p][variant].launch) return e.thr1[p][variant];
  return e.thr[p][variant];
}

// Default choice: first thread variant when the class has one, else the
// warp-per-quartet kernel for single-primitive launches, else team.
const ClassKernel &jk_kernel(int X, int Y, int precision, bool ket1, bool bra1) {
  const JKEntry &e = g_jk_table[X][Y];
  if (precision == 2) return e.team;
  const int p = precision == 1 ? 1 : 0;
  if (ket1 && e.thr1[p][0].launch) return e.thr1[p][0];
  if (e.thr[p][0].launch) return e.thr[p][0];
  if (ket1 && bra1 && e.warp[p].launch) return e.warp[p];
  return precision == 1 ? kNone : e.team;
}

const ClassKernel &jk_stored_kernel(int X, int Y) { return g_jk_table[X][Y].stored; }

cudaError_t jk_prepare_all() {
  for (int X = 0; X < kNumPairClass; ++X)
    for (int Y = 0; Y <= X; ++Y)
      for (int P = 0; P < 3; ++P) {
        if (!g_jk_table[X][Y].prepare[P]) return cudaErrorInitializationError;  // a generated part is missing
        cudaError_t e = g_jk_table[X][Y].prepare[P]();
        if (e != cudaSuccess) return e;
      }
  return cudaSuccess;
}

}  // namespace dgf
