// Quartet selection shared by the Fock kernels: the Schwarz cut of the
// plan's last bin, Dalton's density screen on its blocks, and the precision
// split of the mixed form.
#pragma once

#include "dgf_md.cuh"

namespace dgf {

// Precision bound of the mixed form on working-basis shells:
// Q_AB Q_CD max(4 max(|D|_AB,|D|_CD), |D|_AC,|D|_AD,|D|_BC,|D|_BD), the
// shape of SYMLOP's bound (DALTON/abacus/her2drv.F:2666-2692) with the
// working-basis density.
__device__ __forceinline__ double quartet_bound(const JKArgs &a, const PairRec &b, const PairRec &k) {
  float dj, dk;
  if (a.dmax_w) {  // batches: shell-pair maxima at the shells' first functions in the molecule's block
    const float *dm = a.dmax_w + k.dbase;
    const int n = k.nbfm;
    dj = fmaxf(dm[b.aoA * n + b.aoB], dm[k.aoA * n + k.aoB]);
    dk = fmaxf(fmaxf(dm[b.aoA * n + k.aoA], dm[b.aoA * n + k.aoB]), fmaxf(dm[b.aoB * n + k.aoA], dm[b.aoB * n + k.aoB]));
  } else {
    const float *dm = a.dmax;
    const int n = a.nshell;
    dj = fmaxf(dm[b.shA * n + b.shB], dm[k.shA * n + k.shB]);
    dk = fmaxf(fmaxf(dm[b.shA * n + k.shA], dm[b.shA * n + k.shB]), fmaxf(dm[b.shB * n + k.shA], dm[b.shB * n + k.shB]));
  }
  return b.Q * k.Q * (double)fmaxf(4.0f * dj, dk);
}

// Dalton's density screen (SYMLOP, DALTON/abacus/her2drv.F:2663-2733) on
// the Dalton blocks the quartet's shells lie in: GAB_AB GAB_CD
// max(4 max(|D|_AB,|D|_CD), |D|_AC,|D|_AD,|D|_BC,|D|_BD) with the block
// Schwarz factors and the block maxima of the AO densities.  Every working
// quartet of a block quartet gets the block quartet's decision, so the
// build skips exactly the block quartets Dalton skips.
__device__ __forceinline__ double block_bound(const JKArgs &a, const PairRec *bp, const PairRec *kp) {
  const int4 b = block_of_pair(bp), k = block_of_pair(kp);
  const int n = a.nblk;
  const float *dm = a.blk_dmax;
  const float dj = fmaxf(dm[b.x * n + b.y], dm[k.x * n + k.y]);
  const float dk = fmaxf(fmaxf(dm[b.x * n + k.x], dm[b.x * n + k.y]), fmaxf(dm[b.y * n + k.x], dm[b.y * n + k.y]));
  return a.blk_gab[b.x * n + b.y] * a.blk_gab[k.x * n + k.y] * (double)fmaxf(4.0f * dj, dk);
}

// Returns 0 = evaluate, 1 = outside this launch's precision range, 2 = screened
// out by the density bound, 3 = below the Schwarz threshold (the plan's last bin).
__device__ __forceinline__ int quartet_select(const JKArgs &a, const PairRec &b, const PairRec &k, const PairRec *bp,
                                              const PairRec *kp) {
  if (b.Q * k.Q < a.schwarz_thr) return 3;
  if (a.blk_gab && block_bound(a, bp, kp) < a.dens_thr) return 2;
  if ((!a.dmax && !a.dmax_w) || a.mode == 0) return 0;
  const double bound = quartet_bound(a, b, k);
  if (a.mode == 1 && bound < a.split) return 1;
  if (a.mode == 2 && bound >= a.split) return 1;
  return 0;
}

}  // namespace dgf
