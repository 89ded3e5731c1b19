// AO basis <-> two-electron working basis.
//
// The quartet kernels run in a working basis in which every general
// contraction (a Dalton block whose contracted functions share primitives,
// e.g. the 1s/2s/3s functions of cc-pVDZ oxygen built from one set of nine
// exponents) is resolved into its primitives.  J and K are bilinear, so with
// C the contraction matrix (AO function mu = sum_p C_p,mu working function p)
//   D_w = C D C^T,   F = C^T F_w C
// reproduces the AO-basis Fock matrix exactly, while each primitive integral
// is computed once instead of once per contracted function that uses it.
//
// The maps are sparse rows (a working function feeds at most the handful of
// contracted functions of its block); one kernel launch covers one matrix of
// one molecule or the packed matrices of a whole batch.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace dgf {

struct WorkMaps {
  int nmol;
  const int64_t *w_elem;         // [nmol+1] packed working-matrix offsets
  const int64_t *a_elem;         // [nmol+1] packed AO-matrix offsets
  const int *nw, *na;            // [nmol] working / AO functions per molecule
  const int *wf_base, *af_base;  // [nmol] first global working / AO function of each molecule
  const int *wr_off, *wr_idx;    // rows of C per global working function: local AO index
  const double *wr_c;
  const int *ac_off, *ac_idx;    // columns of C per global AO function: local working index
  const double *ac_c;
};

// Working-basis slot densities from AO densities: for every working element,
// a = (C Din C^T)_pq and t = (C Din C^T)_qp; D = a (op 0), t (op 1),
// (a+t)/2 (op 2), (a-t)/2 (op 3); Ds = a + t (0 for op 3), skipped when null.
void launch_work_prep(const WorkMaps &m, const double *din, double *d, double *ds, int op, int64_t total_w,
                      int nsm, cudaStream_t st);

// AO Fock matrices from working-basis half matrices: F = C^T (F1 + sign F2^T) C.
void launch_work_combine(const WorkMaps &m, const double *f1, const double *f2, double *f, double sign,
                         int64_t total_a, int nsm, cudaStream_t st);

}  // namespace dgf
