// Fock builds from stored integrals: the conventional form of the build
// (Dalton's SIRFCK2 over the AOTWOINT integral file, DALTON/sirius/
// sirfck.F:1122-1342), with the file replaced by a device-memory store.
// dgf_store_integrals evaluates every quartet of the plan once with the
// integral kernels, which write the blocks (layout [a][b][c][d], nint
// values per quartet, in plan order) instead of digesting them; these
// kernels walk the same class queues, read each quartet's block and digest
// it with the same six-block code as the direct kernels (FCKCON,
// DALTON/abacus/herfckcon.F:66-80), so any number of densities, IFCTYP codes
// and HFXFAC values reuse one integral evaluation.
#pragma once

#include "dgf_jk_thread.cuh"
#include "dgf_jk_warp.cuh"

namespace dgf {

// Classes whose Cartesian block has at most this many values are digested
// one quartet per thread (block in registers); larger ones one per warp
// (block staged in shared memory).
constexpr int kStoredThreadMax = 36;

template <int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(kThreadBlock, 2) jk_stored_thread_kernel(const JKArgs a) {
  constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD), NOUT = NA * NB * NC * ND;
  constexpr int FA = nfun(LA, 1), FB = nfun(LB, 1), FC = nfun(LC, 1), FD = nfun(LD, 1);
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int nint = a.store_nint;
  unsigned long long cnt_q = 0, cnt_s = 0;
  // block-contiguous ranges, 32-quartet chunks per warp, as the thread kernels
  const int nw = blockDim.x >> 5, warp = threadIdx.x >> 5;
  const int64_t nq = a.nquartet - a.q_begin;
  const int64_t bspan = ((nq + gridDim.x - 1) / gridDim.x + 31) & ~(int64_t)31;
  const int64_t bbegin = a.q_begin + (int64_t)blockIdx.x * bspan, bend = min(bbegin + bspan, a.nquartet);
  int ibw = -1;
  for (int64_t base = bbegin + (int64_t)warp * 32; base < bend; base += (int64_t)nw * 32) {
    const int64_t q = base + lane;
    const bool active = q < bend;
    int ib0 = ibw;
    if (lane == 0) {
      if (ib0 < 0) {
        ib0 = find_bra(a.qoff, a.nbra, base);
      } else {
        int steps = 0;
        while (base >= a.qoff[ib0 + 1] && steps < 32) {
          ++ib0;
          ++steps;
        }
        if (base >= a.qoff[ib0 + 1]) ib0 = find_bra(a.qoff, a.nbra, base);
      }
    }
    ib0 = __shfl_sync(full, ib0, 0);
    ibw = ib0;
    int ib = ib0, ic = 0, sel = 1;
    PairRec br, kt;
    if (active) {
      int steps = 0;
      while (q >= a.qoff[ib + 1] && steps < 32) {
        ++ib;
        ++steps;
      }
      if (q >= a.qoff[ib + 1]) ib = find_bra(a.qoff, a.nbra, q);
      ic = (int)(q - a.qoff[ib]) + (a.kbase ? a.kbase[ib] : 0);
      br = load_pair_fock(a.bra + ib);
      kt = load_pair_fock(a.ket + ic);
      sel = quartet_select(a, br, kt, a.bra + ib, a.ket + ic);
      if (sel == 2) ++cnt_s;
    }
    const bool work = active && sel == 0;
    double g[NOUT];
    const double *s = a.store_in + a.store_base + q * nint;
#pragma unroll
    for (int k = 0; k < NOUT; ++k) g[k] = (work && k < nint) ? __ldg(s + k) : 0.0;
    if (!__any_sync(full, work)) continue;
    double jnone[1];
    if (a.spherical)
      jk_digest<FA, FB, FC, FD, 1>(a, g, work, ib, ic, ib0, br, kt, 0, jnone, false);
    else
      jk_digest<NA, NB, NC, ND, 1>(a, g, work, ib, ic, ib0, br, kt, 0, jnone, false);
    cnt_q += work ? 1 : 0;
  }
  if (a.counters) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      cnt_q += __shfl_xor_sync(full, cnt_q, off);
      cnt_s += __shfl_xor_sync(full, cnt_s, off);
    }
    if (lane == 0) {
      atomicAdd(a.counters + 0, cnt_q);
      atomicAdd(a.counters + 2, cnt_s);
    }
  }
}

// One warp per quartet: the block (nint values) is staged in shared memory
// with the warp kernel's row stride and digested by its six-block code.
template <int LA, int LB, int LC, int LD>
struct StoredShape {
  using S = wq::Shape<LA, LB, LC, LD, double>;
  static constexpr int PER_WARP = S::NAB * S::PG + S::RD + 8;  // doubles
  static constexpr size_t smem(int warps) { return (size_t)warps * PER_WARP * 8; }
  static constexpr int WPB = smem(4) <= 100 * 1024 ? 4 : smem(2) <= 100 * 1024 ? 2 : 1;
};

template <int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(128) jk_stored_warp_kernel(const JKArgs a) {
  using S = wq::Shape<LA, LB, LC, LD, double>;
  using T = StoredShape<LA, LB, LC, LD>;
  constexpr int PG = S::PG;
  extern __shared__ double sm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  double *Gc = sm + (size_t)warp * T::PER_WARP, *Db = Gc + S::NAB * PG;
  const int ncd = a.spherical ? S::FCD : S::NCD;  // columns of the stored block
  const int nint = a.store_nint;
  unsigned long long cnt_q = 0, cnt_s = 0;
  const int64_t nteam = (int64_t)gridDim.x * nw, team = (int64_t)blockIdx.x * nw + warp;
  const int64_t span = (a.nquartet - a.q_begin + nteam - 1) / nteam;
  const int64_t qbeg = a.q_begin + team * span, qend = min(qbeg + span, a.nquartet);
  int ibw = -1;
  for (int64_t q = qbeg; q < qend; ++q) {
    int ib = 0;
    if (lane == 0) {
      if (ibw < 0) {
        ibw = find_bra(a.qoff, a.nbra, q);
      } else {
        int steps = 0;
        while (q >= a.qoff[ibw + 1] && steps < 32) {
          ++ibw;
          ++steps;
        }
        if (q >= a.qoff[ibw + 1]) ibw = find_bra(a.qoff, a.nbra, q);
      }
      ib = ibw;
    }
    ib = __shfl_sync(0xffffffffu, ib, 0);
    ibw = ib;
    const int ic = (int)(q - a.qoff[ib]) + (a.kbase ? a.kbase[ib] : 0);
    const PairRec br = load_pair_fock(a.bra + ib), kt = load_pair_fock(a.ket + ic);
    const int sel = quartet_select(a, br, kt, a.bra + ib, a.ket + ic);
    if (sel) {
      if (lane == 0 && sel == 2) ++cnt_s;
      continue;
    }
    double w = 1.0;
    if (br.same) w *= 0.5;
    if (kt.same) w *= 0.5;
    if (a.same_class && ib == ic + a.ket_off) w *= 0.5;
    const double *s = a.store_in + a.store_base + q * nint;
    for (int e = lane; e < nint; e += 32) Gc[(e / ncd) * PG + e % ncd] = __ldg(s + e);
    __syncwarp();
    if (a.spherical)
      wq_finish<LA, LB, LC, LD, double, true, true>(a, Gc, nullptr, Db, nullptr, br, kt, ib, ic, w, lane, q);
    else
      wq_finish<LA, LB, LC, LD, double, false>(a, Gc, nullptr, Db, nullptr, br, kt, ib, ic, w, lane, q);
    __syncwarp();
    if (lane == 0) ++cnt_q;
  }
  if (lane == 0 && a.counters) {
    atomicAdd(a.counters + 0, cnt_q);
    atomicAdd(a.counters + 2, cnt_s);
  }
}

}  // namespace dgf
