// Register-resident McMurchie-Davidson J/K quartet kernel: one thread per
// contracted shell quartet (optionally per chunk of its A-shell Cartesian
// components), a warp on 32 consecutive quartets of the class-sorted queue.
//
// Consecutive quartets of the queue share their bra pair, so the bra
// Hermite tables of the current bra primitive are built once per warp in
// shared memory and read by broadcast; Boys function, R_tuv, the ket tables,
// the ket transform and the accumulators stay in registers.  Warps whose
// lanes hold different bra pairs process one bra group after another.
//
// CA splits the A shell's Cartesian components into CA compile-time chunks
// (blockIdx.y); each chunk digests its partial spherical block (digestion is
// linear in the integrals), which bounds the accumulator count per thread.
//
// Tc is the arithmetic type of the Hermite recursion and the Hermite ->
// Cartesian contraction (double: FP64 drop-in; float: FP32 half of the mixed
// form).  Boys function, prefactor and digestion (FP64 atomics into the half
// Fock matrices) are FP64 in both.
#pragma once

#include "dgf_select.cuh"

namespace dgf {

// Segmented sum over runs of adjacent lanes with equal keys: after the call
// the first lane of each run (its head) holds the run's sum.  `end` is the
// last lane of the calling lane's run (seg_end below).
__device__ __forceinline__ double seg_sum(double v, int lane, int end) {
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const double t = __shfl_down_sync(0xffffffffu, v, off);
    if (lane + off <= end) v += t;
  }
  return v;
}

// Runs of adjacent lanes with equal key: whether this lane starts a run and
// the last lane of its run.
__device__ __forceinline__ void seg_end(int key, int lane, bool &head, int &end) {
  const int prev = __shfl_up_sync(0xffffffffu, key, 1);
  head = (lane == 0) || prev != key;
  const unsigned hm = __ballot_sync(0xffffffffu, head);
  const unsigned after = hm & ~((2u << lane) - 1u);
  end = after ? __ffs(after) - 2 : 31;
}

// K_ac/K_bc blocks of kSegMinValues to kSegMaxValues values per lane sum
// runs of lanes before their atomics; from kSegRowsMin values on, through
// shared memory.  Smaller blocks add one atomic per lane: measured on
// (H2O)32 / cc-pVDZ, per-lane atomics were faster for 2 to 10 values
// ((ss|ss) 9%, (ps|ss) 5%, (pp|ss) 7%, (ds|ss) 12%, (dp|ss) 10%, (dd|ss)
// 9%) and slower for the 12 of (ps|ps) (15.5 against 13.4 ms).
constexpr int kSegMinValues = 11;
constexpr int kSegMaxValues = 18;
constexpr int kSegRowsMin = 8;
constexpr int kSegStride = 33;  // doubles per row of a warp's buffer (32 lanes + 1 against bank conflicts)

// Run sums of the group lanes' K_ac / K_bc values, which the lanes wrote as
// columns of sbuf (row e < FA FC: K_ac[x][c], e = x FC + c; after that
// K_bc[y][c]).  Lane e < NV sums row e over each run of lanes with the same
// C shell and adds the total to the group bra's row; the run bounds, the
// C shell and whether the run belongs to the group are warp-uniform.
// Called by the whole warp; returns with sbuf free for reuse.
template <int FA, int FC, int NV>
__device__ __forceinline__ void seg_rows(double *sbuf, bool grp, int cfun, int send, double *Fg, const PairRec &brg,
                                         int a_off) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  __syncwarp();
  unsigned ends = __ballot_sync(full, send == lane);
  const unsigned gmask = __ballot_sync(full, grp);
  const double *row = sbuf + lane * kSegStride;
  int row_f, col_f;  // this lane's row of F (function) and offset within the C shell
  if (lane < FA * FC) {
    row_f = brg.aoA + a_off + lane / FC;
    col_f = lane % FC;
  } else {
    row_f = brg.aoB + (lane - FA * FC) / FC;
    col_f = (lane - FA * FC) % FC;
  }
  int j0 = 0;
  while (ends) {
    const int j1 = __ffs(ends) - 1;
    ends &= ends - 1;
    const int cj = __shfl_sync(full, cfun, j1);
    if ((gmask >> j1) & 1u) {
      double r = 0.0;
      if (lane < NV)
        for (int j = j0; j <= j1; ++j) r += row[j];
      if (lane < NV && r != 0.0) atomicAdd(Fg + (size_t)row_f * brg.nbfm + cj + col_f, r);
    }
    j0 = j1 + 1;
  }
  __syncwarp();
}

// One block of the digestion: s_o = sum_i g[gi(o, i)] d(i) for o < NO,
// i < NI, each density value d(i) loaded once (repeated loads of the same
// element are not merged across the atomics in between).  With NI <= NO
// the NI values are held and each s_o is emitted as it is formed; otherwise
// the NO sums accumulate over the loads.  emit(o, s) is called for every o
// in order by every lane (s = 0 where !on), after the block's loads.
template <int NO, int NI, typename GI, typename DV, typename EMIT>
__device__ __forceinline__ void block_sums(bool on, const double *g, GI gi, DV dv, EMIT emit) {
  if constexpr (NI <= NO) {
    double d[NI];
#pragma unroll
    for (int i = 0; i < NI; ++i) d[i] = on ? dv(i) : 0.0;
#pragma unroll
    for (int o = 0; o < NO; ++o) {
      double s = 0.0;
#pragma unroll
      for (int i = 0; i < NI; ++i) s += g[gi(o, i)] * d[i];
      emit(o, s);
    }
  } else {
    double s[NO];
#pragma unroll
    for (int o = 0; o < NO; ++o) s[o] = 0.0;
    if (on) {
#pragma unroll
      for (int i = 0; i < NI; ++i) {
        const double d = dv(i);
#pragma unroll
        for (int o = 0; o < NO; ++o) s[o] += g[gi(o, i)] * d;
      }
    }
#pragma unroll
    for (int o = 0; o < NO; ++o) emit(o, s[o]);
  }
}

// Digestion of one quartet block g[FA][FB][FC][FD] (FA rows of A starting at
// function a_off) into the half Fock matrices with FP64 atomics: the six J/K
// blocks of FCKCON (DALTON/abacus/herfckcon.F:66-80)
//   J_ab += g Ds_cd,  J_cd += g Ds_ab,
//   K_ac += g D_bd, K_ad += g D_bc, K_bc += g D_ad, K_bd += g D_ac.
// The lanes whose bra pair is the group bra (the warp's first bra) sum J_ab
// with a warp reduction and K_ac,
// K_bc over runs of adjacent lanes with the same C shell (the kets of a
// Schwarz bin are sorted by shell) with a segmented reduction, so that one
// atomic serves the run.  Density screening
// per density (ICEDIF, DALTON/abacus/her2fck.F:221-222,446-466): with
// ice_thr > 0, a lane whose quartet consists of whole Dalton blocks drops
// its Coulomb part of density k when max(|D|_AB,|D|_CD) max|g| < ice_thr
// (bit 1 of icedif) and its exchange part when the exchange blocks' bound
// does (bit 2), with the block maxima of the AO density.
//
// With jon (one density slot), the group lanes add their J_ab terms to the
// registers jacc instead, which the caller reduces across the warp once the
// warp leaves that bra (jk_jab_flush).
//
// With sbuf (the warp's kSegStride x 32 doubles of shared memory) and 8 to
// 18 K_ac/K_bc values per lane, the runs are summed through shared memory
// instead of shuffles: each lane writes its values as one column, then lane
// e sums row e over each run and adds the run's total (seg_rows).
template <int FA, int FB, int FC, int FD, int JN>
__device__ __forceinline__ void jk_digest(const JKArgs &a, const double *g, bool work, int ib, int ic, int gib,
                                          const PairRec &br, const PairRec &kt, int a_off, double (&jacc)[JN],
                                          bool jon, double *sbuf = nullptr) {
  // Segmented reduction of K_ac and K_bc where it is cheap next to the atomics it saves.
  constexpr int NV = (FA + FB) * FC;
  constexpr bool SEG = NV >= kSegMinValues && NV <= kSegMaxValues;
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  double w = 0.0;
  if (work) {
    w = 1.0;
    if (br.same) w *= 0.5;
    if (kt.same) w *= 0.5;
    if (a.same_class && ib == ic + a.ket_off) w *= 0.5;
  }
  // Group: lanes on the group bra reduce their bra-row blocks together.
  const bool grp = work && ib == gib;
  const PairRec brg = load_pair_fock(a.bra + gib);
  // Runs of group lanes with the same C shell (K_ac, K_bc); other lanes are runs of their own.
  bool head = true;
  int send = lane;
  if (SEG) seg_end(grp ? kt.aoA : -1 - lane, lane, head, send);
  // Shared-memory run sums pay a fixed scan of the warp's 32 columns plus
  // one step per run; shuffles pay per value.  The buffer is used when the
  // group's runs are few next to the values (measured: many short runs, as
  // in (ps|ps), make the scan slower than the shuffles).
  bool tseg = false;
  if (SEG && NV >= kSegRowsMin && sbuf != nullptr)
    tseg = 2 * __popc(__ballot_sync(full, grp && head)) <= NV;
  double aomax = 0.0;
  bool ice = false;
  if (a.ice_thr > 0.0 && work) {
    const int4 bb = block_of_pair(a.bra + ib), kb = block_of_pair(a.ket + ic);
    ice = (bb.z & bb.w & kb.z & kb.w) != 0;  // all four shells are whole Dalton blocks
    if (ice) {
#pragma unroll
      for (int e = 0; e < FA * FB * FC * FD; ++e) aomax = fmax(aomax, fabs(g[e]));
    }
  }
  const int N = work ? br.nbfm : brg.nbfm;
  const int64_t db = work ? br.dbase : brg.dbase;
  for (int k = 0; k < a.nslot; ++k) {
    const double *Dk = a.D + k * a.slot_stride + db;
    const double *Dsk = a.Ds + k * a.slot_stride + db;
    double *Fk = a.Fh + k * a.slot_stride + db;
    double *Fg = a.Fh + k * a.slot_stride + brg.dbase;
    // Rows of the bra's functions in D.  D and Ds are read-only during the
    // build, so their gathers take the non-coherent path and stay in
    // registers across the atomics into Fh.
    auto dA = [&](int x, int col) -> double { return __ldg(Dk + (size_t)(br.aoA + a_off + x) * N + col); };
    auto dB = [&](int y, int col) -> double { return __ldg(Dk + (size_t)(br.aoB + y) * N + col); };
    double js = a.jscale[k] * w, ks = -a.kscale[k] * w;
    if (ice) {
      const int4 bb = block_of_pair(a.bra + ib), kb = block_of_pair(a.ket + ic);
      const float *dm = a.blk_dmax_slot + k * a.blk_stride;
      const int n = a.nblk;
      const double dj = fmaxf(dm[bb.x * n + bb.y], dm[kb.x * n + kb.y]);
      const double dk = fmaxf(fmaxf(dm[bb.x * n + kb.x], dm[bb.x * n + kb.y]),
                              fmaxf(dm[bb.y * n + kb.x], dm[bb.y * n + kb.y]));
      if ((a.icedif & 1) && dj * aomax < a.ice_thr) js = 0.0;
      if ((a.icedif & 2) && dk * aomax < a.ice_thr) ks = 0.0;
    }
    if (a.jscale[k] != 0.0) {
      const bool jw = work && js != 0.0;
      // J_ab[x][y] = sum_cd g Ds_cd: group lanes warp-reduced (or held in
      // jacc), others per lane
      block_sums<FA * FB, FC * FD>(
          jw, g, [&](int o, int i) { return o * FC * FD + i; },
          [&](int i) { return __ldg(Dsk + (size_t)(kt.aoA + i / FD) * N + kt.aoB + i % FD); },
          [&](int o, double s) {
            const int x = o / FB, y = o % FB;
            s *= js;
            if constexpr (JN >= FA * FB) {
              if (jon) {
                if (grp) jacc[o] += s;
                else if (work && s != 0.0) atomicAdd(Fk + (size_t)(br.aoA + a_off + x) * N + br.aoB + y, s);
                return;
              }
            }
            double r = grp ? s : 0.0;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) r += __shfl_xor_sync(full, r, off);
            if (lane == 0 && r != 0.0) atomicAdd(Fg + (size_t)(brg.aoA + a_off + x) * brg.nbfm + brg.aoB + y, r);
            if (work && !grp && s != 0.0) atomicAdd(Fk + (size_t)(br.aoA + a_off + x) * N + br.aoB + y, s);
          });
      // J_cd[c][d] = sum_ab g Ds_ab: per lane
      block_sums<FC * FD, FA * FB>(
          jw, g, [&](int o, int i) { return i * FC * FD + o; },
          [&](int i) { return __ldg(Dsk + (size_t)(br.aoA + a_off + i / FB) * N + br.aoB + i % FB); },
          [&](int o, double s) {
            if (jw) atomicAdd(Fk + (size_t)(kt.aoA + o / FD) * N + kt.aoB + o % FD, js * s);
          });
    }
    if (a.kscale[k] != 0.0) {
      const bool kw = work && ks != 0.0;
      // K_ac[x][c] = sum_yd g D_bd: runs of equal C reduced, the run's head adds
      block_sums<FA * FC, FB * FD>(
          kw, g, [&](int o, int i) { return (((o / FC) * FB + i / FD) * FC + o % FC) * FD + i % FD; },
          [&](int i) { return dB(i / FD, kt.aoB + i % FD); },
          [&](int o, double s) {
            const int x = o / FC, c = o % FC;
            s *= ks;
            if (SEG && tseg) {
              sbuf[o * kSegStride + lane] = grp ? s : 0.0;
              if (kw && !grp) atomicAdd(Fk + (size_t)(br.aoA + a_off + x) * N + kt.aoA + c, s);
            } else if (SEG) {
              const double r = seg_sum(grp ? s : 0.0, lane, send);
              if (grp && head && r != 0.0) atomicAdd(Fk + (size_t)(br.aoA + a_off + x) * N + kt.aoA + c, r);
              if (kw && !grp) atomicAdd(Fk + (size_t)(br.aoA + a_off + x) * N + kt.aoA + c, s);
            } else if (kw) {
              atomicAdd(Fk + (size_t)(br.aoA + a_off + x) * N + kt.aoA + c, s);
            }
          });
      // K_ad[x][d] = sum_yc g D_bc: per lane
      block_sums<FA * FD, FB * FC>(
          kw, g, [&](int o, int i) { return (((o / FD) * FB + i / FC) * FC + i % FC) * FD + o % FD; },
          [&](int i) { return dB(i / FC, kt.aoA + i % FC); },
          [&](int o, double s) {
            if (kw) atomicAdd(Fk + (size_t)(br.aoA + a_off + o / FD) * N + kt.aoB + o % FD, ks * s);
          });
      // K_bc[y][c] = sum_xd g D_ad: runs of equal C reduced
      block_sums<FB * FC, FA * FD>(
          kw, g, [&](int o, int i) { return (((i / FD) * FB + o / FC) * FC + o % FC) * FD + i % FD; },
          [&](int i) { return dA(i / FD, kt.aoB + i % FD); },
          [&](int o, double s) {
            const int y = o / FC, c = o % FC;
            s *= ks;
            if (SEG && tseg) {
              sbuf[(FA * FC + o) * kSegStride + lane] = grp ? s : 0.0;
              if (kw && !grp) atomicAdd(Fk + (size_t)(br.aoB + y) * N + kt.aoA + c, s);
            } else if (SEG) {
              const double r = seg_sum(grp ? s : 0.0, lane, send);
              if (grp && head && r != 0.0) atomicAdd(Fk + (size_t)(br.aoB + y) * N + kt.aoA + c, r);
              if (kw && !grp) atomicAdd(Fk + (size_t)(br.aoB + y) * N + kt.aoA + c, s);
            } else if (kw) {
              atomicAdd(Fk + (size_t)(br.aoB + y) * N + kt.aoA + c, s);
            }
          });
      // K_bd[y][d] = sum_xc g D_ac: per lane
      block_sums<FB * FD, FA * FC>(
          kw, g, [&](int o, int i) { return (((i / FC) * FB + o / FD) * FC + i % FC) * FD + o % FD; },
          [&](int i) { return dA(i / FC, kt.aoA + i % FC); },
          [&](int o, double s) {
            if (kw) atomicAdd(Fk + (size_t)(br.aoB + o / FD) * N + kt.aoB + o % FD, ks * s);
          });
      if (SEG && tseg) seg_rows<FA, FC, NV>(sbuf, grp, grp ? kt.aoA : 0, send, Fg, brg, a_off);
    }
  }
}

// J_ab of bra pair jb held in the lanes' registers (slot 0, rows from
// a_off): summed across the warp and added by lane 0, then cleared.  Called
// by the whole warp.
template <int FA, int FB, int JN>
__device__ __forceinline__ void jk_jab_flush(const JKArgs &a, int jb, int a_off, double (&jacc)[JN]) {
  if (jb < 0) return;
  const PairRec bj = load_pair_fock(a.bra + jb);
  double *F = a.Fh + bj.dbase;
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int x = 0; x < FA; ++x)
#pragma unroll
    for (int y = 0; y < FB; ++y) {
      double r = jacc[x * FB + y];
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) r += __shfl_xor_sync(0xffffffffu, r, off);
      if (lane == 0 && r != 0.0) atomicAdd(F + (size_t)(bj.aoA + a_off + x) * bj.nbfm + bj.aoB + y, r);
      jacc[x * FB + y] = 0.0;
    }
}

constexpr int kThreadBlock = 256;
constexpr int kThreadWarps = kThreadBlock / 32;

template <int LA, int LB, int LC, int LD, typename Tc, int CA, int CH, int K1>
__device__ __forceinline__ void jk_thread_body(const JKArgs &a, const double *tab, Tc *ebra, double *sbuf,
                                               double *bsh, unsigned long long &cnt_q, unsigned long long &cnt_p,
                                               unsigned long long &cnt_s) {
  constexpr int L = LA + LB + LC + LD, LAB = LA + LB, LCD = LC + LD;
  constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  constexpr int A0 = CH * NA / CA, A1 = (CH + 1) * NA / CA, NAc = A1 - A0;  // this chunk's A components
  constexpr int NCD = NC * ND, NACC = NAc * NB * NCD;
  constexpr int N3L = n3(L);
  constexpr int EA = (LA + 1) * (LB + 1) * (LAB + 1), EC = (LC + 1) * (LD + 1) * (LCD + 1);
  constexpr bool SPH_NEEDED = (LA >= 2 || LB >= 2 || LC >= 2 || LD >= 2);
  constexpr int FAc = (LA >= 2) ? 2 * LA + 1 : NA, FBc = (LB >= 2) ? 2 * LB + 1 : NB;
  constexpr int FCc = (LC >= 2) ? 2 * LC + 1 : NC, FDc = (LD >= 2) ? 2 * LD + 1 : ND;
  // Buffer for the transformed chunk: spherical A (all m, partial sums) x B x C x D.
  constexpr int NOUT = cmax(NACC, cmax(FAc, NAc) * cmax(NB, FBc) * cmax(NC, FCc) * cmax(ND, FDc));
  const int lane = threadIdx.x & 31;
  const unsigned full = 0xffffffffu;
  // Each block takes one contiguous range of the queue and its warps work
  // on consecutive 32-quartet chunks of it, so that they usually share the
  // bra pair; a warp's chunks only move forward, so its bra index is found
  // once by binary search and then by a short walk along qoff.
  const int nw = blockDim.x >> 5, warp = threadIdx.x >> 5;
  const int64_t nq = a.nquartet - a.q_begin;
  const int64_t bspan = ((nq + gridDim.x - 1) / gridDim.x + 31) & ~(int64_t)31;
  const int64_t bbegin = a.q_begin + (int64_t)blockIdx.x * bspan, bend = min(bbegin + bspan, a.nquartet);
  int ibw = -1;  // the warp's running bra
  // J_ab of the warp's running bra accumulates in registers across its
  // chunks (s and p bras, one density slot); one warp reduction per bra run.
  constexpr bool JACC = !SPH_NEEDED && NAc * NB <= 9;
  constexpr int JN = JACC ? NAc * NB : 1;
  const bool jon = JACC && a.nslot == 1 && a.store_out == nullptr;
  double jacc[JN];
#pragma unroll
  for (int e = 0; e < JN; ++e) jacc[e] = 0.0;
  int jbra = -1;
  int cbra = -1;  // single-primitive bra whose data and tables bsh / ebra hold
  for (int64_t base = bbegin + (int64_t)warp * 32; base < bend; base += (int64_t)nw * 32) {
    const int64_t q = base + lane;
    const bool active = q < bend;
    int ib0 = ibw;
    if (lane == 0) {  // the warp's first bra: a short walk, else a search
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
    PrimPair P2one;  // K1: the ket's only primitive pair, fetched before the bra work
    if (active) {
      int steps = 0;
      while (q >= a.qoff[ib + 1] && steps < 32) {
        ++ib;
        ++steps;
      }
      if (q >= a.qoff[ib + 1]) ib = find_bra(a.qoff, a.nbra, q);
      ic = (int)(q - a.qoff[ib]) + (a.kbase ? a.kbase[ib] : 0);
      br = load_pair_fock(a.bra + ib);
      if (K1 && a.ks_i) {
        // single-primitive kets from the ket table: whole coalesced fields
        const int g = a.ks_base + ic;
        const int4 ki = __ldg(a.ks_i + g);
        kt.aoA = ki.x;
        kt.aoB = ki.y;
        kt.same = ki.z;
        kt.shA = ki.w >> 16;
        kt.shB = ki.w & 0xffff;
        kt.pp0 = 0;
        kt.npp = 1;
        kt.nbfm = a.nbf;
        kt.dbase = 0;
        kt.Q = __ldg(a.ks_q + g);
        const double *pl = a.ks_pp + g;
        const int64_t S = a.ks_stride;
        P2one.p = __ldg(pl);
        P2one.Px = __ldg(pl + S);
        P2one.Py = __ldg(pl + 2 * S);
        P2one.Pz = __ldg(pl + 3 * S);
        P2one.K = __ldg(pl + 4 * S);
        P2one.ea = 0.0;
        if (LC + LD > 0) {
          P2one.PAx = __ldg(pl + 5 * S);
          P2one.PAy = __ldg(pl + 6 * S);
          P2one.PAz = __ldg(pl + 7 * S);
          P2one.PBx = __ldg(pl + 8 * S);
          P2one.PBy = __ldg(pl + 9 * S);
          P2one.PBz = __ldg(pl + 10 * S);
        } else {
          P2one.PAx = P2one.PAy = P2one.PAz = P2one.PBx = P2one.PBy = P2one.PBz = 0.0;
        }
      } else {
        kt = load_pair_fock(a.ket + ic);
        // K1 with a known layout: the ket's primitive pair is fetched alongside its record
        if (K1 && a.ket_pp0 >= 0) P2one = load_prim<(LC + LD > 0)>(a.pp + a.ket_pp0 + ic);
      }
      sel = quartet_select(a, br, kt, a.bra + ib, a.ket + ic);
      if (sel == 2 && CH == 0 && a.mode != 2) ++cnt_s;  // a split class counts its skips in the FP64 launch
    }
    const bool work = active && sel == 0;
    Tc acc[NACC];
#pragma unroll
    for (int k = 0; k < NACC; ++k) acc[k] = Tc(0);
    if (K1 && work && !a.ks_i && a.ket_pp0 < 0) P2one = load_prim<(LC + LD > 0)>(a.pp + kt.pp0);
    // Bra groups: lanes sharing a bra pair run its primitive loop together.
    unsigned pending = __ballot_sync(full, work);
    while (pending) {
      const int leader = __ffs(pending) - 1;
      const int ibl = __shfl_sync(full, ib, leader);
      const bool mine = work && ib == ibl && ((pending >> lane) & 1u);
      pending &= ~__ballot_sync(full, mine);
      // The single-primitive bra the warp met last keeps its primitive data
      // (p, P, K) and Hermite tables in the warp's shared memory, so a run of
      // chunks on one bra loads and tabulates it once.
      const bool cached = (ibl == cbra);
      int npp = 1, pp0 = 0;
      if (!cached) {
        const PairRec brl = load_pair_fock(a.bra + ibl);
        npp = brl.npp;
        pp0 = brl.pp0;
      }
      for (int i = 0; i < npp; ++i) {
        PrimPair P1;
        if (!cached) {
          P1 = load_prim<true>(a.pp + pp0 + i);
          __syncwarp();
          if (lane < 3) {
            const Tc h1 = Tc(0.5 / P1.p);
            const double pa = lane == 0 ? P1.PAx : lane == 1 ? P1.PAy : P1.PAz;
            const double pb = lane == 0 ? P1.PBx : lane == 1 ? P1.PBy : P1.PBz;
            herm_e<LA, LB, 1, Tc>(h1, Tc(pa), Tc(pb), ebra + lane * EA);
          }
          if (lane == 0) {
            bsh[0] = P1.p;
            bsh[1] = P1.Px;
            bsh[2] = P1.Py;
            bsh[3] = P1.Pz;
            bsh[4] = P1.K;
          }
          __syncwarp();
        } else {
          P1.p = bsh[0];
          P1.Px = bsh[1];
          P1.Py = bsh[2];
          P1.Pz = bsh[3];
          P1.K = bsh[4];
        }
        if (!mine) continue;
        const Tc *ex1 = ebra, *ey1 = ebra + EA, *ez1 = ebra + 2 * EA;
        // One ket primitive pair (a zero K makes it contribute nothing).
        auto ket_prim = [&](const PrimPair &P2) {
          // FP32 half: FP32 rsqrt for the prefactor and the low-degree FP64 Boys table
          const double rs = (sizeof(Tc) == 4) ? (double)rsqrtf((float)(P1.p + P2.p)) : rsqrt(P1.p + P2.p);
          double alpha = P1.p * P2.p * rs * rs;
          double s = P1.K * P2.K * rs;
          erf_attenuate(a.erf_mu2, alpha, s);
          const double x = P1.Px - P2.Px, y = P1.Py - P2.Py, z = P1.Pz - P2.Pz;
          double F[L + 1];
          boys_eval<L, (sizeof(Tc) == 4) ? kBoysDegLow : kBoysDeg>(alpha * (x * x + y * y + z * z), tab, F);
          Tc Fs[L + 1];
#pragma unroll
          for (int n = 0; n <= L; ++n) {
            Fs[n] = Tc(s * F[n]);
            s *= -2.0 * alpha;
          }
          Tc R[N3L];
          hermite_r_inplace<L, Tc>(Fs, Tc(x), Tc(y), Tc(z), R);
          Tc ex2[EC], ey2[EC], ez2[EC];
          const Tc h2 = Tc(0.5 / P2.p);
          herm_e<LC, LD, -1, Tc>(h2, Tc(P2.PAx), Tc(P2.PBx), ex2);
          herm_e<LC, LD, -1, Tc>(h2, Tc(P2.PAy), Tc(P2.PBy), ey2);
          herm_e<LC, LD, -1, Tc>(h2, Tc(P2.PAz), Tc(P2.PBz), ez2);
          // (ab|cd) += sum_tuv E^ab_tuv sum_tau E^cd_tau R_{t+tau}: ket first.
#pragma unroll
          for (int c = 0; c < NC; ++c)
#pragma unroll
            for (int d = 0; d < ND; ++d) {
              const int cx = cart_x(LC, c), cy = cart_y(LC, c), cz = cart_z(LC, c);
              const int dx = cart_x(LD, d), dy = cart_y(LD, d), dz = cart_z(LD, d);
              Tc xk[n3(LAB)];
#pragma unroll
              for (int e = 0; e < n3(LAB); ++e) xk[e] = Tc(0);
#pragma unroll
              for (int ta = 0; ta <= cx + dx; ++ta)
#pragma unroll
                for (int na = 0; na <= cy + dy; ++na)
#pragma unroll
                  for (int fa = 0; fa <= cz + dz; ++fa) {
                    const Tc e3 = ex2[(cx * (LD + 1) + dx) * (LCD + 1) + ta] *
                                  ey2[(cy * (LD + 1) + dy) * (LCD + 1) + na] *
                                  ez2[(cz * (LD + 1) + dz) * (LCD + 1) + fa];
#pragma unroll
                    for (int t = 0; t <= LAB; ++t)
#pragma unroll
                      for (int u = 0; u <= LAB - t; ++u)
#pragma unroll
                        for (int v = 0; v <= LAB - t - u; ++v)
                          xk[tuv_index(t, u, v)] += e3 * R[tuv_index(t + ta, u + na, v + fa)];
                  }
#pragma unroll
              for (int ia = A0; ia < A1; ++ia)
#pragma unroll
                for (int jb = 0; jb < NB; ++jb) {
                  const int ax = cart_x(LA, ia), ay = cart_y(LA, ia), az = cart_z(LA, ia);
                  const int bx = cart_x(LB, jb), by = cart_y(LB, jb), bz = cart_z(LB, jb);
                  Tc sum = Tc(0);
#pragma unroll
                  for (int t = 0; t <= ax + bx; ++t)
#pragma unroll
                    for (int u = 0; u <= ay + by; ++u) {
                      const Tc exy = ex1[(ax * (LB + 1) + bx) * (LAB + 1) + t] * ey1[(ay * (LB + 1) + by) * (LAB + 1) + u];
#pragma unroll
                      for (int v = 0; v <= az + bz; ++v)
                        sum += exy * ez1[(az * (LB + 1) + bz) * (LAB + 1) + v] * xk[tuv_index(t, u, v)];
                    }
                  acc[((ia - A0) * NB + jb) * NCD + c * ND + d] += sum;
                }
            }
        };
        if constexpr (K1 != 0) {
          ket_prim(P2one);  // kets of this launch have one primitive pair each
        } else if constexpr (L <= 2) {
          // two independent primitive quartets per iteration for latency hiding
          int j = 0;
          for (; j + 1 < kt.npp; j += 2) {
            const PrimPair P2a = load_prim<(LC + LD > 0)>(a.pp + kt.pp0 + j);
            const PrimPair P2b = load_prim<(LC + LD > 0)>(a.pp + kt.pp0 + j + 1);
            ket_prim(P2a);
            ket_prim(P2b);
          }
          if (j < kt.npp) ket_prim(load_prim<(LC + LD > 0)>(a.pp + kt.pp0 + j));
        } else {
          PrimPair nxt = load_prim<(LC + LD > 0)>(a.pp + kt.pp0);
          for (int j = 0; j < kt.npp; ++j) {
            const PrimPair P2 = nxt;  // the next ket primitive pair is fetched during this one's arithmetic
            if (j + 1 < kt.npp) nxt = load_prim<(LC + LD > 0)>(a.pp + kt.pp0 + j + 1);
            ket_prim(P2);
          }
        }
      }
      cbra = (npp == 1) ? ibl : -1;
    }
    if (work) {
      cnt_q += (CH == 0);
      if (CH == 0) cnt_p += (unsigned long long)br.npp * kt.npp;
    }
    // Chunk block -> the shells' functions: spherical A (partial sums over
    // this chunk's Cartesian components), then B, C, D.
    const bool sphr = SPH_NEEDED && a.spherical;
    double g[NOUT];
#pragma unroll
    for (int k = 0; k < NOUT; ++k) g[k] = 0.0;
#pragma unroll
    for (int k = 0; k < NACC; ++k) g[k] = (double)acc[k];
    if (SPH_NEEDED && sphr && work) {
      // index by index with compile-time coefficients (SPHCO1 convention)
      double tmp[NOUT];
      if constexpr (LA >= 2) {
        sph_index<LA, 1, NAc, A0, NB * NCD>(g, tmp);
#pragma unroll
        for (int k = 0; k < FAc * NB * NCD; ++k) g[k] = tmp[k];
      }
      constexpr int A1r = (LA >= 2) ? FAc : NAc;
      if constexpr (LB >= 2) {
        sph_index<LB, A1r, NB, 0, NCD>(g, tmp);
#pragma unroll
        for (int k = 0; k < A1r * FBc * NCD; ++k) g[k] = tmp[k];
      }
      constexpr int AB1 = A1r * ((LB >= 2) ? FBc : NB);
      if constexpr (LC >= 2) {
        sph_index<LC, AB1, NC, 0, ND>(g, tmp);
#pragma unroll
        for (int k = 0; k < AB1 * FCc * ND; ++k) g[k] = tmp[k];
      }
      constexpr int ABC1 = AB1 * ((LC >= 2) ? FCc : NC);
      if constexpr (LD >= 2) {
        sph_index<LD, ABC1, ND, 0, 1>(g, tmp);
#pragma unroll
        for (int k = 0; k < ABC1 * FDc; ++k) g[k] = tmp[k];
      }
    }
    // Conventional form: the block goes to the store (the host launches only
    // one-chunk variants here, so g holds the whole block).
    if (a.store_out) {
      if (work) {
        double *o = a.store_out + a.store_base + q * a.store_nint;
        if (sphr) {
#pragma unroll
          for (int k = 0; k < FAc * FBc * FCc * FDc; ++k) o[k] = g[k];
        } else {
#pragma unroll
          for (int k = 0; k < NACC; ++k) o[k] = g[k];
        }
      }
      continue;
    }
    // Digestion with compile-time function counts (spherical or Cartesian).
    if (!__any_sync(full, work)) continue;
    if (JACC && jon && ib0 != jbra) {
      jk_jab_flush<NAc, NB, JN>(a, jbra, A0, jacc);
      jbra = ib0;
    }
    if (sphr)
      jk_digest<FAc, FBc, FCc, FDc, JN>(a, g, work, ib, ic, ib0, br, kt, 0, jacc, false, sbuf);
    else
      jk_digest<NAc, NB, NC, ND, JN>(a, g, work, ib, ic, ib0, br, kt, A0, jacc, jon, sbuf);
  }
  if (JACC && jon) jk_jab_flush<NAc, NB, JN>(a, jbra, A0, jacc);
}

template <int LA, int LB, int LC, int LD, typename Tc, int CA, int CH, int K1>
__device__ __forceinline__ void jk_thread_dispatch(int chunk, const JKArgs &a, const double *tab,
                                                   Tc *ebra, double *sbuf, double *bsh, unsigned long long &q,
                                                   unsigned long long &p, unsigned long long &s) {
  if constexpr (CH < CA) {
    if (chunk == CH)
      jk_thread_body<LA, LB, LC, LD, Tc, CA, CH, K1>(a, tab, ebra, sbuf, bsh, q, p, s);
    else
      jk_thread_dispatch<LA, LB, LC, LD, Tc, CA, CH + 1, K1>(chunk, a, tab, ebra, sbuf, bsh, q, p, s);
  }
}

// Rows of the shared-memory run buffer a class needs: the largest K_ac/K_bc
// value count in [max(kSegRowsMin, kSegMinValues), kSegMaxValues] over its A
// chunks, spherical and Cartesian (0: no run buffer).
template <int LA, int LB, int LC, int CA>
constexpr int seg_rows_needed() {
  constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC);
  constexpr int FB = LB >= 2 ? 2 * LB + 1 : NB, FC = LC >= 2 ? 2 * LC + 1 : NC;
  int best = 0;
  for (int ch = 0; ch < CA; ++ch) {
    const int nac = (ch + 1) * NA / CA - ch * NA / CA;
    const int fa = LA >= 2 ? 2 * LA + 1 : nac;
    const int nv[2] = {(nac + NB) * NC, (fa + FB) * FC};
    for (int v : nv)
      if (v >= kSegRowsMin && v >= kSegMinValues && v <= kSegMaxValues && v > best) best = v;
  }
  return best;
}

// Resident blocks per SM the register allocation must allow: the low-L
// classes are latency bound (few FLOPs per quartet, long chains of dependent
// loads), so they trade registers for warps.
#ifndef DGF_THREAD_MINB_L2
#define DGF_THREAD_MINB_L2 2
#endif
#ifndef DGF_THREAD_MINB_L3
#define DGF_THREAD_MINB_L3 1
#endif
constexpr int thread_min_blocks(int L) { return L <= 2 ? DGF_THREAD_MINB_L2 : L == 3 ? DGF_THREAD_MINB_L3 : 1; }

// K1 = 1: every ket pair of the launch has exactly one primitive pair (the
// first primitive-count bucket; all pairs of a basis whose general
// contractions are resolved into primitives), so the ket loop collapses.
template <int LA, int LB, int LC, int LD, typename Tc, int CA, int K1>
__global__ void __launch_bounds__(kThreadBlock, thread_min_blocks(LA + LB + LC + LD))
    jk_thread_kernel(const JKArgs a) {
  constexpr int EA = (LA + 1) * (LB + 1) * (LA + LB + 1);
  // The run buffer only where it fits the 48 KB of static shared memory
  // beside the Boys table and the bra tables, and only in classes that run
  // one block per SM: two blocks with the buffer would not fit the small
  // shared-memory carveout these kernels ask for (the rest of L1 caches the
  // density gathers), which would halve their resident warps.
  constexpr int SR0 = seg_rows_needed<LA, LB, LC, CA>();
  constexpr int kOtherSmem = kBoysTableDoubles * 8 + kThreadWarps * 3 * EA * (int)sizeof(Tc) + kThreadWarps * 64;
  constexpr int SR = (thread_min_blocks(LA + LB + LC + LD) == 1 &&
                      kOtherSmem + kThreadWarps * SR0 * kSegStride * 8 <= 48 * 1024 - 256)
                         ? SR0
                         : 0;
  __shared__ double tab[kBoysTableDoubles];
  __shared__ Tc ebra_all[kThreadWarps][3 * EA];
  __shared__ double bra_sh[kThreadWarps][8];
  __shared__ double segbuf[kThreadWarps][SR > 0 ? SR * kSegStride : 1];
  for (int i = threadIdx.x; i < kBoysTableDoubles; i += blockDim.x) tab[i] = a.boys[i];
  __syncthreads();
  unsigned long long cnt_q = 0, cnt_p = 0, cnt_s = 0;
  double *sbuf = SR > 0 ? segbuf[threadIdx.x >> 5] : nullptr;
  jk_thread_dispatch<LA, LB, LC, LD, Tc, CA, 0, K1>(blockIdx.y, a, tab, ebra_all[threadIdx.x >> 5], sbuf,
                                                bra_sh[threadIdx.x >> 5], cnt_q,
                                                cnt_p, cnt_s);
  if (a.counters) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      cnt_q += __shfl_xor_sync(0xffffffffu, cnt_q, off);
      cnt_p += __shfl_xor_sync(0xffffffffu, cnt_p, off);
      cnt_s += __shfl_xor_sync(0xffffffffu, cnt_s, off);
    }
    if (lane == 0) {
      atomicAdd(a.counters + 0, cnt_q);
      atomicAdd(a.counters + 1, cnt_p);
      atomicAdd(a.counters + 2, cnt_s);
      if (sizeof(Tc) == 4) atomicAdd(a.counters + 3, cnt_q);
    }
  }
}

}  // namespace dgf
