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
template <int FA, int FB, int FC, int FD>
__device__ __forceinline__ void jk_digest(const JKArgs &a, const double *g, bool work, int ib, int ic, int gib,
                                          const PairRec &br, const PairRec &kt, int a_off) {
  // Segmented reduction of K_ac and K_bc where it is cheap next to the atomics it saves.
  constexpr bool SEG = (FA + FB) * FC <= 18;
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
    // Rows of the bra's functions in D.
    auto dA = [&](int x, int col) -> double { return Dk[(size_t)(br.aoA + a_off + x) * N + col]; };
    auto dB = [&](int y, int col) -> double { return Dk[(size_t)(br.aoB + y) * N + col]; };
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
      // J_ab: group lanes warp-reduced, others per lane
#pragma unroll
      for (int x = 0; x < FA; ++x)
#pragma unroll
        for (int y = 0; y < FB; ++y) {
          double s = 0.0;
          if (work && js != 0.0) {
#pragma unroll
            for (int c = 0; c < FC; ++c)
#pragma unroll
              for (int d = 0; d < FD; ++d)
                s += g[((x * FB + y) * FC + c) * FD + d] * Dsk[(size_t)(kt.aoA + c) * N + kt.aoB + d];
            s *= js;
          }
          double r = grp ? s : 0.0;
#pragma unroll
          for (int off = 16; off > 0; off >>= 1) r += __shfl_xor_sync(full, r, off);
          if (lane == 0 && r != 0.0) atomicAdd(Fg + (size_t)(brg.aoA + a_off + x) * brg.nbfm + brg.aoB + y, r);
          if (work && !grp && s != 0.0) atomicAdd(Fk + (size_t)(br.aoA + a_off + x) * N + br.aoB + y, s);
        }
      // J_cd: per lane
      if (work && js != 0.0) {
#pragma unroll
        for (int c = 0; c < FC; ++c)
#pragma unroll
          for (int d = 0; d < FD; ++d) {
            double s = 0.0;
#pragma unroll
            for (int x = 0; x < FA; ++x)
#pragma unroll
              for (int y = 0; y < FB; ++y)
                s += g[((x * FB + y) * FC + c) * FD + d] * Dsk[(size_t)(br.aoA + a_off + x) * N + br.aoB + y];
            atomicAdd(Fk + (size_t)(kt.aoA + c) * N + kt.aoB + d, js * s);
          }
      }
    }
    if (a.kscale[k] != 0.0) {
      const bool kw = work && ks != 0.0;
#pragma unroll
      for (int x = 0; x < FA; ++x) {
        // K_ac: runs of equal C reduced, the run's head adds
#pragma unroll
        for (int c = 0; c < FC; ++c) {
          double s = 0.0;
          if (kw) {
#pragma unroll
            for (int y = 0; y < FB; ++y)
#pragma unroll
              for (int d = 0; d < FD; ++d) s += g[((x * FB + y) * FC + c) * FD + d] * dB(y, kt.aoB + d);
            s *= ks;
          }
          if (SEG) {
            const double r = seg_sum(grp ? s : 0.0, lane, send);
            if (grp && head && r != 0.0) atomicAdd(Fk + (size_t)(br.aoA + a_off + x) * N + kt.aoA + c, r);
            if (kw && !grp) atomicAdd(Fk + (size_t)(br.aoA + a_off + x) * N + kt.aoA + c, s);
          } else if (kw) {
            atomicAdd(Fk + (size_t)(br.aoA + a_off + x) * N + kt.aoA + c, s);
          }
        }
        // K_ad: per lane
#pragma unroll
        for (int d = 0; d < FD; ++d) {
          if (!kw) continue;
          double s = 0.0;
#pragma unroll
          for (int y = 0; y < FB; ++y)
#pragma unroll
            for (int c = 0; c < FC; ++c) s += g[((x * FB + y) * FC + c) * FD + d] * dB(y, kt.aoA + c);
          atomicAdd(Fk + (size_t)(br.aoA + a_off + x) * N + kt.aoB + d, ks * s);
        }
      }
#pragma unroll
      for (int y = 0; y < FB; ++y) {
        // K_bc: runs of equal C reduced
#pragma unroll
        for (int c = 0; c < FC; ++c) {
          double s = 0.0;
          if (kw) {
#pragma unroll
            for (int x = 0; x < FA; ++x)
#pragma unroll
              for (int d = 0; d < FD; ++d) s += g[((x * FB + y) * FC + c) * FD + d] * dA(x, kt.aoB + d);
            s *= ks;
          }
          if (SEG) {
            const double r = seg_sum(grp ? s : 0.0, lane, send);
            if (grp && head && r != 0.0) atomicAdd(Fk + (size_t)(br.aoB + y) * N + kt.aoA + c, r);
            if (kw && !grp) atomicAdd(Fk + (size_t)(br.aoB + y) * N + kt.aoA + c, s);
          } else if (kw) {
            atomicAdd(Fk + (size_t)(br.aoB + y) * N + kt.aoA + c, s);
          }
        }
        // K_bd: per lane
#pragma unroll
        for (int d = 0; d < FD; ++d) {
          if (!kw) continue;
          double s = 0.0;
#pragma unroll
          for (int x = 0; x < FA; ++x)
#pragma unroll
            for (int c = 0; c < FC; ++c) s += g[((x * FB + y) * FC + c) * FD + d] * dA(x, kt.aoA + c);
          atomicAdd(Fk + (size_t)(br.aoB + y) * N + kt.aoB + d, ks * s);
        }
      }
    }
  }
}

constexpr int kThreadBlock = 256;
constexpr int kThreadWarps = kThreadBlock / 32;

template <int LA, int LB, int LC, int LD, typename Tc, int CA, int CH, int K1>
__device__ __forceinline__ void jk_thread_body(const JKArgs &a, const double *tab, Tc *ebra,
                                               unsigned long long &cnt_q, unsigned long long &cnt_p,
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
      const PairRec brl = load_pair_fock(a.bra + ibl);
      for (int i = 0; i < brl.npp; ++i) {
        const PrimPair P1 = load_prim<true>(a.pp + brl.pp0 + i);
        __syncwarp();
        if (lane < 3) {
          const Tc h1 = Tc(0.5 / P1.p);
          const double pa = lane == 0 ? P1.PAx : lane == 1 ? P1.PAy : P1.PAz;
          const double pb = lane == 0 ? P1.PBx : lane == 1 ? P1.PBy : P1.PBz;
          herm_e<LA, LB, 1, Tc>(h1, Tc(pa), Tc(pb), ebra + lane * EA);
        }
        __syncwarp();
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
    if (sphr)
      jk_digest<FAc, FBc, FCc, FDc>(a, g, work, ib, ic, ib0, br, kt, 0);
    else
      jk_digest<NAc, NB, NC, ND>(a, g, work, ib, ic, ib0, br, kt, A0);
  }
}

template <int LA, int LB, int LC, int LD, typename Tc, int CA, int CH, int K1>
__device__ __forceinline__ void jk_thread_dispatch(int chunk, const JKArgs &a, const double *tab,
                                                   Tc *ebra, unsigned long long &q, unsigned long long &p,
                                                   unsigned long long &s) {
  if constexpr (CH < CA) {
    if (chunk == CH)
      jk_thread_body<LA, LB, LC, LD, Tc, CA, CH, K1>(a, tab, ebra, q, p, s);
    else
      jk_thread_dispatch<LA, LB, LC, LD, Tc, CA, CH + 1, K1>(chunk, a, tab, ebra, q, p, s);
  }
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
  __shared__ double tab[kBoysTableDoubles];
  __shared__ Tc ebra_all[kThreadWarps][3 * EA];
  for (int i = threadIdx.x; i < kBoysTableDoubles; i += blockDim.x) tab[i] = a.boys[i];
  __syncthreads();
  unsigned long long cnt_q = 0, cnt_p = 0, cnt_s = 0;
  jk_thread_dispatch<LA, LB, LC, LD, Tc, CA, 0, K1>(blockIdx.y, a, tab, ebra_all[threadIdx.x >> 5], cnt_q, cnt_p,
                                                cnt_s);
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
