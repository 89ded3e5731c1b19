// Warp-per-quartet McMurchie-Davidson J/K kernel for the high angular
// momentum classes (L = la+lb+lc+ld >= 6, up to (fd|fd); also a tuning
// candidate from L = 4), where one thread cannot hold a quartet's
// intermediates in registers.
//
// Each warp of a block works through its own contiguous range of the class
// queue, one quartet at a time; every index pattern is known at compile
// time and the lanes split the work of each step:
//   R_tuv            Hermite recursion level by level in a box in shared
//                    memory (strides chosen per class against bank
//                    conflicts), one (t,u,v) per lane        (HERI, her2her.F)
//   X[cd][tuv]       ket transform, one bra Hermite index tuv per lane: each
//                    R value is read once and applied to every ket
//                    component that uses it, with the ket's Hermite
//                    coefficient products E^cd_{tau nu phi} from a table
//                    built per ket primitive pair (one term per lane, from
//                    per-block index tables); components in register chunks
//                                                          (C2, her2el2.F)
//   (ab|cd)          bra transform, one ket component cd per lane, each X
//                    value read once and applied to every bra component,
//                    with the bra's product table (kept while consecutive
//                    quartets share the bra)               (C1, her2el1.F)
//   spherical        index by index in shared memory, one output element
//                    per lane                              (C1SPHR/C2SPHR)
//   digestion        the six J/K blocks (FCKCON, herfckcon.F:66-80), one
//                    output element per lane, FP64 atomics
// Contracted pairs: the bra primitives form the outer loop and the ket
// primitives the inner one; X sums over the ket primitives and, in the
// classes where a lane holds a whole ket component column (Shape::MP), each
// lane sums its column of the (ab|cd) block over the bra primitives in
// registers (HERMIT's primitive -> contracted step, her2el1.F/her2el2.F).
// Tc is the arithmetic type of R, the transforms and the tables (double:
// FP64 drop-in; float: FP32 half of the mixed form); Boys function,
// prefactor, accumulation across primitive pairs and digestion are FP64.
#pragma once

#include <utility>

#include "dgf_select.cuh"

namespace dgf {
namespace wq {

// (t,u,v) of compact index e (tuv_index order), at compile time.
constexpr int tuv_s(int e) {
  int s = 0;
  while (n3(s) <= e) ++s;
  return s;
}
constexpr int tuv_w(int e) {
  const int r = e - n3(tuv_s(e) - 1 >= 0 ? tuv_s(e) - 1 : 0) * (tuv_s(e) > 0 ? 1 : 0);
  int w = 0;
  while ((w + 1) * (w + 2) / 2 <= r) ++w;
  return w;
}
constexpr int tuv_v(int e) {
  const int r = e - (tuv_s(e) > 0 ? n3(tuv_s(e) - 1) : 0);
  return r - tuv_w(e) * (tuv_w(e) + 1) / 2;
}
constexpr int tuv_u(int e) { return tuv_w(e) - tuv_v(e); }
constexpr int tuv_t(int e) { return tuv_s(e) - tuv_w(e); }

// Hermite terms of Cartesian component pair ij = i*ncart(lb)+j of a shell
// pair (la, lb): (ix+jx+1)(iy+jy+1)(iz+jz+1), and their offsets in a
// compact table ordered by ij, then t, u, v.
constexpr int nterm(int la, int lb, int ij) {
  const int i = ij / ncart(lb), j = ij % ncart(lb);
  return (cart_x(la, i) + cart_x(lb, j) + 1) * (cart_y(la, i) + cart_y(lb, j) + 1) *
         (cart_z(la, i) + cart_z(lb, j) + 1);
}
constexpr int term_off(int la, int lb, int ij) {
  int off = 0;
  for (int k = 0; k < ij; ++k) off += nterm(la, lb, k);
  return off;
}
constexpr int nterm_all(int la, int lb) { return term_off(la, lb, ncart(la) * ncart(lb)); }
// Whether component pair ij uses Hermite index (t,u,v), and the term's index.
constexpr bool uses(int la, int lb, int ij, int t, int u, int v) {
  const int i = ij / ncart(lb), j = ij % ncart(lb);
  return t <= cart_x(la, i) + cart_x(lb, j) && u <= cart_y(la, i) + cart_y(lb, j) &&
         v <= cart_z(la, i) + cart_z(lb, j);
}
constexpr int term_at(int la, int lb, int ij, int t, int u, int v) {
  const int i = ij / ncart(lb), j = ij % ncart(lb);
  const int ny = cart_y(la, i) + cart_y(lb, j) + 1, nz = cart_z(la, i) + cart_z(lb, j) + 1;
  return term_off(la, lb, ij) + (t * ny + u) * nz + v;
}

constexpr int odd(int n) { return n | 1; }

// Components per register chunk of the transforms.
constexpr int kChunk = 36;
// Whether any component pair of [i0, i0+n) uses Hermite index (t,u,v).
constexpr bool chunk_uses(int la, int lb, int i0, int n, int t, int u, int v) {
  for (int ij = i0; ij < i0 + n; ++ij)
    if (uses(la, lb, ij, t, u, v)) return true;
  return false;
}

// One FP64 tensor-core step D(8x8) += A(8x4) B(4x8) (DMMA, mma.sync
// m8n8k4).  Fragments: lane l holds A[l/4][l%4], B[l%4][l/4] and
// D[l/4][2(l%4)], D[l/4][2(l%4)+1].
__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

using ::dgf::static_for;

// Layout of the R box: R_tuv at position SA t + SB u + v (t + u + v <= L).
// The lanes of the ket transform read R at (t,u,v) + (tau,nu,phi) for the
// bra Hermite indices, and the recursion writes one level at a time; the
// strides are chosen per class so that those reads (8-byte values, one
// 16-lane half of the warp per wavefront) fall in distinct banks as far as
// possible, without enlarging the box beyond (L+1)^3.
struct BoxStrides {
  int sa, sb;
};
// Wavefronts of the 16-lane halves reading the positions of Hermite indices
// 0 .. n3(m)-1 (tuv_index order).
constexpr int box_waves(int sa, int sb, int m) {
  int tot = 0, k = 0, mx = 0;
  int cnt[16] = {};
  for (int s = 0; s <= m; ++s)
    for (int t = s; t >= 0; --t)
      for (int u = s - t; u >= 0; --u) {
        const int b = (sa * t + sb * u + (s - t - u)) % 16;
        if (++cnt[b] > mx) mx = cnt[b];
        if (++k == 16) {
          tot += mx;
          k = mx = 0;
          for (int i = 0; i < 16; ++i) cnt[i] = 0;
        }
      }
  return tot + mx;
}
constexpr int box_cost(int sa, int sb, int L, int LAB, int LCD) {
  int c = n3(LCD) * box_waves(sa, sb, LAB);  // ket transform: one read per ket Hermite index
  for (int m = 1; m <= L; ++m) c += 3 * box_waves(sa, sb, m);  // recursion levels
  return c;
}
constexpr BoxStrides box_strides(int L, int LAB, int LCD) {
  const int box = L + 1;
  BoxStrides best{box * box, box};
  int bc = box_cost(best.sa, best.sb, L, LAB, LCD);
  for (int b = L + 1; b < L + 9; ++b)
    for (int a = L * b + 1; a < L * b + 25; ++a) {
      if (a * L + 1 > box * box * box) continue;
      const int c = box_cost(a, b, L, LAB, LCD);
      if (c < bc) {
        bc = c;
        best = BoxStrides{a, b};
      }
    }
  return best;
}

// Per-warp shared memory of class (LA LB | LC LD) in units of 8 bytes.
template <int LA, int LB, int LC, int LD, typename Tc>
struct Shape {
  static constexpr int L = LA + LB + LC + LD, LAB = LA + LB, LCD = LC + LD, BOX = L + 1;
  static constexpr BoxStrides BS = box_strides(L, LAB, LCD);
  static constexpr int SA = BS.sa, SB = BS.sb, RBOX = SA * L + 1;  // R box strides and size
  static constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  static constexpr int NAB = NA * NB, NCD = NC * ND, N3AB = n3(LAB), N3CD = n3(LCD), N3L = n3(L);
  static constexpr int EA = (LA + 1) * (LB + 1) * (LAB + 1), EC = (LC + 1) * (LD + 1) * (LCD + 1);
  static constexpr int TAB = nterm_all(LA, LB), TCD = nterm_all(LC, LD);
  static constexpr int PX = odd(N3AB);  // row stride of X[cd][tuv]
  static constexpr int PG = odd(NCD);   // row stride of the (ab|cd) blocks
  static constexpr int FAm = cmax(NA, LA >= 2 ? 2 * LA + 1 : NA), FBm = cmax(NB, LB >= 2 ? 2 * LB + 1 : NB);
  static constexpr int FCm = cmax(NC, LC >= 2 ? 2 * LC + 1 : NC), FDm = cmax(ND, LD >= 2 ? 2 * LD + 1 : ND);
  static constexpr int W = sizeof(Tc) == 8 ? 1 : 2;  // Tc values per 8-byte unit
  // region A: the two R boxes, later the Cartesian (ab|cd) block and the final block
  static constexpr int RA = cmax((2 * RBOX + W - 1) / W, NAB * PG);
  // region B: X, later the block with spherical bra functions
  static constexpr int RB = cmax((NCD * PX + W - 1) / W, NAB * PG);
  // Hermite 1D tables and product tables of bra and ket (Tc)
  static constexpr int RT = (3 * EA + 3 * EC + TAB + TCD + W - 1) / W;
  // six density blocks (double)
  static constexpr int RD = FAm * FBm + FCm * FDm + FAm * FCm + FAm * FDm + FBm * FCm + FBm * FDm;
  static constexpr int PER_WARP = RA + RB + RT + RD + 8;
  // block-wide: Boys and spherical tables, packed (t,u,v) positions, and the
  // index tables of the bra and ket product tables (ints)
  static constexpr int COMMON = kBoysTableDoubles + kSphTableDoubles + (N3L + TAB + TCD + NAB + NCD + 1) / 2;
  static constexpr size_t smem(int warps) { return ((size_t)COMMON + (size_t)warps * PER_WARP) * 8; }
  // warps per block: four when they fit in 100 KB, else two, else one
  static constexpr int WPB = smem(4) <= 100 * 1024 ? 4 : smem(2) <= 100 * 1024 ? 2 : 1;
  // Primitive loops on both sides: classes whose ket components fit one per
  // lane and whose bra components fit one register chunk, so that a lane
  // keeps its column of the (ab|cd) block in registers across the bra
  // primitives.  Other classes take one primitive pair per side.
  static constexpr bool MP = NCD <= 32 && NAB <= wq::kChunk;
  // spherical function counts; SPHR: the MP form applies the spherical
  // transforms in registers (ket side in the ket transform, bra side when
  // the block leaves the accumulators)
  static constexpr int FA = LA >= 2 ? 2 * LA + 1 : NA, FB = LB >= 2 ? 2 * LB + 1 : NB;
  static constexpr int FC = LC >= 2 ? 2 * LC + 1 : NC, FD = LD >= 2 ? 2 * LD + 1 : ND;
  static constexpr int FAB = FA * FB, FCD = FC * FD;
  static constexpr bool SPHR = MP && (LA >= 2 || LB >= 2 || LC >= 2 || LD >= 2);
  // Tensor-core form (FP64 only): both transforms as DMMA products of dense
  // tiles, the (ab|cd) block in D fragments across the bra primitives.
  static constexpr int MT2 = (N3AB + 7) / 8, KT2 = (N3CD + 3) / 4;  // ket product: rows e, depth f
  static constexpr int MT3 = (NAB + 7) / 8, NT = (NCD + 7) / 8, KT3 = (N3AB + 3) / 4;
  static constexpr bool MMA_OK = sizeof(Tc) == 8 && MT3 * NT * 2 <= 64;
};

// One index of the Cartesian -> spherical transform of a block in shared
// memory (rows ab = a*NB+b, columns cd = c*ND+d, row stride PG), lane-
// parallel over the output elements; T is the M x N table of the index.
// IDX 0: a (rows), 1: b (rows), 2: c (columns), 3: d (columns); NB1/ND1 are
// the current sizes of the b and d indices, NA1/NC1 of a and c.
template <int IDX, int N, int M, int NA1, int NB1, int NC1, int ND1, int PG>
__device__ __forceinline__ void sph_pass(const double *in, double *out, const double *T, int lane) {
  constexpr int NR = (IDX == 0 ? M : NA1) * (IDX == 1 ? M : NB1);  // output rows
  constexpr int NCOL = (IDX == 2 ? M : NC1) * (IDX == 3 ? M : ND1);  // output columns
  for (int e = lane; e < NR * NCOL; e += 32) {
    const int r = e / NCOL, col = e - r * NCOL;
    double s = 0.0;
    if (IDX == 0) {
      const int m = r / NB1, b = r - m * NB1;
#pragma unroll
      for (int n = 0; n < N; ++n) s += T[m * N + n] * in[(n * NB1 + b) * PG + col];
    } else if (IDX == 1) {
      const int a = r / M, m = r - a * M;
#pragma unroll
      for (int n = 0; n < N; ++n) s += T[m * N + n] * in[(a * NB1 + n) * PG + col];
    } else if (IDX == 2) {
      const int m = col / ND1, d = col - m * ND1;
#pragma unroll
      for (int n = 0; n < N; ++n) s += T[m * N + n] * in[r * PG + n * ND1 + d];
    } else {
      const int c = col / M, m = col - c * M;
#pragma unroll
      for (int n = 0; n < N; ++n) s += T[m * N + n] * in[r * PG + c * ND1 + n];
    }
    out[r * PG + col] = s;
  }
}

}  // namespace wq

// Post-processing and digestion of the block Gc[ab][cd] (row stride PG) of
// one quartet: spherical transform (SPH, index by index between Gc and the
// scratch block Gs; PRE: the block is spherical already), then the six J/K
// blocks; Db holds the density blocks.
template <int LA, int LB, int LC, int LD, typename Tc, bool SPH, bool PRE = false>
__device__ __forceinline__ void wq_finish(const JKArgs &a, double *Gc, double *Gs, double *Db,
                                          const double *sph, const PairRec &br, const PairRec &kt, int ib, int ic,
                                          double w, int lane, int64_t q) {
  using S = wq::Shape<LA, LB, LC, LD, Tc>;
  constexpr int NA = S::NA, NB = S::NB, NC = S::NC, ND = S::ND, PG = S::PG;
  constexpr int FA = (SPH && LA >= 2) ? 2 * LA + 1 : NA, FB = (SPH && LB >= 2) ? 2 * LB + 1 : NB;
  constexpr int FC = (SPH && LC >= 2) ? 2 * LC + 1 : NC, FD = (SPH && LD >= 2) ? 2 * LD + 1 : ND;
  constexpr int FAB = FA * FB, FCD = FC * FD;
  const double *G = Gc;
  if (SPH && !PRE) {
    // index by index, ping-pong between Gc and Gs
    constexpr int FA1 = LA >= 2 ? 2 * LA + 1 : NA, FB1 = LB >= 2 ? 2 * LB + 1 : NB;
    constexpr int FC1 = LC >= 2 ? 2 * LC + 1 : NC;
    double *src = Gc, *dst = Gs;
    if constexpr (LA >= 2) {
      wq::sph_pass<0, NA, FA1, NA, NB, NC, ND, PG>(src, dst, sph + sph_offset(LA), lane);
      __syncwarp();
      double *t = src; src = dst; dst = t;
    }
    if constexpr (LB >= 2) {
      wq::sph_pass<1, NB, FB1, FA1, NB, NC, ND, PG>(src, dst, sph + sph_offset(LB), lane);
      __syncwarp();
      double *t = src; src = dst; dst = t;
    }
    if constexpr (LC >= 2) {
      wq::sph_pass<2, NC, FC1, FA1, FB1, NC, ND, PG>(src, dst, sph + sph_offset(LC), lane);
      __syncwarp();
      double *t = src; src = dst; dst = t;
    }
    if constexpr (LD >= 2) {
      wq::sph_pass<3, ND, 2 * LD + 1, FA1, FB1, FC1, ND, PG>(src, dst, sph + sph_offset(LD), lane);
      __syncwarp();
      double *t = src; src = dst; dst = t;
    }
    G = src;
  }
  if (a.store_out) {  // conventional form: the block to the store
    double *o = a.store_out + a.store_base + q * a.store_nint;
    for (int e = lane; e < FAB * FCD; e += 32) o[e] = G[(e / FCD) * PG + e % FCD];
    return;
  }
  // Largest integral for the per-density Coulomb/exchange screen (ICEDIF).
  bool ice = false;
  double aomax = 0.0;
  if (a.ice_thr > 0.0) {
    const int4 bb = block_of_pair(a.bra + ib), kb = block_of_pair(a.ket + ic);
    ice = (bb.z & bb.w & kb.z & kb.w) != 0;
    if (ice) {
      for (int e = lane; e < FAB * FCD; e += 32) aomax = fmax(aomax, fabs(G[(e / FCD) * PG + e % FCD]));
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) aomax = fmax(aomax, __shfl_xor_sync(0xffffffffu, aomax, off));
    }
  }
  const int aoA = br.aoA, aoB = br.aoB, aoC = kt.aoA, aoD = kt.aoB;
  const int N = kt.nbfm;
  double *Dab = Db, *Dcd = Dab + FAB, *Dac = Dcd + FCD, *Dad = Dac + FA * FC, *Dbc = Dad + FA * FD,
         *Dbd = Dbc + FB * FC;
  for (int k = 0; k < a.nslot; ++k) {
    const double *Dk = a.D + k * a.slot_stride + kt.dbase;
    const double *Dsk = a.Ds + k * a.slot_stride + kt.dbase;
    double *Fk = a.Fh + k * a.slot_stride + kt.dbase;
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
    if (js == 0.0 && ks == 0.0) continue;
    // density blocks
    for (int e = lane; e < FAB; e += 32) Dab[e] = Dsk[(size_t)(aoA + e / FB) * N + aoB + e % FB];
    for (int e = lane; e < FCD; e += 32) Dcd[e] = Dsk[(size_t)(aoC + e / FD) * N + aoD + e % FD];
    for (int e = lane; e < FA * FC; e += 32) Dac[e] = Dk[(size_t)(aoA + e / FC) * N + aoC + e % FC];
    for (int e = lane; e < FA * FD; e += 32) Dad[e] = Dk[(size_t)(aoA + e / FD) * N + aoD + e % FD];
    for (int e = lane; e < FB * FC; e += 32) Dbc[e] = Dk[(size_t)(aoB + e / FC) * N + aoC + e % FC];
    for (int e = lane; e < FB * FD; e += 32) Dbd[e] = Dk[(size_t)(aoB + e / FD) * N + aoD + e % FD];
    __syncwarp();
    if (js != 0.0) {
      for (int e = lane; e < FAB; e += 32) {  // J_ab
        const double *row = G + e * PG;
        double s = 0.0;
#pragma unroll
        for (int cd = 0; cd < FCD; ++cd) s += row[cd] * Dcd[cd];
        atomicAdd(Fk + (size_t)(aoA + e / FB) * N + aoB + e % FB, js * s);
      }
      for (int e = lane; e < FCD; e += 32) {  // J_cd
        double s = 0.0;
#pragma unroll
        for (int ab = 0; ab < FAB; ++ab) s += G[ab * PG + e] * Dab[ab];
        atomicAdd(Fk + (size_t)(aoC + e / FD) * N + aoD + e % FD, js * s);
      }
    }
    if (ks != 0.0) {
      for (int e = lane; e < FA * FC; e += 32) {  // K_ac = sum_bd g D_bd
        const int x = e / FC, c = e % FC;
        double s = 0.0;
#pragma unroll
        for (int y = 0; y < FB; ++y)
#pragma unroll
          for (int d = 0; d < FD; ++d) s += G[(x * FB + y) * PG + c * FD + d] * Dbd[y * FD + d];
        atomicAdd(Fk + (size_t)(aoA + x) * N + aoC + c, ks * s);
      }
      for (int e = lane; e < FA * FD; e += 32) {  // K_ad = sum_bc g D_bc
        const int x = e / FD, d = e % FD;
        double s = 0.0;
#pragma unroll
        for (int y = 0; y < FB; ++y)
#pragma unroll
          for (int c = 0; c < FC; ++c) s += G[(x * FB + y) * PG + c * FD + d] * Dbc[y * FC + c];
        atomicAdd(Fk + (size_t)(aoA + x) * N + aoD + d, ks * s);
      }
      for (int e = lane; e < FB * FC; e += 32) {  // K_bc = sum_ad g D_ad
        const int y = e / FC, c = e % FC;
        double s = 0.0;
#pragma unroll
        for (int x = 0; x < FA; ++x)
#pragma unroll
          for (int d = 0; d < FD; ++d) s += G[(x * FB + y) * PG + c * FD + d] * Dad[x * FD + d];
        atomicAdd(Fk + (size_t)(aoB + y) * N + aoC + c, ks * s);
      }
      for (int e = lane; e < FB * FD; e += 32) {  // K_bd = sum_ac g D_ac
        const int y = e / FD, d = e % FD;
        double s = 0.0;
#pragma unroll
        for (int x = 0; x < FA; ++x)
#pragma unroll
          for (int c = 0; c < FC; ++c) s += G[(x * FB + y) * PG + c * FD + d] * Dac[x * FC + c];
        atomicAdd(Fk + (size_t)(aoB + y) * N + aoD + d, ks * s);
      }
    }
    __syncwarp();
  }
}

// Index table of the compact Hermite product table of a shell pair
// (la, lb), built once per block: for term k (ordered by component pair ij,
// then t, u, v as in wq::term_at), the positions of its three factors in the
// 1D tables E (x: ix,jx,t; y; z), packed 10 bits each.
template <int LA, int LB>
__device__ __forceinline__ void wq_term_index(int *idx, int tid, int nt) {
  constexpr int NB = ncart(LB), NIJ = ncart(LA) * NB, LT = LA + LB + 1, EN = (LA + 1) * (LB + 1) * LT;
  for (int ij = tid; ij < NIJ; ij += nt) {
    int ix, iy, iz, jx, jy, jz, off = 0;
    cart_decode(LA, ij / NB, ix, iy, iz);
    cart_decode(LB, ij % NB, jx, jy, jz);
    for (int k = 0; k < ij; ++k) {
      int ax, ay, az, bx, by, bz;
      cart_decode(LA, k / NB, ax, ay, az);
      cart_decode(LB, k % NB, bx, by, bz);
      off += (ax + bx + 1) * (ay + by + 1) * (az + bz + 1);
    }
    const int bxp = (ix * (LB + 1) + jx) * LT, byp = EN + (iy * (LB + 1) + jy) * LT,
              bzp = 2 * EN + (iz * (LB + 1) + jz) * LT;
    for (int t = 0; t <= ix + jx; ++t)
      for (int u = 0; u <= iy + jy; ++u)
        for (int v = 0; v <= iz + jz; ++v) idx[off++] = (bxp + t) | ((byp + u) << 10) | ((bzp + v) << 20);
  }
}

// Compact table of Hermite coefficient products of a shell pair:
// tab[k] = E_x E_y E_z of term k, from the 1D tables E and the index table;
// one term per lane and round.
template <int NT, typename Tc>
__device__ __forceinline__ void wq_product_table(const Tc *E, const int *idx, Tc *tab, int lane) {
  for (int k = lane; k < NT; k += 32) {
    const int p = idx[k];
    tab[k] = E[p & 1023] * E[(p >> 10) & 1023] * E[p >> 20];
  }
}

// Packed positions of the three factors of Cartesian component pair ij
// (i of la, j of lb) in the 1D Hermite tables E (x, y, z blocks of EN
// entries; the Hermite index t is added by the caller), 10 bits each.
template <int LA, int LB>
__device__ __forceinline__ void wq_comp_index(int *idx, int tid, int nt) {
  constexpr int NB = ncart(LB), NIJ = ncart(LA) * NB, LT = LA + LB + 1, EN = (LA + 1) * (LB + 1) * LT;
  for (int ij = tid; ij < NIJ; ij += nt) {
    int ix, iy, iz, jx, jy, jz;
    cart_decode(LA, ij / NB, ix, iy, iz);
    cart_decode(LB, ij % NB, jx, jy, jz);
    idx[ij] = ((ix * (LB + 1) + jx) * LT) | ((EN + (iy * (LB + 1) + jy) * LT) << 10) |
              ((2 * EN + (iz * (LB + 1) + jz) * LT) << 20);
  }
}

// MMA = false: FMA transforms with compact product tables (FP64 and FP32);
// MMA = true: DMMA transforms (FP64, Shape::MMA_OK classes).
template <int LA, int LB, int LC, int LD, typename Tc, bool MMA>
__global__ void __launch_bounds__(128) jk_warp_kernel(const JKArgs a) {
  using S = wq::Shape<LA, LB, LC, LD, Tc>;
  static_assert(!MMA || S::MMA_OK, "DMMA form of a class it does not fit");
  constexpr int L = S::L, SA = S::SA, SB = S::SB, NAB = S::NAB, NCD = S::NCD, N3AB = S::N3AB,
                N3CD = S::N3CD, N3L = S::N3L, EA = S::EA, EC = S::EC, PX = S::PX, PG = S::PG;
  extern __shared__ double sm[];
  double *tab = sm;
  double *sph = tab + kBoysTableDoubles;
  int *tuvt = (int *)(sph + kSphTableDoubles);
  int *idx_ab = tuvt + N3L, *idx_cd = idx_ab + S::TAB;
  int *cmp_ab = idx_cd + S::TCD, *cmp_cd = cmp_ab + NAB;  // packed E positions per Cartesian component pair
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  double *wbase = sm + S::COMMON + (size_t)warp * S::PER_WARP;
  double *regA = wbase, *regB = regA + S::RA;
  Tc *Eb = (Tc *)(regB + S::RB), *Ek = Eb + 3 * EA, *Tb = Ek + 3 * EC, *Tk = Tb + S::TAB;
  double *Db = regB + S::RB + S::RT;
  Tc *R0 = (Tc *)regA, *R1 = R0 + S::RBOX;
  Tc *X = (Tc *)regB;
  double *Gc = regA, *Gs = regB;

  for (int i = threadIdx.x; i < kBoysTableDoubles; i += blockDim.x) tab[i] = a.boys[i];
  for (int i = threadIdx.x; i < kSphTableDoubles; i += blockDim.x) sph[i] = a.sph[i];
  for (int e = threadIdx.x; e < N3L; e += blockDim.x) {
    int t, u, v;
    tuv_decode(e, t, u, v);
    tuvt[e] = t * SA + u * SB + v;  // position of (t,u,v) in the R box
  }
  if constexpr (MMA) {
    wq_comp_index<LA, LB>(cmp_ab, threadIdx.x, blockDim.x);
    wq_comp_index<LC, LD>(cmp_cd, threadIdx.x, blockDim.x);
  } else {
    wq_term_index<LA, LB>(idx_ab, threadIdx.x, blockDim.x);
    wq_term_index<LC, LD>(idx_cd, threadIdx.x, blockDim.x);
  }
  __syncthreads();
  unsigned long long cnt_q = 0, cnt_p = 0, cnt_s = 0;
  // One contiguous range of the queue per warp.
  const int64_t nteam = (int64_t)gridDim.x * nw, team = (int64_t)blockIdx.x * nw + warp;
  const int64_t span = (a.nquartet - a.q_begin + nteam - 1) / nteam;
  const int64_t qbeg = a.q_begin + team * span, qend = min(qbeg + span, a.nquartet);
  int ibw = -1, tb_bra = -1;  // running bra; bra whose product table Tb holds
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
      if (lane == 0 && sel == 2 && a.mode != 2) ++cnt_s;
      continue;
    }
    double w = 1.0;
    if (br.same) w *= 0.5;
    if (kt.same) w *= 0.5;
    if (a.same_class && ib == ic + a.ket_off) w *= 0.5;
    // Primitive pairs: bra i outside, ket j inside.  X accumulates over the
    // ket primitives; the (ab|cd) block over the bra primitives, in each
    // lane's registers where one lane holds a whole ket component column
    // (MP classes; the host launches other classes for one primitive pair
    // per side only).
    constexpr bool LOOPS = MMA || S::MP;
    const int nbp = LOOPS ? br.npp : 1, nkp = LOOPS ? kt.npp : 1;
    Tc gacc[(S::MP && !MMA) ? NAB : 1];
#pragma unroll
    for (int k = 0; k < ((S::MP && !MMA) ? NAB : 1); ++k) gacc[k] = Tc(0);
    double dacc[MMA ? S::MT3 * S::NT * 2 : 1];  // D fragments of the (ab|cd) block
#pragma unroll
    for (int k = 0; k < (MMA ? S::MT3 * S::NT * 2 : 1); ++k) dacc[k] = 0.0;
    for (int i = 0; i < nbp; ++i) {
      const PrimPair P1 = load_prim<true>(a.pp + br.pp0 + i);
      __syncwarp();
      if (nbp > 1 || tb_bra != ib) {
        if (lane < 3) {
          const double pa = lane == 0 ? P1.PAx : lane == 1 ? P1.PAy : P1.PAz;
          const double pb = lane == 0 ? P1.PBx : lane == 1 ? P1.PBy : P1.PBz;
          herm_e<LA, LB, 1, Tc>(Tc(0.5 / P1.p), Tc(pa), Tc(pb), Eb + lane * EA);
        }
        __syncwarp();
        if constexpr (!MMA) wq_product_table<S::TAB, Tc>(Eb, idx_ab, Tb, lane);
        tb_bra = nbp == 1 ? ib : -1;
      }
      for (int j = 0; j < nkp; ++j) {
        const PrimPair P2 = load_prim<true>(a.pp + (a.ket_pp0 >= 0 ? a.ket_pp0 + ic : kt.pp0 + j));
        __syncwarp();
        if (lane < 3) {
          const double pa = lane == 0 ? P2.PAx : lane == 1 ? P2.PAy : P2.PAz;
          const double pb = lane == 0 ? P2.PBx : lane == 1 ? P2.PBy : P2.PBz;
          herm_e<LC, LD, -1, Tc>(Tc(0.5 / P2.p), Tc(pa), Tc(pb), Ek + lane * EC);
        }
        // Boys function and scaled R^n_000 (every lane, the same values)
        const double rs = (sizeof(Tc) == 4) ? (double)rsqrtf((float)(P1.p + P2.p)) : rsqrt(P1.p + P2.p);
        double alpha = P1.p * P2.p * rs * rs;
        double s = P1.K * P2.K * rs;
        erf_attenuate(a.erf_mu2, alpha, s);
        const double x = P1.Px - P2.Px, y = P1.Py - P2.Py, z = P1.Pz - P2.Pz;
        double F[L + 1];
        boys_eval<L, (sizeof(Tc) == 4) ? kBoysDegLow : kBoysDeg>(alpha * (x * x + y * y + z * z), tab, F);
        double Fs[L + 1];
        {
#pragma unroll
          for (int n = 0; n <= L; ++n) {
            Fs[n] = s * F[n];
            s *= -2.0 * alpha;
          }
        }
        __syncwarp();
        if constexpr (!MMA) wq_product_table<S::TCD, Tc>(Ek, idx_cd, Tk, lane);
        // R_tuv, level n = L-1 .. 0 from level n+1, ping-pong between R0 and R1
        Tc *prev = R0, *cur = R1;
        if (lane == 0) prev[0] = Tc(Fs[L]);
        __syncwarp();
        const Tc tx = Tc(x), ty = Tc(y), tz = Tc(z);
#pragma unroll 1
        for (int n = L - 1; n >= 0; --n) {
          const int cnt = n3(L - n);
          for (int e = lane; e < cnt; e += 32) {
            const int pos = tuvt[e];
            const int t = pos / SA, u = (pos % SA) / SB, v = (pos % SA) % SB;
            Tc val;
            if (e == 0) {
              val = Tc(Fs[n]);
            } else if (t > 0) {
              val = tx * prev[pos - SA];
              if (t > 1) val += Tc(t - 1) * prev[pos - 2 * SA];
            } else if (u > 0) {
              val = ty * prev[pos - SB];
              if (u > 1) val += Tc(u - 1) * prev[pos - 2 * SB];
            } else {
              val = tz * prev[pos - 1];
              if (v > 1) val += Tc(v - 1) * prev[pos - 2];
            }
            cur[pos] = val;
          }
          __syncwarp();
          Tc *sw = prev;
          prev = cur;
          cur = sw;
        }
        const Tc *R = prev;
        if constexpr (MMA) {
          // ket product X[cd][e] (+)= sum_f R[e+f] E^cd[f]: rows e, columns
          // cd, depth f; A from the R box, B the dense ket coefficient
          // products (zero where a component does not reach f).
          const int g = lane >> 2, t4 = lane & 3;
          wq::static_for<S::NT>([&](auto NT_) {
            constexpr int nt = decltype(NT_)::value;
            const int cd = nt * 8 + g;
            const int pc = cd < NCD ? cmp_cd[cd] : 0;
            double bf[S::KT2];
#pragma unroll
            for (int kk = 0; kk < S::KT2; ++kk) {
              const int f = kk * 4 + t4;
              double v = 0.0;
              if (cd < NCD && f < N3CD) {
                const int pos = tuvt[f];
                const int ft = pos / SA, fu = (pos % SA) / SB, fv = (pos % SA) % SB;
                v = (double)Ek[(pc & 1023) + ft] * (double)Ek[((pc >> 10) & 1023) + fu] * (double)Ek[(pc >> 20) + fv];
              }
              bf[kk] = v;
            }
#pragma unroll
            for (int mt = 0; mt < S::MT2; ++mt) {
              const int e = mt * 8 + g;
              const int pe = e < N3AB ? tuvt[e] : 0;
              double d0 = 0.0, d1 = 0.0;
#pragma unroll
              for (int kk = 0; kk < S::KT2; ++kk) {
                const int f = kk * 4 + t4;
                const double av = (e < N3AB && f < N3CD) ? (double)R[pe + tuvt[f]] : 0.0;
                wq::dmma(d0, d1, av, bf[kk]);
              }
              const int c0 = nt * 8 + 2 * t4;
              if (e < N3AB) {
                if (c0 < NCD) X[c0 * PX + e] = Tc(j > 0 ? d0 + (double)X[c0 * PX + e] : d0);
                if (c0 + 1 < NCD) X[(c0 + 1) * PX + e] = Tc(j > 0 ? d1 + (double)X[(c0 + 1) * PX + e] : d1);
              }
            }
          });
        } else {
          // ket transform: lane = bra Hermite index, every ket component (in
          // chunks of kChunk components, R re-read per chunk)
          for (int e = lane; e < N3AB; e += 32) {
            const int base = tuvt[e];
            wq::static_for<(NCD + wq::kChunk - 1) / wq::kChunk>([&](auto CH_) {
              constexpr int c0 = decltype(CH_)::value * wq::kChunk;
              constexpr int nc = NCD - c0 < wq::kChunk ? NCD - c0 : wq::kChunk;
              Tc xa[nc];
#pragma unroll
              for (int k = 0; k < nc; ++k) xa[k] = Tc(0);
              wq::static_for<N3CD>([&](auto F_) {
                constexpr int f = decltype(F_)::value;
                constexpr int ft = wq::tuv_t(f), fu = wq::tuv_u(f), fv = wq::tuv_v(f);
                if constexpr (wq::chunk_uses(LC, LD, c0, nc, ft, fu, fv)) {
                  const Tc r = R[base + ft * SA + fu * SB + fv];
                  wq::static_for<nc>([&](auto K_) {
                    constexpr int cd = c0 + decltype(K_)::value;
                    if constexpr (wq::uses(LC, LD, cd, ft, fu, fv))
                      xa[cd - c0] += Tk[wq::term_at(LC, LD, cd, ft, fu, fv)] * r;
                  });
                }
              });
              if constexpr (S::SPHR && !MMA) {
                if (a.spherical) {  // one chunk holds all ket components: spherical rows of X
                  Tc xs[S::FCD];
                  sph_pair<LC, LD>(xa, xs);
                  if (j > 0) {
#pragma unroll
                    for (int k = 0; k < S::FCD; ++k) xs[k] += X[k * PX + e];
                  }
#pragma unroll
                  for (int k = 0; k < S::FCD; ++k) X[k * PX + e] = xs[k];
                  return;
                }
              }
              if (j > 0) {  // later ket primitives add to X
#pragma unroll
                for (int k = 0; k < nc; ++k) xa[k] += X[(c0 + k) * PX + e];
              }
#pragma unroll
              for (int k = 0; k < nc; ++k) X[(c0 + k) * PX + e] = xa[k];
            });
          }
        }
        __syncwarp();
      }
      if constexpr (MMA) {
        // bra product G[ab][cd] += sum_e E^ab[e] X[cd][e]: rows ab, columns
        // cd, depth e; A the dense bra coefficient products, B from X, D in
        // the lane's accumulators across the bra primitives.
        const int g = lane >> 2, t4 = lane & 3;
#pragma unroll
        for (int mt = 0; mt < S::MT3; ++mt) {
          const int ab = mt * 8 + g;
          const int pa = ab < NAB ? cmp_ab[ab] : 0;
          double af[S::KT3];
#pragma unroll
          for (int kk = 0; kk < S::KT3; ++kk) {
            const int e = kk * 4 + t4;
            double v = 0.0;
            if (ab < NAB && e < N3AB) {
              const int pos = tuvt[e];
              const int et = pos / SA, eu = (pos % SA) / SB, ev = (pos % SA) % SB;
              v = (double)Eb[(pa & 1023) + et] * (double)Eb[((pa >> 10) & 1023) + eu] * (double)Eb[(pa >> 20) + ev];
            }
            af[kk] = v;
          }
#pragma unroll
          for (int nt = 0; nt < S::NT; ++nt) {
            const int cd = nt * 8 + g;
#pragma unroll
            for (int kk = 0; kk < S::KT3; ++kk) {
              const int e = kk * 4 + t4;
              const double bv = (cd < NCD && e < N3AB) ? (double)X[cd * PX + e] : 0.0;
              wq::dmma(dacc[(mt * S::NT + nt) * 2], dacc[(mt * S::NT + nt) * 2 + 1], af[kk], bv);
            }
          }
        }
      } else if constexpr (S::MP) {
        // bra transform into the lane's accumulators: lane = ket component
        // (spherical ones when the ket transform produced them)
        if (lane < ((S::SPHR && a.spherical) ? S::FCD : NCD)) {
          wq::static_for<N3AB>([&](auto E_) {
            constexpr int e = decltype(E_)::value;
            constexpr int et = wq::tuv_t(e), eu = wq::tuv_u(e), ev = wq::tuv_v(e);
            const Tc xv = X[lane * PX + e];
            wq::static_for<NAB>([&](auto K_) {
              constexpr int ab = decltype(K_)::value;
              if constexpr (wq::uses(LA, LB, ab, et, eu, ev)) gacc[ab] += Tb[wq::term_at(LA, LB, ab, et, eu, ev)] * xv;
            });
          });
        }
      } else {
        // bra transform: lane = ket component, every bra component (in chunks)
        for (int cd = lane; cd < NCD; cd += 32) {
          wq::static_for<(NAB + wq::kChunk - 1) / wq::kChunk>([&](auto CH_) {
            constexpr int a0 = decltype(CH_)::value * wq::kChunk;
            constexpr int na = NAB - a0 < wq::kChunk ? NAB - a0 : wq::kChunk;
            Tc acc[na];
#pragma unroll
            for (int k = 0; k < na; ++k) acc[k] = Tc(0);
            wq::static_for<N3AB>([&](auto E_) {
              constexpr int e = decltype(E_)::value;
              constexpr int et = wq::tuv_t(e), eu = wq::tuv_u(e), ev = wq::tuv_v(e);
              if constexpr (wq::chunk_uses(LA, LB, a0, na, et, eu, ev)) {
                const Tc xv = X[cd * PX + e];
                wq::static_for<na>([&](auto K_) {
                  constexpr int ab = a0 + decltype(K_)::value;
                  if constexpr (wq::uses(LA, LB, ab, et, eu, ev))
                    acc[ab - a0] += Tb[wq::term_at(LA, LB, ab, et, eu, ev)] * xv;
                });
              }
            });
#pragma unroll
            for (int k = 0; k < na; ++k) Gc[(a0 + k) * PG + cd] = (double)acc[k];
          });
        }
      }
      __syncwarp();
    }
    if constexpr (MMA) {
      // D fragments to the Cartesian block (R, in region A, is no longer needed)
      const int g = lane >> 2, t4 = lane & 3;
#pragma unroll
      for (int mt = 0; mt < S::MT3; ++mt)
#pragma unroll
        for (int nt = 0; nt < S::NT; ++nt) {
          const int ab = mt * 8 + g, c0 = nt * 8 + 2 * t4;
          if (ab < NAB) {
            if (c0 < NCD) Gc[ab * PG + c0] = dacc[(mt * S::NT + nt) * 2];
            if (c0 + 1 < NCD) Gc[ab * PG + c0 + 1] = dacc[(mt * S::NT + nt) * 2 + 1];
          }
        }
      __syncwarp();
    } else if constexpr (S::MP) {
      // the accumulated block to shared memory (R, in region A, is no longer needed)
      if (S::SPHR && a.spherical) {
        if (lane < S::FCD) {
          Tc gs[S::FAB];
          sph_pair<LA, LB>(gacc, gs);
#pragma unroll
          for (int k = 0; k < S::FAB; ++k) Gc[k * PG + lane] = (double)gs[k];
        }
      } else if (lane < NCD) {
#pragma unroll
        for (int k = 0; k < NAB; ++k) Gc[k * PG + lane] = (double)gacc[k];
      }
      __syncwarp();
    }
    if (lane == 0) {
      cnt_q += 1;
      cnt_p += (unsigned long long)nbp * nkp;
    }
    if (a.spherical)
      wq_finish<LA, LB, LC, LD, Tc, true, S::SPHR && !MMA>(a, Gc, Gs, Db, sph, br, kt, ib, ic, w, lane, q);
    else
      wq_finish<LA, LB, LC, LD, Tc, false>(a, Gc, Gs, Db, sph, br, kt, ib, ic, w, lane, q);
    __syncwarp();
  }
  if (lane == 0 && a.counters) {
    atomicAdd(a.counters + 0, cnt_q);
    atomicAdd(a.counters + 1, cnt_p);
    atomicAdd(a.counters + 2, cnt_s);
    if (sizeof(Tc) == 4) atomicAdd(a.counters + 3, cnt_q);
  }
}

}  // namespace dgf
