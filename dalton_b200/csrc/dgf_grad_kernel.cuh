// Two-electron part of the RHF nuclear gradient (pattern 3, the backward
// kernel): for every canonical shell quartet the derivative integrals are
// recomputed (never stored) and contracted with the symmetrised density
// product
//   G_abcd = w [2 (D1_ab D2_cd + D2_ab D1_cd)
//             - hfx/2 (D1_ac D2_bd + D2_ac D1_bd + D1_ad D2_bc + D2_ad D1_bc)],
// so that with D1 = D2 = D the sum is d/dx of 1/2 sum (pq|rs)[D_pq D_rs -
// hfx/2 D_pr D_qs] (TWOEXP -> INTEX1 -> DEROUT, DALTON/abacus/aba2tex.F:242,
// her2ave.F:91-830), and for D1 = C (a cotangent) it is half the derivative
// of <C, G(D)>.
//
// Derivatives of the Gaussians enter through shifted Hermite expansions:
// d/dA_x of the bra is 2a E^{a+1x,b} - a_x E^{a-1x,b} (and alike for B and
// for C on the ket); the centre-D derivative follows from translational
// invariance.  One thread per quartet; quartets come from the Fock build's
// Schwarz-screened class plan.  The lanes of a warp share their bra pair (as
// in the Fock kernels), so the bra's plain and derivative Hermite tables are
// built once per bra primitive in shared memory; the density product is
// formed from Cartesian 2-index blocks with compile-time sizes; the bra sums
// over (t, u, v) are nested one direction at a time.
#pragma once

#include <utility>

#include "dgf_md.cuh"

namespace dgf {
namespace grad {

constexpr int kGradBlock = 128;
constexpr int kGradWarps = kGradBlock / 32;
// Gradients of molecules up to this many atoms are summed per block in
// shared memory and flushed once per block (every quartet adds to four
// centres, so a global accumulator of 3 natom doubles is a hot spot).
constexpr int kGradSmemAtoms = 256;

// Per-warp shared tables of the current bra primitive pair: the Hermite
// coefficients E^{ij}_t of herm_e<LA+1, LB+1> per direction (stage), and
// derived from them, per direction and (i, j) with i <= LA, j <= LB, t <=
// LA+LB+1: the plain E^{ij}_t, the A-derivative 2a E^{i+1,j}_t - i E^{i-1,j}_t
// and the B-derivative 2b E^{i,j+1}_t - j E^{i,j-1}_t (zero past the range).
template <int LA, int LB>
struct GradBra {
  static constexpr int LAB = LA + LB;
  static constexpr int T1 = LAB + 3;
  static constexpr int EA1 = (LA + 2) * (LB + 2) * T1;
  static constexpr int TT = LAB + 2;
  static constexpr int NT = (LA + 1) * (LB + 1) * TT;
  static constexpr int kSize = 3 * EA1 + 9 * NT;
};

// The (lx, ly) block of density D (rows p0.., columns q0.., row stride N) in
// Cartesian components: spherical blocks are mapped back with the transposed
// Cartesian -> spherical tables, so that sum_sph G_sph I_sph = sum_cart G I.
template <int LX, int LY, bool SPH>
__device__ __forceinline__ void cart_block(const double *__restrict__ D, int N, int p0, int q0, double *out) {
  constexpr int NX = ncart(LX), NY = ncart(LY);
  constexpr bool TX = SPH && LX >= 2, TY = SPH && LY >= 2;
  constexpr int FX = TX ? 2 * LX + 1 : NX, FY = TY ? 2 * LY + 1 : NY;
  double f[FX * FY];
#pragma unroll
  for (int x = 0; x < FX; ++x)
#pragma unroll
    for (int y = 0; y < FY; ++y) f[x * FY + y] = D[(size_t)(p0 + x) * N + q0 + y];
  // transposed tables with compile-time coefficients (zero ones drop out)
  double t1[NX * FY];
#pragma unroll
  for (int y = 0; y < FY; ++y)
    static_for<NX>([&](auto I_) {
      constexpr int i = decltype(I_)::value;
      if constexpr (TX) {
        double s = 0.0;
        static_for<FX>([&](auto X_) {
          constexpr int x = decltype(X_)::value;
          constexpr double c = sph::coef<LX>(x, i);
          if constexpr (c != 0.0) s += c * f[x * FY + y];
        });
        t1[i * FY + y] = s;
      } else {
        t1[i * FY + y] = f[i * FY + y];
      }
    });
#pragma unroll
  for (int i = 0; i < NX; ++i)
    static_for<NY>([&](auto J_) {
      constexpr int j = decltype(J_)::value;
      if constexpr (TY) {
        double s = 0.0;
        static_for<FY>([&](auto Y_) {
          constexpr int y = decltype(Y_)::value;
          constexpr double c = sph::coef<LY>(y, j);
          if constexpr (c != 0.0) s += t1[i * FY + y] * c;
        });
        out[i * NY + j] = s;
      } else {
        out[i * NY + j] = t1[i * FY + j];
      }
    });
}

// Chunks of the ket's Cartesian (c, d) components a launch is split into
// (grid.y): the high-L classes have few quartets and much work per quartet,
// so they are spread over more threads, each recomputing the quartet's R_tuv.
constexpr int grad_chunks(int LA, int LB, int LC, int LD) { return (LA + LB + LC + LD) >= 4 ? ncart(LC) : 1; }

// Chunk CH of CDN handles the ket components cd = c ND + d in [CD0, CD1).
template <int LA, int LB, int LC, int LD, bool SPH, int CDN, int CH>
__device__ __forceinline__ void grad_body(const JKArgs &a, const double *tab, double *bt,
                                          double *gsh) {
  constexpr int L = LA + LB + LC + LD, LAB = LA + LB, LCD = LC + LD;
  constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  constexpr int NCD = NC * ND;
  constexpr int CD0 = CH * NCD / CDN, CD1 = (CH + 1) * NCD / CDN, NCDc = CD1 - CD0;
  constexpr int TC = LCD + 2;                       // t extent of the ket tables herm_e<LC+1, LD>
  constexpr int EC1 = (LC + 2) * (LD + 1) * TC;
  using S = GradBra<LA, LB>;
  const int lane = threadIdx.x & 31;
  const unsigned full = 0xffffffffu;
  const int N = a.nbf;
  const double h = 0.5 * a.hfx;
  double *stage = bt, *pl = bt + 3 * S::EA1, *da = pl + 3 * S::NT, *db = da + 3 * S::NT;
  // one contiguous range of the queue per warp (the bra index only moves forward)
  const int64_t nwarp = (int64_t)gridDim.x * (blockDim.x >> 5);
  const int64_t wid = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int64_t span = (((a.nquartet - a.q_begin) + nwarp - 1) / nwarp + 31) & ~(int64_t)31;
  const int64_t wbegin = a.q_begin + wid * span, wend = min(wbegin + span, a.nquartet);
  int ibw = 0;
  if (wbegin < wend && lane == 0) ibw = find_bra(a.qoff, a.nbra, wbegin);
  ibw = __shfl_sync(full, ibw, 0);
  for (int64_t base = wbegin; base < wend; base += 32) {
    const int64_t q = base + lane;
    bool work = q < wend;
    int ib0 = ibw;
    if (lane == 0) {
      int steps = 0;
      while (base >= a.qoff[ib0 + 1] && steps < 32) {
        ++ib0;
        ++steps;
      }
      if (base >= a.qoff[ib0 + 1]) ib0 = find_bra(a.qoff, a.nbra, base);
    }
    ib0 = __shfl_sync(full, ib0, 0);
    ibw = ib0;
    int ib = ib0, ic = 0;
    PairRec br, kt;
    double G[NA * NB * NCDc];  // this chunk's (c, d) components
    if (work) {
      int steps = 0;
      while (q >= a.qoff[ib + 1] && steps < 32) {
        ++ib;
        ++steps;
      }
      if (q >= a.qoff[ib + 1]) ib = find_bra(a.qoff, a.nbra, q);
      ic = (int)(q - a.qoff[ib]);
      br = load_pair(a.bra + ib);
      kt = load_pair(a.ket + ic);
      work = br.Q * kt.Q >= a.schwarz_thr;  // the plan's last Schwarz bin may reach below the threshold
    }
    if (work) {
      double w = 1.0;
      if (br.same) w *= 0.5;
      if (kt.same) w *= 0.5;
      if (a.same_class && ib == ic + a.ket_off) w *= 0.5;
      // G_abcd = w [2 (D1_ab D2_cd + D2_ab D1_cd) - hfx/2 (D1_ac D2_bd + D2_ac D1_bd + D1_ad D2_bc + D2_ad D1_bc)]
      double ab1[NA * NB], ab2[NA * NB], cd1[NCD], cd2[NCD];
      cart_block<LA, LB, SPH>(a.G1, N, br.aoA, br.aoB, ab1);
      cart_block<LA, LB, SPH>(a.G2, N, br.aoA, br.aoB, ab2);
      cart_block<LC, LD, SPH>(a.G1, N, kt.aoA, kt.aoB, cd1);
      cart_block<LC, LD, SPH>(a.G2, N, kt.aoA, kt.aoB, cd2);
#pragma unroll
      for (int x = 0; x < NA * NB; ++x)
#pragma unroll
        for (int y = CD0; y < CD1; ++y) G[x * NCDc + y - CD0] = 2.0 * w * (ab1[x] * cd2[y] + ab2[x] * cd1[y]);
      if (h != 0.0) {
        double ac1[NA * NC], ac2[NA * NC], bd1[NB * ND], bd2[NB * ND];
        cart_block<LA, LC, SPH>(a.G1, N, br.aoA, kt.aoA, ac1);
        cart_block<LA, LC, SPH>(a.G2, N, br.aoA, kt.aoA, ac2);
        cart_block<LB, LD, SPH>(a.G1, N, br.aoB, kt.aoB, bd1);
        cart_block<LB, LD, SPH>(a.G2, N, br.aoB, kt.aoB, bd2);
#pragma unroll
        for (int i = 0; i < NA; ++i)
#pragma unroll
          for (int j = 0; j < NB; ++j)
#pragma unroll
            for (int k = 0; k < NC; ++k)
#pragma unroll
              for (int l = 0; l < ND; ++l) {
                if (k * ND + l < CD0 || k * ND + l >= CD1) continue;
                G[(i * NB + j) * NCDc + k * ND + l - CD0] -=
                    w * h * (ac1[i * NC + k] * bd2[j * ND + l] + ac2[i * NC + k] * bd1[j * ND + l]);
              }
        double ad1[NA * ND], ad2[NA * ND], bc1[NB * NC], bc2[NB * NC];
        cart_block<LA, LD, SPH>(a.G1, N, br.aoA, kt.aoB, ad1);
        cart_block<LA, LD, SPH>(a.G2, N, br.aoA, kt.aoB, ad2);
        cart_block<LB, LC, SPH>(a.G1, N, br.aoB, kt.aoA, bc1);
        cart_block<LB, LC, SPH>(a.G2, N, br.aoB, kt.aoA, bc2);
#pragma unroll
        for (int i = 0; i < NA; ++i)
#pragma unroll
          for (int j = 0; j < NB; ++j)
#pragma unroll
            for (int k = 0; k < NC; ++k)
#pragma unroll
              for (int l = 0; l < ND; ++l) {
                if (k * ND + l < CD0 || k * ND + l >= CD1) continue;
                G[(i * NB + j) * NCDc + k * ND + l - CD0] -=
                    w * h * (ad1[i * ND + l] * bc2[j * NC + k] + ad2[i * ND + l] * bc1[j * NC + k]);
              }
      }
    }
    double acc[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) acc[k] = 0.0;
    unsigned pending = __ballot_sync(full, work);
    while (pending) {
      const int leader = __ffs(pending) - 1;
      const int ibl = __shfl_sync(full, ib, leader);
      const bool mine = work && ib == ibl && ((pending >> lane) & 1u);
      pending &= ~__ballot_sync(full, mine);
      const PairRec brl = load_pair(a.bra + ibl);
      for (int i = 0; i < brl.npp; ++i) {
        const PrimPair P1 = load_prim<true>(a.pp + brl.pp0 + i);
        const double ea = P1.ea, eb = P1.p - P1.ea;
        __syncwarp();
        if (lane < 3) {
          const double pa = lane == 0 ? P1.PAx : lane == 1 ? P1.PAy : P1.PAz;
          const double pb = lane == 0 ? P1.PBx : lane == 1 ? P1.PBy : P1.PBz;
          herm_e<LA + 1, LB + 1, 1, double>(0.5 / P1.p, pa, pb, stage + lane * S::EA1);
        }
        __syncwarp();
        for (int e = lane; e < 3 * S::NT; e += 32) {
          const int dir = e / S::NT, r = e - dir * S::NT;
          const int t = r % S::TT, ij = r / S::TT, j0 = ij % (LB + 1), i0 = ij / (LB + 1);
          const double *Et = stage + dir * S::EA1;
          auto E = [&](int i, int j) { return (t <= i + j) ? Et[(i * (LB + 2) + j) * S::T1 + t] : 0.0; };
          pl[e] = E(i0, j0);
          da[e] = 2.0 * ea * E(i0 + 1, j0) - (i0 > 0 ? i0 * E(i0 - 1, j0) : 0.0);
          db[e] = 2.0 * eb * E(i0, j0 + 1) - (j0 > 0 ? j0 * E(i0, j0 - 1) : 0.0);
        }
        __syncwarp();
        if (!mine) continue;
        for (int j = 0; j < kt.npp; ++j) {
          const PrimPair P2 = load_prim<true>(a.pp + kt.pp0 + j);
          const double ecx = P2.ea;
          const double rs = rsqrt(P1.p + P2.p);
          const double alpha = P1.p * P2.p * rs * rs;
          const double x = P1.Px - P2.Px, y = P1.Py - P2.Py, z = P1.Pz - P2.Pz;
          double F[L + 2];
          boys_eval<L + 1>(alpha * (x * x + y * y + z * z), tab, F);
          double Fs[L + 2];
          double sc = P1.K * P2.K * rs;
#pragma unroll
          for (int n = 0; n <= L + 1; ++n) {
            Fs[n] = sc * F[n];
            sc *= -2.0 * alpha;
          }
          double R[n3(L + 1)];
          hermite_r_inplace<L + 1, double>(Fs, x, y, z, R);
          double e2x[EC1], e2y[EC1], e2z[EC1];
          const double h2 = 0.5 / P2.p;
          herm_e<LC + 1, LD, -1, double>(h2, P2.PAx, P2.PBx, e2x);
          herm_e<LC + 1, LD, -1, double>(h2, P2.PAy, P2.PBy, e2y);
          herm_e<LC + 1, LD, -1, double>(h2, P2.PAz, P2.PBz, e2z);
          const double *E2[3] = {e2x, e2y, e2z};
#pragma unroll
          for (int c = 0; c < NC; ++c)
#pragma unroll
            for (int d = 0; d < ND; ++d) {
              if (c * ND + d < CD0 || c * ND + d >= CD1) continue;
              const int cc[3] = {cart_x(LC, c), cart_y(LC, c), cart_z(LC, c)};
              const int dd[3] = {cart_x(LD, d), cart_y(LD, d), cart_z(LD, d)};
              // ket transforms: plain (bra range t+u+v <= LAB+1) and C-derivative (<= LAB)
              double xk[n3(LAB + 1)];
              double xc[3][n3(LAB)];
#pragma unroll
              for (int e = 0; e < n3(LAB + 1); ++e) xk[e] = 0.0;
#pragma unroll
              for (int k = 0; k < 3; ++k)
#pragma unroll
                for (int e = 0; e < n3(LAB); ++e) xc[k][e] = 0.0;
#pragma unroll
              for (int ta = 0; ta <= cc[0] + dd[0] + 1; ++ta)
#pragma unroll
                for (int na = 0; na <= cc[1] + dd[1] + 1; ++na)
#pragma unroll
                  for (int fa = 0; fa <= cc[2] + dd[2] + 1; ++fa) {
                    const int tt[3] = {ta, na, fa};
                    double ev[3], dv[3];
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                      const double *Et = E2[k];
                      ev[k] = (tt[k] <= cc[k] + dd[k]) ? Et[(cc[k] * (LD + 1) + dd[k]) * TC + tt[k]] : 0.0;
                      double dvk = 2.0 * ecx * Et[((cc[k] + 1) * (LD + 1) + dd[k]) * TC + tt[k]];
                      if (cc[k] > 0 && tt[k] <= cc[k] - 1 + dd[k])
                        dvk -= cc[k] * Et[((cc[k] - 1) * (LD + 1) + dd[k]) * TC + tt[k]];
                      dv[k] = dvk;
                    }
                    const double e0 = ev[0] * ev[1] * ev[2];
                    const double d0 = dv[0] * ev[1] * ev[2], d1 = ev[0] * dv[1] * ev[2], d2 = ev[0] * ev[1] * dv[2];
#pragma unroll
                    for (int t = 0; t <= LAB + 1; ++t)
#pragma unroll
                      for (int u = 0; u <= LAB + 1 - t; ++u)
#pragma unroll
                        for (int v = 0; v <= LAB + 1 - t - u; ++v) {
                          if (t + ta + u + na + v + fa > L + 1) continue;  // past the R range: zero
                          const double r = R[tuv_index(t + ta, u + na, v + fa)];
                          xk[tuv_index(t, u, v)] += e0 * r;
                          if (t + u + v <= LAB) {
                            xc[0][tuv_index(t, u, v)] += d0 * r;
                            xc[1][tuv_index(t, u, v)] += d1 * r;
                            xc[2][tuv_index(t, u, v)] += d2 * r;
                          }
                        }
                  }
              // bra side from the shared tables, sums nested v -> u -> t; the
              // (a, b) component loop stays rolled to bound code size and registers
#pragma unroll 1
              for (int ab = 0; ab < NA * NB; ++ab) {
                const int ia = ab / NB, jb = ab - ia * NB;
                const double g = G[ab * NCDc + c * ND + d - CD0];
                int ax0, ax1, ax2, bx0, bx1, bx2;
                cart_decode(LA, ia, ax0, ax1, ax2);
                cart_decode(LB, jb, bx0, bx1, bx2);
                const double *P0 = pl + 0 * S::NT + (ax0 * (LB + 1) + bx0) * S::TT;
                const double *P1t = pl + 1 * S::NT + (ax1 * (LB + 1) + bx1) * S::TT;
                const double *P2t = pl + 2 * S::NT + (ax2 * (LB + 1) + bx2) * S::TT;
                const double *A0 = da + 0 * S::NT + (ax0 * (LB + 1) + bx0) * S::TT;
                const double *A1 = da + 1 * S::NT + (ax1 * (LB + 1) + bx1) * S::TT;
                const double *A2 = da + 2 * S::NT + (ax2 * (LB + 1) + bx2) * S::TT;
                const double *B0 = db + 0 * S::NT + (ax0 * (LB + 1) + bx0) * S::TT;
                const double *B1 = db + 1 * S::NT + (ax1 * (LB + 1) + bx1) * S::TT;
                const double *B2 = db + 2 * S::NT + (ax2 * (LB + 1) + bx2) * S::TT;
                // tables are zero past t = i + j + 1, so the full ranges are safe
                double sA[3] = {0, 0, 0}, sB[3] = {0, 0, 0}, sC[3] = {0, 0, 0};
#pragma unroll
                for (int t = 0; t <= LAB + 1; ++t) {
                  double b00 = 0, b01 = 0, b02 = 0, b10 = 0, b20 = 0, q0 = 0, q1 = 0, q2 = 0;
#pragma unroll
                  for (int u = 0; u <= LAB + 1 - t; ++u) {
                    double a0 = 0, a1 = 0, a2 = 0, c0 = 0, c1 = 0, c2 = 0;
#pragma unroll
                    for (int v = 0; v <= LAB + 1 - t - u; ++v) {
                      const double xv = xk[tuv_index(t, u, v)];
                      const double p2v = P2t[v];
                      a0 += p2v * xv;
                      a1 += A2[v] * xv;
                      a2 += B2[v] * xv;
                      if (t + u + v <= LAB) {
                        c0 += p2v * xc[0][tuv_index(t, u, v)];
                        c1 += p2v * xc[1][tuv_index(t, u, v)];
                        c2 += p2v * xc[2][tuv_index(t, u, v)];
                      }
                    }
                    const double p1u = P1t[u];
                    b00 += p1u * a0;
                    b01 += p1u * a1;
                    b02 += p1u * a2;
                    b10 += A1[u] * a0;
                    b20 += B1[u] * a0;
                    q0 += p1u * c0;
                    q1 += p1u * c1;
                    q2 += p1u * c2;
                  }
                  const double p0t = P0[t];
                  sA[0] += A0[t] * b00;
                  sB[0] += B0[t] * b00;
                  sA[1] += p0t * b10;
                  sB[1] += p0t * b20;
                  sA[2] += p0t * b01;
                  sB[2] += p0t * b02;
                  sC[0] += p0t * q0;
                  sC[1] += p0t * q1;
                  sC[2] += p0t * q2;
                }
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                  acc[k] += g * sA[k];
                  acc[3 + k] += g * sB[k];
                  acc[6 + k] += g * sC[k];
                }
              }
            }
        }
      }
    }
    // Centres A and B (warp-reduced when every working lane has the warp's
    // bra pair), C, and D by translational invariance.
    const bool uniform = __all_sync(full, !work || ib == ib0) && __any_sync(full, work);
    const bool smem_acc = gsh != nullptr;
    auto add = [&](int atom, int k, double v) {
      if (smem_acc)
        atomicAdd(gsh + 3 * atom + k, v);
      else
        atomicAdd(a.grad + 3 * atom + k, v);
    };
    if (uniform) {
      const PairRec brw = load_pair(a.bra + ib0);
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        double v = work ? acc[k] : 0.0;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(full, v, off);
        if (lane == 0) add(k < 3 ? brw.atA : brw.atB, k % 3, v);
      }
    } else if (work) {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        add(br.atA, k, acc[k]);
        add(br.atB, k, acc[3 + k]);
      }
    }
    if (work) {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        add(kt.atA, k, acc[6 + k]);
        add(kt.atB, k, -(acc[k] + acc[3 + k] + acc[6 + k]));
      }
    }
  }
}

// One thread per quartet, 32 consecutive quartets of the class queue per
// warp; SPH selects the spherical (1) or Cartesian (0) density blocks.
template <int LA, int LB, int LC, int LD, bool SPH, int CDN, int CH>
__device__ __forceinline__ void grad_dispatch(int chunk, const JKArgs &a, const double *tab, double *bt,
                                              double *gsh) {
  if constexpr (CH < CDN) {
    if (chunk == CH)
      grad_body<LA, LB, LC, LD, SPH, CDN, CH>(a, tab, bt, gsh);
    else
      grad_dispatch<LA, LB, LC, LD, SPH, CDN, CH + 1>(chunk, a, tab, bt, gsh);
  }
}

template <int LA, int LB, int LC, int LD, bool SPH>
__global__ void __launch_bounds__(kGradBlock) grad_thread_kernel(const JKArgs a) {
  constexpr int CDN = grad_chunks(LA, LB, LC, LD);
  using S = GradBra<LA, LB>;
  __shared__ double tab[kBoysTableDoubles];
  __shared__ double bt_all[kGradWarps][S::kSize];
  __shared__ double gsh_all[3 * kGradSmemAtoms];
  const bool smem_acc = a.natom <= kGradSmemAtoms;
  for (int i = threadIdx.x; i < kBoysTableDoubles; i += blockDim.x) tab[i] = a.boys[i];
  if (smem_acc)
    for (int i = threadIdx.x; i < 3 * a.natom; i += blockDim.x) gsh_all[i] = 0.0;
  __syncthreads();
  grad_dispatch<LA, LB, LC, LD, SPH, CDN, 0>(blockIdx.y, a, tab, bt_all[threadIdx.x >> 5],
                                             smem_acc ? gsh_all : nullptr);
  if (smem_acc) {
    __syncthreads();
    for (int i = threadIdx.x; i < 3 * a.natom; i += blockDim.x)
      if (gsh_all[i] != 0.0) atomicAdd(a.grad + i, gsh_all[i]);
  }
}

constexpr int cls_la(int X) { return X == 0 ? 0 : X <= 2 ? 1 : X <= 5 ? 2 : 3; }
constexpr int cls_lb(int X) { return X - cls_la(X) * (cls_la(X) + 1) / 2; }
constexpr int kGradClasses = 6;  // pair classes up to (dd)

typedef void (*GradLauncher)(const JKArgs &, int, int, cudaStream_t);
extern GradLauncher g_grad_table[kGradClasses][kGradClasses];  // dgf_grad2e.cu; filled by DGF_GRAD_CLASS units

template <int LA, int LB, int LC, int LD>
void launch_grad(const JKArgs &a, int grid, int block, cudaStream_t s) {
  const dim3 g(grid, grad_chunks(LA, LB, LC, LD));
  if (a.spherical)
    grad_thread_kernel<LA, LB, LC, LD, true><<<g, block, 0, s>>>(a);
  else
    grad_thread_kernel<LA, LB, LC, LD, false><<<g, block, 0, s>>>(a);
}


}  // namespace grad
}  // namespace dgf

// Defines the static initialiser that fills entry (X, Y) of the gradient
// table (one generated translation unit per class pair).
#define DGF_GRAD_CLASS(X, Y)                                                                       \
  namespace dgf {                                                                                  \
  namespace grad {                                                                                 \
  namespace {                                                                                      \
  struct GradClassInit_##X##_##Y {                                                                 \
    GradClassInit_##X##_##Y() { g_grad_table[X][Y] = &launch_grad<cls_la(X), cls_lb(X), cls_la(Y), cls_lb(Y)>; } \
  } g_grad_class_init_##X##_##Y;                                                                   \
  }                                                                                                \
  }                                                                                                \
  }
