// Cooperative ("team") McMurchie-Davidson J/K quartet kernel: one thread
// block per contracted shell quartet, intermediates staged in shared memory.
//
// Per quartet (AB|CD) and primitive pairs i (bra), j (ket):
//   R^n_000 = K_i K_j (p+q)^-1/2 (-2 alpha)^n F_n(alpha |PQ|^2)      (R0001)
//   R_tuv by the Hermite recursion                                   (HERI)
//   X_i[tuv][cd] = sum_j sum_tau (-1)^(tau+nu+phi) E^cd_tau R_{t+tau}  (C2: ket)
//   (ab|cd)     = sum_i sum_tuv E^ab_tuv X_i[tuv][cd]                 (C1: bra)
// then Cartesian -> spherical and digestion into the half Fock matrices
// (DALTON/abacus/her2her.F:248-1245, her2el1.F, her2el2.F, herfckcon.F).
// The same kernel computes the Schwarz diagonal (ab|ab) in diag mode.
#pragma once

#include "dgf_select.cuh"

namespace dgf {

template <int LA, int LB, int LC, int LD>
struct TeamShape {
  static constexpr int L = LA + LB + LC + LD, LAB = LA + LB, LCD = LC + LD;
  static constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  static constexpr int NAB = NA * NB, NCD = NC * ND;
  static constexpr int N3L = n3(L), N3AB = n3(LAB);
  static constexpr int EA = (LA + 1) * (LB + 1) * (LAB + 1), EC = (LC + 1) * (LD + 1) * (LCD + 1);
  static constexpr int XS = cmax(N3AB * NCD, NAB * NCD);
  static constexpr int DST = 6 * 100;  // six density blocks of up to 10x10 (Cartesian f)
  // per quartet in flight: R ping-pong, Hermite tables, half-transformed and
  // final blocks, density blocks, and the scalars (F_n, P-Q, weight)
  static constexpr int PQ = 2 * N3L + 3 * EA + 3 * EC + XS + NAB * NCD + DST + (L + 1) + 4;
  // shared by the block: Boys and spherical tables, packed (t,u,v) of R
  static constexpr size_t smem_w(int nq) {
    return ((size_t)kBoysTableDoubles + kSphTableDoubles + (size_t)nq * PQ) * 8 + (size_t)N3L * 4;
  }
  static constexpr size_t smem() { return smem_w(1); }
  // warp teams (one quartet per warp) per block, 0 when four or two do not fit in 96 KB
  static constexpr int kWarpTeams = smem_w(4) <= 96 * 1024 ? 4 : smem_w(2) <= 96 * 1024 ? 2 : 0;
};

// One step of the Cartesian->spherical transform of index k of a 4-index block.
__device__ __forceinline__ void sph_step(const double *in, double *outb, int pre, int nin, int nout, int post,
                                         const double *T, int tid, int nt) {
  const int tot = pre * nout * post;
  for (int e = tid; e < tot; e += nt) {
    int i = e / (nout * post), r = e - i * (nout * post);
    int o = r / post, j = r - o * post;
    double s = 0.0;
    for (int x = 0; x < nin; ++x) s += T[o * nin + x] * in[(i * nin + x) * post + j];
    outb[e] = s;
  }
}

// WT = 0: the whole block works on one quartet at a time.  WT > 0: each of
// the block's WT warps works on its own quartet (its own slice of shared
// memory, warp-level synchronisation), which keeps several light quartets
// (single primitive pairs) in flight per block instead of one.
template <int LA, int LB, int LC, int LD, int WT = 0>
__global__ void __launch_bounds__(128) jk_team_kernel(const JKArgs a) {
  using S = TeamShape<LA, LB, LC, LD>;
  constexpr int L = S::L, LAB = S::LAB, LCD = S::LCD;
  constexpr int NB = S::NB, ND = S::ND, NAB = S::NAB, NCD = S::NCD;
  constexpr int N3L = S::N3L, N3AB = S::N3AB, EA = S::EA, EC = S::EC;
  constexpr int NQ = WT ? WT : 1;
  extern __shared__ double sm[];
  const int sub = WT ? (int)(threadIdx.x >> 5) : 0;
  double *tab = sm;
  double *sph = tab + kBoysTableDoubles;
  double *Ra = sph + kSphTableDoubles + (size_t)sub * S::PQ;
  double *Rb = Ra + N3L;
  double *eab = Rb + N3L;
  double *ecd = eab + 3 * EA;
  double *X = ecd + 3 * EC;
  double *out = X + S::XS;
  double *dst = out + NAB * NCD;
  double *sF = dst + S::DST;
  double *sPQ = sF + (L + 1);
  double &s_w = sPQ[3];
  int *tuvt = (int *)(sph + kSphTableDoubles + (size_t)NQ * S::PQ);
  __shared__ int s_int[NQ][3];
  int &s_ib = s_int[sub][0], &s_ic = s_int[sub][1], &s_sel = s_int[sub][2];

  for (int i = threadIdx.x; i < kBoysTableDoubles; i += blockDim.x) tab[i] = a.boys[i];
  for (int i = threadIdx.x; i < kSphTableDoubles; i += blockDim.x) sph[i] = a.sph[i];
  for (int e = threadIdx.x; e < N3L; e += blockDim.x) {
    int t, u, v;
    tuv_decode(e, t, u, v);
    tuvt[e] = t | (u << 8) | (v << 16);
  }
  __syncthreads();
  const int tid = WT ? (int)(threadIdx.x & 31) : (int)threadIdx.x;
  const int nt = WT ? 32 : (int)blockDim.x;
  auto team_sync = [&]() {
    if constexpr (WT != 0)
      __syncwarp();
    else
      __syncthreads();
  };
  const int FA = nfun(LA, a.spherical), FB = nfun(LB, a.spherical);
  const int FC = nfun(LC, a.spherical), FD = nfun(LD, a.spherical);
  unsigned long long cnt_q = 0, cnt_p = 0, cnt_s = 0;

  // One contiguous range of the queue per team: its thread 0 finds the first
  // bra once and then walks forward along the prefix sums.
  const int64_t nteam = (int64_t)gridDim.x * NQ, team = (int64_t)blockIdx.x * NQ + sub;
  const int64_t span = (a.nquartet - a.q_begin + nteam - 1) / nteam;
  const int64_t qbeg = a.q_begin + team * span, qend = min(qbeg + span, a.nquartet);
  int ibw = -1;
  for (int64_t q = qbeg; q < qend; ++q) {
    team_sync();
    if (tid == 0) {
      int ib, ic;
      if (a.diag_out) {
        ib = ic = (int)q;
      } else {
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
        ic = (int)(q - a.qoff[ib]) + (a.kbase ? a.kbase[ib] : 0);
      }
      s_ib = ib;
      s_ic = ic;
      const PairRec br = load_pair(a.bra + ib), kt = load_pair(a.ket + ic);
      s_sel = a.diag_out ? 0 : quartet_select(a, br, kt, a.bra + ib, a.ket + ic);
      double w = 1.0;
      if (br.same) w *= 0.5;
      if (kt.same) w *= 0.5;
      if (a.same_class && ib == ic + a.ket_off) w *= 0.5;
      s_w = w;
    }
    team_sync();
    if (s_sel) {
      if (tid == 0 && s_sel == 2) ++cnt_s;
      continue;
    }
    const PairRec br = load_pair(a.bra + s_ib), kt = load_pair(a.ket + s_ic);
    for (int e = tid; e < NAB * NCD; e += nt) out[e] = 0.0;
    for (int i = 0; i < br.npp; ++i) {
      const PrimPair P1 = a.pp[br.pp0 + i];
      if (tid < 3) {
        const double pa = tid == 0 ? P1.PAx : tid == 1 ? P1.PAy : P1.PAz;
        const double pb = tid == 0 ? P1.PBx : tid == 1 ? P1.PBy : P1.PBz;
        herm_e<LA, LB, 1, double>(0.5 / P1.p, pa, pb, eab + tid * EA);
      }
      for (int e = tid; e < N3AB * NCD; e += nt) X[e] = 0.0;
      for (int j = 0; j < kt.npp; ++j) {
        const PrimPair P2 = a.pp[kt.pp0 + j];
        if (tid < 3) {
          const double pa = tid == 0 ? P2.PAx : tid == 1 ? P2.PAy : P2.PAz;
          const double pb = tid == 0 ? P2.PBx : tid == 1 ? P2.PBy : P2.PBz;
          herm_e<LC, LD, -1, double>(0.5 / P2.p, pa, pb, ecd + tid * EC);
        }
        if (tid == (nt > 32 ? 32 : 3)) {
          const double p = P1.p, qq = P2.p;
          const double rs = rsqrt(p + qq);
          double alpha = p * qq * rs * rs;
          double s = P1.K * P2.K * rs;
          erf_attenuate(a.erf_mu2, alpha, s);
          const double x = P1.Px - P2.Px, y = P1.Py - P2.Py, z = P1.Pz - P2.Pz;
          double F[L + 1];
          boys_eval<L>(alpha * (x * x + y * y + z * z), tab, F);
          for (int n = 0; n <= L; ++n) {
            sF[n] = s * F[n];
            s *= -2.0 * alpha;
          }
          sPQ[0] = x;
          sPQ[1] = y;
          sPQ[2] = z;
        }
        team_sync();
        double *prev = Ra;
        if (tid == 0) prev[0] = sF[L];
        team_sync();
        const double px = sPQ[0], py = sPQ[1], pz = sPQ[2];
        for (int n = L - 1; n >= 0; --n) {
          double *cur = (prev == Ra) ? Rb : Ra;
          const int cnt = n3(L - n);
          for (int e = tid; e < cnt; e += nt) {
            double val;
            if (e == 0) {
              val = sF[n];
            } else {
              const int pk = tuvt[e];
              const int t = pk & 255, u = (pk >> 8) & 255, v = pk >> 16;
              if (t > 0) {
                val = px * prev[tuv_index(t - 1, u, v)];
                if (t > 1) val += (t - 1) * prev[tuv_index(t - 2, u, v)];
              } else if (u > 0) {
                val = py * prev[tuv_index(t, u - 1, v)];
                if (u > 1) val += (u - 1) * prev[tuv_index(t, u - 2, v)];
              } else {
                val = pz * prev[tuv_index(t, u, v - 1)];
                if (v > 1) val += (v - 1) * prev[tuv_index(t, u, v - 2)];
              }
            }
            cur[e] = val;
          }
          team_sync();
          prev = cur;
        }
        const double *R = prev;
        for (int e = tid; e < N3AB * NCD; e += nt) {
          const int tuv = e / NCD, cd = e - tuv * NCD;
          const int pk = tuvt[tuv];
          const int t = pk & 255, u = (pk >> 8) & 255, v = pk >> 16;
          const int c = cd / ND, d = cd - c * ND;
          int cx, cy, cz, dx, dy, dz;
          cart_decode(LC, c, cx, cy, cz);
          cart_decode(LD, d, dx, dy, dz);
          const double *ex = ecd + (cx * (LD + 1) + dx) * (LCD + 1);
          const double *ey = ecd + EC + (cy * (LD + 1) + dy) * (LCD + 1);
          const double *ez = ecd + 2 * EC + (cz * (LD + 1) + dz) * (LCD + 1);
          double s = 0.0;
          for (int ta = 0; ta <= cx + dx; ++ta)
            for (int na = 0; na <= cy + dy; ++na) {
              const double exy = ex[ta] * ey[na];
              for (int fa = 0; fa <= cz + dz; ++fa) s += exy * ez[fa] * R[tuv_index(t + ta, u + na, v + fa)];
            }
          X[e] += s;
        }
        team_sync();
      }
      for (int e = tid; e < NAB * NCD; e += nt) {
        const int ab = e / NCD, cd = e - ab * NCD;
        const int ia = ab / NB, ib = ab - ia * NB;
        int ax, ay, az, bx, by, bz;
        cart_decode(LA, ia, ax, ay, az);
        cart_decode(LB, ib, bx, by, bz);
        const double *ex = eab + (ax * (LB + 1) + bx) * (LAB + 1);
        const double *ey = eab + EA + (ay * (LB + 1) + by) * (LAB + 1);
        const double *ez = eab + 2 * EA + (az * (LB + 1) + bz) * (LAB + 1);
        double s = 0.0;
        for (int t = 0; t <= ax + bx; ++t)
          for (int u = 0; u <= ay + by; ++u) {
            const double exy = ex[t] * ey[u];
            for (int v = 0; v <= az + bz; ++v) s += exy * ez[v] * X[tuv_index(t, u, v) * NCD + cd];
          }
        out[e] += s;
      }
      team_sync();
    }
    cnt_q += 1;
    cnt_p += (unsigned long long)br.npp * kt.npp;

    // Cartesian -> spherical, index by index, ping-pong between out and X.
    double *res = out, *tmp = X;
    if (a.spherical && (LA >= 2 || LB >= 2 || LC >= 2 || LD >= 2)) {
      int dims[4] = {S::NA, S::NB, S::NC, S::ND};
      const int ls[4] = {LA, LB, LC, LD};
      for (int k = 0; k < 4; ++k) {
        if (ls[k] < 2) continue;
        int pre = 1, post = 1;
        for (int m = 0; m < k; ++m) pre *= dims[m];
        for (int m = k + 1; m < 4; ++m) post *= dims[m];
        sph_step(res, tmp, pre, dims[k], 2 * ls[k] + 1, post, sph + sph_offset(ls[k]), tid, nt);
        team_sync();
        dims[k] = 2 * ls[k] + 1;
        double *sw = res;
        res = tmp;
        tmp = sw;
      }
    }

    if (a.store_out) {  // conventional form: the block to the store
      double *o = a.store_out + a.store_base + q * a.store_nint;
      for (int e = tid; e < FA * FB * FC * FD; e += nt) o[e] = res[e];
      continue;
    }
    if (a.diag_out) {
      if (tid == 0) {
        double mx = 0.0;
        for (int x = 0; x < FA; ++x)
          for (int y = 0; y < FB; ++y) mx = fmax(mx, fabs(res[((x * FB + y) * FA + x) * FB + y]));
        a.diag_out[s_ib] = sqrt(mx);
      }
      continue;
    }

    const double w = s_w;
    const int aoA = br.aoA, aoB = br.aoB, aoC = kt.aoA, aoD = kt.aoB;
    const int64_t db = kt.dbase;
    const int N = kt.nbfm;
    double *Dcd = dst, *Dab = dst + 100, *Dbd = dst + 200, *Dbc = dst + 300, *Dad = dst + 400, *Dac = dst + 500;
    for (int k = 0; k < a.nslot; ++k) {
      const double *Dk = a.D + k * a.slot_stride + db;
      const double *Dsk = a.Ds + k * a.slot_stride + db;
      double *Fk = a.Fh + k * a.slot_stride + db;
      const double js = a.jscale[k] * w, ks = -a.kscale[k] * w;
      for (int e = tid; e < 100; e += nt) {
        int r = e / 10, c = e % 10;
        if (r < FC && c < FD) Dcd[r * FD + c] = Dsk[(size_t)(aoC + r) * N + aoD + c];
        if (r < FA && c < FB) Dab[r * FB + c] = Dsk[(size_t)(aoA + r) * N + aoB + c];
        if (r < FB && c < FD) Dbd[r * FD + c] = Dk[(size_t)(aoB + r) * N + aoD + c];
        if (r < FB && c < FC) Dbc[r * FC + c] = Dk[(size_t)(aoB + r) * N + aoC + c];
        if (r < FA && c < FD) Dad[r * FD + c] = Dk[(size_t)(aoA + r) * N + aoD + c];
        if (r < FA && c < FC) Dac[r * FC + c] = Dk[(size_t)(aoA + r) * N + aoC + c];
      }
      team_sync();
      const int FCD = FC * FD, FAB = FA * FB;
      if (js != 0.0) {
        for (int e = tid; e < FAB; e += nt) {
          double s = 0.0;
          for (int cd = 0; cd < FCD; ++cd) s += res[e * FCD + cd] * Dcd[cd];
          const int x = e / FB, y = e - x * FB;
          atomicAdd(Fk + (size_t)(aoA + x) * N + aoB + y, js * s);
        }
        for (int e = tid; e < FCD; e += nt) {
          double s = 0.0;
          for (int ab = 0; ab < FAB; ++ab) s += res[ab * FCD + e] * Dab[ab];
          const int x = e / FD, y = e - x * FD;
          atomicAdd(Fk + (size_t)(aoC + x) * N + aoD + y, js * s);
        }
      }
      if (ks != 0.0) {
        for (int e = tid; e < FA * FC; e += nt) {
          const int x = e / FC, c = e - x * FC;
          double s = 0.0;
          for (int b = 0; b < FB; ++b)
            for (int d = 0; d < FD; ++d) s += res[((x * FB + b) * FC + c) * FD + d] * Dbd[b * FD + d];
          atomicAdd(Fk + (size_t)(aoA + x) * N + aoC + c, ks * s);
        }
        for (int e = tid; e < FA * FD; e += nt) {
          const int x = e / FD, d = e - x * FD;
          double s = 0.0;
          for (int b = 0; b < FB; ++b)
            for (int c = 0; c < FC; ++c) s += res[((x * FB + b) * FC + c) * FD + d] * Dbc[b * FC + c];
          atomicAdd(Fk + (size_t)(aoA + x) * N + aoD + d, ks * s);
        }
        for (int e = tid; e < FB * FC; e += nt) {
          const int b = e / FC, c = e - b * FC;
          double s = 0.0;
          for (int x = 0; x < FA; ++x)
            for (int d = 0; d < FD; ++d) s += res[((x * FB + b) * FC + c) * FD + d] * Dad[x * FD + d];
          atomicAdd(Fk + (size_t)(aoB + b) * N + aoC + c, ks * s);
        }
        for (int e = tid; e < FB * FD; e += nt) {
          const int b = e / FD, d = e - b * FD;
          double s = 0.0;
          for (int x = 0; x < FA; ++x)
            for (int c = 0; c < FC; ++c) s += res[((x * FB + b) * FC + c) * FD + d] * Dac[x * FC + c];
          atomicAdd(Fk + (size_t)(aoB + b) * N + aoD + d, ks * s);
        }
      }
      team_sync();
    }
  }
  if (tid == 0 && a.counters) {
    atomicAdd(a.counters + 0, cnt_q);
    atomicAdd(a.counters + 1, cnt_p);
    atomicAdd(a.counters + 2, cnt_s);
  }
}

}  // namespace dgf
