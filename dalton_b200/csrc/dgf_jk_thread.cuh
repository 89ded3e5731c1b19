// Register-resident McMurchie-Davidson J/K quartet kernel for the low
// angular-momentum classes: one thread per contracted shell quartet, a warp
// on 32 consecutive quartets of the class-sorted queue (mostly one bra pair
// against 32 ket pairs, so bra data and the bra-side Coulomb block are
// shared across the warp).
//
// Tc is the arithmetic type of the Hermite recursion and the Hermite ->
// Cartesian contraction (double for the FP64 drop-in, float for the FP32 half
// of the mixed form).  The Boys function, the prefactor and the digestion
// (FP64 atomics into the half Fock matrices) are always FP64.
#pragma once

#include "dgf_jk_team.cuh"

namespace dgf {

// R_tuv for t+u+v <= L in place (compact index), from Fs[n] = pref (-2a)^n F_n:
// level by level from n = L-1 down to 0, each level in decreasing t+u+v so
// the level-(n+1) values it reads are still in place.
template <int L, typename T>
__device__ __forceinline__ void hermite_r_inplace(const T *Fs, T x, T y, T z, T *R) {
  R[0] = Fs[L];
#pragma unroll
  for (int n = L - 1; n >= 0; --n) {
#pragma unroll
    for (int s = L - n; s >= 1; --s) {
#pragma unroll
      for (int w = 0; w <= s; ++w) {
#pragma unroll
        for (int v = 0; v <= w; ++v) {
          const int u = w - v, t = s - w;
          T val;
          if (t > 0) {
            val = x * R[tuv_index(t - 1, u, v)];
            if (t > 1) val += T(t - 1) * R[tuv_index(t - 2, u, v)];
          } else if (u > 0) {
            val = y * R[tuv_index(t, u - 1, v)];
            if (u > 1) val += T(u - 1) * R[tuv_index(t, u - 2, v)];
          } else {
            val = z * R[tuv_index(t, u, v - 1)];
            if (v > 1) val += T(v - 1) * R[tuv_index(t, u, v - 2)];
          }
          R[tuv_index(t, u, v)] = val;
        }
      }
    }
    R[0] = Fs[n];
  }
}

__host__ __device__ constexpr int cart_x(int l, int k) {
  int s = 0;
  while ((s + 1) * (s + 2) / 2 <= k) ++s;
  return l - s;
}
__host__ __device__ constexpr int cart_z(int l, int k) {
  int s = 0;
  while ((s + 1) * (s + 2) / 2 <= k) ++s;
  return k - s * (s + 1) / 2;
}
__host__ __device__ constexpr int cart_y(int l, int k) { return l - cart_x(l, k) - cart_z(l, k); }

template <int LA, int LB, int LC, int LD, typename Tc>
__global__ void __launch_bounds__(128) jk_thread_kernel(const JKArgs a) {
  constexpr int L = LA + LB + LC + LD, LAB = LA + LB, LCD = LC + LD;
  constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  constexpr int NAB = NA * NB, NCD = NC * ND;
  constexpr int N3L = n3(L);
  constexpr int EA = (LA + 1) * (LB + 1) * (LAB + 1), EC = (LC + 1) * (LD + 1) * (LCD + 1);
  constexpr bool SPH_NEEDED = (LA >= 2 || LB >= 2 || LC >= 2 || LD >= 2);
  __shared__ double tab[kBoysTableDoubles];
  __shared__ double sph[kSphTableDoubles];
  for (int i = threadIdx.x; i < kBoysTableDoubles; i += blockDim.x) tab[i] = a.boys[i];
  for (int i = threadIdx.x; i < kSphTableDoubles; i += blockDim.x) sph[i] = a.sph[i];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int N = a.nbf;
  unsigned long long cnt_q = 0, cnt_p = 0, cnt_s = 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = a.q_begin + (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < a.nquartet;
       base += stride) {
    const int64_t q = base + lane;
    const bool active = q < a.nquartet;
    int ib0 = 0;
    if (lane == 0) ib0 = find_bra(a.qoff, a.nbra, base);
    ib0 = __shfl_sync(0xffffffffu, ib0, 0);
    int ib = ib0, ic = 0;
    int sel = 1;
    if (active) {
      int steps = 0;
      while (q >= a.qoff[ib + 1] && steps < 32) {
        ++ib;
        ++steps;
      }
      if (q >= a.qoff[ib + 1]) ib = find_bra(a.qoff, a.nbra, q);
      ic = (int)(q - a.qoff[ib]);
      sel = quartet_select(a, a.bra[ib], a.ket[ic]);
      if (sel == 2) ++cnt_s;
    }
    const bool work = active && sel == 0;
    double g[NAB * NCD];
#pragma unroll
    for (int k = 0; k < NAB * NCD; ++k) g[k] = 0.0;
    PairRec br, kt;
    if (work) {
      br = a.bra[ib];
      kt = a.ket[ic];
      Tc acc[NAB * NCD];
#pragma unroll
      for (int k = 0; k < NAB * NCD; ++k) acc[k] = Tc(0);
      for (int i = 0; i < br.npp; ++i) {
        const PrimPair P1 = a.pp[br.pp0 + i];
        Tc ex1[EA], ey1[EA], ez1[EA];
        const Tc h1 = Tc(0.5 / P1.p);
        herm_e<LA, LB, 1, Tc>(h1, Tc(P1.PAx), Tc(P1.PBx), ex1);
        herm_e<LA, LB, 1, Tc>(h1, Tc(P1.PAy), Tc(P1.PBy), ey1);
        herm_e<LA, LB, 1, Tc>(h1, Tc(P1.PAz), Tc(P1.PBz), ez1);
        for (int j = 0; j < kt.npp; ++j) {
          const PrimPair P2 = a.pp[kt.pp0 + j];
          const double rs = rsqrt(P1.p + P2.p);
          const double alpha = P1.p * P2.p * rs * rs;
          const double x = P1.Px - P2.Px, y = P1.Py - P2.Py, z = P1.Pz - P2.Pz;
          double F[L + 1];
          boys_eval<L>(alpha * (x * x + y * y + z * z), tab, F);
          Tc Fs[L + 1];
          double s = P1.K * P2.K * rs;
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
              for (int ia = 0; ia < NA; ++ia)
#pragma unroll
                for (int jb = 0; jb < NB; ++jb) {
                  const int ax = cart_x(LA, ia), ay = cart_y(LA, ia), az = cart_z(LA, ia);
                  const int bx = cart_x(LB, jb), by = cart_y(LB, jb), bz = cart_z(LB, jb);
                  Tc sum = Tc(0);
#pragma unroll
                  for (int t = 0; t <= ax + bx; ++t)
#pragma unroll
                    for (int u = 0; u <= ay + by; ++u)
#pragma unroll
                      for (int v = 0; v <= az + bz; ++v)
                        sum += ex1[(ax * (LB + 1) + bx) * (LAB + 1) + t] * ey1[(ay * (LB + 1) + by) * (LAB + 1) + u] *
                               ez1[(az * (LB + 1) + bz) * (LAB + 1) + v] * xk[tuv_index(t, u, v)];
                  acc[(ia * NB + jb) * NCD + c * ND + d] += sum;
                }
            }
        }
      }
#pragma unroll
      for (int k = 0; k < NAB * NCD; ++k) g[k] = (double)acc[k];
      cnt_q += 1;
      cnt_p += (unsigned long long)br.npp * kt.npp;
    }
    // Cartesian -> spherical for d/f shells (in registers, compile-time sizes).
    constexpr int FAc = (LA >= 2) ? 2 * LA + 1 : NA, FBc = (LB >= 2) ? 2 * LB + 1 : NB;
    constexpr int FCc = (LC >= 2) ? 2 * LC + 1 : NC, FDc = (LD >= 2) ? 2 * LD + 1 : ND;
    const bool sphr = SPH_NEEDED && a.spherical;
    if (SPH_NEEDED && sphr && work) {
      // index-by-index transform into a buffer of spherical sizes (<= Cartesian sizes)
      double tmp[NAB * NCD];
      constexpr int dims0[4] = {NA, NB, NC, ND};
      int d0 = dims0[0], d1 = dims0[1], d2 = dims0[2], d3 = dims0[3];
      (void)d0;
      if (LA >= 2) {
        const double *T = sph + sph_offset(LA);
#pragma unroll
        for (int o = 0; o < FAc; ++o)
#pragma unroll
          for (int r = 0; r < NB * NCD; ++r) {
            double s = 0.0;
#pragma unroll
            for (int x = 0; x < NA; ++x) s += T[o * NA + x] * g[x * NB * NCD + r];
            tmp[o * NB * NCD + r] = s;
          }
#pragma unroll
        for (int k = 0; k < FAc * NB * NCD; ++k) g[k] = tmp[k];
      }
      constexpr int A1 = (LA >= 2) ? FAc : NA;
      if (LB >= 2) {
        const double *T = sph + sph_offset(LB);
#pragma unroll
        for (int i = 0; i < A1; ++i)
#pragma unroll
          for (int o = 0; o < FBc; ++o)
#pragma unroll
            for (int r = 0; r < NCD; ++r) {
              double s = 0.0;
#pragma unroll
              for (int x = 0; x < NB; ++x) s += T[o * NB + x] * g[(i * NB + x) * NCD + r];
              tmp[(i * FBc + o) * NCD + r] = s;
            }
#pragma unroll
        for (int k = 0; k < A1 * FBc * NCD; ++k) g[k] = tmp[k];
      }
      constexpr int AB1 = A1 * ((LB >= 2) ? FBc : NB);
      if (LC >= 2) {
        const double *T = sph + sph_offset(LC);
#pragma unroll
        for (int i = 0; i < AB1; ++i)
#pragma unroll
          for (int o = 0; o < FCc; ++o)
#pragma unroll
            for (int r = 0; r < ND; ++r) {
              double s = 0.0;
#pragma unroll
              for (int x = 0; x < NC; ++x) s += T[o * NC + x] * g[(i * NC + x) * ND + r];
              tmp[(i * FCc + o) * ND + r] = s;
            }
#pragma unroll
        for (int k = 0; k < AB1 * FCc * ND; ++k) g[k] = tmp[k];
      }
      constexpr int ABC1 = AB1 * ((LC >= 2) ? FCc : NC);
      if (LD >= 2) {
        const double *T = sph + sph_offset(LD);
#pragma unroll
        for (int i = 0; i < ABC1; ++i)
#pragma unroll
          for (int o = 0; o < FDc; ++o) {
            double s = 0.0;
#pragma unroll
            for (int x = 0; x < ND; ++x) s += T[o * ND + x] * g[i * ND + x];
            tmp[i * FDc + o] = s;
          }
#pragma unroll
        for (int k = 0; k < ABC1 * FDc; ++k) g[k] = tmp[k];
      }
      (void)d1;
      (void)d2;
      (void)d3;
    }
    // Function counts of this launch (spherical or Cartesian basis).
    const int FA = sphr ? FAc : NA, FB = sphr ? FBc : NB, FC = sphr ? FCc : NC, FD = sphr ? FDc : ND;
    // Digestion: per slot, J_ab (warp-reduced when the warp shares its bra pair),
    // J_cd, K_ac, K_ad, K_bc, K_bd as FP64 atomics into the half Fock matrices.
    const unsigned full = 0xffffffffu;
    const bool uniform = __all_sync(full, !work || ib == ib0) && __any_sync(full, work);
    if (!__any_sync(full, work)) continue;
    double w = 0.0;
    if (work) {
      w = 1.0;
      if (br.same) w *= 0.5;
      if (kt.same) w *= 0.5;
      if (a.same_class && ib == ic) w *= 0.5;
    }
    const PairRec brw = a.bra[ib0];
    for (int k = 0; k < a.nslot; ++k) {
      const double *Dk = a.D + (size_t)k * N * N;
      const double *Dsk = a.Ds + (size_t)k * N * N;
      double *Fk = a.Fh + (size_t)k * N * N;
      const double js = a.jscale[k] * w, ks = -a.kscale[k] * w;
      if (a.jscale[k] != 0.0) {
        // J_ab
#pragma unroll
        for (int x = 0; x < NA; ++x)
#pragma unroll
          for (int y = 0; y < NB; ++y) {
            if (x >= FA || y >= FB) continue;
            double s = 0.0;
            if (work) {
#pragma unroll
              for (int c = 0; c < NC; ++c)
#pragma unroll
                for (int d = 0; d < ND; ++d)
                  if (c < FC && d < FD)
                    s += g[((x * FB + y) * FC + c) * FD + d] * Dsk[(size_t)(kt.aoA + c) * N + kt.aoB + d];
              s *= js;
            }
            if (uniform) {
#pragma unroll
              for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(full, s, off);
              if (lane == 0) atomicAdd(Fk + (size_t)(brw.aoA + x) * N + brw.aoB + y, s);
            } else if (work) {
              atomicAdd(Fk + (size_t)(br.aoA + x) * N + br.aoB + y, s);
            }
          }
        if (work) {
          // J_cd
#pragma unroll
          for (int c = 0; c < NC; ++c)
#pragma unroll
            for (int d = 0; d < ND; ++d) {
              if (c >= FC || d >= FD) continue;
              double s = 0.0;
#pragma unroll
              for (int x = 0; x < NA; ++x)
#pragma unroll
                for (int y = 0; y < NB; ++y)
                  if (x < FA && y < FB)
                    s += g[((x * FB + y) * FC + c) * FD + d] * Dsk[(size_t)(br.aoA + x) * N + br.aoB + y];
              atomicAdd(Fk + (size_t)(kt.aoA + c) * N + kt.aoB + d, js * s);
            }
        }
      }
      if (work && a.kscale[k] != 0.0) {
        // K_ac and K_ad
#pragma unroll
        for (int x = 0; x < NA; ++x) {
          if (x >= FA) continue;
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            if (c >= FC) continue;
            double s = 0.0;
#pragma unroll
            for (int y = 0; y < NB; ++y)
#pragma unroll
              for (int d = 0; d < ND; ++d)
                if (y < FB && d < FD)
                  s += g[((x * FB + y) * FC + c) * FD + d] * Dk[(size_t)(br.aoB + y) * N + kt.aoB + d];
            atomicAdd(Fk + (size_t)(br.aoA + x) * N + kt.aoA + c, ks * s);
          }
#pragma unroll
          for (int d = 0; d < ND; ++d) {
            if (d >= FD) continue;
            double s = 0.0;
#pragma unroll
            for (int y = 0; y < NB; ++y)
#pragma unroll
              for (int c = 0; c < NC; ++c)
                if (y < FB && c < FC)
                  s += g[((x * FB + y) * FC + c) * FD + d] * Dk[(size_t)(br.aoB + y) * N + kt.aoA + c];
            atomicAdd(Fk + (size_t)(br.aoA + x) * N + kt.aoB + d, ks * s);
          }
        }
        // K_bc and K_bd
#pragma unroll
        for (int y = 0; y < NB; ++y) {
          if (y >= FB) continue;
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            if (c >= FC) continue;
            double s = 0.0;
#pragma unroll
            for (int x = 0; x < NA; ++x)
#pragma unroll
              for (int d = 0; d < ND; ++d)
                if (x < FA && d < FD)
                  s += g[((x * FB + y) * FC + c) * FD + d] * Dk[(size_t)(br.aoA + x) * N + kt.aoB + d];
            atomicAdd(Fk + (size_t)(br.aoB + y) * N + kt.aoA + c, ks * s);
          }
#pragma unroll
          for (int d = 0; d < ND; ++d) {
            if (d >= FD) continue;
            double s = 0.0;
#pragma unroll
            for (int x = 0; x < NA; ++x)
#pragma unroll
              for (int c = 0; c < NC; ++c)
                if (x < FA && c < FC)
                  s += g[((x * FB + y) * FC + c) * FD + d] * Dk[(size_t)(br.aoA + x) * N + kt.aoA + c];
            atomicAdd(Fk + (size_t)(br.aoB + y) * N + kt.aoB + d, ks * s);
          }
        }
      }
    }
  }
  // warp-aggregated counters
  if (a.counters) {
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
