// Device building blocks of the McMurchie-Davidson quartet kernels:
// Boys function from the shared-memory table, Hermite expansion
// coefficients, index helpers.  Shared by the Fock, Schwarz and gradient
// kernels.
#pragma once

#include <utility>

#include "dgf_internal.h"
#include "dgf_sph.h"

namespace dgf {

// Calls f(std::integral_constant<int, i>) for i = 0 .. N-1, so that the loop
// index is a constant expression inside f (index arithmetic and term
// selection at compile time).
template <typename F, int... I>
__device__ __forceinline__ void static_for_impl(F &&f, std::integer_sequence<int, I...>) {
  (f(std::integral_constant<int, I>{}), ...);
}
template <int N, typename F>
__device__ __forceinline__ void static_for(F &&f) {
  static_for_impl(f, std::make_integer_sequence<int, N>{});
}

// One index of the Cartesian -> spherical transform with compile-time
// coefficients (zero ones drop out): for i < NI, spherical m < 2L+1, r < NR,
//   out[(i * (2L+1) + m) * NR + r] = sum_{x < N} C_L[m][X0 + x] in[(i * N + x) * NR + r]
// (X0 > 0: a chunk of the Cartesian components, the partial sums of which
// add up across chunks).
template <int L, int NI, int N, int X0, int NR, typename TI, typename TO>
__device__ __forceinline__ void sph_index(const TI *in, TO *out) {
  constexpr int M = 2 * L + 1;
#pragma unroll
  for (int i = 0; i < NI; ++i)
#pragma unroll
    for (int r = 0; r < NR; ++r)
      static_for<M>([&](auto M_) {
        constexpr int m = decltype(M_)::value;
        TO s = TO(0);
        static_for<N>([&](auto X_) {
          constexpr int x = decltype(X_)::value;
          constexpr double c = sph::coef<L>(m, X0 + x);
          if constexpr (c != 0.0) s += TO(c) * TO(in[(i * N + x) * NR + r]);
        });
        out[(i * M + m) * NR + r] = s;
      });
}

// Both indices of a shell pair block in[ncart(L1)][ncart(L2)] to spherical
// functions, out[F1][F2] (F = 2L+1 for L >= 2, ncart(L) for s and p).
template <int L1, int L2, typename T>
__device__ __forceinline__ void sph_pair(const T *in, T *out) {
  constexpr int N1 = ncart(L1), N2 = ncart(L2);
  constexpr int F1 = L1 >= 2 ? 2 * L1 + 1 : N1, F2 = L2 >= 2 ? 2 * L2 + 1 : N2;
  T t[F1 * N2];
  if constexpr (L1 >= 2) {
    sph_index<L1, 1, N1, 0, N2>(in, t);
  } else {
#pragma unroll
    for (int k = 0; k < N1 * N2; ++k) t[k] = in[k];
  }
  if constexpr (L2 >= 2) {
    sph_index<L2, F1, N2, 0, 1>(t, out);
  } else {
#pragma unroll
    for (int k = 0; k < F1 * F2; ++k) out[k] = t[k];
  }
}


__host__ __device__ constexpr int nfun(int l, int spherical) { return (spherical && l >= 2) ? 2 * l + 1 : ncart(l); }

// Compact index of (t,u,v) with t+u+v = s: s-major, then u+v, then v.
__host__ __device__ __forceinline__ int tuv_index(int t, int u, int v) {
  int s = t + u + v, w = u + v;
  return s * (s + 1) * (s + 2) / 6 + w * (w + 1) / 2 + v;
}

// Inverse of tuv_index.
__host__ __device__ __forceinline__ void tuv_decode(int e, int &t, int &u, int &v) {
  int s = 0;
  while (n3(s) <= e) ++s;
  int r = e - s * (s + 1) * (s + 2) / 6;
  int w = 0;
  while ((w + 1) * (w + 2) / 2 <= r) ++w;
  v = r - w * (w + 1) / 2;
  u = w - v;
  t = s - w;
}

// Cartesian exponents of component k of shell l in Dalton order
// (xx, xy, xz, yy, yz, zz): k = s(s+1)/2 + z with s = y + z.
__host__ __device__ __forceinline__ void cart_decode(int l, int k, int &x, int &y, int &z) {
  int s = 0;
  while ((s + 1) * (s + 2) / 2 <= k) ++s;
  z = k - s * (s + 1) / 2;
  y = s - z;
  x = l - s;
}

// Polynomial of degree DEG in x (coefficients c[0..DEG]) by Estrin's scheme:
// the dependency depth grows with log2(DEG) instead of DEG.
template <int DEG>
__device__ __forceinline__ double poly_estrin(const double *__restrict__ c, double x) {
  static_assert(DEG == 11 || DEG == 5, "Boys tables are degree 11 or 5");
  const double x2 = x * x;
  if (DEG == 5) {
    const double p01 = fma(c[1], x, c[0]), p23 = fma(c[3], x, c[2]), p45 = fma(c[5], x, c[4]);
    return fma(fma(p45, x2, p23), x2, p01);
  }
  const double x4 = x2 * x2;
  const double p01 = fma(c[1], x, c[0]), p23 = fma(c[3], x, c[2]), p45 = fma(c[5], x, c[4]);
  const double p67 = fma(c[7], x, c[6]), p89 = fma(c[9], x, c[8]), pab = fma(c[11], x, c[10]);
  const double q0 = fma(p23, x2, p01), q1 = fma(p67, x2, p45), q2 = fma(pab, x2, p89);
  return fma(fma(q2, x4, q1), x4, q0);
}

// F_0..F_M(T): table polynomial for F_M below kBoysTmax then downward
// recursion F_m = (2T F_{m+1} + e^-T)/(2m+1); above it F_0 = sqrt(pi/T)/2
// and upward recursion F_{m+1} = ((2m+1) F_m - e^-T)/(2T).  DEG 11 is the
// full-accuracy table (relative error ~1e-16); DEG 5 is the table of the
// FP32 half of the mixed form (relative error ~2e-8, FP64 arithmetic).
template <int M, int DEG = kBoysDeg>
__device__ __forceinline__ void boys_eval(double T, const double *__restrict__ tab, double *F) {
  // e^-T is formed once, ahead of the branch: the lanes of a warp often fall
  // on both sides of kBoysTmax, and then both branches run.
  double et = 0.0;
  if (M > 0) et = exp(-T);
  if (T < kBoysTmax) {
    int i = (int)(T * kBoysPerUnit);
    double x = (T - (i + 0.5) * (1.0 / kBoysPerUnit)) * (2.0 * kBoysPerUnit);
    F[M] = poly_estrin<DEG>(tab + i * kBoysNcoef, x);
    if (M > 0) {
      const double t2 = 2.0 * T;
#pragma unroll
      for (int m = M - 1; m >= 0; --m) F[m] = fma(t2, F[m + 1], et) * (1.0 / (2 * m + 1));
    }
  } else {
    double rt = rsqrt(T);
    F[0] = 0.88622692545275801364908374167057 * rt;
    if (M > 0) {
      const double h = 0.5 * rt * rt;
#pragma unroll
      for (int m = 0; m < M; ++m) F[m + 1] = fma((double)(2 * m + 1), F[m], -et) * h;
    }
  }
}

// The attenuated Coulomb operator erf(mu r12)/r12 of range-separated
// exchange (Dalton's HFXMU pass, DALTON/abacus/her2her.F:344-353): with
// beta = mu^2 / (alpha + mu^2), R^n_000 takes alpha * beta in place of alpha,
// in the Boys argument and in (-2 alpha)^n, and its prefactor gains
// sqrt(beta).  mu2 = 0 leaves the plain 1/r12 operator.
__device__ __forceinline__ void erf_attenuate(double mu2, double &alpha, double &pref) {
  if (mu2 > 0.0) {
    const double beta = mu2 / (alpha + mu2);
    alpha *= beta;
    pref *= sqrt(beta);
  }
}

// Hermite expansion coefficients of one direction, E^{ij}_t for i <= LA,
// j <= LB, t <= i+j, E^{00}_0 = 1; layout E[(i*(LB+1)+j)*(LA+LB+1)+t].
// h = 1/(2p).  SIGN = -1 multiplies E_t by (-1)^t (ket side of the MD sum).
template <int LA, int LB, int SIGN, typename T>
__device__ __forceinline__ void herm_e(T h, T pa, T pb, T *E) {
  constexpr int NT = LA + LB + 1;
#pragma unroll
  for (int k = 0; k < (LA + 1) * (LB + 1) * NT; ++k) E[k] = T(0);
  E[0] = T(1);
#pragma unroll
  for (int i = 0; i <= LA; ++i) {
#pragma unroll
    for (int j = 0; j <= LB; ++j) {
      if (i == 0 && j == 0) continue;
      const int pi = (i > 0) ? i - 1 : 0, pj = (i > 0) ? j : j - 1;
      const T x = (i > 0) ? pa : pb;
      const int top = pi + pj;
      const T *prev = E + (pi * (LB + 1) + pj) * NT;
      T *cur = E + (i * (LB + 1) + j) * NT;
#pragma unroll
      for (int t = 0; t <= i + j; ++t) {
        T v = (t <= top) ? x * prev[t] : T(0);
        if (t > 0) v += h * prev[t - 1];
        if (t + 1 <= top) v += T(t + 1) * prev[t + 1];
        cur[t] = v;
      }
    }
  }
  if (SIGN < 0) {
#pragma unroll
    for (int k = 0; k < (LA + 1) * (LB + 1) * NT; ++k)
      if ((k % NT) & 1) E[k] = -E[k];
  }
}

// Maps a flattened quartet index to (bra, ket) through the prefix array.
// Pair records through the read-only data path, 16 bytes at a time (the
// records are 16-byte aligned); load_prim<false> skips P-A and P-B, which
// (ss) pairs do not use.
__device__ __forceinline__ PairRec load_pair(const PairRec *p) {
  PairRec r;
  const int4 *s = reinterpret_cast<const int4 *>(p);
  int4 *d = reinterpret_cast<int4 *>(&r);
#pragma unroll
  for (int k = 0; k < (int)(sizeof(PairRec) / 16); ++k) d[k] = __ldg(s + k);
  return r;
}

// The fields of a pair record the Fock kernels read (all but the atoms).
__device__ __forceinline__ PairRec load_pair_fock(const PairRec *p) {
  PairRec r;
  const int4 *s = reinterpret_cast<const int4 *>(p);
  int4 *d = reinterpret_cast<int4 *>(&r);
#pragma unroll
  for (int k = 0; k < 3; ++k) d[k] = __ldg(s + k);
  d[3] = make_int4(0, 0, 0, 0);
  return r;
}

// Dalton blocks of a pair's shells: {block A, block B, A whole, B whole}.
__device__ __forceinline__ int4 block_of_pair(const PairRec *p) {
  const int4 v = __ldg(reinterpret_cast<const int4 *>(p) + 3);  // atA, atB, blkA, blkB
  return make_int4(v.z & (kWholeBlock - 1), v.w & (kWholeBlock - 1), (v.z & kWholeBlock) ? 1 : 0,
                   (v.w & kWholeBlock) ? 1 : 0);
}

template <bool PAB>
__device__ __forceinline__ PrimPair load_prim(const PrimPair *p) {
  PrimPair r;
  const double2 *s = reinterpret_cast<const double2 *>(p);
  double2 *d = reinterpret_cast<double2 *>(&r);
  d[0] = __ldg(s + 0);  // p, Px
  d[1] = __ldg(s + 1);  // Py, Pz
  if (PAB) {
    d[2] = __ldg(s + 2);  // PAx, PAy
    d[3] = __ldg(s + 3);  // PAz, PBx
    d[4] = __ldg(s + 4);  // PBy, PBz
  } else {
    d[2] = d[3] = d[4] = make_double2(0.0, 0.0);
  }
  d[5] = __ldg(s + 5);  // K, ea
  return r;
}

__device__ __forceinline__ int find_bra(const int64_t *__restrict__ qoff, int nbra, int64_t q) {
  int lo = 0, hi = nbra;
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (qoff[mid] <= q)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

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

}  // namespace dgf
