// Cartesian -> real spherical harmonic transformation coefficients in
// Dalton's convention, computed at compile time so that kernels can use
// them as immediate constants (zero coefficients drop out of the code).
//
// The generator follows SPHCO1 (DALTON/abacus/her1pro.F:4716-4770) with
// MINTEG = 2 and MORDER = 1: Legendre coefficients PL, the COSSIN
// recurrence of (x + i y)^m, the normalisation CM = sqrt(2 (l-m)!/(l+m)!)
// / sqrt((2l-1)!!) (1 for m = 0), and Dalton's row order (m = -l..l, the
// cosine component of m at row l+m, the sine component at row l-m) and
// Cartesian column order.  The host table of the kernels' shared-memory
// copy (sph_table_host) is filled from the same generator.
#pragma once

namespace dgf {
namespace sph {

constexpr int kMaxL = 4;  // tables for l = 0..4 (f shells and their gradient)

constexpr int ncart_c(int l) { return (l + 1) * (l + 2) / 2; }

// Square root by Newton's iteration in double (a constant-expression
// stand-in for std::sqrt; it stops when the iterates stop falling, within
// an ulp of the rounded root).
constexpr double csqrt(double x) {
  if (x <= 0.0) return 0.0;
  double r = x > 1.0 ? x : 1.0;  // from above, the iterates fall monotonically
  for (int i = 0; i < 200; ++i) {
    const double n = 0.5 * (r + x / r);
    if (!(n < r)) break;
    r = n;
  }
  return r;
}

constexpr double binom(int n, int k) {
  if (k < 0 || k > n) return 0.0;
  double r = 1.0;
  for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
  return r;
}

constexpr double fact(int n) {
  double r = 1.0;
  for (int i = 2; i <= n; ++i) r *= i;
  return r;
}

// (2l+1) x ncart(l) coefficients of one l, row-major.
struct Table {
  double c[(2 * kMaxL + 1) * ((kMaxL + 1) * (kMaxL + 2) / 2)] = {};
};

constexpr Table make(int l) {
  Table t{};
  const int nx = ncart_c(l);
  if (l <= 1) {
    for (int i = 0; i < nx; ++i) t.c[i * nx + i] = 1.0;
    return t;
  }
  double pl[kMaxL + 2] = {};
  double cs[(kMaxL + 1) * (kMaxL + 1)] = {};
  double two_l = 1.0;
  for (int i = 0; i < l; ++i) two_l *= 2.0;
  for (int k = 0; k <= l / 2; ++k)
    pl[l - 2 * k] = ((k % 2) ? -1.0 : 1.0) / two_l * binom(l, k) * binom(2 * (l - k), l);
  cs[0] = 1.0;
  for (int m = 1; m <= l; ++m) {
    cs[m * (l + 1)] = 1.0;
    for (int k = 1; k <= m; ++k) {
      cs[m * (l + 1) + k] = cs[(m - 1) * (l + 1) + k - 1] * (((k - 1) % 2) ? -1.0 : 1.0);
      if (m > k) cs[m * (l + 1) + k] += cs[(m - 1) * (l + 1) + k];
    }
  }
  double df = 1.0;
  for (int v = 2 * l - 1; v > 0; v -= 2) df *= v;
  for (int m = 0; m <= l; ++m) {
    double cm = (m == 0) ? 1.0 : csqrt(2.0 * fact(l - m) / fact(l + m));
    cm /= csqrt(df);
    for (int k = (l - m) % 2; k <= l - m; k += 2) {
      if (m > 0) pl[k] = (k + 1) * pl[k + 1];
      const double cmk = cm * pl[k];
      for (int i = 0; i <= (l - k - m) / 2; ++i) {
        const double cmki = cmk * binom((l - k - m) / 2, i);
        for (int j = 0; j <= i; ++j) {
          const double cmkij = cmki * binom(i, j);
          for (int nn = 0; nn <= m; ++nn) {
            int ix = l - 2 * j - m + nn;
            ix = ix * (ix + 1) / 2 + l + 1 - m - 2 * i;          // 1-based Cartesian index
            const int ilm = (nn % 2 == 1) ? (l - m) : (l + m);  // 0-based row
            t.c[ilm * nx + (ix - 1)] += cmkij * cs[m * (l + 1) + nn];
          }
        }
      }
    }
  }
  return t;
}

template <int L>
struct Tab {
  static constexpr Table t = make(L);
};

// Coefficient of Cartesian component x in spherical component m (row) of l.
template <int L>
constexpr double coef(int m, int x) {
  return Tab<L>::t.c[m * ncart_c(L) + x];
}

}  // namespace sph
}  // namespace dgf
