// CPU oracle for the direct J/K Fock build — TEST INFRASTRUCTURE ONLY.
//
// A plain restatement of Dalton's HERMIT McMurchie-Davidson two-electron path
// and of the one-electron/gradient pieces a full RHF energy and gradient
// need.  It is the checker for the CUDA library; nothing in the product links
// it.  Each function names the Dalton routine (path inside the Dalton tree)
// whose arithmetic it restates.  Parity pins: see oracle.h.
#include "oracle.h"

#include <omp.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <vector>

namespace {

const double kPi = 3.14159265358979323846264338327950288;
int g_threads = 0;

inline int ncart(int l) { return (l + 1) * (l + 2) / 2; }

// Dalton Cartesian order: x-exponent descending, then y descending
// (xx, xy, xz, yy, yz, zz) — DALTON/abacus/hergam.F:164-218.
// Tables are built once (l <= 8) and returned by reference.
const std::vector<std::array<int, 3>> &cart_list(int l) {
  static const std::vector<std::vector<std::array<int, 3>>> tab = [] {
    std::vector<std::vector<std::array<int, 3>>> t(9);
    for (int ll = 0; ll <= 8; ++ll)
      for (int i = ll; i >= 0; --i)
        for (int j = ll - i; j >= 0; --j) t[ll].push_back({i, j, ll - i - j});
    return t;
  }();
  return tab[l];
}

double binom(int n, int k) {
  if (k < 0 || k > n) return 0.0;
  double r = 1.0;
  for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
  return r;
}
double fact(int n) {
  double r = 1.0;
  for (int i = 2; i <= n; ++i) r *= i;
  return r;
}

// Cartesian -> spherical (SPHCO1, DALTON/abacus/her1pro.F:4697-4770, MORDER=1,
// MINTEG=2): out[(m+l)*ncart + ix].
std::vector<double> sph_matrix(int l) {
  int nx = ncart(l), nlm = 2 * l + 1;
  std::vector<double> tr(nx * nlm, 0.0);  // tr[ix*nlm + ilm]
  if (l <= 1) {
    std::vector<double> out(nlm * nx, 0.0);
    for (int i = 0; i < nx; ++i) out[i * nx + i] = 1.0;
    return out;
  }
  std::vector<double> pl(l + 2, 0.0);
  for (int k = 0; k <= l / 2; ++k)
    pl[l - 2 * k] = std::pow(-1.0, k) * std::pow(2.0, -l) * binom(l, k) * binom(2 * (l - k), l);
  std::vector<double> cs((l + 1) * (l + 1), 0.0);
  auto CS = [&](int m, int k) -> double & { return cs[m * (l + 1) + k]; };
  CS(0, 0) = 1.0;
  for (int m = 1; m <= l; ++m) {
    CS(m, 0) = 1.0;
    for (int k = 1; k <= m; ++k) {
      CS(m, k) = CS(m - 1, k - 1) * std::pow(-1.0, k - 1);
      if (m > k) CS(m, k) += CS(m - 1, k);
    }
  }
  double df = 1.0;
  for (int v = 2 * l - 1; v > 0; v -= 2) df *= v;
  for (int m = 0; m <= l; ++m) {
    double cm = (m == 0) ? 1.0 : std::sqrt(2.0 * fact(l - m) / fact(l + m));
    cm /= std::sqrt(df);
    for (int k = (l - m) % 2; k <= l - m; k += 2) {
      if (m > 0) pl[k] = (k + 1) * pl[k + 1];
      double cmk = cm * pl[k];
      for (int i = 0; i <= (l - k - m) / 2; ++i) {
        double cmki = cmk * binom((l - k - m) / 2, i);
        for (int j = 0; j <= i; ++j) {
          double cmkij = cmki * binom(i, j);
          for (int n = 0; n <= m; ++n) {
            int ix = l - 2 * j - m + n;
            ix = ix * (ix + 1) / 2 + l + 1 - m - 2 * i;
            int ilm = (n % 2 == 1) ? (1 + l - m) : (1 + l + m);
            tr[(ix - 1) * nlm + (ilm - 1)] += cmkij * CS(m, n);
          }
        }
      }
    }
  }
  std::vector<double> out(nlm * nx);
  for (int i = 0; i < nlm; ++i)
    for (int x = 0; x < nx; ++x) out[i * nx + x] = tr[x * nlm + i];
  return out;
}

// Boys function F_0..F_m(t): series for the top order then downward
// recursion for t < 50; F_0 from erf and upward recursion beyond.  Written
// from the defining integral, not from Dalton's tabulation (GETGAM,
// DALTON/abacus/her2her.F:856).
void boys(int m, double t, double *f) {
  if (t < 50.0) {
    double et = std::exp(-t);
    double term = 1.0 / (2 * m + 1), sum = term;
    for (int k = 1; k < 2000; ++k) {
      term *= 2.0 * t / (2 * m + 2 * k + 1);
      sum += term;
      if (term < 1e-18 * sum) break;
    }
    f[m] = et * sum;
    for (int j = m - 1; j >= 0; --j) f[j] = (2.0 * t * f[j + 1] + et) / (2 * j + 1);
  } else {
    double et = std::exp(-t);
    f[0] = 0.5 * std::sqrt(kPi / t) * std::erf(std::sqrt(t));
    for (int j = 0; j < m; ++j) f[j + 1] = ((2 * j + 1) * f[j] - et) / (2.0 * t);
  }
}

// Hermite expansion coefficients E^{ij}_t of one Cartesian direction
// (ODCOEF/EXCOEF, DALTON/abacus/her2odc.F:805,890), E^{00}_0 = 1.
// Layout: E[(i*(lb+1)+j)*(la+lb+1)+t].
void hermite_e(int la, int lb, double p, double pa, double pb, std::vector<double> &E) {
  int nt = la + lb + 1;
  E.assign((la + 1) * (lb + 1) * nt, 0.0);
  auto at = [&](int i, int j, int t) -> double & { return E[(i * (lb + 1) + j) * nt + t]; };
  double h = 0.5 / p;
  at(0, 0, 0) = 1.0;
  for (int i = 0; i <= la; ++i) {
    for (int j = 0; j <= lb; ++j) {
      if (i == 0 && j == 0) continue;
      if (i > 0) {
        for (int t = 0; t <= i + j; ++t) {
          double v = pa * ((t <= i - 1 + j) ? at(i - 1, j, t) : 0.0);
          if (t > 0) v += h * at(i - 1, j, t - 1);
          if (t + 1 <= i - 1 + j) v += (t + 1) * at(i - 1, j, t + 1);
          at(i, j, t) = v;
        }
      } else {
        for (int t = 0; t <= j; ++t) {
          double v = pb * ((t <= j - 1) ? at(0, j - 1, t) : 0.0);
          if (t > 0) v += h * at(0, j - 1, t - 1);
          if (t + 1 <= j - 1) v += (t + 1) * at(0, j - 1, t + 1);
          at(0, j, t) = v;
        }
      }
    }
  }
}

// Hermite Coulomb integrals R_{tuv} (HERI/HRECUR, DALTON/abacus/her2her.F:991,1086):
// R^n_{000} = (-2 alpha)^n F_n(alpha |PQ|^2); out R[(t*(L+1)+u)*(L+1)+v] for t+u+v <= L.
struct RWork {
  std::vector<double> r, f;
};
void hermite_r(int L, double alpha, double x, double y, double z, RWork &w, std::vector<double> &out) {
  int n1 = L + 1;
  size_t lev = (size_t)n1 * n1 * n1;
  w.r.assign(lev * n1, 0.0);
  w.f.resize(L + 1);
  boys(L, alpha * (x * x + y * y + z * z), w.f.data());
  auto R = [&](int n, int t, int u, int v) -> double & { return w.r[n * lev + (t * n1 + u) * n1 + v]; };
  double s = 1.0;
  for (int n = 0; n <= L; ++n) {
    R(n, 0, 0, 0) = s * w.f[n];
    s *= -2.0 * alpha;
  }
  for (int n = L - 1; n >= 0; --n) {
    int top = L - n;
    for (int t = 0; t <= top; ++t)
      for (int u = 0; u <= top - t; ++u)
        for (int v = 0; v <= top - t - u; ++v) {
          if (t + u + v == 0) continue;
          double val;
          if (t > 0) {
            val = x * R(n + 1, t - 1, u, v);
            if (t > 1) val += (t - 1) * R(n + 1, t - 2, u, v);
          } else if (u > 0) {
            val = y * R(n + 1, t, u - 1, v);
            if (u > 1) val += (u - 1) * R(n + 1, t, u - 2, v);
          } else {
            val = z * R(n + 1, t, u, v - 1);
            if (v > 1) val += (v - 1) * R(n + 1, t, u, v - 2);
          }
          R(n, t, u, v) = val;
        }
  }
  out.assign(lev, 0.0);
  for (size_t i = 0; i < lev; ++i) out[i] = w.r[i];
}

struct Shell {
  int l, atom, nprim, ao, nf;
  int blk;  // Dalton block (atom, l, general contraction) the shell comes from
  double xyz[3];
  std::vector<double> a, c;
};

struct Basis {
  int nbf, natom, spherical, maxl;
  std::vector<Shell> sh;
  std::vector<int> blk_ao0, blk_nfun;  // per Dalton block: first AO function, number of functions
  std::vector<double> xyz, charge;
  std::vector<std::vector<double>> sph;  // per l: nf x ncart
};

// Split Dalton's general-contraction blocks into one shell per contracted
// function, dropping zero coefficients; AO offsets keep Dalton's C1 order.
Basis make_basis(const orc_basis *b) {
  Basis B;
  B.nbf = (int)b->nbf;
  B.natom = (int)b->natom;
  B.spherical = (int)b->spherical;
  B.maxl = 0;
  B.xyz.assign(b->atom_xyz, b->atom_xyz + 3 * b->natom);
  B.charge.assign(b->atom_charge, b->atom_charge + b->natom);
  for (int ib = 0; ib < b->nblock; ++ib) {
    int l = (int)b->block_l[ib];
    int np = (int)b->block_nprim[ib], nc = (int)b->block_ncontr[ib];
    int nf = (B.spherical && l >= 2) ? 2 * l + 1 : ncart(l);
    B.maxl = std::max(B.maxl, l);
    B.blk_ao0.push_back((int)b->block_ao_offset[ib]);
    B.blk_nfun.push_back(nc * nf);
    for (int k = 0; k < nc; ++k) {
      Shell s;
      s.l = l;
      s.blk = ib;
      s.atom = (int)b->block_atom[ib];
      s.ao = (int)b->block_ao_offset[ib] + k * nf;
      s.nf = nf;
      for (int d = 0; d < 3; ++d) s.xyz[d] = B.xyz[3 * s.atom + d];
      for (int i = 0; i < np; ++i) {
        double cc = b->coef[b->block_coef_offset[ib] + (size_t)k * np + i];
        if (cc != 0.0) {
          s.a.push_back(b->prim_exp[b->block_prim_offset[ib] + i]);
          s.c.push_back(cc);
        }
      }
      s.nprim = (int)s.a.size();
      B.sh.push_back(s);
    }
  }
  for (int l = 0; l <= B.maxl + 1; ++l) {
    if (B.spherical && l >= 2)
      B.sph.push_back(sph_matrix(l));
    else {
      int n = ncart(l);
      std::vector<double> e(n * n, 0.0);
      for (int i = 0; i < n; ++i) e[i * n + i] = 1.0;
      B.sph.push_back(e);
    }
  }
  return B;
}

// Primitive Cartesian ERI block for arbitrary (la lb|lc ld) (R0001 prefactor,
// HERI, C1/C2 Hermite->Cartesian: DALTON/abacus/her2her.F:248-854,
// her2el1.F, her2el2.F).  out[((a*ncb+b)*ncc+c)*ncd+d] += scale*(ab|cd).
struct EriWork {
  std::vector<double> ex1, ey1, ez1, ex2, ey2, ez2, R, X;
  RWork rw;
  // > 0: the attenuated operator erf(mu r12)/r12 with mu^2 = mu2 (HFXMU
  // branch of R0001, DALTON/abacus/her2her.F:344-353); 0: 1/r12.
  double mu2 = 0.0;
};
void prim_eri(int la, int lb, int lc, int ld, double a, double b, double c, double d, const double *A,
              const double *Bc, const double *C, const double *D, double scale, double *out, EriWork &w) {
  double p = a + b, q = c + d;
  double P[3], Q[3];
  for (int i = 0; i < 3; ++i) {
    P[i] = (a * A[i] + b * Bc[i]) / p;
    Q[i] = (c * C[i] + d * D[i]) / q;
  }
  double ab2 = 0, cd2 = 0;
  for (int i = 0; i < 3; ++i) {
    ab2 += (A[i] - Bc[i]) * (A[i] - Bc[i]);
    cd2 += (C[i] - D[i]) * (C[i] - D[i]);
  }
  double kab = std::exp(-a * b / p * ab2), kcd = std::exp(-c * d / q * cd2);
  double alpha = p * q / (p + q);
  double pref = 2.0 * std::pow(kPi, 2.5) / (p * q * std::sqrt(p + q)) * kab * kcd * scale;
  if (w.mu2 > 0.0) {  // BETA = HFXMU^2 / (ALPHA + HFXMU^2): alpha -> alpha*beta, prefactor * sqrt(beta)
    const double beta = w.mu2 / (alpha + w.mu2);
    alpha *= beta;
    pref *= std::sqrt(beta);
  }
  hermite_e(la, lb, p, P[0] - A[0], P[0] - Bc[0], w.ex1);
  hermite_e(la, lb, p, P[1] - A[1], P[1] - Bc[1], w.ey1);
  hermite_e(la, lb, p, P[2] - A[2], P[2] - Bc[2], w.ez1);
  hermite_e(lc, ld, q, Q[0] - C[0], Q[0] - D[0], w.ex2);
  hermite_e(lc, ld, q, Q[1] - C[1], Q[1] - D[1], w.ey2);
  hermite_e(lc, ld, q, Q[2] - C[2], Q[2] - D[2], w.ez2);
  int L = la + lb + lc + ld, n1 = L + 1;
  hermite_r(L, alpha, P[0] - Q[0], P[1] - Q[1], P[2] - Q[2], w.rw, w.R);
  int Lab = la + lb, Lcd = lc + ld;
  const auto &ca = cart_list(la), &cb = cart_list(lb), &cc = cart_list(lc), &cd = cart_list(ld);
  int nab1 = Lab + 1, ncd1 = Lcd + 1;
  size_t box = (size_t)nab1 * nab1 * nab1;
  int ncc = (int)cc.size(), ncdd = (int)cd.size();
  w.X.assign(box * ncc * ncdd, 0.0);
  // ket transform: X[(c,d)][tuv] = sum (-1)^(tau+nu+phi) Ecd R[t+tau,u+nu,v+phi]
  for (int ic = 0; ic < ncc; ++ic)
    for (int id = 0; id < ncdd; ++id) {
      int cx = cc[ic][0], cy = cc[ic][1], cz = cc[ic][2];
      int dx = cd[id][0], dy = cd[id][1], dz = cd[id][2];
      double *Xcd = &w.X[(ic * ncdd + id) * box];
      for (int tau = 0; tau <= cx + dx; ++tau) {
        double e1 = w.ex2[(cx * (ld + 1) + dx) * ncd1 + tau];
        if (e1 == 0.0) continue;
        for (int nu = 0; nu <= cy + dy; ++nu) {
          double e2 = e1 * w.ey2[(cy * (ld + 1) + dy) * ncd1 + nu];
          if (e2 == 0.0) continue;
          for (int phi = 0; phi <= cz + dz; ++phi) {
            double e3 = e2 * w.ez2[(cz * (ld + 1) + dz) * ncd1 + phi];
            if ((tau + nu + phi) & 1) e3 = -e3;
            for (int t = 0; t <= Lab; ++t)
              for (int u = 0; u <= Lab - t; ++u)
                for (int v = 0; v <= Lab - t - u; ++v)
                  Xcd[(t * nab1 + u) * nab1 + v] += e3 * w.R[((t + tau) * n1 + (u + nu)) * n1 + (v + phi)];
          }
        }
      }
    }
  int ncbb = (int)cb.size();
  for (int ia = 0; ia < (int)ca.size(); ++ia)
    for (int ib = 0; ib < ncbb; ++ib) {
      int ax = ca[ia][0], ay = ca[ia][1], az = ca[ia][2];
      int bx = cb[ib][0], by = cb[ib][1], bz = cb[ib][2];
      double *o = out + (size_t)(ia * ncbb + ib) * ncc * ncdd;
      for (int t = 0; t <= ax + bx; ++t) {
        double e1 = w.ex1[(ax * (lb + 1) + bx) * nab1 + t];
        if (e1 == 0.0) continue;
        for (int u = 0; u <= ay + by; ++u) {
          double e2 = e1 * w.ey1[(ay * (lb + 1) + by) * nab1 + u];
          if (e2 == 0.0) continue;
          for (int v = 0; v <= az + bz; ++v) {
            double e3 = pref * e2 * w.ez1[(az * (lb + 1) + bz) * nab1 + v];
            size_t idx = (t * nab1 + u) * nab1 + v;
            for (int k = 0; k < ncc * ncdd; ++k) o[k] += e3 * w.X[k * box + idx];
          }
        }
      }
    }
}

// Transform a Cartesian 4-index block to the shells' (spherical) functions.
void cart_to_sph4(const Basis &B, int la, int lb, int lc, int ld, const std::vector<double> &cart,
                  std::vector<double> &out, std::vector<double> &tmp) {
  int n[4] = {ncart(la), ncart(lb), ncart(lc), ncart(ld)};
  int ls[4] = {la, lb, lc, ld};
  int f[4];
  for (int i = 0; i < 4; ++i) f[i] = (B.spherical && ls[i] >= 2) ? 2 * ls[i] + 1 : n[i];
  // transform index by index: dims cur[0..3]
  std::vector<double> cur = cart;
  int dims[4] = {n[0], n[1], n[2], n[3]};
  for (int k = 0; k < 4; ++k) {
    const std::vector<double> &T = B.sph[ls[k]];
    int nin = dims[k], nout = f[k];
    int pre = 1, post = 1;
    for (int i = 0; i < k; ++i) pre *= dims[i];
    for (int i = k + 1; i < 4; ++i) post *= dims[i];
    tmp.assign((size_t)pre * nout * post, 0.0);
    for (int i = 0; i < pre; ++i)
      for (int o = 0; o < nout; ++o)
        for (int x = 0; x < nin; ++x) {
          double t = T[o * nin + x];
          if (t == 0.0) continue;
          const double *src = &cur[((size_t)i * nin + x) * post];
          double *dst = &tmp[((size_t)i * nout + o) * post];
          for (int j = 0; j < post; ++j) dst[j] += t * src[j];
        }
    cur.swap(tmp);
    dims[k] = nout;
  }
  out.swap(cur);
}

// Contracted spherical ERI block of a segmented shell quartet.
void shell_eri(const Basis &B, int iA, int iB, int iC, int iD, std::vector<double> &out, EriWork &w,
               std::vector<double> &cart, std::vector<double> &tmp) {
  const Shell &A = B.sh[iA], &Bs = B.sh[iB], &C = B.sh[iC], &D = B.sh[iD];
  size_t nc = (size_t)ncart(A.l) * ncart(Bs.l) * ncart(C.l) * ncart(D.l);
  cart.assign(nc, 0.0);
  for (int i = 0; i < A.nprim; ++i)
    for (int j = 0; j < Bs.nprim; ++j)
      for (int k = 0; k < C.nprim; ++k)
        for (int m = 0; m < D.nprim; ++m)
          prim_eri(A.l, Bs.l, C.l, D.l, A.a[i], Bs.a[j], C.a[k], D.a[m], A.xyz, Bs.xyz, C.xyz, D.xyz,
                   A.c[i] * Bs.c[j] * C.c[k] * D.c[m], cart.data(), w);
  cart_to_sph4(B, A.l, Bs.l, C.l, D.l, cart, out, tmp);
}

// Schwarz factors on segmented shell pairs (GABGEN/GABDRV, DALTON/abacus/her2gab.F:36,1776).
std::vector<double> schwarz(const Basis &B) {
  int ns = (int)B.sh.size();
  std::vector<double> Q((size_t)ns * ns, 0.0);
#pragma omp parallel
  {
    EriWork w;
    std::vector<double> out, cart, tmp;
#pragma omp for schedule(dynamic)
    for (int a = 0; a < ns; ++a)
      for (int b = 0; b <= a; ++b) {
        shell_eri(B, a, b, a, b, out, w, cart, tmp);
        int fa = B.sh[a].nf, fb = B.sh[b].nf;
        double mx = 0;
        for (int i = 0; i < fa; ++i)
          for (int j = 0; j < fb; ++j) mx = std::max(mx, std::fabs(out[((i * fb + j) * fa + i) * fb + j]));
        Q[(size_t)a * ns + b] = Q[(size_t)b * ns + a] = std::sqrt(mx);
      }
  }
  return Q;
}

void set_threads() {
  if (g_threads > 0) omp_set_num_threads(g_threads);
}

}  // namespace

extern "C" {

void orc_set_threads(int n) { g_threads = n; }
int orc_get_threads(void) {
  set_threads();
  int n = 1;
#pragma omp parallel
  {
#pragma omp single
    n = omp_get_num_threads();
  }
  return n;
}

void orc_boys(int m, double t, double *f) { boys(m, t, f); }

void orc_sph_matrix(int l, double *out) {
  auto m = sph_matrix(l);
  std::memcpy(out, m.data(), m.size() * sizeof(double));
}

int orc_nshell(const orc_basis *b) { return (int)make_basis(b).sh.size(); }

int orc_schwarz(const orc_basis *b, double *q, int64_t *shell_l, int64_t *shell_nprim, int64_t *shell_atom) {
  set_threads();
  Basis B = make_basis(b);
  std::vector<double> Q = schwarz(B);
  std::memcpy(q, Q.data(), Q.size() * sizeof(double));
  for (size_t i = 0; i < B.sh.size(); ++i) {
    shell_l[i] = B.sh[i].l;
    shell_nprim[i] = B.sh[i].nprim;
    shell_atom[i] = B.sh[i].atom;
  }
  return 0;
}

int orc_eri_full(const orc_basis *b, double *eri) {
  set_threads();
  Basis B = make_basis(b);
  int ns = (int)B.sh.size();
  size_t N = B.nbf;
#pragma omp parallel
  {
    EriWork w;
    std::vector<double> out, cart, tmp;
#pragma omp for schedule(dynamic) collapse(2)
    for (int a = 0; a < ns; ++a)
      for (int bb = 0; bb < ns; ++bb)
        for (int c = 0; c < ns; ++c)
          for (int d = 0; d < ns; ++d) {
            shell_eri(B, a, bb, c, d, out, w, cart, tmp);
            const Shell &A = B.sh[a], &Bs = B.sh[bb], &C = B.sh[c], &D = B.sh[d];
            for (int i = 0; i < A.nf; ++i)
              for (int j = 0; j < Bs.nf; ++j)
                for (int k = 0; k < C.nf; ++k)
                  for (int m = 0; m < D.nf; ++m)
                    eri[(((A.ao + i) * N + Bs.ao + j) * N + C.ao + k) * N + D.ao + m] =
                        out[((i * Bs.nf + j) * C.nf + k) * D.nf + m];
          }
  }
  return 0;
}

// HERFCK semantics through FCKD03-style digestion of unique integrals
// (DALTON/sirius/sirfck.F:1496-1547; IFCTYP decoding sirfck.F:45-57 and
// DALTON/abacus/herfckcon.F:20-220).
//
// Density screening restates Dalton's direct-Fock screening, which is on
// when IFTHRS < 16 (DALTON/abacus/her2drv.F:520-540; IFTHRS < 4 is reset to
// 14 there):
//  * SYMLOP (her2drv.F:2663-2733): per Dalton block quartet, with GAB the
//    block Schwarz factors and DMRAO the block maxima of |D| per density,
//    DNSBUF(1) = max |D| over the AB, BA, CD, DC blocks (Coulomb),
//    DNSBUF(2) = max over the CA, AC, CB, BC, DA, AD, BD, DB blocks
//    (exchange, 0 when HFXFAC = 0), DNSMAX = max over densities of
//    max(4 DNSBUF(1), DNSBUF(2)); the quartet is skipped when
//    GAB_AB GAB_CD DNSMAX < 10^-IFTHRS.
//  * INTFCK/INTFC1 (DALTON/abacus/her2fck.F:84-90, 221-222, 446-466):
//    integrals with |g| <= max(10^-IFTHRS / DNSMAX, 1e-15) are dropped; with
//    AOMAX the largest kept |g|, density I's Coulomb part is skipped when
//    bit 1 of ICEDIF is set and DNSBUF(1,I) AOMAX < 10^-IFTHRS, its exchange
//    part when bit 2 is set and DNSBUF(2,I) AOMAX < 10^-IFTHRS.
// The block quantities use Dalton's blocks (one atom's shell of angular
// momentum l with all its contracted functions); AOMAX is taken per
// segmented shell quartet, the unit this restatement evaluates.  Whatever
// IFTHRS is, quartets whose density bound is exactly zero contribute nothing
// and are skipped without evaluation.
struct FockOpts {
  double hfxfac = 1.0, thrs = 1e-12;
  int ifthrs = 20, icedif = 3;
  int stride = 1, offset = 0;
  // attenuated pass of HERFCK_1 (DALTON/abacus/herdirect.F:815-835): the
  // operator erf(mu r12)/r12 (mu2 = HFXMU^2) and exchange only for every
  // density (FCKCON sets IY = 2, herfckcon.F:66), hfxfac = HFXATT.
  double mu2 = 0.0;
  bool exchange_only = false;
};

struct FockCounts {
  int64_t evaluated = 0, skipped_screen = 0, skipped_zero = 0, dropped_j = 0, dropped_k = 0;
};

// Block Schwarz factors and block density maxima.
struct BlockBounds {
  int nb = 0;
  std::vector<double> gab;    // nb x nb
  std::vector<double> dmax;   // ndmat x nb x nb, max |D_pq| over p in block A, q in block B
};

static BlockBounds block_bounds(const Basis &B, const std::vector<double> &Q, const double *D, int ndmat) {
  BlockBounds bb;
  bb.nb = (int)B.blk_ao0.size();
  const int nb = bb.nb, ns = (int)B.sh.size();
  const size_t N = B.nbf;
  bb.gab.assign((size_t)nb * nb, 0.0);
  for (int a = 0; a < ns; ++a)
    for (int b = 0; b < ns; ++b) {
      double &g = bb.gab[(size_t)B.sh[a].blk * nb + B.sh[b].blk];
      g = std::max(g, Q[(size_t)a * ns + b]);
    }
  bb.dmax.assign((size_t)ndmat * nb * nb, 0.0);
  for (int k = 0; k < ndmat; ++k)
    for (int A = 0; A < nb; ++A)
      for (int Bk = 0; Bk < nb; ++Bk) {
        double m = 0.0;
        for (int p = B.blk_ao0[A]; p < B.blk_ao0[A] + B.blk_nfun[A]; ++p)
          for (int q = B.blk_ao0[Bk]; q < B.blk_ao0[Bk] + B.blk_nfun[Bk]; ++q)
            m = std::max(m, std::fabs(D[k * N * N + p * N + q]));
        bb.dmax[((size_t)k * nb + A) * nb + Bk] = m;
      }
  return bb;
}

static int fock_core(const orc_basis *b, int ndmat, const int64_t *ifctyp, const double *dmat, double *fmat,
                     const FockOpts &o, FockCounts *counts);

int orc_fock(const orc_basis *b, int ndmat, const int64_t *ifctyp, const double *dmat, double *fmat,
             double hfxfac, double thrs) {
  FockOpts o;
  o.hfxfac = hfxfac;
  o.thrs = thrs;
  return fock_core(b, ndmat, ifctyp, dmat, fmat, o, nullptr);
}

int orc_fock_screened(const orc_basis *b, int ndmat, const int64_t *ifctyp, const double *dmat, double *fmat,
                      double hfxfac, double thrs, int64_t ifthrs, int64_t icedif, int64_t *counts) {
  FockOpts o;
  o.hfxfac = hfxfac;
  o.thrs = thrs;
  o.ifthrs = (int)ifthrs;
  o.icedif = (int)icedif;
  FockCounts c;
  int r = fock_core(b, ndmat, ifctyp, dmat, fmat, o, &c);
  if (counts) {
    counts[0] = c.evaluated;
    counts[1] = c.skipped_screen;
    counts[2] = c.skipped_zero;
    counts[3] = c.dropped_j;
    counts[4] = c.dropped_k;
  }
  return r;
}

// HERFCK_1 with range-separated exchange (DALTON/abacus/herdirect.F:792-835):
// the 1/r12 build with HFXFAC, then, when HFXMU != 0, a second TWOINT pass
// with the operator erf(HFXMU r12)/r12, HFXFAC replaced by HFXATT and only
// the exchange part of every density, added to the same FMAT.
int orc_fock_attenuated(const orc_basis *b, int ndmat, const int64_t *ifctyp, const double *dmat, double *fmat,
                        double hfxfac, double thrs, double hfxmu, double hfxatt) {
  FockOpts o;
  o.hfxfac = hfxfac;
  o.thrs = thrs;
  int r = fock_core(b, ndmat, ifctyp, dmat, fmat, o, nullptr);
  if (r || hfxmu == 0.0) return r;
  const size_t n2 = (size_t)ndmat * b->nbf * b->nbf;
  std::vector<double> f2(n2);
  FockOpts o2;
  o2.hfxfac = hfxatt;
  o2.thrs = thrs;
  o2.mu2 = hfxmu * hfxmu;
  o2.exchange_only = true;
  r = fock_core(b, ndmat, ifctyp, dmat, f2.data(), o2, nullptr);
  for (size_t i = 0; i < n2; ++i) fmat[i] += f2[i];
  return r;
}

// One primitive (la lb|lc ld) Cartesian block with the operator erf(mu r12)/r12
// (mu = 0: 1/r12), out[((a*nb+b)*nc+c)*nd+d]; for tests of the attenuation.
void orc_prim_eri(int la, int lb, int lc, int ld, const double *exps, const double *centers, double mu, double *out) {
  EriWork w;
  w.mu2 = mu * mu;
  const size_t n = (size_t)ncart(la) * ncart(lb) * ncart(lc) * ncart(ld);
  for (size_t i = 0; i < n; ++i) out[i] = 0.0;
  prim_eri(la, lb, lc, ld, exps[0], exps[1], exps[2], exps[3], centers, centers + 3, centers + 6, centers + 9, 1.0,
           out, w);
}

int orc_fock_sampled(const orc_basis *b, const double *dmat, double *fmat, double thrs, int stride, int offset,
                     int64_t *nquartet) {
  const int64_t ift = 13;
  FockOpts o;
  o.thrs = thrs;
  o.stride = stride;
  o.offset = offset;
  FockCounts c;
  int r = fock_core(b, 1, &ift, dmat, fmat, o, &c);
  if (nquartet) *nquartet = c.evaluated;
  return r;
}

// Decoded IFCTYP of each density: symmetrised / antisymmetrised / general D,
// and whether it takes Coulomb and exchange parts.
struct DensitySet {
  std::vector<double> D;
  std::vector<int> doJ, doK;
};

static DensitySet decode_densities(size_t N, int ndmat, const int64_t *ifctyp, const double *dmat, double hfxfac) {
  DensitySet ds;
  const size_t N2 = N * N;
  ds.D.assign(ndmat * N2, 0.0);
  ds.doJ.assign(ndmat, 0);
  ds.doK.assign(ndmat, 0);
  for (int k = 0; k < ndmat; ++k) {
    int X = (int)(ifctyp[k] / 10), Y = (int)(ifctyp[k] % 10);
    if (X == 2) Y &= 2;
    if (hfxfac == 0.0) Y &= 1;
    ds.doJ[k] = Y & 1;
    ds.doK[k] = (Y & 2) ? 1 : 0;
    for (size_t p = 0; p < N; ++p)
      for (size_t q = 0; q < N; ++q) {
        double dpq = dmat[k * N2 + p * N + q], dqp = dmat[k * N2 + q * N + p];
        ds.D[k * N2 + p * N + q] = (X == 1) ? 0.5 * (dpq + dqp) : (X == 2) ? 0.5 * (dpq - dqp) : dpq;
      }
  }
  return ds;
}

// Digestion of one segmented shell quartet block g (FCKCON, herfckcon.F:66-80,
// in the FCKD03 form that handles general densities), with Dalton's
// per-density Coulomb/exchange skips; Fl accumulates (ndmat x N x N).
static void digest_quartet(const Basis &B, int sA, int sB, int sC, int sD, bool same_pair, const std::vector<double> &g,
                           const DensitySet &ds, int ndmat, double efac, const double *jkeep, const double *kkeep,
                           double fcktol, double *Fl) {
  const size_t N = B.nbf, N2 = N * N;
  const Shell &A = B.sh[sA], &Bs = B.sh[sB], &C = B.sh[sC], &Dd = B.sh[sD];
  for (int i = 0; i < A.nf; ++i) {
    size_t p = A.ao + i;
    for (int j = 0; j < Bs.nf; ++j) {
      size_t q = Bs.ao + j;
      if (sA == sB && q > p) continue;
      for (int kk = 0; kk < C.nf; ++kk) {
        size_t r = C.ao + kk;
        for (int m = 0; m < Dd.nf; ++m) {
          size_t s = Dd.ao + m;
          if (sC == sD && s > r) continue;
          if (same_pair && (r * (r + 1) / 2 + s) > (p * (p + 1) / 2 + q)) continue;
          double gint = g[((i * Bs.nf + j) * C.nf + kk) * Dd.nf + m];
          if (std::fabs(gint) <= fcktol) continue;
          if (p == q) gint *= 0.5;
          if (r == s) gint *= 0.5;
          if (p == r && q == s) gint *= 0.5;
          for (int k = 0; k < ndmat; ++k) {
            const double *Dk = &ds.D[k * N2];
            double *Fk = &Fl[k * N2];
            if (ds.doJ[k] && jkeep[k] != 0.0) {
              double fadd = gint * (Dk[r * N + s] + Dk[s * N + r]);
              Fk[p * N + q] += fadd;
              Fk[q * N + p] += fadd;
              fadd = gint * (Dk[p * N + q] + Dk[q * N + p]);
              Fk[r * N + s] += fadd;
              Fk[s * N + r] += fadd;
            }
            if (ds.doK[k] && kkeep[k] != 0.0) {
              double e = efac * gint;
              Fk[p * N + r] -= e * Dk[q * N + s];
              Fk[r * N + p] -= e * Dk[s * N + q];
              Fk[p * N + s] -= e * Dk[q * N + r];
              Fk[s * N + p] -= e * Dk[r * N + q];
              Fk[q * N + r] -= e * Dk[p * N + s];
              Fk[r * N + q] -= e * Dk[s * N + p];
              Fk[q * N + s] -= e * Dk[p * N + r];
              Fk[s * N + q] -= e * Dk[r * N + p];
            }
          }
        }
      }
    }
  }
}

// Screening decision of one segmented quartet (SYMLOP on its Dalton
// blocks): returns 0 = evaluate, 1 = screened out, 2 = zero density bound;
// dJ/dK receive DNSBUF(1/2, I), *dnsmax DNSMAX.
static int quartet_screen(const Basis &B, const BlockBounds &bb, int sA, int sB, int sC, int sD, int ndmat,
                          double hfxfac, bool doscrn, double fckthr, double *dJ, double *dK, double *dnsmax) {
  const int nb = bb.nb;
  const int a = B.sh[sA].blk, b = B.sh[sB].blk, c = B.sh[sC].blk, d = B.sh[sD].blk;
  double dm = 0.0;
  for (int k = 0; k < ndmat; ++k) {
    const double *M = &bb.dmax[(size_t)k * nb * nb];
    auto at = [&](int x, int y) { return M[(size_t)x * nb + y]; };
    dJ[k] = std::max(std::max(at(a, b), at(b, a)), std::max(at(c, d), at(d, c)));
    dK[k] = 0.0;
    if (hfxfac != 0.0)
      dK[k] = std::max(std::max(std::max(at(c, a), at(a, c)), std::max(at(c, b), at(b, c))),
                       std::max(std::max(at(d, a), at(a, d)), std::max(at(b, d), at(d, b))));
    dm = std::max(dm, std::max(4.0 * dJ[k], dK[k]));
  }
  *dnsmax = dm;
  if (dm == 0.0) return 2;
  if (doscrn && dm * bb.gab[(size_t)a * nb + b] * bb.gab[(size_t)c * nb + d] < fckthr) return 1;
  return 0;
}

static int fock_core(const orc_basis *b, int ndmat, const int64_t *ifctyp, const double *dmat, double *fmat,
                     const FockOpts &o, FockCounts *counts) {
  set_threads();
  Basis B = make_basis(b);
  int ns = (int)B.sh.size();
  size_t N = B.nbf, N2 = N * N;
  DensitySet ds = decode_densities(N, ndmat, ifctyp, dmat, o.hfxfac);
  if (o.exchange_only)
    for (int k = 0; k < ndmat; ++k) {
      ds.doJ[k] = 0;
      ds.doK[k] = o.hfxfac != 0.0;
    }
  std::vector<double> Q = schwarz(B);
  const BlockBounds bb = block_bounds(B, Q, ds.D.data(), ndmat);
  int ifthrs = o.ifthrs;
  if (ifthrs < 4) ifthrs = 14;
  const bool doscrn = ifthrs < 16;
  const double fckthr = std::pow(10.0, -(double)ifthrs);
  std::vector<std::pair<int, int>> pairs;
  for (int a = 0; a < ns; ++a)
    for (int bb2 = 0; bb2 <= a; ++bb2) pairs.push_back({a, bb2});
  int npair = (int)pairs.size();
  std::vector<double> F(ndmat * N2, 0.0);
  double efac = 0.5 * o.hfxfac;
  int64_t nq = 0, nscr = 0, nzero = 0, ndj = 0, ndk = 0;
#pragma omp parallel reduction(+ : nq, nscr, nzero, ndj, ndk)
  {
    std::vector<double> Fl(ndmat * N2, 0.0);
    std::vector<double> dJ(ndmat), dK(ndmat), jkeep(ndmat), kkeep(ndmat);
    EriWork w;
    w.mu2 = o.mu2;
    std::vector<double> g, cart, tmp;
#pragma omp for schedule(dynamic)
    for (int ab = npair - 1; ab >= 0; --ab) {
      if (ab % o.stride != o.offset) continue;
      int sA = pairs[ab].first, sB = pairs[ab].second;
      double qab = Q[(size_t)sA * ns + sB];
      for (int cd = 0; cd <= ab; ++cd) {
        int sC = pairs[cd].first, sD = pairs[cd].second;
        if (qab * Q[(size_t)sC * ns + sD] < o.thrs) continue;
        double dnsmax = 0.0;
        const int scr = quartet_screen(B, bb, sA, sB, sC, sD, ndmat, o.hfxfac, doscrn, fckthr, dJ.data(),
                                       dK.data(), &dnsmax);
        if (scr == 2) {
          ++nzero;
          continue;
        }
        if (scr == 1) {
          ++nscr;
          continue;
        }
        ++nq;
        shell_eri(B, sA, sB, sC, sD, g, w, cart, tmp);
        double fcktol = -1.0;  // keep every integral unless screening is on
        for (int k = 0; k < ndmat; ++k) jkeep[k] = kkeep[k] = 1.0;
        if (doscrn) {
          fcktol = std::max(fckthr / dnsmax, 1e-15);
          double aomax = 0.0;
          for (double v : g)
            if (std::fabs(v) > fcktol) aomax = std::max(aomax, std::fabs(v));
          for (int k = 0; k < ndmat; ++k) {
            if ((o.icedif & 1) && ds.doJ[k] && dJ[k] * aomax < fckthr) {
              jkeep[k] = 0.0;
              ++ndj;
            }
            if ((o.icedif & 2) && ds.doK[k] && dK[k] * aomax < fckthr) {
              kkeep[k] = 0.0;
              ++ndk;
            }
          }
        }
        digest_quartet(B, sA, sB, sC, sD, ab == cd, g, ds, ndmat, efac, jkeep.data(), kkeep.data(), fcktol,
                       Fl.data());
      }
    }
#pragma omp critical
    for (size_t i = 0; i < F.size(); ++i) F[i] += Fl[i];
  }
  std::memcpy(fmat, F.data(), F.size() * sizeof(double));
  if (counts) {
    counts->evaluated = nq;
    counts->skipped_screen = nscr;
    counts->skipped_zero = nzero;
    counts->dropped_j = ndj;
    counts->dropped_k = ndk;
  }
  return 0;
}

// Timing sample of the J+K build (IFCTYP 13, hfxfac 1, no density
// screening) for the CPU baseline: the significant canonical quartets
// (ab|cd) of the segmented shells whose hash of (ab, cd) falls below
// 2^(64 - k) -- a fixed pseudo-random subset of about 2^-k of the quartet
// list, so its class mix is the workload's -- are evaluated and digested on
// all threads.  *nsample receives the quartets evaluated, *seconds the wall
// time of that evaluation (the selection scan, which a full build spends
// about a nanosecond per quartet on, the Schwarz pre-pass and set-up
// excluded), *total the number of significant quartets.  k = 0 evaluates
// every quartet.
static inline uint64_t quartet_hash(uint64_t ab, uint64_t cd) {
  uint64_t x = ab * 0x9E3779B97F4A7C15ull ^ (cd + 0x632BE59BD9B4E019ull);
  x ^= x >> 31;
  x *= 0xD6E8FEB86659FD93ull;
  x ^= x >> 32;
  x *= 0xD6E8FEB86659FD93ull;
  x ^= x >> 32;
  return x;
}

int orc_fock_hash_sample(const orc_basis *b, const double *dmat, double thrs, int k, int64_t *nsample,
                         double *seconds, int64_t *total) {
  set_threads();
  Basis B = make_basis(b);
  const int ns = (int)B.sh.size();
  const size_t N = B.nbf, N2 = N * N;
  const int64_t ift = 13;
  const DensitySet ds = decode_densities(N, 1, &ift, dmat, 1.0);
  std::vector<double> Q = schwarz(B);
  std::vector<std::pair<int, int>> pairs;
  for (int a = 0; a < ns; ++a)
    for (int c = 0; c <= a; ++c) pairs.push_back({a, c});
  const int npair = (int)pairs.size();
  const uint64_t cut = k <= 0 ? ~0ull : (k >= 64 ? 0ull : (~0ull >> k));
  int64_t ntot = 0;
  std::vector<std::pair<int, int>> smp;
#pragma omp parallel reduction(+ : ntot)
  {
    std::vector<std::pair<int, int>> mine;
#pragma omp for schedule(dynamic, 64)
    for (int ab = npair - 1; ab >= 0; --ab) {
      const int sA = pairs[ab].first, sB = pairs[ab].second;
      const double qab = Q[(size_t)sA * ns + sB];
      for (int cd = 0; cd <= ab; ++cd) {
        const int sC = pairs[cd].first, sD = pairs[cd].second;
        if (qab * Q[(size_t)sC * ns + sD] < thrs) continue;
        ++ntot;
        if (quartet_hash((uint64_t)ab, (uint64_t)cd) <= cut) mine.push_back({ab, cd});
      }
    }
#pragma omp critical
    smp.insert(smp.end(), mine.begin(), mine.end());
  }
  std::sort(smp.begin(), smp.end(), [](const std::pair<int, int> &x, const std::pair<int, int> &y) {
    return x.first != y.first ? x.first > y.first : x.second < y.second;
  });
  int64_t nq = 0;
  const double t0 = omp_get_wtime();
#pragma omp parallel reduction(+ : nq)
  {
    std::vector<double> Fl(N2, 0.0);
    const double keep = 1.0;
    EriWork w;
    std::vector<double> g, cart, tmp;
#pragma omp for schedule(dynamic, 8)
    for (int64_t i = 0; i < (int64_t)smp.size(); ++i) {
      const int ab = smp[i].first, cd = smp[i].second;
      const int sA = pairs[ab].first, sB = pairs[ab].second, sC = pairs[cd].first, sD = pairs[cd].second;
      ++nq;
      shell_eri(B, sA, sB, sC, sD, g, w, cart, tmp);
      digest_quartet(B, sA, sB, sC, sD, ab == cd, g, ds, 1, 0.5, &keep, &keep, -1.0, Fl.data());
    }
  }
  *seconds = omp_get_wtime() - t0;
  *nsample = nq;
  *total = ntot;
  return 0;
}

// ---------------------------------------------------------------- gradient
// Derivative integrals by differentiating the Gaussians:
// d/dA_x [x_A^i e^{-a x_A^2}] = 2a x_A^{i+1} e^{..} - i x_A^{i-1} e^{..}
// (INTEXP/INTEX1/DEROUT, DALTON/abacus/her2ave.F:20,91,784-830).

// Cartesian-component shift: index of (ax+dx, ay+dy, az+dz) in shell l+-1.
static int cart_index(int l, int x, int y, int z) {
  (void)l;
  int s = y + z;
  return s * (s + 1) / 2 + z;
}

int orc_grad2e(const orc_basis *b, const double *dmat, double hfxfac, double thrs, double *grad) {
  set_threads();
  Basis B = make_basis(b);
  int ns = (int)B.sh.size();
  size_t N = B.nbf;
  std::vector<double> Q = schwarz(B);
  std::vector<std::pair<int, int>> pairs;
  for (int a = 0; a < ns; ++a)
    for (int bb = 0; bb <= a; ++bb) pairs.push_back({a, bb});
  int npair = (int)pairs.size();
  std::vector<double> G(3 * B.natom, 0.0);
#pragma omp parallel
  {
    std::vector<double> Gl(3 * B.natom, 0.0);
    EriWork w;
    std::vector<double> tmp, sphd;
#pragma omp for schedule(dynamic)
    for (int ab = npair - 1; ab >= 0; --ab) {
      int s4[4];
      s4[0] = pairs[ab].first;
      s4[1] = pairs[ab].second;
      double qab = Q[(size_t)s4[0] * ns + s4[1]];
      for (int cd = 0; cd <= ab; ++cd) {
        s4[2] = pairs[cd].first;
        s4[3] = pairs[cd].second;
        if (qab * Q[(size_t)s4[2] * ns + s4[3]] < thrs) continue;
        const Shell *S[4] = {&B.sh[s4[0]], &B.sh[s4[1]], &B.sh[s4[2]], &B.sh[s4[3]]};
        int l[4] = {S[0]->l, S[1]->l, S[2]->l, S[3]->l};
        int nc[4] = {ncart(l[0]), ncart(l[1]), ncart(l[2]), ncart(l[3])};
        size_t ntot = (size_t)nc[0] * nc[1] * nc[2] * nc[3];
        // derivative Cartesian blocks for centres 0..2, x/y/z
        std::vector<double> dcart(9 * ntot, 0.0);
        for (int cen = 0; cen < 3; ++cen) {
          int lp[4] = {l[0], l[1], l[2], l[3]};
          lp[cen] += 1;
          int lm[4] = {l[0], l[1], l[2], l[3]};
          lm[cen] -= 1;
          size_t np_ = (size_t)ncart(lp[0]) * ncart(lp[1]) * ncart(lp[2]) * ncart(lp[3]);
          size_t nm_ = lm[cen] >= 0 ? (size_t)ncart(lm[0]) * ncart(lm[1]) * ncart(lm[2]) * ncart(lm[3]) : 0;
          std::vector<double> cp(np_, 0.0), cm(nm_, 0.0);
          for (int i0 = 0; i0 < S[0]->nprim; ++i0)
            for (int i1 = 0; i1 < S[1]->nprim; ++i1)
              for (int i2 = 0; i2 < S[2]->nprim; ++i2)
                for (int i3 = 0; i3 < S[3]->nprim; ++i3) {
                  double ex[4] = {S[0]->a[i0], S[1]->a[i1], S[2]->a[i2], S[3]->a[i3]};
                  double cc = S[0]->c[i0] * S[1]->c[i1] * S[2]->c[i2] * S[3]->c[i3];
                  prim_eri(lp[0], lp[1], lp[2], lp[3], ex[0], ex[1], ex[2], ex[3], S[0]->xyz, S[1]->xyz,
                           S[2]->xyz, S[3]->xyz, 2.0 * ex[cen] * cc, cp.data(), w);
                  if (nm_)
                    prim_eri(lm[0], lm[1], lm[2], lm[3], ex[0], ex[1], ex[2], ex[3], S[0]->xyz, S[1]->xyz,
                             S[2]->xyz, S[3]->xyz, cc, cm.data(), w);
                }
          const std::vector<std::array<int, 3>> *Ls[4] = {&cart_list(l[0]), &cart_list(l[1]), &cart_list(l[2]),
                                                          &cart_list(l[3])};
          int ncp[4], ncm[4];
          for (int i = 0; i < 4; ++i) {
            ncp[i] = ncart(lp[i]);
            ncm[i] = lm[i] >= 0 ? ncart(lm[i]) : 0;
          }
          for (int i0 = 0; i0 < nc[0]; ++i0)
            for (int i1 = 0; i1 < nc[1]; ++i1)
              for (int i2 = 0; i2 < nc[2]; ++i2)
                for (int i3 = 0; i3 < nc[3]; ++i3) {
                  int idx[4] = {i0, i1, i2, i3};
                  size_t o = (((size_t)i0 * nc[1] + i1) * nc[2] + i2) * nc[3] + i3;
                  for (int dir = 0; dir < 3; ++dir) {
                    std::array<int, 3> e = (*Ls[cen])[idx[cen]];
                    int ep[3] = {e[0], e[1], e[2]};
                    ep[dir] += 1;
                    int ip[4] = {i0, i1, i2, i3};
                    ip[cen] = cart_index(lp[cen], ep[0], ep[1], ep[2]);
                    double v = cp[(((size_t)ip[0] * ncp[1] + ip[1]) * ncp[2] + ip[2]) * ncp[3] + ip[3]];
                    if (e[dir] > 0) {
                      int em[3] = {e[0], e[1], e[2]};
                      em[dir] -= 1;
                      int im[4] = {i0, i1, i2, i3};
                      im[cen] = cart_index(lm[cen], em[0], em[1], em[2]);
                      v -= e[dir] * cm[(((size_t)im[0] * ncm[1] + im[1]) * ncm[2] + im[2]) * ncm[3] + im[3]];
                    }
                    dcart[(cen * 3 + dir) * ntot + o] = v;
                  }
                }
        }
        // contract with density products over unique function tuples
        const Shell &A = *S[0], &Bs = *S[1], &C = *S[2], &Dd = *S[3];
        std::vector<std::vector<double>> dsph(9);
        for (int k = 0; k < 9; ++k) {
          std::vector<double> blk(dcart.begin() + k * ntot, dcart.begin() + (k + 1) * ntot);
          cart_to_sph4(B, l[0], l[1], l[2], l[3], blk, dsph[k], tmp);
        }
        double acc[9] = {0};
        for (int i = 0; i < A.nf; ++i) {
          size_t p = A.ao + i;
          for (int j = 0; j < Bs.nf; ++j) {
            size_t q = Bs.ao + j;
            if (s4[0] == s4[1] && q > p) continue;
            for (int kk = 0; kk < C.nf; ++kk) {
              size_t r = C.ao + kk;
              for (int m = 0; m < Dd.nf; ++m) {
                size_t s = Dd.ao + m;
                if (s4[2] == s4[3] && s > r) continue;
                if (ab == cd && (r * (r + 1) / 2 + s) > (p * (p + 1) / 2 + q)) continue;
                double f = 1.0;
                if (p == q) f *= 0.5;
                if (r == s) f *= 0.5;
                if (p == r && q == s) f *= 0.5;
                double gam = 4.0 * dmat[p * N + q] * dmat[r * N + s] -
                             hfxfac * (dmat[p * N + r] * dmat[q * N + s] + dmat[p * N + s] * dmat[q * N + r]);
                size_t o = ((i * Bs.nf + j) * C.nf + kk) * Dd.nf + m;
                for (int k = 0; k < 9; ++k) acc[k] += f * gam * dsph[k][o];
              }
            }
          }
        }
        for (int dir = 0; dir < 3; ++dir) {
          double da = acc[dir], db = acc[3 + dir], dc = acc[6 + dir];
          Gl[3 * A.atom + dir] += da;
          Gl[3 * Bs.atom + dir] += db;
          Gl[3 * C.atom + dir] += dc;
          Gl[3 * Dd.atom + dir] -= da + db + dc;
        }
      }
    }
#pragma omp critical
    for (size_t i = 0; i < G.size(); ++i) G[i] += Gl[i];
  }
  std::memcpy(grad, G.data(), G.size() * sizeof(double));
  return 0;
}

// ----------------------------------------------------------- one-electron
// S, T, V by Hermite expansions (HER1 one-electron integrals restated from
// the McMurchie-Davidson formulas; used for full SCF energies).
namespace {
struct OneWork {
  std::vector<double> ex, ey, ez, R;
  RWork rw;
};

// Primitive Cartesian one-electron block for (la|lb): kind 0 = S, 1 = T, 2 = V
// (V summed over all nuclei, or only nucleus `only` if >= 0; scale applied).
void prim_one(const Basis &B, int kind, int la, int lb, double a, double b, const double *A, const double *Bc,
              double scale, double *out, OneWork &w, int only = -1) {
  double p = a + b, P[3], ab2 = 0;
  for (int i = 0; i < 3; ++i) {
    P[i] = (a * A[i] + b * Bc[i]) / p;
    ab2 += (A[i] - Bc[i]) * (A[i] - Bc[i]);
  }
  double kab = std::exp(-a * b / p * ab2) * scale;
  const auto &ca = cart_list(la), &cb = cart_list(lb);
  int ncb = (int)cb.size();
  int lbe = (kind == 1) ? lb + 2 : lb;
  hermite_e(la, lbe, p, P[0] - A[0], P[0] - Bc[0], w.ex);
  hermite_e(la, lbe, p, P[1] - A[1], P[1] - Bc[1], w.ey);
  hermite_e(la, lbe, p, P[2] - A[2], P[2] - Bc[2], w.ez);
  int nt = la + lbe + 1;
  auto E = [&](const std::vector<double> &e, int i, int j, int t) -> double {
    if (j < 0) return 0.0;
    return e[(i * (lbe + 1) + j) * nt + t];
  };
  if (kind == 0 || kind == 1) {
    double s0 = std::pow(kPi / p, 1.5) * kab;
    for (int ia = 0; ia < (int)ca.size(); ++ia)
      for (int ib = 0; ib < ncb; ++ib) {
        int ax = ca[ia][0], ay = ca[ia][1], az = ca[ia][2], bx = cb[ib][0], by = cb[ib][1], bz = cb[ib][2];
        double sx = E(w.ex, ax, bx, 0), sy = E(w.ey, ay, by, 0), sz = E(w.ez, az, bz, 0);
        if (kind == 0) {
          out[ia * ncb + ib] += s0 * sx * sy * sz;
        } else {
          auto kin = [&](const std::vector<double> &e, int i, int j) {
            return -0.5 * (j * (j - 1) * E(e, i, j - 2, 0) - 2.0 * b * (2 * j + 1) * E(e, i, j, 0) +
                           4.0 * b * b * E(e, i, j + 2, 0));
          };
          double tx = kin(w.ex, ax, bx), ty = kin(w.ey, ay, by), tz = kin(w.ez, az, bz);
          out[ia * ncb + ib] += s0 * (tx * sy * sz + sx * ty * sz + sx * sy * tz);
        }
      }
  } else {
    int L = la + lb, n1 = L + 1;
    for (int c = 0; c < B.natom; ++c) {
      if (only >= 0 && c != only) continue;
      const double *C = &B.xyz[3 * c];
      hermite_r(L, p, P[0] - C[0], P[1] - C[1], P[2] - C[2], w.rw, w.R);
      double pref = -B.charge[c] * 2.0 * kPi / p * kab;
      for (int ia = 0; ia < (int)ca.size(); ++ia)
        for (int ib = 0; ib < ncb; ++ib) {
          int ax = ca[ia][0], ay = ca[ia][1], az = ca[ia][2], bx = cb[ib][0], by = cb[ib][1], bz = cb[ib][2];
          double sum = 0;
          for (int t = 0; t <= ax + bx; ++t)
            for (int u = 0; u <= ay + by; ++u)
              for (int v = 0; v <= az + bz; ++v)
                sum += E(w.ex, ax, bx, t) * E(w.ey, ay, by, u) * E(w.ez, az, bz, v) * w.R[(t * n1 + u) * n1 + v];
          out[ia * ncb + ib] += pref * sum;
        }
    }
  }
}

void sph2(const Basis &B, int la, int lb, const std::vector<double> &cart, std::vector<double> &out) {
  int na = ncart(la), nb = ncart(lb);
  int fa = (B.spherical && la >= 2) ? 2 * la + 1 : na, fb = (B.spherical && lb >= 2) ? 2 * lb + 1 : nb;
  const auto &Ta = B.sph[la], &Tb = B.sph[lb];
  out.assign(fa * fb, 0.0);
  for (int i = 0; i < fa; ++i)
    for (int j = 0; j < fb; ++j) {
      double s = 0;
      for (int x = 0; x < na; ++x)
        for (int y = 0; y < nb; ++y) s += Ta[i * na + x] * Tb[j * nb + y] * cart[x * nb + y];
      out[i * fb + j] = s;
    }
}
}  // namespace

int orc_oneint(const orc_basis *b, double *S, double *T, double *V) {
  set_threads();
  Basis B = make_basis(b);
  int ns = (int)B.sh.size();
  size_t N = B.nbf;
  double *outs[3] = {S, T, V};
#pragma omp parallel
  {
    OneWork w;
    std::vector<double> cart, sph;
#pragma omp for schedule(dynamic) collapse(2)
    for (int a = 0; a < ns; ++a)
      for (int bb = 0; bb < ns; ++bb) {
        const Shell &A = B.sh[a], &Bs = B.sh[bb];
        for (int kind = 0; kind < 3; ++kind) {
          if (!outs[kind]) continue;
          cart.assign(ncart(A.l) * ncart(Bs.l), 0.0);
          for (int i = 0; i < A.nprim; ++i)
            for (int j = 0; j < Bs.nprim; ++j)
              prim_one(B, kind, A.l, Bs.l, A.a[i], Bs.a[j], A.xyz, Bs.xyz, A.c[i] * Bs.c[j], cart.data(), w);
          sph2(B, A.l, Bs.l, cart, sph);
          for (int i = 0; i < A.nf; ++i)
            for (int j = 0; j < Bs.nf; ++j) outs[kind][(A.ao + i) * N + Bs.ao + j] = sph[i * Bs.nf + j];
        }
      }
  }
  return 0;
}

int orc_grad1e(const orc_basis *b, const double *dmat, const double *wmat, double *grad) {
  set_threads();
  Basis B = make_basis(b);
  int ns = (int)B.sh.size();
  size_t N = B.nbf;
  std::vector<double> G(3 * B.natom, 0.0);
  // nuclear repulsion
  for (int i = 0; i < B.natom; ++i)
    for (int j = 0; j < B.natom; ++j) {
      if (i == j) continue;
      double d[3], r2 = 0;
      for (int k = 0; k < 3; ++k) {
        d[k] = B.xyz[3 * i + k] - B.xyz[3 * j + k];
        r2 += d[k] * d[k];
      }
      double r3 = r2 * std::sqrt(r2);
      for (int k = 0; k < 3; ++k) G[3 * i + k] -= B.charge[i] * B.charge[j] * d[k] / r3;
    }
#pragma omp parallel
  {
    std::vector<double> Gl(3 * B.natom, 0.0);
    OneWork w;
    std::vector<double> cp, cm, dc, sph;
#pragma omp for schedule(dynamic) collapse(2)
    for (int a = 0; a < ns; ++a)
      for (int bb = 0; bb < ns; ++bb) {
        const Shell &A = B.sh[a], &Bs = B.sh[bb];
        int na = ncart(A.l), nb = ncart(Bs.l);
        const auto &La = cart_list(A.l);
        // derivative w.r.t. centre of A (the bra function); the ket-centre
        // derivative is covered by the (b,a) ordered pair of the full loop.
        // kinds: S (weight -W), T (weight D), V per nucleus (weight D).
        for (int kind = 0; kind < 3; ++kind) {
          int nnuc = (kind == 2) ? B.natom : 1;
          for (int cn = 0; cn < nnuc; ++cn) {
            int only = (kind == 2) ? cn : -1;
            cp.assign(ncart(A.l + 1) * nb, 0.0);
            cm.assign(A.l > 0 ? ncart(A.l - 1) * nb : 0, 0.0);
            for (int i = 0; i < A.nprim; ++i)
              for (int j = 0; j < Bs.nprim; ++j) {
                double cc = A.c[i] * Bs.c[j];
                prim_one(B, kind, A.l + 1, Bs.l, A.a[i], Bs.a[j], A.xyz, Bs.xyz, 2.0 * A.a[i] * cc, cp.data(), w,
                         only);
                if (A.l > 0)
                  prim_one(B, kind, A.l - 1, Bs.l, A.a[i], Bs.a[j], A.xyz, Bs.xyz, cc, cm.data(), w, only);
              }
            const double *M = (kind == 0) ? wmat : dmat;
            double sgn = (kind == 0) ? -2.0 : 2.0;  // bra and ket derivatives are equal by symmetry
            for (int dir = 0; dir < 3; ++dir) {
              dc.assign(na * nb, 0.0);
              for (int ia = 0; ia < na; ++ia) {
                auto e = La[ia];
                int ep[3] = {e[0], e[1], e[2]};
                ep[dir] += 1;
                int ip = cart_index(A.l + 1, ep[0], ep[1], ep[2]);
                for (int ib = 0; ib < nb; ++ib) {
                  double v = cp[ip * nb + ib];
                  if (e[dir] > 0) {
                    int em[3] = {e[0], e[1], e[2]};
                    em[dir] -= 1;
                    v -= e[dir] * cm[cart_index(A.l - 1, em[0], em[1], em[2]) * nb + ib];
                  }
                  dc[ia * nb + ib] = v;
                }
              }
              sph2(B, A.l, Bs.l, dc, sph);
              double s = 0;
              for (int i = 0; i < A.nf; ++i)
                for (int j = 0; j < Bs.nf; ++j) s += M[(A.ao + i) * N + Bs.ao + j] * sph[i * Bs.nf + j];
              s *= sgn;
              Gl[3 * A.atom + dir] += s;
              if (kind == 2) {
                // operator (Hellmann-Feynman) term by translational invariance:
                // dV^C/dC = -(d/dA + d/dB) V^C; this ordered pair supplies -d/dA.
                Gl[3 * cn + dir] -= s;
              }
            }
          }
        }
      }
#pragma omp critical
    for (size_t i = 0; i < G.size(); ++i) G[i] += Gl[i];
  }
  std::memcpy(grad, G.data(), G.size() * sizeof(double));
  return 0;
}

}  // extern "C"
