// One-electron integrals (S, T, V) and the one-electron part of the RHF
// gradient: the HER1 pieces the SCF host needs next to the Fock build.
// One thread per ordered shell pair; McMurchie-Davidson Hermite expansions.
#include <cmath>
#include <vector>

#include "dgf_ctx.h"
#include "dgf_md.cuh"

using namespace dgf;

namespace {

constexpr int kMaxLE = kMaxShellL + 2;  // bra l+1 (derivative) / ket l+2 (kinetic)
constexpr int kEStride = (kMaxLE + 1) * (kMaxLE + 3) * (2 * kMaxLE + 3);

struct OneArgs {
  const int *sh_l, *sh_atom, *sh_ao, *sh_nprim, *sh_p0;
  const double *sh_a, *sh_c, *xyz, *charge;
  const double *boys;  // all orders
  const double *sph;
  int nshell, natom, nbf, spherical;
  double *S, *T, *V;   // outputs (N x N) or null
  // gradient mode
  const double *D, *W;
  double *grad;        // (natom, 3)
};

// E^{ij}_t for i <= la, j <= lb (runtime), layout [(i*(lb+1)+j)*(la+lb+1)+t].
__device__ void herm_e_rt(int la, int lb, double h, double pa, double pb, double *E) {
  const int nt = la + lb + 1;
  for (int k = 0; k < (la + 1) * (lb + 1) * nt; ++k) E[k] = 0.0;
  E[0] = 1.0;
  for (int i = 0; i <= la; ++i)
    for (int j = 0; j <= lb; ++j) {
      if (i == 0 && j == 0) continue;
      const int pi = (i > 0) ? i - 1 : 0, pj = (i > 0) ? j : j - 1;
      const double x = (i > 0) ? pa : pb;
      const int top = pi + pj;
      const double *prev = E + (pi * (lb + 1) + pj) * nt;
      double *cur = E + (i * (lb + 1) + j) * nt;
      for (int t = 0; t <= i + j; ++t) {
        double v = (t <= top) ? x * prev[t] : 0.0;
        if (t > 0) v += h * prev[t - 1];
        if (t + 1 <= top) v += (t + 1) * prev[t + 1];
        cur[t] = v;
      }
    }
}

__device__ void boys_rt(int M, double T, const double *boys, double *F) {
  const double *tab = boys + (size_t)M * kBoysTableDoubles;
  switch (M) {
    case 0: boys_eval<0>(T, tab, F); break;
    case 1: boys_eval<1>(T, tab, F); break;
    case 2: boys_eval<2>(T, tab, F); break;
    case 3: boys_eval<3>(T, tab, F); break;
    case 4: boys_eval<4>(T, tab, F); break;
    case 5: boys_eval<5>(T, tab, F); break;
    case 6: boys_eval<6>(T, tab, F); break;
    case 7: boys_eval<7>(T, tab, F); break;
    default: boys_eval<8>(T, tab, F); break;
  }
}

// R_tuv(p, PC) for t+u+v <= L (runtime L <= 8), compact index.
__device__ void hermite_r_rt(int L, double p, double x, double y, double z, const double *boys, double pref,
                             double *R) {
  double F[9];
  boys_rt(L, p * (x * x + y * y + z * z), boys, F);
  double Fs[9], s = pref;
  for (int n = 0; n <= L; ++n) {
    Fs[n] = s * F[n];
    s *= -2.0 * p;
  }
  R[0] = Fs[L];
  for (int n = L - 1; n >= 0; --n) {
    for (int ss = L - n; ss >= 1; --ss)
      for (int w = 0; w <= ss; ++w)
        for (int v = 0; v <= w; ++v) {
          const int u = w - v, t = ss - w;
          double val;
          if (t > 0) {
            val = x * R[tuv_index(t - 1, u, v)];
            if (t > 1) val += (t - 1) * R[tuv_index(t - 2, u, v)];
          } else if (u > 0) {
            val = y * R[tuv_index(t, u - 1, v)];
            if (u > 1) val += (u - 1) * R[tuv_index(t, u - 2, v)];
          } else {
            val = z * R[tuv_index(t, u, v - 1)];
            if (v > 1) val += (v - 1) * R[tuv_index(t, u, v - 2)];
          }
          R[tuv_index(t, u, v)] = val;
        }
    R[0] = Fs[n];
  }
}

// Cartesian one-electron block (la|lb) of one primitive pair, scaled by `scale`:
// kind 0 = overlap, 1 = kinetic, 2 = nuclear attraction summed over nuclei
// (only nucleus `only` when >= 0).  out[ia*ncart(lb)+ib] +=.
__device__ void prim_one(const OneArgs &a, int kind, int la, int lb, double ea, double eb, const double *A,
                         const double *B, double scale, double *out, int only, double *E) {
  const double p = ea + eb;
  double P[3], ab2 = 0.0;
  for (int i = 0; i < 3; ++i) {
    P[i] = (ea * A[i] + eb * B[i]) / p;
    ab2 += (A[i] - B[i]) * (A[i] - B[i]);
  }
  const double kab = exp(-ea * eb / p * ab2) * scale;
  const int lbe = (kind == 1) ? lb + 2 : lb;
  const int nt = la + lbe + 1, es = (la + 1) * (lbe + 1) * nt;
  double *ex = E, *ey = E + es, *ez = E + 2 * es;
  const double h = 0.5 / p;
  herm_e_rt(la, lbe, h, P[0] - A[0], P[0] - B[0], ex);
  herm_e_rt(la, lbe, h, P[1] - A[1], P[1] - B[1], ey);
  herm_e_rt(la, lbe, h, P[2] - A[2], P[2] - B[2], ez);
  auto Ev = [&](const double *e, int i, int j, int t) -> double {
    return (j < 0) ? 0.0 : e[(i * (lbe + 1) + j) * nt + t];
  };
  const int na = ncart(la), nb = ncart(lb);
  if (kind <= 1) {
    const double s0 = pow(3.14159265358979323846 / p, 1.5) * kab;
    for (int ia = 0; ia < na; ++ia) {
      int ax, ay, az;
      cart_decode(la, ia, ax, ay, az);
      for (int ib = 0; ib < nb; ++ib) {
        int bx, by, bz;
        cart_decode(lb, ib, bx, by, bz);
        const double sx = Ev(ex, ax, bx, 0), sy = Ev(ey, ay, by, 0), sz = Ev(ez, az, bz, 0);
        if (kind == 0) {
          out[ia * nb + ib] += s0 * sx * sy * sz;
        } else {
          auto kin = [&](const double *e, int i, int j) {
            return -0.5 * (j * (j - 1) * Ev(e, i, j - 2, 0) - 2.0 * eb * (2 * j + 1) * Ev(e, i, j, 0) +
                           4.0 * eb * eb * Ev(e, i, j + 2, 0));
          };
          out[ia * nb + ib] +=
              s0 * (kin(ex, ax, bx) * sy * sz + sx * kin(ey, ay, by) * sz + sx * sy * kin(ez, az, bz));
        }
      }
    }
  } else {
    const int L = la + lb;
    double R[n3(8)];
    for (int c = 0; c < a.natom; ++c) {
      if (only >= 0 && c != only) continue;
      const double *C = a.xyz + 3 * c;
      hermite_r_rt(L, p, P[0] - C[0], P[1] - C[1], P[2] - C[2], a.boys, 1.0, R);
      const double pref = -a.charge[c] * 2.0 * 3.14159265358979323846 / p * kab;
      for (int ia = 0; ia < na; ++ia) {
        int ax, ay, az;
        cart_decode(la, ia, ax, ay, az);
        for (int ib = 0; ib < nb; ++ib) {
          int bx, by, bz;
          cart_decode(lb, ib, bx, by, bz);
          double s = 0.0;
          for (int t = 0; t <= ax + bx; ++t)
            for (int u = 0; u <= ay + by; ++u)
              for (int v = 0; v <= az + bz; ++v)
                s += Ev(ex, ax, bx, t) * Ev(ey, ay, by, u) * Ev(ez, az, bz, v) * R[tuv_index(t, u, v)];
          out[ia * nb + ib] += pref * s;
        }
      }
    }
  }
}

// (fa, fb) block of the shells' functions from a Cartesian (la|lb) block.
__device__ void to_sph2(const OneArgs &a, int la, int lb, const double *cart, double *out, int &fa, int &fb) {
  const int na = ncart(la), nb = ncart(lb);
  fa = nfun(la, a.spherical);
  fb = nfun(lb, a.spherical);
  const bool ta = a.spherical && la >= 2, tb = a.spherical && lb >= 2;
  const double *Ta = a.sph + sph_offset(la), *Tb = a.sph + sph_offset(lb);
  for (int i = 0; i < fa; ++i)
    for (int j = 0; j < fb; ++j) {
      double s = 0.0;
      for (int x = 0; x < na; ++x) {
        const double cx = ta ? Ta[i * na + x] : (x == i ? 1.0 : 0.0);
        if (cx == 0.0) continue;
        for (int y = 0; y < nb; ++y) {
          const double cy = tb ? Tb[j * nb + y] : (y == j ? 1.0 : 0.0);
          if (cy != 0.0) s += cx * cy * cart[x * nb + y];
        }
      }
      out[i * fb + j] = s;
    }
}

__global__ void oneint_kernel(const OneArgs a) {
  const int64_t tot = (int64_t)a.nshell * a.nshell;
  double E[3 * kEStride];
  double cart[100], sph[100];
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
    const int A = (int)(e / a.nshell), B = (int)(e - (int64_t)A * a.nshell);
    const int la = a.sh_l[A], lb = a.sh_l[B];
    const double *XA = a.xyz + 3 * a.sh_atom[A], *XB = a.xyz + 3 * a.sh_atom[B];
    double *outs[3] = {a.S, a.T, a.V};
    for (int kind = 0; kind < 3; ++kind) {
      if (!outs[kind]) continue;
      for (int k = 0; k < 100; ++k) cart[k] = 0.0;
      for (int i = 0; i < a.sh_nprim[A]; ++i)
        for (int j = 0; j < a.sh_nprim[B]; ++j)
          prim_one(a, kind, la, lb, a.sh_a[a.sh_p0[A] + i], a.sh_a[a.sh_p0[B] + j], XA, XB,
                   a.sh_c[a.sh_p0[A] + i] * a.sh_c[a.sh_p0[B] + j], cart, -1, E);
      int fa, fb;
      to_sph2(a, la, lb, cart, sph, fa, fb);
      for (int i = 0; i < fa; ++i)
        for (int j = 0; j < fb; ++j) outs[kind][(size_t)(a.sh_ao[A] + i) * a.nbf + a.sh_ao[B] + j] = sph[i * fb + j];
    }
  }
}

// Bra-centre derivatives of S (weight -W), T and V (weight D), doubled for
// the equal ket term, plus the Hellmann-Feynman operator term of V by
// translational invariance (d/dC = -(d/dA + d/dB)); atomics into grad.
__global__ void grad1e_kernel(const OneArgs a) {
  const int64_t tot = (int64_t)a.nshell * a.nshell;
  double E[3 * kEStride];
  double cp[150], cm[100], dc[100], sph[100];
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
    const int A = (int)(e / a.nshell), B = (int)(e - (int64_t)A * a.nshell);
    const int la = a.sh_l[A], lb = a.sh_l[B];
    const int na = ncart(la), nb = ncart(lb);
    const double *XA = a.xyz + 3 * a.sh_atom[A], *XB = a.xyz + 3 * a.sh_atom[B];
    for (int kind = 0; kind < 3; ++kind) {
      const int nnuc = (kind == 2) ? a.natom : 1;
      for (int cn = 0; cn < nnuc; ++cn) {
        const int only = (kind == 2) ? cn : -1;
        for (int k = 0; k < 150; ++k) cp[k] = 0.0;
        for (int k = 0; k < 100; ++k) cm[k] = 0.0;
        for (int i = 0; i < a.sh_nprim[A]; ++i)
          for (int j = 0; j < a.sh_nprim[B]; ++j) {
            const double ea = a.sh_a[a.sh_p0[A] + i], eb = a.sh_a[a.sh_p0[B] + j];
            const double cc = a.sh_c[a.sh_p0[A] + i] * a.sh_c[a.sh_p0[B] + j];
            prim_one(a, kind, la + 1, lb, ea, eb, XA, XB, 2.0 * ea * cc, cp, only, E);
            if (la > 0) prim_one(a, kind, la - 1, lb, ea, eb, XA, XB, cc, cm, only, E);
          }
        const double *M = (kind == 0) ? a.W : a.D;
        const double sgn = (kind == 0) ? -2.0 : 2.0;
        for (int dir = 0; dir < 3; ++dir) {
          for (int ia = 0; ia < na; ++ia) {
            int ex, ey, ez;
            cart_decode(la, ia, ex, ey, ez);
            int ep[3] = {ex, ey, ez}, em[3] = {ex, ey, ez};
            ep[dir] += 1;
            em[dir] -= 1;
            const int ip = (ep[1] + ep[2]) * (ep[1] + ep[2] + 1) / 2 + ep[2];
            const int lm = (ep[dir] - 1);
            for (int ib = 0; ib < nb; ++ib) {
              double v = cp[ip * nb + ib];
              if (lm > 0) {
                const int im = (em[1] + em[2]) * (em[1] + em[2] + 1) / 2 + em[2];
                v -= lm * cm[im * nb + ib];
              }
              dc[ia * nb + ib] = v;
            }
          }
          int fa, fb;
          to_sph2(a, la, lb, dc, sph, fa, fb);
          double s = 0.0;
          for (int i = 0; i < fa; ++i)
            for (int j = 0; j < fb; ++j) s += M[(size_t)(a.sh_ao[A] + i) * a.nbf + a.sh_ao[B] + j] * sph[i * fb + j];
          s *= sgn;
          atomicAdd(a.grad + 3 * a.sh_atom[A] + dir, s);
          if (kind == 2) atomicAdd(a.grad + 3 * cn + dir, -s);
        }
      }
    }
  }
}

}  // namespace

static int one_args(dgf_ctx *c, OneArgs &a, std::vector<void *> &owned) {
  memset(&a, 0, sizeof(a));
  const int ns = c->nshell;
  auto up = [&](const void *src, size_t bytes, void **dst) -> int {
    if (cudaMalloc(dst, std::max<size_t>(bytes, 8)) != cudaSuccess) {
      cudaGetLastError();
      return DGF_ERR_NOMEM;
    }
    owned.push_back(*dst);
    if (cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice) != cudaSuccess) return DGF_ERR_CUDA;
    return DGF_OK;
  };
  int r = 0;
  r |= up(c->sh_l.data(), ns * 4, (void **)&a.sh_l);
  r |= up(c->sh_atom.data(), ns * 4, (void **)&a.sh_atom);
  r |= up(c->sh_ao.data(), ns * 4, (void **)&a.sh_ao);
  r |= up(c->sh_nprim.data(), ns * 4, (void **)&a.sh_nprim);
  r |= up(c->sh_p0.data(), ns * 4, (void **)&a.sh_p0);
  r |= up(c->sh_a.data(), c->sh_a.size() * 8, (void **)&a.sh_a);
  r |= up(c->sh_c.data(), c->sh_c.size() * 8, (void **)&a.sh_c);
  r |= up(c->xyz.data(), c->xyz.size() * 8, (void **)&a.xyz);
  r |= up(c->charge.data(), c->charge.size() * 8, (void **)&a.charge);
  if (r) {
    dgf::set_error(__FILE__, __LINE__, "device upload of shell data failed");
    return DGF_ERR_NOMEM;
  }
  a.boys = c->d_boys;
  a.sph = c->d_sph;
  a.nshell = ns;
  a.natom = c->natom;
  a.nbf = c->nbf;
  a.spherical = c->spherical;
  return DGF_OK;
}

static void free_owned(std::vector<void *> &owned) {
  for (void *p : owned) cudaFree(p);
  owned.clear();
}

extern "C" int dgf_oneint(dgf_ctx *c, double *S, double *T, double *V) {
  if (!c) {
    dgf::set_error(__FILE__, __LINE__, "ctx is NULL");
    return DGF_ERR_ARG;
  }
  DeviceGuard g(c->device);
  OneArgs a;
  std::vector<void *> owned;
  int r = one_args(c, a, owned);
  if (r) {
    free_owned(owned);
    return r;
  }
  const size_t n2 = (size_t)c->nbf * c->nbf;
  double *d = nullptr;
  if (cudaMalloc(&d, 3 * n2 * 8) != cudaSuccess) {
    cudaGetLastError();
    free_owned(owned);
    dgf::set_error(__FILE__, __LINE__, "device allocation failed");
    return DGF_ERR_NOMEM;
  }
  owned.push_back(d);
  a.S = S ? d : nullptr;
  a.T = T ? d + n2 : nullptr;
  a.V = V ? d + 2 * n2 : nullptr;
  const int64_t tot = (int64_t)c->nshell * c->nshell;
  oneint_kernel<<<(int)std::min<int64_t>((tot + 63) / 64, 4096), 64>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  double *outs[3] = {S, T, V};
  for (int k = 0; k < 3 && e == cudaSuccess; ++k)
    if (outs[k]) e = cudaMemcpy(outs[k], d + k * n2, n2 * 8, cudaMemcpyDeviceToHost);
  free_owned(owned);
  if (e != cudaSuccess) {
    dgf::set_error(__FILE__, __LINE__, std::string("oneint: ") + cudaGetErrorString(e));
    return DGF_ERR_CUDA;
  }
  return DGF_OK;
}

extern "C" int dgf_grad1e(dgf_ctx *c, const double *dmat, const double *wmat, double *grad) {
  if (!c || !dmat || !wmat || !grad) {
    dgf::set_error(__FILE__, __LINE__, "NULL argument");
    return DGF_ERR_ARG;
  }
  DeviceGuard g(c->device);
  OneArgs a;
  std::vector<void *> owned;
  int r = one_args(c, a, owned);
  if (r) {
    free_owned(owned);
    return r;
  }
  const size_t n2 = (size_t)c->nbf * c->nbf;
  double *d = nullptr;
  if (cudaMalloc(&d, (2 * n2 + 3 * (size_t)c->natom) * 8) != cudaSuccess) {
    cudaGetLastError();
    free_owned(owned);
    dgf::set_error(__FILE__, __LINE__, "device allocation failed");
    return DGF_ERR_NOMEM;
  }
  owned.push_back(d);
  cudaError_t e = cudaMemcpy(d, dmat, n2 * 8, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + n2, wmat, n2 * 8, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(d + 2 * n2, 0, 3 * (size_t)c->natom * 8);
  a.D = d;
  a.W = d + n2;
  a.grad = d + 2 * n2;
  const int64_t tot = (int64_t)c->nshell * c->nshell;
  if (e == cudaSuccess) {
    grad1e_kernel<<<(int)std::min<int64_t>((tot + 63) / 64, 4096), 64>>>(a);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  std::vector<double> gr(3 * (size_t)c->natom);
  if (e == cudaSuccess) e = cudaMemcpy(gr.data(), a.grad, gr.size() * 8, cudaMemcpyDeviceToHost);
  free_owned(owned);
  if (e != cudaSuccess) {
    dgf::set_error(__FILE__, __LINE__, std::string("grad1e: ") + cudaGetErrorString(e));
    return DGF_ERR_CUDA;
  }
  // nuclear repulsion gradient
  for (int i = 0; i < c->natom; ++i)
    for (int j = 0; j < c->natom; ++j) {
      if (i == j) continue;
      double dx[3], r2 = 0.0;
      for (int k = 0; k < 3; ++k) {
        dx[k] = c->xyz[3 * i + k] - c->xyz[3 * j + k];
        r2 += dx[k] * dx[k];
      }
      const double r3 = r2 * std::sqrt(r2);
      for (int k = 0; k < 3; ++k) gr[3 * i + k] -= c->charge[i] * c->charge[j] * dx[k] / r3;
    }
  memcpy(grad, gr.data(), gr.size() * 8);
  return DGF_OK;
}
