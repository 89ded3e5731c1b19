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
// Schwarz-screened class plan.
#include <cmath>
#include <cstring>
#include <utility>
#include <vector>

#include "dgf_ctx.h"
#include "dgf_md.cuh"

using namespace dgf;

namespace {

template <int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(128) grad_thread_kernel(const JKArgs a) {
  constexpr int L = LA + LB + LC + LD, LAB = LA + LB, LCD = LC + LD;
  constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  constexpr int NAB = NA * NB, NCD = NC * ND;
  constexpr int FA = (LA >= 2) ? 2 * LA + 1 : NA, FB = (LB >= 2) ? 2 * LB + 1 : NB;
  constexpr int FC = (LC >= 2) ? 2 * LC + 1 : NC, FD = (LD >= 2) ? 2 * LD + 1 : ND;
  constexpr int TA = LAB + 3, TC = LCD + 2;        // t extents of the shifted tables
  constexpr int EA1 = (LA + 2) * (LB + 2) * TA;     // herm_e<LA+1, LB+1>
  constexpr int EC1 = (LC + 2) * (LD + 1) * TC;     // herm_e<LC+1, LD>
  __shared__ double tab[kBoysTableDoubles];
  __shared__ double sph[kSphTableDoubles];
  for (int i = threadIdx.x; i < kBoysTableDoubles; i += blockDim.x) tab[i] = a.boys[i];
  for (int i = threadIdx.x; i < kSphTableDoubles; i += blockDim.x) sph[i] = a.sph[i];
  __syncthreads();
  const int N = a.nbf;
  const bool sphr = a.spherical != 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t q = a.q_begin + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < a.nquartet; q += stride) {
    const int ib = find_bra(a.qoff, a.nbra, q);
    const int ic = (int)(q - a.qoff[ib]);
    const PairRec br = a.bra[ib], kt = a.ket[ic];
    double w = 1.0;
    if (br.same) w *= 0.5;
    if (kt.same) w *= 0.5;
    if (a.same_class && ib == ic + a.ket_off) w *= 0.5;
    // Density product in the shells' own functions, then back to Cartesians.
    const int fa = sphr ? FA : NA, fb = sphr ? FB : NB, fc = sphr ? FC : NC, fd = sphr ? FD : ND;
    double G[NAB * NCD];
    const double h4 = 0.5 * a.hfx;
    for (int x = 0; x < fa; ++x)
      for (int y = 0; y < fb; ++y) {
        const size_t pa = br.aoA + x, pb = br.aoB + y;
        const double d1ab = a.G1[pa * N + pb], d2ab = a.G2[pa * N + pb];
        for (int c = 0; c < fc; ++c)
          for (int d = 0; d < fd; ++d) {
            const size_t pc = kt.aoA + c, pd = kt.aoB + d;
            const double v = 2.0 * (d1ab * a.G2[pc * N + pd] + d2ab * a.G1[pc * N + pd]) -
                             h4 * (a.G1[pa * N + pc] * a.G2[pb * N + pd] + a.G2[pa * N + pc] * a.G1[pb * N + pd] +
                                   a.G1[pa * N + pd] * a.G2[pb * N + pc] + a.G2[pa * N + pd] * a.G1[pb * N + pc]);
            G[((x * fb + y) * fc + c) * fd + d] = w * v;
          }
      }
    if (sphr && (LA >= 2 || LB >= 2 || LC >= 2 || LD >= 2)) {
      // Cartesian G = (T_a x T_b x T_c x T_d)^T G_sph, index by index from d back to a.
      double tmp[NAB * NCD];
      int dims[4] = {fa, fb, fc, fd};
      const int ls[4] = {LA, LB, LC, LD};
      const int nc[4] = {NA, NB, NC, ND};
      for (int k = 3; k >= 0; --k) {
        if (ls[k] < 2) continue;
        const double *T = sph + sph_offset(ls[k]);
        int pre = 1, post = 1;
        for (int m = 0; m < k; ++m) pre *= dims[m];
        for (int m = k + 1; m < 4; ++m) post *= dims[m];
        const int nin = dims[k], nout = nc[k];
        for (int i = 0; i < pre; ++i)
          for (int o = 0; o < nout; ++o)
            for (int j = 0; j < post; ++j) {
              double s = 0.0;
              for (int x = 0; x < nin; ++x) s += T[x * nout + o] * G[(i * nin + x) * post + j];
              tmp[(i * nout + o) * post + j] = s;
            }
        const int tot = pre * nout * post;
        for (int e = 0; e < tot; ++e) G[e] = tmp[e];
        dims[k] = nout;
      }
    }
    double acc[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) acc[k] = 0.0;
    for (int i = 0; i < br.npp; ++i) {
      const PrimPair P1 = a.pp[br.pp0 + i];
      const double ea = P1.ea, eb = P1.p - P1.ea;
      double e1x[EA1], e1y[EA1], e1z[EA1];
      const double h1 = 0.5 / P1.p;
      herm_e<LA + 1, LB + 1, 1, double>(h1, P1.PAx, P1.PBx, e1x);
      herm_e<LA + 1, LB + 1, 1, double>(h1, P1.PAy, P1.PBy, e1y);
      herm_e<LA + 1, LB + 1, 1, double>(h1, P1.PAz, P1.PBz, e1z);
      for (int j = 0; j < kt.npp; ++j) {
        const PrimPair P2 = a.pp[kt.pp0 + j];
        const double ecx = P2.ea;
        const double rs = rsqrt(P1.p + P2.p);
        const double alpha = P1.p * P2.p * rs * rs;
        const double x = P1.Px - P2.Px, y = P1.Py - P2.Py, z = P1.Pz - P2.Pz;
        double F[L + 2];
        boys_eval<L + 1>(alpha * (x * x + y * y + z * z), tab, F);
        double Fs[L + 2];
        double s = P1.K * P2.K * rs;
#pragma unroll
        for (int n = 0; n <= L + 1; ++n) {
          Fs[n] = s * F[n];
          s *= -2.0 * alpha;
        }
        double R[n3(L + 1)];
        hermite_r_inplace<L + 1, double>(Fs, x, y, z, R);
        double e2x[EC1], e2y[EC1], e2z[EC1];
        const double h2 = 0.5 / P2.p;
        herm_e<LC + 1, LD, -1, double>(h2, P2.PAx, P2.PBx, e2x);
        herm_e<LC + 1, LD, -1, double>(h2, P2.PAy, P2.PBy, e2y);
        herm_e<LC + 1, LD, -1, double>(h2, P2.PAz, P2.PBz, e2z);
        const double *E2[3] = {e2x, e2y, e2z};
        const double *E1[3] = {e1x, e1y, e1z};
#pragma unroll
        for (int c = 0; c < NC; ++c)
#pragma unroll
          for (int d = 0; d < ND; ++d) {
            const int cc[3] = {cart_x(LC, c), cart_y(LC, c), cart_z(LC, c)};
            const int dd[3] = {cart_x(LD, d), cart_y(LD, d), cart_z(LD, d)};
            // normal ket transform, bra Hermite range t+u+v <= LAB+1
            double xk[n3(LAB + 1)];
#pragma unroll
            for (int e = 0; e < n3(LAB + 1); ++e) xk[e] = 0.0;
            // C-derivative ket transforms, range <= LAB
            double xc[3][n3(LAB)];
#pragma unroll
            for (int k = 0; k < 3; ++k)
#pragma unroll
              for (int e = 0; e < n3(LAB); ++e) xc[k][e] = 0.0;
#pragma unroll
            for (int ta = 0; ta <= cc[0] + dd[0] + 1; ++ta)
#pragma unroll
              for (int na = 0; na <= cc[1] + dd[1] + 1; ++na)
#pragma unroll
                for (int fa2 = 0; fa2 <= cc[2] + dd[2] + 1; ++fa2) {
                  const int tt[3] = {ta, na, fa2};
                  // plain E^{cd} and the derivative combination per direction
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
                        if (t + ta + u + na + v + fa2 > L + 1) continue;  // zero terms past the R range
                        const double r = R[tuv_index(t + ta, u + na, v + fa2)];
                        xk[tuv_index(t, u, v)] += e0 * r;
                        if (t + u + v <= LAB) {
                          xc[0][tuv_index(t, u, v)] += d0 * r;
                          xc[1][tuv_index(t, u, v)] += d1 * r;
                          xc[2][tuv_index(t, u, v)] += d2 * r;
                        }
                      }
                }
#pragma unroll
            for (int ia = 0; ia < NA; ++ia)
#pragma unroll
              for (int jb = 0; jb < NB; ++jb) {
                const double g = G[(ia * NB + jb) * NCD + c * ND + d];
                const int ax[3] = {cart_x(LA, ia), cart_y(LA, ia), cart_z(LA, ia)};
                const int bx[3] = {cart_x(LB, jb), cart_y(LB, jb), cart_z(LB, jb)};
                // per direction: plain, A-derivative and B-derivative 1D tables (t <= ax+bx+1)
                double pl[3][LAB + 2], da[3][LAB + 2], db[3][LAB + 2];
#pragma unroll
                for (int k = 0; k < 3; ++k)
#pragma unroll
                  for (int t = 0; t <= LAB + 1; ++t) {
                    const double *Et = E1[k];
                    const int i0 = ax[k], j0 = bx[k];
                    pl[k][t] = (t <= i0 + j0) ? Et[(i0 * (LB + 2) + j0) * TA + t] : 0.0;
                    double va = (t <= i0 + 1 + j0) ? 2.0 * ea * Et[((i0 + 1) * (LB + 2) + j0) * TA + t] : 0.0;
                    if (i0 > 0 && t <= i0 - 1 + j0) va -= i0 * Et[((i0 - 1) * (LB + 2) + j0) * TA + t];
                    double vb = (t <= i0 + j0 + 1) ? 2.0 * eb * Et[(i0 * (LB + 2) + j0 + 1) * TA + t] : 0.0;
                    if (j0 > 0 && t <= i0 + j0 - 1) vb -= j0 * Et[(i0 * (LB + 2) + j0 - 1) * TA + t];
                    da[k][t] = va;
                    db[k][t] = vb;
                  }
                double sA[3] = {0, 0, 0}, sB[3] = {0, 0, 0}, sC[3] = {0, 0, 0};
#pragma unroll
                for (int t = 0; t <= LAB + 1; ++t)
#pragma unroll
                  for (int u = 0; u <= LAB + 1 - t; ++u)
#pragma unroll
                    for (int v = 0; v <= LAB + 1 - t - u; ++v) {
                      const double xv = xk[tuv_index(t, u, v)];
                      sA[0] += da[0][t] * pl[1][u] * pl[2][v] * xv;
                      sA[1] += pl[0][t] * da[1][u] * pl[2][v] * xv;
                      sA[2] += pl[0][t] * pl[1][u] * da[2][v] * xv;
                      sB[0] += db[0][t] * pl[1][u] * pl[2][v] * xv;
                      sB[1] += pl[0][t] * db[1][u] * pl[2][v] * xv;
                      sB[2] += pl[0][t] * pl[1][u] * db[2][v] * xv;
                      if (t + u + v <= LAB) {
                        const double pp = pl[0][t] * pl[1][u] * pl[2][v];
                        sC[0] += pp * xc[0][tuv_index(t, u, v)];
                        sC[1] += pp * xc[1][tuv_index(t, u, v)];
                        sC[2] += pp * xc[2][tuv_index(t, u, v)];
                      }
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
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      atomicAdd(a.grad + 3 * br.atA + k, acc[k]);
      atomicAdd(a.grad + 3 * br.atB + k, acc[3 + k]);
      atomicAdd(a.grad + 3 * kt.atA + k, acc[6 + k]);
      atomicAdd(a.grad + 3 * kt.atB + k, -(acc[k] + acc[3 + k] + acc[6 + k]));
    }
  }
}

constexpr int cls_la(int X) { return X == 0 ? 0 : X <= 2 ? 1 : X <= 5 ? 2 : 3; }
constexpr int cls_lb(int X) { return X - cls_la(X) * (cls_la(X) + 1) / 2; }
constexpr int kGradClasses = 6;  // pair classes up to (dd)

typedef void (*GradLauncher)(const JKArgs &, int, int, cudaStream_t);
GradLauncher g_grad[kGradClasses][kGradClasses];

template <int LA, int LB, int LC, int LD>
void launch_grad(const JKArgs &a, int grid, int block, cudaStream_t s) {
  grad_thread_kernel<LA, LB, LC, LD><<<grid, block, 0, s>>>(a);
}

template <int X, int Y>
void fill_one() {
  g_grad[X][Y] = &launch_grad<cls_la(X), cls_lb(X), cls_la(Y), cls_lb(Y)>;
}
template <int X, int... Ys>
void fill_row(std::integer_sequence<int, Ys...>) {
  (fill_one<X, Ys>(), ...);
}
template <int... Xs>
void fill_all(std::integer_sequence<int, Xs...>) {
  (fill_row<Xs>(std::make_integer_sequence<int, Xs + 1>{}), ...);
}
struct Init {
  Init() { fill_all(std::make_integer_sequence<int, kGradClasses>{}); }
} g_init;

}  // namespace

int dgf_plan_for(dgf_ctx *c, double thrs);  // dgf_api.cu

static int grad_impl(dgf_ctx *c, const double *d1, const double *d2, double hfx, double thrs, double *grad,
                     cudaStream_t st) {
  if (c->maxl > 2) {
    dgf::set_error(__FILE__, __LINE__, "the two-electron gradient covers s, p and d shells");
    return DGF_ERR_UNSUPPORTED;
  }
  int r = dgf_plan_for(c, thrs);
  if (r) return r;
  cudaError_t e = cudaMemsetAsync(grad, 0, 3 * (size_t)c->natom * sizeof(double), st);
  if (e != cudaSuccess) {
    dgf::set_error(__FILE__, __LINE__, cudaGetErrorString(e));
    return DGF_ERR_CUDA;
  }
  // The densities in the working basis (D_w = C D C^T; the derivative
  // integrals do not act on the contraction coefficients).
  const size_t n2w = (size_t)c->nwf * c->nwf;
  if (!c->d_gw) {
    if (cudaMalloc(&c->d_gw, 2 * n2w * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      c->d_gw = nullptr;
      dgf::set_error(__FILE__, __LINE__, "device allocation of the working-basis densities failed");
      return DGF_ERR_NOMEM;
    }
  }
  const WorkMaps maps = ctx_maps(c);
  const bool same = (d2 == d1);
  launch_work_prep(maps, d1, c->d_gw, nullptr, 0, (int64_t)n2w, c->nsm, st);
  if (!same) launch_work_prep(maps, d2, c->d_gw + n2w, nullptr, 0, (int64_t)n2w, c->nsm, st);
  d1 = c->d_gw;
  d2 = same ? c->d_gw : c->d_gw + n2w;
  JKArgs a;
  memset(&a, 0, sizeof(a));
  a.pp = c->d_pp;
  a.sph = c->d_sph;
  a.spherical = c->spherical;
  a.nbf = c->nwf;
  a.G1 = d1;
  a.G2 = d2;
  a.grad = grad;
  a.hfx = hfx;
  for (const ClassPlan &cp : c->plan) {
    a.bra = c->d_pairs + c->cls_off[cp.X];
    a.ket = c->d_pairs + c->cls_off[cp.Y] + cp.kb0;
    a.ket_off = cp.kb0;
    a.nbra = c->cls_off[cp.X + 1] - c->cls_off[cp.X];
    a.same_class = (cp.X == cp.Y);
    a.qoff = c->d_qoff + cp.off;
    a.q_begin = 0;
    a.nquartet = cp.nquartet;
    const int L = cls_la(cp.X) + cls_lb(cp.X) + cls_la(cp.Y) + cls_lb(cp.Y);
    a.boys = c->d_boys + (size_t)(L + 1) * kBoysTableDoubles;
    const int block = 128;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((cp.nquartet + block - 1) / block, c->nsm * 16));
    g_grad[cp.X][cp.Y](a, grid, block, st);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
      dgf::set_error(__FILE__, __LINE__, cudaGetErrorString(e));
      return DGF_ERR_CUDA;
    }
  }
  return DGF_OK;
}

extern "C" int dgf_grad2e_bilinear_device(dgf_ctx *c, const double *d1, const double *d2, double hfxfac, double thrs,
                                          double *grad_device, void *stream) {
  if (!c || !d1 || !d2 || !grad_device) {
    dgf::set_error(__FILE__, __LINE__, "NULL argument");
    return DGF_ERR_ARG;
  }
  DeviceGuard g(c->device);
  return grad_impl(c, d1, d2, hfxfac, thrs, grad_device, (cudaStream_t)stream);
}

extern "C" int dgf_grad2e_device(dgf_ctx *c, const double *dmat_device, double hfxfac, double thrs,
                                 double *grad_device, void *stream) {
  return dgf_grad2e_bilinear_device(c, dmat_device, dmat_device, hfxfac, thrs, grad_device, stream);
}

extern "C" int dgf_grad2e(dgf_ctx *c, const double *dmat, double hfxfac, double thrs, double *grad) {
  if (!c || !dmat || !grad) {
    dgf::set_error(__FILE__, __LINE__, "NULL argument");
    return DGF_ERR_ARG;
  }
  DeviceGuard g(c->device);
  const size_t n2 = (size_t)c->nbf * c->nbf;
  double *d = nullptr;
  if (cudaMalloc(&d, (n2 + 3 * (size_t)c->natom) * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    dgf::set_error(__FILE__, __LINE__, "device allocation failed");
    return DGF_ERR_NOMEM;
  }
  cudaError_t e = cudaMemcpyAsync(d, dmat, n2 * 8, cudaMemcpyHostToDevice, c->stream);
  int r = (e == cudaSuccess) ? grad_impl(c, d, d, hfxfac, thrs, d + n2, c->stream) : DGF_ERR_CUDA;
  if (r == DGF_OK) {
    e = cudaMemcpyAsync(grad, d + n2, 3 * (size_t)c->natom * 8, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
      dgf::set_error(__FILE__, __LINE__, cudaGetErrorString(e));
      r = DGF_ERR_CUDA;
    }
  }
  cudaFree(d);
  return r;
}
