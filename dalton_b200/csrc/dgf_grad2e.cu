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
//
// Host side; the kernels are in dgf_grad_kernel.cuh, instantiated one class
// pair per translation unit (DGF_GRAD_CLASS, generated by the build).
#include <cmath>
#include <cstring>
#include <vector>

#include "dgf_ctx.h"
#include "dgf_grad_kernel.cuh"

using namespace dgf;
using namespace dgf::grad;

namespace dgf {
namespace grad {
GradLauncher g_grad_table[kGradClasses][kGradClasses];
}  // namespace grad
}  // namespace dgf

int dgf_plan_for(dgf_ctx *c, double thrs);         // dgf_api.cu
int dgf_finish_profile(dgf_ctx *c, cudaStream_t st);  // dgf_api.cu

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
  a.natom = c->natom;
  a.schwarz_thr = thrs;
  a.ket_pp0 = -1;
  // Per-launch profile (dgf_set_profiling): one record per class launch,
  // kernel 5 = gradient; quartets are the plan's, primitive quartets from the
  // classes' mean primitive-pair counts.
  if (c->profiling) {
    for (cudaEvent_t ev : c->prof_ev) cudaEventDestroy(ev);
    c->prof_ev.clear();
    c->prof.clear();
  }
  static const double kBucketPrims[kNumBuckets] = {1, 2, 4, 8, 16, 32, 64};
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
    const int block = kGradBlock;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((cp.nquartet + block - 1) / block, c->nsm * 8));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (c->profiling) {
      cudaEventCreate(&e0);
      cudaEventCreate(&e1);
      c->prof_ev.push_back(e0);
      c->prof_ev.push_back(e1);
      cudaEventRecord(e0, st);
    }
    g_grad_table[cp.X][cp.Y](a, grid, block, st);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
      dgf::set_error(__FILE__, __LINE__, cudaGetErrorString(e));
      return DGF_ERR_CUDA;
    }
    if (c->profiling) {
      cudaEventRecord(e1, st);
      dgf_class_time r;
      r.la = cls_la(cp.X);
      r.lb = cls_lb(cp.X);
      r.lc = cls_la(cp.Y);
      r.ld = cls_lb(cp.Y);
      r.precision = 64;
      r.kernel = 5;
      r.quartets = r.evaluated = cp.nquartet;
      const double bra = c->cls_avg_npp[cp.X] > 0 ? c->cls_avg_npp[cp.X] : 1.0;
      r.prim_quartets = (int64_t)std::llround((double)cp.nquartet * bra * kBucketPrims[cp.bucket]);
      r.ms = 0.0;
      c->prof.push_back(r);
    }
  }
  if (c->profiling) return dgf_finish_profile(c, st);
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
