// AO basis <-> two-electron working basis transforms (see dgf_work.h).
//
// Both transforms are element-parallel and HBM/L2-bound: each output element
// is a short double sum over the sparse rows of its two functions (one term
// each for a contracted function kept as it is, up to ncontr^2 terms for a
// resolved general contraction), reading the input matrix through L2.
#include <algorithm>

#include "dgf_work.h"

namespace dgf {

namespace {

__device__ __forceinline__ int mol_index(const int64_t *__restrict__ off, int nmol, int64_t e) {
  int lo = 0, hi = nmol;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (off[mid] <= e)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

__global__ void work_prep_kernel(const WorkMaps m, const double *__restrict__ din, double *__restrict__ d,
                                 double *__restrict__ ds, int op, int64_t total) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int mol = (m.nmol == 1) ? 0 : mol_index(m.w_elem, m.nmol, e);
    const int64_t loc = e - m.w_elem[mol];
    const int n = m.nw[mol], na = m.na[mol];
    const int p = (int)(loc / n), q = (int)(loc - (int64_t)p * n);
    const int gp = m.wf_base[mol] + p, gq = m.wf_base[mol] + q;
    const double *dm = din + m.a_elem[mol];
    const int i0 = m.wr_off[gp], i1 = m.wr_off[gp + 1], j0 = m.wr_off[gq], j1 = m.wr_off[gq + 1];
    double a = 0.0, t = 0.0;
    for (int i = i0; i < i1; ++i) {
      const int mu = m.wr_idx[i];
      const double ci = m.wr_c[i];
      double sa = 0.0, st = 0.0;
      for (int j = j0; j < j1; ++j) {
        const int nu = m.wr_idx[j];
        const double cj = m.wr_c[j];
        sa += cj * dm[(int64_t)mu * na + nu];
        st += cj * dm[(int64_t)nu * na + mu];
      }
      a += ci * sa;
      t += ci * st;
    }
    d[e] = (op == 0) ? a : (op == 1) ? t : (op == 2) ? 0.5 * (a + t) : 0.5 * (a - t);
    if (ds) ds[e] = (op == 3) ? 0.0 : a + t;
  }
}

__global__ void work_combine_kernel(const WorkMaps m, const double *__restrict__ f1, const double *__restrict__ f2,
                                    double *__restrict__ f, double sign, int64_t total) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int mol = (m.nmol == 1) ? 0 : mol_index(m.a_elem, m.nmol, e);
    const int64_t loc = e - m.a_elem[mol];
    const int n = m.na[mol], nw = m.nw[mol];
    const int mu = (int)(loc / n), nu = (int)(loc - (int64_t)mu * n);
    const int gmu = m.af_base[mol] + mu, gnu = m.af_base[mol] + nu;
    const double *w1 = f1 + m.w_elem[mol], *w2 = f2 + m.w_elem[mol];
    const int i0 = m.ac_off[gmu], i1 = m.ac_off[gmu + 1], j0 = m.ac_off[gnu], j1 = m.ac_off[gnu + 1];
    double s = 0.0;
    for (int i = i0; i < i1; ++i) {
      const int p = m.ac_idx[i];
      double r = 0.0;
      for (int j = j0; j < j1; ++j) {
        const int q = m.ac_idx[j];
        r += m.ac_c[j] * (w1[(int64_t)p * nw + q] + sign * w2[(int64_t)q * nw + p]);
      }
      s += m.ac_c[i] * r;
    }
    f[e] = s;
  }
}

int grid_for(int64_t total, int block, int nsm) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((total + block - 1) / block, (int64_t)nsm * 8));
}

}  // namespace

void launch_work_prep(const WorkMaps &m, const double *din, double *d, double *ds, int op, int64_t total_w, int nsm,
                      cudaStream_t st) {
  if (total_w <= 0) return;
  work_prep_kernel<<<grid_for(total_w, 256, nsm), 256, 0, st>>>(m, din, d, ds, op, total_w);
}

void launch_work_combine(const WorkMaps &m, const double *f1, const double *f2, double *f, double sign,
                         int64_t total_a, int nsm, cudaStream_t st) {
  if (total_a <= 0) return;
  work_combine_kernel<<<grid_for(total_a, 256, nsm), 256, 0, st>>>(m, f1, f2, f, sign, total_a);
}

}  // namespace dgf
