// Host runtime and C ABI of libdgfock: context (device-resident shell-pair
// data, Schwarz factors, class-sorted pair lists), the HERFCK-semantics Fock
// build, and the Boys/spherical tables.
#include <algorithm>
#include <functional>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "dgf_ctx.h"
#include "dgf_sph.h"
#include "dgf_md.cuh"

using namespace dgf;

// ------------------------------------------------------------------ errors
namespace dgf {
static thread_local std::string g_last_error;
void set_error(const char *file, int line, const std::string &msg) {
  const char *f = strrchr(file, '/');
  g_last_error = std::string(f ? f + 1 : file) + ":" + std::to_string(line) + ": " + msg;
}
}  // namespace dgf

#define DGF_FAIL(code, msg)                \
  do {                                     \
    ::dgf::set_error(__FILE__, __LINE__, msg); \
    return code;                           \
  } while (0)

// Test hook: DGF_FAULT_INJECT=alloc makes every device allocation of the
// library fail, so callers' error paths can be exercised without a GPU fault.
static bool alloc_fault_injected() {
  const char *e = getenv("DGF_FAULT_INJECT");
  return e && strcmp(e, "alloc") == 0;
}

template <typename T>
static cudaError_t dev_alloc(T **p, size_t n) {
  if (alloc_fault_injected()) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMalloc((void **)p, std::max<size_t>(n, 1) * sizeof(T));
}

// ------------------------------------------------------------------ tables
namespace dgf {

// F_m(t) by its power series, e^-t sum_k (2t)^k / ((2m+1)(2m+3)...(2m+2k+1)),
// in long double (all terms positive; accurate to ~1e-18 relative for t < 60).
static long double boys_series(int m, long double t) {
  long double term = 1.0L / (2 * m + 1), sum = term;
  for (int k = 1; k < 4000; ++k) {
    term *= 2.0L * t / (2 * m + 2 * k + 1);
    sum += term;
    if (term < 1e-22L * sum) break;
  }
  return expl(-t) * sum;
}

double boys_reference(int m, double t) {
  if (t < 60.0) return (double)boys_series(m, t);
  long double f = 0.5L * sqrtl(3.14159265358979323846264338327950288L / t);
  long double et = expl(-(long double)t);
  for (int j = 0; j < m; ++j) f = ((2 * j + 1) * f - et) / (2.0L * t);
  return (double)f;
}

// Chebyshev interpolant of F_M on each interval at kBoysNcoef nodes, written
// out as a polynomial in the interval's local variable x in [-1, 1].
void boys_table_host(std::vector<double> &out) {
  const long double pi = 3.14159265358979323846264338327950288L;
  out.assign(kBoysAllDoubles, 0.0);
  const long double h = 1.0L / kBoysPerUnit;
  // Two table sets: full degree kBoysDeg and low degree kBoysDegLow.
  for (int set = 0; set < 2; ++set) {
    const int n = (set == 0 ? kBoysDeg : kBoysDegLow) + 1;
    std::vector<long double> f(n), c(n), tk(n * n, 0.0L), pw(n);
    // monomial coefficients of T_j(x): tk[j*n + k]
    tk[0] = 1.0L;
    if (n > 1) tk[1 * n + 1] = 1.0L;
    for (int j = 2; j < n; ++j)
      for (int k = 0; k < n; ++k) {
        long double v = -tk[(j - 2) * n + k];
        if (k > 0) v += 2.0L * tk[(j - 1) * n + k - 1];
        tk[j * n + k] = v;
      }
    for (int M = 0; M <= kBoysMaxM; ++M)
      for (int i = 0; i < kBoysNint; ++i) {
        const long double mid = (i + 0.5L) * h;
        for (int k = 0; k < n; ++k) {
          long double x = cosl(pi * (k + 0.5L) / n);
          f[k] = boys_series(M, mid + 0.5L * h * x);
        }
        for (int j = 0; j < n; ++j) {
          long double sm = 0;
          for (int k = 0; k < n; ++k) sm += f[k] * cosl(pi * j * (k + 0.5L) / n);
          c[j] = sm * 2.0L / n;
        }
        c[0] *= 0.5L;
        std::fill(pw.begin(), pw.end(), 0.0L);
        for (int j = 0; j < n; ++j)
          for (int k = 0; k < n; ++k) pw[k] += c[j] * tk[j * n + k];
        const size_t base = (set == 0 ? (size_t)M * kBoysTableDoubles : boys_low_offset(M)) + (size_t)i * kBoysNcoef;
        for (int k = 0; k < n; ++k) out[base + k] = (double)pw[k];
      }
  }
}

// Cartesian -> real spherical coefficients with Dalton's conventions (SPHCO1,
// DALTON/abacus/her1pro.F:4697-4770, MORDER=1 so m = -l..l, MINTEG=2 so the
// functions are normalised given Cartesians carrying the x^l norm), from the
// compile-time generator the kernels' immediate coefficients come from; p
// and s are identities.  Layout per l: rows m, columns Cartesian components.
void sph_table_host(std::vector<double> &out) {
  out.assign(kSphTableDoubles, 0.0);
  for (int l = 0; l <= kMaxShellL + 1; ++l) {
    const sph::Table t = sph::make(l);
    const int n = (2 * l + 1) * ncart(l);
    for (int k = 0; k < n; ++k) out[sph_offset(l) + k] = t.c[k];
  }
}

}  // namespace dgf

static void free_ctx(dgf_ctx *c) {
  if (!c) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(c->device);
  void *ptrs[] = {c->d_pairs, c->d_pp,     c->d_boys,   c->d_sph,   c->d_D,     c->d_Ds,    c->d_Fh, c->d_io,
                  c->d_dmax,  c->d_cnt,    c->d_qoff,   c->d_wmap_i, c->d_wmap_c, c->d_wmeta, c->d_wdims, c->d_gw,
                  c->d_shinfo, c->d_blk_gab, c->d_blk_info, c->d_blk_dmax, c->d_ks_i, c->d_ks_q, c->d_ks_pp,
                  c->d_store};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (c->stream) cudaStreamDestroy(c->stream);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  for (cudaEvent_t e : c->prof_ev) cudaEventDestroy(e);
  cudaSetDevice(prev);
  delete c;
}


static int cls_l1(int X) { return (X == 0) ? 0 : (X <= 2) ? 1 : (X <= 5) ? 2 : 3; }

// Kernel for class pair (X, Y): precision 0 = FP64 (the context's choice),
// 1 = FP32 thread kernel, 2 = FP64 team kernel (Schwarz pre-pass).
static const ClassKernel &select_kernel(const dgf_ctx *c, int X, int Y, int precision, bool ket1) {
  if (precision == 2) return jk_kernel(X, Y, 2);
  const int p = precision ? 1 : 0;
  const int v = c->choice[X][Y][p];
  const bool bra1 = c->cls_max_npp[X] == 1;
  const ClassKernel &k = jk_kernel_variant(X, Y, p, v, ket1, bra1);
  if (k.launch) return k;
  return jk_kernel(X, Y, precision, ket1, bra1);
}

static int launch_kernel(dgf_ctx *c, const ClassKernel &k, int X, int Y, JKArgs &args, cudaStream_t st,
                         int precision);

static int launch_class(dgf_ctx *c, int X, int Y, JKArgs &args, cudaStream_t st, int precision,
                        bool ket1 = false) {
  return launch_kernel(c, select_kernel(c, X, Y, precision, ket1), X, Y, args, st, precision);
}

static int launch_kernel(dgf_ctx *c, const ClassKernel &k, int X, int Y, JKArgs &args, cudaStream_t st,
                         int precision) {
  if (!k.launch) DGF_FAIL(DGF_ERR_UNSUPPORTED, "no kernel for this class and precision");
  const bool thread_kernel = (k.kind == kKindThread);
  const int64_t per_block = k.qpb;  // thread kernels: a quartet per thread; team kernels: per block or per warp
  const int64_t nq = args.nquartet - args.q_begin;
  if (nq <= 0 && !args.diag_out) return DGF_OK;
  int64_t grid64 = std::min<int64_t>((nq + per_block - 1) / per_block, (int64_t)c->nsm * (thread_kernel ? 8 : 16));
  int grid = (int)std::max<int64_t>(grid64, 1);
  const bool prof = c->profiling && !args.diag_out;
  if (prof) {
    cudaEvent_t e0, e1;
    DGF_CUDA_CHECK(cudaEventCreate(&e0));
    DGF_CUDA_CHECK(cudaEventCreate(&e1));
    c->prof_ev.push_back(e0);
    c->prof_ev.push_back(e1);
    DGF_CUDA_CHECK(cudaEventRecord(e0, st));
  }
  k.launch(args, grid, k.block, k.smem, st);
  DGF_CUDA_CHECK(cudaGetLastError());
  if (prof) {
    DGF_CUDA_CHECK(cudaEventRecord(c->prof_ev.back(), st));
    dgf_class_time r;
    r.la = cls_l1(X);
    r.lb = X - r.la * (r.la + 1) / 2;
    r.lc = cls_l1(Y);
    r.ld = Y - r.lc * (r.lc + 1) / 2;
    r.precision = (precision == 1) ? 32 : 64;
    r.kernel = thread_kernel                 ? 0
               : k.kind == kKindWarpTeam   ? 2
               : k.kind == kKindWarp       ? 4
               : k.kind == kKindWarpMma    ? 6
                                           : 1;
    (void)k;
    r.quartets = args.nquartet - args.q_begin;
    r.evaluated = 0;
    r.prim_quartets = 0;
    r.ms = 0.0;
    c->prof.push_back(r);
  }
  return DGF_OK;
}

int dgf_finish_profile(dgf_ctx *c, cudaStream_t st);
static int finish_profile(dgf_ctx *c, cudaStream_t st) { return dgf_finish_profile(c, st); }

// Waits for the profiled launches of the last call and stores their device times.
int dgf_finish_profile(dgf_ctx *c, cudaStream_t st) {
  if (!c->profiling) return DGF_OK;
  DGF_CUDA_CHECK(cudaStreamSynchronize(st));
  for (size_t i = 0; i < c->prof.size(); ++i) {
    float ms = 0.f;
    DGF_CUDA_CHECK(cudaEventElapsedTime(&ms, c->prof_ev[2 * i], c->prof_ev[2 * i + 1]));
    c->prof[i].ms = ms;
  }
  for (cudaEvent_t e : c->prof_ev) cudaEventDestroy(e);
  c->prof_ev.clear();
  return DGF_OK;
}

extern "C" int dgf_set_profiling(dgf_ctx *c, int on) {
  if (!c) DGF_FAIL(DGF_ERR_ARG, "ctx is NULL");
  c->profiling = on ? 1 : 0;
  return DGF_OK;
}

extern "C" int dgf_get_profile(const dgf_ctx *c, dgf_class_time *out, int max, int *count) {
  if (!c || (max > 0 && !out)) DGF_FAIL(DGF_ERR_ARG, "NULL argument");
  const int n = std::min<int>(max, (int)c->prof.size());
  for (int i = 0; i < n; ++i) out[i] = c->prof[i];
  if (count) *count = (int)c->prof.size();
  return DGF_OK;
}

// Register-resident FMA chains: 8 independent accumulators per thread.
template <typename T>
__global__ void fma_peak_kernel(T *out, int iters, T a, T b) {
  T x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      x0 = x0 * a + b; x1 = x1 * a + b; x2 = x2 * a + b; x3 = x3 * a + b;
      x4 = x4 * a + b; x5 = x5 * a + b; x6 = x6 * a + b; x7 = x7 * a + b;
    }
  }
  const T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == T(-1)) out[0] = s;  // keeps the chains live
}

template <typename T>
static int fma_peak(int device, double *tflops) {
  cudaDeviceProp prop;
  DGF_CUDA_CHECK(cudaGetDeviceProperties(&prop, device));
  T *d = nullptr;
  DGF_CUDA_CHECK(cudaMalloc(&d, sizeof(T)));
  const int block = 256, grid = prop.multiProcessorCount * 8, iters = 4096;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  fma_peak_kernel<T><<<grid, block>>>(d, 64, T(0.999999), T(1e-7));
  float best = 1e30f;
  for (int rep = 0; rep < 3; ++rep) {
    cudaEventRecord(e0);
    fma_peak_kernel<T><<<grid, block>>>(d, iters, T(0.999999), T(1e-7));
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    best = std::min(best, ms);
  }
  cudaError_t err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d);
  DGF_CUDA_CHECK(err);
  const double flops = 2.0 * 8 * 16 * (double)iters * block * grid;
  *tflops = flops / (best * 1e-3) / 1e12;
  return DGF_OK;
}

extern "C" int dgf_measure_fma_peak(int device, double *fp64_tflops, double *fp32_tflops) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    DGF_FAIL(DGF_ERR_NODEVICE, "no such CUDA device");
  }
  DeviceGuard g(device);
  int r = DGF_OK;
  if (fp64_tflops) r = fma_peak<double>(device, fp64_tflops);
  if (!r && fp32_tflops) r = fma_peak<float>(device, fp32_tflops);
  return r;
}

static JKArgs base_args(dgf_ctx *c) {
  JKArgs a;
  memset(&a, 0, sizeof(a));
  a.pp = c->d_pp;
  a.sph = c->d_sph;
  a.spherical = c->spherical;
  a.nbf = c->nwf;
  a.nshell = c->nwshell;
  a.slot_stride = (int64_t)c->nwf * c->nwf;
  a.ket_pp0 = -1;
  return a;
}

// Schwarz factors: (ab|ab) of every pair of a class-major pair list with the
// diag mode of the kernels (GABGEN/GABDRV, DALTON/abacus/her2gab.F:36,1776).
static int schwarz_of(dgf_ctx *c, const PairRec *d_pairs, const PrimPair *d_pp, const int *cls_off,
                      std::vector<double> &q) {
  const int np = cls_off[kNumPairClass];
  q.assign(np, 0.0);
  if (np == 0) return DGF_OK;
  double *d_q = nullptr;
  DGF_CUDA_CHECK(dev_alloc(&d_q, np));
  for (int X = 0; X < kNumPairClass; ++X) {
    const int n = cls_off[X + 1] - cls_off[X];
    if (!n) continue;
    const int la = (X == 0) ? 0 : (X <= 2) ? 1 : (X <= 5) ? 2 : 3;
    JKArgs a = base_args(c);
    a.pp = d_pp;
    a.bra = a.ket = d_pairs + cls_off[X];
    a.nbra = n;
    a.nquartet = n;
    a.same_class = 1;
    a.boys = c->d_boys + (size_t)(2 * (la + (X - la * (la + 1) / 2))) * kBoysTableDoubles;
    a.diag_out = d_q + cls_off[X];
    int st = launch_class(c, X, X, a, c->stream, 2);
    if (st) {
      cudaFree(d_q);
      return st;
    }
  }
  cudaError_t e = cudaMemcpyAsync(q.data(), d_q, np * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(d_q);
  DGF_CUDA_CHECK(e);
  return DGF_OK;
}

static int compute_schwarz(dgf_ctx *c) {
  std::vector<double> q;
  int st = schwarz_of(c, c->d_pairs, c->d_pp, c->cls_off, q);
  if (st) return st;
  for (size_t i = 0; i < q.size(); ++i) c->pairs[i].Q = q[i];
  return DGF_OK;
}

struct ShellList {
  const std::vector<int> &l, &atom, &ao, &nprim, &p0;
  const std::vector<double> &a, &c;
  const std::vector<int> *blk = nullptr;  // Dalton block of each shell (PairRec blkA/blkB), with kWholeBlock
};

// Shell pairs A >= B (the higher l first) with their primitive pairs, class
// by class; primitive pairs with mu |AB|^2 > 40 (e^-40 ~ 4e-18) are dropped.
static void build_pairs(const dgf_ctx *c, const ShellList &sh, int nbfm, std::vector<PairRec> &pairs,
                        int *cls_off, std::vector<PrimPair> &pp) {
  const double r2pi52 = std::sqrt(2.0 * std::pow(3.14159265358979323846, 2.5));
  std::vector<std::vector<PairRec>> bycls(kNumPairClass);
  pp.clear();
  pairs.clear();
  const int nsh = (int)sh.l.size();
  for (int A = 0; A < nsh; ++A)
    for (int B = 0; B <= A; ++B) {
      int sa = A, sb = B;
      if (sh.l[sb] > sh.l[sa]) std::swap(sa, sb);
      const int la = sh.l[sa], lb = sh.l[sb];
      const double *xa = &c->xyz[3 * sh.atom[sa]], *xb = &c->xyz[3 * sh.atom[sb]];
      const double ab2 = (xa[0] - xb[0]) * (xa[0] - xb[0]) + (xa[1] - xb[1]) * (xa[1] - xb[1]) +
                         (xa[2] - xb[2]) * (xa[2] - xb[2]);
      PairRec r;
      memset(&r, 0, sizeof(r));
      r.shA = sa;
      r.shB = sb;
      r.aoA = sh.ao[sa];
      r.aoB = sh.ao[sb];
      r.same = (A == B);
      r.atA = sh.atom[sa];
      r.atB = sh.atom[sb];
      r.blkA = sh.blk ? (*sh.blk)[sa] : 0;
      r.blkB = sh.blk ? (*sh.blk)[sb] : 0;
      r.nbfm = nbfm;
      r.dbase = 0;
      r.pp0 = (int)pp.size();
      for (int i = 0; i < sh.nprim[sa]; ++i)
        for (int j = 0; j < sh.nprim[sb]; ++j) {
          const double ea = sh.a[sh.p0[sa] + i], eb = sh.a[sh.p0[sb] + j];
          const double p = ea + eb, mu = ea * eb / p;
          if (mu * ab2 > 40.0) continue;
          PrimPair q;
          q.p = p;
          q.Px = (ea * xa[0] + eb * xb[0]) / p;
          q.Py = (ea * xa[1] + eb * xb[1]) / p;
          q.Pz = (ea * xa[2] + eb * xb[2]) / p;
          q.PAx = q.Px - xa[0];
          q.PAy = q.Py - xa[1];
          q.PAz = q.Pz - xa[2];
          q.PBx = q.Px - xb[0];
          q.PBy = q.Py - xb[1];
          q.PBz = q.Pz - xb[2];
          q.K = sh.c[sh.p0[sa] + i] * sh.c[sh.p0[sb] + j] * std::exp(-mu * ab2) * r2pi52 / p;
          q.ea = ea;
          pp.push_back(q);
        }
      r.npp = (int)pp.size() - r.pp0;
      if (r.npp == 0) continue;
      bycls[pair_class(la, lb)].push_back(r);
    }
  cls_off[0] = 0;
  for (int X = 0; X < kNumPairClass; ++X) {
    cls_off[X + 1] = cls_off[X] + (int)bycls[X].size();
    pairs.insert(pairs.end(), bycls[X].begin(), bycls[X].end());
  }
}

// Working basis (see dgf_work.h).  A block is a general contraction when
// some primitive has a nonzero coefficient in two or more of its contracted
// functions; such a block becomes one single-primitive shell per primitive,
// scaled by its largest coefficient so that the working functions keep the
// magnitude of the contracted ones (C entries = coefficient / scale, at most
// 1 in size).  Other blocks keep one shell per contracted function with its
// nonzero primitives (C entries 1).  Working functions are numbered block by
// block, shell by shell, component by component.
static int build_working_basis(dgf_ctx *c, const dgf_basis *b) {
  WorkMapHost &wm = c->wmap;
  std::vector<std::vector<std::pair<int, double>>> rows;
  int wao = 0;
  c->w_identity = 1;
  for (dgf_int ib = 0; ib < b->nblock; ++ib) {
    const int l = (int)b->block_l[ib], np = (int)b->block_nprim[ib], nc = (int)b->block_ncontr[ib];
    const int at = (int)b->block_atom[ib], nf = nfun(l, c->spherical);
    const double *cf = b->coef + b->block_coef_offset[ib];  // column-major (np, nc)
    const double *ex = b->prim_exp + b->block_prim_offset[ib];
    bool general = false;
    for (int i = 0; i < np && !general; ++i) {
      int used = 0;
      for (int k = 0; k < nc; ++k) used += (cf[(size_t)k * np + i] != 0.0);
      general = used >= 2;
    }
    if (general) {
      c->w_identity = 0;
      for (int i = 0; i < np; ++i) {
        double scale = 0.0;
        for (int k = 0; k < nc; ++k) scale = std::max(scale, std::fabs(cf[(size_t)k * np + i]));
        if (scale == 0.0) continue;
        c->ws_l.push_back(l);
        c->ws_atom.push_back(at);
        c->ws_ao.push_back(wao);
        c->ws_p0.push_back((int)c->ws_a.size());
        c->ws_blk.push_back((int)ib);
        c->ws_nprim.push_back(1);
        c->ws_a.push_back(ex[i]);
        c->ws_c.push_back(scale);
        for (int m = 0; m < nf; ++m) {
          std::vector<std::pair<int, double>> r;
          for (int k = 0; k < nc; ++k) {
            const double v = cf[(size_t)k * np + i];
            if (v != 0.0) r.push_back({(int)b->block_ao_offset[ib] + k * nf + m, v / scale});
          }
          rows.push_back(std::move(r));
        }
        wao += nf;
      }
    } else {
      for (int k = 0; k < nc; ++k) {
        c->ws_l.push_back(l);
        c->ws_atom.push_back(at);
        c->ws_ao.push_back(wao);
        c->ws_p0.push_back((int)c->ws_a.size());
        c->ws_blk.push_back((int)ib);
        int cnt = 0;
        for (int i = 0; i < np; ++i) {
          const double v = cf[(size_t)k * np + i];
          if (v == 0.0) continue;
          c->ws_a.push_back(ex[i]);
          c->ws_c.push_back(v);
          ++cnt;
        }
        c->ws_nprim.push_back(cnt);
        for (int m = 0; m < nf; ++m) {
          const int ao = (int)b->block_ao_offset[ib] + k * nf + m;
          if (ao != wao + m) c->w_identity = 0;
          rows.push_back({{ao, 1.0}});
        }
        wao += nf;
      }
    }
  }
  c->nwf = wao;
  c->nwshell = (int)c->ws_l.size();
  if (c->nwf != (int)rows.size()) DGF_FAIL(DGF_ERR_ARG, "inconsistent working basis");
  wm = WorkMapHost();
  wm.wr_off.assign(c->nwf + 1, 0);
  for (int p = 0; p < c->nwf; ++p) {
    wm.wr_off[p + 1] = wm.wr_off[p] + (int)rows[p].size();
    for (const auto &e : rows[p]) {
      wm.wr_idx.push_back(e.first);
      wm.wr_c.push_back(e.second);
    }
  }
  // transpose: AO function -> working functions
  wm.ac_off.assign(c->nbf + 1, 0);
  for (int mu : wm.wr_idx) ++wm.ac_off[mu + 1];
  for (int mu = 0; mu < c->nbf; ++mu) wm.ac_off[mu + 1] += wm.ac_off[mu];
  wm.ac_idx.assign(wm.wr_idx.size(), 0);
  wm.ac_c.assign(wm.wr_idx.size(), 0.0);
  std::vector<int> fill(wm.ac_off.begin(), wm.ac_off.end() - 1);
  for (int p = 0; p < c->nwf; ++p)
    for (int i = wm.wr_off[p]; i < wm.wr_off[p + 1]; ++i) {
      const int pos = fill[wm.wr_idx[i]]++;
      wm.ac_idx[pos] = p;
      wm.ac_c[pos] = wm.wr_c[i];
    }
  return DGF_OK;
}

static int upload_working_maps(dgf_ctx *c) {
  const WorkMapHost &wm = c->wmap;
  std::vector<int> ints;
  ints.insert(ints.end(), wm.wr_off.begin(), wm.wr_off.end());
  ints.insert(ints.end(), wm.wr_idx.begin(), wm.wr_idx.end());
  ints.insert(ints.end(), wm.ac_off.begin(), wm.ac_off.end());
  ints.insert(ints.end(), wm.ac_idx.begin(), wm.ac_idx.end());
  std::vector<double> cs(wm.wr_c);
  cs.insert(cs.end(), wm.ac_c.begin(), wm.ac_c.end());
  const int64_t meta[4] = {0, (int64_t)c->nwf * c->nwf, 0, (int64_t)c->nbf * c->nbf};
  const int dims[4] = {c->nwf, c->nbf, 0, 0};
  if (dev_alloc(&c->d_wmap_i, ints.size()) != cudaSuccess || dev_alloc(&c->d_wmap_c, std::max<size_t>(cs.size(), 1)) != cudaSuccess ||
      dev_alloc(&c->d_wmeta, 4) != cudaSuccess || dev_alloc(&c->d_wdims, 4) != cudaSuccess) {
    cudaGetLastError();
    DGF_FAIL(DGF_ERR_NOMEM, "device allocation of the working-basis maps failed");
  }
  DGF_CUDA_CHECK(cudaMemcpy(c->d_wmap_i, ints.data(), ints.size() * sizeof(int), cudaMemcpyHostToDevice));
  if (!cs.empty()) DGF_CUDA_CHECK(cudaMemcpy(c->d_wmap_c, cs.data(), cs.size() * 8, cudaMemcpyHostToDevice));
  DGF_CUDA_CHECK(cudaMemcpy(c->d_wmeta, meta, sizeof(meta), cudaMemcpyHostToDevice));
  DGF_CUDA_CHECK(cudaMemcpy(c->d_wdims, dims, sizeof(dims), cudaMemcpyHostToDevice));
  std::vector<int> shinfo(c->ws_ao);
  for (int s = 0; s < c->nwshell; ++s) shinfo.push_back(nfun(c->ws_l[s], c->spherical));
  if (dev_alloc(&c->d_shinfo, std::max<size_t>(shinfo.size(), 1)) != cudaSuccess) {
    cudaGetLastError();
    DGF_FAIL(DGF_ERR_NOMEM, "device allocation of the shell table failed");
  }
  if (!shinfo.empty())
    DGF_CUDA_CHECK(cudaMemcpy(c->d_shinfo, shinfo.data(), shinfo.size() * sizeof(int), cudaMemcpyHostToDevice));
  for (int X = 0; X < kNumPairClass; ++X)
    for (int Y = 0; Y < kNumPairClass; ++Y) c->split_ok[X][Y] = 1;
  return DGF_OK;
}

extern "C" void dgf_default_options(dgf_options *opt) {
  if (!opt) return;
  opt->thrs = 1e-12;
  opt->ifthrs = 20;
  opt->hfxfac = 1.0;
  opt->mixed_cutoff = 0.0;
  opt->shard_index = 0;
  opt->shard_count = 1;
  opt->icedif = 3;
  opt->hfxmu = 0.0;
  opt->hfxatt = 0.0;
}

extern "C" int dgf_create(const dgf_basis *b, int device, dgf_ctx **out) {
  if (!out) DGF_FAIL(DGF_ERR_ARG, "out is NULL");
  *out = nullptr;
  if (!b || b->nblock <= 0 || b->natom <= 0 || b->nbf <= 0) DGF_FAIL(DGF_ERR_ARG, "empty or invalid basis");
  if (!b->block_l || !b->block_atom || !b->block_nprim || !b->block_ncontr || !b->block_ao_offset ||
      !b->block_prim_offset || !b->block_coef_offset || !b->prim_exp || !b->coef || !b->atom_xyz ||
      !b->atom_charge)
    DGF_FAIL(DGF_ERR_ARG, "basis has a NULL array");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    DGF_FAIL(DGF_ERR_NODEVICE, "no CUDA device");
  }
  if (device < 0 || device >= ndev) DGF_FAIL(DGF_ERR_ARG, "device index out of range");
  std::unique_ptr<dgf_ctx, void (*)(dgf_ctx *)> c(new dgf_ctx, free_ctx);
  c->device = device;
  DeviceGuard g(device);
  cudaDeviceProp prop;
  DGF_CUDA_CHECK(cudaGetDeviceProperties(&prop, device));
  c->nsm = prop.multiProcessorCount;
  c->nbf = (int)b->nbf;
  c->natom = (int)b->natom;
  c->spherical = b->spherical ? 1 : 0;
  c->xyz.assign(b->atom_xyz, b->atom_xyz + 3 * b->natom);
  c->charge.assign(b->atom_charge, b->atom_charge + b->natom);

  // Segment Dalton's general-contraction blocks into one shell per
  // contracted function (zero coefficients dropped).
  for (dgf_int ib = 0; ib < b->nblock; ++ib) {
    const int l = (int)b->block_l[ib];
    if (l < 0 || l > kMaxShellL) DGF_FAIL(DGF_ERR_UNSUPPORTED, "angular momentum above f is not supported");
    const int np = (int)b->block_nprim[ib], nc = (int)b->block_ncontr[ib];
    const int at = (int)b->block_atom[ib];
    if (np <= 0 || nc <= 0 || at < 0 || at >= c->natom) DGF_FAIL(DGF_ERR_ARG, "invalid block");
    const int nf = nfun(l, c->spherical);
    for (int k = 0; k < nc; ++k) {
      const int ao = (int)b->block_ao_offset[ib] + k * nf;
      if (ao < 0 || ao + nf > c->nbf) DGF_FAIL(DGF_ERR_ARG, "AO offset out of range");
      c->sh_l.push_back(l);
      c->sh_atom.push_back(at);
      c->sh_ao.push_back(ao);
      c->sh_p0.push_back((int)c->sh_a.size());
      c->sh_blk.push_back((int)ib);
      int cnt = 0;
      for (int i = 0; i < np; ++i) {
        const double cc = b->coef[b->block_coef_offset[ib] + (dgf_int)k * np + i];
        const double ex = b->prim_exp[b->block_prim_offset[ib] + i];
        if (cc == 0.0) continue;
        if (!(ex > 0.0)) DGF_FAIL(DGF_ERR_ARG, "non-positive exponent");
        c->sh_a.push_back(ex);
        c->sh_c.push_back(cc);
        ++cnt;
      }
      c->sh_nprim.push_back(cnt);
      c->maxl = std::max(c->maxl, l);
    }
  }
  c->nshell = (int)c->sh_l.size();

  // Two-electron working basis and its map to the AO basis.
  int st_wb = build_working_basis(c.get(), b);
  if (st_wb) return st_wb;

  // Dalton blocks: working shells per block (a block that is one working
  // shell is "whole"), and each block's AO functions.
  c->nblk = (int)b->nblock;
  {
    std::vector<int> nws(c->nblk, 0);
    for (int blk : c->ws_blk) ++nws[blk];
    c->ws_blk_flag.resize(c->ws_blk.size());
    for (size_t i = 0; i < c->ws_blk.size(); ++i)
      c->ws_blk_flag[i] = c->ws_blk[i] | (nws[c->ws_blk[i]] == 1 ? kWholeBlock : 0);
    c->blk_ao0.resize(c->nblk);
    c->blk_nf.resize(c->nblk);
    for (int ib = 0; ib < c->nblk; ++ib) {
      c->blk_ao0[ib] = (int)b->block_ao_offset[ib];
      c->blk_nf[ib] = (int)b->block_ncontr[ib] * nfun((int)b->block_l[ib], c->spherical);
    }
  }
  // Working-basis shell pairs with their primitive pairs.
  build_pairs(c.get(),
              ShellList{c->ws_l, c->ws_atom, c->ws_ao, c->ws_nprim, c->ws_p0, c->ws_a, c->ws_c, &c->ws_blk_flag},
              c->nwf, c->pairs, c->cls_off, c->pp);

  DGF_CUDA_CHECK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  DGF_CUDA_CHECK(cudaEventCreate(&c->ev0));
  DGF_CUDA_CHECK(cudaEventCreate(&c->ev1));
  DGF_CUDA_CHECK(jk_prepare_all());
  std::vector<double> boys, sph;
  boys_table_host(boys);
  sph_table_host(sph);
  if (dev_alloc(&c->d_boys, boys.size()) != cudaSuccess || dev_alloc(&c->d_sph, sph.size()) != cudaSuccess ||
      dev_alloc(&c->d_pp, c->pp.size()) != cudaSuccess || dev_alloc(&c->d_pairs, c->pairs.size()) != cudaSuccess ||
      dev_alloc(&c->d_cnt, 4 * kCounterSlots) != cudaSuccess) {
    cudaGetLastError();
    DGF_FAIL(DGF_ERR_NOMEM, "device allocation failed while creating the context");
  }
  DGF_CUDA_CHECK(cudaMemcpy(c->d_boys, boys.data(), boys.size() * 8, cudaMemcpyHostToDevice));
  DGF_CUDA_CHECK(cudaMemcpy(c->d_sph, sph.data(), sph.size() * 8, cudaMemcpyHostToDevice));
  DGF_CUDA_CHECK(cudaMemcpy(c->d_pp, c->pp.data(), c->pp.size() * sizeof(PrimPair), cudaMemcpyHostToDevice));
  DGF_CUDA_CHECK(
      cudaMemcpy(c->d_pairs, c->pairs.data(), c->pairs.size() * sizeof(PairRec), cudaMemcpyHostToDevice));
  int st = upload_working_maps(c.get());
  if (st) return st;
  st = compute_schwarz(c.get());
  if (st) return st;
  // Sort each class by (primitive-count bucket, Schwarz bin descending, shells)
  // and record the bucket boundaries, then re-upload.
  for (int X = 0; X < kNumPairClass; ++X) {
    std::stable_sort(c->pairs.begin() + c->cls_off[X], c->pairs.begin() + c->cls_off[X + 1],
                     [](const PairRec &u, const PairRec &v) {
                       const int bu = npp_bucket(u.npp), bv = npp_bucket(v.npp);
                       if (bu != bv) return bu < bv;
                       const int qu = q_bin(u.Q), qv = q_bin(v.Q);
                       if (qu != qv) return qu > qv;
                       return u.shA != v.shA ? u.shA < v.shA : u.shB < v.shB;
                     });
    const int n = c->cls_off[X + 1] - c->cls_off[X];
    int pos = 0;
    for (int b = 0; b <= kNumBuckets; ++b) {
      while (b < kNumBuckets && pos < n && npp_bucket(c->pairs[c->cls_off[X] + pos].npp) < b) ++pos;
      c->bkt_off[X][b] = (b == kNumBuckets) ? n : pos;
    }
  }
  for (int X = 0; X < kNumPairClass; ++X) {
    double sum = 0.0;
    for (int i = c->cls_off[X]; i < c->cls_off[X + 1]; ++i) sum += c->pairs[i].npp;
    c->cls_avg_npp[X] = c->cls_off[X + 1] > c->cls_off[X] ? sum / (c->cls_off[X + 1] - c->cls_off[X]) : 0.0;
    c->cls_max_npp[X] = 0;
    for (int i = c->cls_off[X]; i < c->cls_off[X + 1]; ++i) c->cls_max_npp[X] = std::max(c->cls_max_npp[X], c->pairs[i].npp);
  }
  // Primitive pairs in the order of the sorted pair list.
  {
    std::vector<PrimPair> pp2;
    pp2.reserve(c->pp.size());
    for (PairRec &r : c->pairs) {
      const int p0 = (int)pp2.size();
      pp2.insert(pp2.end(), c->pp.begin() + r.pp0, c->pp.begin() + r.pp0 + r.npp);
      r.pp0 = p0;
    }
    c->pp.swap(pp2);
  }
  DGF_CUDA_CHECK(cudaMemcpy(c->d_pp, c->pp.data(), c->pp.size() * sizeof(PrimPair), cudaMemcpyHostToDevice));
  DGF_CUDA_CHECK(
      cudaMemcpy(c->d_pairs, c->pairs.data(), c->pairs.size() * sizeof(PairRec), cudaMemcpyHostToDevice));
  // Ket table of single-primitive kets (first primitive pair of every pair).
  if (c->nwshell < 65536 && !c->pairs.empty()) {
    const size_t np = c->pairs.size();
    std::vector<int4> ki(np);
    std::vector<double> kq(np), kp(11 * np);
    for (size_t g = 0; g < np; ++g) {
      const PairRec &r = c->pairs[g];
      ki[g] = make_int4(r.aoA, r.aoB, r.same, (r.shA << 16) | r.shB);
      kq[g] = r.Q;
      const PrimPair &q = c->pp[r.pp0];
      const double v[11] = {q.p, q.Px, q.Py, q.Pz, q.K, q.PAx, q.PAy, q.PAz, q.PBx, q.PBy, q.PBz};
      for (int k = 0; k < 11; ++k) kp[k * np + g] = v[k];
    }
    if (dev_alloc(&c->d_ks_i, np) != cudaSuccess || dev_alloc(&c->d_ks_q, np) != cudaSuccess ||
        dev_alloc(&c->d_ks_pp, 11 * np) != cudaSuccess) {
      cudaGetLastError();
      DGF_FAIL(DGF_ERR_NOMEM, "device allocation of the ket table failed");
    }
    DGF_CUDA_CHECK(cudaMemcpy(c->d_ks_i, ki.data(), np * sizeof(int4), cudaMemcpyHostToDevice));
    DGF_CUDA_CHECK(cudaMemcpy(c->d_ks_q, kq.data(), np * 8, cudaMemcpyHostToDevice));
    DGF_CUDA_CHECK(cudaMemcpy(c->d_ks_pp, kp.data(), 11 * np * 8, cudaMemcpyHostToDevice));
  }
  *out = c.release();
  return DGF_OK;
}

extern "C" void dgf_destroy(dgf_ctx *c) { free_ctx(c); }

extern "C" int dgf_info(const dgf_ctx *c, dgf_int *nbf, dgf_int *natom, dgf_int *nshell) {
  if (!c) DGF_FAIL(DGF_ERR_ARG, "ctx is NULL");
  if (nbf) *nbf = c->nbf;
  if (natom) *natom = c->natom;
  if (nshell) *nshell = c->nshell;
  return DGF_OK;
}

// Significant contracted shell quartets of the AO basis (one shell per
// contracted function, canonical A >= B, C >= D, AB >= CD, Q_AB Q_CD >= thrs):
// the size of a Fock build in the units Dalton-style codes count, independent
// of the working basis the kernels use.  Builds the AO pair list and its
// Schwarz factors once per call; not meant for a hot loop.
extern "C" int dgf_count_ao_quartets(dgf_ctx *c, double thrs, dgf_int *count) {
  if (!c || !count) DGF_FAIL(DGF_ERR_ARG, "NULL argument");
  if (!(thrs >= 0.0)) DGF_FAIL(DGF_ERR_ARG, "thrs must be >= 0");
  DeviceGuard g(c->device);
  std::vector<PairRec> pairs;
  std::vector<PrimPair> pp;
  int cls_off[kNumPairClass + 1];
  build_pairs(c, ShellList{c->sh_l, c->sh_atom, c->sh_ao, c->sh_nprim, c->sh_p0, c->sh_a, c->sh_c}, c->nbf, pairs,
              cls_off, pp);
  PairRec *d_pairs = nullptr;
  PrimPair *d_pp = nullptr;
  if (dev_alloc(&d_pairs, std::max<size_t>(pairs.size(), 1)) != cudaSuccess ||
      dev_alloc(&d_pp, std::max<size_t>(pp.size(), 1)) != cudaSuccess) {
    cudaGetLastError();
    if (d_pairs) cudaFree(d_pairs);
    DGF_FAIL(DGF_ERR_NOMEM, "device allocation of the AO pair list failed");
  }
  cudaError_t e = cudaMemcpy(d_pairs, pairs.data(), pairs.size() * sizeof(PairRec), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d_pp, pp.data(), pp.size() * sizeof(PrimPair), cudaMemcpyHostToDevice);
  std::vector<double> q;
  int st = (e == cudaSuccess) ? schwarz_of(c, d_pairs, d_pp, cls_off, q) : DGF_ERR_CUDA;
  cudaFree(d_pairs);
  cudaFree(d_pp);
  if (e != cudaSuccess) DGF_FAIL(DGF_ERR_CUDA, cudaGetErrorString(e));
  if (st) return st;
  int64_t total = 0;
  for (int X = 0; X < kNumPairClass; ++X) {
    std::vector<double> qb(q.begin() + cls_off[X], q.begin() + cls_off[X + 1]);
    std::sort(qb.begin(), qb.end(), std::greater<double>());
    for (int Y = 0; Y <= X; ++Y) {
      std::vector<double> qk(q.begin() + cls_off[Y], q.begin() + cls_off[Y + 1]);
      std::sort(qk.begin(), qk.end(), std::greater<double>());
      for (size_t i = 0; i < qb.size(); ++i) {
        size_t lo = 0, hi = qk.size();  // kets with qb * Q >= thrs form a prefix
        while (lo < hi) {
          const size_t mid = (lo + hi) >> 1;
          if (qb[i] * qk[mid] >= thrs)
            lo = mid + 1;
          else
            hi = mid;
        }
        total += (int64_t)((X == Y) ? std::min(lo, i + 1) : lo);
      }
    }
  }
  *count = total;
  return DGF_OK;
}

// Quartet plan: for every class pair X >= Y and bra pair, the number of ket
// pairs whose Schwarz bin can reach Q_AB Q_CD >= thrs (a prefix of the
// bin-sorted ket bucket; the kernels drop the quartets below thrs), and
// only kets up to the bra itself when X == Y), as prefix sums.
// First primitive pair of a plan entry's kets when every ket of the entry
// has one primitive pair (bucket 0): the primitive pairs are stored in pair
// order, so ket ic's is pp[base + ic]; -1 otherwise.
static int ket_pp0_of(const dgf_ctx *c, const ClassPlan &cp) {
  if (cp.bucket != 0 || cp.kb1 <= cp.kb0) return -1;
  return c->pairs[c->cls_off[cp.Y] + cp.kb0].pp0;
}

// Ket-table arguments of a plan entry: set for entries whose kets have one
// primitive pair each (bucket 0), cleared otherwise.
static void set_ket_table(const dgf_ctx *c, const ClassPlan &cp, JKArgs &a) {
  const bool on = c->d_ks_i && cp.bucket == 0 && cp.kb1 > cp.kb0;
  a.ks_i = on ? c->d_ks_i : nullptr;
  a.ks_q = on ? c->d_ks_q : nullptr;
  a.ks_pp = on ? c->d_ks_pp : nullptr;
  a.ks_stride = (int64_t)c->pairs.size();
  a.ks_base = c->cls_off[cp.Y] + cp.kb0;
}

static int build_plan(dgf_ctx *c, double thrs) {
  if (c->plan_thrs == thrs && !c->plan.empty()) return DGF_OK;
  std::vector<int64_t> all;
  std::vector<ClassPlan> plan;
  for (int X = 0; X < kNumPairClass; ++X)
    for (int Y = 0; Y <= X; ++Y) {
      const int nb = c->cls_off[X + 1] - c->cls_off[X], nk = c->cls_off[Y + 1] - c->cls_off[Y];
      if (!nb || !nk) continue;
      const PairRec *bra = &c->pairs[c->cls_off[X]], *ket = &c->pairs[c->cls_off[Y]];
      for (int kb = 0; kb < kNumBuckets; ++kb) {
        const int k0 = c->bkt_off[Y][kb], k1 = c->bkt_off[Y][kb + 1];
        if (k0 == k1) continue;
        ClassPlan cp;
        cp.X = X;
        cp.Y = Y;
        cp.bucket = kb;
        cp.kb0 = k0;
        cp.kb1 = k1;
        cp.off = (int64_t)all.size();
        int64_t acc = 0;
        all.push_back(0);
        for (int i = 0; i < nb; ++i) {
          const double qb = bra[i].Q;
          int lo = k0, hi = k1;  // first ket whose whole Schwarz bin has qb*Q < thrs
          while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (qb * q_bin_upper(q_bin(ket[mid].Q)) >= thrs)
              lo = mid + 1;
            else
              hi = mid;
          }
          int n = lo - k0;
          // X == Y: canonical pairs, ket position <= bra position in the class order
          if (X == Y) n = std::max(0, std::min(n, i - k0 + 1));
          acc += n;
          all.push_back(acc);
        }
        cp.nquartet = acc;
        if (acc > 0) plan.push_back(cp);
      }
    }
  if (all.size() > c->qoff_cap) {
    if (c->d_qoff) cudaFree(c->d_qoff);
    c->d_qoff = nullptr;
    if (dev_alloc(&c->d_qoff, all.size()) != cudaSuccess) {
      cudaGetLastError();
      c->qoff_cap = 0;
      DGF_FAIL(DGF_ERR_NOMEM, "device allocation of the quartet plan failed");
    }
    c->qoff_cap = all.size();
  }
  DGF_CUDA_CHECK(cudaMemcpy(c->d_qoff, all.data(), all.size() * 8, cudaMemcpyHostToDevice));
  c->plan.swap(plan);
  c->plan_thrs = thrs;
  return DGF_OK;
}

int dgf_plan_for(dgf_ctx *c, double thrs) { return build_plan(c, thrs); }

static int ensure_slots(dgf_ctx *c, int nslot) {
  if (nslot <= c->cap_slots) return DGF_OK;
  const size_t n2 = (size_t)c->nwf * c->nwf;
  for (double **p : {&c->d_D, &c->d_Ds, &c->d_Fh}) {
    if (*p) cudaFree(*p);
    *p = nullptr;
  }
  c->cap_slots = 0;
  if (dev_alloc(&c->d_D, n2 * nslot) != cudaSuccess || dev_alloc(&c->d_Ds, n2 * nslot) != cudaSuccess ||
      dev_alloc(&c->d_Fh, n2 * nslot) != cudaSuccess) {
    cudaGetLastError();
    DGF_FAIL(DGF_ERR_NOMEM, "device allocation of density/Fock scratch failed");
  }
  c->cap_slots = nslot;
  if (!c->d_dmax) {
    if (dev_alloc(&c->d_dmax, (size_t)c->nwshell * c->nwshell) != cudaSuccess) {
      cudaGetLastError();
      DGF_FAIL(DGF_ERR_NOMEM, "device allocation of the density bound failed");
    }
  }
  return DGF_OK;
}

// Block maxima of |D| per working shell pair over all slots, for the mixed
// form's precision bound; stored in FP32 rounded up, so that a bound never
// shrinks below the FP64 value it stands for.
__global__ void dmax_kernel(const double *__restrict__ D, int nslot, int n, const int *__restrict__ sh_ao,
                            const int *__restrict__ sh_nf, int ns, float *__restrict__ dm) {
  const int64_t tot = (int64_t)ns * ns;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
    const int A = (int)(e / ns), B = (int)(e - (int64_t)A * ns);
    double m = 0.0;
    for (int s = 0; s < nslot; ++s) {
      const double *Dk = D + (size_t)s * n * n;
      for (int i = 0; i < sh_nf[A]; ++i)
        for (int j = 0; j < sh_nf[B]; ++j) {
          const int p = sh_ao[A] + i, q = sh_ao[B] + j;
          m = fmax(m, fmax(fabs(Dk[(size_t)p * n + q]), fabs(Dk[(size_t)q * n + p])));
        }
    }
    dm[e] = __double2float_ru(m);
  }
}

struct SlotSources {
  int src[kMaxSlots];
  int nslot;
};

// Dalton's block density maxima DMRAO (MKDRAO, DALTON/abacus/her2gab.F:1213)
// of the AO densities: for every pair of Dalton blocks, max |D_pq| over the
// functions of the two blocks in both orientations, per density slot (the
// slot's source matrix) into dm_slot[s] and over the chunk's slots into dm.
// FP32 rounded up.
__global__ void blk_dmax_kernel(const double *__restrict__ Dao, int n, const int *__restrict__ blk_ao0,
                                const int *__restrict__ blk_nf, int nb, SlotSources ss, float *__restrict__ dm,
                                float *__restrict__ dm_slot) {
  const int64_t tot = (int64_t)nb * nb;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
    const int A = (int)(e / nb), B = (int)(e - (int64_t)A * nb);
    double m = 0.0;
    for (int s = 0; s < ss.nslot; ++s) {
      const double *Dk = Dao + (size_t)ss.src[s] * n * n;
      double ms = 0.0;
      for (int i = 0; i < blk_nf[A]; ++i)
        for (int j = 0; j < blk_nf[B]; ++j) {
          const int p = blk_ao0[A] + i, q = blk_ao0[B] + j;
          ms = fmax(ms, fmax(fabs(Dk[(size_t)p * n + q]), fabs(Dk[(size_t)q * n + p])));
        }
      dm_slot[(size_t)s * tot + e] = __double2float_ru(ms);
      m = fmax(m, ms);
    }
    dm[e] = __double2float_ru(m);
  }
}

// Block Schwarz factors GAB (GABGEN, DALTON/abacus/her2gab.F:1776) for the
// density screen, once per context: sqrt(max |(ab|ab)|) over the contracted
// functions of each pair of Dalton blocks, from the Schwarz factors of the
// AO basis's segmented shells; and the device buffers of the block bounds.
static int schwarz_of(dgf_ctx *c, const PairRec *d_pairs, const PrimPair *d_pp, const int *cls_off,
                      std::vector<double> &q);

static int ensure_block_screen(dgf_ctx *c, int nslot) {
  const size_t nb2 = (size_t)c->nblk * c->nblk;
  if (!c->d_blk_gab) {
    std::vector<PairRec> pairs;
    std::vector<PrimPair> pp;
    int cls_off[kNumPairClass + 1];
    build_pairs(c, ShellList{c->sh_l, c->sh_atom, c->sh_ao, c->sh_nprim, c->sh_p0, c->sh_a, c->sh_c, &c->sh_blk},
                c->nbf, pairs, cls_off, pp);
    PairRec *d_pairs = nullptr;
    PrimPair *d_pp = nullptr;
    if (dev_alloc(&d_pairs, std::max<size_t>(pairs.size(), 1)) != cudaSuccess ||
        dev_alloc(&d_pp, std::max<size_t>(pp.size(), 1)) != cudaSuccess) {
      cudaGetLastError();
      if (d_pairs) cudaFree(d_pairs);
      DGF_FAIL(DGF_ERR_NOMEM, "device allocation of the AO pair list failed");
    }
    cudaError_t e = cudaMemcpy(d_pairs, pairs.data(), pairs.size() * sizeof(PairRec), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_pp, pp.data(), pp.size() * sizeof(PrimPair), cudaMemcpyHostToDevice);
    std::vector<double> q;
    int st = (e == cudaSuccess) ? schwarz_of(c, d_pairs, d_pp, cls_off, q) : DGF_ERR_CUDA;
    cudaFree(d_pairs);
    cudaFree(d_pp);
    if (e != cudaSuccess) DGF_FAIL(DGF_ERR_CUDA, cudaGetErrorString(e));
    if (st) return st;
    std::vector<double> gab(nb2, 0.0);
    for (size_t i = 0; i < pairs.size(); ++i) {
      const int A = pairs[i].blkA, B = pairs[i].blkB;
      gab[(size_t)A * c->nblk + B] = std::max(gab[(size_t)A * c->nblk + B], q[i]);
      gab[(size_t)B * c->nblk + A] = gab[(size_t)A * c->nblk + B];
    }
    std::vector<int> info(c->blk_ao0);
    info.insert(info.end(), c->blk_nf.begin(), c->blk_nf.end());
    if (dev_alloc(&c->d_blk_gab, nb2) != cudaSuccess || dev_alloc(&c->d_blk_info, info.size()) != cudaSuccess) {
      cudaGetLastError();
      DGF_FAIL(DGF_ERR_NOMEM, "device allocation of the block Schwarz factors failed");
    }
    DGF_CUDA_CHECK(cudaMemcpy(c->d_blk_gab, gab.data(), nb2 * 8, cudaMemcpyHostToDevice));
    DGF_CUDA_CHECK(cudaMemcpy(c->d_blk_info, info.data(), info.size() * sizeof(int), cudaMemcpyHostToDevice));
  }
  if (nslot > c->cap_blk_slots) {
    if (c->d_blk_dmax) cudaFree(c->d_blk_dmax);
    c->d_blk_dmax = nullptr;
    c->cap_blk_slots = 0;
    if (dev_alloc(&c->d_blk_dmax, (size_t)(nslot + 1) * nb2) != cudaSuccess) {
      cudaGetLastError();
      DGF_FAIL(DGF_ERR_NOMEM, "device allocation of the block density bounds failed");
    }
    c->cap_blk_slots = nslot;
  }
  return DGF_OK;
}

struct SlotSpec {
  int src, op;
  double js, ks;  // Coulomb and exchange scales of the 1/r12 pass
  double ka;      // exchange scale of the attenuated erf(mu r12)/r12 pass
};

// Model cost of one quartet of a plan entry: the fixed FLOP model of the
// McMurchie-Davidson kernels (Boys + prefactor, R_tuv, ket and bra
// contractions per primitive quartet; spherical transform and six-block
// digestion per contracted quartet), times the primitive quartets of the
// entry's bucket.  Deterministic, so that every rank cuts the same shards.
static double entry_cost_per_quartet(const dgf_ctx *c, const ClassPlan &cp) {
  const int la = cls_l1(cp.X), lb = cp.X - la * (la + 1) / 2, lc = cls_l1(cp.Y), ld = cp.Y - lc * (lc + 1) / 2;
  const int L = la + lb + lc + ld, lab = la + lb, lcd = lc + ld;
  double rt = 0.0;
  for (int j = 1; j <= L; ++j) rt += 3.0 * n3(j);
  const double prim = 40.0 + 3.0 * L + rt + 2.0 * n3(lab) * n3(lcd) * ncart(lc) * ncart(ld) +
                      2.0 * n3(lab) * ncart(la) * ncart(lb) * ncart(lc) * ncart(ld);
  const double nint = (double)nfun(la, c->spherical) * nfun(lb, c->spherical) * nfun(lc, c->spherical) *
                      nfun(ld, c->spherical);
  static const double kBucketPrims[kNumBuckets] = {1, 2, 4, 8, 16, 32, 64};
  const double bra_prims = c->cls_avg_npp[cp.X] > 0 ? c->cls_avg_npp[cp.X] : 1.0;
  return prim * bra_prims * kBucketPrims[cp.bucket] + 12.0 * nint;
}

// Quartet range [q0, q1) of plan entry `e` that shard `r` of `n` evaluates:
// the plan entries in order form one queue whose cost (entry_cost_per_quartet
// x quartets) is cut into n equal parts, as Dalton's parallel Fock build
// distributes cost-sorted shell-pair tasks over its workers
// (DALTON/abacus/herpar.F:457,1165).  Consecutive shards share their cut
// points, so the ranges of all shards tile every entry exactly.
static void shard_range(const dgf_ctx *c, size_t e, int64_t r, int64_t n, int64_t *q0, int64_t *q1) {
  const ClassPlan &cp = c->plan[e];
  if (n <= 1) {
    *q0 = 0;
    *q1 = cp.nquartet;
    return;
  }
  double total = 0.0, before = 0.0;
  for (size_t i = 0; i < c->plan.size(); ++i) {
    const double w = (double)c->plan[i].nquartet * entry_cost_per_quartet(c, c->plan[i]);
    if (i < e) before += w;
    total += w;
  }
  const double w = (double)cp.nquartet * entry_cost_per_quartet(c, cp);
  auto cut = [&](int64_t k) -> int64_t {
    if (k <= 0) return 0;
    if (k >= n) return cp.nquartet;
    const double x = total * (double)k / (double)n;
    if (x <= before) return 0;
    if (x >= before + w) return cp.nquartet;
    return std::min<int64_t>(cp.nquartet, (int64_t)std::floor((x - before) / w * (double)cp.nquartet));
  };
  *q0 = cut(r);
  *q1 = cut(r + 1);
}

// Values of one quartet's integral block of class pair (X, Y) in the store.
static int64_t store_nint(const dgf_ctx *c, int X, int Y) {
  const int la = cls_l1(X), lb = X - la * (la + 1) / 2, lc = cls_l1(Y), ld = Y - lc * (lc + 1) / 2;
  return (int64_t)nfun(la, c->spherical) * nfun(lb, c->spherical) * nfun(lc, c->spherical) * nfun(ld, c->spherical);
}

// stored = true: the conventional form, digesting the blocks of the integral
// store (dgf_store_integrals) instead of evaluating integrals.
static int fock_impl(dgf_ctx *c, int ndmat, const dgf_int *ifctyp, const double *dmat_dev, double *fmat_dev,
                     const dgf_options *opt, cudaStream_t st, dgf_stats *stats, bool stored = false) {
  dgf_options o;
  dgf_default_options(&o);
  if (opt) o = *opt;
  if (stored) {
    if (!c->d_store) DGF_FAIL(DGF_ERR_ARG, "no integral store: call dgf_store_integrals first");
    if (o.thrs != c->store_thrs) DGF_FAIL(DGF_ERR_ARG, "the integral store was made for another Schwarz threshold");
    if (o.mixed_cutoff > 0.0 || o.hfxmu != 0.0)
      DGF_FAIL(DGF_ERR_UNSUPPORTED, "stored integrals are FP64 1/r12 integrals: no mixed form, no range separation");
  }
  if (!(o.thrs >= 0.0)) DGF_FAIL(DGF_ERR_ARG, "thrs must be >= 0");
  if (o.shard_count <= 0) o.shard_count = 1;
  if (o.shard_index < 0 || o.shard_index >= o.shard_count) DGF_FAIL(DGF_ERR_ARG, "shard_index out of range");
  const int N = c->nwf;                            // working basis
  const size_t n2 = (size_t)N * N;
  const size_t n2ao = (size_t)c->nbf * c->nbf;     // AO-basis inputs and outputs
  const WorkMaps wmaps = ctx_maps(c);
  // Decode IFCTYP into density slots and output combinations.
  std::vector<SlotSpec> slots;
  struct OutSpec {
    int s1, s2;
    double sign;
    bool zero;
  };
  std::vector<OutSpec> outs;
  if (!std::isfinite(o.hfxmu) || !std::isfinite(o.hfxatt)) DGF_FAIL(DGF_ERR_ARG, "hfxmu and hfxatt must be finite");
  const bool attenuated = o.hfxmu != 0.0 && o.hfxatt != 0.0;
  for (int k = 0; k < ndmat; ++k) {
    const int X = (int)(ifctyp[k] / 10), Y0 = (int)(ifctyp[k] % 10);
    if (X < 0 || X > 2 || Y0 < 1 || Y0 > 3) DGF_FAIL(DGF_ERR_UNSUPPORTED, "unsupported IFCTYP");
    int Y = Y0;
    if (X == 2) Y &= 2;                 // antisymmetric density: no Coulomb part
    if (o.hfxfac == 0.0) Y &= 1;        // no exchange
    const double js = (Y & 1) ? 1.0 : 0.0, ks = (Y & 2) ? 0.5 * o.hfxfac : 0.0;
    // attenuated pass: exchange only, scaled by HFXATT (herfckcon.F:59-66)
    const double ka = attenuated ? 0.5 * o.hfxatt : 0.0;
    if (Y == 0 && ka == 0.0) {
      outs.push_back({0, 0, 0.0, true});
      continue;
    }
    if (X == 1) {
      slots.push_back({k, 2, js, ks, ka});
      const int s = (int)slots.size() - 1;
      outs.push_back({s, s, 1.0, false});
    } else if (X == 2) {
      slots.push_back({k, 3, js, ks, ka});
      const int s = (int)slots.size() - 1;
      outs.push_back({s, s, -1.0, false});
    } else {
      slots.push_back({k, 0, js, ks, ka});
      slots.push_back({k, 1, js, ks, ka});
      const int s = (int)slots.size() - 2;
      outs.push_back({s, s + 1, 1.0, false});
    }
  }
  int st_code = build_plan(c, o.thrs);
  if (st_code) return st_code;
  // Density screening as Dalton's direct Fock build: on when IFTHRS < 16,
  // IFTHRS < 4 taken as 14 (DALTON/abacus/her2drv.F:520-540).
  int64_t ifthrs = o.ifthrs;
  if (ifthrs < 4) ifthrs = 14;
  const bool doscrn = ifthrs < 16;
  const bool ice = doscrn && (o.icedif & 3) != 0;
  const bool need_dmax = o.mixed_cutoff > 0.0;
  const int nslot_total = (int)slots.size();
  const int chunk = std::min(kMaxSlots, std::max(nslot_total, 1));
  st_code = ensure_slots(c, chunk);
  if (st_code) return st_code;
  if (doscrn) {
    st_code = ensure_block_screen(c, chunk);
    if (st_code) return st_code;
  }
  if (c->profiling) {
    for (cudaEvent_t e : c->prof_ev) cudaEventDestroy(e);
    c->prof_ev.clear();
    c->prof.clear();
  }
  DGF_CUDA_CHECK(cudaMemsetAsync(c->d_cnt, 0, 4 * kCounterSlots * sizeof(unsigned long long), st));
  DGF_CUDA_CHECK(cudaEventRecord(c->ev0, st));
  int64_t launches = 0, total_q = 0, nlaunch_class = 0;
  std::vector<int64_t> sq0(c->plan.size()), sq1(c->plan.size());
  for (size_t e = 0; e < c->plan.size(); ++e) {
    shard_range(c, e, o.shard_index, o.shard_count, &sq0[e], &sq1[e]);
    total_q += sq1[e] - sq0[e];
  }
  // Zero outputs that have no contributions.
  for (int k = 0; k < ndmat; ++k)
    if (outs[k].zero) DGF_CUDA_CHECK(cudaMemsetAsync(fmat_dev + (size_t)k * n2ao, 0, n2ao * 8, st));
  const int nws = c->nwshell;
  const int *d_shinfo = c->d_shinfo;
  for (int s0 = 0; s0 < nslot_total; s0 += chunk) {
    const int ns = std::min(chunk, nslot_total - s0);
    for (int s = 0; s < ns; ++s) {
      const SlotSpec &sp = slots[s0 + s];
      launch_work_prep(wmaps, dmat_dev + (size_t)sp.src * n2ao, c->d_D + s * n2, c->d_Ds + s * n2, sp.op,
                       (int64_t)n2, c->nsm, st);
      ++launches;
    }
    DGF_CUDA_CHECK(cudaMemsetAsync(c->d_Fh, 0, ns * n2 * 8, st));
    if (need_dmax) {
      dmax_kernel<<<std::max(1, std::min(nws * nws / 128 + 1, c->nsm * 8)), 128, 0, st>>>(
          c->d_D, ns, N, d_shinfo, d_shinfo + nws, nws, c->d_dmax);
      ++launches;
    }
    const int64_t nb2 = (int64_t)c->nblk * c->nblk;
    if (doscrn) {
      SlotSources ss;
      ss.nslot = ns;
      for (int s = 0; s < ns; ++s) ss.src[s] = slots[s0 + s].src;
      blk_dmax_kernel<<<(int)std::max<int64_t>(1, std::min<int64_t>(nb2 / 128 + 1, c->nsm * 8)), 128, 0, st>>>(
          dmat_dev, c->nbf, c->d_blk_info, c->d_blk_info + c->nblk, c->nblk, ss, c->d_blk_dmax, c->d_blk_dmax + nb2);
      ++launches;
    }
    JKArgs a = base_args(c);
    a.nslot = ns;
    a.D = c->d_D;
    a.Ds = c->d_Ds;
    a.Fh = c->d_Fh;
    a.dmax = need_dmax ? c->d_dmax : nullptr;
    a.dens_thr = doscrn ? std::pow(10.0, -(double)ifthrs) : 0.0;
    a.blk_gab = doscrn ? c->d_blk_gab : nullptr;
    a.blk_dmax = doscrn ? c->d_blk_dmax : nullptr;
    a.blk_dmax_slot = doscrn ? c->d_blk_dmax + nb2 : nullptr;
    a.blk_stride = nb2;
    a.nblk = c->nblk;
    a.ice_thr = ice ? a.dens_thr : 0.0;
    a.icedif = (int)(o.icedif & 3);
    a.split = o.mixed_cutoff;
    a.schwarz_thr = o.thrs;
    a.mode = 0;
    // Pass 0: 1/r12 with the slots' Coulomb and exchange scales; pass 1
    // (range-separated exchange): erf(mu r12)/r12, exchange only.
    for (int pass = 0; pass < (attenuated ? 2 : 1); ++pass) {
      bool any = false;
      for (int s = 0; s < ns; ++s) {
        a.jscale[s] = pass == 0 ? slots[s0 + s].js : 0.0;
        a.kscale[s] = pass == 0 ? slots[s0 + s].ks : slots[s0 + s].ka;
        any = any || a.jscale[s] != 0.0 || a.kscale[s] != 0.0;
      }
      a.erf_mu2 = pass == 0 ? 0.0 : o.hfxmu * o.hfxmu;
      if (!any) continue;
      for (size_t e = 0; e < c->plan.size(); ++e) {
        const ClassPlan &cp = c->plan[e];
        if (sq1[e] <= sq0[e]) continue;  // not in this shard
        a.bra = c->d_pairs + c->cls_off[cp.X];
        a.ket = c->d_pairs + c->cls_off[cp.Y] + cp.kb0;
        a.ket_off = cp.kb0;
        a.ket_pp0 = ket_pp0_of(c, cp);
        set_ket_table(c, cp, a);
        a.nbra = c->cls_off[cp.X + 1] - c->cls_off[cp.X];
        a.same_class = (cp.X == cp.Y);
        a.qoff = c->d_qoff + cp.off;
        a.q_begin = sq0[e];
        a.nquartet = sq1[e];
        // Boys table of order L = la+lb+lc+ld.
        const int la = (cp.X == 0) ? 0 : (cp.X <= 2) ? 1 : (cp.X <= 5) ? 2 : 3;
        const int lb = cp.X - la * (la + 1) / 2;
        const int lc = (cp.Y == 0) ? 0 : (cp.Y <= 2) ? 1 : (cp.Y <= 5) ? 2 : 3;
        const int ld = cp.Y - lc * (lc + 1) / 2;
        a.boys = c->d_boys + (size_t)(la + lb + lc + ld) * kBoysTableDoubles;
        const bool split = o.mixed_cutoff > 0.0 && c->split_ok[cp.X][cp.Y] &&
                           select_kernel(c, cp.X, cp.Y, 1, cp.bucket == 0).launch != nullptr;
        const int Lq = la + lb + lc + ld;
        if (stored) {  // conventional form: digest the stored blocks
          a.store_in = c->d_store;
          a.store_base = c->store_off[e];
          a.store_nint = (int)store_nint(c, cp.X, cp.Y);
          a.mode = 0;
          a.counters = c->d_cnt + 4 * (nlaunch_class % kCounterSlots);
          ++nlaunch_class;
          int r = launch_kernel(c, jk_stored_kernel(cp.X, cp.Y), cp.X, cp.Y, a, st, 0);
          if (r) return r;
          ++launches;
          continue;
        }
        for (int part = 0; part < (split ? 2 : 1); ++part) {
          a.mode = split ? 1 + part : 0;
          // the FP32 half reads the low-degree Boys table
          a.boys = c->d_boys + ((split && part == 1) ? boys_low_offset(Lq) : (size_t)Lq * kBoysTableDoubles);
          a.counters = c->d_cnt + 4 * (nlaunch_class % kCounterSlots);
          ++nlaunch_class;
          int r = launch_class(c, cp.X, cp.Y, a, st, split && part == 1 ? 1 : 0, cp.bucket == 0);
          if (r) return r;
          ++launches;
        }
      }
    }
    // Combine the slots of this chunk into the outputs they belong to.
    for (int k = 0; k < ndmat; ++k) {
      const OutSpec &os = outs[k];
      if (os.zero || os.s1 < s0 || os.s1 >= s0 + ns) continue;
      launch_work_combine(wmaps, c->d_Fh + (os.s1 - s0) * n2, c->d_Fh + (os.s2 - s0) * n2,
                          fmat_dev + (size_t)k * n2ao, os.sign, (int64_t)n2ao, c->nsm, st);
      ++launches;
    }
  }
  DGF_CUDA_CHECK(cudaGetLastError());
  DGF_CUDA_CHECK(cudaEventRecord(c->ev1, st));
  st_code = finish_profile(c, st);
  if (st_code) return st_code;
  if (stats || c->profiling) {
    std::vector<unsigned long long> all(4 * kCounterSlots);
    DGF_CUDA_CHECK(cudaMemcpyAsync(all.data(), c->d_cnt, all.size() * 8, cudaMemcpyDeviceToHost, st));
    DGF_CUDA_CHECK(cudaStreamSynchronize(st));
    unsigned long long cnt[4] = {0, 0, 0, 0};
    for (int i = 0; i < kCounterSlots; ++i)
      for (int k = 0; k < 4; ++k) cnt[k] += all[4 * i + k];
    if (c->profiling)
      for (size_t i = 0; i < c->prof.size() && i < (size_t)kCounterSlots; ++i) {
        c->prof[i].evaluated = (int64_t)all[4 * i];
        c->prof[i].prim_quartets = (int64_t)all[4 * i + 1];
      }
    if (!stats) return DGF_OK;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    (void)total_q;
    stats->quartets_total = (int64_t)(cnt[0] + cnt[2]);  // passed Schwarz: evaluated or density-skipped
    stats->quartets_fp64 = (int64_t)(cnt[0] - cnt[3]);
    stats->quartets_fp32 = (int64_t)cnt[3];
    stats->quartets_skipped = (int64_t)cnt[2];
    stats->prim_quartets = (int64_t)cnt[1];
    stats->kernel_launches = launches;
    stats->ms_device = ms;
  }
  return DGF_OK;
}

static int check_fock_args(dgf_ctx *c, dgf_int ndmat, const dgf_int *ifctyp, const void *d, const void *f) {
  if (!c) DGF_FAIL(DGF_ERR_ARG, "ctx is NULL");
  if (ndmat < 0) DGF_FAIL(DGF_ERR_ARG, "ndmat < 0");
  if (ndmat > 0 && (!ifctyp || !d || !f)) DGF_FAIL(DGF_ERR_ARG, "NULL matrix or IFCTYP array");
  return DGF_OK;
}

extern "C" int dgf_fock_device(dgf_ctx *c, dgf_int ndmat, const dgf_int *ifctyp, const double *dmat_device,
                               double *fmat_device, const dgf_options *opt, void *stream, dgf_stats *stats) {
  int r = check_fock_args(c, ndmat, ifctyp, dmat_device, fmat_device);
  if (r || ndmat == 0) return r;
  DeviceGuard g(c->device);
  return fock_impl(c, (int)ndmat, ifctyp, dmat_device, fmat_device, opt, (cudaStream_t)stream, stats);
}

// An integral kernel that writes whole blocks: the tuned choice unless it is
// a thread kernel split into A-component chunks, else a one-chunk thread
// variant, else the warp-per-quartet kernel, else the cooperative one.
static const ClassKernel &store_kernel(const dgf_ctx *c, int X, int Y, bool ket1) {
  const bool bra1 = c->cls_max_npp[X] == 1;
  const ClassKernel &t = jk_kernel_variant(X, Y, 0, c->choice[X][Y][0], ket1, bra1);
  if (t.launch && (t.kind != kKindThread || t.chunks == 1)) return t;
  for (int v = 0; v < kThreadVariants; ++v) {
    const ClassKernel &k = jk_kernel_variant(X, Y, 0, v, ket1, bra1);
    if (k.launch && k.chunks == 1) return k;
  }
  const ClassKernel &w = jk_kernel_variant(X, Y, 0, -3, ket1, bra1);
  if (w.launch) return w;
  return jk_kernel_variant(X, Y, 0, -1, ket1, bra1);
}

extern "C" int dgf_store_integrals(dgf_ctx *c, double thrs, int64_t max_bytes, void *stream, int64_t *bytes) {
  if (!c) DGF_FAIL(DGF_ERR_ARG, "ctx is NULL");
  if (!(thrs >= 0.0)) DGF_FAIL(DGF_ERR_ARG, "thrs must be >= 0");
  DeviceGuard g(c->device);
  int r = build_plan(c, thrs);
  if (r) return r;
  std::vector<int64_t> off(c->plan.size());
  int64_t tot = 0;
  for (size_t e = 0; e < c->plan.size(); ++e) {
    off[e] = tot;
    tot += c->plan[e].nquartet * store_nint(c, c->plan[e].X, c->plan[e].Y);
  }
  if (bytes) *bytes = tot * 8;
  if (max_bytes > 0 && tot * 8 > max_bytes)
    DGF_FAIL(DGF_ERR_NOMEM, "the integral store needs " + std::to_string(tot * 8) + " bytes, more than max_bytes");
  if (c->d_store) cudaFree(c->d_store);
  c->d_store = nullptr;
  c->store_doubles = 0;
  c->store_thrs = -1.0;
  if (dev_alloc(&c->d_store, (size_t)std::max<int64_t>(tot, 1)) != cudaSuccess) {
    cudaGetLastError();
    c->d_store = nullptr;
    DGF_FAIL(DGF_ERR_NOMEM, "device allocation of the integral store (" + std::to_string(tot * 8) + " bytes) failed");
  }
  r = ensure_slots(c, 1);
  if (r) return r;
  cudaStream_t st = (cudaStream_t)stream;
  JKArgs a = base_args(c);
  a.nslot = 1;
  a.D = c->d_D;
  a.Ds = c->d_Ds;
  a.Fh = c->d_Fh;
  a.schwarz_thr = thrs;
  a.store_out = c->d_store;
  const int saved_prof = c->profiling;
  c->profiling = 0;
  for (size_t e = 0; e < c->plan.size(); ++e) {
    const ClassPlan &cp = c->plan[e];
    if (cp.nquartet <= 0) continue;
    a.bra = c->d_pairs + c->cls_off[cp.X];
    a.ket = c->d_pairs + c->cls_off[cp.Y] + cp.kb0;
    a.ket_off = cp.kb0;
    a.ket_pp0 = ket_pp0_of(c, cp);
    set_ket_table(c, cp, a);
    a.nbra = c->cls_off[cp.X + 1] - c->cls_off[cp.X];
    a.same_class = (cp.X == cp.Y);
    a.qoff = c->d_qoff + cp.off;
    a.q_begin = 0;
    a.nquartet = cp.nquartet;
    const int Lq = cls_l1(cp.X) + (cp.X - cls_l1(cp.X) * (cls_l1(cp.X) + 1) / 2) + cls_l1(cp.Y) +
                   (cp.Y - cls_l1(cp.Y) * (cls_l1(cp.Y) + 1) / 2);
    a.boys = c->d_boys + (size_t)Lq * kBoysTableDoubles;
    a.store_base = off[e];
    a.store_nint = (int)store_nint(c, cp.X, cp.Y);
    a.counters = c->d_cnt;
    r = launch_kernel(c, store_kernel(c, cp.X, cp.Y, cp.bucket == 0), cp.X, cp.Y, a, st, 0);
    if (r) {
      c->profiling = saved_prof;
      return r;
    }
  }
  c->profiling = saved_prof;
  DGF_CUDA_CHECK(cudaGetLastError());
  c->store_off.swap(off);
  c->store_doubles = tot;
  c->store_thrs = thrs;
  return DGF_OK;
}

extern "C" int dgf_store_release(dgf_ctx *c) {
  if (!c) DGF_FAIL(DGF_ERR_ARG, "ctx is NULL");
  DeviceGuard g(c->device);
  if (c->d_store) cudaFree(c->d_store);
  c->d_store = nullptr;
  c->store_doubles = 0;
  c->store_thrs = -1.0;
  c->store_off.clear();
  return DGF_OK;
}

extern "C" int dgf_fock_stored(dgf_ctx *c, dgf_int ndmat, const dgf_int *ifctyp, const double *dmat_device,
                               double *fmat_device, const dgf_options *opt, void *stream, dgf_stats *stats) {
  int r = check_fock_args(c, ndmat, ifctyp, dmat_device, fmat_device);
  if (r || ndmat == 0) return r;
  DeviceGuard g(c->device);
  return fock_impl(c, (int)ndmat, ifctyp, dmat_device, fmat_device, opt, (cudaStream_t)stream, stats, true);
}

extern "C" int dgf_fock(dgf_ctx *c, dgf_int ndmat, const dgf_int *ifctyp, const double *dmat, double *fmat,
                        const dgf_options *opt, dgf_stats *stats) {
  int r = check_fock_args(c, ndmat, ifctyp, dmat, fmat);
  if (r || ndmat == 0) return r;
  DeviceGuard g(c->device);
  const size_t n2 = (size_t)c->nbf * c->nbf;
  if ((int)ndmat * 2 > c->cap_io) {
    if (c->d_io) cudaFree(c->d_io);
    c->d_io = nullptr;
    c->cap_io = 0;
    if (dev_alloc(&c->d_io, 2 * ndmat * n2) != cudaSuccess) {
      cudaGetLastError();
      DGF_FAIL(DGF_ERR_NOMEM, "device allocation of the D/F staging buffers failed");
    }
    c->cap_io = (int)ndmat * 2;
  }
  double *dD = c->d_io, *dF = c->d_io + ndmat * n2;
  DGF_CUDA_CHECK(cudaMemcpyAsync(dD, dmat, ndmat * n2 * 8, cudaMemcpyHostToDevice, c->stream));
  r = fock_impl(c, (int)ndmat, ifctyp, dD, dF, opt, c->stream, stats);
  if (r) return r;
  DGF_CUDA_CHECK(cudaMemcpyAsync(fmat, dF, ndmat * n2 * 8, cudaMemcpyDeviceToHost, c->stream));
  DGF_CUDA_CHECK(cudaStreamSynchronize(c->stream));
  return DGF_OK;
}

extern "C" const char *dgf_strerror(int s) {
  switch (s) {
    case DGF_OK: return "success";
    case DGF_ERR_ARG: return "invalid argument";
    case DGF_ERR_NOMEM: return "out of memory";
    case DGF_ERR_CUDA: return "CUDA runtime error";
    case DGF_ERR_UNSUPPORTED: return "unsupported angular momentum, IFCTYP or option";
    case DGF_ERR_TIMEOUT: return "bounded device wait timed out";
    case DGF_ERR_NODEVICE: return "no usable CUDA device";
    default: return "unknown status";
  }
}

extern "C" const char *dgf_last_error(void) { return dgf::g_last_error.c_str(); }

// Copy the per-class kernel choices of one context to another (contexts of
// similar molecules share a tuning run).
extern "C" int dgf_copy_tuning(dgf_ctx *dst, const dgf_ctx *src) {
  if (!dst || !src) DGF_FAIL(DGF_ERR_ARG, "NULL context");
  memcpy(dst->choice, src->choice, sizeof(dst->choice));
  memcpy(dst->split_ok, src->split_ok, sizeof(dst->split_ok));
  return DGF_OK;
}

extern "C" int dgf_set_class_kernel(dgf_ctx *c, int la, int lb, int lc, int ld, int precision, int variant) {
  if (!c) DGF_FAIL(DGF_ERR_ARG, "NULL context");
  if (la < lb || lc < ld || lb < 0 || ld < 0 || la > kMaxShellL || lc > kMaxShellL)
    DGF_FAIL(DGF_ERR_ARG, "class angular momenta must satisfy la >= lb >= 0, lc >= ld >= 0, at most f");
  if (precision != 64 && precision != 32) DGF_FAIL(DGF_ERR_ARG, "precision must be 64 or 32");
  int X = la * (la + 1) / 2 + lb, Y = lc * (lc + 1) / 2 + ld;
  if (X < Y) std::swap(X, Y);
  const int p = precision == 32 ? 1 : 0;
  const bool bra1 = c->cls_max_npp[X] == 1;
  if (!jk_kernel_variant(X, Y, p, variant, false, bra1).launch && !jk_kernel_variant(X, Y, p, variant, true, bra1).launch)
    DGF_FAIL(DGF_ERR_UNSUPPORTED, "no such kernel variant for this class and precision");
  c->choice[X][Y][p] = variant;
  return DGF_OK;
}

// Per-class autotuner: times every candidate kernel of every class pair of
// the current plan on the given density (team kernel and each thread-kernel
// chunk variant, FP64 and FP32) with CUDA events and keeps the fastest.
extern "C" int dgf_autotune(dgf_ctx *c, const double *dmat_device, const dgf_options *opt, void *stream,
                            char *report, size_t report_len) {
  if (!c || !dmat_device) DGF_FAIL(DGF_ERR_ARG, "NULL argument");
  DeviceGuard g(c->device);
  dgf_options o;
  dgf_default_options(&o);
  if (opt) o = *opt;
  cudaStream_t st = (cudaStream_t)stream;
  int r = build_plan(c, o.thrs);
  if (r) return r;
  r = ensure_slots(c, 1);
  if (r) return r;
  launch_work_prep(ctx_maps(c), dmat_device, c->d_D, c->d_Ds, 2, (int64_t)c->nwf * c->nwf, c->nsm, st);
  if (o.mixed_cutoff > 0.0) {
    const int nws = c->nwshell;
    dmax_kernel<<<std::max(1, std::min(nws * nws / 128 + 1, c->nsm * 8)), 128, 0, st>>>(
        c->d_D, 1, c->nwf, c->d_shinfo, c->d_shinfo + nws, nws, c->d_dmax);
  }
  DGF_CUDA_CHECK(cudaGetLastError());
  cudaEvent_t e0, e1;
  DGF_CUDA_CHECK(cudaEventCreate(&e0));
  DGF_CUDA_CHECK(cudaEventCreate(&e1));
  std::string rep = "[";
  const int saved_prof = c->profiling;
  c->profiling = 0;
  // candidates are timed over all bucket entries of a class pair
  for (size_t ip = 0; ip < c->plan.size();) {
    size_t jp = ip;
    while (jp < c->plan.size() && c->plan[jp].X == c->plan[ip].X && c->plan[jp].Y == c->plan[ip].Y) ++jp;
    const ClassPlan &cp = c->plan[ip];
    JKArgs a = base_args(c);
    a.schwarz_thr = o.thrs;
    a.nslot = 1;
    a.D = c->d_D;
    a.Ds = c->d_Ds;
    a.Fh = c->d_Fh;
    a.jscale[0] = 1.0;
    a.kscale[0] = 0.5 * o.hfxfac;
    a.bra = c->d_pairs + c->cls_off[cp.X];
    a.nbra = c->cls_off[cp.X + 1] - c->cls_off[cp.X];
    a.same_class = (cp.X == cp.Y);
    a.q_begin = 0;
    const int la = cls_l1(cp.X), lb = cp.X - la * (la + 1) / 2, lc = cls_l1(cp.Y), ld = cp.Y - lc * (lc + 1) / 2;
    a.boys = c->d_boys + (size_t)(la + lb + lc + ld) * kBoysTableDoubles;
    float best_prec[2] = {1e30f, 1e30f};
    for (int p = 0; p < 2; ++p) {
      float best = 1e30f;
      int bestv = c->choice[cp.X][cp.Y][p];
      a.boys = c->d_boys + (p ? boys_low_offset(la + lb + lc + ld) : (size_t)(la + lb + lc + ld) * kBoysTableDoubles);
      const bool bra1 = c->cls_max_npp[cp.X] == 1;
      // With the warp-per-quartet kernel available for the class's
      // single-primitive launches, the cooperative kernels are not timed
      // (they are several times slower wherever both exist).
      const bool has_warp = bra1 && jk_kernel_variant(cp.X, cp.Y, p, -3, true, bra1).launch != nullptr;
      for (int v = -4; v < kThreadVariants; ++v) {
        if (!jk_kernel_variant(cp.X, cp.Y, p, v, false, bra1).launch &&
            !jk_kernel_variant(cp.X, cp.Y, p, v, true, bra1).launch)
          continue;
        if (has_warp && (v == -1 || v == -2)) continue;
        int chunks = 1;
        float ms = 0.f;
        for (int rep2 = 0; rep2 < 2; ++rep2) {  // a first pass warms caches unless it is long
          if (rep2 == 1 && ms > 20.f) break;
          DGF_CUDA_CHECK(cudaEventRecord(e0, st));
          for (size_t q = ip; q < jp; ++q) {
            const ClassPlan &cq = c->plan[q];
            a.ket = c->d_pairs + c->cls_off[cq.Y] + cq.kb0;
            a.ket_off = cq.kb0;
            a.ket_pp0 = ket_pp0_of(c, cq);
            set_ket_table(c, cq, a);
            a.qoff = c->d_qoff + cq.off;
            a.nquartet = cq.nquartet;
            // entries this candidate has no kernel for run the FP64 default (same for every candidate)
            const ClassKernel &kv = jk_kernel_variant(cq.X, cq.Y, p, v, cq.bucket == 0, bra1);
            const ClassKernel &k = kv.launch ? kv : jk_kernel(cq.X, cq.Y, 0, cq.bucket == 0, bra1);
            if (kv.launch) chunks = k.chunks;
            r = launch_kernel(c, k, cq.X, cq.Y, a, st, kv.launch ? p : 0);
            if (r) return r;
          }
          DGF_CUDA_CHECK(cudaEventRecord(e1, st));
          DGF_CUDA_CHECK(cudaEventSynchronize(e1));
          DGF_CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
        }
        char buf[160];
        snprintf(buf, sizeof(buf), "%s{\"class\":[%d,%d,%d,%d],\"precision\":%d,\"variant\":%d,\"chunks\":%d,\"ms\":%.4f}",
                 rep.size() > 1 ? "," : "", la, lb, lc, ld, p ? 32 : 64, v, chunks, ms);
        rep += buf;
        if (ms < best) {
          best = ms;
          bestv = v;
        }
      }
      c->choice[cp.X][cp.Y][p] = bestv;
      best_prec[p] = best;
    }
    // Mixed form: split the class into FP64 and FP32 launches only where
    // that beats one FP64 pass (both walk all of the class's quartets).
    // The split runs an FP64 and an FP32 launch over the whole queue; it can
    // only win when the FP32 kernel is faster than the FP64 one.
    if (o.mixed_cutoff > 0.0) c->split_ok[cp.X][cp.Y] = 0;
    if (o.mixed_cutoff > 0.0 && best_prec[1] < best_prec[0] &&
        (select_kernel(c, cp.X, cp.Y, 1, false).launch || select_kernel(c, cp.X, cp.Y, 1, true).launch)) {
      const int Lq = la + lb + lc + ld;
      float t[2] = {0.f, 0.f};
      for (int cfg = 0; cfg < 2; ++cfg) {  // 0: FP64 only, 1: FP64 + FP32 halves
        for (int rep2 = 0; rep2 < 2; ++rep2) {
          if (rep2 == 1 && t[cfg] > 20.f) break;
          DGF_CUDA_CHECK(cudaEventRecord(e0, st));
          for (size_t q = ip; q < jp; ++q) {
            const ClassPlan &cq = c->plan[q];
            a.ket = c->d_pairs + c->cls_off[cq.Y] + cq.kb0;
            a.ket_off = cq.kb0;
            a.ket_pp0 = ket_pp0_of(c, cq);
            set_ket_table(c, cq, a);
            a.qoff = c->d_qoff + cq.off;
            a.nquartet = cq.nquartet;
            a.dmax = c->d_dmax;
            a.split = o.mixed_cutoff;
            // as in the build: entries without an FP32 kernel are not split
            const bool cansplit = select_kernel(c, cq.X, cq.Y, 1, cq.bucket == 0).launch != nullptr;
            for (int part = 0; part < (cfg && cansplit ? 2 : 1); ++part) {
              const int prec = (cfg && part == 1) ? 1 : 0;
              a.mode = (cfg && cansplit) ? 1 + part : 0;
              a.boys = c->d_boys + (prec ? boys_low_offset(Lq) : (size_t)Lq * kBoysTableDoubles);
              r = launch_class(c, cq.X, cq.Y, a, st, prec, cq.bucket == 0);
              if (r) return r;
            }
          }
          DGF_CUDA_CHECK(cudaEventRecord(e1, st));
          DGF_CUDA_CHECK(cudaEventSynchronize(e1));
          DGF_CUDA_CHECK(cudaEventElapsedTime(&t[cfg], e0, e1));
        }
      }
      a.dmax = nullptr;
      a.mode = 0;
      c->split_ok[cp.X][cp.Y] = t[1] < t[0] ? 1 : 0;
      char buf[160];
      snprintf(buf, sizeof(buf), "%s{\"class\":[%d,%d,%d,%d],\"split\":%d,\"ms_fp64\":%.4f,\"ms_split\":%.4f}",
               rep.size() > 1 ? "," : "", la, lb, lc, ld, c->split_ok[cp.X][cp.Y], t[0], t[1]);
      rep += buf;
    }
    ip = jp;
  }
  c->profiling = saved_prof;
  rep += "]";
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (report && report_len) {
    strncpy(report, rep.c_str(), report_len - 1);
    report[report_len - 1] = 0;
  }
  return DGF_OK;
}
