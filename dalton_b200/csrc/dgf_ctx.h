// Context of libdgfock (the opaque dgf_ctx of the C ABI): device-resident
// shell-pair data and the per-call scratch of one molecule/basis.
#pragma once

#include "../../include/dgfock.h"
#include "dgf_internal.h"
#include "dgf_work.h"

#define DGF_CUDA_CHECK(expr)                                                   \
  do {                                                                         \
    cudaError_t _e = (expr);                                                   \
    if (_e != cudaSuccess) {                                                   \
      ::dgf::set_error(__FILE__, __LINE__, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
      return DGF_ERR_CUDA;                                                     \
    }                                                                          \
  } while (0)


constexpr int kCounterSlots = 256;

struct ClassPlan {
  int X, Y;
  int bucket;         // primitive-count bucket of the kets (0: one primitive pair each)
  int kb0, kb1;       // ket range of this entry: one primitive-count bucket of class Y (relative to its start)
  int64_t off;        // offset of this entry's qoff array in the plan buffer
  int64_t nquartet;
};

// Map between the AO basis (Dalton's contracted functions) and the
// two-electron working basis, as sparse rows: wr_* gives, for every working
// function, the AO functions it contributes to with the contraction
// coefficient (D_w = C D C^T); ac_* gives, for every AO function, the working
// functions it is made of (F = C^T F_w C).  Device copies in one allocation.
struct WorkMapHost {
  std::vector<int> wr_off, wr_idx, ac_off, ac_idx;
  std::vector<double> wr_c, ac_c;
};

struct dgf_ctx {
  int device = 0, nbf = 0, natom = 0, nshell = 0, spherical = 1, maxl = 0, nsm = 148;
  std::vector<double> xyz, charge;
  // AO shells: one per contracted function of a Dalton block (one-electron
  // integrals and gradients work on these)
  std::vector<int> sh_l, sh_atom, sh_ao, sh_nprim, sh_p0;
  std::vector<double> sh_a, sh_c;
  // Two-electron working basis: a block whose contracted functions share
  // primitives (a general contraction) is resolved into one shell per
  // primitive; every other block keeps one shell per contracted function.
  // nwf functions in nwshell shells; w_identity when no block was resolved
  // (the working basis is then the AO basis, function for function).
  int nwf = 0, nwshell = 0, w_identity = 1;
  std::vector<int> ws_l, ws_atom, ws_ao, ws_nprim, ws_p0;
  std::vector<double> ws_a, ws_c;
  WorkMapHost wmap;
  int *d_wmap_i = nullptr;      // wr_off | wr_idx | ac_off | ac_idx
  double *d_wmap_c = nullptr;   // wr_c | ac_c
  int64_t *d_wmeta = nullptr;   // {0, nwf^2} {0, nbf^2} element offsets of the single-molecule form
  int *d_wdims = nullptr;       // {nwf, nbf, 0, 0}
  double *d_gw = nullptr;       // working-basis densities of the two-electron gradient (2 nwf^2)
  int *d_shinfo = nullptr;      // per working shell: first function | function count (density bounds)
  // conventional form: the integral store (dgf_store_integrals) for the plan
  // of store_thrs, one block of store_nint(X, Y) values per quartet, plan
  // entry e starting at store_off[e]
  double *d_store = nullptr;
  int64_t store_doubles = 0;
  double store_thrs = -1.0;
  std::vector<int64_t> store_off;
  std::vector<dgf::PairRec> pairs;  // class-major, Schwarz-descending inside a class
  int cls_off[dgf::kNumPairClass + 1] = {0};
  // per class: bucket boundaries (relative to the class start), pairs sorted by (bucket, -Schwarz bin, shells)
  int bkt_off[dgf::kNumPairClass][dgf::kNumBuckets + 1] = {};
  double cls_avg_npp[dgf::kNumPairClass] = {};  // mean primitive pairs of a class's pairs (shard cost model)
  int cls_max_npp[dgf::kNumPairClass] = {};     // most primitive pairs of a class's pairs
  std::vector<dgf::PrimPair> pp;
  dgf::PairRec *d_pairs = nullptr;
  // ket table of single-primitive kets (JKArgs::ks_*), one entry per pair of
  // d_pairs; null when a shell index does not fit 16 bits
  int4 *d_ks_i = nullptr;
  double *d_ks_q = nullptr, *d_ks_pp = nullptr;
  dgf::PrimPair *d_pp = nullptr;
  double *d_boys = nullptr, *d_sph = nullptr;
  // per-call buffers
  int cap_slots = 0, cap_io = 0;
  double *d_D = nullptr, *d_Ds = nullptr, *d_Fh = nullptr, *d_io = nullptr;
  float *d_dmax = nullptr;
  // Dalton blocks and the density screen on them: block of each AO shell
  // and working shell (ws_blk_flag with kWholeBlock where the shell is its
  // whole block), each block's first AO function and function count; device
  // block Schwarz factors (nblk^2, built at the first screened call), block
  // info (ao0 | nf) and block density maxima ((1 + cap_blk_slots) x nblk^2)
  int nblk = 0;
  std::vector<int> sh_blk, ws_blk, ws_blk_flag, blk_ao0, blk_nf;
  double *d_blk_gab = nullptr;
  int *d_blk_info = nullptr;
  float *d_blk_dmax = nullptr;
  int cap_blk_slots = 0;
  unsigned long long *d_cnt = nullptr;  // kCounterSlots x 4 per-launch counters
  // quartet plan, cached by Schwarz threshold
  double plan_thrs = -1.0;
  std::vector<ClassPlan> plan;
  int64_t *d_qoff = nullptr;
  size_t qoff_cap = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // kernel choice per class pair and precision (-1 = team kernel, >= 0 =
  // thread-kernel variant), set by the autotuner; 0 by default
  int choice[dgf::kNumPairClass][dgf::kNumPairClass][2] = {};
  // mixed form: whether a class pair is split into FP64 and FP32 launches
  // (set by the autotuner where the FP32 half pays for the second pass over
  // the class's quartets; every class splits by default)
  int split_ok[dgf::kNumPairClass][dgf::kNumPairClass];
  // per-class launch profiling (dgf_set_profiling)
  int profiling = 0;
  std::vector<cudaEvent_t> prof_ev;
  std::vector<dgf_class_time> prof;
};


// The single-molecule form of the AO <-> working-basis maps of a context.
inline dgf::WorkMaps ctx_maps(const dgf_ctx *c) {
  dgf::WorkMaps m;
  const size_t nr = c->wmap.wr_idx.size();
  m.nmol = 1;
  m.w_elem = c->d_wmeta;
  m.a_elem = c->d_wmeta + 2;
  m.nw = c->d_wdims;
  m.na = c->d_wdims + 1;
  m.wf_base = c->d_wdims + 2;
  m.af_base = c->d_wdims + 3;
  m.wr_off = c->d_wmap_i;
  m.wr_idx = c->d_wmap_i + (c->nwf + 1);
  m.ac_off = c->d_wmap_i + (c->nwf + 1) + nr;
  m.ac_idx = c->d_wmap_i + (c->nwf + 1) + nr + (c->nbf + 1);
  m.wr_c = c->d_wmap_c;
  m.ac_c = c->d_wmap_c + nr;
  return m;
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

