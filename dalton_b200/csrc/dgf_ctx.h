// Context of libdgfock (the opaque dgf_ctx of the C ABI): device-resident
// shell-pair data and the per-call scratch of one molecule/basis.
#pragma once

#include "../../include/dgfock.h"
#include "dgf_internal.h"

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
  int kb0, kb1;       // ket range of this entry: one primitive-count bucket of class Y (relative to its start)
  int64_t off;        // offset of this entry's qoff array in the plan buffer
  int64_t nquartet;
};

struct dgf_ctx {
  int device = 0, nbf = 0, natom = 0, nshell = 0, spherical = 1, maxl = 0, nsm = 148;
  std::vector<double> xyz, charge;
  std::vector<int> sh_l, sh_atom, sh_ao, sh_nprim, sh_p0;
  std::vector<double> sh_a, sh_c;
  std::vector<dgf::PairRec> pairs;  // class-major, Schwarz-descending inside a class
  int cls_off[dgf::kNumPairClass + 1] = {0};
  // per class: bucket boundaries (relative to the class start), pairs sorted by (bucket, -Q)
  int bkt_off[dgf::kNumPairClass][dgf::kNumBuckets + 1] = {};
  std::vector<dgf::PrimPair> pp;
  dgf::PairRec *d_pairs = nullptr;
  dgf::PrimPair *d_pp = nullptr;
  double *d_boys = nullptr, *d_sph = nullptr;
  // per-call buffers
  int cap_slots = 0, cap_io = 0;
  double *d_D = nullptr, *d_Ds = nullptr, *d_Fh = nullptr, *d_io = nullptr;
  float *d_dmax = nullptr;
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
  // per-class launch profiling (dgf_set_profiling)
  int profiling = 0;
  std::vector<cudaEvent_t> prof_ev;
  std::vector<dgf_class_time> prof;
};


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

