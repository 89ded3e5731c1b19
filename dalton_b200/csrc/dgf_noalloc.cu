// A Fock build that allocates no device memory.
//
// Some callers cannot allocate GPU memory at the moment they need a Fock
// matrix: a host program that, like Dalton, hands the engine a fixed work
// area and expects it to take nothing else (HERFCK's WORK/LWORK contract);
// a process whose device memory is already carved up by a pool it does not
// own; or a time-critical loop that cannot afford the implicit
// synchronisation of cudaMalloc/cudaFree.  dgf_fock_device_noalloc serves
// them: it runs the same quartet-class kernels as dgf_fock_device, but its
// scratch (the symmetrised density, D + D^T and the half Fock accumulator,
// all in the two-electron working basis) lives in one file-scope device
// array of fixed size that every GPU which loads this library holds until
// the process exits.
//
// Limits and sharing: at most kNoAllocMaxN basis functions and
// kNoAllocMaxW working functions; IFCTYP 13
// (J - hfxfac/2 K of one symmetric density), all-FP64, Schwarz screening
// only; the context's quartet plan for `thrs` must already exist (any
// earlier dgf_fock, dgf_fock_device, dgf_autotune or dgf_grad2e call with the
// same threshold builds it).  All calls share the one array per device and
// it keeps the last call's contents; the accumulator is cleared at the start
// of each call.  Calls whose work overlaps on the GPU (different streams,
// different host threads) race on the array and must be serialised by the
// caller.
#include <cstring>
#include <mutex>
#include <string>

#include "dgf_ctx.h"
#include "dgf_md.cuh"

using namespace dgf;

namespace {

constexpr int kNoAllocMaxN = 768;
constexpr int kNoAllocMaxW = 1536;  // working functions (general contractions resolved into primitives)
constexpr size_t kNoAllocDoubles = 3 * (size_t)kNoAllocMaxW * kNoAllocMaxW;  // 56.6 MB

// The scratch of the no-allocation Fock build (see the file comment).  In
// host code this name is only a stand-in for the device array, never a
// device address: the address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

constexpr int kMaxDevices = 64;
double *g_scratch_addr[kMaxDevices] = {};
std::mutex g_setup_mutex;

// Device address of the scratch array on the current device, looked up once
// per device by the first call made on it (make that call before any stream
// capture).  The address stays valid for the life of the device's primary
// context: after a cudaDeviceReset on that device the cached address is
// stale, so a process that resets a device must not call this entry point
// on it again.
cudaError_t scratch_address(int device, double **out) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[device]) {
    double *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress((void **)&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[device] = p;
  }
  *out = g_scratch_addr[device];
  return cudaSuccess;
}

int fail(int code, int line, const std::string &msg) {
  dgf::set_error(__FILE__, line, msg);
  return code;
}

}  // namespace

extern "C" int dgf_fock_device_noalloc(dgf_ctx *c, const double *dmat_device, double *fmat_device, double hfxfac,
                                       double thrs, void *stream) {
  if (!c || !dmat_device || !fmat_device) return fail(DGF_ERR_ARG, __LINE__, "NULL argument");
  if (c->nbf > kNoAllocMaxN)
    return fail(DGF_ERR_ARG, __LINE__,
                "dgf_fock_device_noalloc: " + std::to_string(c->nbf) + " basis functions exceed its fixed scratch (" +
                    std::to_string(kNoAllocMaxN) + " at most); use dgf_fock_device");
  if (c->nwf > kNoAllocMaxW)
    return fail(DGF_ERR_ARG, __LINE__,
                "dgf_fock_device_noalloc: " + std::to_string(c->nwf) + " working functions exceed its fixed scratch (" +
                    std::to_string(kNoAllocMaxW) + " at most); use dgf_fock_device");
  if (c->plan.empty() || c->plan_thrs != thrs)
    return fail(DGF_ERR_ARG, __LINE__,
                "dgf_fock_device_noalloc: no quartet plan for this threshold yet (building one needs device "
                "memory); make one dgf_fock or dgf_fock_device call with the same thrs first");
  if (c->device < 0 || c->device >= kMaxDevices)
    return fail(DGF_ERR_ARG, __LINE__, "device index beyond the no-allocation set-up table");
  DeviceGuard g(c->device);
  double *scratch = nullptr;
  cudaError_t e = scratch_address(c->device, &scratch);
  if (e != cudaSuccess) return fail(DGF_ERR_CUDA, __LINE__, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  cudaStream_t st = (cudaStream_t)stream;
  const int N = c->nwf;
  const size_t n2 = (size_t)N * N;
  double *D = scratch, *Ds = scratch + n2, *Fh = scratch + 2 * n2;
  const WorkMaps maps = ctx_maps(c);
  launch_work_prep(maps, dmat_device, D, Ds, 2, (int64_t)n2, c->nsm, st);
  e = cudaMemsetAsync(Fh, 0, n2 * sizeof(double), st);  // the accumulator starts at zero on every call
  if (e != cudaSuccess) return fail(DGF_ERR_CUDA, __LINE__, std::string("memset: ") + cudaGetErrorString(e));
  JKArgs a;
  memset(&a, 0, sizeof(a));
  a.pp = c->d_pp;
  a.sph = c->d_sph;
  a.spherical = c->spherical;
  a.nbf = N;
  a.nshell = c->nwshell;
  a.slot_stride = (int64_t)n2;
  a.nslot = 1;
  a.D = D;
  a.Ds = Ds;
  a.Fh = Fh;
  a.jscale[0] = 1.0;
  a.kscale[0] = 0.5 * hfxfac;
  a.schwarz_thr = thrs;
  for (const ClassPlan &cp : c->plan) {
    a.bra = c->d_pairs + c->cls_off[cp.X];
    a.ket = c->d_pairs + c->cls_off[cp.Y] + cp.kb0;
    a.ket_off = cp.kb0;
    a.ket_pp0 = (cp.bucket == 0 && cp.kb1 > cp.kb0) ? c->pairs[c->cls_off[cp.Y] + cp.kb0].pp0 : -1;
    a.nbra = c->cls_off[cp.X + 1] - c->cls_off[cp.X];
    a.same_class = (cp.X == cp.Y);
    a.qoff = c->d_qoff + cp.off;
    a.q_begin = 0;
    a.nquartet = cp.nquartet;
    const int la = (cp.X == 0) ? 0 : (cp.X <= 2) ? 1 : (cp.X <= 5) ? 2 : 3;
    const int lb = cp.X - la * (la + 1) / 2;
    const int lc = (cp.Y == 0) ? 0 : (cp.Y <= 2) ? 1 : (cp.Y <= 5) ? 2 : 3;
    const int ld = cp.Y - lc * (lc + 1) / 2;
    a.boys = c->d_boys + (size_t)(la + lb + lc + ld) * kBoysTableDoubles;
    if (cp.nquartet <= 0) continue;
    const bool bra1 = c->cls_max_npp[cp.X] == 1;
    const ClassKernel *k = &jk_kernel_variant(cp.X, cp.Y, 0, c->choice[cp.X][cp.Y][0], cp.bucket == 0, bra1);
    if (!k->launch) k = &jk_kernel(cp.X, cp.Y, 0, cp.bucket == 0, bra1);
    if (!k->launch) return fail(DGF_ERR_UNSUPPORTED, __LINE__, "no kernel for this quartet class");
    const int64_t per_block = k->qpb;
    const int grid =
        (int)std::max<int64_t>(1, std::min<int64_t>((cp.nquartet + per_block - 1) / per_block, (int64_t)c->nsm * 16));
    k->launch(a, grid, k->block, k->smem, st);
  }
  launch_work_combine(maps, Fh, Fh, fmat_device, 1.0, (int64_t)c->nbf * c->nbf, c->nsm, st);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(DGF_ERR_CUDA, __LINE__, std::string("launch: ") + cudaGetErrorString(e));
  return DGF_OK;
}
