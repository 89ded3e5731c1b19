// Batched Fock builds (pattern 2): many molecules of uneven size evaluated
// by one launch per quartet class over a merged, class-sorted quartet queue,
// the launches spread over forked streams (so that their tails overlap) and
// the whole sequence captured once as a CUDA graph and replayed.  The mixed
// form splits the classes the tuned context splits into FP64 and FP32
// launches, with per-shell-pair density bounds of every molecule.
//
// Every molecule keeps its own canonical quartet list (no cross-molecule
// quartets): the merged pair list of a class is the concatenation of the
// molecules' lists in their contexts' order (primitive-count bucket, Schwarz
// bin, shells), the plan has one entry per (class pair, ket bucket) over
// every molecule's bras, each pair record carries its molecule's
// offset and size in the packed working-basis D/F storage, and the plan
// stores, per bra pair, the first ket of its molecule in the merged ket
// list.  The packed AO-basis matrices of the caller are mapped to and from
// the packed working-basis ones by one transform launch each.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "dgf_ctx.h"
#include "dgf_md.cuh"

using namespace dgf;

struct BatchPlan {
  int X, Y;
  int bucket;        // primitive-count bucket of the kets (0: one primitive pair each)
  int64_t off;       // into the qoff buffer (nbra+1 entries)
  int64_t koff;      // into the kbase buffer (nbra entries)
  int64_t nquartet;
};

struct dgf_batch {
  int device = 0, nmol = 0, spherical = 1, nsm = 148;
  std::vector<int64_t> offsets;   // nmol+1 packed AO-matrix offsets (the caller's layout)
  std::vector<int64_t> woffsets;  // nmol+1 packed working-matrix offsets
  std::vector<int> nbf, nwf;
  int64_t total = 0, total_w = 0;
  std::vector<PairRec> pairs;
  int cls_off[kNumPairClass + 1] = {0};
  std::vector<int> mol_cls_off;  // [X * nmol + m]: start of molecule m's class-X pairs in the merged list
  std::vector<int> mol_bkt;      // [(X * nmol + m) * (kNumBuckets + 1) + k]: bucket starts inside that list
  PairRec *d_pairs = nullptr;
  PrimPair *d_pp = nullptr;
  double *d_boys = nullptr, *d_sph = nullptr;
  int64_t *d_offsets = nullptr;  // AO offsets | working offsets
  int *d_dims = nullptr;          // nwf | nbf | working base | AO base, nmol each
  int *d_wmap_i = nullptr;
  double *d_wmap_c = nullptr;
  WorkMaps maps;
  double *d_D = nullptr, *d_Ds = nullptr, *d_Fh = nullptr;
  unsigned long long *d_cnt = nullptr;
  double plan_thrs = -1.0;
  std::vector<BatchPlan> plan;
  int64_t *d_qoff = nullptr;
  int *d_kbase = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  const double *g_in = nullptr;
  double *g_out = nullptr;
  double g_thrs = -1.0, g_hfx = 0.0, g_mixed = 0.0;
  cudaStream_t g_stream = nullptr;
  int64_t launches = 0;
  int choice[kNumPairClass][kNumPairClass] = {};  // FP64 kernel per class pair (from the largest context)
  int choice32[kNumPairClass][kNumPairClass] = {};  // FP32 kernel per class pair (mixed form)
  int split_ok[kNumPairClass][kNumPairClass] = {};  // mixed form: split the class into FP64 + FP32 launches
  int cls_max_npp[kNumPairClass] = {};             // most primitive pairs of any pair of the class
  // mixed form: working shells of all molecules (first function | count),
  // per molecule {shell offset, shells, working functions} and the prefix
  // sums of shells^2, and the shell-pair maxima of |D| in the packed
  // working-matrix layout (allocated on the first mixed call)
  int *d_bsh = nullptr, *d_bmol = nullptr;
  int64_t *d_bpref = nullptr;
  int64_t nshpair = 0;
  int nshell_all = 0;
  float *d_dmw = nullptr;
  // The class launches are spread over kBatchStreams streams forked from
  // the caller's (or the capture) stream and joined back before the
  // epilogue, so that the tail of one launch overlaps the next ones.
  static constexpr int kBatchStreams = 4;
  cudaStream_t aux[kBatchStreams] = {};
  cudaEvent_t ev_fork = nullptr, ev_join[kBatchStreams] = {};
};

static void batch_free(dgf_batch *b) {
  if (!b) return;
  DeviceGuard g(b->device);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  void *ptrs[] = {b->d_pairs, b->d_pp,  b->d_boys, b->d_sph,  b->d_offsets, b->d_dims,  b->d_wmap_i,
                  b->d_wmap_c, b->d_D,   b->d_Ds,   b->d_Fh,   b->d_cnt,     b->d_qoff,  b->d_kbase,
                  b->d_bsh,    b->d_bmol, b->d_bpref, b->d_dmw};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (b->stream) cudaStreamDestroy(b->stream);
  for (int k = 0; k < dgf_batch::kBatchStreams; ++k) {
    if (b->aux[k]) cudaStreamDestroy(b->aux[k]);
    if (b->ev_join[k]) cudaEventDestroy(b->ev_join[k]);
  }
  if (b->ev_fork) cudaEventDestroy(b->ev_fork);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  delete b;
}

#define BFAIL(code, msg)                       \
  do {                                         \
    ::dgf::set_error(__FILE__, __LINE__, msg); \
    return code;                               \
  } while (0)

extern "C" void dgf_batch_destroy(dgf_batch *b) { batch_free(b); }

extern "C" int dgf_batch_create(dgf_ctx *const *ctxs, dgf_int nmol, dgf_batch **out) {
  if (!out) BFAIL(DGF_ERR_ARG, "out is NULL");
  *out = nullptr;
  if (!ctxs || nmol <= 0) BFAIL(DGF_ERR_ARG, "empty batch");
  for (dgf_int m = 0; m < nmol; ++m)
    if (!ctxs[m]) BFAIL(DGF_ERR_ARG, "NULL context in batch");
  const int dev = ctxs[0]->device, sph = ctxs[0]->spherical;
  for (dgf_int m = 0; m < nmol; ++m)
    if (ctxs[m]->device != dev || ctxs[m]->spherical != sph)
      BFAIL(DGF_ERR_ARG, "batch contexts must share device and spherical flag");
  dgf_batch *b = new dgf_batch;
  b->device = dev;
  b->nmol = (int)nmol;
  b->spherical = sph;
  b->nsm = ctxs[0]->nsm;
  DeviceGuard g(dev);
  b->offsets.assign(nmol + 1, 0);
  b->woffsets.assign(nmol + 1, 0);
  for (dgf_int m = 0; m < nmol; ++m) {
    b->nbf.push_back(ctxs[m]->nbf);
    b->nwf.push_back(ctxs[m]->nwf);
    b->offsets[m + 1] = b->offsets[m] + (int64_t)ctxs[m]->nbf * ctxs[m]->nbf;
    b->woffsets[m + 1] = b->woffsets[m] + (int64_t)ctxs[m]->nwf * ctxs[m]->nwf;
  }
  b->total = b->offsets[nmol];
  b->total_w = b->woffsets[nmol];
  dgf_int big = 0;
  for (dgf_int m = 1; m < nmol; ++m)
    if (ctxs[m]->nbf > ctxs[big]->nbf) big = m;
  for (int X = 0; X < kNumPairClass; ++X)
    for (int Y = 0; Y < kNumPairClass; ++Y) {
      b->choice[X][Y] = ctxs[big]->choice[X][Y][0];
      b->choice32[X][Y] = ctxs[big]->choice[X][Y][1];
      b->split_ok[X][Y] = ctxs[big]->split_ok[X][Y];
    }
  // Concatenated AO <-> working maps (offsets made global, indices stay local).
  std::vector<int> wr_off{0}, wr_idx, ac_off{0}, ac_idx, wbase, abase;
  std::vector<double> wr_c, ac_c;
  for (dgf_int m = 0; m < nmol; ++m) {
    const WorkMapHost &wm = ctxs[m]->wmap;
    wbase.push_back((int)wr_off.size() - 1);
    abase.push_back((int)ac_off.size() - 1);
    const int r0 = (int)wr_idx.size(), c0 = (int)ac_idx.size();
    for (int p = 0; p < ctxs[m]->nwf; ++p) wr_off.push_back(r0 + wm.wr_off[p + 1]);
    for (int mu = 0; mu < ctxs[m]->nbf; ++mu) ac_off.push_back(c0 + wm.ac_off[mu + 1]);
    wr_idx.insert(wr_idx.end(), wm.wr_idx.begin(), wm.wr_idx.end());
    wr_c.insert(wr_c.end(), wm.wr_c.begin(), wm.wr_c.end());
    ac_idx.insert(ac_idx.end(), wm.ac_idx.begin(), wm.ac_idx.end());
    ac_c.insert(ac_c.end(), wm.ac_c.begin(), wm.ac_c.end());
  }
  std::vector<int> ints(wr_off);
  ints.insert(ints.end(), wr_idx.begin(), wr_idx.end());
  ints.insert(ints.end(), ac_off.begin(), ac_off.end());
  ints.insert(ints.end(), ac_idx.begin(), ac_idx.end());
  std::vector<double> cs(wr_c);
  cs.insert(cs.end(), ac_c.begin(), ac_c.end());
  std::vector<int> dims(b->nwf);
  dims.insert(dims.end(), b->nbf.begin(), b->nbf.end());
  dims.insert(dims.end(), wbase.begin(), wbase.end());
  dims.insert(dims.end(), abase.begin(), abase.end());
  std::vector<int64_t> offs(b->offsets);
  offs.insert(offs.end(), b->woffsets.begin(), b->woffsets.end());
  size_t npp_all = 0;
  for (dgf_int m = 0; m < nmol; ++m) npp_all += ctxs[m]->pp.size();
  if (npp_all > (size_t)0x7fffffff) {
    batch_free(b);
    BFAIL(DGF_ERR_UNSUPPORTED, "batch too large (primitive pairs exceed 2^31)");
  }
  std::vector<PrimPair> pp;  // in the order of the merged pair list
  pp.reserve(npp_all);
  b->mol_cls_off.assign((size_t)kNumPairClass * nmol, 0);
  b->mol_bkt.assign((size_t)kNumPairClass * nmol * (kNumBuckets + 1), 0);
  for (int X = 0; X < kNumPairClass; ++X) {
    b->cls_off[X] = (int)b->pairs.size();
    for (dgf_int m = 0; m < nmol; ++m) {
      const dgf_ctx *c = ctxs[m];
      b->mol_cls_off[(size_t)X * nmol + m] = (int)b->pairs.size();
      // The molecule's class list in its context's order: primitive-count
      // bucket, Schwarz bin, shells (a bra's partners in one bucket are a
      // prefix of whole bins).
      for (int k = 0; k <= kNumBuckets; ++k) b->mol_bkt[((size_t)X * nmol + m) * (kNumBuckets + 1) + k] = c->bkt_off[X][k];
      std::vector<PairRec> lst(c->pairs.begin() + c->cls_off[X], c->pairs.begin() + c->cls_off[X + 1]);
      for (const PairRec &src : lst) {
        PairRec r = src;
        r.pp0 = (int)pp.size();
        pp.insert(pp.end(), c->pp.begin() + src.pp0, c->pp.begin() + src.pp0 + src.npp);
        r.nbfm = c->nwf;
        r.dbase = b->woffsets[m];
        b->pairs.push_back(r);
      }
    }
  }
  b->cls_off[kNumPairClass] = (int)b->pairs.size();
  std::vector<int> bsh, bmol;
  std::vector<int64_t> bpref{0};
  {
    std::vector<int> nf;
    for (dgf_int m = 0; m < nmol; ++m) {
      const dgf_ctx *c = ctxs[m];
      bmol.push_back((int)(bsh.size()));
      bmol.push_back(c->nwshell);
      bmol.push_back(c->nwf);
      bsh.insert(bsh.end(), c->ws_ao.begin(), c->ws_ao.end());
      for (int k = 0; k < c->nwshell; ++k) nf.push_back(nfun(c->ws_l[k], c->spherical));
      bpref.push_back(bpref.back() + (int64_t)c->nwshell * c->nwshell);
    }
    bsh.insert(bsh.end(), nf.begin(), nf.end());  // first functions, then counts
  }
  b->nshpair = bpref.back();
  b->nshell_all = (int)(bsh.size() / 2);
  for (int X = 0; X < kNumPairClass; ++X)
    for (int i = b->cls_off[X]; i < b->cls_off[X + 1]; ++i) b->cls_max_npp[X] = std::max(b->cls_max_npp[X], b->pairs[i].npp);
  const size_t n_boys = kBoysAllDoubles;  // full-degree and low-degree (FP32 half) tables
  cudaError_t e = cudaSuccess;
  auto alloc = [&](void **p, size_t bytes) {
    if (e == cudaSuccess) e = cudaMalloc(p, std::max<size_t>(bytes, 8));
  };
  alloc((void **)&b->d_pairs, b->pairs.size() * sizeof(PairRec));
  alloc((void **)&b->d_pp, pp.size() * sizeof(PrimPair));
  alloc((void **)&b->d_boys, n_boys * 8);
  alloc((void **)&b->d_sph, kSphTableDoubles * 8);
  alloc((void **)&b->d_offsets, offs.size() * 8);
  alloc((void **)&b->d_dims, dims.size() * 4);
  alloc((void **)&b->d_wmap_i, ints.size() * 4);
  alloc((void **)&b->d_wmap_c, cs.size() * 8);
  alloc((void **)&b->d_D, b->total_w * 8);
  alloc((void **)&b->d_Ds, b->total_w * 8);
  alloc((void **)&b->d_Fh, b->total_w * 8);
  alloc((void **)&b->d_cnt, 4 * kCounterSlots * 8);
  alloc((void **)&b->d_bsh, bsh.size() * 4);
  alloc((void **)&b->d_bmol, bmol.size() * 4);
  alloc((void **)&b->d_bpref, bpref.size() * 8);
  if (e != cudaSuccess) {
    cudaGetLastError();
    batch_free(b);
    BFAIL(DGF_ERR_NOMEM, "device allocation for the batch failed");
  }
  e = cudaMemcpy(b->d_pairs, b->pairs.data(), b->pairs.size() * sizeof(PairRec), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->d_pp, pp.data(), pp.size() * sizeof(PrimPair), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->d_boys, ctxs[0]->d_boys, n_boys * 8, cudaMemcpyDeviceToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->d_sph, ctxs[0]->d_sph, kSphTableDoubles * 8, cudaMemcpyDeviceToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->d_offsets, offs.data(), offs.size() * 8, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->d_dims, dims.data(), dims.size() * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->d_wmap_i, ints.data(), ints.size() * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !cs.empty()) e = cudaMemcpy(b->d_wmap_c, cs.data(), cs.size() * 8, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->d_bsh, bsh.data(), bsh.size() * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->d_bmol, bmol.data(), bmol.size() * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->d_bpref, bpref.data(), bpref.size() * 8, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  for (int k = 0; k < dgf_batch::kBatchStreams; ++k) {
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->aux[k], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_join[k], cudaEventDisableTiming);
  }
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreate(&b->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&b->ev1);
  if (e != cudaSuccess) {
    std::string msg = cudaGetErrorString(e);
    batch_free(b);
    BFAIL(DGF_ERR_CUDA, msg);
  }
  WorkMaps &mp = b->maps;
  const int nm = (int)nmol;
  const size_t nr = wr_idx.size();
  mp.nmol = nm;
  mp.a_elem = b->d_offsets;
  mp.w_elem = b->d_offsets + (nm + 1);
  mp.nw = b->d_dims;
  mp.na = b->d_dims + nm;
  mp.wf_base = b->d_dims + 2 * nm;
  mp.af_base = b->d_dims + 3 * nm;
  mp.wr_off = b->d_wmap_i;
  mp.wr_idx = b->d_wmap_i + wr_off.size();
  mp.ac_off = b->d_wmap_i + wr_off.size() + nr;
  mp.ac_idx = b->d_wmap_i + wr_off.size() + nr + ac_off.size();
  mp.wr_c = b->d_wmap_c;
  mp.ac_c = b->d_wmap_c + nr;
  *out = b;
  return DGF_OK;
}

extern "C" int dgf_batch_layout(const dgf_batch *b, dgf_int *offsets) {
  if (!b || !offsets) BFAIL(DGF_ERR_ARG, "NULL argument");
  for (int m = 0; m <= b->nmol; ++m) offsets[m] = b->offsets[m];
  return DGF_OK;
}

// Per-molecule quartet queues, merged per class pair.
static int batch_plan(dgf_batch *b, double thrs) {
  if (b->plan_thrs == thrs && !b->plan.empty()) return DGF_OK;
  std::vector<int64_t> qoff;
  std::vector<int> kbase;
  std::vector<BatchPlan> plan;
  const int nm = b->nmol;
  auto mol_end = [&](int X, int m) {
    return (m + 1 < nm) ? b->mol_cls_off[(size_t)X * nm + m + 1] : b->cls_off[X + 1];
  };
  for (int X = 0; X < kNumPairClass; ++X)
    for (int Y = 0; Y <= X; ++Y)
      for (int kb = 0; kb < kNumBuckets; ++kb) {
        const int nb = b->cls_off[X + 1] - b->cls_off[X];
        const int nk = b->cls_off[Y + 1] - b->cls_off[Y];
        if (!nb || !nk) continue;
        BatchPlan bp;
        bp.X = X;
        bp.Y = Y;
        bp.bucket = kb;
        bp.off = (int64_t)qoff.size();
        bp.koff = (int64_t)kbase.size();
        int64_t acc = 0;
        qoff.push_back(0);
        for (int m = 0; m < nm; ++m) {
          const int b0 = b->mol_cls_off[(size_t)X * nm + m], b1 = mol_end(X, m);
          const int ky = b->mol_cls_off[(size_t)Y * nm + m];  // molecule's class-Y list start
          const int *bk = &b->mol_bkt[((size_t)Y * nm + m) * (kNumBuckets + 1)];
          const int k0 = ky + bk[kb], k1 = ky + bk[kb + 1];
          for (int i = b0; i < b1; ++i) {
            const double qb = b->pairs[i].Q;
            int lo = k0, hi = k1;  // first ket whose whole Schwarz bin has qb*Q < thrs
            while (lo < hi) {
              const int mid = (lo + hi) >> 1;
              if (qb * q_bin_upper(q_bin(b->pairs[mid].Q)) >= thrs)
                lo = mid + 1;
              else
                hi = mid;
            }
            int n = lo - k0;
            // X == Y: ket position <= bra position inside the molecule's class list
            if (X == Y) n = std::max(0, std::min(n, (i - b0) - bk[kb] + 1));
            acc += n;
            qoff.push_back(acc);
            kbase.push_back(k0 - b->cls_off[Y]);
          }
        }
        bp.nquartet = acc;
        if (acc > 0)
          plan.push_back(bp);
        else {
          qoff.resize(bp.off);
          kbase.resize(bp.koff);
        }
      }
  if (b->d_qoff) cudaFree(b->d_qoff);
  if (b->d_kbase) cudaFree(b->d_kbase);
  b->d_qoff = nullptr;
  b->d_kbase = nullptr;
  if (cudaMalloc(&b->d_qoff, std::max<size_t>(qoff.size(), 1) * 8) != cudaSuccess ||
      cudaMalloc(&b->d_kbase, std::max<size_t>(kbase.size(), 1) * 4) != cudaSuccess) {
    cudaGetLastError();
    BFAIL(DGF_ERR_NOMEM, "device allocation of the batch plan failed");
  }
  if (cudaMemcpy(b->d_qoff, qoff.data(), qoff.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
      (kbase.size() && cudaMemcpy(b->d_kbase, kbase.data(), kbase.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess))
    BFAIL(DGF_ERR_CUDA, "upload of the batch plan failed");
  b->plan.swap(plan);
  b->plan_thrs = thrs;
  if (b->exec) {  // a captured graph refers to the old plan
    cudaGraphExecDestroy(b->exec);
    cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
  }
  return DGF_OK;
}

// Mixed form of a batch: max |D| over the working functions of every shell
// pair of every molecule (both orientations), rounded up to FP32 and stored
// at (first function of A, first function of B) of the molecule's block of
// the packed working matrix.  e runs over the molecules' shell pairs;
// pref holds the prefix sums of shells^2, mol {shell offset, shells,
// functions} per molecule, sh the shells' first functions then counts.
__global__ void batch_dmax_kernel(const double *__restrict__ D, const int64_t *__restrict__ woff,
                                  const int64_t *__restrict__ pref, const int *__restrict__ mol,
                                  const int *__restrict__ sh, int nshell_all, int nmol, int64_t npair,
                                  float *__restrict__ dm) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < npair; e += (int64_t)gridDim.x * blockDim.x) {
    int lo = 0, hi = nmol - 1;  // the molecule: last m with pref[m] <= e
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (pref[mid] <= e) lo = mid; else hi = mid - 1;
    }
    const int m = lo, s0 = mol[3 * m], ns = mol[3 * m + 1], n = mol[3 * m + 2];
    const int64_t local = e - pref[m];
    const int A = s0 + (int)(local / ns), B = s0 + (int)(local % ns);
    const int pa = sh[A], na = sh[nshell_all + A], pb = sh[B], nb = sh[nshell_all + B];
    const double *Dm = D + woff[m];
    double v = 0.0;
    for (int i = 0; i < na; ++i)
      for (int j = 0; j < nb; ++j) {
        const int p = pa + i, q = pb + j;
        v = fmax(v, fmax(fabs(Dm[(size_t)p * n + q]), fabs(Dm[(size_t)q * n + p])));
      }
    dm[woff[m] + (int64_t)pa * n + pb] = __double2float_ru(v);
  }
}

// la + lb of pair class X (classes ordered (s,s), (p,s), (p,p), (d,s), ...).
static int pair_class_l(int X) {
  const int la = (X == 0) ? 0 : (X <= 2) ? 1 : (X <= 5) ? 2 : 3;
  return la + (X - la * (la + 1) / 2);
}

static int batch_enqueue(dgf_batch *b, const double *din, double *fout, double hfx, double mixed_cutoff,
                         cudaStream_t st) {
  int64_t launches = 0;
  launch_work_prep(b->maps, din, b->d_D, b->d_Ds, 2, b->total_w, b->nsm, st);  // symmetric part, IFCTYP 13
  ++launches;
  const bool mixed = mixed_cutoff > 0.0;
  if (mixed) {
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(b->nshpair / 128 + 1, (int64_t)b->nsm * 8));
    batch_dmax_kernel<<<grid, 128, 0, st>>>(b->d_D, b->d_offsets + b->nmol + 1, b->d_bpref, b->d_bmol, b->d_bsh,
                                             b->nshell_all, b->nmol, b->nshpair, b->d_dmw);
    ++launches;
  }
  if (cudaMemsetAsync(b->d_Fh, 0, b->total_w * 8, st) != cudaSuccess) BFAIL(DGF_ERR_CUDA, "memset failed");
  JKArgs a;
  memset(&a, 0, sizeof(a));
  a.pp = b->d_pp;
  a.sph = b->d_sph;
  a.spherical = b->spherical;
  a.nslot = 1;
  a.slot_stride = b->total_w;
  a.D = b->d_D;
  a.Ds = b->d_Ds;
  a.Fh = b->d_Fh;
  a.jscale[0] = 1.0;
  a.kscale[0] = 0.5 * hfx;
  a.schwarz_thr = b->plan_thrs;  // the plan's last Schwarz bin may reach below the threshold
  a.ket_pp0 = -1;                 // a molecule's kets are not adjacent to the next molecule's
  a.dmax_w = mixed ? b->d_dmw : nullptr;
  a.split = mixed_cutoff;
  // Longest-first assignment of the plan entries to the forked streams by
  // model cost (quartets x a per-class weight).
  const int ns = dgf_batch::kBatchStreams;
  std::vector<int> order(b->plan.size()), stream_of(b->plan.size(), 0);
  std::vector<double> cost(b->plan.size());
  for (size_t i = 0; i < b->plan.size(); ++i) {
    const BatchPlan &bp = b->plan[i];
    const int L = pair_class_l(bp.X) + pair_class_l(bp.Y);
    cost[i] = (double)bp.nquartet * (double)n3(L) * (double)(1 << std::min(bp.bucket, 6));
    order[i] = (int)i;
  }
  std::stable_sort(order.begin(), order.end(), [&](int u, int v) { return cost[u] > cost[v]; });
  {
    double load[dgf_batch::kBatchStreams] = {};
    for (int i : order) {
      int k = 0;
      for (int t = 1; t < ns; ++t)
        if (load[t] < load[k]) k = t;
      stream_of[i] = k;
      load[k] += cost[i];
    }
  }
  if (cudaEventRecord(b->ev_fork, st) != cudaSuccess) BFAIL(DGF_ERR_CUDA, "event record failed");
  for (int k = 0; k < ns; ++k)
    if (cudaStreamWaitEvent(b->aux[k], b->ev_fork, 0) != cudaSuccess) BFAIL(DGF_ERR_CUDA, "stream fork failed");
  int slot = 0;
  for (int i : order) {
    const BatchPlan &bp = b->plan[i];
    cudaStream_t ls = b->aux[stream_of[i]];
    a.bra = b->d_pairs + b->cls_off[bp.X];
    a.ket = b->d_pairs + b->cls_off[bp.Y];
    a.ket_off = 0;
    a.nbra = b->cls_off[bp.X + 1] - b->cls_off[bp.X];
    a.same_class = (bp.X == bp.Y);
    a.qoff = b->d_qoff + bp.off;
    a.kbase = b->d_kbase + bp.koff;
    a.q_begin = 0;
    a.nquartet = bp.nquartet;
    const int Lq = pair_class_l(bp.X) + pair_class_l(bp.Y);
    const bool bra1 = b->cls_max_npp[bp.X] == 1;
    const ClassKernel *kp = &jk_kernel_variant(bp.X, bp.Y, 0, b->choice[bp.X][bp.Y], bp.bucket == 0, bra1);
    if (!kp->launch) kp = &jk_kernel(bp.X, bp.Y, 0, bp.bucket == 0, bra1);
    // Mixed form: the classes the tuned context splits run an FP64 launch
    // for quartets whose bound is at or above the cutoff and an FP32 launch
    // for the rest.
    const ClassKernel *k32 = nullptr;
    if (mixed && b->split_ok[bp.X][bp.Y]) {
      k32 = &jk_kernel_variant(bp.X, bp.Y, 1, b->choice32[bp.X][bp.Y], bp.bucket == 0, bra1);
      if (!k32->launch) k32 = &jk_kernel(bp.X, bp.Y, 1, bp.bucket == 0, bra1);
      if (!k32->launch) k32 = nullptr;
    }
    for (int part = 0; part < (k32 ? 2 : 1); ++part) {
      const ClassKernel &k = part ? *k32 : *kp;
      a.mode = k32 ? 1 + part : 0;
      a.boys = b->d_boys + (part ? boys_low_offset(Lq) : (size_t)Lq * kBoysTableDoubles);
      a.counters = b->d_cnt + 4 * (slot++ % kCounterSlots);
      const int64_t per_block = k.qpb;
      const int grid = (int)std::max<int64_t>(
          1, std::min<int64_t>((bp.nquartet + per_block - 1) / per_block, (int64_t)b->nsm * 16));
      k.launch(a, grid, k.block, k.smem, ls);
      ++launches;
    }
  }
  for (int k = 0; k < ns; ++k) {
    if (cudaEventRecord(b->ev_join[k], b->aux[k]) != cudaSuccess || cudaStreamWaitEvent(st, b->ev_join[k], 0) != cudaSuccess)
      BFAIL(DGF_ERR_CUDA, "stream join failed");
  }
  launch_work_combine(b->maps, b->d_Fh, b->d_Fh, fout, 1.0, b->total, b->nsm, st);  // F = C^T (Fh + Fh^T) C
  ++launches;
  if (cudaGetLastError() != cudaSuccess) BFAIL(DGF_ERR_CUDA, "launch failed in the batched build");
  b->launches = launches;
  return DGF_OK;
}

extern "C" int dgf_fock_batch(dgf_batch *b, const double *dmat_packed_device, double *fmat_packed_device,
                              const dgf_options *opt, int use_graph, void *stream, dgf_stats *stats) {
  if (!b || !dmat_packed_device || !fmat_packed_device) BFAIL(DGF_ERR_ARG, "NULL argument");
  DeviceGuard g(b->device);
  dgf_options o;
  dgf_default_options(&o);
  if (opt) o = *opt;
  if (o.ifthrs < 16 || o.shard_count > 1 || o.hfxmu != 0.0)
    BFAIL(DGF_ERR_UNSUPPORTED, "batched builds take the Schwarz-screened form without range separation only");
  if (!(o.mixed_cutoff >= 0.0)) BFAIL(DGF_ERR_ARG, "mixed_cutoff must be >= 0");
  if (o.mixed_cutoff > 0.0 && !b->d_dmw) {
    if (cudaMalloc(&b->d_dmw, std::max<int64_t>(b->total_w, 1) * sizeof(float)) != cudaSuccess) {
      cudaGetLastError();
      b->d_dmw = nullptr;
      BFAIL(DGF_ERR_NOMEM, "device allocation of the batch density bounds failed");
    }
  }
  cudaStream_t st = (cudaStream_t)stream;  // NULL: the legacy default stream, as in dgf_fock_device
  int r = batch_plan(b, o.thrs);
  if (r) return r;
  if (cudaMemsetAsync(b->d_cnt, 0, 4 * kCounterSlots * 8, st) != cudaSuccess) BFAIL(DGF_ERR_CUDA, "memset failed");
  if (cudaEventRecord(b->ev0, st) != cudaSuccess) BFAIL(DGF_ERR_CUDA, "event record failed");
  if (use_graph) {
    const bool stale = !b->exec || b->g_in != dmat_packed_device || b->g_out != fmat_packed_device ||
                       b->g_thrs != o.thrs || b->g_hfx != o.hfxfac || b->g_mixed != o.mixed_cutoff ||
                       b->g_stream != st;
    if (stale) {
      if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        cudaGraphDestroy(b->graph);
        b->exec = nullptr;
        b->graph = nullptr;
      }
      // capture on the batch's own stream, replay on st (the counters are reset outside the graph)
      cudaStream_t cs = b->stream;
      if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        BFAIL(DGF_ERR_CUDA, "stream capture failed to begin");
      r = batch_enqueue(b, dmat_packed_device, fmat_packed_device, o.hfxfac, o.mixed_cutoff, cs);
      cudaGraph_t gr = nullptr;
      cudaError_t e = cudaStreamEndCapture(cs, &gr);
      if (r) {
        if (gr) cudaGraphDestroy(gr);
        return r;
      }
      if (e != cudaSuccess) BFAIL(DGF_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
      e = cudaGraphInstantiate(&b->exec, gr, 0);
      if (e != cudaSuccess) {
        cudaGraphDestroy(gr);
        BFAIL(DGF_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
      }
      b->graph = gr;
      b->g_in = dmat_packed_device;
      b->g_out = fmat_packed_device;
      b->g_thrs = o.thrs;
      b->g_hfx = o.hfxfac;
      b->g_mixed = o.mixed_cutoff;
      b->g_stream = st;
    }
    if (cudaGraphLaunch(b->exec, st) != cudaSuccess) BFAIL(DGF_ERR_CUDA, "graph launch failed");
  } else {
    r = batch_enqueue(b, dmat_packed_device, fmat_packed_device, o.hfxfac, o.mixed_cutoff, st);
    if (r) return r;
  }
  if (cudaEventRecord(b->ev1, st) != cudaSuccess) BFAIL(DGF_ERR_CUDA, "event record failed");
  if (stats) {
    std::vector<unsigned long long> cnt(4 * kCounterSlots);
    if (cudaMemcpyAsync(cnt.data(), b->d_cnt, cnt.size() * 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      BFAIL(DGF_ERR_CUDA, "stats copy failed");
    unsigned long long s[4] = {0, 0, 0, 0};
    for (int i = 0; i < kCounterSlots; ++i)
      for (int k = 0; k < 4; ++k) s[k] += cnt[4 * i + k];
    const int64_t tq = (int64_t)(s[0] + s[2]);  // quartets that passed Schwarz
    float ms = 0.f;
    cudaEventElapsedTime(&ms, b->ev0, b->ev1);
    stats->quartets_total = tq;
    stats->quartets_fp64 = (int64_t)(s[0] - s[3]);
    stats->quartets_fp32 = (int64_t)s[3];
    stats->quartets_skipped = 0;
    stats->prim_quartets = (int64_t)s[1];
    stats->kernel_launches = b->launches;
    stats->ms_device = ms;
  }
  return DGF_OK;
}
