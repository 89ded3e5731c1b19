/* dgfock — B200-native direct J/K Fock build, C ABI.
 *
 * Drop-in for the two-electron Fock call of Dalton's SCF:
 *   SUBROUTINE HERFCK(FMAT,DMAT,NDMT,ISYMDM,IFCTYP,IPRFCK,WORK,LWORK)
 *   (DALTON/abacus/herdirect.F:431-551), reached from SIRFCK
 *   (DALTON/sirius/sirfck.F:387) and from FCK2AO (DALTON/sirius/sirgrad.F:714).
 *
 * Contract kept from HERFCK:
 *   - FMAT(N,N,NDMT) is overwritten (HERFCK_1 zeroes it, herdirect.F:686);
 *     DMAT(N,N,NDMT) is read only.  Matrices are full squares in Dalton's C1
 *     AO order; a symmetric matrix reads the same in C (row-major) and
 *     Fortran (column-major) order, and general ones are documented per call.
 *   - IFCTYP = 10*X + Y per matrix (sirfck.F:45-57): X = 1 symmetric,
 *     0 general, 2 antisymmetric density; Y = 1 Coulomb, 2 exchange, 3 both.
 *     F = [Y&1] J[D] - [Y&2] (hfxfac/2) K[D] with
 *       J_pq = sum_rs (pq|rs) D_rs,   K_pq = sum_rs (pr|qs) D_rs
 *     (FCKD03, sirfck.F:1496-1547; FCKCON, herfckcon.F:20-220).
 *   - Shell quartets with Q_AB*Q_CD < thrs are skipped (Schwarz, THRS
 *     default 1e-12, herrdn.F:359; her2gab.F GABGEN); with ifthrs < 16 also
 *     those with Q_AB*Q_CD*max(4|D|_Coulomb, |D|_exchange) < 10^-ifthrs
 *     (SYMLOP screening, her2drv.F:2663-2733).
 *   - Errors are returned as status codes (0 = success), never by aborting;
 *     the Fortran shim maps a nonzero status to QUIT (gptrygve.F:256).
 *
 * All pointers are host pointers unless a name says _device.  A context is
 * not thread-safe; separate contexts are independent.
 */
#ifndef DGFOCK_H
#define DGFOCK_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Integer width of the ABI.  Dalton is built with 4-byte INTEGER unless
 * -DVAR_INT64 (cmake/Definitions.cmake:30); this library takes int64 and a
 * 4-byte-INTEGER Dalton widens its arrays in the shim. */
typedef int64_t dgf_int;

typedef struct dgf_ctx dgf_ctx;

/* Status codes. */
enum {
  DGF_OK = 0,
  DGF_ERR_ARG = 1,         /* invalid argument */
  DGF_ERR_NOMEM = 2,       /* device or host allocation failed */
  DGF_ERR_CUDA = 3,        /* CUDA runtime error */
  DGF_ERR_UNSUPPORTED = 4, /* angular momentum, IFCTYP or option not supported */
  DGF_ERR_TIMEOUT = 5,     /* a bounded device-side wait gave up */
  DGF_ERR_NODEVICE = 6     /* no CUDA device / extension unusable */
};

/* Basis in Dalton block form (one block = one atom's shell of angular
 * momentum l: nprim primitives shared by ncontr contracted functions, CPRIM
 * coefficients already normalised as NRMORB does, herrdn.F:3263-3290).
 * AO offsets follow Dalton's C1 order: atom -> l -> contraction -> component
 * (p as x,y,z; d and higher as real spherical m=-l..l when spherical=1,
 * SPHCOM MINTEG=2, her1pro.F:4671-4790; Cartesian xx,xy,xz,yy,yz,zz,...
 * otherwise).  This is what a Fortran shim gathers from /SHELLS/ and
 * /PRIMIT/. */
typedef struct {
  dgf_int nblock, natom, nbf, spherical;
  const dgf_int *block_l, *block_atom, *block_nprim, *block_ncontr;
  const dgf_int *block_ao_offset, *block_prim_offset, *block_coef_offset;
  const double *prim_exp;   /* concatenated exponents */
  const double *coef;       /* per block, column-major (nprim, ncontr) */
  const double *atom_xyz;   /* (natom, 3) bohr */
  const double *atom_charge;/* (natom) nuclear charges */
} dgf_basis;

/* Work counters of one call (HERFCK's DINTSKP/SCRSTA statistics,
 * her2drv.F:495-541, her2gab.F:1486, in this library's units: shell quartets
 * of the two-electron working basis, in which general contractions are
 * resolved into primitives; dgf_count_ao_quartets gives the AO-basis count). */
typedef struct {
  int64_t quartets_total;    /* canonical shell quartets with Q_AB*Q_CD >= thrs */
  int64_t quartets_fp64;     /* evaluated in FP64 */
  int64_t quartets_fp32;     /* evaluated in FP32 (mixed form) */
  int64_t quartets_skipped;  /* skipped by density screening */
  int64_t prim_quartets;     /* primitive quartets evaluated */
  int64_t kernel_launches;   /* device kernels launched by the call */
  double ms_device;          /* device time of the Fock build (CUDA events) */
} dgf_stats;

/* Fock-build options (no globals; Dalton's COMMON values passed in).
 * thrs: Schwarz threshold (THRS, 1e-12 default);
 * ifthrs: density screening exponent (HR2INP .IFTHRS): on when ifthrs < 16
 *   as in Dalton's direct Fock build (values below 4 are taken as 14,
 *   DALTON/abacus/her2drv.F:520-540);
 * hfxfac: exchange factor (HFXFAC, 1 for HF);
 * mixed_cutoff: 0 = all-FP64 drop-in; > 0 = quartets whose bound
 *   Q_AB*Q_CD*Dmax is below it are evaluated in FP32 (Boys function,
 *   accumulation and digestion stay FP64). */
typedef struct {
  double thrs;
  dgf_int ifthrs;
  double hfxfac;
  double mixed_cutoff;
  /* Shard of the quartet queue this call evaluates: the class-sorted queue
   * (all classes in order) is cut into shard_count contiguous ranges of equal
   * model cost (a fixed FLOP model per class, the same on every rank) and
   * range shard_index is evaluated, as Dalton's parallel Fock build hands
   * cost-sorted shell-pair tasks to its workers (herpar.F:457,1165); F is
   * then the partial sum of that shard (sum the shards, e.g. with an NCCL
   * all-reduce, for the full matrix).  0 and 1 = everything. */
  dgf_int shard_index;
  dgf_int shard_count;
  /* ICEDIF (HR2INP .ICEDIF, DALTON/abacus/herdrv.F:2042-2044,2131): with
   * density screening on, bit 1 drops a quartet's Coulomb contribution of a
   * density when max|D| over its Coulomb blocks times the quartet's largest
   * integral is below 10^-ifthrs, bit 2 likewise its exchange contribution
   * (INTFC1, DALTON/abacus/her2fck.F:221-222,446-466).  Dalton's default is
   * 3.  The thread- and warp-per-quartet kernels apply it; quartets of the
   * cooperative kernels are always digested whole (the conservative side). */
  dgf_int icedif;
  /* Range-separated exchange of CAM-type functionals (Dalton's HFXMU and
   * HFXATT, set by dftsetcam, DALTON/dft/dft_aux.F:346-351): with hfxmu != 0
   * a second pass over the quartets adds -hfxatt/2 K[D] computed with the
   * attenuated operator erf(hfxmu r12)/r12, exchange only whatever the
   * Coulomb digit of IFCTYP (HERFCK_1, DALTON/abacus/herdirect.F:792-835;
   * FCKCON forces IY = 2, herfckcon.F:59-66; attenuated R^n_000,
   * her2her.F:344-353).  The Schwarz factors of 1/r12 bound the attenuated
   * integrals too (erf(mu r)/r <= 1/r, positive definite), so the same
   * quartet plan serves both passes.  hfxmu = 0: no second pass. */
  double hfxmu;
  double hfxatt;
} dgf_options;

/* Default options: thrs 1e-12, ifthrs 20, hfxfac 1, mixed_cutoff 0, one
 * shard, icedif 3, hfxmu 0, hfxatt 0. */
void dgf_default_options(dgf_options *opt);

/* Create a context on CUDA device `device`: copies the basis to the device,
 * builds the shell-pair records, Schwarz factors and class-sorted pair lists
 * (the GETGAB/GABGEN pre-pass, her2gab.F:1776-1928, once per geometry). */
int dgf_create(const dgf_basis *basis, int device, dgf_ctx **out);

/* Free a context (and all its device memory). NULL is ignored. */
void dgf_destroy(dgf_ctx *ctx);

/* HERFCK: F(N,N,ndmat) from D(N,N,ndmat), host pointers.  Replaces the
 * HERFCK_1 / ERIFCK dispatch (herdirect.F:514-553).  stats may be NULL. */
int dgf_fock(dgf_ctx *ctx, dgf_int ndmat, const dgf_int *ifctyp, const double *dmat, double *fmat,
             const dgf_options *opt, dgf_stats *stats);

/* Same with device pointers, enqueued on `stream` (a cudaStream_t, NULL for
 * the legacy default stream); no host synchronisation except what screening
 * set-up needs.  dmat_device/fmat_device hold ndmat N*N doubles. */
int dgf_fock_device(dgf_ctx *ctx, dgf_int ndmat, const dgf_int *ifctyp, const double *dmat_device,
                    double *fmat_device, const dgf_options *opt, void *stream, dgf_stats *stats);

/* Fock build that allocates no device memory.  No counterpart in Dalton:
 * an addition for callers that cannot allocate GPU memory when they need a
 * Fock matrix, such as a host that, like Dalton, gives the engine one fixed
 * work area and nothing more, or a process whose device memory is owned by
 * another pool.  Same result as dgf_fock_device with ndmat = 1, IFCTYP 13,
 * ifthrs >= 16, mixed_cutoff = 0: F = J[D] - hfxfac/2 K[D] of one density
 * (symmetrised), device pointers.  Its scratch is a fixed device array of
 * 3 x 1536 x 1536 doubles (56.6 MB: density, D + D^T and half Fock matrix of
 * the two-electron working basis, in which general contractions are resolved
 * into primitives) that every GPU loading this library holds until exit;
 * contexts with more than 768 basis functions, or more than 1536 working
 * functions, are rejected (DGF_ERR_ARG).  The context's quartet plan for `thrs` must exist already
 * (an earlier dgf_fock, dgf_fock_device, dgf_autotune or dgf_grad2e call
 * with this threshold builds it), else DGF_ERR_ARG.  The first call on a
 * device looks up the array's device address; make it before any CUDA
 * stream capture.  The address is kept for the life of the device's
 * context: after a cudaDeviceReset of that device do not call it again.  All calls share the array and leave its contents behind;
 * calls that overlap on the GPU (other streams or host threads) race and
 * must be serialised by the caller. */
int dgf_fock_device_noalloc(dgf_ctx *ctx, const double *dmat_device, double *fmat_device, double hfxfac,
                            double thrs, void *stream);

/* Two-electron part of the RHF nuclear gradient (TWOEXP -> INTEX1 -> DEROUT,
 * aba2tex.F:242, her2ave.F:91-830): grad(natom,3) is overwritten with
 *   1/2 sum_pqrs d(pq|rs)/dx [D_pq D_rs - hfxfac/2 D_pr D_qs],
 * D the symmetric total density (host pointers). */
int dgf_grad2e(dgf_ctx *ctx, const double *dmat, double hfxfac, double thrs, double *grad);

/* Device-pointer form of dgf_grad2e. */
int dgf_grad2e_device(dgf_ctx *ctx, const double *dmat_device, double hfxfac, double thrs, double *grad_device,
                      void *stream);

/* Bilinear form of the two-electron gradient, device pointers: grad = sum
 * over canonical quartets of d(ab|cd)/dx times the symmetrised product
 * 2 (D1_ab D2_cd + D2_ab D1_cd) - hfxfac/2 (D1_ac D2_bd + D2_ac D1_bd +
 * D1_ad D2_bc + D2_ad D1_bc) (weighted for coinciding shells).  With
 * D1 = D2 = D it equals dgf_grad2e; with D1 = C a symmetric cotangent of
 * G = F(D) it is half of d<C, G(D)>/dx (the backward pass of the build).
 * No counterpart in Dalton, which only forms the D1 = D2 case (INTEX1). */
int dgf_grad2e_bilinear_device(dgf_ctx *ctx, const double *d1_device, const double *d2_device, double hfxfac,
                               double thrs, double *grad_device, void *stream);

/* One-electron integrals S, T, V (N x N each, host pointers, any may be
 * NULL): the HER1 integrals the SCF host needs next to the Fock build. */
int dgf_oneint(dgf_ctx *ctx, double *S, double *T, double *V);

/* One-electron + nuclear-repulsion part of the RHF gradient:
 * sum D_pq dh_pq/dx - sum W_pq dS_pq/dx + dVnn/dx, grad(natom,3). */
int dgf_grad1e(dgf_ctx *ctx, const double *dmat, const double *wmat, double *grad);

/* Per-launch profile of the last Fock build (enabled by dgf_set_profiling):
 * one record per quartet-class kernel launch, timed with CUDA events on the
 * launching stream. */
typedef struct {
  int32_t la, lb, lc, ld;   /* angular momenta of the class (ab|cd) */
  int32_t precision;        /* 64 = FP64, 32 = FP32 contraction */
  int32_t kernel;           /* 0 = thread-per-quartet, 1 = cooperative team, 2 = warp teams,
                               4 = warp-per-quartet (L >= 4), 6 = warp-per-quartet with
                               FP64 tensor-core (DMMA) transforms,
                               5 = two-electron gradient (dgf_grad2e*: quartets are the plan's,
                               primitive quartets estimated from the classes' mean primitive
                               pairs) */
  int64_t quartets;         /* quartets of the class in the plan */
  int64_t evaluated;        /* quartets this launch evaluated */
  int64_t prim_quartets;    /* primitive quartets this launch evaluated */
  double ms;                /* device time of the launch */
} dgf_class_time;

/* Turn per-launch profiling of dgf_fock / dgf_fock_device and of the
 * two-electron gradient calls on (1) or off (0).  While on, each call
 * synchronises its stream at the end. */
int dgf_set_profiling(dgf_ctx *ctx, int on);

/* Copy up to `max` records of the last profiled call; *count = records. */
int dgf_get_profile(const dgf_ctx *ctx, dgf_class_time *out, int max, int *count);

/* Conventional (stored-integral) form: Dalton's SIRFCK2 path over the
 * AOTWOINT integral file (DALTON/sirius/sirfck.F:1122-1342), with the file
 * held in device memory.  dgf_store_integrals evaluates the integral block
 * of every quartet of the plan for Schwarz threshold thrs once (spherical or
 * Cartesian functions as the basis, FP64, 1/r12) and keeps them on the
 * device; *bytes receives the store's size (also on DGF_ERR_NOMEM, so that a
 * caller can size max_bytes; max_bytes <= 0 means no limit besides the
 * device).  dgf_fock_stored then builds Fock matrices as dgf_fock_device
 * does (any IFCTYP codes, HFXFAC, IFTHRS/ICEDIF screening, shards) by
 * digesting the stored blocks; its opt->thrs must equal the store's thrs,
 * mixed_cutoff must be 0 and hfxmu 0.  A store made before a change of the
 * context's tuning stays valid.  dgf_store_release frees it. */
int dgf_store_integrals(dgf_ctx *ctx, double thrs, int64_t max_bytes, void *stream, int64_t *bytes);
int dgf_fock_stored(dgf_ctx *ctx, dgf_int ndmat, const dgf_int *ifctyp, const double *dmat_device,
                    double *fmat_device, const dgf_options *opt, void *stream, dgf_stats *stats);
int dgf_store_release(dgf_ctx *ctx);

/* Batched Fock builds of many molecules (no counterpart in Dalton, which
 * builds one molecule per run): one launch per quartet class covers every
 * molecule's canonical quartet queue, merged class by class; the launches
 * run on four streams forked from the caller's stream and joined back
 * before the epilogue, and the sequence can be captured once as a CUDA
 * graph and replayed.  Contexts must
 * live on one device with the same spherical flag and stay alive while the
 * batch exists.  Matrices are packed: molecule k's N_k x N_k block starts at
 * offsets[k] (offsets[nmol] = total doubles), see dgf_batch_layout. */
typedef struct dgf_batch dgf_batch;
int dgf_batch_create(dgf_ctx *const *ctxs, dgf_int nmol, dgf_batch **out);
void dgf_batch_destroy(dgf_batch *batch);
int dgf_batch_layout(const dgf_batch *batch, dgf_int *offsets /* nmol + 1 */);

/* J+K (IFCTYP 13, HFXFAC from opt) of every molecule of the batch, device
 * pointers to packed D and F.  use_graph = 1: the first call captures the
 * launch sequence into a CUDA graph, later calls with the same pointers,
 * options and stream replay it.  `stream` is a cudaStream_t (NULL for the
 * legacy default stream).  Kernel choices per class, and with mixed_cutoff
 * > 0 the classes split into FP64 and FP32 launches, come from the context
 * with the most basis functions at dgf_batch_create time (tune it with
 * dgf_autotune first, with the same mixed_cutoff).  Schwarz-screened form
 * only: ifthrs >= 16, one shard, hfxmu = 0. */
int dgf_fock_batch(dgf_batch *batch, const double *dmat_packed_device, double *fmat_packed_device,
                   const dgf_options *opt, int use_graph, void *stream, dgf_stats *stats);

/* Per-class autotuner (no counterpart in Dalton): times every candidate
 * kernel of every quartet class of the plan for opt->thrs on the density
 * dmat_device (N x N, device) -- the cooperative team kernel and the
 * thread-per-quartet kernel in its A-chunk variants, FP64 and FP32 -- and
 * keeps the fastest per class and precision in the context for later builds.
 * A JSON list of the timings is written to `report` (may be NULL). */
int dgf_autotune(dgf_ctx *ctx, const double *dmat_device, const dgf_options *opt, void *stream, char *report,
                 size_t report_len);

/* Copy the kernel choices dgf_autotune stored in `src` to `dst` (no
 * counterpart in Dalton), so that contexts of similar molecules share one
 * tuning run. */
int dgf_copy_tuning(dgf_ctx *dst, const dgf_ctx *src);

/* Pin the kernel of one quartet class (la lb|lc ld), as the autotuner would:
 * precision 64 or 32; variant -4 warp per quartet with FP64 tensor-core
 * (DMMA) transforms, -3 warp per quartet, -2 warp team, -1
 * cooperative team, 0.. thread-kernel chunk variants.  Launches the chosen
 * kernel cannot serve (e.g. a warp kernel restricted to one primitive pair
 * per side) fall back to the default kernel.  DGF_ERR_UNSUPPORTED when the
 * variant does not exist for the class. */
int dgf_set_class_kernel(dgf_ctx *ctx, int la, int lb, int lc, int ld, int precision, int variant);

/* Measurement helper (not part of the HERFCK contract): FP64 and FP32 FMA
 * throughput of device `device` in TFLOP/s from a register-resident FMA
 * loop, the denominator of the FP64-pipe roofline. */
int dgf_measure_fma_peak(int device, double *fp64_tflops, double *fp32_tflops);

/* Number of basis functions, atoms and segmented shells of a context. */
int dgf_info(const dgf_ctx *ctx, dgf_int *nbf, dgf_int *natom, dgf_int *nshell);

/* Workload statistic (no counterpart in Dalton): the number of contracted
 * shell quartets of the AO basis that survive Schwarz screening at `thrs`,
 * one shell per contracted function, canonical (A>=B, C>=D, AB>=CD).  The
 * kernels work in a basis where general contractions are resolved into
 * primitives, so dgf_stats.quartets_total counts that basis's quartets; this
 * count is the implementation-independent size of the build.  Computes the
 * AO pairs' Schwarz factors on the device on every call. */
int dgf_count_ao_quartets(dgf_ctx *ctx, double thrs, dgf_int *count);

/* Message text of a status code. */
const char *dgf_strerror(int status);

/* Text of the last error recorded on this thread (file/line and CUDA text). */
const char *dgf_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* DGFOCK_H */
