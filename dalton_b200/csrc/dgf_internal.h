// Internal definitions shared by the host runtime and the device kernels of
// libdgfock (the B200 direct J/K Fock build).
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <string>
#include <vector>


namespace dgf {

constexpr int kMaxShellL = 3;                                         // s, p, d, f
constexpr int kNumPairClass = (kMaxShellL + 1) * (kMaxShellL + 2) / 2;  // (la >= lb) classes
constexpr int kMaxSlots = 8;  // density slots processed together by one kernel pass
constexpr int kNumBuckets = 7;  // primitive-pair-count buckets of a class list

// Bucket of a pair by its primitive-pair count (1, 2, <=4, <=8, <=16, <=32, more):
// lanes of a warp then loop over similar ket primitive counts.
__host__ __device__ inline int npp_bucket(int n) {
  return n <= 1 ? 0 : n <= 2 ? 1 : n <= 4 ? 2 : n <= 8 ? 3 : n <= 16 ? 4 : n <= 32 ? 5 : 6;
}

// Schwarz bins: inside a primitive-count bucket, pairs are ordered by bin of
// log2 Q (descending), then by shell indices, so that the kets of a warp's
// lanes are neighbours in the density and Fock matrices.  A bra's significant
// kets are then a prefix of whole bins, and the kernels drop the few quartets
// of the last bin below the threshold.
constexpr int kQBinsPerOctave = 2;
inline int q_bin(double q) {
  if (!(q > 0.0)) return -(1 << 20);
  int e = 0;
  const double m = std::frexp(q, &e);  // q = m 2^e, m in [0.5, 1)
  return (int)std::floor(((double)e + std::log2(m)) * kQBinsPerOctave);
}
inline double q_bin_upper(int bin) {  // every Q of the bin is below this
  return bin <= -(1 << 20) ? 0.0 : std::exp2((double)(bin + 1) / kQBinsPerOctave);
}

// Boys-function table: F_M(T) on [0, kBoysTmax) in kBoysNint intervals of
// width 1/kBoysPerUnit, a degree-kBoysDeg polynomial in x = (T - mid) * 2 *
// kBoysPerUnit per interval (Chebyshev interpolant converted to powers of x).
constexpr int kBoysMaxM = 17;
constexpr int kBoysPerUnit = 2;
constexpr double kBoysTmax = 40.0;
constexpr int kBoysNint = 80;
constexpr int kBoysDeg = 11;
constexpr int kBoysNcoef = kBoysDeg + 1;
constexpr int kBoysTableDoubles = kBoysNint * kBoysNcoef;
constexpr int kBoysDegLow = 5;  // tables of the FP32 half of the mixed form
// Device table layout: orders 0..kBoysMaxM at full degree, then the same
// orders at degree kBoysDegLow (same interval layout, unused coefficients 0).
constexpr size_t kBoysAllDoubles = 2 * (size_t)(kBoysMaxM + 1) * kBoysTableDoubles;
__host__ __device__ constexpr size_t boys_low_offset(int M) {
  return ((size_t)(kBoysMaxM + 1) + M) * kBoysTableDoubles;
}

__host__ __device__ constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }
__host__ __device__ constexpr int n3(int L) { return (L + 1) * (L + 2) * (L + 3) / 6; }
__host__ __device__ constexpr int pair_class(int la, int lb) { return la * (la + 1) / 2 + lb; }
__host__ __device__ constexpr int cmax(int a, int b) { return a > b ? a : b; }

// Primitive pair of a shell pair (A first, the higher angular momentum).
// K = c_a c_b exp(-mu |AB|^2) sqrt(2 pi^(5/2)) / p, Dalton's FAC12 with R2PI52
// (DALTON/abacus/her2odc.F:229-231, DALTON/include/pi.h:9-14).  96 bytes,
// 16-byte aligned so that a lane reads one with 128-bit loads; the primitive
// pairs of a context are stored in the order of the class-sorted pair list,
// so the kets of consecutive lanes are adjacent in memory.
struct __align__(16) PrimPair {
  double p, Px, Py, Pz, PAx, PAy, PAz, PBx, PBy, PBz, K, ea;  // ea: exponent of A (B's is p - ea)
};

// Shell pair record in a class list (sorted by Schwarz factor, descending),
// 64 bytes in four 16-byte groups, the fields every quartet reads first.
struct __align__(16) PairRec {
  int aoA, aoB;    // first function of each shell (within its molecule's working basis)
  int pp0, npp;    // primitive-pair range
  int same;        // A == B
  int shA, shB;    // working-basis shell indices (A has l >= l of B)
  int nbfm;        // basis size of the pair's molecule (row stride of its D/F blocks)
  double Q;        // Schwarz factor sqrt(max |(ab|ab)|)
  int64_t dbase;   // offset of the molecule's N x N block in packed D/F storage (0 for one molecule)
  int atA, atB;    // atoms of A and B
  int blkA, blkB;  // Dalton blocks of A and B, bit kWholeBlock set when the shell is its whole block
};
constexpr int kWholeBlock = 1 << 30;

static_assert(sizeof(PrimPair) == 96 && sizeof(PairRec) == 64, "pair records are read 16 bytes at a time");

// Arguments of one quartet-class launch.
struct JKArgs {
  const PairRec *bra;
  const PairRec *ket;
  const int64_t *qoff;      // prefix sums of ket partners per bra (nbra+1), device
  const int *kbase;         // per bra: first ket of its molecule in the ket list (batches), or null
  int ket_off;              // position of ket[0] in its class list (same-class weight compares ib, ic + ket_off)
  int ket_pp0;              // >= 0: kets of one primitive pair each, ket ic's primitive pair is pp[ket_pp0 + ic]
  int64_t slot_stride;      // elements between density slots in D, Ds, Fh
  int nbra;
  int same_class;           // bra class == ket class (canonical ket <= bra)
  int64_t q_begin;          // first quartet of this launch (shard start)
  int64_t nquartet;         // one past the last quartet of this launch
  const PrimPair *pp;
  const double *boys;       // table for M = L of this class
  const double *sph;        // Cartesian->spherical tables, see sph_offset()
  int spherical;
  int nbf;
  int nslot;
  const double *D;          // [nslot][N*N] densities (exchange)
  const double *Ds;         // [nslot][N*N] D + D^T (Coulomb)
  double *Fh;               // [nslot][N*N] half Fock accumulators
  double jscale[kMaxSlots];
  double kscale[kMaxSlots];
  // screening / precision split
  const float *dmax;        // [nshell*nshell] max |D| per shell pair, or null
  // batches: max |D| per shell pair stored in the packed working-matrix
  // layout, at (first function of A, first function of B) of the pair's
  // molecule (offset dbase, stride nbfm); null: dmax above
  const float *dmax_w;
  int nshell;
  double dens_thr;          // skip if bound < dens_thr (0: no density screening)
  double split;             // precision split bound
  double schwarz_thr;       // skip quartets with Q_AB Q_CD below this (0: the plan is exact)
  double erf_mu2;           // > 0: the attenuated operator erf(mu r12)/r12 with mu^2 = erf_mu2; 0: 1/r12
  // conventional (stored-integral) form: store_out non-null makes the
  // integral kernels write each evaluated quartet's block (layout [a][b][c][d],
  // spherical or Cartesian functions, store_nint values) to store_out +
  // store_base + q store_nint instead of digesting it; the digest kernels
  // read the blocks from store_in the same way
  double *store_out;
  const double *store_in;
  int64_t store_base;
  int store_nint;
  int mode;                 // 0: all, 1: bound >= split only, 2: bound < split only
  double *diag_out;         // Schwarz mode: sqrt(max |(ab|ab)|) per bra pair, no digestion
  unsigned long long *counters;  // [0] quartets done, [1] primitive quartets, [2] skipped
  // Dalton's density screen on its blocks (an atom's shell of angular
  // momentum l with all its contracted functions; every working shell lies
  // in one): block Schwarz factors GAB (nblk x nblk), block maxima of |D| of
  // the AO densities, over all slots and per slot (blk_stride apart), the
  // ICEDIF threshold (0: off) and bits.  blk_gab null: no density screen.
  const double *blk_gab;
  const float *blk_dmax;
  const float *blk_dmax_slot;
  int64_t blk_stride;
  int nblk;
  double ice_thr;
  int icedif;
  // ket table of single-primitive kets (kets of one primitive pair, one
  // molecule): per pair index, {aoA, aoB, same, shA << 16 | shB}, the
  // Schwarz factor, and the primitive pair's p, P, K, P-A, P-B as eleven
  // planes of ks_stride doubles; ket ic of the launch is entry ks_base + ic.
  // ks_i null: the kernels read the pair and primitive-pair records.
  const int4 *ks_i;
  const double *ks_q;
  const double *ks_pp;
  int64_t ks_stride;
  int ks_base;
  // gradient mode (dgf_grad2e): densities D1, D2 (N*N) and grad (natom*3)
  const double *G1, *G2;
  double *grad;
  double hfx;
  int natom;
};

// Offset of the l-block of the Cartesian->spherical table: rows m=-l..l,
// ncart(l) columns, l = 0..kMaxShellL+1.
__host__ __device__ inline int sph_offset(int l) {
  int off = 0;
  for (int k = 0; k < l; ++k) off += (2 * k + 1) * ncart(k);
  return off;
}
constexpr int kSphTableDoubles = 1 * 1 + 3 * 3 + 5 * 6 + 7 * 10 + 9 * 15;

typedef void (*JKLauncher)(const JKArgs &, int grid, int block, size_t smem, cudaStream_t);

enum { kKindThread = 0, kKindTeam = 1, kKindWarpTeam = 2, kKindWarp = 4, kKindWarpMma = 6 };

struct ClassKernel {
  JKLauncher launch;
  int block;
  size_t smem;   // dynamic shared memory (team and warp kernels); 0 for thread kernels
  int chunks;    // thread kernels: A-component chunks (grid.y)
  int qpb;       // quartets a block works on at a time (grid sizing)
  int kind;      // kKindThread, kKindTeam, kKindWarpTeam, kKindWarp or kKindWarpMma
};

constexpr int kThreadVariants = 2;

// Per-class launch table (filled by dgf_jk.cu): index [X][Y] of pair classes.
// precision: 0 = default FP64 kernel, 1 = FP32 kernel, 2 = team kernel.
// ket1: the launch's kets have one primitive pair each (thread kernels then
// use their single-ket-primitive form); bra1: so do all pairs of the bra
// class (with ket1, the condition of the warp-per-quartet kernel).
const ClassKernel &jk_kernel(int X, int Y, int precision, bool ket1 = false, bool bra1 = false);
// Digestion kernel of stored integral blocks of class pair (X, Y).
const ClassKernel &jk_stored_kernel(int X, int Y);
// variant -3 = warp-per-quartet kernel, -2 = warp-team kernel, -1 = team
// kernel, >= 0 = thread-kernel variant (precision 0/1).
const ClassKernel &jk_kernel_variant(int X, int Y, int precision, int variant, bool ket1 = false,
                                     bool bra1 = false);
cudaError_t jk_prepare_all();

void boys_table_host(std::vector<double> &out);       // [kBoysMaxM+1][kBoysTableDoubles]
void sph_table_host(std::vector<double> &out);        // kSphTableDoubles
double boys_reference(int m, double t);               // accurate host F_m(t)

void set_error(const char *file, int line, const std::string &msg);

}  // namespace dgf

