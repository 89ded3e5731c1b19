/* CPU oracle for the direct J/K Fock build — TEST INFRASTRUCTURE ONLY.
 *
 * A plain C++ restatement of Dalton's HERMIT two-electron Fock path, used by
 * tests/, __graft_entry__.smoke() and the CPU-baseline legs of bench.py as the
 * checker.  Nothing in the product (dalton_b200/, include/) links or calls it.
 *
 * Parity is pinned by Dalton's stored golden outputs: the H2O/cc-pVDZ direct
 * RHF energy (DALTON/test/trueresult/energy_direct.ref:659) and the acrolein
 * HF/STO-3G energy and molecular gradient
 * (DALTON/test/geoopt_preopt2/result/preopt_acrolein.out:637,840-850).
 *
 * The basis arrives in Dalton block form (one block = one atom's shell of
 * angular momentum l with nprim primitives and ncontr contracted functions,
 * CPRIM coefficients already NRMORB-normalised), AOs in Dalton C1 order.
 */
#ifndef DGF_ORACLE_H
#define DGF_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int64_t nblock, natom, nbf, spherical;
  const int64_t *block_l, *block_atom, *block_nprim, *block_ncontr;
  const int64_t *block_ao_offset, *block_prim_offset, *block_coef_offset;
  const double *prim_exp, *coef; /* coef: per block column-major (nprim, ncontr) */
  const double *atom_xyz;        /* (natom, 3) bohr */
  const double *atom_charge;     /* (natom,) */
} orc_basis;

/* Number of OpenMP threads the oracle uses (0 = all). */
void orc_set_threads(int n);
int orc_get_threads(void);

/* Boys function F_0..F_m(T) (own series / asymptotic evaluation). */
void orc_boys(int m, double t, double *f);

/* Cartesian -> spherical matrix, (2l+1) x ncart(l) row-major (SPHCO1, MINTEG=2). */
void orc_sph_matrix(int l, double *out);

/* One-electron S, T, V (N x N, row-major; symmetric). */
int orc_oneint(const orc_basis *b, double *S, double *T, double *V);

/* Full ERI tensor (N^4, (pq|rs) at ((p*N+q)*N+r)*N+s) for small checks. */
int orc_eri_full(const orc_basis *b, double *eri);

/* Schwarz factors per segmented shell pair: Q_AB = sqrt(max |(ab|ab)|).
 * Returns the number of segmented shells in *nshell. */
int orc_nshell(const orc_basis *b);
int orc_schwarz(const orc_basis *b, double *q /* nshell^2 */, int64_t *shell_l, int64_t *shell_nprim,
                int64_t *shell_atom);

/* Fock build with HERFCK semantics (FMAT overwritten):
 *   IFCTYP = 10*X + Y; X = 1 symmetric D, 0 general, 2 antisymmetric;
 *   Y = 1 Coulomb, 2 exchange, 3 both.
 *   F = [Y&1] J[D] - [Y&2] (hfxfac/2) K[D],
 *   J_pq = sum_rs (pq|rs) (D_rs + D_sr)/2, K_pq = sum_rs (pr|qs) D_rs.
 * Shell quartets with Q_AB * Q_CD < thrs are skipped (segmented shells).
 * Matrices are N x N row-major; ndmat densities back to back. */
int orc_fock(const orc_basis *b, int ndmat, const int64_t *ifctyp, const double *dmat,
             double *fmat, double hfxfac, double thrs);

/* orc_fock with Dalton's direct-Fock density screening (IFTHRS < 16 turns it
 * on): the SYMLOP quartet skip on Dalton's blocks (her2drv.F:2663-2733), the
 * FCKTOL integral drop and the per-density Coulomb/exchange skips selected by
 * the bits of ICEDIF (her2fck.F:84-90, 221-222, 446-466).  counts (may be
 * NULL) receives 5 values: quartets evaluated, skipped by the screen, skipped
 * because their density bound is exactly zero, density Coulomb parts
 * dropped, density exchange parts dropped. */
int orc_fock_screened(const orc_basis *b, int ndmat, const int64_t *ifctyp, const double *dmat, double *fmat,
                      double hfxfac, double thrs, int64_t ifthrs, int64_t icedif, int64_t *counts);

/* HERFCK_1 with range-separated exchange (DALTON/abacus/herdirect.F:792-835):
 * orc_fock, then for hfxmu != 0 a second pass with the operator
 * erf(hfxmu r12)/r12 adding -hfxatt/2 K[D] (exchange only for every
 * density, FCKCON's IY = 2 of herfckcon.F:66). */
int orc_fock_attenuated(const orc_basis *b, int ndmat, const int64_t *ifctyp, const double *dmat, double *fmat,
                        double hfxfac, double thrs, double hfxmu, double hfxatt);

/* One primitive Cartesian block (la lb|lc ld) of unnormalised Gaussians with
 * exponents exps[4] at centers[4][3], operator erf(mu r12)/r12 (mu = 0:
 * 1/r12), out[((a*nb+b)*nc+c)*nd+d]. */
void orc_prim_eri(int la, int lb, int lc, int ld, const double *exps, const double *centers, double mu, double *out);

/* Timing sample of a J+K build (IFCTYP 13, hfxfac 1) for the CPU baseline:
 * the significant quartets whose hash falls in a fixed 2^-k fraction (the
 * workload's class mix), evaluated and digested on all threads; *nsample
 * quartets in *seconds, *total significant quartets (see oracle.cpp). */
int orc_fock_hash_sample(const orc_basis *b, const double *dmat, double thrs, int k, int64_t *nsample,
                         double *seconds, int64_t *total);

/* Sampled J+K build (IFCTYP 13, hfxfac 1) over the bra pairs ab with
 * ab % stride == offset, for CPU-baseline timing; *nquartet = quartets done. */
int orc_fock_sampled(const orc_basis *b, const double *dmat, double *fmat, double thrs, int stride, int offset,
                     int64_t *nquartet);

/* Two-electron part of the RHF gradient: 1/2 sum (pq|rs)^x [D_pq D_rs - hfx/2 D_pr D_qs],
 * D the total (symmetric) density; grad (natom, 3) overwritten. */
int orc_grad2e(const orc_basis *b, const double *dmat, double hfxfac, double thrs, double *grad);

/* One-electron + nuclear-repulsion part of the RHF gradient:
 *   sum D_pq h_pq^x - sum W_pq S_pq^x + dVnn/dx; grad (natom, 3) overwritten. */
int orc_grad1e(const orc_basis *b, const double *dmat, const double *wmat, double *grad);

#ifdef __cplusplus
}
#endif
#endif
