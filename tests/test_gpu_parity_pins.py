"""Parity of the GPU build with the oracle at the sizes and options the
benchmarks use: a mid-size water cluster, an f-shell alkane that reaches
every class with L >= 6, the (H2O)32 / cc-pVDZ plan of the headline
workload, Dalton's IFTHRS density screen and ICEDIF Coulomb/exchange skips,
and the mixed form.  Every GPU call goes through the C ABI."""
import numpy as np
import pytest

from dalton_b200 import molecules
from dalton_b200.basis import build_basis
from dalton_b200.fock import FockBuilder

pytestmark = pytest.mark.gpu

TOL = 1e-10  # max-abs on F, FP64 form


def scf_density(bs, conv=1e-7):
    from dalton_b200.scf import rhf

    res = rhf(bs, conv=conv, incremental=False)
    return res["dmat"].cpu().numpy(), res


def energy2(D, F):
    """Two-electron energy 1/2 sum D G of a Fock contribution G."""
    return 0.5 * float(np.sum(D * F))


@pytest.fixture(scope="module")
def h2o8(cuda, orc):
    bs = build_basis(molecules.water_cluster(8, (2, 2, 2), seed=8), "cc-pVDZ")
    D, res = scf_density(bs)
    ref = orc.fock(bs, D, 13, 1.0, 1e-12)
    return bs, D, res["builder"], ref


def test_fock_h2o8_ccpvdz_fp64(h2o8):
    """(H2O)8 / cc-pVDZ (192 basis functions), converged RHF density: FP64
    J - K/2 equals the oracle to 1e-10."""
    bs, D, fb, ref = h2o8
    f = fb.herfck(D, 13)
    err = np.abs(f - ref).max()
    assert err < TOL, f"max |dF| = {err:.3e}"


def test_fock_h2o8_ccpvdz_mixed(h2o8):
    """Mixed form (quartets with Q_AB Q_CD |D| < 1e-6 in FP32) against the
    FP64 oracle: max-element and two-electron energy error."""
    bs, D, fb, ref = h2o8
    f = fb.herfck(D, 13, mixed_cutoff=1e-6)
    st = fb.last_stats
    assert st["quartets_fp32"] > 0
    err = np.abs(f - ref).max()
    de = abs(energy2(D, f) - energy2(D, ref))
    print(f"mixed vs oracle: max |dF| = {err:.3e}, |dE| = {de:.3e} Eh, FP32 quartets {st['quartets_fp32']}")
    assert err < 1e-6
    assert de < 1e-6


@pytest.fixture(scope="module")
def h2o4(cuda, orc):
    bs = build_basis(molecules.water_cluster(4, (2, 2, 1), seed=1), "cc-pVDZ")
    D, res = scf_density(bs)
    full = orc.fock(bs, D, 13, 1.0, 1e-12)
    return bs, D, res["builder"], full


@pytest.mark.parametrize("ifthrs", [6, 8, 9, 10, 11])
def test_ifthrs_screen_against_oracle(h2o4, orc, ifthrs):
    """Dalton's density screen (SYMLOP quartet skip on Dalton's blocks plus
    the ICEDIF Coulomb/exchange skips, IFTHRS < 16) in the GPU build against
    the same screen in the oracle on (H2O)4 / cc-pVDZ.  The GPU skips every
    working-basis quartet of the block quartets Dalton skips, so the error
    each screen leaves in F against the unscreened oracle build is the same
    up to the ICEDIF skips (which the GPU applies only to quartets of whole
    blocks); both skip work."""
    bs, D, fb, full = h2o4
    scr, cnt = orc.fock_screened(bs, D, 13, 1.0, 1e-12, ifthrs=ifthrs, icedif=3)
    f = fb.herfck(D, 13, ifthrs=ifthrs)
    st = fb.last_stats
    err_orc = np.abs(scr - full).max()
    err_gpu = np.abs(f - full).max()
    de_gpu = abs(energy2(D, f) - energy2(D, full))
    frac_gpu = st["quartets_skipped"] / max(st["quartets_total"], 1)
    frac_orc = cnt["skipped_screen"] / max(cnt["skipped_screen"] + cnt["evaluated"], 1)
    print(f"IFTHRS {ifthrs}: max |dF| oracle {err_orc:.2e} GPU {err_gpu:.2e}; GPU |dE| {de_gpu:.2e}; "
          f"skipped quartets oracle {frac_orc:.3f} GPU {frac_gpu:.3f}")
    thr = 10.0 ** -ifthrs
    assert err_orc < 100 * thr
    assert err_gpu <= 1.5 * err_orc + 1e-11
    assert de_gpu < 100 * thr
    if ifthrs <= 9:
        assert st["quartets_skipped"] > 0 and cnt["skipped_screen"] > 0


def test_icedif_bits(h2o4, orc):
    """ICEDIF = 0 (no separate Coulomb/exchange skips) and 3 (both) give
    results within the screen's error of each other and of the unscreened
    build; ICEDIF = 3 drops contributions the quartet skip kept."""
    bs, D, fb, full = h2o4
    f0 = fb.herfck(D, 13, ifthrs=9, icedif=0)
    f3 = fb.herfck(D, 13, ifthrs=9, icedif=3)
    _, c0 = orc.fock_screened(bs, D, 13, 1.0, 1e-12, ifthrs=9, icedif=0)
    _, c3 = orc.fock_screened(bs, D, 13, 1.0, 1e-12, ifthrs=9, icedif=3)
    assert c0["dropped_coulomb"] == c0["dropped_exchange"] == 0
    assert c3["dropped_coulomb"] + c3["dropped_exchange"] > 0
    assert np.abs(f0 - full).max() < 3e-7
    assert np.abs(f3 - full).max() < 3e-7
    assert np.abs(f3 - f0).max() > 0.0


@pytest.fixture(scope="module")
def c4h10(cuda, orc):
    bs = build_basis(molecules.alkane(4, seed=4), "cc-pVTZ")
    rng = np.random.default_rng(40)
    d = rng.normal(size=(bs.nbf, bs.nbf)) * 0.05
    d = d + d.T
    return bs, d, FockBuilder(bs), orc.fock(bs, d, 13, 1.0, 1e-12)


@pytest.mark.parametrize("ifthrs", [20, 11, 9])
def test_fock_c4h10_ccpvtz(c4h10, ifthrs):
    """Butane / cc-pVTZ (f shells): every quartet class up to (ff|ff),
    including all classes with L >= 6 that run in the cooperative kernels.
    Random symmetric density of a physical scale; unscreened to 1e-10 and
    with the IFTHRS screen within 100 x 10^-IFTHRS of the unscreened oracle."""
    bs, d, fb, ref = c4h10
    f = fb.herfck(d, 13, ifthrs=ifthrs)
    err = np.abs(f - ref).max()
    print(f"C4H10/cc-pVTZ IFTHRS {ifthrs}: max |dF| {err:.3e}, skipped {fb.last_stats['quartets_skipped']}")
    if ifthrs >= 16:
        assert err < TOL
    else:
        assert err < 100 * 10.0 ** -ifthrs


def test_h2o32_plan_with_localized_density(cuda, orc):
    """The headline workload's quartet plan, (H2O)32 / cc-pVDZ (768 basis
    functions), checked whole against the oracle: the density is the
    converged monomer RHF density of one water near the cluster's centre
    placed in that water's block (zero elsewhere).  The GPU evaluates every
    quartet of the plan; a quartet contributes only where one of its six
    density blocks touches that water, and the oracle evaluates exactly
    those (it skips quartets whose density bound is exactly zero), so the two
    F agree to 1e-10 everywhere."""
    from dalton_b200.scf import rhf

    mol, basis = molecules.config("h2o32_ccpvdz")
    bs = build_basis(mol, basis)
    k = 21  # a water in the middle layer of the 4 x 4 x 2 grid
    from dalton_b200.basis import Molecule

    sub = Molecule(mol.charges[3 * k:3 * k + 3], mol.coords[3 * k:3 * k + 3], mol.symbols[3 * k:3 * k + 3])
    bsm = build_basis(sub, basis)
    dm = rhf(bsm, conv=1e-8, incremental=False)["dmat"].cpu().numpy()
    lo = [i for i, a in enumerate(bs.ao_atom()) if 3 * k <= a < 3 * k + 3]
    assert len(lo) == bsm.nbf
    D = np.zeros((bs.nbf, bs.nbf))
    D[np.ix_(lo, lo)] = dm
    fb = FockBuilder(bs)
    f = fb.herfck(D, 13)
    ref, cnt = orc.fock_screened(bs, D, 13, 1.0, 1e-12, ifthrs=20)
    err = np.abs(f - ref).max()
    print(f"(H2O)32 plan, one-water density: max |dF| {err:.3e}; oracle evaluated {cnt['evaluated']} quartets, "
          f"skipped {cnt['skipped_zero']} with zero density bound; GPU evaluated {fb.last_stats['quartets_total']}")
    assert cnt["evaluated"] > 0
    assert err < TOL
