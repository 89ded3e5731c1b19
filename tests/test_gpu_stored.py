"""The conventional (stored-integral) form of the Fock build, Dalton's
SIRFCK2 over the AOTWOINT integral file (DALTON/sirius/sirfck.F:1122-1342)
with the file held in device memory: the integral blocks are evaluated once
(dgf_store_integrals) and digested for any densities (dgf_fock_stored).
Checked against the direct build and the oracle through the C ABI."""
import numpy as np
import pytest

from dalton_b200 import _lib, molecules
from dalton_b200.basis import Molecule, build_basis
from dalton_b200.fock import FockBuilder

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _density(n, seed, scale=0.05, nd=None):
    rng = np.random.default_rng(seed)
    shape = (n, n) if nd is None else (nd, n, n)
    d = rng.normal(size=shape) * scale
    return d + np.swapaxes(d, -1, -2)


def _methane():
    r = 0.63
    return Molecule.from_angstrom(["C", "H", "H", "H", "H"],
                                  [[0, 0, 0], [r, r, r], [-r, -r, r], [-r, r, -r], [r, -r, -r]])


@pytest.fixture(scope="module")
def h2o4(cuda):
    bs = build_basis(molecules.water_cluster(4, (2, 2, 1), seed=1), "cc-pVDZ")
    fb = FockBuilder(bs)
    nbytes = fb.store_integrals()
    assert nbytes > 0
    return bs, fb


@pytest.mark.parametrize("ifctyp,hfxfac", [(13, 1.0), (11, 1.0), (12, 0.3), (13, 0.25)])
def test_stored_equals_direct(h2o4, ifctyp, hfxfac):
    import torch

    bs, fb = h2o4
    d = torch.tensor(_density(bs.nbf, 5), device="cuda")
    ref = fb.herfck_device(d, ifctyp=ifctyp, hfxfac=hfxfac).clone()
    f = fb.herfck_stored(d, ifctyp=ifctyp, hfxfac=hfxfac)
    assert float(torch.max(torch.abs(f - ref))) < 1e-12
    assert fb.last_stats["quartets_total"] > 0


def test_stored_several_densities(h2o4, orc):
    """A general and an antisymmetric density at once (IFCTYP 3 and 22)."""
    import torch

    bs, fb = h2o4
    rng = np.random.default_rng(8)
    d = rng.normal(size=(2, bs.nbf, bs.nbf)) * 0.05
    f = fb.herfck_stored(torch.tensor(d, device="cuda"), ifctyp=[3, 22], hfxfac=0.5).cpu().numpy()
    ref = orc.fock(bs, d, [3, 22], 0.5, 1e-12)
    assert np.abs(f - ref).max() < TOL


def test_stored_density_screen(h2o4, orc):
    """IFTHRS / ICEDIF screening on the stored blocks: the error against the
    unscreened build is that of the oracle's screen."""
    import torch

    bs, fb = h2o4
    d = _density(bs.nbf, 9, scale=0.01)
    full = orc.fock(bs, d, 13, 1.0, 1e-12)
    scr, _ = orc.fock_screened(bs, d, 13, 1.0, 1e-12, ifthrs=9, icedif=3)
    f = fb.herfck_stored(torch.tensor(d, device="cuda"), ifthrs=9).cpu().numpy()
    assert fb.last_stats["quartets_skipped"] > 0
    assert np.abs(f - full).max() <= 1.5 * np.abs(scr - full).max() + 1e-11


@pytest.mark.parametrize("basis,spherical", [("cc-pVTZ", True), ("cc-pVTZ", False)])
def test_stored_f_shells(cuda, orc, basis, spherical):
    """CH4 / cc-pVTZ: every class up to (ff|ff), so blocks come from the
    thread, warp and cooperative kernels, spherical and Cartesian."""
    import torch

    bs = build_basis(_methane(), basis, spherical=spherical)
    fb = FockBuilder(bs)
    fb.store_integrals()
    d = _density(bs.nbf, 21)
    f = fb.herfck_stored(torch.tensor(d, device="cuda")).cpu().numpy()
    assert np.abs(f - orc.fock(bs, d, 13, 1.0, 1e-12)).max() < TOL


def test_stored_contracted_pairs_and_tuning(cuda, orc):
    """6-31G* (contracted s/sp shells): blocks of multi-primitive pairs, and a
    store made with tuned kernel choices."""
    import torch

    bs = build_basis(molecules.water_cluster(2, seed=5), "6-31G*")
    fb = FockBuilder(bs)
    d = _density(bs.nbf, 3)
    dt = torch.tensor(d, device="cuda")
    fb.autotune(dt)
    fb.store_integrals()
    f = fb.herfck_stored(dt).cpu().numpy()
    assert np.abs(f - orc.fock(bs, d, 13, 1.0, 1e-12)).max() < TOL


def test_stored_scf_energy(cuda):
    """An RHF built on stored integrals reaches the direct build's energy."""
    from dalton_b200.scf import rhf

    bs = build_basis(molecules.water_cluster(2, seed=7), "cc-pVDZ")
    direct = rhf(bs, conv=1e-8, incremental=False)
    fb = FockBuilder(bs)
    fb.store_integrals()
    stored = rhf(bs, fb, conv=1e-8, incremental=False, stored=True)
    assert abs(stored["energy"] - direct["energy"]) < 1e-10


def test_stored_errors(cuda):
    import torch

    bs = build_basis(molecules.water_dalton_test(), "cc-pVDZ")
    fb = FockBuilder(bs)
    d = torch.tensor(_density(bs.nbf, 2), device="cuda")
    with pytest.raises(_lib.DgfError):
        fb.herfck_stored(d)  # no store yet
    nbytes = fb.store_integrals(thrs=1e-12)
    with pytest.raises(_lib.DgfError):
        fb.herfck_stored(d, thrs=1e-10)  # another threshold
    with pytest.raises(_lib.DgfError) as e:
        fb.store_integrals(thrs=1e-12, max_bytes=nbytes // 2)
    assert e.value.status == _lib.DGF_ERR_NOMEM
    fb.store_integrals(thrs=1e-12)
    ref = fb.herfck_device(d).clone()
    assert float(torch.max(torch.abs(fb.herfck_stored(d) - ref))) < 1e-12
    fb.release_store()
    with pytest.raises(_lib.DgfError):
        fb.herfck_stored(d)
