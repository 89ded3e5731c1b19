"""Range-separated exchange on the GPU (Dalton's HFXMU/HFXATT pass of
HERFCK_1, DALTON/abacus/herdirect.F:792-835): the two-pass Fock build
through the C ABI against the oracle's restatement, for s/p/d shells (thread
kernels), f shells (warp and cooperative kernels), several IFCTYP codes and
the mixed form."""
import numpy as np
import pytest

from dalton_b200 import molecules
from dalton_b200.basis import build_basis
from dalton_b200.fock import FockBuilder

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _methane():
    from dalton_b200.basis import Molecule

    r = 0.63
    return Molecule.from_angstrom(["C", "H", "H", "H", "H"],
                                  [[0, 0, 0], [r, r, r], [-r, -r, r], [-r, r, -r], [r, -r, -r]])


def _density(n, seed, scale=0.05):
    rng = np.random.default_rng(seed)
    d = rng.normal(size=(n, n)) * scale
    return d + d.T


@pytest.mark.parametrize("ifctyp", [13, 11, 12])
def test_attenuated_exchange_water_pair(cuda, orc, ifctyp):
    bs = build_basis(molecules.water_cluster(2, seed=3), "cc-pVDZ")
    d = _density(bs.nbf, 60 + ifctyp)
    fb = FockBuilder(bs)
    f = fb.herfck(d, ifctyp, hfxfac=0.19, hfxmu=0.33, hfxatt=0.46)
    ref = orc.fock_attenuated(bs, d, ifctyp, 0.19, 1e-12, 0.33, 0.46)
    err = np.abs(f - ref).max()
    print(f"IFCTYP {ifctyp}: max |dF| {err:.2e}")
    assert err < TOL
    # the attenuated pass changes the result
    assert np.abs(f - fb.herfck(d, ifctyp, hfxfac=0.19)).max() > 1e-4


def test_attenuated_exchange_f_shells(cuda, orc):
    """CH4 / cc-pVTZ: every class up to (ff|ff), so the warp-per-quartet and
    cooperative kernels take the attenuated operator too."""
    bs = build_basis(_methane(), "cc-pVTZ")
    d = _density(bs.nbf, 71)
    fb = FockBuilder(bs)
    f = fb.herfck(d, 13, hfxfac=0.0, hfxmu=0.4, hfxatt=1.0)
    ref = orc.fock_attenuated(bs, d, 13, 0.0, 1e-12, 0.4, 1.0)
    assert np.abs(f - ref).max() < TOL


def test_attenuated_exchange_general_densities(cuda, orc):
    """Two densities at once, a general and an antisymmetric one (IFCTYP 3, 22)."""
    bs = build_basis(molecules.water_cluster(2, seed=3), "cc-pVDZ")
    rng = np.random.default_rng(81)
    d = rng.normal(size=(2, bs.nbf, bs.nbf)) * 0.05
    fb = FockBuilder(bs)
    f = fb.herfck(d, [3, 22], hfxfac=0.5, hfxmu=0.8, hfxatt=0.3)
    ref = orc.fock_attenuated(bs, d, [3, 22], 0.5, 1e-12, 0.8, 0.3)
    assert np.abs(f - ref).max() < TOL


def test_attenuated_exchange_mixed(cuda, orc):
    """Mixed form: quartets below the cutoff in FP32 in both passes."""
    bs = build_basis(molecules.water_cluster(4, (2, 2, 1), seed=1), "cc-pVDZ")
    d = _density(bs.nbf, 91, scale=0.02)
    fb = FockBuilder(bs)
    f = fb.herfck(d, 13, hfxfac=0.2, hfxmu=0.33, hfxatt=0.8, mixed_cutoff=1e-6)
    assert fb.last_stats["quartets_fp32"] > 0
    ref = orc.fock_attenuated(bs, d, 13, 0.2, 1e-12, 0.33, 0.8)
    err = np.abs(f - ref).max()
    print(f"mixed: max |dF| {err:.2e}")
    assert err < 1e-6
