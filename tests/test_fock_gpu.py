"""GPU parity of the J/K Fock build (libdgfock through its C ABI) against
the CPU oracle, on the same seeded inputs."""
import numpy as np
import pytest

from dalton_b200.basis import Molecule, build_basis
from dalton_b200.fock import FockBuilder
from dalton_b200 import molecules

pytestmark = pytest.mark.gpu

TOL = 1e-10  # max-abs on F, FP64 form


def rand_density(n, seed, sym=True):
    rng = np.random.default_rng(seed)
    d = rng.normal(size=(n, n)) * 0.1
    if sym:
        d = d + d.T
    return d


def methane():
    return Molecule.from_angstrom(["C", "H", "H", "H", "H"],
                                  [[0, 0, 0], [0.63, 0.63, 0.63], [-0.63, -0.63, 0.63], [-0.63, 0.63, -0.63],
                                   [0.63, -0.63, -0.63]])


CASES = [
    ("h2o_ccpvdz", lambda: molecules.water_dalton_test(), "cc-pVDZ"),
    ("h2o_sto3g", lambda: molecules.water_dalton_test(), "STO-3G"),
    ("ch4_ccpvtz", methane, "cc-pVTZ"),
    ("h2o2_631gs", lambda: molecules.water_cluster(2, seed=3), "6-31G*"),
]


@pytest.mark.parametrize("name,molf,basis", CASES, ids=[c[0] for c in CASES])
def test_fock_symmetric_matches_oracle(cuda, orc, name, molf, basis):
    bs = build_basis(molf(), basis)
    fb = FockBuilder(bs)
    d = rand_density(bs.nbf, 1)
    f_gpu = fb.herfck(d, 13, thrs=1e-12)
    f_ref = orc.fock(bs, d, 13, 1.0, 1e-12)
    err = np.abs(f_gpu - f_ref).max()
    assert err < TOL, f"{name}: max |dF| = {err:.3e}"
    assert np.abs(f_gpu - f_gpu.T).max() < 1e-13


@pytest.mark.parametrize("ifctyp", [11, 12, 13, 1, 2, 3, 22, 23])
def test_fock_ifctyp_matches_oracle(cuda, orc, ifctyp):
    bs = build_basis(molecules.water_dalton_test(), "cc-pVDZ")
    fb = FockBuilder(bs)
    d = rand_density(bs.nbf, 7, sym=False)
    f_gpu = fb.herfck(d, ifctyp, hfxfac=0.7)
    f_ref = orc.fock(bs, d, ifctyp, 0.7, 1e-12)
    assert np.abs(f_gpu - f_ref).max() < TOL


def test_fock_many_densities(cuda, orc):
    bs = build_basis(molecules.water_dalton_test(), "cc-pVDZ")
    fb = FockBuilder(bs)
    ds = np.stack([rand_density(bs.nbf, s, sym=(s % 2 == 0)) for s in range(5)])
    ift = [13, 3, 11, 12, 23]
    f_gpu = fb.herfck(ds, ift)
    f_ref = orc.fock(bs, ds, ift, 1.0, 1e-12)
    assert np.abs(f_gpu - f_ref).max() < TOL


def test_fock_water_cluster_ccpvdz(cuda, orc):
    bs = build_basis(molecules.water_cluster(4, (2, 2, 1), seed=1), "cc-pVDZ")
    fb = FockBuilder(bs)
    d = rand_density(bs.nbf, 4)
    f_gpu = fb.herfck(d)
    f_ref = orc.fock(bs, d, 13, 1.0, 1e-12)
    assert np.abs(f_gpu - f_ref).max() < TOL
    st = fb.last_stats
    assert st["quartets_fp64"] == st["quartets_total"] > 0


def test_f_shells_mixed_and_tuned_match_fp64(cuda, orc):
    """cc-pVTZ (f shells): the single-primitive thread kernels of the f
    classes, their FP32 half and the warp-team candidates, once autotuned,
    reproduce the FP64 oracle (FP64 to 1e-10, mixed to 1e-5)."""
    import torch

    bs = build_basis(methane(), "cc-pVTZ")
    fb = FockBuilder(bs)
    d = rand_density(bs.nbf, 12)
    ref = orc.fock(bs, d, 13, 1.0, 1e-12)
    dt = torch.tensor(d, device=cuda)
    fb.autotune(dt, mixed_cutoff=1e-6)
    f64 = fb.herfck_device(dt).cpu().numpy()
    assert np.abs(f64 - ref).max() < TOL
    fmx = fb.herfck_device(dt, mixed_cutoff=1e-6).cpu().numpy()
    assert np.abs(fmx - ref).max() < 1e-5
    assert abs(0.5 * float(np.sum(d * (fmx - f64)))) < 1e-6


@pytest.mark.parametrize("name,molf,basis", [
    ("h2o3_ccpvdz_cart", lambda: molecules.water_cluster(3, seed=2), "cc-pVDZ"),
    ("ch4_ccpvtz_cart", methane, "cc-pVTZ"),
], ids=["h2o3_ccpvdz_cart", "ch4_ccpvtz_cart"])
def test_cartesian_direct_matches_oracle(cuda, orc, name, molf, basis):
    """Cartesian d and f functions through the direct build: the thread
    kernels digest their Cartesian blocks, A-component chunks included (the
    chunk's rows of F start at an offset inside the A shell), by the default
    kernels, the tuned ones, the mixed split, and two densities at once."""
    import torch

    bs = build_basis(molf(), basis, spherical=False)
    fb = FockBuilder(bs)
    d = rand_density(bs.nbf, 31)
    ref = orc.fock(bs, d, 13, 1.0, 1e-12)
    dt = torch.tensor(d, device=cuda)
    assert np.abs(fb.herfck_device(dt).cpu().numpy() - ref).max() < TOL
    fb.autotune(dt, mixed_cutoff=1e-6)
    assert np.abs(fb.herfck_device(dt).cpu().numpy() - ref).max() < TOL
    fmx = fb.herfck_device(dt, mixed_cutoff=1e-6).cpu().numpy()
    assert np.abs(fmx - ref).max() < 1e-5
    d2 = rand_density(bs.nbf, 32, sym=False)
    f2 = fb.herfck(np.stack([d, d2]), ifctyp=[13, 3])
    assert np.abs(f2[0] - ref).max() < TOL
    assert np.abs(f2[1] - orc.fock(bs, d2, 3, 1.0, 1e-12)).max() < TOL
