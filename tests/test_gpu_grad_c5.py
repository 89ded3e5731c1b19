"""RHF gradient at the gradient benchmark's size and with the mixed forward
build: the analytic gradient of (H2O)16 / cc-pVDZ (384 basis functions)
against central finite differences of the SCF energy, and the gradient of a
mixed-precision SCF against the all-FP64 one."""
import numpy as np
import pytest

from dalton_b200 import molecules
from dalton_b200.basis import build_basis

pytestmark = pytest.mark.gpu


def test_mixed_forward_gradient_h2o4(cuda):
    """Mixed form in the forward SCF (FP32 for quartets with Q_AB Q_CD |D| <
    1e-6, incremental builds winning the accuracy back): the RHF gradient
    matches the all-FP64 SCF's to 1e-6 Eh/bohr."""
    from dalton_b200.grad import rhf_gradient
    from dalton_b200.scf import rhf

    bs = build_basis(molecules.water_cluster(4, (2, 2, 1), seed=1), "cc-pVDZ")
    r64 = rhf(bs, conv=1e-9, incremental=False)
    rmx = rhf(bs, r64["builder"], conv=1e-9, mixed_cutoff=1e-6)
    g64 = rhf_gradient(r64["builder"], r64["dmat"], r64["wmat"])
    gmx = rhf_gradient(r64["builder"], rmx["dmat"], rmx["wmat"])
    err = np.abs(gmx - g64).max()
    print(f"mixed-forward gradient vs FP64: max diff {err:.2e} Eh/bohr; energy diff "
          f"{abs(rmx['energy'] - r64['energy']):.2e} Eh")
    assert err < 1e-6
    assert abs(rmx["energy"] - r64["energy"]) < 1e-6


def test_rhf_gradient_h2o16_finite_difference(cuda):
    """(H2O)16 / cc-pVDZ: three Cartesian components of the analytic RHF
    gradient (one- and two-electron parts, backward kernel) against central
    differences (h = 1e-4 bohr) of fully converged SCF energies."""
    from dalton_b200.grad import rhf_gradient
    from dalton_b200.scf import rhf

    mol, basis = molecules.config("h2o16_ccpvdz")
    bs = build_basis(mol, basis)
    res = rhf(bs, conv=1e-10, incremental=False)
    g = rhf_gradient(res["builder"], res["dmat"], res["wmat"])
    res["builder"].close()
    h = 1e-4
    for atom, k in ((0, 0), (7, 1), (29, 2)):
        e = []
        for sgn in (1.0, -1.0):
            c = bs.molecule.coords.copy()
            c[atom, k] += sgn * h
            r = rhf(bs.with_coords(c), conv=1e-10, incremental=False)
            e.append(r["energy"])
            r["builder"].close()
        fd = (e[0] - e[1]) / (2 * h)
        print(f"atom {atom} axis {k}: analytic {g[atom, k]:.9f} finite difference {fd:.9f}")
        assert abs(fd - g[atom, k]) < 1e-6
