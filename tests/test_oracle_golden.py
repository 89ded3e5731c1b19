"""The oracle (CPU restatement of Dalton's HERMIT path) against Dalton's own
stored golden outputs, and against brute-force and finite-difference checks
of itself.  Golden values are Dalton test outputs:
  DALTON/test/trueresult/energy_direct.ref:659 (H2O/cc-pVDZ direct RHF)
  DALTON/test/geoopt_preopt2/result/preopt_acrolein.out:637,840-850
  (acrolein HF/STO-3G energy and molecular gradient)."""
import json
import os

import numpy as np
import pytest

from dalton_b200 import molecules
from dalton_b200.basis import build_basis

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def golden(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def test_h2o_ccpvdz_direct_rhf_energy(orc):
    g = golden("dalton_energies.json")["energy_direct"]
    bs = build_basis(molecules.water_dalton_test(), "cc-pVDZ")
    assert bs.nbf == 24
    assert abs(bs.molecule.nuclear_repulsion() - g["nuclear_repulsion"]) < 1e-11
    r = orc.rhf(bs, conv=1e-10)
    assert abs(r["energy"] - g["energy"]) < 1e-9


def test_acrolein_sto3g_energy_and_gradient(orc):
    g = golden("dalton_energies.json")["preopt_acrolein"]
    bs = build_basis(molecules.acrolein(), "STO-3G")
    assert np.abs(bs.molecule.coords - np.array(g["coords_bohr"])).max() < 1e-9
    r = orc.rhf(bs, conv=1e-10)
    assert abs(r["energy"] - g["energy"]) < 1e-9
    grad = orc.rhf_gradient(bs, r)
    # Dalton's gradient is printed at its own (looser) SCF convergence; the
    # gradient is linear in the density error, hence 1e-6 Eh/bohr.
    assert np.abs(grad - np.array(g["gradient"])).max() < 1e-6
    assert np.abs(grad.sum(0)).max() < 1e-10


def test_boys_against_mpmath(orc):
    mpmath = pytest.importorskip("mpmath")
    mpmath.mp.dps = 40
    for m in (0, 1, 4, 8, 12, 16):
        for t in (0.0, 1e-9, 0.3, 5.0, 17.3, 35.9, 49.9, 50.1, 80.0, 300.0):
            f = orc.boys(m, t)[m]
            if t == 0.0:
                ref = mpmath.mpf(1) / (2 * m + 1)
            else:
                ref = mpmath.quad(lambda u: u ** (2 * m) * mpmath.e ** (-t * u * u), [0, 1])
            assert abs(f - float(ref)) <= 1e-14 * float(ref) + 1e-300, (m, t)


def test_spherical_functions_orthonormal(orc):
    from dalton_b200.basis import Molecule

    for bas in ("cc-pVTZ",):
        bs = build_basis(Molecule.from_bohr(["C"], [[0.0, 0.0, 0.0]]), bas)
        S, _, _ = orc.oneint(bs)
        # functions of one contracted shell are orthonormal
        for i in range(bs.nblock):
            l, nc = int(bs.block_l[i]), int(bs.block_ncontr[i])
            nf = 2 * l + 1 if l >= 2 else (l + 1) * (l + 2) // 2
            for k in range(nc):
                o = int(bs.block_ao_offset[i]) + k * nf
                blk = S[o:o + nf, o:o + nf]
                assert np.abs(blk - np.eye(nf)).max() < 1e-12


def brute_jk(eri, d):
    j = np.einsum("pqrs,rs->pq", eri, d)
    k = np.einsum("prqs,rs->pq", eri, d)
    return j, k


@pytest.mark.parametrize("ifctyp", [13, 11, 12, 3, 1, 2, 23, 22])
def test_oracle_fock_matches_brute_force(orc, ifctyp):
    bs = build_basis(molecules.water_dalton_test(), "6-31G*")
    eri = orc.eri_full(bs)
    rng = np.random.default_rng(ifctyp)
    d = rng.normal(size=(bs.nbf, bs.nbf))
    X, Y = divmod(ifctyp, 10)
    dd = {1: 0.5 * (d + d.T), 2: 0.5 * (d - d.T), 0: d}[X]
    if X == 2:
        Y &= 2
    j, k = brute_jk(eri, dd)
    ref = (j if Y & 1 else 0) - (0.35 * k if Y & 2 else 0)
    f = orc.fock(bs, d, ifctyp, 0.7, 0.0)
    assert np.abs(f - ref).max() < 1e-11


def test_eri_permutational_symmetry(orc):
    bs = build_basis(molecules.water_dalton_test(), "cc-pVDZ")
    eri = orc.eri_full(bs)
    for perm in ("qprs", "pqsr", "rspq"):
        assert np.abs(eri - np.einsum(f"pqrs->{perm}", eri)).max() < 1e-12


def test_oracle_gradient_finite_difference(orc):
    bs = build_basis(molecules.water_dalton_test(), "STO-3G")
    r = orc.rhf(bs, conv=1e-11)
    g = orc.rhf_gradient(bs, r, thrs=0.0)
    h = 1e-4
    for atom, k in ((0, 1), (1, 0), (2, 2)):
        e = []
        for s in (1, -1):
            c = bs.molecule.coords.copy()
            c[atom, k] += s * h
            e.append(orc.rhf(bs.with_coords(c), conv=1e-11, thrs=0.0)["energy"])
        fd = (e[0] - e[1]) / (2 * h)
        assert abs(fd - g[atom, k]) < 2e-7
