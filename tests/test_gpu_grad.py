"""Backward kernel (two-electron gradient) and the autograd harness against
the oracle, Dalton's acrolein golden gradient and finite differences."""
import json
import os

import numpy as np
import pytest

from dalton_b200 import molecules
from dalton_b200.basis import build_basis
from dalton_b200.fock import FockBuilder

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mol,basis", [("h2o", "cc-pVDZ"), ("acrolein", "STO-3G"), ("w2", "6-31G*")])
def test_grad2e_matches_oracle(cuda, orc, mol, basis):
    m = {"h2o": molecules.water_dalton_test, "acrolein": molecules.acrolein,
         "w2": lambda: molecules.water_cluster(2, seed=4)}[mol]()
    bs = build_basis(m, basis)
    r = orc.rhf(bs)
    fb = FockBuilder(bs)
    g = fb.grad2e(r["dmat"], 1.0, 1e-12)
    ref = orc.grad2e(bs, r["dmat"], 1.0, 1e-12)
    assert np.abs(g - ref).max() < 1e-9


def test_bilinear_symmetry_and_autograd_density(cuda):
    import torch

    from dalton_b200.grad import FockJK, grad2e_bilinear

    bs = build_basis(molecules.water_cluster(2, seed=1), "cc-pVDZ")
    fb = FockBuilder(bs)
    rng = np.random.default_rng(0)
    d1 = rng.normal(size=(bs.nbf, bs.nbf)) * 0.1
    d2 = rng.normal(size=(bs.nbf, bs.nbf)) * 0.1
    d1, d2 = torch.tensor(d1 + d1.T, device=cuda), torch.tensor(d2 + d2.T, device=cuda)
    k12 = grad2e_bilinear(fb, d1, d2)
    k21 = grad2e_bilinear(fb, d2, d1)
    assert float(torch.max(torch.abs(k12 - k21))) < 1e-11
    kdd = grad2e_bilinear(fb, d1, d1).cpu().numpy()
    assert np.abs(kdd - fb.grad2e(d1.cpu().numpy())).max() < 1e-11
    D = d1.clone().requires_grad_(True)
    X = d2
    coords = torch.tensor(bs.molecule.coords, device=cuda)
    L = torch.sum(X * FockJK.apply(D, coords, fb))
    (gD,) = torch.autograd.grad(L, D)
    assert float(torch.max(torch.abs(gD - fb.herfck_device(X)))) < 1e-12


def test_rhf_gradient_acrolein_dalton_golden(cuda):
    from dalton_b200.grad import rhf_gradient
    from dalton_b200.scf import rhf

    with open(os.path.join(os.path.dirname(__file__), "golden", "dalton_energies.json")) as f:
        gold = json.load(f)["preopt_acrolein"]
    bs = build_basis(molecules.acrolein(), "STO-3G")
    res = rhf(bs, conv=1e-10)
    assert abs(res["energy"] - gold["energy"]) < 1e-9
    g = rhf_gradient(res["builder"], res["dmat"], res["wmat"])
    assert np.abs(g - np.array(gold["gradient"])).max() < 1e-6
    assert np.abs(g.sum(0)).max() < 1e-10


def test_autograd_coords_finite_difference(cuda):
    import torch

    from dalton_b200.grad import FockJK

    bs = build_basis(molecules.water_cluster(2, seed=7), "cc-pVDZ")
    rng = np.random.default_rng(3)
    d = rng.normal(size=(bs.nbf, bs.nbf)) * 0.05
    D = torch.tensor(d + d.T, device=cuda)

    def energy(coords_np):
        fb = FockBuilder(bs.with_coords(coords_np))
        return 0.5 * float(torch.sum(D * fb.herfck_device(D, thrs=0.0)))

    fb = FockBuilder(bs)
    coords = torch.tensor(bs.molecule.coords, device=cuda, requires_grad=True)
    e2 = 0.5 * torch.sum(D * FockJK.apply(D, coords, fb, 1.0, 0.0))
    (g,) = torch.autograd.grad(e2, coords)
    g = g.cpu().numpy()
    h = 1e-4
    for atom, k in ((0, 0), (1, 1), (4, 2)):
        c = bs.molecule.coords.copy()
        c[atom, k] += h
        ep = energy(c)
        c[atom, k] -= 2 * h
        em = energy(c)
        assert abs((ep - em) / (2 * h) - g[atom, k]) < 1e-7
