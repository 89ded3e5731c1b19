"""GPU checks beyond the Fock parity: one-electron integrals and gradient,
the SCF energy against Dalton's golden value, the mixed form's accuracy,
quartet-queue shards, the device-pointer entry point, determinism and a
host-injected allocation failure."""
import os
import subprocess
import sys

import numpy as np
import pytest

from dalton_b200 import _lib, molecules
from dalton_b200.basis import build_basis
from dalton_b200.fock import FockBuilder

pytestmark = pytest.mark.gpu


def rdens(n, seed):
    rng = np.random.default_rng(seed)
    d = rng.normal(size=(n, n)) * 0.1
    return d + d.T


@pytest.mark.parametrize("basis", ["cc-pVDZ", "cc-pVTZ", "6-31G*"])
def test_oneint_matches_oracle(cuda, orc, basis):
    bs = build_basis(molecules.water_cluster(2, seed=2), basis)
    fb = FockBuilder(bs)
    got = fb.oneint()
    ref = orc.oneint(bs)
    for g, r in zip(got, ref):
        assert np.abs(g - r).max() < 1e-11


def test_grad1e_matches_oracle(cuda, orc):
    bs = build_basis(molecules.acrolein(), "STO-3G")
    r = orc.rhf(bs)
    fb = FockBuilder(bs)
    g = fb.grad1e(r["dmat"], r["wmat"])
    ref = orc.grad1e(bs, r["dmat"], r["wmat"])
    assert np.abs(g - ref).max() < 1e-11


def test_scf_energy_dalton_golden(cuda):
    import json

    from dalton_b200.scf import rhf

    with open(os.path.join(os.path.dirname(__file__), "golden", "dalton_energies.json")) as f:
        gold = json.load(f)["energy_direct"]["energy"]
    bs = build_basis(molecules.water_dalton_test(), "cc-pVDZ")
    res = rhf(bs, conv=1e-10, incremental=False)
    assert abs(res["energy"] - gold) < 1e-9
    res2 = rhf(bs, conv=1e-10, incremental=True)
    assert abs(res2["energy"] - gold) < 1e-9


def test_mixed_precision_accuracy(cuda, orc):
    import torch

    from dalton_b200.scf import rhf

    bs = build_basis(molecules.water_cluster(4, (2, 2, 1), seed=1), "cc-pVDZ")
    res = rhf(bs, conv=1e-9)
    fb = res["builder"]
    D = res["dmat"]
    f64 = fb.herfck_device(D)
    q64 = fb.last_stats
    fmx = fb.herfck_device(D, mixed_cutoff=1e-6)
    st = fb.last_stats
    assert st["quartets_fp32"] > 0 and st["quartets_fp64"] + st["quartets_fp32"] == q64["quartets_total"]
    dE = 0.5 * float(torch.sum(D * (fmx - f64)))
    assert abs(dE) < 1e-6
    assert float(torch.max(torch.abs(fmx - f64))) < 1e-5
    ref = orc.fock(bs, D.cpu().numpy(), 13, 1.0, 1e-12)
    assert np.abs(f64.cpu().numpy() - ref).max() < 1e-10


def test_ifthrs_schedule_scf_energy(cuda):
    """Dalton's direct-SCF screening schedule (loose while the orbital
    gradient is large, tight near convergence) with incremental and mixed
    builds reaches the energy of plain full FP64 builds."""
    from dalton_b200.scf import rhf

    bs = build_basis(molecules.water_cluster(4, (2, 2, 1), seed=1), "cc-pVDZ")
    ref = rhf(bs, conv=1e-8, incremental=False)
    fb = ref["builder"]
    sch = rhf(bs, fb, conv=1e-8, ifthrs_schedule=True)
    mix = rhf(bs, fb, conv=1e-8, ifthrs_schedule=True, mixed_cutoff=1e-6)
    assert abs(sch["energy"] - ref["energy"]) < 1e-8
    assert abs(mix["energy"] - ref["energy"]) < 1e-7
    assert min(sch["ifthrs"]) < max(sch["ifthrs"]) <= 20  # the threshold tightened along the way


def test_shards_sum_to_full(cuda):
    bs = build_basis(molecules.water_cluster(4, (2, 2, 1), seed=1), "cc-pVDZ")
    fb = FockBuilder(bs)
    d = rdens(bs.nbf, 3)
    full = fb.herfck(d)
    parts = [fb.herfck(d, shard=(k, 3)) for k in range(3)]
    assert np.abs(sum(parts) - full).max() < 1e-12


def test_device_entry_point_and_determinism(cuda):
    import torch

    bs = build_basis(molecules.water_cluster(2, seed=9), "cc-pVDZ")
    fb = FockBuilder(bs)
    d = rdens(bs.nbf, 4)
    fh = fb.herfck(d)
    fd = fb.herfck_device(torch.tensor(d, device=cuda)).cpu().numpy()
    fd2 = fb.herfck_device(torch.tensor(d, device=cuda)).cpu().numpy()
    assert np.abs(fh - fd).max() < 1e-13
    assert np.abs(fd - fd2).max() < 1e-13  # FP64 atomics: order only


def test_density_screening_ifthrs(cuda, orc):
    bs = build_basis(molecules.water_cluster(4, (2, 2, 1), seed=1), "cc-pVDZ")
    fb = FockBuilder(bs)
    d = rdens(bs.nbf, 5) * 1e-3
    full = fb.herfck(d)
    scr = fb.herfck(d, ifthrs=10)
    st = fb.last_stats
    assert st["quartets_skipped"] > 0
    assert np.abs(scr - full).max() < 1e-7


def test_alloc_fault_injection_reports_nomem(cuda):
    code = ("import sys; sys.path.insert(0, %r)\n"
            "from dalton_b200 import molecules, _lib\n"
            "from dalton_b200.basis import build_basis\n"
            "from dalton_b200.fock import FockBuilder\n"
            "try:\n"
            "    FockBuilder(build_basis(molecules.water_dalton_test(), 'STO-3G'))\n"
            "    print('NO ERROR')\n"
            "except _lib.DgfError as e:\n"
            "    print('STATUS', e.status)\n") % os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, DGF_FAULT_INJECT="alloc")
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert f"STATUS {_lib.DGF_ERR_NOMEM}" in out.stdout, out.stdout + out.stderr


def test_batched_build_matches_per_molecule(cuda):
    import torch

    from dalton_b200.batch import BatchBuilder

    mols = molecules.water_batch(6, 1, 4, seed=11)
    fbs = [FockBuilder(build_basis(m, "6-31G*")) for m in mols]
    ds = [torch.tensor(rdens(fb.nbf, 20 + k), device=cuda) for k, fb in enumerate(fbs)]
    ref = [fb.herfck_device(d).clone() for fb, d in zip(fbs, ds)]
    nq = sum(fb.herfck_device(d) is not None and fb.last_stats["quartets_total"] for fb, d in zip(fbs, ds))
    bb = BatchBuilder(fbs)
    dp = bb.pack(ds)
    for use_graph in (False, True, True):
        fp = bb.herfck_batch(dp, use_graph=use_graph)
        for a, b in zip(bb.unpack(fp), ref):
            assert float(torch.max(torch.abs(a - b))) < 1e-12
        assert bb.last_stats["quartets_total"] == nq
