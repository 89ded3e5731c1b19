"""The two-electron working basis (general contractions resolved into
primitives) behind the C ABI: batched builds over general-contraction bases,
the AO-basis quartet count, shared kernel tuning."""
import numpy as np
import pytest

from dalton_b200 import molecules
from dalton_b200.basis import build_basis
from dalton_b200.fock import FockBuilder

pytestmark = pytest.mark.gpu


def rdens(n, seed):
    rng = np.random.default_rng(seed)
    a = rng.normal(size=(n, n)) * 0.05
    return a + a.T + np.eye(n) * 0.3


def test_batched_general_contraction_matches_per_molecule_and_oracle(cuda, orc):
    """cc-pVDZ blocks are general contractions: the packed AO <-> working maps
    of a batch must reproduce each molecule's own build and the oracle."""
    import torch

    from dalton_b200.batch import BatchBuilder

    mols = molecules.water_batch(5, 1, 3, seed=21)
    bss = [build_basis(m, "cc-pVDZ") for m in mols]
    fbs = [FockBuilder(bs) for bs in bss]
    ds = [torch.tensor(rdens(fb.nbf, 40 + k), device=cuda) for k, fb in enumerate(fbs)]
    ref = [fb.herfck_device(d).clone() for fb, d in zip(fbs, ds)]
    bb = BatchBuilder(fbs)
    dp = bb.pack(ds)
    for use_graph in (False, True):
        fp = bb.herfck_batch(dp, use_graph=use_graph)
        for a, b in zip(bb.unpack(fp), ref):
            assert float(torch.max(torch.abs(a - b))) < 1e-12
    k = 0
    fo = orc.fock(bss[k], ds[k].cpu().numpy(), 13, 1.0, 1e-12)
    assert np.abs(ref[k].cpu().numpy() - fo).max() < 1e-10


def test_ao_quartet_count_matches_oracle(cuda, orc):
    """dgf_count_ao_quartets counts the oracle's segmented-shell quartets
    (Schwarz factors computed independently on both sides; equal up to
    quartets whose Q_AB Q_CD sits within rounding of the threshold)."""
    bs = build_basis(molecules.water_cluster(2, seed=3), "cc-pVDZ")
    fb = FockBuilder(bs)
    d = rdens(bs.nbf, 5)
    _, nq_oracle = orc.fock_sampled(bs, d, 1, 0, 1e-12)
    nq = fb.ao_quartets(1e-12)
    assert abs(nq - nq_oracle) <= max(2, nq_oracle // 10000), (nq, nq_oracle)
    # the working basis resolves general contractions: more (single-primitive) quartets
    fb.herfck(d)
    assert fb.last_stats["quartets_total"] > nq


def test_copy_tuning_keeps_results(cuda):
    import torch

    bs = build_basis(molecules.water_cluster(2, seed=6), "cc-pVDZ")
    fa, fbb = FockBuilder(bs), FockBuilder(bs)
    d = torch.tensor(rdens(bs.nbf, 8), device=cuda)
    before = fbb.herfck_device(d).clone()
    fa.autotune(d, mixed_cutoff=1e-6)
    fbb.copy_tuning_from(fa)
    after = fbb.herfck_device(d)
    assert float(torch.max(torch.abs(after - before))) < 1e-12
