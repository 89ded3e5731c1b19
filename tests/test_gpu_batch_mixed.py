"""The warp-per-quartet kernel on contracted (multi-primitive) pairs, and the
batched build with the warp kernel and with the mixed form, through the C
ABI.  6-31G* has contracted s/sp shells (3 and 6 primitives) and
uncontracted d shells, so its d-containing classes mix one- and
multi-primitive pairs."""
import numpy as np
import pytest

from dalton_b200 import molecules
from dalton_b200.basis import build_basis
from dalton_b200.fock import FockBuilder

pytestmark = pytest.mark.gpu

# classes whose warp kernel loops over primitive pairs, with L >= 4
MP_CLASSES = [(2, 1, 1, 0), (2, 1, 1, 1), (1, 1, 1, 1), (2, 2, 2, 0), (2, 2, 0, 0), (2, 1, 2, 0), (2, 1, 2, 1)]


def _density(n, seed, scale=0.05):
    rng = np.random.default_rng(seed)
    d = rng.normal(size=(n, n)) * scale
    return d + d.T


@pytest.fixture(scope="module")
def pair631(cuda, orc):
    bs = build_basis(molecules.water_cluster(2, seed=5), "6-31G*")
    d = _density(bs.nbf, 3)
    return bs, d, orc.fock(bs, d, 13, 1.0, 1e-12)


@pytest.mark.parametrize("precision", [64, 32])
def test_warp_kernel_primitive_loops_match_oracle(pair631, precision):
    bs, d, ref = pair631
    fb = FockBuilder(bs)
    for cls in MP_CLASSES:
        fb.set_class_kernel(cls, -3, precision=precision)
    if precision == 64:
        f = fb.herfck(d, 13)
        err = np.abs(f - ref).max()
        assert err < 1e-10, f"max |dF| {err:.2e}"
    else:
        # every class that splits runs its small quartets in the FP32 warp kernel
        f = fb.herfck(d, 13, mixed_cutoff=1e3)
        assert fb.last_stats["quartets_fp32"] > 0
        err = np.abs(f - ref).max()
        assert err < 1e-5, f"max |dF| {err:.2e}"


def test_set_class_kernel_rejects_missing_variants(cuda):
    from dalton_b200 import _lib

    fb = FockBuilder(build_basis(molecules.water_dalton_test(), "6-31G*"))
    with pytest.raises(_lib.DgfError):
        fb.set_class_kernel((1, 0, 0, 0), -3)  # L = 1: no warp kernel
    with pytest.raises(_lib.DgfError):
        fb.set_class_kernel((1, 2, 0, 0), 0)   # la < lb


def _batch(cuda, nmol=6, seed=11):
    import torch

    mols = molecules.water_batch(nmol, 1, 4, seed=seed)
    fbs = [FockBuilder(build_basis(m, "6-31G*")) for m in mols]
    ds = [torch.tensor(_density(fb.nbf, 50 + k, scale=0.02), device=cuda) for k, fb in enumerate(fbs)]
    big = max(range(len(fbs)), key=lambda k: fbs[k].nbf)
    return fbs, ds, big


def test_batch_with_warp_kernels_matches_per_molecule(cuda):
    import torch

    from dalton_b200.batch import BatchBuilder

    fbs, ds, big = _batch(cuda)
    for cls in MP_CLASSES:
        fbs[big].set_class_kernel(cls, -3)
    for fb in fbs:
        fb.copy_tuning_from(fbs[big])
    ref = [fb.herfck_device(d).clone() for fb, d in zip(fbs, ds)]
    bb = BatchBuilder(fbs)
    dp = bb.pack(ds)
    for use_graph in (False, True, True):
        fp = bb.herfck_batch(dp, use_graph=use_graph)
        for a, b in zip(bb.unpack(fp), ref):
            assert float(torch.max(torch.abs(a - b))) < 1e-11


def test_batch_mixed_form(cuda):
    """Mixed batch: the tuned context's split classes run their small
    quartets in FP32; F within 1e-6 of the FP64 per-molecule builds, and the
    graph replays it."""
    import torch

    from dalton_b200.batch import BatchBuilder

    fbs, ds, big = _batch(cuda, nmol=8, seed=12)
    fbs[big].autotune(ds[big], mixed_cutoff=1e-6)
    ref = [fb.herfck_device(d).clone() for fb, d in zip(fbs, ds)]
    bb = BatchBuilder(fbs)
    dp = bb.pack(ds)
    f64 = bb.unpack(bb.herfck_batch(dp, use_graph=False).clone())
    for a, b in zip(f64, ref):
        assert float(torch.max(torch.abs(a - b))) < 1e-11
    for use_graph in (False, True, True):
        fp = bb.herfck_batch(dp, use_graph=use_graph, mixed_cutoff=1e-6)
        st = bb.last_stats
        err = max(float(torch.max(torch.abs(a - b))) for a, b in zip(bb.unpack(fp), ref))
        de = max(abs(0.5 * float(torch.sum(d * (a - b)))) for d, a, b in zip(ds, bb.unpack(fp), ref))
        print(f"mixed batch: max |dF| {err:.2e}, max |dE| {de:.2e}, FP32 quartets {st['quartets_fp32']}")
        assert err < 1e-6 and de < 1e-6
    # the FP64 form is unchanged after mixed calls (a separate graph)
    fp = bb.herfck_batch(dp, use_graph=True)
    for a, b in zip(bb.unpack(fp), ref):
        assert float(torch.max(torch.abs(a - b))) < 1e-11


def _pin_all(fb, variant, precision=64):
    """Pin `variant` on every class (L >= 4) that has it; returns the classes."""
    from dalton_b200 import _lib

    pinned = []
    for la in range(4):
        for lb in range(la + 1):
            for lc in range(4):
                for ld in range(lc + 1):
                    if la + lb + lc + ld < 4 or (la * (la + 1) // 2 + lb) < (lc * (lc + 1) // 2 + ld):
                        continue
                    try:
                        fb.set_class_kernel((la, lb, lc, ld), variant, precision=precision)
                        pinned.append((la, lb, lc, ld))
                    except _lib.DgfError:
                        pass
    return pinned


def _methane():
    from dalton_b200.basis import Molecule

    r = 0.63
    return Molecule.from_angstrom(["C", "H", "H", "H", "H"],
                                  [[0, 0, 0], [r, r, r], [-r, -r, r], [-r, r, -r], [r, -r, -r]])


def test_tensor_core_transforms_f_shells(cuda, orc):
    """The DMMA form of the warp kernel (FP64 tensor cores for the ket and
    bra Hermite contractions) on every class that has it, CH4 / cc-pVTZ
    (single-primitive pairs up to f), against the oracle."""
    bs = build_basis(_methane(), "cc-pVTZ")
    d = _density(bs.nbf, 17)
    fb = FockBuilder(bs)
    pinned = _pin_all(fb, -4)
    assert (2, 1, 2, 1) in pinned and (3, 0, 3, 0) in pinned
    f = fb.herfck(d, 13)
    err = np.abs(f - orc.fock(bs, d, 13, 1.0, 1e-12)).max()
    print(f"DMMA on {len(pinned)} classes: max |dF| {err:.2e}")
    assert err < 1e-10


def test_tensor_core_transforms_contracted_pairs(pair631):
    """The DMMA form loops over the primitive pairs of 6-31G*'s contracted
    shells, against the oracle."""
    bs, d, ref = pair631
    fb = FockBuilder(bs)
    assert len(_pin_all(fb, -4)) > 0
    f = fb.herfck(d, 13)
    assert np.abs(f - ref).max() < 1e-10
