"""CPU-side checks: the C-ABI library loads and exports every symbol its
header declares, error paths without a device, host-side basis/molecule
logic, the FLOP model, and the shard-and-sum pattern across 2 gloo ranks."""
import os
import re

import numpy as np
import pytest

from dalton_b200 import _lib, molecules, perfmodel
from dalton_b200.basis import XTANG, build_basis, cart_exponents, nrmorb, sph_transform

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    with open(os.path.join(ROOT, "include", "dgfock.h")) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dgf_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = header_functions()
    assert len(names) >= 10
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(_lib.EXPORTS) == names


def test_strerror_and_options():
    assert _lib.strerror(0) == "success"
    assert "argument" in _lib.strerror(1)
    o = _lib.default_options()
    assert o.thrs == 1e-12 and o.ifthrs == 20 and o.hfxfac == 1.0 and o.mixed_cutoff == 0.0
    assert o.shard_index == 0 and o.shard_count == 1


def test_create_fails_cleanly_without_device():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    from dalton_b200.fock import FockBuilder

    with pytest.raises(_lib.DgfError) as ei:
        FockBuilder(build_basis(molecules.water_dalton_test(), "STO-3G"))
    assert ei.value.status == _lib.DGF_ERR_NODEVICE


def test_null_arguments_rejected():
    import ctypes

    lib = _lib.load()
    h = ctypes.c_void_p()
    assert lib.dgf_create(None, 0, ctypes.byref(h)) == _lib.DGF_ERR_ARG
    assert lib.dgf_fock(None, 1, None, None, None, None, None) == _lib.DGF_ERR_ARG
    assert lib.dgf_info(None, None, None, None) == _lib.DGF_ERR_ARG
    assert "NULL" in _lib.last_error() or "null" in _lib.last_error()


def test_basis_counts_and_order():
    counts = {"h2o4_ccpvdz": 96, "h2o32_ccpvdz": 768, "h2o16_ccpvdz": 384, "c20h42_ccpvtz": 1188}
    for name, nbf in counts.items():
        mol, bas = molecules.config(name)
        assert build_basis(mol, bas).nbf == nbf
    bs = build_basis(molecules.water_dalton_test(), "cc-pVDZ")
    # Dalton C1 order: O 1s 1s 1s 2p(x,y,z) x2 3d(5), H1 1s 1s 2p, H2 ...
    assert list(bs.block_l) == [0, 1, 2, 0, 1, 0, 1]
    assert list(bs.block_ao_offset) == [0, 3, 9, 14, 16, 19, 21]
    assert cart_exponents(2) == [(2, 0, 0), (1, 1, 0), (1, 0, 1), (0, 2, 0), (0, 1, 1), (0, 0, 2)]


def test_nrmorb_single_primitive_norm():
    # one primitive: coefficient (4a)^(l/2+3/4) (2 pi)^(-3/4), the x^l norm
    for l in range(4):
        c = nrmorb(l, np.array([0.7]), np.array([[1.0]]))
        assert abs(c[0, 0] - (4 * 0.7) ** (0.5 * l + 0.75) * (2 * np.pi) ** -0.75) < 1e-14


def test_sph_transform_matches_oracle(orc):
    for l in (2, 3):
        assert np.abs(sph_transform(l) - orc.sph_matrix(l)).max() < 1e-15
    t = sph_transform(2)
    assert abs(t[4, 0] - 0.5) < 1e-15 and abs(t[4, 3] + 0.5) < 1e-15  # d2+ = (xx - yy)/2


def test_water_cluster_geometry():
    mol = molecules.water_cluster(8, (2, 2, 2), seed=3)
    xyz = mol.coords * XTANG
    for k in range(8):
        o, h1, h2 = xyz[3 * k: 3 * k + 3]
        assert abs(np.linalg.norm(h1 - o) - 0.96) < 1e-12
        assert abs(np.linalg.norm(h2 - o) - 0.96) < 1e-12
        cosang = np.dot(h1 - o, h2 - o) / 0.96 ** 2
        assert abs(np.degrees(np.arccos(cosang)) - 104.5) < 1e-9


def test_alkane_geometry():
    mol = molecules.alkane(20, seed=0, jitter=0.0)
    assert mol.natom == 62 and mol.symbols.count("H") == 42
    xyz = mol.coords * XTANG
    c = xyz[:20]
    assert np.allclose(np.linalg.norm(np.diff(c, axis=0), axis=1), 1.54)
    d = np.linalg.norm(xyz[:, None] - xyz[None], axis=-1) + np.eye(62) * 9
    assert d.min() > 1.08


def test_flop_model_monotone():
    assert perfmodel.flops_per_primitive(0, 0, 0, 0) == 44  # Boys 40 + ket 2 + bra 2
    assert perfmodel.flops_per_primitive(2, 2, 2, 2) > perfmodel.flops_per_primitive(1, 1, 1, 1)
    assert perfmodel.flops_per_contracted(0, 0, 0, 0) == 12


def _gloo_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import sys

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import orc

    orc.set_threads(1)
    bs = build_basis(molecules.water_cluster(2, seed=5), "STO-3G")
    rng = np.random.default_rng(0)
    d = rng.normal(size=(bs.nbf, bs.nbf))
    d = d + d.T
    part, nq = orc.fock_sampled(bs, d, world, rank)
    t = torch.from_numpy(part)
    dist.all_reduce(t)
    if rank == 0:
        full = orc.fock(bs, d, 13, 1.0, 1e-12)
        q.put(float(np.abs(t.numpy() - full).max()))
    dist.barrier()
    dist.destroy_process_group()


def test_shard_partial_fock_allreduce_gloo(orc):
    import socket

    import torch.multiprocessing as mp

    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    assert all(p.exitcode == 0 for p in procs)
    assert q.get(timeout=10) < 1e-12
