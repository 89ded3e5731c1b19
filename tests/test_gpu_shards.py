"""The product's quartet-queue shards across processes: two ranks (gloo on
the host, both on cuda:0, no peer memory) each build the partial Fock
matrix of their cost-weighted shard through the C ABI and sum them with an
all-reduce, as bench.py's multi-GPU path does with NCCL."""
import datetime
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, dmat, out_path):
    import sys

    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist

    from dalton_b200 import molecules
    from dalton_b200.basis import build_basis
    from dalton_b200.fock import FockBuilder

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        bs = build_basis(molecules.water_cluster(4, (2, 2, 1), seed=1), "cc-pVDZ")
        fb = FockBuilder(bs, device=0)
        part = fb.herfck(dmat, 13, shard=(rank, world))
        quartets = torch.tensor([fb.last_stats["quartets_total"]], dtype=torch.int64)
        t = torch.from_numpy(part.copy())
        dist.all_reduce(t)
        dist.all_reduce(quartets)
        if rank == 0:
            np.save(out_path, t.numpy())
            np.save(out_path + ".q.npy", quartets.numpy())
        fb.close()
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_process_shards_match_oracle(cuda, orc, tmp_path):
    import torch.multiprocessing as mp

    from dalton_b200 import molecules
    from dalton_b200.basis import build_basis
    from dalton_b200.fock import FockBuilder

    bs = build_basis(molecules.water_cluster(4, (2, 2, 1), seed=1), "cc-pVDZ")
    rng = np.random.default_rng(31)
    d = rng.normal(size=(bs.nbf, bs.nbf)) * 0.1
    d = d + d.T
    out = str(tmp_path / "f.npy")
    mp.spawn(_rank_main, args=(2, _free_port(), d, out), nprocs=2, join=True)
    f = np.load(out)
    ref = orc.fock(bs, d, 13, 1.0, 1e-12)
    assert np.abs(f - ref).max() < 1e-10
    fb = FockBuilder(bs)
    fb.herfck(d, 13)
    assert int(np.load(out + ".q.npy")[0]) == fb.last_stats["quartets_total"]  # the shards tile the queue


@pytest.mark.parametrize("n", [2, 3, 5, 8])
def test_cost_weighted_shards_tile_the_queue(cuda, n):
    """Every quartet in exactly one shard: shard sums equal the full build and
    the shards' quartet counts add up to the full count; the shards' model
    costs are balanced, so no shard is empty for small n."""
    from dalton_b200 import molecules
    from dalton_b200.basis import build_basis
    from dalton_b200.fock import FockBuilder

    bs = build_basis(molecules.water_cluster(4, (2, 2, 1), seed=1), "cc-pVDZ")
    fb = FockBuilder(bs)
    rng = np.random.default_rng(5)
    d = rng.normal(size=(bs.nbf, bs.nbf)) * 0.1
    d = d + d.T
    full = fb.herfck(d)
    nq = fb.last_stats["quartets_total"]
    parts, counts = [], []
    for r in range(n):
        parts.append(fb.herfck(d, shard=(r, n)))
        counts.append(fb.last_stats["quartets_total"])
    assert sum(counts) == nq
    assert min(counts) > 0
    assert np.abs(sum(parts) - full).max() < 1e-12
