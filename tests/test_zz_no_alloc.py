"""The Fock build that allocates no device memory, checked against the
regular device entry point through the C ABI.

Some callers cannot allocate GPU memory when they need a Fock matrix: a
host that hands the engine one fixed work area (as Dalton does with
WORK/LWORK), or a process whose device memory belongs to another pool.  They
call dgf_fock_device_noalloc, whose scratch is a fixed array inside the
library.  This file is named so that pytest collects it last."""
import ctypes

import numpy as np
import pytest

from dalton_b200 import _lib, molecules
from dalton_b200.basis import build_basis
from dalton_b200.fock import FockBuilder

pytestmark = pytest.mark.gpu

TOL = 1e-10  # the FP64 parity tolerance of the other Fock tests


def _noalloc(fb, d, f, hfxfac=1.0, thrs=1e-12):
    import torch

    fn = fb._lib.dgf_fock_device_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_double,
                   ctypes.c_void_p]
    fn.restype = ctypes.c_int
    stream = torch.cuda.current_stream(d.device).cuda_stream
    return fn(fb._h, ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(f.data_ptr()), float(hfxfac), float(thrs),
              ctypes.c_void_p(stream))


def _density(n, seed, device):
    import torch

    rng = np.random.default_rng(seed)
    d = rng.normal(size=(n, n)) * 0.1
    return torch.tensor(d + d.T, device=device)


def test_noalloc_matches_regular_build_on_two_calls(cuda):
    import torch

    bs = build_basis(molecules.water_cluster(4, (2, 2, 1), seed=1), "cc-pVDZ")
    fb = FockBuilder(bs)
    ds = [_density(bs.nbf, 31, cuda), _density(bs.nbf, 32, cuda)]
    refs = [fb.herfck_device(d).clone() for d in ds]  # also builds the plan for thrs = 1e-12
    out = torch.full_like(ds[0], float("nan"))
    # two calls in a row with different densities: the second must not see the first's scratch
    for d, ref in zip(ds, refs):
        assert _noalloc(fb, d, out) == _lib.DGF_OK, _lib.last_error()
        torch.cuda.synchronize()
        assert float(torch.max(torch.abs(out - ref))) < TOL


def test_noalloc_rejects_oversized_and_unplanned(cuda):
    import torch

    big = FockBuilder(build_basis(molecules.water_cluster(33, (4, 4, 3), seed=5), "cc-pVDZ"))
    assert big.nbf > 768
    d = torch.zeros((big.nbf, big.nbf), dtype=torch.float64, device=cuda)
    f = torch.empty_like(d)
    assert _noalloc(big, d, f) == _lib.DGF_ERR_ARG
    assert "768" in _lib.last_error()
    small = FockBuilder(build_basis(molecules.water_dalton_test(), "cc-pVDZ"))
    d = _density(small.nbf, 3, cuda)
    f = torch.empty_like(d)
    assert _noalloc(small, d, f, thrs=1e-12) == _lib.DGF_ERR_ARG  # no plan for this threshold yet


@pytest.mark.parametrize("hfxfac", [1.0, 0.25, 0.0])
def test_noalloc_hfxfac(cuda, hfxfac):
    """The exchange scale: full exchange, a hybrid fraction and J only, each
    against the regular device build with the same HFXFAC."""
    import torch

    bs = build_basis(molecules.water_cluster(2, seed=4), "cc-pVDZ")
    fb = FockBuilder(bs)
    d = _density(bs.nbf, 41, cuda)
    ref = fb.herfck_device(d, hfxfac=hfxfac).clone()
    out = torch.full_like(d, float("nan"))
    assert _noalloc(fb, d, out, hfxfac=hfxfac) == _lib.DGF_OK, _lib.last_error()
    torch.cuda.synchronize()
    assert float(torch.max(torch.abs(out - ref))) < TOL


@pytest.mark.parametrize("planner", ["autotune", "grad2e"])
def test_noalloc_uses_plan_of_autotune_or_gradient(cuda, planner):
    """A quartet plan made by the autotuner or by the gradient (not by a Fock
    build) serves the no-allocation call; the autotuner's kernel choices apply."""
    import torch

    bs = build_basis(molecules.water_cluster(2, seed=6), "cc-pVDZ")
    fb = FockBuilder(bs)
    d = _density(bs.nbf, 43, cuda)
    if planner == "autotune":
        fb.autotune(d)
    else:
        fb.grad2e(d.cpu().numpy())
    out = torch.full_like(d, float("nan"))
    assert _noalloc(fb, d, out) == _lib.DGF_OK, _lib.last_error()
    torch.cuda.synchronize()
    ref = fb.herfck_device(d)
    assert float(torch.max(torch.abs(out - ref))) < TOL
