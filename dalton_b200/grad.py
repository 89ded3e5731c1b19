"""Differentiable Fock build and the RHF nuclear gradient.

``FockJK.apply(D, coords, builder)`` returns G = J[D] - hfx/2 K[D]
(IFCTYP 13) on the device.  Its backward pass recomputes integrals instead
of storing them:

* w.r.t. the density: the build is self-adjoint (<X, G(D)> = <D, G(X)> for
  symmetric X), so dL/dD = G(sym(dL/dG)) -- one more J/K build of the
  cotangent;
* w.r.t. the nuclear coordinates: d<C, G(D)>/dR = 2 K(C, D), where K is the
  bilinear derivative-integral contraction of ``dgf_grad2e_bilinear_device``
  (K(D, D) is the two-electron part of the HF gradient, Dalton's
  TWOEXP/INTEX1, DALTON/abacus/aba2tex.F:242, her2ave.F:91-830).

``rhf_gradient`` assembles the full RHF nuclear gradient
sum D dh - sum W dS + dVnn + K(D, D) from the library's one- and
two-electron parts (the one-electron part as Dalton's HER1 derivative
integrals, the two-electron part through the backward kernel).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .fock import FockBuilder


def grad2e_bilinear(fb: FockBuilder, d1, d2, hfxfac=1.0, thrs=1e-12):
    """K(D1, D2) on the device: (natom, 3) tensor."""
    import torch

    out = torch.empty((fb.natom, 3), dtype=torch.float64, device=d1.device)
    stream = torch.cuda.current_stream(d1.device).cuda_stream
    a, b = d1.contiguous(), d2.contiguous()
    _lib.check(fb._lib.dgf_grad2e_bilinear_device(fb._h, ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(b.data_ptr()),
                                                  float(hfxfac), float(thrs), ctypes.c_void_p(out.data_ptr()),
                                                  ctypes.c_void_p(stream)), "dgf_grad2e_bilinear_device")
    return out


class FockJK:
    """torch.autograd.Function wrapper (built lazily so importing needs no torch)."""

    _fn = None

    @classmethod
    def apply(cls, D, coords, builder: FockBuilder, hfxfac: float = 1.0, thrs: float = 1e-12,
              mixed_cutoff: float = 0.0):
        if cls._fn is None:
            cls._fn = _make_function()
        return cls._fn.apply(D, coords, builder, hfxfac, thrs, mixed_cutoff)


def _make_function():
    import torch

    class _FockJK(torch.autograd.Function):
        @staticmethod
        def forward(ctx, D, coords, builder, hfxfac, thrs, mixed_cutoff):
            ctx.builder, ctx.hfx, ctx.thrs = builder, hfxfac, thrs
            G = builder.herfck_device(D.detach().contiguous(), ifctyp=13, hfxfac=hfxfac, thrs=thrs,
                                      mixed_cutoff=mixed_cutoff)
            ctx.save_for_backward(D)
            return G

        @staticmethod
        def backward(ctx, gbar):
            (D,) = ctx.saved_tensors
            fb = ctx.builder
            C = (0.5 * (gbar + gbar.T)).contiguous()
            dD = dR = None
            if ctx.needs_input_grad[0]:
                dD = fb.herfck_device(C, ifctyp=13, hfxfac=ctx.hfx, thrs=ctx.thrs)
            if ctx.needs_input_grad[1]:
                dR = 2.0 * grad2e_bilinear(fb, C, D.detach().contiguous(), ctx.hfx, ctx.thrs)
            return dD, dR, None, None, None, None

    return _FockJK


def rhf_gradient(fb: FockBuilder, dmat, wmat, hfxfac=1.0, thrs=1e-12, use_autograd=True):
    """Full RHF nuclear gradient (natom, 3) as numpy: one-electron + nuclear
    repulsion from the library, two-electron through the backward kernel."""
    import torch

    D = dmat if hasattr(dmat, "device") else torch.tensor(dmat, device="cuda")
    W = wmat.detach().cpu().numpy() if hasattr(wmat, "device") else np.asarray(wmat)
    g1 = fb.grad1e(D.detach().cpu().numpy(), W)
    if use_autograd:
        coords = torch.tensor(fb.basis.molecule.coords, dtype=torch.float64, device=D.device, requires_grad=True)
        G = FockJK.apply(D, coords, fb, hfxfac, thrs)
        e2 = 0.5 * torch.sum(D * G)
        (g2,) = torch.autograd.grad(e2, coords)
    else:
        g2 = grad2e_bilinear(fb, D, D, hfxfac, thrs)
    return g1 + g2.detach().cpu().numpy()
