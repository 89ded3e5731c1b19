"""Batched Fock builds of many molecules (one launch per quartet class over
the merged queue, optionally replayed as a CUDA graph)."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .fock import FockBuilder


class BatchBuilder:
    """J+K builds for a list of FockBuilder contexts (same device)."""

    def __init__(self, builders: list[FockBuilder]):
        self.builders = builders
        self._lib = _lib.load()
        arr = (ctypes.c_void_p * len(builders))(*[fb._h.value for fb in builders])
        h = ctypes.c_void_p()
        _lib.check(self._lib.dgf_batch_create(arr, len(builders), ctypes.byref(h)), "dgf_batch_create")
        self._h = h
        off = (_lib.dgf_int * (len(builders) + 1))()
        _lib.check(self._lib.dgf_batch_layout(self._h, off), "dgf_batch_layout")
        self.offsets = np.array(off[:], dtype=np.int64)
        self.nbf = [fb.nbf for fb in builders]
        self.last_stats: dict = {}

    @property
    def total(self) -> int:
        return int(self.offsets[-1])

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._lib.dgf_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass

    def pack(self, mats):
        """List of (N_k, N_k) CUDA tensors -> one packed float64 tensor."""
        import torch

        return torch.cat([m.reshape(-1) for m in mats]).contiguous()

    def unpack(self, packed):
        return [packed[self.offsets[k]:self.offsets[k + 1]].view(n, n) for k, n in enumerate(self.nbf)]

    def herfck_batch(self, dpacked, fpacked=None, hfxfac=1.0, thrs=1e-12, use_graph=True, stream=None,
                     stats=True, mixed_cutoff=0.0):
        """F = J - hfxfac/2 K of every molecule, packed device tensors.  With
        ``mixed_cutoff`` > 0 the classes that the tuned context splits run
        their quartets with bound Q_AB Q_CD max|D| below it in FP32."""
        import torch

        if fpacked is None:
            fpacked = torch.empty_like(dpacked)
        opt = _lib.default_options(thrs=float(thrs), hfxfac=float(hfxfac), mixed_cutoff=float(mixed_cutoff))
        if stream is None:
            stream = torch.cuda.current_stream(dpacked.device).cuda_stream
        st = _lib.DgfStats()
        _lib.check(self._lib.dgf_fock_batch(self._h, ctypes.c_void_p(dpacked.data_ptr()),
                                            ctypes.c_void_p(fpacked.data_ptr()), ctypes.byref(opt),
                                            1 if use_graph else 0, ctypes.c_void_p(stream),
                                            ctypes.byref(st) if stats else None), "dgf_fock_batch")
        if stats:
            self.last_stats = st.as_dict()
        return fpacked
