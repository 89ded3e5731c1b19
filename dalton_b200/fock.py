"""HERFCK-style host interface over libdgfock (the B200 J/K Fock build).

``FockBuilder.herfck`` mirrors Dalton's two-electron Fock call
``HERFCK(FMAT, DMAT, NDMT, ISYMDM, IFCTYP, ...)`` (DALTON/abacus/herdirect.F:431):
AO densities in, Fock matrices out, Dalton's C1 AO order and normalisation,
IFCTYP = 10*X + Y codes, Schwarz threshold THRS and density screening
IFTHRS.  ``herfck_device`` takes and returns CUDA tensors already resident in
device memory (the data stays in HBM between SCF iterations).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .basis import BasisSet


class _BasisArrays:
    def __init__(self, bs: BasisSet):
        c = lambda a, dt: np.ascontiguousarray(a, dtype=dt)
        i64 = np.int64
        self.arrs = [c(bs.block_l, i64), c(bs.block_atom, i64), c(bs.block_nprim, i64), c(bs.block_ncontr, i64),
                     c(bs.block_ao_offset, i64), c(bs.block_prim_offset, i64), c(bs.block_coef_offset, i64),
                     c(bs.prim_exp, np.float64), c(bs.coef, np.float64), c(bs.molecule.coords, np.float64),
                     c(bs.molecule.charges, np.float64)]
        ip = ctypes.POINTER(_lib.dgf_int)
        dp = ctypes.POINTER(ctypes.c_double)
        ptrs = [a.ctypes.data_as(ip) for a in self.arrs[:7]] + [a.ctypes.data_as(dp) for a in self.arrs[7:]]
        self.struct = _lib.DgfBasis(bs.nblock, bs.molecule.natom, bs.nbf, int(bs.spherical), *ptrs)


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class FockBuilder:
    """A device context for one molecule/basis (geometry-dependent pair data)."""

    def __init__(self, basis: BasisSet, device: int = 0):
        self.basis = basis
        self.nbf = basis.nbf
        self.natom = basis.molecule.natom
        self.device = device
        self._lib = _lib.load()
        self._arrays = _BasisArrays(basis)
        h = ctypes.c_void_p()
        _lib.check(self._lib.dgf_create(ctypes.byref(self._arrays.struct), int(device), ctypes.byref(h)),
                   "dgf_create")
        self._h = h
        self.last_stats: dict = {}

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._lib.dgf_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass

    def info(self):
        n, a, s = _lib.dgf_int(), _lib.dgf_int(), _lib.dgf_int()
        _lib.check(self._lib.dgf_info(self._h, ctypes.byref(n), ctypes.byref(a), ctypes.byref(s)), "dgf_info")
        return dict(nbf=n.value, natom=a.value, nshell=s.value)

    def ao_quartets(self, thrs=1e-12) -> int:
        """Significant contracted shell quartets of the AO basis at ``thrs``
        (the implementation-independent size of one build)."""
        n = _lib.dgf_int()
        _lib.check(self._lib.dgf_count_ao_quartets(self._h, float(thrs), ctypes.byref(n)), "dgf_count_ao_quartets")
        return int(n.value)

    def copy_tuning_from(self, other: "FockBuilder"):
        """Use the kernel choices (and mixed-form splits) ``other.autotune`` found."""
        _lib.check(self._lib.dgf_copy_tuning(self._h, other._h), "dgf_copy_tuning")

    def set_class_kernel(self, cls, variant, precision=64):
        """Pin the kernel of quartet class ``cls`` = (la, lb, lc, ld): variant
        -4 warp per quartet with FP64 tensor-core (DMMA) transforms, -3 warp
        per quartet, -2 warp team, -1 cooperative team, 0.. thread chunk
        variants."""
        la, lb, lc, ld = (int(x) for x in cls)
        _lib.check(self._lib.dgf_set_class_kernel(self._h, la, lb, lc, ld, int(precision), int(variant)),
                   "dgf_set_class_kernel")

    @staticmethod
    def _ifctyp(ifctyp, nd):
        return np.ascontiguousarray(np.broadcast_to(np.asarray(ifctyp, dtype=np.int64), (nd,)))

    def herfck(self, dmat, ifctyp=13, hfxfac=1.0, thrs=1e-12, ifthrs=20, mixed_cutoff=0.0, shard=(0, 1),
               icedif=3, hfxmu=0.0, hfxatt=0.0) -> np.ndarray:
        """F = [Y&1] J[D] - [Y&2] hfxfac/2 K[D] for host matrices (N,N) or (ndmat,N,N).
        Density screening (Dalton's .IFTHRS) is on for ifthrs < 16, with
        Dalton's separate Coulomb/exchange skips per ``icedif`` (.ICEDIF).
        With ``hfxmu`` != 0 (range-separated hybrids) F also gets
        -hfxatt/2 K[D] of the operator erf(hfxmu r12)/r12."""
        d = np.ascontiguousarray(dmat, dtype=np.float64)
        single = d.ndim == 2
        if single:
            d = d[None]
        if d.shape[1:] != (self.nbf, self.nbf):
            raise ValueError(f"density must be ({self.nbf},{self.nbf}), got {d.shape[1:]}")
        nd = d.shape[0]
        ift = self._ifctyp(ifctyp, nd)
        f = np.empty_like(d)
        opt = _lib.default_options(thrs=float(thrs), ifthrs=int(ifthrs), hfxfac=float(hfxfac),
                                   mixed_cutoff=float(mixed_cutoff), shard_index=int(shard[0]),
                                   shard_count=int(shard[1]), icedif=int(icedif), hfxmu=float(hfxmu),
                                   hfxatt=float(hfxatt))
        st = _lib.DgfStats()
        _lib.check(self._lib.dgf_fock(self._h, nd, ift.ctypes.data_as(ctypes.POINTER(_lib.dgf_int)), _dp(d), _dp(f),
                                      ctypes.byref(opt), ctypes.byref(st)), "dgf_fock")
        self.last_stats = st.as_dict()
        return f[0] if single else f

    def herfck_device(self, dmat, fmat=None, ifctyp=13, hfxfac=1.0, thrs=1e-12, ifthrs=20, mixed_cutoff=0.0,
                      stream=None, stats=True, shard=(0, 1), icedif=3, hfxmu=0.0, hfxatt=0.0):
        """Device form: ``dmat`` a CUDA float64 tensor (N,N) or (ndmat,N,N)."""
        import torch

        if dmat.device.type != "cuda" or dmat.dtype != torch.float64:
            raise ValueError("dmat must be a CUDA float64 tensor")
        d = dmat.contiguous()
        nd = 1 if d.dim() == 2 else d.shape[0]
        if fmat is None:
            fmat = torch.empty_like(d)
        ift = self._ifctyp(ifctyp, nd)
        opt = _lib.default_options(thrs=float(thrs), ifthrs=int(ifthrs), hfxfac=float(hfxfac),
                                   mixed_cutoff=float(mixed_cutoff), shard_index=int(shard[0]),
                                   shard_count=int(shard[1]), icedif=int(icedif), hfxmu=float(hfxmu),
                                   hfxatt=float(hfxatt))
        if stream is None:
            stream = torch.cuda.current_stream(d.device).cuda_stream
        st = _lib.DgfStats()
        _lib.check(self._lib.dgf_fock_device(self._h, nd, ift.ctypes.data_as(ctypes.POINTER(_lib.dgf_int)),
                                             ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(fmat.data_ptr()),
                                             ctypes.byref(opt), ctypes.c_void_p(stream),
                                             ctypes.byref(st) if stats else None), "dgf_fock_device")
        if stats:
            self.last_stats = st.as_dict()
        return fmat

    def store_integrals(self, thrs=1e-12, max_bytes=0, stream=None):
        """Conventional form: evaluate the integral blocks of every quartet of
        the plan for ``thrs`` once and keep them in device memory (Dalton's
        AOTWOINT file, held on the GPU).  Returns the store's size in bytes."""
        import torch

        if stream is None:
            stream = torch.cuda.current_stream().cuda_stream
        nbytes = ctypes.c_int64()
        _lib.check(self._lib.dgf_store_integrals(self._h, float(thrs), int(max_bytes), ctypes.c_void_p(stream),
                                                 ctypes.byref(nbytes)), "dgf_store_integrals")
        return nbytes.value

    def release_store(self):
        _lib.check(self._lib.dgf_store_release(self._h), "dgf_store_release")

    def herfck_stored(self, dmat, fmat=None, ifctyp=13, hfxfac=1.0, thrs=1e-12, ifthrs=20, stream=None, stats=True,
                      shard=(0, 1), icedif=3):
        """HERFCK from the integral store (Dalton's SIRFCK2 over AOTWOINT):
        ``dmat`` a CUDA float64 tensor (N,N) or (ndmat,N,N); same results as
        ``herfck_device`` with the store's Schwarz threshold."""
        import torch

        if dmat.device.type != "cuda" or dmat.dtype != torch.float64:
            raise ValueError("dmat must be a CUDA float64 tensor")
        d = dmat.contiguous()
        nd = 1 if d.dim() == 2 else d.shape[0]
        if fmat is None:
            fmat = torch.empty_like(d)
        ift = self._ifctyp(ifctyp, nd)
        opt = _lib.default_options(thrs=float(thrs), ifthrs=int(ifthrs), hfxfac=float(hfxfac),
                                   shard_index=int(shard[0]), shard_count=int(shard[1]), icedif=int(icedif))
        if stream is None:
            stream = torch.cuda.current_stream(d.device).cuda_stream
        st = _lib.DgfStats()
        _lib.check(self._lib.dgf_fock_stored(self._h, nd, ift.ctypes.data_as(ctypes.POINTER(_lib.dgf_int)),
                                             ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(fmat.data_ptr()),
                                             ctypes.byref(opt), ctypes.c_void_p(stream),
                                             ctypes.byref(st) if stats else None), "dgf_fock_stored")
        if stats:
            self.last_stats = st.as_dict()
        return fmat

    def autotune(self, dmat, thrs=1e-12, hfxfac=1.0, mixed_cutoff=0.0):
        """Time every candidate kernel per quartet class on this density (a
        CUDA float64 tensor) and keep the fastest; with ``mixed_cutoff`` > 0
        also decide per class whether the mixed form splits it into FP64 and
        FP32 launches.  Returns the timing list."""
        import json

        import torch

        d = dmat.contiguous()
        opt = _lib.default_options(thrs=float(thrs), hfxfac=float(hfxfac), mixed_cutoff=float(mixed_cutoff))
        buf = ctypes.create_string_buffer(1 << 16)
        stream = torch.cuda.current_stream(d.device).cuda_stream
        _lib.check(self._lib.dgf_autotune(self._h, ctypes.c_void_p(d.data_ptr()), ctypes.byref(opt),
                                          ctypes.c_void_p(stream), buf, len(buf)), "dgf_autotune")
        try:
            return json.loads(buf.value.decode())
        except ValueError:
            return []

    def set_profiling(self, on: bool = True):
        _lib.check(self._lib.dgf_set_profiling(self._h, 1 if on else 0), "dgf_set_profiling")

    def profile(self) -> list[dict]:
        """Per-class launch records of the last profiled Fock build."""
        n = ctypes.c_int()
        _lib.check(self._lib.dgf_get_profile(self._h, None, 0, ctypes.byref(n)), "dgf_get_profile")
        arr = (_lib.DgfClassTime * max(n.value, 1))()
        _lib.check(self._lib.dgf_get_profile(self._h, arr, n.value, ctypes.byref(n)), "dgf_get_profile")
        return [arr[i].as_dict() for i in range(n.value)]

    def oneint(self):
        n = self.nbf
        S, T, V = (np.empty((n, n)) for _ in range(3))
        _lib.check(self._lib.dgf_oneint(self._h, _dp(S), _dp(T), _dp(V)), "dgf_oneint")
        return S, T, V

    def grad2e(self, dmat, hfxfac=1.0, thrs=1e-12) -> np.ndarray:
        d = np.ascontiguousarray(dmat, dtype=np.float64)
        g = np.empty((self.natom, 3))
        _lib.check(self._lib.dgf_grad2e(self._h, _dp(d), float(hfxfac), float(thrs), _dp(g)), "dgf_grad2e")
        return g

    def grad1e(self, dmat, wmat) -> np.ndarray:
        d = np.ascontiguousarray(dmat, dtype=np.float64)
        w = np.ascontiguousarray(wmat, dtype=np.float64)
        g = np.empty((self.natom, 3))
        _lib.check(self._lib.dgf_grad1e(self._h, _dp(d), _dp(w), _dp(g)), "dgf_grad1e")
        return g
