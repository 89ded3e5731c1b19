"""ctypes front end of the CPU oracle — TEST INFRASTRUCTURE ONLY.

Loads ``oracle/_build/liboracle.so`` (built by ``oracle/Makefile``) and
offers the oracle's integrals, HERFCK-semantics Fock build and RHF gradient,
plus a numpy RHF/DIIS driver restating Dalton's SIRIUS DIIS loop
(``DALTON/sirius/sirdiis.F:282``) closely enough to reproduce its converged
energies.  Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU
baseline use this module; the product never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
_lib = None

_i64p = ctypes.POINTER(ctypes.c_int64)
_dp = ctypes.POINTER(ctypes.c_double)


class OrcBasis(ctypes.Structure):
    _fields_ = [("nblock", ctypes.c_int64), ("natom", ctypes.c_int64), ("nbf", ctypes.c_int64),
                ("spherical", ctypes.c_int64),
                ("block_l", _i64p), ("block_atom", _i64p), ("block_nprim", _i64p), ("block_ncontr", _i64p),
                ("block_ao_offset", _i64p), ("block_prim_offset", _i64p), ("block_coef_offset", _i64p),
                ("prim_exp", _dp), ("coef", _dp), ("atom_xyz", _dp), ("atom_charge", _dp)]


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.orc_fock.argtypes = [ctypes.POINTER(OrcBasis), ctypes.c_int, _i64p, _dp, _dp, ctypes.c_double,
                                  ctypes.c_double]
        _lib.orc_grad2e.argtypes = [ctypes.POINTER(OrcBasis), _dp, ctypes.c_double, ctypes.c_double, _dp]
        _lib.orc_grad1e.argtypes = [ctypes.POINTER(OrcBasis), _dp, _dp, _dp]
        _lib.orc_oneint.argtypes = [ctypes.POINTER(OrcBasis), _dp, _dp, _dp]
        _lib.orc_eri_full.argtypes = [ctypes.POINTER(OrcBasis), _dp]
        _lib.orc_boys.argtypes = [ctypes.c_int, ctypes.c_double, _dp]
        _lib.orc_sph_matrix.argtypes = [ctypes.c_int, _dp]
        _lib.orc_set_threads.argtypes = [ctypes.c_int]
        _lib.orc_nshell.argtypes = [ctypes.POINTER(OrcBasis)]
        _lib.orc_fock_sampled.argtypes = [ctypes.POINTER(OrcBasis), _dp, _dp, ctypes.c_double, ctypes.c_int,
                                          ctypes.c_int, _i64p]
        _lib.orc_schwarz.argtypes = [ctypes.POINTER(OrcBasis), _dp, _i64p, _i64p, _i64p]
        _lib.orc_fock_screened.argtypes = [ctypes.POINTER(OrcBasis), ctypes.c_int, _i64p, _dp, _dp,
                                           ctypes.c_double, ctypes.c_double, ctypes.c_int64, ctypes.c_int64, _i64p]
        _lib.orc_fock_hash_sample.argtypes = [ctypes.POINTER(OrcBasis), _dp, ctypes.c_double, ctypes.c_int, _i64p,
                                              _dp, _i64p]
        _lib.orc_fock_attenuated.argtypes = [ctypes.POINTER(OrcBasis), ctypes.c_int, _i64p, _dp, _dp,
                                             ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        _lib.orc_prim_eri.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp,
                                      ctypes.c_double, _dp]
        _lib.orc_prim_eri.restype = None
    return _lib


def _p(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


class _Holder:
    """Keeps the numpy arrays behind an OrcBasis alive."""

    def __init__(self, bs):
        c = lambda a, dt: np.ascontiguousarray(a, dtype=dt)
        self.arrs = dict(
            block_l=c(bs.block_l, np.int64), block_atom=c(bs.block_atom, np.int64),
            block_nprim=c(bs.block_nprim, np.int64), block_ncontr=c(bs.block_ncontr, np.int64),
            block_ao_offset=c(bs.block_ao_offset, np.int64), block_prim_offset=c(bs.block_prim_offset, np.int64),
            block_coef_offset=c(bs.block_coef_offset, np.int64), prim_exp=c(bs.prim_exp, np.float64),
            coef=c(bs.coef, np.float64), atom_xyz=c(bs.molecule.coords, np.float64),
            atom_charge=c(bs.molecule.charges, np.float64))
        a = self.arrs
        self.s = OrcBasis(bs.nblock, bs.molecule.natom, bs.nbf, int(bs.spherical),
                          *[_p(a[k], ctypes.c_int64) for k in ("block_l", "block_atom", "block_nprim",
                                                               "block_ncontr", "block_ao_offset",
                                                               "block_prim_offset", "block_coef_offset")],
                          *[_p(a[k], ctypes.c_double) for k in ("prim_exp", "coef", "atom_xyz", "atom_charge")])


def set_threads(n: int):
    lib().orc_set_threads(int(n))


def threads() -> int:
    return lib().orc_get_threads()


def boys(m: int, t: float) -> np.ndarray:
    f = np.zeros(m + 1)
    lib().orc_boys(m, float(t), _p(f, ctypes.c_double))
    return f


def sph_matrix(l: int) -> np.ndarray:
    nc = (l + 1) * (l + 2) // 2
    out = np.zeros((2 * l + 1) * nc if l >= 2 else nc * nc)
    lib().orc_sph_matrix(l, _p(out, ctypes.c_double))
    return out.reshape(2 * l + 1 if l >= 2 else nc, nc)


def nshell(bs) -> int:
    h = _Holder(bs)
    return lib().orc_nshell(ctypes.byref(h.s))


def schwarz(bs):
    """Schwarz factors of the segmented shells: (Q (ns,ns), l (ns,), nprim (ns,), atom (ns,))."""
    h = _Holder(bs)
    ns = lib().orc_nshell(ctypes.byref(h.s))
    q = np.zeros((ns, ns))
    l, n, a = (np.zeros(ns, dtype=np.int64) for _ in range(3))
    lib().orc_schwarz(ctypes.byref(h.s), _p(q, ctypes.c_double), _p(l, ctypes.c_int64), _p(n, ctypes.c_int64),
                      _p(a, ctypes.c_int64))
    return q, l, n, a


def oneint(bs):
    h = _Holder(bs)
    n = bs.nbf
    S, T, V = np.zeros((n, n)), np.zeros((n, n)), np.zeros((n, n))
    lib().orc_oneint(ctypes.byref(h.s), _p(S, ctypes.c_double), _p(T, ctypes.c_double), _p(V, ctypes.c_double))
    return S, T, V


def eri_full(bs) -> np.ndarray:
    h = _Holder(bs)
    n = bs.nbf
    out = np.zeros(n ** 4)
    lib().orc_eri_full(ctypes.byref(h.s), _p(out, ctypes.c_double))
    return out.reshape(n, n, n, n)


def fock_screened(bs, dmat, ifctyp=13, hfxfac=1.0, thrs=1e-12, ifthrs=20, icedif=3):
    """HERFCK-semantics Fock build with Dalton's density screening (IFTHRS,
    ICEDIF; see oracle.h).  Returns (F, counts) with counts a dict of the
    screening statistics."""
    h = _Holder(bs)
    d = np.ascontiguousarray(dmat, dtype=np.float64)
    single = d.ndim == 2
    if single:
        d = d[None]
    nd = d.shape[0]
    ift = np.ascontiguousarray(np.broadcast_to(np.asarray(ifctyp, dtype=np.int64), (nd,)))
    f = np.zeros_like(d)
    c = np.zeros(5, dtype=np.int64)
    lib().orc_fock_screened(ctypes.byref(h.s), nd, _p(ift, ctypes.c_int64), _p(d, ctypes.c_double),
                            _p(f, ctypes.c_double), float(hfxfac), float(thrs), int(ifthrs), int(icedif),
                            _p(c, ctypes.c_int64))
    counts = dict(zip(("evaluated", "skipped_screen", "skipped_zero", "dropped_coulomb", "dropped_exchange"),
                      (int(x) for x in c)))
    return (f[0] if single else f), counts


def fock_attenuated(bs, dmat, ifctyp=13, hfxfac=1.0, thrs=1e-12, hfxmu=0.0, hfxatt=0.0):
    """HERFCK with range-separated exchange: the 1/r12 build plus, for
    hfxmu != 0, -hfxatt/2 K[D] of erf(hfxmu r12)/r12 (see oracle.h)."""
    h = _Holder(bs)
    d = np.ascontiguousarray(dmat, dtype=np.float64)
    single = d.ndim == 2
    if single:
        d = d[None]
    nd = d.shape[0]
    ift = np.ascontiguousarray(np.broadcast_to(np.asarray(ifctyp, dtype=np.int64), (nd,)))
    f = np.zeros_like(d)
    lib().orc_fock_attenuated(ctypes.byref(h.s), nd, _p(ift, ctypes.c_int64), _p(d, ctypes.c_double),
                              _p(f, ctypes.c_double), float(hfxfac), float(thrs), float(hfxmu), float(hfxatt))
    return f[0] if single else f


def prim_eri(ls, exps, centers, mu=0.0):
    """One primitive Cartesian (la lb|lc ld) block of unnormalised Gaussians
    with the operator erf(mu r12)/r12 (mu = 0: 1/r12); shape (na, nb, nc, nd)."""
    ls = [int(x) for x in ls]
    nc = [(x + 1) * (x + 2) // 2 for x in ls]
    e = np.ascontiguousarray(exps, dtype=np.float64)
    c = np.ascontiguousarray(centers, dtype=np.float64).reshape(12)
    out = np.zeros(int(np.prod(nc)))
    lib().orc_prim_eri(ls[0], ls[1], ls[2], ls[3], _p(e, ctypes.c_double), _p(c, ctypes.c_double), float(mu),
                       _p(out, ctypes.c_double))
    return out.reshape(nc)


def fock_hash_sample(bs, dmat, k, thrs=1e-12):
    """Timing sample of the J+K build (see oracle.h): a fixed pseudo-random
    2^-k fraction of the significant quartets.  Returns (quartets evaluated,
    seconds, significant quartets in all)."""
    h = _Holder(bs)
    d = np.ascontiguousarray(dmat, dtype=np.float64)
    nq, tot = ctypes.c_int64(), ctypes.c_int64()
    sec = ctypes.c_double()
    lib().orc_fock_hash_sample(ctypes.byref(h.s), _p(d, ctypes.c_double), float(thrs), int(k), ctypes.byref(nq),
                               ctypes.byref(sec), ctypes.byref(tot))
    return nq.value, sec.value, tot.value


def fock(bs, dmat, ifctyp=13, hfxfac=1.0, thrs=1e-12) -> np.ndarray:
    """HERFCK-semantics Fock build (see oracle.h).  dmat: (N,N) or (ndmat,N,N)."""
    h = _Holder(bs)
    d = np.ascontiguousarray(dmat, dtype=np.float64)
    single = d.ndim == 2
    if single:
        d = d[None]
    nd = d.shape[0]
    ift = np.ascontiguousarray(np.broadcast_to(np.asarray(ifctyp, dtype=np.int64), (nd,)))
    f = np.zeros_like(d)
    lib().orc_fock(ctypes.byref(h.s), nd, _p(ift, ctypes.c_int64), _p(d, ctypes.c_double),
                   _p(f, ctypes.c_double), float(hfxfac), float(thrs))
    return f[0] if single else f


def fock_sampled(bs, dmat, stride, offset=0, thrs=1e-12):
    """J+K over every stride-th bra pair; returns (partial F, quartets done)."""
    h = _Holder(bs)
    d = np.ascontiguousarray(dmat, dtype=np.float64)
    f = np.zeros_like(d)
    nq = ctypes.c_int64()
    lib().orc_fock_sampled(ctypes.byref(h.s), _p(d, ctypes.c_double), _p(f, ctypes.c_double), float(thrs),
                           int(stride), int(offset), ctypes.byref(nq))
    return f, nq.value


def grad2e(bs, dmat, hfxfac=1.0, thrs=1e-12) -> np.ndarray:
    h = _Holder(bs)
    d = np.ascontiguousarray(dmat, dtype=np.float64)
    g = np.zeros((bs.molecule.natom, 3))
    lib().orc_grad2e(ctypes.byref(h.s), _p(d, ctypes.c_double), float(hfxfac), float(thrs), _p(g, ctypes.c_double))
    return g


def grad1e(bs, dmat, wmat) -> np.ndarray:
    h = _Holder(bs)
    d = np.ascontiguousarray(dmat, dtype=np.float64)
    w = np.ascontiguousarray(wmat, dtype=np.float64)
    g = np.zeros((bs.molecule.natom, 3))
    lib().orc_grad1e(ctypes.byref(h.s), _p(d, ctypes.c_double), _p(w, ctypes.c_double), _p(g, ctypes.c_double))
    return g


def rhf(bs, thrs=1e-12, conv=1e-10, maxiter=100, fock_fn=None, verbose=False):
    """Closed-shell RHF with DIIS on the oracle's integrals.

    Returns dict(energy, dmat (total density D = 2 C_occ C_occ^T), C, eps, wmat,
    S, H, fock, niter).  ``fock_fn(D) -> G`` replaces the oracle Fock build.
    """
    S, T, V = oneint(bs)
    H = T + V
    enuc = bs.molecule.nuclear_repulsion()
    nocc = bs.molecule.nelectrons() // 2
    s, U = np.linalg.eigh(S)
    X = U / np.sqrt(s)
    build = fock_fn or (lambda D: fock(bs, D, 13, 1.0, thrs))

    def solve(F):
        e, Cp = np.linalg.eigh(X.T @ F @ X)
        return e, X @ Cp

    eps, C = solve(H)
    D = 2.0 * C[:, :nocc] @ C[:, :nocc].T
    errs, focks = [], []
    energy = 0.0
    for it in range(1, maxiter + 1):
        G = build(D)
        F = H + G
        energy = 0.5 * np.sum(D * (H + F)) + enuc
        err = X.T @ (F @ D @ S - S @ D @ F) @ X
        en = np.linalg.norm(err)
        if verbose:
            print(f"iter {it:3d}  E = {energy:.12f}  |err| = {en:.3e}")
        if en < conv:
            break
        errs.append(err)
        focks.append(F)
        errs, focks = errs[-8:], focks[-8:]
        n = len(errs)
        if n >= 2:
            Bm = -np.ones((n + 1, n + 1))
            Bm[n, n] = 0.0
            for i in range(n):
                for j in range(n):
                    Bm[i, j] = np.sum(errs[i] * errs[j])
            rhs = np.zeros(n + 1)
            rhs[n] = -1.0
            cvec = np.linalg.solve(Bm, rhs)[:n]
            F = sum(c * f for c, f in zip(cvec, focks))
        eps, C = solve(F)
        D = 2.0 * C[:, :nocc] @ C[:, :nocc].T
    eps, C = solve(F)
    Cocc = C[:, :nocc]
    W = 2.0 * (Cocc * eps[:nocc]) @ Cocc.T
    return dict(energy=energy, dmat=D, C=C, eps=eps, wmat=W, S=S, H=H, fock=F, niter=it, nocc=nocc, enuc=enuc)


def rhf_gradient(bs, res, thrs=1e-12):
    return grad1e(bs, res["dmat"], res["wmat"]) + grad2e(bs, res["dmat"], 1.0, thrs)
