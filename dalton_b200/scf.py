"""Closed-shell RHF driver around the device Fock build.

Mirrors the parts of Dalton's SIRIUS SCF that call the two-electron Fock
build (``DIIS_CTL``, DALTON/sirius/sirdiis.F:282):

* AO density ``D = 2 C_occ C_occ^T`` (FCKDEN, DALTON/sirius/sirgrad.F:247);
* ``G(D)`` through the HERFCK-semantics build with IFCTYP = 13
  (FCK2AO, sirgrad.F:714-860);
* incremental difference-density Fock builds: ``G(D_n) = G(D_{n-1}) +
  G(D_n - D_{n-1})`` (DIFDEN, sirdiis.F:551-567, 733-773, 811-825), with a
  full rebuild every ``full_every`` iterations;
* optionally Dalton's integral-screening schedule for direct SCF
  (``ifthrs_schedule``, sirdiis.F:520-523, 1224-1248): the density screen
  Q_AB Q_CD |D| < 10^-IFTHRS is loose while the orbital gradient is large
  and tightens with it, IFTHRS = -log10(|g| / SCRFAC) + 3 clamped to
  [IFTMIN, IFTMAX], SCRFAC = 100 N^2; a tightened threshold forces a full
  build, otherwise the build is incremental;
* DIIS extrapolation on the orbital gradient ``FDS - SDF``;
* energy ``E = 1/2 sum D (H + F) + E_nuc`` (EMY, sirdiis.F:825).

Matrices live on the GPU (torch float64); the linear algebra is torch's.
With ``mixed_cutoff > 0`` the Fock builds run in the mixed form: quartets
whose bound Q_AB Q_CD |D| is below the cutoff are contracted in FP32.  The
incremental build makes that bound shrink with the density change, which
is how the mixed form wins back its accuracy.
"""
from __future__ import annotations

import time

import numpy as np

from .basis import BasisSet
from .fock import FockBuilder


def rhf(bs: BasisSet, fb: FockBuilder | None = None, conv: float = 1e-8, maxiter: int = 50, thrs: float = 1e-12,
        mixed_cutoff: float = 0.0, incremental: bool = True, full_every: int = 8, diis_size: int = 8,
        device: str = "cuda", verbose: bool = False, fixed_iterations: int | None = None,
        ifthrs_schedule: bool = False, stored: bool = False):
    """Run RHF; returns a dict with energy, density, orbitals, timings.
    ``stored``: Fock builds from the builder's integral store (the
    conventional form; ``fb.store_integrals(thrs)`` first)."""
    import torch

    fb = fb or FockBuilder(bs)
    dev = torch.device(device)
    S_np, T_np, V_np = fb.oneint()
    S = torch.tensor(S_np, device=dev)
    H = torch.tensor(T_np + V_np, device=dev)
    enuc = bs.molecule.nuclear_repulsion()
    nocc = bs.molecule.nelectrons() // 2
    s, U = torch.linalg.eigh(S)
    X = U / torch.sqrt(s)

    def solve(F):
        e, Cp = torch.linalg.eigh(X.T @ F @ X)
        return e, X @ Cp

    eps, C = solve(H)
    D = 2.0 * C[:, :nocc] @ C[:, :nocc].T
    D_prev = None
    G_prev = None
    errs, focks = [], []
    energy = 0.0
    history = []
    fock_ms = 0.0
    nbuild = 0
    it = 0
    # Dalton's screening limits (sirdiis.F:520-523), conv playing THDIIS
    scrfac = 100.0 * bs.nbf * bs.nbf
    iftmax = int(-np.log10(conv / scrfac)) + 1
    iftmin = int(-np.log10(0.1 / scrfac)) + 1
    ifthrs = iftmin if ifthrs_schedule else 20
    newthr = False
    ifthrs_used = []
    for it in range(1, maxiter + 1):
        full = (not incremental) or G_prev is None or (it % full_every == 0) or newthr
        t0 = time.perf_counter()
        if stored:
            build = lambda dm: fb.herfck_stored(dm, ifctyp=13, thrs=thrs, ifthrs=ifthrs)
        else:
            build = lambda dm: fb.herfck_device(dm, ifctyp=13, thrs=thrs, ifthrs=ifthrs, mixed_cutoff=mixed_cutoff)
        if full:
            G = build(D)
        else:
            G = G_prev + build(D - D_prev)
        ifthrs_used.append(ifthrs)
        torch.cuda.synchronize(dev)
        fock_ms += (time.perf_counter() - t0) * 1e3
        nbuild += 1
        G_prev, D_prev = G, D
        F = H + G
        err = X.T @ (F @ D @ S - S @ D @ F) @ X
        # the iteration's one device-to-host read: energy and error norm together
        e_and_norm = torch.stack([0.5 * torch.sum(D * (H + F)), torch.linalg.norm(err)]).cpu()
        energy = float(e_and_norm[0]) + enuc
        en = float(e_and_norm[1])
        history.append((energy, en, bool(full)))
        if ifthrs_schedule:  # next build's screening threshold (sirdiis.F:1224-1248, DIFDEN form)
            ithrs = int(-np.log10(max(en, 1e-300) / scrfac)) + 3
            if ithrs >= iftmax - 2:
                ithrs = iftmax
            newthr = abs(ithrs - ifthrs) >= 2
            if newthr:
                ifthrs = min(iftmax, max(iftmin, ithrs))
        if verbose:
            print(f"iter {it:3d}  E = {energy:.12f}  |g| = {en:.3e}  {'full' if full else 'incr'}")
        if fixed_iterations is None and en < conv:
            break
        if fixed_iterations is not None and it >= fixed_iterations:
            break
        errs.append(err)
        focks.append(F)
        errs, focks = errs[-diis_size:], focks[-diis_size:]
        n = len(errs)
        Fx = F
        if n >= 2:
            Bm = -torch.ones((n + 1, n + 1), dtype=F.dtype, device=dev)
            Bm[n, n] = 0.0
            for i in range(n):
                for j in range(n):
                    Bm[i, j] = torch.sum(errs[i] * errs[j])
            rhs = torch.zeros(n + 1, dtype=F.dtype, device=dev)
            rhs[n] = -1.0
            cvec = torch.linalg.solve(Bm, rhs)[:n]
            Fx = sum(c * f for c, f in zip(cvec, focks))
        eps, C = solve(Fx)
        D = 2.0 * C[:, :nocc] @ C[:, :nocc].T
    eps, C = solve(F)
    Cocc = C[:, :nocc]
    W = 2.0 * (Cocc * eps[:nocc]) @ Cocc.T
    return dict(energy=energy, dmat=D, C=C, eps=eps, wmat=W, S=S, H=H, fock=F, niter=it, nocc=nocc, enuc=enuc,
                history=history, fock_ms=fock_ms, nbuild=nbuild, builder=fb, ifthrs=ifthrs_used)


def energy_of(D, H, G, enuc: float) -> float:
    """E = 1/2 sum D (2H + G) + E_nuc for a fixed density."""
    import torch

    return float(0.5 * torch.sum(D * (2.0 * H + G))) + enuc


def to_numpy(x):
    return x.detach().cpu().numpy() if hasattr(x, "detach") else np.asarray(x)
