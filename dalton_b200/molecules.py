"""Seeded synthetic molecules for the J/K Fock-build workloads.

All geometries are generated, never read from a dataset:

* water clusters: O-H 0.96 A, H-O-H 104.5 deg, each molecule rotated by a
  seeded random rotation about its oxygen, oxygens on a 3.0 A cubic grid with
  +-0.3 A uniform jitter per axis;
* all-trans linear alkanes CnH2n+2: C-C 1.54 A, C-H 1.09 A, tetrahedral
  angles, +-0.02 A seeded jitter on every atom;
* the H2O geometry of Dalton's ``energy_direct`` test
  (``DALTON/test/energy_direct:36-43``) and acrolein of ``geoopt_preopt2``
  (``DALTON/test/geoopt_preopt2/acrolein.mol``), the golden-value inputs.
"""
from __future__ import annotations

import math

import numpy as np

from .basis import Molecule

OH = 0.96
HOH = math.radians(104.5)


def _rotation(rng: np.random.Generator) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([
        [a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
        [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
        [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d],
    ])


def water_cluster(n: int, grid=None, seed: int = 0, spacing: float = 3.0, jitter: float = 0.3) -> Molecule:
    """n water molecules on a cubic grid (first n points of ``grid``, x fastest)."""
    if grid is None:
        grid = _default_grid(n)
    gx, gy, gz = grid
    if gx * gy * gz < n:
        raise ValueError("grid too small")
    rng = np.random.default_rng(seed)
    h1 = np.array([OH, 0.0, 0.0])
    h2 = np.array([OH * math.cos(HOH), OH * math.sin(HOH), 0.0])
    symbols, xyz = [], []
    k = 0
    for iz in range(gz):
        for iy in range(gy):
            for ix in range(gx):
                if k >= n:
                    break
                centre = np.array([ix, iy, iz], dtype=np.float64) * spacing
                centre += rng.uniform(-jitter, jitter, size=3)
                R = _rotation(rng)
                symbols += ["O", "H", "H"]
                xyz += [centre, centre + R @ h1, centre + R @ h2]
                k += 1
    return Molecule.from_angstrom(symbols, np.array(xyz))


def _default_grid(n: int):
    table = {1: (1, 1, 1), 2: (2, 1, 1), 4: (2, 2, 1), 8: (2, 2, 2), 16: (4, 2, 2), 32: (4, 4, 2),
             64: (4, 4, 4)}
    if n in table:
        return table[n]
    side = math.ceil(n ** (1 / 3))
    return (side, side, side)


def alkane(nc: int, seed: int = 0, jitter: float = 0.02) -> Molecule:
    """All-trans linear CnH2n+2 (zig-zag backbone in the xy plane)."""
    rng = np.random.default_rng(seed)
    cc, ch = 1.54, 1.09
    tet = math.acos(-1.0 / 3.0)
    half = 0.5 * tet
    dx = cc * math.sin(half)
    dy = cc * math.cos(half)
    carbons = [np.array([i * dx, (0.0 if i % 2 == 0 else dy), 0.0]) for i in range(nc)]
    symbols = ["C"] * nc
    xyz = list(carbons)
    for i, c in enumerate(carbons):
        # the two in-plane bonds of carbon i point to its neighbours; the hydrogens
        # complete the tetrahedron
        nbrs = []
        if i > 0:
            nbrs.append(carbons[i - 1] - c)
        if i < nc - 1:
            nbrs.append(carbons[i + 1] - c)
        if len(nbrs) == 1:
            # terminal carbon: virtual neighbour continuing the zig-zag
            v = nbrs[0]
            mirror = np.array([-v[0], v[1], 0.0])
            nbrs.append(mirror)
        u1, u2 = (v / np.linalg.norm(v) for v in nbrs)
        bis = -(u1 + u2)
        bis /= np.linalg.norm(bis)
        perp = np.cross(u1, u2)
        perp /= np.linalg.norm(perp)
        hdirs = [math.cos(half) * bis + math.sin(half) * perp, math.cos(half) * bis - math.sin(half) * perp]
        for hd in hdirs:
            symbols.append("H")
            xyz.append(c + ch * hd)
        if i in (0, nc - 1):
            # third hydrogen of a methyl group along the virtual neighbour
            v = nbrs[-1] / np.linalg.norm(nbrs[-1])
            symbols.append("H")
            xyz.append(c + ch * v)
    xyz = np.array(xyz) + rng.uniform(-jitter, jitter, size=(len(xyz), 3))
    return Molecule.from_angstrom(symbols, xyz)


def water_dalton_test() -> Molecule:
    """H2O of Dalton's energy_direct test (bohr)."""
    return Molecule.from_bohr(["O", "H", "H"], [[0.0, -0.2249058930, 0.0], [1.45235, 0.899623, 0.0],
                                                [-1.45235, 0.899623, 0.0]])


def acrolein() -> Molecule:
    """Acrolein of Dalton's geoopt_preopt2 test (Angstrom input)."""
    ang = [[-0.145335, -0.546770, 0.000607], [1.274009, -0.912471, -0.000167], [1.630116, -2.207690, -0.000132],
           [-0.560104, 0.608977, 0.000534], [-0.871904, -1.386459, 0.001253], [2.004448, -0.101417, -0.000710],
           [0.879028, -3.000685, 0.000484], [2.675323, -2.516779, -0.000673]]
    return Molecule.from_angstrom(["C", "C", "C", "O", "H", "H", "H", "H"], ang)


def water_batch(count: int = 256, lo: int = 1, hi: int = 16, seed: int = 0) -> list[Molecule]:
    """Batch of water clusters with sizes drawn uniformly from [lo, hi]."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(lo, hi + 1, size=count)
    return [water_cluster(int(n), grid=(4, 2, 2) if n <= 16 else None, seed=seed * 100003 + i)
            for i, n in enumerate(sizes)]


# Named workloads (sizes as used by the bench and the parity tests).
def config(name: str):
    """Return (molecule or list of molecules, basis name) of a named workload."""
    if name == "h2o4_ccpvdz":
        return water_cluster(4, (2, 2, 1), seed=1), "cc-pVDZ"
    if name == "h2o32_ccpvdz":
        return water_cluster(32, (4, 4, 2), seed=32), "cc-pVDZ"
    if name == "c20h42_ccpvtz":
        return alkane(20, seed=20), "cc-pVTZ"
    if name == "h2o16_ccpvdz":
        return water_cluster(16, (4, 2, 2), seed=16), "cc-pVDZ"
    if name == "batch256_631gs":
        return water_batch(256, 1, 16, seed=256), "6-31G*"
    raise KeyError(name)
