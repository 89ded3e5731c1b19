"""Dalton basis-library reader and HERMIT C1 shell conventions.

This module plays the part Dalton's HERMIT input stage plays for the
two-electron Fock build: it reads a basis set in the Dalton basis-library
text format, normalises the contraction coefficients the way HERMIT does and
lays the atomic orbitals out in Dalton's C1 order.  Its output is the shell
description the C ABI (``include/dgfock.h``) takes, i.e. what a Fortran shim
would gather from Dalton's ``/SHELLS/``/``/PRIMIT/`` common blocks.

Conventions restated from the Dalton sources (paths inside the Dalton tree):

* basis-library format: ``a <Z>`` element cards, blocks of
  ``nprim ncontr 0`` headers followed by ``nprim`` rows of an exponent and
  ``ncontr`` coefficients read free-format (``DALTON/abacus/herbas.F:593-640``,
  READ_NU); consecutive blocks of one element are s, p, d, ... shells.
* normalisation: NRMORB (``DALTON/abacus/herrdn.F:3263-3290``); each
  contracted function is normalised and each primitive coefficient carries
  ``(4 alpha)^(l/2+3/4) (2 pi)^(-3/4)``, the norm of the axial Cartesian
  component ``x^l``.
* AO order in C1: atom -> angular momentum -> contracted function ->
  component, p as x, y, z and spherical components m = -l..l (MORDER=1)
  (``DALTON/test/trueresult/energy_nosymm.ref:899-924``,
  ``DALTON/abacus/herrdn.F:5444-5530``).  p shells are Cartesian; d and higher
  are spherical unless ``spherical=False`` (Dalton's ``Cartesian`` keyword).
* Angstrom to bohr: Dalton's ``XTANG = 0.5291772108`` (``DALTON/include/codata.h:35``).
"""
from __future__ import annotations

import math
import os
import re
from dataclasses import dataclass, field

import numpy as np

XTANG = 0.5291772108
DATA_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "basis_data")
ELEMENT_SYMBOL = {1: "H", 2: "He", 6: "C", 7: "N", 8: "O"}
SYMBOL_Z = {v: k for k, v in ELEMENT_SYMBOL.items()}


@dataclass
class Block:
    """One basis-library block: angular momentum, exponents, raw coefficients."""
    l: int
    exps: np.ndarray          # (nprim,)
    coefs: np.ndarray         # (nprim, ncontr), as read (unnormalised)


def parse_dalton_basis(text: str) -> dict[int, list[Block]]:
    """Parse the Dalton basis-library text format into {Z: [Block, ...]}."""
    elements: dict[int, list[Block]] = {}
    tokens_by_element: dict[int, list[str]] = {}
    current = None
    for raw in text.splitlines():
        line = raw.strip()
        if not line or line.startswith("$") or line.startswith("!"):
            continue
        m = re.match(r"^[aA]\s+(\d+)\s*$", line)
        if m:
            current = int(m.group(1))
            tokens_by_element[current] = []
            continue
        if current is None:
            continue
        tokens_by_element[current].extend(line.replace("D", "E").replace("d", "e").split())
    for z, toks in tokens_by_element.items():
        blocks = []
        pos = 0
        l = 0
        while pos < len(toks):
            nprim, ncontr = int(toks[pos]), int(toks[pos + 1])
            pos += 3
            exps = np.zeros(nprim)
            coefs = np.zeros((nprim, ncontr))
            for i in range(nprim):
                exps[i] = float(toks[pos])
                coefs[i, :] = [float(t) for t in toks[pos + 1: pos + 1 + ncontr]]
                pos += 1 + ncontr
            blocks.append(Block(l, exps, coefs))
            l += 1
        elements[z] = blocks
    return elements


_CACHE: dict[str, dict[int, list[Block]]] = {}


def load_basis(name: str) -> dict[int, list[Block]]:
    """Load a basis set shipped in ``basis_data`` (a subset of Dalton's library)."""
    if name not in _CACHE:
        fname = os.path.join(DATA_DIR, name.replace("*", "_star") + ".dalton")
        if not os.path.exists(fname):
            raise FileNotFoundError(f"basis set {name!r} not shipped (looked for {fname})")
        with open(fname) as f:
            _CACHE[name] = parse_dalton_basis(f.read())
    return _CACHE[name]


def nrmorb(l: int, exps: np.ndarray, coefs: np.ndarray) -> np.ndarray:
    """Normalised contraction coefficients (HERMIT NRMORB, herrdn.F:3263-3290).

    Returns CPRIM with the same shape as ``coefs``: each column is scaled so
    the contracted axial Cartesian function is normalised, and each primitive
    row carries ``(4 a)^(l/2 + 3/4) * (2 pi)^(-3/4)``.
    """
    exps = np.asarray(exps, dtype=np.float64)
    coefs = np.asarray(coefs, dtype=np.float64)
    nprim, ncontr = coefs.shape
    out = np.zeros_like(coefs)
    if nprim == 1 and abs(exps[0]) <= 1e-10:
        out[0, 0] = 1.0
        return out
    pippi = (0.5 / math.pi) ** 0.75
    aa = exps[:, None]
    bb = exps[None, :]
    t = (2.0 * np.sqrt(aa * bb) / (aa + bb)) ** (l + 1.5)
    for n in range(ncontr):
        c = coefs[:, n]
        s = float(c @ t @ c)
        if math.sqrt(abs(s)) < 1e-17:
            raise ValueError(f"contracted function {n} of an l={l} block has zero norm")
        out[:, n] = c / math.sqrt(s) * (4.0 * exps) ** (0.5 * l + 0.75) * pippi
    return out


@dataclass
class Molecule:
    """Atoms as nuclear charges and Cartesian coordinates in bohr."""
    charges: np.ndarray       # (natom,) float
    coords: np.ndarray        # (natom, 3) bohr
    symbols: list[str] = field(default_factory=list)

    @property
    def natom(self):
        return len(self.charges)

    @staticmethod
    def from_angstrom(symbols, xyz_angstrom):
        z = np.array([float(SYMBOL_Z[s]) for s in symbols])
        return Molecule(z, np.asarray(xyz_angstrom, dtype=np.float64) / XTANG, list(symbols))

    @staticmethod
    def from_bohr(symbols, xyz_bohr):
        z = np.array([float(SYMBOL_Z[s]) for s in symbols])
        return Molecule(z, np.asarray(xyz_bohr, dtype=np.float64), list(symbols))

    def nuclear_repulsion(self) -> float:
        e = 0.0
        for i in range(self.natom):
            for j in range(i):
                e += self.charges[i] * self.charges[j] / np.linalg.norm(self.coords[i] - self.coords[j])
        return float(e)

    def nelectrons(self) -> int:
        return int(round(self.charges.sum()))


def ncart(l: int) -> int:
    return (l + 1) * (l + 2) // 2


def nfunc(l: int, spherical: bool) -> int:
    if spherical and l >= 2:
        return 2 * l + 1
    return ncart(l)


@dataclass
class BasisSet:
    """A molecule's AO basis in Dalton C1 order, as Dalton-style shell blocks.

    Each block is one (atom, l) basis-library block with ``nprim`` primitives
    shared by ``ncontr`` contracted functions (a general contraction, as in
    Dalton's CPRIM).  Arrays follow the C ABI's ``dgf_basis`` struct.
    """
    molecule: Molecule
    name: str
    spherical: bool
    block_l: np.ndarray
    block_atom: np.ndarray
    block_nprim: np.ndarray
    block_ncontr: np.ndarray
    block_ao_offset: np.ndarray
    block_prim_offset: np.ndarray
    block_coef_offset: np.ndarray
    prim_exp: np.ndarray
    coef: np.ndarray           # concatenated column-major (nprim, ncontr) CPRIM blocks
    nbf: int

    @property
    def nblock(self):
        return len(self.block_l)

    def max_l(self):
        return int(self.block_l.max()) if self.nblock else 0

    def block_coefs(self, i):
        off = int(self.block_coef_offset[i])
        n, c = int(self.block_nprim[i]), int(self.block_ncontr[i])
        return self.coef[off: off + n * c].reshape(c, n).T

    def block_exps(self, i):
        off = int(self.block_prim_offset[i])
        return self.prim_exp[off: off + int(self.block_nprim[i])]

    def ao_atom(self) -> np.ndarray:
        """Atom index of every AO."""
        out = np.zeros(self.nbf, dtype=np.int64)
        for i in range(self.nblock):
            n = int(self.block_ncontr[i]) * nfunc(int(self.block_l[i]), self.spherical)
            out[self.block_ao_offset[i]: self.block_ao_offset[i] + n] = self.block_atom[i]
        return out

    def with_coords(self, coords: np.ndarray) -> "BasisSet":
        mol = Molecule(self.molecule.charges.copy(), np.asarray(coords, dtype=np.float64).reshape(-1, 3),
                       list(self.molecule.symbols))
        return build_basis(mol, self.name, self.spherical)


def build_basis(mol: Molecule, name: str, spherical: bool = True) -> BasisSet:
    """Lay out the basis of ``mol`` in Dalton C1 order (atom -> l -> contraction -> component)."""
    lib = load_basis(name)
    bl, ba, bn, bc, bao, bpo, bco = [], [], [], [], [], [], []
    exps, coefs = [], []
    ao = po = co = 0
    for ia in range(mol.natom):
        z = int(round(mol.charges[ia]))
        if z not in lib:
            raise KeyError(f"element Z={z} not in basis {name}")
        for blk in lib[z]:
            cprim = nrmorb(blk.l, blk.exps, blk.coefs)
            nprim, ncontr = cprim.shape
            bl.append(blk.l)
            ba.append(ia)
            bn.append(nprim)
            bc.append(ncontr)
            bao.append(ao)
            bpo.append(po)
            bco.append(co)
            exps.append(blk.exps)
            coefs.append(cprim.T.reshape(-1))   # column-major (nprim, ncontr)
            ao += ncontr * nfunc(blk.l, spherical)
            po += nprim
            co += nprim * ncontr
    as_i = lambda v: np.asarray(v, dtype=np.int64)
    return BasisSet(mol, name, spherical, as_i(bl), as_i(ba), as_i(bn), as_i(bc), as_i(bao), as_i(bpo),
                    as_i(bco), np.concatenate(exps), np.concatenate(coefs), ao)


def cart_exponents(l: int) -> list[tuple[int, int, int]]:
    """Dalton's Cartesian component order (xx, xy, xz, yy, yz, zz for l=2)."""
    out = []
    for i in range(l, -1, -1):
        for j in range(l - i, -1, -1):
            out.append((i, j, l - i - j))
    return out


def sph_transform(l: int) -> np.ndarray:
    """Cartesian -> normalised real spherical matrix, shape (2l+1, ncart(l)).

    Restates SPHCO1 (``DALTON/abacus/her1pro.F:4697-4770``) for MORDER=1,
    MINTEG=2: rows are m = -l..l; columns follow ``cart_exponents``.
    """
    if l == 0:
        return np.ones((1, 1))
    if l == 1:
        return np.eye(3)
    binom = math.comb
    pl = [0.0] * (l + 1)
    for k in range(l // 2 + 1):
        pl[l - 2 * k] = ((-1.0) ** k) * 2.0 ** (-l) * binom(l, k) * binom(2 * (l - k), l)
    cs = np.zeros((l + 1, l + 1))
    cs[0, 0] = 1.0
    for m in range(1, l + 1):
        cs[m, 0] = 1.0
        for k in range(1, m + 1):
            cs[m, k] = cs[m - 1, k - 1] * ((-1.0) ** (k - 1))
            if m > k:
                cs[m, k] += cs[m - 1, k]
    nx = ncart(l)
    tr = np.zeros((nx, 2 * l + 1))
    dfact = 1.0
    for v in range(2 * l - 1, 0, -2):
        dfact *= v
    for m in range(l + 1):
        cm = 1.0 if m == 0 else math.sqrt(2.0 * math.factorial(l - m) / math.factorial(l + m))
        cm /= math.sqrt(dfact)
        for k in range((l - m) % 2, l - m + 1, 2):
            if m > 0:
                pl[k] = (k + 1) * pl[k + 1]
            cmk = cm * pl[k]
            for i in range((l - k - m) // 2 + 1):
                cmki = cmk * binom((l - k - m) // 2, i)
                for j in range(i + 1):
                    cmkij = cmki * binom(i, j)
                    for n in range(m + 1):
                        ix = l - 2 * j - m + n
                        ix = ix * (ix + 1) // 2 + l + 1 - m - 2 * i
                        ilm = (1 + l - m) if (n % 2 == 1) else (1 + l + m)
                        tr[ix - 1, ilm - 1] += cmkij * cs[m, n]
    return tr.T.copy()
