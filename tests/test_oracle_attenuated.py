"""The oracle's range-separated exchange (the attenuated operator
erf(mu r12)/r12 of Dalton's HFXMU pass, DALTON/abacus/her2her.F:344-353,
herdirect.F:792-835) pinned against closed forms and limits (CPU only):

* (ss|ss): the interaction of two Gaussian charge clouds through
  erf(mu r)/r is erf(sqrt(a') R)/R with 1/a' = 1/p + 1/q + 1/mu^2 (the
  form of Dalton's long-range MC-srDFT branch, her2her.F:417-431);
* mu -> infinity gives the 1/r12 integrals, for every angular momentum;
* mu -> 0: erf(mu r)/r = 2 mu/sqrt(pi) (1 - mu^2 r^2/3 + ...), so the
  integral over 2 mu/sqrt(pi) tends to the product of the bra and ket
  overlap distributions' integrals, for every angular momentum;
* the two-pass HERFCK_1 Fock matrix at mu -> infinity equals the one-pass
  build with HFXFAC + HFXATT."""
import math

import numpy as np
import pytest

from dalton_b200 import molecules
from dalton_b200.basis import build_basis


def _random_quartet(seed):
    rng = np.random.default_rng(seed)
    return rng.uniform(0.3, 2.5, 4), rng.normal(scale=0.8, size=(4, 3))


def _cart(l):
    return [(x, y, l - x - y) for x in range(l, -1, -1) for y in range(l - x, -1, -1)]


def _overlap_1d(i, j, a, b, A, B):
    """Integral of (x-A)^i (x-B)^j exp(-a (x-A)^2 - b (x-B)^2) by Gauss-Hermite
    quadrature (exact for these polynomial degrees)."""
    p = a + b
    P = (a * A + b * B) / p
    pref = math.exp(-a * b / p * (A - B) ** 2)
    x, w = np.polynomial.hermite.hermgauss(20)
    t = x / math.sqrt(p) + P
    return pref / math.sqrt(p) * float(np.sum(w * (t - A) ** i * (t - B) ** j))


def _pair_integral(la, lb, a, b, A, B):
    out = np.zeros((len(_cart(la)), len(_cart(lb))))
    for i, ci in enumerate(_cart(la)):
        for j, cj in enumerate(_cart(lb)):
            out[i, j] = np.prod([_overlap_1d(ci[k], cj[k], a, b, A[k], B[k]) for k in range(3)])
    return out


def test_ss_closed_form(orc):
    for seed in range(5):
        e, c = _random_quartet(seed)
        a, b, cc, d = e
        A, B, C, D = c
        p, q = a + b, cc + d
        P, Q = (a * A + b * B) / p, (cc * C + d * D) / q
        K = math.exp(-a * b / p * np.sum((A - B) ** 2) - cc * d / q * np.sum((C - D) ** 2))
        R = float(np.linalg.norm(P - Q))
        for mu in (0.0, 0.11, 0.4, 1.7, 9.0):
            inv = 1 / p + 1 / q + (1 / mu ** 2 if mu > 0 else 0.0)
            ref = (math.pi / p) ** 1.5 * (math.pi / q) ** 1.5 * K * math.erf(math.sqrt(1 / inv) * R) / R
            got = orc.prim_eri((0, 0, 0, 0), e, c, mu)[0, 0, 0, 0]
            assert abs(got - ref) <= 1e-14 * abs(ref)


@pytest.mark.parametrize("ls", [(1, 0, 0, 0), (1, 1, 1, 0), (2, 1, 2, 0), (3, 2, 1, 1), (3, 3, 2, 0)])
def test_large_mu_gives_coulomb(orc, ls):
    e, c = _random_quartet(sum(ls))
    full = orc.prim_eri(ls, e, c, 0.0)
    att = orc.prim_eri(ls, e, c, 1e6)
    assert np.abs(att - full).max() <= 1e-9 * np.abs(full).max()


@pytest.mark.parametrize("ls", [(1, 0, 1, 0), (2, 1, 1, 1), (3, 0, 2, 1)])
def test_small_mu_gives_overlap_product(orc, ls):
    e, c = _random_quartet(7 + sum(ls))
    mu = 1e-4
    att = orc.prim_eri(ls, e, c, mu) / (2 * mu / math.sqrt(math.pi))
    sab = _pair_integral(ls[0], ls[1], e[0], e[1], c[0], c[1])
    scd = _pair_integral(ls[2], ls[3], e[2], e[3], c[2], c[3])
    ref = np.einsum("ab,cd->abcd", sab, scd)
    assert np.abs(att - ref).max() <= 1e-6 * np.abs(ref).max()


def test_fock_two_pass_limits(orc):
    bs = build_basis(molecules.water_cluster(2, seed=3), "cc-pVDZ")
    rng = np.random.default_rng(9)
    d = rng.normal(size=(bs.nbf, bs.nbf)) * 0.05
    d = d + d.T
    # no attenuated pass
    f0 = orc.fock_attenuated(bs, d, 13, 0.3, 1e-12, 0.0, 0.7)
    assert np.abs(f0 - orc.fock(bs, d, 13, 0.3, 1e-12)).max() < 1e-13
    # mu -> infinity: the attenuated exchange is the full exchange
    big = orc.fock_attenuated(bs, d, 13, 0.25, 1e-12, 1e8, 0.5)
    assert np.abs(big - orc.fock(bs, d, 13, 0.75, 1e-12)).max() < 1e-8
    # Coulomb-only IFCTYP: the attenuated pass still adds exchange (FCKCON's IY = 2)
    j_plus = orc.fock_attenuated(bs, d, 11, 1.0, 1e-12, 1e8, 1.0)
    assert np.abs(j_plus - orc.fock(bs, d, 13, 1.0, 1e-12)).max() < 1e-8
    # a finite mu lies between: smaller exchange than the full operator
    mid = orc.fock_attenuated(bs, d, 13, 0.0, 1e-12, 0.33, 1.0)
    kfull = orc.fock(bs, d, 13, 1.0, 1e-12) - orc.fock(bs, d, 11, 1.0, 1e-12)
    katt = mid - orc.fock(bs, d, 11, 1.0, 1e-12)
    assert 0.0 < np.abs(katt).max() < np.abs(kfull).max()
    assert np.sum(d * katt) / np.sum(d * kfull) > 0.0


def test_attenuated_exchange_is_symmetric_in_its_permutations(orc):
    """The attenuated primitive block keeps the 8-fold permutation symmetry."""
    e, c = _random_quartet(21)
    ls = (2, 1, 1, 0)
    g = orc.prim_eri(ls, e, c, 0.6)
    perm = [1, 0, 3, 2]
    h = orc.prim_eri([ls[i] for i in perm], e[perm], c[perm], 0.6)
    assert np.abs(g - h.transpose(1, 0, 3, 2)).max() < 1e-14 * np.abs(g).max()
    swap = [2, 3, 0, 1]
    k = orc.prim_eri([ls[i] for i in swap], e[swap], c[swap], 0.6)
    assert np.abs(g - k.transpose(2, 3, 0, 1)).max() < 1e-13 * np.abs(g).max()
