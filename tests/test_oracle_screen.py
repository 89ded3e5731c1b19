"""The oracle's restatement of Dalton's density screen (IFTHRS, ICEDIF) and
its class-stratified timing of the CPU baseline (CPU only)."""
import numpy as np

from dalton_b200 import molecules
from dalton_b200.basis import build_basis


def _water_pair():
    return build_basis(molecules.water_cluster(2, seed=3), "cc-pVDZ")


def _density(n, seed, scale=0.05):
    rng = np.random.default_rng(seed)
    d = rng.normal(size=(n, n)) * scale
    return d + d.T


def test_screen_off_is_the_plain_build(orc):
    """IFTHRS >= 16 turns the screen off (DALTON/abacus/her2drv.F:520-540):
    the result is the unscreened build (up to the order in which the threads'
    partial matrices are summed)."""
    bs = _water_pair()
    d = _density(bs.nbf, 1)
    ref = orc.fock(bs, d, 13, 1.0, 1e-12)
    for ifthrs in (16, 20):
        f, c = orc.fock_screened(bs, d, 13, 1.0, 1e-12, ifthrs=ifthrs, icedif=3)
        assert np.abs(f - ref).max() < 1e-13
        assert c["skipped_screen"] == 0 and c["dropped_coulomb"] == 0 and c["dropped_exchange"] == 0


def test_screen_error_tracks_threshold(orc):
    """The error the screen leaves falls with IFTHRS, and the screen skips
    fewer quartets as it tightens."""
    bs = _water_pair()
    d = _density(bs.nbf, 2, scale=0.01)
    ref = orc.fock(bs, d, 13, 1.0, 1e-12)
    errs, skips = [], []
    for ifthrs in (6, 8, 10, 12):
        f, c = orc.fock_screened(bs, d, 13, 1.0, 1e-12, ifthrs=ifthrs, icedif=3)
        errs.append(np.abs(f - ref).max())
        skips.append(c["skipped_screen"])
        assert errs[-1] < 1e3 * 10.0 ** -ifthrs
    assert errs == sorted(errs, reverse=True)
    assert skips == sorted(skips, reverse=True) and skips[0] > 0


def test_ifthrs_below_four_means_fourteen(orc):
    bs = _water_pair()
    d = _density(bs.nbf, 3)
    f3, _ = orc.fock_screened(bs, d, 13, 1.0, 1e-12, ifthrs=3)
    f14, _ = orc.fock_screened(bs, d, 13, 1.0, 1e-12, ifthrs=14)
    assert np.abs(f3 - f14).max() < 1e-13


def test_zero_density_blocks_are_skipped_exactly(orc):
    """Quartets whose density bound is exactly zero contribute nothing: with a
    density on one water only the result equals the full evaluation."""
    bs = _water_pair()
    d = np.zeros((bs.nbf, bs.nbf))
    atoms = bs.ao_atom()
    idx = np.where(atoms < 3)[0]
    d[np.ix_(idx, idx)] = _density(len(idx), 4)
    f, c = orc.fock_screened(bs, d, 13, 1.0, 1e-12, ifthrs=20)
    ref = orc.fock(bs, d, 13, 1.0, 1e-12)
    assert c["skipped_zero"] > 0
    assert np.abs(f - ref).max() < 1e-13


def test_hash_sample_is_a_fixed_uniform_subset(orc):
    """The CPU-baseline sample: k = 0 evaluates every significant quartet; a
    2^-k sample holds about that fraction of them, the same subset every
    time."""
    bs = _water_pair()
    d = _density(bs.nbf, 5)
    n0, _, tot = orc.fock_hash_sample(bs, d, 0)
    _, nq = orc.fock_sampled(bs, d, 1, 0, 1e-12)
    assert n0 == tot == nq
    n4, s4, tot4 = orc.fock_hash_sample(bs, d, 4)
    assert tot4 == tot
    assert abs(n4 - tot / 16) < 5 * (tot / 16) ** 0.5
    assert orc.fock_hash_sample(bs, d, 4)[0] == n4
    assert s4 > 0.0
