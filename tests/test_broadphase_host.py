"""Host-side logic of the broadphase (no GPU): cell hash, stripe bounds and
the stripe load regulator, against the reference's behaviour."""
import numpy as np

from solarsystemsimulator_b200 import broadphase as bp


def test_cell_hash_wraps_like_int64():
    cx = np.array([0, 1, -1, 2**40, -(2**40), 123456789012], np.int64)
    cy = np.array([0, -1, 1, 2**41, 7, -987654321098], np.int64)
    k = bp._zellschluessel(cx, cy)
    # reference: cx * int64(73856093) ^ cy * int64(19349663) with wrap-around
    want = [((int(a) * 73856093) ^ (int(b) * 19349663)) & (2**64 - 1) for a, b in zip(cx, cy)]
    want = [w - 2**64 if w >= 2**63 else w for w in want]
    assert k.tolist() == want


def test_stripes_cover_the_line():
    g = np.random.default_rng(1).normal(size=1000)
    assert bp._streifengrenzen(g, [1.0]) == [(-np.inf, np.inf)]
    s = bp._streifengrenzen(g, [0.25, 0.25, 0.5])
    assert s[0][0] == -np.inf and s[-1][1] == np.inf
    assert all(s[i][1] == s[i + 1][0] for i in range(len(s) - 1))


def test_load_regulator_converges_and_respects_floor():
    # a skewed load narrows the loaded stripe; shares stay normalised and >= 5 %
    a = [0.5, 0.5]
    for _ in range(30):
        dichte = [4.0, 1.0]                     # stripe 0 is four times denser
        last = [d * x for d, x in zip(dichte, a)]
        a = bp._lastanteile(a, last)
    assert abs(sum(a) - 1.0) < 1e-12
    assert a[0] < 0.3 and a[1] > 0.7
    b = bp._lastanteile([0.9, 0.1], [1, 10**9])
    assert min(b) >= bp.LAST_MIN_ANTEIL - 1e-12 and abs(sum(b) - 1) < 1e-12
    assert bp._lastanteile([0.5, 0.5], [0, 0]) == [0.5, 0.5]
