"""Host-side logic of the broadphase (no GPU): the cell hash and the
percentile arithmetic of the search cell, against NumPy and the reference."""
import numpy as np
import pytest
import torch

from solarsystemsimulator_b200 import broadphase as bp


def test_cell_hash_wraps_like_int64():
    cx = np.array([0, 1, -1, 2**40, -(2**40), 123456789012], np.int64)
    cy = np.array([0, -1, 1, 2**41, 7, -987654321098], np.int64)
    k = bp._zellschluessel(cx, cy)
    # reference: cx * int64(73856093) ^ cy * int64(19349663) with wrap-around
    want = [((int(a) * 73856093) ^ (int(b) * 19349663)) & (2**64 - 1) for a, b in zip(cx, cy)]
    want = [w - 2**64 if w >= 2**63 else w for w in want]
    assert k.tolist() == want


@pytest.mark.parametrize("seed", range(6))
def test_percentile_matches_numpy_on_f32(seed):
    """percentile_linear reproduces np.percentile(f32 speeds, 95), the
    reference's v95 (film_producer.py:357), bit for bit: every size from 1
    to 60 and a few large ones, ties, NaN."""
    rng = np.random.default_rng(seed)
    sizes = list(range(1, 61)) + [1000, 4097, 200_000]
    for n in sizes:
        v = np.hypot(rng.normal(0, 3, n), rng.normal(0, 3, n)).astype(np.float32)
        if seed == 1:
            v = np.round(v, 1).astype(np.float32)            # ties
        if seed == 2 and n > 3:
            v[n // 2] = np.nan
        for q in (95, 50, 0, 100, 99.9):
            want = np.percentile(v, q)
            got = bp.percentile_linear(np.sort(v), q)
            assert (np.isnan(want) and np.isnan(got)) or got == float(want), (n, q, got, want)
            # a tensor takes the one-readback path
            got_t = bp.percentile_linear(torch.from_numpy(np.sort(v)), q)
            assert (np.isnan(want) and np.isnan(got_t)) or got_t == float(want), (n, q, got_t, want)
