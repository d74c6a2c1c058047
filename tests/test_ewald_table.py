"""The host-built table of the Ewald real-space factor g(x) = erfc(x) +
2 x exp(-x^2) / sqrt(pi) (ewald.cu, read through sss_ewald_gtab; host code,
no device): the quintic pieces reproduce g to 1e-15 (absolute; g(0) = 1)
over the whole range the real-space sum uses, and join across interval
boundaries."""
import ctypes
import math

import numpy as np
import pytest

scipy_special = pytest.importorskip("scipy.special")


def _table():
    from solarsystemsimulator_b200 import _lib
    lib = _lib.load()
    cap = 64 * 1024
    buf = (ctypes.c_double * cap)()
    n = ctypes.c_int()
    h = ctypes.c_double()
    assert lib.sss_ewald_gtab(buf, cap, ctypes.byref(n), ctypes.byref(h)) == 0
    return np.frombuffer(buf, np.float64, n.value * 6).reshape(n.value, 6).copy(), n.value, h.value


def _piece(tab, k, h, x):
    d = x - (k + 0.5) * h
    a = tab[k]
    r = a[:, 5]
    for j in (4, 3, 2, 1, 0):
        r = a[:, j] + d * r
    return r


def test_table_matches_erfc():
    tab, n, h = _table()
    assert n * h >= 6.0 - 1e-12             # covers alpha r_cut up to 6
    sp = 2.0 / math.sqrt(math.pi)
    x = np.concatenate([np.random.default_rng(0).uniform(0.0, n * h, 400_000), np.arange(n + 1) * h])
    x = np.minimum(x, n * h)
    k = np.minimum((x / h).astype(np.int64), n - 1)
    ref = scipy_special.erfc(x) + sp * x * np.exp(-x * x)
    assert np.max(np.abs(_piece(tab, k, h, x) - ref)) < 1e-15


def test_pieces_join():
    tab, n, h = _table()
    kk = np.arange(1, n)
    edges = kk * h
    left = _piece(tab, kk - 1, h, edges)
    right = _piece(tab, kk, h, edges)
    assert np.max(np.abs(left - right)) < 1e-15
