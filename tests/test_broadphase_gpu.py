"""GPU broadphase: the colliding-pair list must be bit-exact.

Against the reference's own `_hits` outputs (golden fixtures: same pairs,
same (i, j) orientation, same order, same candidate count) and against the
CPU oracle on further seeded scenes (dense clumps, hidden bodies, stripes,
degenerate inputs). Mirrors the reference's test_erkennung_streifen.py.
"""
import numpy as np
import pytest

from oracle import broadphase as obp

pytestmark = pytest.mark.gpu

SCENES = ["wolke", "klumpen", "zwei_wolken", "auf_der_grenze"]


def _bp():
    from solarsystemsimulator_b200 import broadphase as bp
    return bp


def _same(res, ref):
    if ref is None or res is None:
        return res is None and ref is None
    return np.array_equal(res[0], ref[0]) and np.array_equal(res[1], ref[1])


@pytest.mark.parametrize("scene", SCENES)
def test_hits_bit_exact_against_reference_golden(load_golden, scene):
    bp = _bp()
    g = load_golden(f"broadphase_{scene}.npz")
    karte = bp.Erkennungskarte(0, np.ones(len(g["x"]), bool), -np.inf, np.inf)
    karte.stammdaten(np.ones(len(g["x"]), np.uint8), g["rr"])
    res, cand = karte.bounce_hits(g["x"], g["y"], g["vx"], g["vy"], float(g["dt_y"]), float(g["h"]),
                                  float(g["halo"]))
    assert cand == int(g["n_cand"])
    assert _same(res, (g["hit_i"], g["hit_j"]))


@pytest.mark.parametrize("scene", SCENES)
def test_stripe_union_equals_single_card(load_golden, scene):
    # test_erkennung_streifen.py: the union of stripe hits is exactly the full set
    bp = _bp()
    g = load_golden(f"broadphase_{scene}.npz")
    n = len(g["x"])
    karte = bp.Erkennungskarte(0, np.ones(n, bool), -np.inf, np.inf)
    karte.stammdaten(np.ones(n, np.uint8), g["rr"])
    full = set(zip(g["hit_i"].tolist(), g["hit_j"].tolist()))
    for k in (2, 3, 5):
        got, count = set(), 0
        for lo, hi in g[f"stripes{k}_bounds"]:
            karte.streifen(lo, hi)
            res, _ = karte.bounce_hits(g["x"], g["y"], g["vx"], g["vy"], float(g["dt_y"]), float(g["h"]),
                                       float(g["halo"]))
            if res is not None:
                part = set(zip(res[0].tolist(), res[1].tolist()))
                assert not (got & part)
                got |= part
                count += len(res[0])
        assert got == full and count == int(g[f"stripes{k}_count"])


def _scene(seed, n, kind):
    rng = np.random.default_rng(seed)
    if kind == "clumps":
        cen = rng.uniform(1, 5, (8, 2))
        which = rng.integers(0, 8, n)
        x = cen[which, 0] + rng.normal(0, 0.01, n)
        y = cen[which, 1] + rng.normal(0, 0.01, n)
        vx = rng.normal(0, 2, n); vy = rng.normal(5, 2, n)
        rr = 10 ** rng.uniform(-7, -4, n)
    else:
        x = rng.uniform(-5, 5, n); y = rng.uniform(-5, 5, n)
        vx = rng.normal(0, 6, n); vy = rng.normal(0, 6, n)
        rr = np.full(n, 2e-3)
    return [a.astype(np.float32) for a in (x, y, vx, vy, rr)]


@pytest.mark.parametrize("kind,n", [("clumps", 60000), ("uniform", 120000)])
def test_hits_bit_exact_against_oracle(kind, n):
    bp = _bp()
    x, y, vx, vy, rr = _scene(5, n, kind)
    rng = np.random.default_rng(6)
    is_ast = rng.random(n) > 0.02
    vis = (rng.random(n) > 0.02).astype(np.uint8)
    dt = 0.5 / 365.25
    v95 = float(np.percentile(np.hypot(vx, vy), 95))
    h = max(1e-4, 2.0 * v95 * dt)
    halo = 2.0 * h + 2.0 * float(rr.max())
    ref, cand_ref = obp.hits(x, y, vx, vy, rr, dt, h, halo, is_ast=is_ast, vis=vis)
    res, cand = bp.bounce_hits(x, y, vx, vy, dt, h, halo, rr=rr, is_ast=is_ast, vis=vis)
    assert cand == cand_ref
    assert _same(res, ref)
    # a stripe with a finite window
    lo, hi = np.percentile(x, [30, 60])
    ref, cand_ref = obp.hits(x, y, vx, vy, rr, dt, h, halo, is_ast=is_ast, vis=vis, lo=lo, hi=hi)
    res, cand = bp.bounce_hits(x, y, vx, vy, dt, h, halo, rr=rr, is_ast=is_ast, vis=vis, lo=lo, hi=hi)
    assert cand == cand_ref and _same(res, ref)


def test_degenerate_inputs():
    bp = _bp()
    one = np.ones(1, np.float32)
    assert bp.bounce_hits(one, one, one, one, 0.01, 0.1, 0.2, rr=one) == (None, 0)
    x = np.zeros(5, np.float32)
    hidden = np.zeros(5, np.uint8)
    assert bp.bounce_hits(x, x, x, x, 0.01, 0.1, 0.2, rr=x + 1e-3, vis=hidden) == (None, 0)
    # all bodies in one cell: every pair is a candidate and touches
    res, cand = bp.bounce_hits(x, x, x, x, 0.01, 0.1, 0.2, rr=x + 1e-3)
    ref, cref = obp.hits(x, x, x, x, x + 1e-3, 0.01, 0.1, 0.2)
    assert cand == cref and _same(res, ref) and len(res[0]) == 10


def test_more_hits_than_the_first_buffer():
    # a dense clump with far more hits than bodies exercises the capacity retry
    bp = _bp()
    rng = np.random.default_rng(8)
    n = 3000
    x = (2 + rng.normal(0, 1e-4, n)).astype(np.float32)
    y = rng.normal(0, 1e-4, n).astype(np.float32)
    v = rng.normal(0, 1, n).astype(np.float32)
    rr = np.full(n, 1e-3, np.float32)
    res, cand = bp.bounce_hits(x, y, v, v, 0.001, 1e-3, 4e-3, rr=rr)
    ref, cref = obp.hits(x, y, v, v, rr, 0.001, 1e-3, 4e-3)
    assert cand == cref and _same(res, ref) and len(res[0]) > 4096


def test_colliding_cell_keys():
    """Cells (-34, 38) and (34, -38) have the same hash key at h = 0.01 AU,
    so their bodies share one key range, interleaved in body order: runs of
    a few bodies, tiles mixing two clusters 0.7 AU apart (where the line test
    may not skip), a neighbour range that holds both, and many pairs through
    the exact tests."""
    bp = _bp()
    A, B = np.int64(73856093), np.int64(19349663)
    assert (np.int64(-34) * A) ^ (np.int64(38) * B) == (np.int64(34) * A) ^ (np.int64(-38) * B)
    rng = np.random.default_rng(12)
    n = 4000
    h = 0.01
    side = rng.integers(0, 2, n)                       # interleaved body indices
    cx = np.where(side == 0, -34, 34) + 0.5
    cy = np.where(side == 0, 38, -38) + 0.5
    x = ((cx + rng.uniform(-0.45, 0.45, n)) * h).astype(np.float32)
    y = ((cy + rng.uniform(-0.45, 0.45, n)) * h).astype(np.float32)
    vx = rng.normal(0, 1e-2, n).astype(np.float32)
    vy = rng.normal(0, 1e-2, n).astype(np.float32)
    rr = np.full(n, 3e-5, np.float32)
    dt = 0.05
    halo = 2.0 * h + 2.0 * float(rr.max())
    ref, cref = obp.hits(x, y, vx, vy, rr, dt, h, halo)
    res, cand = bp.bounce_hits(x, y, vx, vy, dt, h, halo, rr=rr)
    assert cand == cref and _same(res, ref)
    assert ref is not None and len(ref[0]) > 0


def test_non_finite_and_far_bodies():
    """NaN positions and radii and bodies far from the origin: the line test
    never skips what the exact tests would keep."""
    bp = _bp()
    x, y, vx, vy, rr = _scene(9, 20000, "clumps")
    rng = np.random.default_rng(13)
    bad = rng.choice(len(x), 40, replace=False)
    x[bad[:10]] = np.nan
    vy[bad[10:20]] = np.nan
    rr[bad[20:30]] = np.nan
    far = bad[30:]
    x[far] = 3000.0 + rng.normal(0, 1e-3, len(far)).astype(np.float32)
    dt = 0.5 / 365.25
    v95 = float(np.nanpercentile(np.hypot(vx, vy), 95))
    h = max(1e-4, 2.0 * v95 * dt)
    halo = 2.0 * h + 2.0 * float(np.nanmax(rr))
    ref, cref = obp.hits(x, y, vx, vy, rr, dt, h, halo)
    res, cand = bp.bounce_hits(x, y, vx, vy, dt, h, halo, rr=rr)
    assert cand == cref and _same(res, ref)


@pytest.mark.parametrize("k,n", [(1, 10), (5_000, 200_000), (70_000, 3_000), (20_000, (1 << 30) - 1)])
def test_hit_order_on_the_device(k, n):
    """sss_broadphase_order sorts (offset, a, b) triples exactly as
    np.lexsort does, duplicates and the largest body index included."""
    import ctypes
    import torch
    from solarsystemsimulator_b200 import _lib
    rng = np.random.default_rng(k)
    h = np.stack([rng.integers(0, 5, k), rng.integers(0, n, k), rng.integers(0, n, k)], 1).astype(np.int32)
    h[: k // 10] = h[0]                                   # repeated triples
    h[-1, 1:] = n - 1
    d = torch.as_tensor(h).cuda()
    ctx = _lib.context(0)
    ctx.check(ctx.lib.sss_broadphase_order(ctx.ptr, d.data_ptr(), k, n, ctypes.c_void_p(_lib.stream_handle(0))))
    want = h[np.lexsort((h[:, 2], h[:, 1], h[:, 0]))]
    assert np.array_equal(d.cpu().numpy(), want)


def test_hit_order_rejects_bad_sizes():
    import ctypes
    from solarsystemsimulator_b200 import _lib
    ctx = _lib.context(0)
    assert ctx.lib.sss_broadphase_order(ctx.ptr, None, -1, 10, None) == _lib.SSS_ERR_ARG
    assert ctx.lib.sss_broadphase_order(ctx.ptr, None, 5, 10, None) == _lib.SSS_ERR_ARG
    assert ctx.lib.sss_broadphase_order(ctx.ptr, None, 0, 1 << 30, None) == _lib.SSS_ERR_ARG
    # more hits than the 32-bit sort index holds (checked before any access)
    assert ctx.lib.sss_broadphase_order(ctx.ptr, ctypes.c_void_p(16), (1 << 31), 10, None) == _lib.SSS_ERR_ARG


def _clouds_scene(n_per_cloud=40_000):
    """The asteroid-cloud configuration's broadphase input, built as
    tests/golden/make_golden.py builds it for the reference's `_hits`."""
    import hashlib
    from solarsystemsimulator_b200 import workloads
    w = workloads.asteroid_clouds(n_per_cloud=n_per_cloud)
    a = np.flatnonzero(w["is_ast"] != 0)
    f = [np.ascontiguousarray(v, dtype=np.float32) for v in
         (w["pos"][0, a], w["pos"][1, a], w["vel"][0, a], w["vel"][1, a], w["radius"][a])]
    d = hashlib.sha256()
    for v in f:
        d.update(v.tobytes())
    return f, d.hexdigest()


def test_asteroid_clouds_200k_bit_exact_against_reference(load_golden):
    """The configured scene (200,000 asteroids in 5 Gaussian clouds, 3.1e9
    candidate pairs): pairs, order and candidate count equal to the
    reference's own `_hits` on it; h and the halo come from bounce_suche and
    equal the reference's (film_producer.py:357-362)."""
    bp = _bp()
    g = load_golden("broadphase_asteroid_clouds_200k.npz")
    f, digest = _clouds_scene(int(g["n_per_cloud"]))
    assert digest == str(g["digest"])                  # the same f32 input as the reference saw
    x, y, vx, vy, rr = f
    n = len(x)
    karte = bp.Erkennungskarte(0, np.ones(n, bool), -np.inf, np.inf)
    karte.stammdaten(np.ones(n, np.uint8), rr)
    res, cand, h, shares = bp.bounce_suche([karte], None, [(x, y, vx, vy)], float(g["dt"]), float(rr.max()))
    assert h == float(g["h"]) and shares == [1.0]
    assert cand == int(g["n_cand"])
    assert _same(res, (g["hit_i"].astype(np.int64), g["hit_j"].astype(np.int64)))
    assert len(res[0]) == 5192


def test_bounce_suche_matches_reference_arithmetic():
    """bounce_suche's cell size from the living asteroids' speeds (hidden
    bodies and non-asteroids excluded) equals max(1e-4, 2 v95 dt) with v95 =
    np.percentile(np.hypot(f32, f32), 95), and its hits equal the oracle's."""
    bp = _bp()
    for seed, n in ((3, 50_000), (4, 7), (5, 2)):
        x, y, vx, vy, rr = _scene(seed, n, "clumps")
        rng = np.random.default_rng(seed)
        is_ast = rng.random(n) > 0.1
        vis = (rng.random(n) > 0.1).astype(np.uint8)
        if n == 2:
            is_ast[:] = True
            vis[:] = 1
        lebt = np.flatnonzero(is_ast & (vis != 0))
        dt = 0.5 / 365.25
        v95 = float(np.percentile(np.hypot(vx[lebt], vy[lebt]), 95))
        h_ref = max(1e-4, 2.0 * v95 * dt)
        karte = bp.Erkennungskarte(0, is_ast, -np.inf, np.inf)
        karte.stammdaten(vis, rr)
        res, cand, h, shares = bp.bounce_suche([karte], None, [(x, y, vx, vy)], dt, float(rr.max()))
        assert h == h_ref and shares == [1.0]
        ref, cref = obp.hits(x, y, vx, vy, rr, dt, h_ref, 2.0 * h_ref + 2.0 * float(rr.max()), is_ast=is_ast, vis=vis)
        assert cand == cref and _same(res, ref)


def test_one_alive_body_among_many():
    """Exactly one living asteroid among many bodies (hidden ones and
    non-asteroids around it, in the same cell): no pair, no candidate."""
    bp = _bp()
    n = 5000
    x = np.full(n, 1.0, np.float32)
    rr = np.full(n, 1e-3, np.float32)
    for is_ast, vis in ((np.zeros(n, bool), np.ones(n, np.uint8)), (np.ones(n, bool), np.zeros(n, np.uint8))):
        is_ast = is_ast.copy()
        vis = vis.copy()
        is_ast[1234] = True
        vis[1234] = 1
        ref = obp.hits(x, x, x, x, rr, 0.01, 0.1, 0.2, is_ast=is_ast, vis=vis)
        assert ref == (None, 0)
        assert bp.bounce_hits(x, x, x, x, 0.01, 0.1, 0.2, rr=rr, is_ast=is_ast, vis=vis) == (None, 0)
    # one alive body inside the stripe window, many outside it
    x2 = np.concatenate([np.full(n - 1, 50.0, np.float32), np.array([1.0], np.float32)])
    assert bp.bounce_hits(x2, x2, x2, x2, 0.01, 0.1, 0.2, rr=rr, lo=0.0, hi=2.0) == \
        obp.hits(x2, x2, x2, x2, rr, 0.01, 0.1, 0.2, lo=0.0, hi=2.0) == (None, 0)
