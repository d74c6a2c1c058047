"""CPU checks of the collision-response oracle (oracle/collide.py): NumPy's
summation order restated bit for bit, the sweep geometry, and the
conservation laws of the bounce and merge restatements
(film_producer.py:707-1019)."""
import numpy as np

from oracle import collide as oc


def test_pairwise_sum_is_numpys_order():
    rng = np.random.default_rng(0)
    for n in list(range(0, 40)) + [63, 64, 65, 127, 128, 129, 200, 255, 256, 1000, 1031]:
        a = rng.normal(0, 1, n) * 10.0 ** rng.uniform(-8, 8, n)
        assert oc.np_pairwise_sum(a) == a.sum(), n


def _scene():
    # star, one planet at (1, 0), asteroids with known fates
    n = 8
    x = np.zeros(n, np.float32); y = np.zeros(n, np.float32)
    vx = np.zeros(n, np.float32); vy = np.zeros(n, np.float32)
    rr = np.zeros(n, np.float32)
    mass = np.zeros(n)
    is_ast = np.ones(n, np.uint8); is_ast[:2] = 0
    vis = np.ones(n, np.uint8)
    mass[0], rr[0] = 1.0, 0.00465
    x[1], mass[1], rr[1] = 1.0, 3e-6, 4.3e-5
    px = x.copy(); py = y.copy()
    # 2: crossed the planet between the previous and this sample
    x[2], y[2], px[2], py[2] = 1.0, 0.001, 1.0, -0.001
    # 3: will reach it within dt (extrapolated segment)
    x[3], y[3], vx[3], vy[3] = 1.0, -0.002, 0.0, 1.0
    px[3], py[3] = 1.0, -0.002
    # 4: far away, slow
    x[4], y[4], px[4], py[4], vx[4] = 2.5, 0.0, 2.5, 0.0, 0.1
    # 5: would cross, but invisible
    x[5], y[5], px[5], py[5] = 1.0, 0.001, 1.0, -0.001
    vis[5] = 0
    # 6: runaway (far above escape speed)
    x[6], y[6], vx[6], px[6] = 3.0, 0.0, 500.0, 3.0
    # 7: at rest at 2 AU
    x[7], px[7] = 2.0, 2.0
    mass[2:] = 1e-12
    return x, y, vx, vy, px, py, rr, vis, is_ast, mass


def test_sweep_finds_the_crossings_and_the_runaway():
    x, y, vx, vy, px, py, rr, vis, is_ast, mass = _scene()
    pairs, run = oc.merge_sweep(x, y, vx, vy, px, py, rr, vis, is_ast, mass, np.array([0, 1]), 0.01)
    got = {(a, b) for a, b, _ in pairs}
    assert (1, 2) in got and (1, 3) in got and (1, 5) not in got and (1, 4) not in got
    fr = {(a, b): f for a, b, f in pairs}
    assert -1.0 <= fr[(1, 2)] <= 0.0          # before this sample
    assert 0.0 <= fr[(1, 3)] <= 1.0           # after it
    assert run is not None and list(run) == [6]
    # row-major order: massive 0 rows before massive 1 rows, bodies ascending
    assert pairs == sorted(pairs, key=lambda p: ([0, 1].index(p[0]), p[1]))


def test_bounce_keeps_one_hit_per_body_and_conserves_momentum():
    rng = np.random.default_rng(3)
    n = 60
    x = rng.uniform(0, 1e-3, n).astype(np.float32)
    y = rng.uniform(0, 1e-3, n).astype(np.float32)
    vx = rng.normal(0, 1.0, n).astype(np.float32)
    vy = rng.normal(0, 1.0, n).astype(np.float32)
    rr = np.full(n, 2e-4)
    mass = rng.uniform(1e-12, 1e-11, n)
    hi = rng.integers(0, n, 200)
    hj = rng.integers(0, n, 200)
    keep = hi != hj
    hi, hj = hi[keep], hj[keep]
    k = oc.bounce_filter(hi, hj)
    seen = set()
    for t in k:
        assert hi[t] not in seen and hj[t] not in seen
        seen |= {hi[t], hj[t]}
    res = oc.bounce_deltas(x, y, vx, vy, rr, mass, hi, hj, 0.01)
    assert res is not None
    a, b, touched, d = res
    assert np.all(np.diff(touched) > 0)
    # impulses are equal and opposite: sum m dv = 0
    p = (mass[touched][:, None] * d[:, 2:4]).sum(0)
    scale = (mass[touched][:, None] * np.abs(d[:, 2:4])).sum()
    assert np.abs(p).max() <= 1e-12 * scale


def test_merges_conserve_mass_and_momentum():
    n = 4
    sample = np.zeros(4 * n, np.float32)
    sample[0:n] = [1.0, 1.00001, 3.0, 4.0]
    sample[2 * n:3 * n] = [0.0, 2.0, 0.0, 0.0]
    mass = np.array([3e-6, 1e-9, 1e-9, 1e-9])
    vis = np.ones(n, np.uint8)
    rr = np.array([4e-5, 1e-6, 1e-6, 1e-6])
    is_ast = np.array([0, 1, 1, 1], bool)
    star = np.zeros(n, bool)
    m01 = mass[0] + mass[1]
    p0 = (mass * sample[2 * n:3 * n]).sum()       # bodies 2, 3 are at rest
    ev, states, deact, sh = oc.apply_merges(sample, n, [(0, 1, -0.5)], np.array([3]), mass, vis, rr, is_ast, star)
    assert sh is None and deact == [1, 3]
    a, nx, ny, nvx, nvy, m, r = states[0]
    assert a == 0 and m == m01                    # the heavier body takes both masses
    assert abs(m * nvx - p0) <= 1e-15 * abs(p0)
    assert abs(r - (4e-5 ** 3 + 1e-6 ** 3) ** (1 / 3)) <= 1e-18
    assert [e[3] for e in ev] == [0, 2]


def test_fast_body_impact_stops_for_the_shatter():
    n = 2
    sample = np.zeros(4 * n, np.float32)
    sample[2 * n:3 * n] = [0.0, 1000.0]
    mass = np.array([1e-6, 1e-7])
    ev, states, deact, sh = oc.apply_merges(sample, n, [(0, 1, 0.0)], None, mass, np.ones(n, np.uint8),
                                            np.array([1e-5, 1e-5]), np.zeros(n, bool), np.zeros(n, bool))
    assert sh == (0, 1, 0.0) and not states and mass[1] == 1e-7


# ---------------------------------------------------------------- pinned by the reference's own outputs
# tests/golden/make_golden.py ran producer_main's analyze_merge, bounce_deltas
# and apply_merges (film_producer.py:707-1019; closures run from their own
# code objects) on the scenes below; the oracle must reproduce them exactly.

def test_sweep_matches_reference_golden(load_golden):
    g = load_golden("collide_sweep.npz")
    m_idx = np.arange(int(g["n_m"]), dtype=np.int64)
    px, py = g["x0"], g["y0"]
    for k in range(2):
        gx, gy = g[f"x{k}"], g[f"y{k}"]
        pairs, run = oc.merge_sweep(gx, gy, g[f"vx{k}"], g[f"vy{k}"], px if k else gx, py if k else gy, g["rr"],
                                    g["vis"], g["is_ast"], g["mass"], m_idx, float(g["dt_years"]), G=float(g["G"]))
        got = np.array([(a, b) for a, b, _ in pairs], np.int64).reshape(-1, 2)
        assert np.array_equal(got, g[f"pairs{k}"])
        assert np.array_equal(np.array([f for _, _, f in pairs]), g[f"frac{k}"])
        assert np.array_equal(np.asarray(run if run is not None else [], np.int64), g[f"run{k}"])
        assert len(got) > 100 and len(g[f"run{k}"]) > 10


import pytest  # noqa: E402


@pytest.mark.parametrize("scene", ["clump", "massless", "cases"])
def test_bounce_matches_reference_golden(load_golden, scene):
    g = load_golden(f"collide_bounce_{scene}.npz")
    s = g["sample"]
    n = len(g["mass"])
    with np.errstate(invalid="ignore", divide="ignore"):
        res = oc.bounce_deltas(s[0:n], s[n:2 * n], s[2 * n:3 * n], s[3 * n:4 * n], g["rr"], g["mass"], g["hit_i"],
                               g["hit_j"], float(g["raster_days"]) / 365.25)
    if "none" in g:
        assert res is None
        return
    hi, hj, touched, d = res
    assert np.array_equal(hi, g["kept_i"]) and np.array_equal(hj, g["kept_j"])
    assert np.array_equal(touched, g["touched"])
    assert np.array_equal(d, g["deltas"], equal_nan=True)


@pytest.mark.parametrize("scene", ["chain", "chain_noshatter", "shatter"])
def test_merges_match_reference_golden(load_golden, scene):
    g = load_golden(f"collide_merges_{scene}.npz")
    n = len(g["mass0"])
    mass, vis, rr = g["mass0"].copy(), g["vis0"].copy(), g["rr0"].copy()
    pairs = [(int(a), int(b), float(f)) for (a, b), f in zip(g["pairs"], g["frac"])]
    runs = g["runaways"] if len(g["runaways"]) or scene != "shatter" else None
    contact = {int(k): float(v) for k, v in g["contact"]}
    k_ev = int(g["k_ev"])
    ev, states, deact, sh = oc.apply_merges(g["sample"], n, pairs, runs, mass, vis, rr, g["is_ast"], g["star"],
                                            k_ev=k_ev, contact=contact, shatter=bool(g["shatter"]))
    calls = eval(str(g["calls"]))                       # the reference's recorded sim calls, in order
    want_states = [c[1:] for c in calls if c[0] == "state"]
    want_radius = [c[1:] for c in calls if c[0] == "radius"]
    want_off = [c[1] for c in calls if c[0] == "off"]
    assert [s[:6] for s in states] == [tuple(w) for w in want_states]
    assert [(s[0], s[6]) for s in states] == [tuple(w) for w in want_radius]
    assert deact == want_off
    events = eval(str(g["events"]))                     # (a, b, new_mass, kind, k_ev, x, y, frac)
    assert [(e[0], e[1], e[2], e[3], e[5], e[6], e[4]) for e in ev] == \
        [(a, b, m, kd, x, y, fr) for a, b, m, kd, _k, x, y, fr in events]
    assert np.array_equal(mass, g["mass1"]) and np.array_equal(vis, g["vis1"]) and np.array_equal(rr, g["rr1"])
    if int(g["shatter_flag"]):
        a, b, fr = sh
        assert (a, b) == tuple(int(v) for v in g["shatter_ab"]) and int(g["dumps"]) == 1
        assert 0.0 + (k_ev + 1 + fr) * 0.5 == float(g["shatter_t"])
    else:
        assert sh is None
