"""GPU parity of the collision response (sss_collide_sweep,
sss_collide_bounce, CollisionResponse) against oracle/collide.py, the
restatement of the reference's analyze_merge / bounce_deltas / apply_merges
(film_producer.py:707-1019).

Integer results (pairs, their order, runaways, kept and active hits,
touched bodies) must be identical; the f32 fractions bit-identical; the f64
deltas within 1e-12 relative (hypot is the one operation whose last bit may
differ between CUDA and the host C library).
"""
import numpy as np
import pytest
import torch

from oracle import collide as oc

pytestmark = pytest.mark.gpu


def _film(seed, n_per=3000, clouds=3, sigma=0.01, crossers=40, runaways=12, hidden=50):
    from solarsystemsimulator_b200.workloads import asteroid_clouds
    w = asteroid_clouds(n_per_cloud=n_per, n_clouds=clouds, seed=seed)
    rng = np.random.default_rng(seed + 1)
    pos = w["pos"][:2].copy()
    vel = w["vel"][:2] * 365.25                     # AU / yr, the film's units
    n = pos.shape[1]
    if sigma != 0.01:
        # tighter clouds: shrink about each cloud centre
        for c in range(clouds):
            s = slice(8 + c * n_per, 8 + (c + 1) * n_per)
            cen = pos[:, s].mean(1, keepdims=True)
            pos[:, s] = cen + (pos[:, s] - cen) * (sigma / 0.01)
    rr = w["radius"].copy()
    rr[0] = 0.00465
    rr[1:8] = 10 ** rng.uniform(-5, -4.3, 7)
    dt_y = 0.5 / 365.25
    prev = pos - vel * dt_y
    ast = np.flatnonzero(w["is_ast"])
    # asteroids whose last segment crosses a planet
    for j in rng.choice(ast, crossers, replace=False):
        k = int(rng.integers(1, 8))
        off = rng.normal(0, 1, 2)
        off *= 3 * rr[k] / np.linalg.norm(off)
        pos[:, j] = pos[:, k] + off
        prev[:, j] = pos[:, k] - off + rng.normal(0, rr[k] * 0.3, 2)
    # runaways
    fast = rng.choice(ast, runaways, replace=False)
    vel[:, fast] *= 60.0
    vis = np.ones(n, np.uint8)
    vis[rng.choice(ast, hidden, replace=False)] = 0
    g = np.stack([pos[0], pos[1], vel[0], vel[1]]).astype(np.float32)
    return {"g": g, "prev": prev.astype(np.float32), "rr": rr, "mass": w["mass"].copy(), "is_ast": w["is_ast"],
            "vis": vis, "dt_y": dt_y, "m_idx": np.arange(8)}


def _cr(f):
    from solarsystemsimulator_b200.collide import CollisionResponse
    return CollisionResponse(f["mass"], f["rr"], f["vis"], f["is_ast"], m_idx=f["m_idx"])


@pytest.mark.parametrize("seed", [11, 12])
def test_sweep_matches_oracle(seed):
    f = _film(seed)
    cr = _cr(f)
    g = torch.as_tensor(f["g"]).cuda()
    cr.prev = (torch.as_tensor(f["prev"][0]).cuda(), torch.as_tensor(f["prev"][1]).cuda())
    pairs, run = cr.analyze_merge(g, f["dt_y"])
    ref_pairs, ref_run = oc.merge_sweep(*f["g"], f["prev"][0], f["prev"][1], f["rr"].astype(np.float32), f["vis"],
                                        f["is_ast"], f["mass"], f["m_idx"], f["dt_y"])
    assert len(ref_pairs) >= 30
    assert pairs == ref_pairs
    assert ref_run is not None and run is not None and np.array_equal(run, ref_run)
    # the next sample sweeps from this one's positions
    g2 = f["g"].copy()
    g2[0:2] += g2[2:4] * np.float32(f["dt_y"])
    pairs2, run2 = cr.analyze_merge(torch.as_tensor(g2).cuda(), f["dt_y"])
    ref2, rrun2 = oc.merge_sweep(*g2, f["g"][0], f["g"][1], f["rr"].astype(np.float32), f["vis"], f["is_ast"],
                                 f["mass"], f["m_idx"], f["dt_y"])
    assert pairs2 == ref2
    assert (run2 is None and rrun2 is None) or np.array_equal(run2, rrun2)


def _bounce_case(seed, n_per=20000, sigma=0.002, massless=False):
    from solarsystemsimulator_b200 import broadphase as bp
    f = _film(seed, n_per=n_per, clouds=2, sigma=sigma, crossers=0, runaways=0, hidden=100)
    if massless:
        f["mass"][8:8 + n_per // 2] = 0.0
    g = f["g"]
    ast = f["is_ast"] != 0
    alive = ast & (f["vis"] != 0)
    speed = np.hypot(g[2][alive], g[3][alive]).astype(np.float64)
    h = max(1e-4, 2.0 * float(np.quantile(speed, 0.95)) * f["dt_y"])
    halo = 2.0 * h + 2.0 * float(f["rr"][ast].max())
    rr32 = f["rr"].astype(np.float32)
    buf, k, _ = bp.bounce_hits_device(*g, f["dt_y"], h, halo, rr=rr32, is_ast=f["is_ast"], vis=f["vis"])
    ref_hits, _ = bp.bounce_hits(*g, f["dt_y"], h, halo, rr=rr32, is_ast=f["is_ast"], vis=f["vis"])
    return f, buf, k, ref_hits


@pytest.mark.parametrize("massless", [False, True])
def test_bounce_matches_oracle(massless):
    f, buf, k, ref_hits = _bounce_case(21, massless=massless)
    assert k >= 200
    cr = _cr(f)
    res = cr.bounce_deltas(torch.as_tensor(f["g"]).cuda(), buf, k, f["dt_y"])
    ref = oc.bounce_deltas(*f["g"], f["rr"], f["mass"], ref_hits[0], ref_hits[1], f["dt_y"])
    assert res is not None and ref is not None
    hi, hj, touched, d = (t.cpu().numpy() for t in res)
    assert np.array_equal(hi, ref[0]) and np.array_equal(hj, ref[1])
    assert np.array_equal(touched, ref[2])
    # the reference's arithmetic gives NaN for a bounce of two massless bodies; so does this one
    assert np.allclose(d, ref[3], rtol=1e-12, atol=0.0, equal_nan=True)


def test_bounce_deltas_apply_on_the_device():
    from solarsystemsimulator_b200.nbody_kernel import NBodyCuda
    f, buf, k, _ = _bounce_case(22, n_per=8000, sigma=0.001)
    cr = _cr(f)
    g = torch.as_tensor(f["g"]).cuda()
    res = cr.bounce_deltas(g, buf, k, f["dt_y"])
    assert res is not None
    x, y, vx, vy = (f["g"][c].astype(np.float64) for c in range(4))
    sims = []
    for _ in range(2):
        sim = NBodyCuda([0])
        st = sim.load_state(x, y, vx, vy, f["mass"], f["vis"], f["is_ast"], f["rr"])
        sims.append((sim, st))
    cr.apply_bounce(*sims[0], res)
    sims[1][0].apply_deltas(sims[1][1], res[2].cpu().numpy(), res[3].cpu().numpy())
    a, b = sims[0][0].export_f64(sims[0][1]), sims[1][0].export_f64(sims[1][1])
    assert np.array_equal(a, b)
    assert not np.array_equal(a[:len(x)], x)


def test_merges_match_oracle_and_reach_the_simulation():
    from solarsystemsimulator_b200.nbody_kernel import NBodyCuda
    f = _film(31, n_per=2000, clouds=2, crossers=30, runaways=8)
    cr = _cr(f)
    g = torch.as_tensor(f["g"]).cuda()
    cr.prev = (torch.as_tensor(f["prev"][0]).cuda(), torch.as_tensor(f["prev"][1]).cuda())
    pairs, run = cr.analyze_merge(g, f["dt_y"])
    assert pairs and run is not None
    sample = f["g"].reshape(-1)
    x, y, vx, vy = (f["g"][c].astype(np.float64) for c in range(4))
    sim = NBodyCuda([0])
    st = sim.load_state(x, y, vx, vy, f["mass"], f["vis"], f["is_ast"], f["rr"])
    events, shatter = cr.apply_merges(sim, st, sample, pairs, run, k_ev=5)
    mass, vis, rr = f["mass"].copy(), f["vis"].copy(), f["rr"].copy()
    ev_ref, states, deact, sh = oc.apply_merges(sample, len(x), pairs, run, mass, vis, rr, f["is_ast"] != 0,
                                                np.zeros(len(x), bool), k_ev=5)
    assert shatter is None and sh is None
    assert events == ev_ref
    assert np.array_equal(cr.mass, mass) and np.array_equal(cr.vis, vis) and np.array_equal(cr.real_r, rr)
    out = sim.export_f64(st)
    n = len(x)
    last = {s[0]: s for s in states}          # a planet may absorb several asteroids
    assert last
    for a, nx, ny, nvx, nvy, m, r in last.values():
        assert out[a] == nx and out[n + a] == ny and out[2 * n + a] == nvx and out[3 * n + a] == nvy


def test_one_hit_rule_long_chains():
    """The one-hit-per-body rule on a hit list with a 600-hit chain in index
    order ((i, i+1): each round of the parallel filter settles one link, so
    the sequential finish runs) and 3000 random hits among other bodies:
    kept/active hits, touched bodies and deltas as the oracle's."""
    from solarsystemsimulator_b200.collide import CollisionResponse
    rng = np.random.default_rng(31)
    n = 2000
    x = np.arange(n) * 1e-5
    y = rng.normal(0, 1e-7, n)
    vx = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    vy = rng.normal(0, 0.1, n)
    g = np.stack([x, y, vx, vy]).astype(np.float32)
    rr = np.full(n, 6e-6)
    mass = 10 ** rng.uniform(-14, -12, n)
    ones = np.ones(n, np.uint8)
    chain = {(i, i + 1) for i in range(600)}
    extra = set()
    while len(extra) < 3000:
        a, b = sorted(rng.choice(np.arange(600, n), 2, replace=False).tolist())
        extra.add((a, b))
    pairs = sorted(chain | extra)
    hits = np.array([(0, a, b) for a, b in pairs], np.int32)
    cr = CollisionResponse(mass, rr, ones, ones, m_idx=np.zeros(0, np.int64))
    res = cr.bounce_deltas(torch.as_tensor(g).cuda(), torch.as_tensor(hits).cuda(), len(hits), 0.5 / 365.25)
    hi = np.array([a for a, b in pairs])
    hj = np.array([b for a, b in pairs])
    ref = oc.bounce_deltas(*g, rr, mass, hi, hj, 0.5 / 365.25)
    assert res is not None and ref is not None
    ghi, ghj, touched, d = (t.cpu().numpy() for t in res)
    assert np.array_equal(ghi, ref[0]) and np.array_equal(ghj, ref[1])
    assert np.array_equal(touched, ref[2])
    assert np.allclose(d, ref[3], rtol=1e-12, atol=0.0, equal_nan=True)
    assert len(ghi) > 300


# ------------------------------------------------ against the reference's own outputs
# Fixtures written by tests/golden/make_golden.py from producer_main's own
# analyze_merge, bounce_deltas and apply_merges (film_producer.py:707-1019).

def test_sweep_matches_reference_golden(load_golden):
    from solarsystemsimulator_b200.collide import CollisionResponse
    g = load_golden("collide_sweep.npz")
    cr = CollisionResponse(g["mass"], g["rr"].astype(np.float64), g["vis"], g["is_ast"],
                           m_idx=np.arange(int(g["n_m"])), G=float(g["G"]))
    # the reference sweeps with the f32 radii it holds on the detection card
    cr.d_rr32 = torch.as_tensor(g["rr"]).cuda()
    for k in range(2):
        s = torch.as_tensor(np.stack([g[f"x{k}"], g[f"y{k}"], g[f"vx{k}"], g[f"vy{k}"]])).cuda()
        pairs, run = cr.analyze_merge(s, float(g["dt_years"]))
        assert np.array_equal(np.array([(a, b) for a, b, _ in pairs], np.int64).reshape(-1, 2), g[f"pairs{k}"])
        assert np.array_equal(np.array([f for _, _, f in pairs]), g[f"frac{k}"])
        assert np.array_equal(np.asarray(run if run is not None else [], np.int64), g[f"run{k}"])


@pytest.mark.parametrize("scene", ["clump", "massless", "cases"])
def test_bounce_matches_reference_golden(load_golden, scene):
    """The device hit list (bit-exact broadphase) through sss_collide_bounce:
    kept and active hits and touched bodies identical to the reference's,
    deltas within 1e-12 (f64 hypot may differ in the last bit from the
    host C library's), NaN where the reference's arithmetic gives NaN."""
    from solarsystemsimulator_b200 import broadphase as bp
    from solarsystemsimulator_b200.collide import CollisionResponse
    g = load_golden(f"collide_bounce_{scene}.npz")
    n = len(g["mass"])
    s = g["sample"].reshape(4, n)
    dt_y = float(g["raster_days"]) / 365.25
    v95 = float(np.percentile(np.hypot(s[2], s[3]), 95))
    h = max(1e-4, 2.0 * v95 * dt_y)
    rr32 = g["rr"].astype(np.float32)
    buf, k, _ = bp.bounce_hits_device(*s, dt_y, h, 2.0 * h + 2.0 * float(g["rr"].max()), rr=rr32)
    ones = np.ones(n, np.uint8)
    cr = CollisionResponse(g["mass"], g["rr"], ones, ones, m_idx=np.zeros(0, np.int64))
    res = cr.bounce_deltas(torch.as_tensor(s).cuda(), buf, k, dt_y)
    hi, hj, touched, d = (t.cpu().numpy() for t in res)
    assert np.array_equal(hi, g["kept_i"]) and np.array_equal(hj, g["kept_j"])
    assert np.array_equal(touched, g["touched"])
    assert np.allclose(d, g["deltas"], rtol=1e-12, atol=0.0, equal_nan=True)
    assert np.array_equal(np.isnan(d), np.isnan(g["deltas"]))


@pytest.mark.parametrize("scene", ["chain", "chain_noshatter", "shatter"])
def test_merges_match_reference_golden(load_golden, scene):
    """CollisionResponse.apply_merges issues the reference's simulation calls
    in the reference's order and leaves the same host mirrors."""
    from solarsystemsimulator_b200.collide import CollisionResponse
    g = load_golden(f"collide_merges_{scene}.npz")
    n = len(g["mass0"])
    calls = []

    class _Sim:
        def apply_body_state(self, st, a, x, y, vx, vy, m):
            calls.append(("state", int(a), float(x), float(y), float(vx), float(vy), float(m)))

        def deactivate_body(self, st, b):
            calls.append(("off", int(b)))

        def set_radius(self, st, a, r):
            calls.append(("radius", int(a), float(r)))

    cr = CollisionResponse(g["mass0"], g["rr0"], g["vis0"], g["is_ast"], is_star_bh=g["star"],
                           m_idx=np.flatnonzero(~g["is_ast"]), shatter=bool(g["shatter"]))
    pairs = [(int(a), int(b), float(f)) for (a, b), f in zip(g["pairs"], g["frac"])]
    runs = g["runaways"] if len(g["runaways"]) or scene != "shatter" else None
    events, sh = cr.apply_merges(_Sim(), {}, g["sample"], pairs, runs, k_ev=int(g["k_ev"]),
                                 contact={int(k): float(v) for k, v in g["contact"]})
    assert calls == eval(str(g["calls"]))
    want = eval(str(g["events"]))
    assert [(a, b, m, kd, x, y, fr) for a, b, m, kd, fr, x, y in events] == \
        [(a, b, m, kd, x, y, fr) for a, b, m, kd, _k, x, y, fr in want]
    assert np.array_equal(cr.mass, g["mass1"]) and np.array_equal(cr.vis, g["vis1"])
    assert np.array_equal(cr.real_r, g["rr1"])
    assert (sh is not None) == bool(int(g["shatter_flag"]))


# ------------------------------------------------ fragmentation of fast impacts

def _fast_impacts(seed=41, n=3000):
    """A clump of small asteroids (2 g/cm^3) with random speeds: most bounce
    pairs hit far above their escape speed, slow ones below it; some bodies
    hidden (free slots for fragments)."""
    rng = np.random.default_rng(seed)
    x = (1.5 + rng.normal(0, 1e-4, n)).astype(np.float32)
    y = rng.normal(0, 1e-4, n).astype(np.float32)
    sp = 10 ** rng.uniform(-3, 0.5, n)                     # AU / yr: v_esc is ~0.02 AU / yr at r = 1e-6 AU
    th = rng.uniform(0, 2 * np.pi, n)
    vx, vy = (sp * np.cos(th)).astype(np.float32), (sp * np.sin(th)).astype(np.float32)
    rr = 10 ** rng.uniform(-6.5, -5.5, n)
    mass = (4.0 / 3.0) * np.pi * (rr * 1.495978707e13) ** 3 * 2.0 / 1.98847e33
    vis = np.ones(n, np.uint8)
    vis[rng.choice(n, n // 3, replace=False)] = 0
    return np.stack([x, y, vx, vy]), rr, mass, vis


def test_fragments_match_oracle_and_conserve():
    from solarsystemsimulator_b200 import broadphase as bp
    from solarsystemsimulator_b200.collide import CollisionResponse, FRAG_V_ESC, G_AU
    g, rr, mass, vis = _fast_impacts()
    n = g.shape[1]
    ones = np.ones(n, np.uint8)
    dt_y = 0.5 / 365.25
    h = max(1e-4, 2.0 * float(np.percentile(np.hypot(g[2], g[3]), 95)) * dt_y)
    buf, k, _ = bp.bounce_hits_device(*g, dt_y, h, 2 * h + 2 * float(rr.max()), rr=rr.astype(np.float32), vis=vis)
    cr = CollisionResponse(mass, rr, vis, ones, m_idx=np.zeros(0, np.int64))
    gd = torch.as_tensor(g).cuda()
    res = cr.bounce_deltas(gd, buf, k, dt_y)
    assert res is not None
    parents, frags = cr.fragment(gd, res, FRAG_V_ESC, seed=1234)
    act = np.stack([res[0].cpu().numpy(), res[1].cpu().numpy()], 1)
    ref = oc.fragment_events(*g, rr, mass, act, G_AU, FRAG_V_ESC, 1234)
    assert 0 < len(ref) < len(act)                          # some pairs fragment, some only bounce
    assert np.array_equal(parents, np.array([(a, b) for a, b, _ in ref]))
    want = np.stack([f for _, _, f in ref])
    scale = np.abs(want).max(axis=(0, 1))
    assert np.all(np.abs(frags - want) <= 1e-12 * scale)
    # mass and momentum of every event are those of its parents
    for (a, b), f in zip(parents, frags):
        mt = mass[a] + mass[b]
        assert abs(f[:, 4].sum() - mt) <= 1e-15 * mt
        for c, vc in ((2, 2), (3, 3)):
            p0 = mass[a] * float(g[vc][a]) + mass[b] * float(g[vc][b])
            assert abs((f[:, 4] * f[:, c]).sum() - p0) <= 1e-13 * mt * np.abs(f[:, c]).max()
    # a different seed scatters differently; factor 0 turns it off
    p2, f2 = cr.fragment(gd, res, FRAG_V_ESC, seed=99)
    assert np.array_equal(p2, parents) and not np.array_equal(f2, frags)
    assert len(cr.fragment(gd, res, 0.0, seed=1)[0]) == 0


def test_fragments_enter_the_simulation():
    from solarsystemsimulator_b200 import broadphase as bp
    from solarsystemsimulator_b200.collide import CollisionResponse, FRAG_V_ESC
    from solarsystemsimulator_b200.nbody_kernel import NBodyCuda
    g, rr, mass, vis = _fast_impacts(seed=42, n=2000)
    n = g.shape[1]
    is_ast = np.ones(n, np.uint8)
    is_ast[0] = 0                                          # a star far away keeps the film's shape
    x = g[0].astype(np.float64); y = g[1].astype(np.float64)
    x[0], y[0] = 0.0, 0.0
    mass = mass.copy(); mass[0] = 1.0
    vis[0] = 1
    gg = np.stack([x, y, g[2], g[3]]).astype(np.float32)
    dt_y = 0.5 / 365.25
    h = max(1e-4, 2.0 * float(np.percentile(np.hypot(gg[2], gg[3]), 95)) * dt_y)
    buf, k, _ = bp.bounce_hits_device(*gg, dt_y, h, 2 * h + 2 * float(rr.max()), rr=rr.astype(np.float32),
                                      is_ast=is_ast, vis=vis)
    cr = CollisionResponse(mass, rr, vis, is_ast, m_idx=np.array([0]))
    sim = NBodyCuda([0])
    st = sim.load_state(x, y, gg[2].astype(np.float64), gg[3].astype(np.float64), mass, vis, is_ast, rr)
    gd = torch.as_tensor(gg).cuda()
    res = cr.bounce_deltas(gd, buf, k, dt_y)
    cr.apply_bounce(sim, st, res)
    parents, frags = cr.fragment(gd, res, FRAG_V_ESC, seed=7)
    n_hidden = int(((vis == 0) & (is_ast != 0)).sum())
    events, used, skipped = cr.apply_fragments(sim, st, parents, frags)
    assert len(events) + skipped == len(parents) and len(events) > 0
    assert skipped == max(0, len(parents) - n_hidden // 3)
    out = sim.export_f64(st)
    slots = np.array(used)
    assert len(np.unique(slots)) == slots.size                 # every fragment has its own slot
    new_slots = np.array([q for sl in used for q in sl[2:]])
    assert np.all(cr.vis[new_slots] == 0) and np.all(cr.pending[new_slots])   # visible from the next batch
    assert np.array_equal(np.sort(cr.activate_fragments(gd)), np.sort(new_slots))
    for sl, f in zip(used, frags[:len(used)]):
        assert np.array_equal(out[sl], f[:, 0]) and np.array_equal(out[n + np.array(sl)], f[:, 1])
        assert np.array_equal(out[2 * n + np.array(sl)], f[:, 2])
        assert np.all(cr.vis[sl] == 1) and np.array_equal(cr.mass[sl], f[:, 4])
    # the fragments fly on with the rest
    sim.step_batch(st, dt_y, 1)


def test_fragment_events_sharing_a_body():
    """A body in two fast active pairs fragments once: the later event that
    names an already fragmented body is left out (its bounce stands), so is
    an event with a hidden parent, and the slots stay distinct."""
    from solarsystemsimulator_b200.collide import CollisionResponse, FRAG_V_ESC, N_FRAG
    from solarsystemsimulator_b200.nbody_kernel import NBodyCuda
    g, rr, mass, vis = _fast_impacts(seed=43, n=600)
    n = g.shape[1]
    is_ast = np.ones(n, np.uint8)
    is_ast[0] = 0
    x = g[0].astype(np.float64)
    y = g[1].astype(np.float64)
    x[0], y[0] = 0.0, 0.0
    mass = mass.copy()
    mass[0] = 1.0
    vis[0] = 1
    gg = np.stack([x, y, g[2], g[3]]).astype(np.float32)
    cr = CollisionResponse(mass, rr, vis, is_ast, m_idx=np.array([0]))
    sim = NBodyCuda([0])
    st = sim.load_state(x, y, gg[2].astype(np.float64), gg[3].astype(np.float64), mass, vis, is_ast, rr)
    a, b, c, d, e5 = [int(q) for q in np.flatnonzero((vis != 0) & (is_ast != 0))[:5]]
    hid = int(np.flatnonzero((vis == 0) & (is_ast != 0))[0])
    # (b, c) shares b with the first event; (hid, e5) names a body hidden since the broadphase
    parents = np.array([[a, b], [b, c], [c, d], [hid, e5]], np.int64)
    frags = np.zeros((4, N_FRAG, 6))
    for e, (p, q) in enumerate(parents):
        frags[e, :, 0] = x[p] + 1e-6 * np.arange(N_FRAG)
        frags[e, :, 1] = y[q]
        frags[e, :, 4] = (mass[p] + mass[q]) / N_FRAG
        frags[e, :, 5] = rr[p]
    events, used, skipped = cr.apply_fragments(sim, st, parents, frags)
    assert [ev[:2] for ev in events] == [(a, b), (c, d)] and skipped == 2
    slots = np.array(used)
    assert len(np.unique(slots)) == slots.size
    out = sim.export_f64(st)
    assert np.array_equal(out[slots[1]], frags[2, :, 0])
    assert FRAG_V_ESC > 0


def test_batched_merges_equal_immediate_updates():
    # apply_merges with the sample's columns gathered on the device, the
    # simulation's updates in one batch and the changed mirrors refreshed
    # alone leaves exactly the state of the reference's immediate updates
    # with the whole sample on the host and a full refresh
    from solarsystemsimulator_b200.nbody_kernel import NBodyCuda
    f = _film(31, n_per=2000, clouds=2, crossers=30, runaways=8)
    g = f["g"]
    x, y, vx, vy = (g[i].astype(np.float64) for i in range(4))
    runs = {}
    for batched in (False, True):
        cr = _cr(f)
        sim = NBodyCuda([0])
        st = sim.load_state(x, y, vx, vy, f["mass"], f["vis"], f["is_ast"], f["rr"])
        gd = torch.as_tensor(g).cuda()
        cr.prev = (torch.as_tensor(f["prev"][0]).cuda(), torch.as_tensor(f["prev"][1]).cuda())
        pairs, run = cr.analyze_merge(gd, f["dt_y"])
        assert len(pairs) > 0 and run is not None and len(run) > 0
        if batched:
            events, shatter = cr.apply_merges(sim, st, gd, pairs, run, batched=True)
            cr.refresh(cr.changed)
            fresh = np.flatnonzero((cr.vis == 0) & cr.is_ast & ~cr.pending)
            assert np.array_equal(cr._free_slots(), fresh)
        else:
            events, shatter = cr.apply_merges(sim, st, g.reshape(-1), pairs, run, batched=False)
            cr.refresh()
        snap = sim.step_batch(st, f["dt_y"], 2)
        runs[batched] = dict(
            events=events, shatter=shatter, f64=sim.export_f64(st), snap=snap,
            mirrors=[cr.mass.copy(), cr.vis.copy(), cr.real_r.copy(), st["am_h"].copy(), st["avis_h"].copy()],
            device=[t.cpu().numpy() for t in (cr.d_vis, cr.d_rr32, cr.d_rr, cr.d_mass)] +
                   [st[k].cpu().numpy() for k in ("am", "avis", "ar", "mm", "mvis", "mr")])
    a, b = runs[False], runs[True]
    assert a["events"] == b["events"] and a["shatter"] == b["shatter"]
    assert any(e[3] == 0 for e in a["events"]) and any(e[3] == 2 for e in a["events"])
    assert np.array_equal(a["f64"], b["f64"]) and np.array_equal(a["snap"], b["snap"])
    for u, v in zip(a["mirrors"] + a["device"], b["mirrors"] + b["device"]):
        assert np.array_equal(u, v)
