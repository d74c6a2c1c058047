"""Generate the golden fixtures in tests/golden/ from the reference's OWN code.

Run in the build container (where the reference checkout exists):

    python tests/golden/make_golden.py /path/to/reference [which ...]

The reference's array-level Python (NumPy oracles in backend/test_*.py,
backend/pm_kernel.py, the broadphase of backend/film_producer.py) is
imported unmodified through cupy_shim (cupy -> numpy, stable argsort) and
run on seeded inputs; inputs and outputs are written as small .npz files.
The GPU box has no reference checkout, so tests read only these files.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import cupy_shim  # noqa: E402


def _save(name, **arrays):
    path = os.path.join(HERE, name)
    np.savez_compressed(path, **arrays)
    print(f"wrote {name}: " + ", ".join(f"{k}{np.shape(v)}" for k, v in arrays.items()))


def selfgrav(ref):
    import test_pm
    import test_selfgrav as ts
    from nbody_kernel import G_AU

    # 1) the dense all-pairs force of the reference (test_pm.py:32-41) on
    #    the test_selfgrav cloud (test_selfgrav.py:33-51), two sizes
    for n, seed in ((256, 7), (1000, 11)):
        x, y, vx, vy, m = ts.wolke(n, 0.5, seed=seed)
        eps2 = ts.EPS ** 2
        ax, ay = test_pm.allpairs_accel(x, y, m, eps2, G_AU)
        _save(f"selfgrav_accel_n{n}.npz", x=x, y=y, m=m, eps2=eps2, G=G_AU,
              ax=np.asarray(ax), ay=np.asarray(ay))

    # 2) the reference's KDK oracle (test_selfgrav.py:66-88) + energy (:54-63)
    n, steps, dt = 128, 25, 0.0055
    x, y, vx, vy, m = ts.wolke(n, 0.4, seed=7)
    eps2 = ts.EPS ** 2
    e0 = ts.energie(x, y, vx, vy, m, eps2)
    rx, ry, rvx, rvy = ts.referenz(x, y, vx, vy, m, eps2, dt, steps)
    e1 = ts.energie(rx, ry, rvx, rvy, m, eps2)
    _save("selfgrav_kdk_n128.npz", x=x, y=y, vx=vx, vy=vy, m=m, eps2=eps2, dt=dt, steps=steps,
          G=G_AU, rx=rx, ry=ry, rvx=rvx, rvy=rvy, e0=e0, e1=e1)


def frame(ref):
    import test_kernel as tk
    from nbody_kernel import G_AU, MAX_SUB_DT_YEARS, SOFTENING, YOSHIDA_W0, YOSHIDA_W1

    # 3) make_system(200) advanced 5 days (test_kernel.py:112-131)
    state = tk.make_system(200)
    dt = 5 / 365.25
    rx, ry, rvx, rvy = tk.reference_advance(dt, *state)
    x, y, vx, vy, mass, vis, is_ast = state
    _save("frame_system200_5d.npz", x=x, y=y, vx=vx, vy=vy, mass=mass, vis=vis, is_ast=is_ast,
          dt=dt, rx=rx, ry=ry, rvx=rvx, rvy=rvy, G=G_AU, soft=SOFTENING,
          max_sub_dt=MAX_SUB_DT_YEARS, w1=YOSHIDA_W1, w0=YOSHIDA_W0)

    # 4) the sun-diver scene (test_kernel.py:190-219)
    rng = np.random.default_rng(3)
    nd = 20
    x = np.zeros(1 + nd); y = np.zeros(1 + nd)
    vx = np.zeros(1 + nd); vy = np.zeros(1 + nd)
    mass = np.full(1 + nd, 1e-12); mass[0] = 1.0
    vis = np.ones(1 + nd, np.uint8)
    is_ast = np.ones(1 + nd, np.uint8); is_ast[0] = 0
    th = rng.random(nd) * 2 * np.pi
    r0 = 0.25 + 0.1 * rng.random(nd)
    x[1:] = r0 * np.cos(th); y[1:] = r0 * np.sin(th)
    dt8 = 8 / 365.25
    rx, ry, rvx, rvy = tk.reference_advance(dt8, x, y, vx, vy, mass, vis, is_ast)
    _save("frame_sundiver_8d.npz", x=x, y=y, vx=vx, vy=vy, mass=mass, vis=vis, is_ast=is_ast,
          dt=dt8, rx=rx, ry=ry, rvx=rvx, rvy=rvy)


def pm(ref):
    import pm_kernel as pk
    from nbody_kernel import G_AU

    # 5) 2-D isolated PM forces (pm_kernel.py:34-163) on a seeded cloud
    rng = np.random.default_rng(42)
    n, grid_n = 2000, 128
    x = rng.uniform(-40000, 40000, n)
    y = rng.uniform(-40000, 40000, n)
    m = rng.uniform(1e6, 2e7, n)
    x0, y0, h = pk.grid_fuer(x, y, grid_n)
    eps2 = (2 * h) ** 2
    ax, ay = pk.pm_accelerations(x, y, m, grid_n, x0, y0, h, eps2)
    rho = pk._cic_deposit(x, y, m, grid_n, x0, y0, h)
    _save("pm2d_n2000_g128.npz", x=x, y=y, m=m, grid_n=grid_n, x0=x0, y0=y0, h=h, eps2=eps2,
          G=G_AU, ax=np.asarray(ax), ay=np.asarray(ay), rho=np.asarray(rho))

    # 6) NBodyPM KDK: 5 steps of the adaptive-grid integrator (pm_kernel.py:166-293)
    rng = np.random.default_rng(5)
    n = 1500
    R = 30000.0
    Mtot = 5.6e9
    r = R * np.sqrt(rng.uniform(0, 1, n))
    th = rng.uniform(0, 2 * np.pi, n)
    x = r * np.cos(th); y = r * np.sin(th)
    m = np.full(n, Mtot / n)
    vvir = np.sqrt(G_AU * Mtot / R)
    ang = rng.uniform(0, 2 * np.pi, n)
    vx = 0.7 * vvir * np.cos(ang); vy = 0.7 * vvir * np.sin(ang)
    tx = rng.uniform(-R, R, 64); ty = rng.uniform(-R, R, 64)
    tvx = np.zeros(64); tvy = np.zeros(64)
    sim = pk.NBodyPM([0], grid_n=256, softening_zellen=1.5)
    st = sim.load_state(x, y, vx, vy, m, tracer=(tx, ty, tvx, tvy))
    dt = (R / vvir) / 1000.0
    out = sim.step_batch(st, dt, 5)
    f = sim.export_f64(st)
    _save("pm2d_kdk_n1500.npz", x=x, y=y, vx=vx, vy=vy, m=m, tx=tx, ty=ty, tvx=tvx, tvy=tvy,
          grid_n=256, soft_cells=1.5, rand_cells=4.0, dt=dt, steps=5, out=out, f64=f, G=G_AU)


def broadphase(ref):
    import film_producer as fp

    dt_y = 0.5 / 365.25

    def run(name, x, y, vx, vy, rr):
        n = len(x)
        is_ast = np.ones(n, bool)
        vis = np.ones(n, np.uint8)
        f = [a.astype(np.float32) for a in (x, y, vx, vy)]
        v95 = float(np.percentile(np.hypot(f[2], f[3]), 95))
        h = max(1e-4, 2.0 * v95 * dt_y)
        halo = 2.0 * h + 2.0 * float(rr.max())
        karte = fp.Erkennungskarte(0, is_ast, -np.inf, np.inf)
        karte.stammdaten(vis, rr.astype(np.float32))
        hits, kand = karte.bounce_hits(*f, dt_y, h, halo)
        hi = np.empty(0, np.int64) if hits is None else np.asarray(hits[0], np.int64)
        hj = np.empty(0, np.int64) if hits is None else np.asarray(hits[1], np.int64)
        # the striped variants (film_producer.py:382-405): union must equal the full set
        stripes = {}
        for anzahl in (2, 3, 5):
            grenzen = fp._streifengrenzen(f[0], [1.0 / anzahl] * anzahl)
            parts = []
            for lo, hi_ in grenzen:
                karte.streifen(lo, hi_)
                t, _k = karte.bounce_hits(*f, dt_y, h, halo)
                parts.append(np.zeros((0, 2), np.int64) if t is None
                             else np.stack([np.asarray(t[0]), np.asarray(t[1])], 1).astype(np.int64))
            stripes[f"stripes{anzahl}_bounds"] = np.array(grenzen, np.float64)
            union = np.concatenate(parts) if parts else np.zeros((0, 2), np.int64)
            # the reference's own invariant: the stripe union is the full set
            stripes[f"stripes{anzahl}_count"] = np.int64(len(union))
        _save(f"broadphase_{name}.npz", x=f[0], y=f[1], vx=f[2], vy=f[3], rr=rr.astype(np.float32),
              dt_y=dt_y, h=h, halo=halo, hit_i=hi, hit_j=hj, n_cand=kand, **stripes)

    rng = np.random.default_rng(4711)
    nb = 20_000
    run("wolke", rng.uniform(-3, 3, nb), rng.uniform(-3, 3, nb), rng.normal(0, 4, nb),
        rng.normal(0, 4, nb), np.full(nb, 3e-3))
    nb = 8_000
    run("klumpen", rng.normal(2.0, 0.02, nb), rng.normal(0.0, 0.02, nb), rng.normal(0, 6, nb),
        rng.normal(0, 6, nb), np.full(nb, 2e-4))
    nb = 5_000
    x = np.concatenate([rng.normal(-4.0, 0.1, nb), rng.normal(4.0, 0.1, nb)])
    y = rng.normal(0.0, 0.1, 2 * nb)
    run("zwei_wolken", x, y, rng.normal(0, 3, 2 * nb), rng.normal(0, 3, 2 * nb), np.full(2 * nb, 1e-3))
    run("auf_der_grenze", np.array([5.0 - 5e-4, 5.0 + 5e-4]), np.zeros(2), np.array([0.5, -0.5]),
        np.zeros(2), np.full(2, 1e-4))


def clouds_scene(n_per_cloud=40_000):
    """The asteroid-cloud configuration's broadphase input: 5 Gaussian clouds
    of n_per_cloud asteroids from the seeded generator, the f32 snapshot of
    x, y, vx, vy and radii, dt = 0.5 day, h from the 95th speed percentile
    (film_producer.py:357-359)."""
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from solarsystemsimulator_b200 import workloads
    w = workloads.asteroid_clouds(n_per_cloud=n_per_cloud)
    a = np.flatnonzero(w["is_ast"] != 0)
    f = [np.ascontiguousarray(v, dtype=np.float32) for v in
         (w["pos"][0, a], w["pos"][1, a], w["vel"][0, a], w["vel"][1, a], w["radius"][a])]
    dt = 0.5
    v95 = float(np.percentile(np.hypot(f[2], f[3]), 95))
    h = max(1e-4, 2.0 * v95 * dt)
    halo = 2.0 * h + 2.0 * float(f[4].max())
    return f, dt, h, halo


def scene_digest(f):
    import hashlib
    d = hashlib.sha256()
    for v in f:
        d.update(np.ascontiguousarray(v, dtype=np.float32).tobytes())
    return d.hexdigest()


def broadphase_clouds(ref):
    """The 200,000-asteroid cloud scene through the reference's own `_hits`
    (film_producer.py:223-317). Only the hit list, the candidate count, the
    scalars and a digest of the input are stored; the test rebuilds the
    scene from the seeded generator and checks the digest first."""
    import time
    import film_producer as fp
    f, dt, h, halo = clouds_scene()
    n = len(f[0])
    karte = fp.Erkennungskarte(0, np.ones(n, bool), -np.inf, np.inf)
    karte.stammdaten(np.ones(n, np.uint8), f[4])
    t0 = time.time()
    hits, kand = karte.bounce_hits(f[0], f[1], f[2], f[3], dt, h, halo)
    print(f"_hits on {n} asteroids: {kand} candidates, {time.time() - t0:.0f} s")
    hi = np.empty(0, np.int64) if hits is None else np.asarray(hits[0], np.int64)
    hj = np.empty(0, np.int64) if hits is None else np.asarray(hits[1], np.int64)
    _save("broadphase_asteroid_clouds_200k.npz", n_per_cloud=40_000, dt=dt, h=h, halo=halo,
          digest=np.array(scene_digest(f)), hit_i=hi.astype(np.int32), hit_j=hj.astype(np.int32),
          n_cand=np.int64(kand))


class _Val:
    def __init__(self, v=0):
        self.value = v


def _producer_closure(fp, name, **cells):
    """One of producer_main's nested functions (the film producer keeps its
    per-sample analysis as closures) as a callable: the reference's own code
    object, with the enclosing variables it reads given as cells."""
    import types

    def find(code):
        for c in code.co_consts:
            if isinstance(c, types.CodeType):
                if c.co_name == name:
                    return c
                r = find(c)
                if r is not None:
                    return r
        return None

    code = find(fp.producer_main.__code__)
    missing = [v for v in code.co_freevars if v not in cells]
    if missing:
        raise KeyError(f"{name} needs {missing}")
    closure = tuple(types.CellType(cells[v]) for v in code.co_freevars)
    return types.FunctionType(code, fp.__dict__, name, None, closure)


def _cell(fn, name):
    return fn.__closure__[fn.__code__.co_freevars.index(name)].cell_contents


def collide(ref):
    """The film producer's collision response through its own code:
    analyze_merge (film_producer.py:707-779) over two samples,
    bounce_deltas (:916-1019) on broadphase hit lists, apply_merges
    (:781-861) with recorded state changes and events."""
    import film_producer as fp
    from nbody_kernel import G_AU

    class _Karte:
        pass

    # ---- merge sweep: star, 7 planets (one hidden, one massless), asteroids
    rng = np.random.default_rng(20261204)
    n_m, n_a = 8, 4000
    n = n_m + n_a
    x = np.zeros(n); y = np.zeros(n); vx = np.zeros(n); vy = np.zeros(n)
    rr = np.zeros(n); mass = np.zeros(n)
    is_ast = np.zeros(n, bool); is_ast[n_m:] = True
    vis = np.ones(n, np.uint8)
    mass[0], rr[0] = 1.0, 0.00465
    for k in range(1, n_m):
        a = 0.5 + 0.6 * k
        th = rng.uniform(0, 2 * np.pi)
        v = np.sqrt(G_AU / a)
        x[k], y[k] = a * np.cos(th), a * np.sin(th)
        vx[k], vy[k] = -v * np.sin(th), v * np.cos(th)
        mass[k] = 10 ** rng.uniform(-6, -3)
        rr[k] = 10 ** rng.uniform(-4.5, -3.3)
    vis[3] = 0                                        # a hidden planet
    mass[5] = 0.0                                     # a massless one
    host = rng.integers(0, n_m, n_a)                  # asteroids crowd around the massive bodies
    d = rng.normal(0, 1, (n_a, 2)) * 10 ** rng.uniform(-3.5, -1.5, (n_a, 1))
    x[n_m:] = x[host] + d[:, 0]
    y[n_m:] = y[host] + d[:, 1]
    vx[n_m:] = vx[host] + rng.normal(0, 3.0, n_a)
    vy[n_m:] = vy[host] + rng.normal(0, 3.0, n_a)
    fast = rng.choice(np.arange(n_m, n), 25, replace=False)
    vx[fast] *= 60.0                                  # runaways
    rr[n_m:] = 10 ** rng.uniform(-7, -5, n_a)
    mass[n_m:] = 1e-14
    vis[rng.choice(np.arange(n_m, n), 40, replace=False)] = 0
    dt_years = 0.5 / 365.25
    karte = _Karte()
    karte.g_vis = vis.copy()
    karte.g_rr = rr.astype(np.float32)
    karte.g_ast = is_ast.copy()
    st = {"m_idx_h": np.arange(n_m, dtype=np.int64)}
    sweep = _producer_closure(fp, "analyze_merge", G_AU=G_AU, det=[karte], dt_years=dt_years, mass=mass,
                              prev_det=None, st=st, vis=vis)
    rec = {"n": n, "n_m": n_m, "rr": rr.astype(np.float32), "mass": mass, "is_ast": is_ast, "vis": vis,
           "dt_years": dt_years, "G": G_AU}
    for k in range(2):
        f = [v.astype(np.float32) for v in (x, y, vx, vy)]
        pairs, run = sweep(f[0], f[1], f[0], f[1], f[2], f[3])
        rec.update({f"x{k}": f[0], f"y{k}": f[1], f"vx{k}": f[2], f"vy{k}": f[3],
                    f"pairs{k}": np.array([(a, b) for a, b, _ in pairs], np.int64).reshape(-1, 2),
                    f"frac{k}": np.array([fr for _, _, fr in pairs], np.float64),
                    f"run{k}": np.empty(0, np.int64) if run is None else np.asarray(run, np.int64)})
        print(f"sweep sample {k}: {len(pairs)} pairs, {0 if run is None else len(run)} runaways")
        x = x + vx * dt_years
        y = y + vy * dt_years
    _save("collide_sweep.npz", **rec)

    # ---- bounce response on broadphase hit lists (the reference's order)
    def bounce_scene(name, n, xs, ys, vxs, vys, rr, mass, dt_days):
        f = [v.astype(np.float32) for v in (xs, ys, vxs, vys)]
        karte = fp.Erkennungskarte(0, np.ones(n, bool), -np.inf, np.inf)
        karte.stammdaten(np.ones(n, np.uint8), rr.astype(np.float32))
        dt_y = dt_days / 365.25
        v95 = float(np.percentile(np.hypot(f[2], f[3]), 95))
        h = max(1e-4, 2.0 * v95 * dt_y)
        hits, _ = karte.bounce_hits(*f, dt_y, h, 2.0 * h + 2.0 * float(rr.max()))
        sample = np.concatenate(f).astype(np.float32)
        bd = _producer_closure(fp, "bounce_deltas", mass=mass, n=n, raster_days=dt_days, real_r=rr)
        res = bd(sample, hits)
        out = {"sample": sample, "rr": rr, "mass": mass, "raster_days": dt_days,
               "hit_i": np.asarray(hits[0], np.int64), "hit_j": np.asarray(hits[1], np.int64)}
        if res is None:
            out["none"] = True
        else:
            hi, hj, touched, deltas = res
            out.update({"kept_i": hi, "kept_j": hj, "touched": touched, "deltas": deltas})
        print(f"bounce {name}: {len(hits[0])} hits, {0 if res is None else len(res[0])} active")
        _save(f"collide_bounce_{name}.npz", **out)

    rng = np.random.default_rng(20261205)
    nb = 3000                                         # a dense clump: many more hits than bodies
    bounce_scene("clump", nb, 2.0 + rng.normal(0, 2e-4, nb), rng.normal(0, 2e-4, nb), rng.normal(0, 2.0, nb),
                 rng.normal(0, 2.0, nb), 10 ** rng.uniform(-5.3, -4.7, nb), 10 ** rng.uniform(-13, -11, nb), 0.5)
    nb = 400                                          # massless bodies among them (NaN impulses)
    m = 10 ** rng.uniform(-13, -11, nb)
    m[rng.choice(nb, 60, replace=False)] = 0.0
    bounce_scene("massless", nb, 1.0 + rng.normal(0, 1e-4, nb), rng.normal(0, 1e-4, nb), rng.normal(0, 1.0, nb),
                 rng.normal(0, 1.0, nb), np.full(nb, 2e-5), m, 0.5)
    # head-on, resting overlap, receding, and a grazing pass
    xs = np.array([0.0, 3e-5, 1.0, 1.0 + 1e-5, 2.0, 2.0 + 3e-5, 3.0, 3.0 + 1.9e-5])
    ys = np.array([0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.5e-5])
    vxs = np.array([1.0, -1.0, 0.0, 0.0, -1.0, 1.0, 2.0, -2.0])
    vys = np.zeros(8)
    bounce_scene("cases", 8, xs, ys, vxs, vys, np.full(8, 1e-5), np.array([1e-12, 3e-12] * 4), 0.5)

    # ---- apply_merges with recorded calls
    def merges_scene(name, sample, pairs, runaways, mass, vis, rr, is_ast, star, contact, k_ev, shatter):
        n = len(mass)
        calls, events = [], []

        class _Sim:
            def apply_body_state(self, st, a, x, y, vx, vy, m):
                calls.append(("state", int(a), float(x), float(y), float(vx), float(vy), float(m)))

            def deactivate_body(self, st, b):
                calls.append(("off", int(b)))

            def set_radius(self, st, a, r):
                calls.append(("radius", int(a), float(r)))

        def emit(a, b, new_mass, kind, k_ev, ex, ey, frac=0.0):
            events.append((int(a), int(b), float(new_mass), int(kind), int(k_ev), float(ex), float(ey), float(frac)))

        dumps = []
        flag = _Val(0) if shatter else None
        sa, sb, sti = _Val(-1), _Val(-1), _Val(0.0)
        mass0, vis0, rr0 = mass, vis, rr
        mass, vis, rr = mass.copy(), vis.copy(), rr.copy()
        am = _producer_closure(fp, "apply_merges", G_AU=G_AU, coll_val=_Val(0), collisions=0, det_dirty=[False],
                               dump_state=lambda: dumps.append(1), emit_event=emit, is_ast=is_ast,
                               is_star_bh=star, kernel_kontakt=dict(contact), mass=mass, n=n, raster_days=0.5,
                               real_r=rr, shatter_a=sa, shatter_b=sb, shatter_flag=flag, shatter_t=sti, sim=_Sim(),
                               st={}, t0_days=0.0, vis=vis)
        am(sample, pairs, runaways, k_ev)
        _save(f"collide_merges_{name}.npz", sample=sample, pairs=np.array([(a, b) for a, b, _ in pairs], np.int64),
              frac=np.array([f for _, _, f in pairs]), runaways=np.asarray(runaways if runaways is not None else [],
                                                                         np.int64),
              mass0=mass0, vis0=vis0, rr0=rr0,
              is_ast=is_ast, star=star, contact=np.array(sorted(contact.items()), np.float64).reshape(-1, 2),
              k_ev=k_ev, shatter=shatter, mass1=mass, vis1=vis, rr1=rr,
              calls=np.array(repr(calls)), events=np.array(repr(events)), dumps=len(dumps),
              shatter_ab=np.array([sa.value, sb.value]), shatter_t=sti.value, shatter_flag=0 if flag is None else
              flag.value, collisions=_cell(am, "collisions"))
        print(f"merges {name}: {len(events)} events, {len(calls)} calls, shatter {flag.value if flag else None}")

    n = 10
    s = np.zeros(4 * n, np.float32)
    rng = np.random.default_rng(20261206)
    s[:] = rng.normal(0, 1, 4 * n).astype(np.float32)
    mass = np.array([1.0, 3e-6, 1e-3, 2e-9, 1e-12, 1e-12, 1e-12, 1e-12, 0.0, 1e-12])
    vis = np.ones(n, np.uint8); vis[7] = 0
    rr = np.array([4.65e-3, 4.3e-5, 4.8e-4, 1e-6, 1e-7, 2e-7, 3e-7, 1e-7, 1e-7, 5e-8])
    is_ast = np.array([0, 0, 0, 0, 1, 1, 1, 1, 1, 1], bool)
    star = np.array([1, 0, 0, 0, 0, 0, 0, 0, 0, 0], bool)
    # star eats 4; planet 1 eats 5 (kernel contact time inside the raster) and
    # 6 (contact time outside: the sweep's fraction stays); 2 eats 4 again
    # (already gone: skipped); hidden 7 skipped; 8 massless partner; planet 3
    # absorbed by 2 (slow); then the runaways 9 and the already dead 4
    pairs = [(0, 4, -0.25), (1, 5, 0.5), (1, 6, -0.75), (2, 4, 0.1), (1, 7, 0.2), (8, 9, 0.0), (2, 3, 0.3)]
    s[2 * n + 3] = s[2 * n + 2]                      # 3 moves with 2: a slow merge
    s[3 * n + 3] = s[3 * n + 2]
    merges_scene("chain", s, pairs, np.array([9, 4], np.int64), mass, vis, rr, is_ast, star, {5: 1.6, 6: 3.5}, 0,
                 True)
    merges_scene("chain_noshatter", s, pairs, np.array([9, 4], np.int64), mass, vis, rr, is_ast, star,
                 {5: 1.6, 6: 3.5}, 0, False)
    # a fast impact of two planets stops the sample for the shatter
    s2 = s.copy()
    s2[2 * n + 1] = np.float32(900.0)
    pairs2 = [(0, 4, 0.0), (2, 1, 0.4), (2, 3, 0.1)]
    merges_scene("shatter", s2, pairs2, None, mass, vis, rr, is_ast, star, {}, 3, True)


def ring(ref):
    """Ring slots written by schreibe_slot (film_producer.py:87-123) and the
    self-gravity row reorder of the producer loop (:1245-1261, run from the
    reference's source lines)."""
    import textwrap
    import film_producer as fp
    rng = np.random.default_rng(20261207)
    n, m_sub = 5000, 8
    out_i = rng.normal(0, 3, 4 * n).astype(np.float32)
    cases = {"none": None, "few": 37, "overflow": 900}
    rec = {"n": n, "m_sub": m_sub, "out_i": out_i}
    for name, nh in cases.items():
        sub_max = 0 if name == "none" else 256
        if nh is None:
            sub_i = None
        else:
            idx = rng.choice(n, nh, replace=False).astype(np.int64)        # unsorted, as collected
            pos = rng.normal(0, 3, (m_sub, 2, nh)).astype(np.float32)
            sub_i = (idx, pos)
            rec[f"{name}_idx"] = idx
            rec[f"{name}_pos"] = pos
        buf = bytearray(fp.slot_bytes(n, m_sub, sub_max) + 16)
        over = fp.schreibe_slot(buf, 16, n, sub_max, out_i, sub_i)
        rec[f"{name}_sub_max"] = sub_max
        rec[f"{name}_slot"] = np.frombuffer(bytes(buf[16:]), np.uint8)
        rec[f"{name}_overflow"] = bool(over)
    # the reorder block of producer_main, run as written
    src = open(os.path.join(ref, "backend", "film_producer.py")).read().splitlines()
    a = next(i for i, l in enumerate(src) if "voll = np.zeros((outs.shape[0], 4 * n), np.float32)" in l) - 1
    b = next(i for i in range(a, len(src)) if src[i].strip() == "outs = voll")
    block = textwrap.dedent("\n".join(src[a:b + 1]))
    nn = 3000
    perm = rng.permutation(nn)
    sg_m, sg_t = np.sort(perm[:1200]).astype(np.int64), np.sort(perm[1200:]).astype(np.int64)
    outs = rng.normal(0, 1, (3, 4 * 1200 + 2 * 1800)).astype(np.float32)
    ns = {"np": np, "outs": outs, "sg_m": sg_m, "sg_t": sg_t, "n": nn}
    exec(block, ns)
    rec.update({"sg_n": nn, "sg_m": sg_m, "sg_t": sg_t, "sg_outs": outs, "sg_full": ns["outs"]})
    _save("ring_slots.npz", **rec)


def batched(ref):
    """test_kernel.reference_advance (test_kernel.py:16-81) on all-massive
    planetary systems whose substep stays at MAX_SUB_DT_YEARS (every
    encounter time / 20 is longer): one call per substep, so each call is one
    fixed Yoshida-4 step, the batched integrator's scheme."""
    import test_kernel as tk
    from nbody_kernel import G_AU, MAX_SUB_DT_YEARS, SOFTENING
    rng = np.random.default_rng(20261208)
    out = {"G": G_AU, "eps2": SOFTENING, "dt": MAX_SUB_DT_YEARS, "steps": 400}
    for s, nb in enumerate((3, 7, 12)):
        a = np.sort(rng.uniform(1.2, 12.0, nb - 1))
        a = a * (1.0 + 0.25 * np.arange(nb - 1) / max(nb - 2, 1))      # keep the orbits apart
        th = rng.uniform(0, 2 * np.pi, nb - 1)
        e = rng.uniform(0, 0.08, nb - 1)
        m = np.concatenate([[1.0], 10 ** rng.uniform(-7, -3.5, nb - 1)])
        v = np.sqrt(G_AU / a) * (1 + e)
        x = np.concatenate([[0.0], a * np.cos(th)])
        y = np.concatenate([[0.0], a * np.sin(th)])
        vx = np.concatenate([[0.0], -v * np.sin(th)])
        vy = np.concatenate([[0.0], v * np.cos(th)])
        vis = np.ones(nb, np.uint8)
        is_ast = np.zeros(nb, np.uint8)
        out.update({f"x{s}": x, f"y{s}": y, f"vx{s}": vx, f"vy{s}": vy, f"m{s}": m})
        st = (x, y, vx, vy)
        for _ in range(out["steps"]):
            st = tk.reference_advance(MAX_SUB_DT_YEARS, *st, m, vis, is_ast)
        out.update({f"rx{s}": st[0], f"ry{s}": st[1], f"rvx{s}": st[2], f"rvy{s}": st[3]})
    _save("batched_reference_advance.npz", **out)


def main():
    if len(sys.argv) < 2 or not os.path.isdir(os.path.join(sys.argv[1], "backend")):
        sys.exit("usage: make_golden.py REFERENCE_CHECKOUT [selfgrav|frame|pm|broadphase|broadphase_clouds|"
                 "collide|ring|batched ...]")
    ref = sys.argv[1]
    sys.path.insert(0, os.path.join(ref, "backend"))
    cupy_shim.install()
    which = sys.argv[2:] or ["selfgrav", "frame", "pm", "broadphase", "broadphase_clouds", "collide", "ring", "batched"]
    for w in which:
        globals()[w](ref)


if __name__ == "__main__":
    main()
