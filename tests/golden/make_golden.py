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


def main():
    if len(sys.argv) < 2 or not os.path.isdir(os.path.join(sys.argv[1], "backend")):
        sys.exit("usage: make_golden.py REFERENCE_CHECKOUT [selfgrav|frame|pm|broadphase|broadphase_clouds ...]")
    ref = sys.argv[1]
    sys.path.insert(0, os.path.join(ref, "backend"))
    cupy_shim.install()
    which = sys.argv[2:] or ["selfgrav", "frame", "pm", "broadphase", "broadphase_clouds"]
    for w in which:
        globals()[w](ref)


if __name__ == "__main__":
    main()
