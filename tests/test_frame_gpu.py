"""GPU parity of the few-massive-body integrator (NBodyCuda) .

Against the reference's own oracle outputs (golden fixtures) with the
reference's tolerances (test_kernel.py, test_subsamples.py,
test_bewegter_stern.py), and against the CPU restatement of frame_kernel
(oracle/frame.py) with tight tolerances: f64 state within 1e-9 relative,
f32 snapshots within 2 f32 ulps of the oracle's f64 values, identical
sub-sample sets and contact partners.
"""
import numpy as np
import pytest

from oracle import frame as of

pytestmark = pytest.mark.gpu


def _nk():
    from solarsystemsimulator_b200 import nbody_kernel as nk
    return nk


def make_system(n_ast, seed=7):
    """The calm test system of the reference's test_kernel (sun, 9 planets,
    one frozen, asteroids at 2-4 AU on circular orbits)."""
    rng = np.random.default_rng(seed)
    n = 10 + n_ast
    x = np.zeros(n); y = np.zeros(n); vx = np.zeros(n); vy = np.zeros(n)
    mass = np.full(n, 1e-6); mass[0] = 1.0
    is_ast = np.zeros(n, np.uint8); is_ast[10:] = 1
    visible = np.ones(n, np.uint8); visible[3] = 0
    rp = np.arange(1, 10, dtype=np.float64)
    x[1:10] = rp
    vy[1:10] = np.sqrt(of.G_AU / rp)
    r = 2 + 2 * rng.random(n_ast)
    th = rng.random(n_ast) * 2 * np.pi
    x[10:] = r * np.cos(th); y[10:] = r * np.sin(th)
    v = np.sqrt(of.G_AU / r)
    vx[10:] = -v * np.sin(th); vy[10:] = v * np.cos(th)
    mass[10:] = 1e-12
    return x, y, vx, vy, mass, visible, is_ast


def oracle_state(x, y, vx, vy, mass, vis, is_ast, rr=None, z=None, vz=None):
    ast = np.asarray(is_ast) != 0
    a, m = np.flatnonzero(ast), np.flatnonzero(~ast)
    rr = np.zeros(len(x)) if rr is None else np.asarray(rr, float)
    P = [x, y] + ([z] if z is not None else [])
    V = [vx, vy] + ([vz] if z is not None else [])
    st = of.FrameState(np.stack([p[a] for p in P]), np.stack([v[a] for v in V]), mass[a], vis[a] != 0, rr[a],
                       np.stack([p[m] for p in P]), np.stack([v[m] for v in V]), mass[m], vis[m] != 0, rr[m])
    return st, a, m


def full_order(st, a, m, n):
    d = st.dim
    out = np.empty(2 * d * n)
    for c in range(d):
        out[c * n + a] = st.ax[c]; out[(d + c) * n + a] = st.av[c]
        out[c * n + m] = st.mx[c]; out[(d + c) * n + m] = st.mv[c]
    return out


def diver_scene(n_div=12, seed=3, with_planets=True):
    """Sun + (planets) + asteroids diving close to the sun (hot)."""
    rng = np.random.default_rng(seed)
    bodies = []
    x = [0.0]; y = [0.0]; vx = [0.0]; vy = [0.0]; mass = [1.0]; is_ast = [0]
    if with_planets:
        for r in (0.7, 1.5, 5.2):
            x.append(r); y.append(0.0); vx.append(0.0); vy.append(np.sqrt(of.G_AU / r))
            mass.append(3e-6); is_ast.append(0)
    th = rng.random(n_div) * 2 * np.pi
    r0 = 0.05 + 0.05 * rng.random(n_div)
    b = 0.02 * rng.random(n_div)                # impact parameter: small ones touch the sun
    speed = 20.0 + 20.0 * rng.random(n_div)
    for t, r, bb, sp in zip(th, r0, b, speed):
        px, py = r * np.cos(t), r * np.sin(t)
        ux, uy = -np.cos(t), -np.sin(t)         # inward, offset sideways by b
        x.append(px - bb * uy); y.append(py + bb * ux)
        vx.append(sp * ux); vy.append(sp * uy)
        mass.append(0.0); is_ast.append(1)
    # a few calm belt asteroids
    for k in range(20):
        r = 2.5 + 0.01 * k
        t = 0.3 * k
        v = np.sqrt(of.G_AU / r)
        x.append(r * np.cos(t)); y.append(r * np.sin(t)); vx.append(-v * np.sin(t)); vy.append(v * np.cos(t))
        mass.append(0.0); is_ast.append(1)
    n = len(x)
    return (np.array(x), np.array(y), np.array(vx), np.array(vy), np.array(mass), np.ones(n, np.uint8),
            np.array(is_ast, np.uint8))


def test_calm_system_matches_reference_golden(load_golden):
    # test_kernel.py:112-131: |dpos|, |dvel| < 5e-6 (f32 output), frozen body unchanged
    nk = _nk()
    g = load_golden("frame_system200_5d.npz")
    sim = nk.NBodyCuda(0)
    st = sim.load_state(g["x"], g["y"], g["vx"], g["vy"], g["mass"], g["vis"], g["is_ast"])
    out = sim.step(st, float(g["dt"]))
    n = len(g["x"])
    gx, gy, gvx, gvy = out[:n], out[n:2 * n], out[2 * n:3 * n], out[3 * n:]
    assert np.abs(np.concatenate([gx - g["rx"], gy - g["ry"]])).max() < 5e-6
    assert np.abs(np.concatenate([gvx - g["rvx"], gvy - g["rvy"]])).max() < 5e-6
    assert abs(gx[3] - g["x"][3]) < 1e-5 and abs(gy[3] - g["y"][3]) < 1e-5


def test_sun_diver_matches_reference_golden(load_golden):
    # test_kernel.py:190-219: |dpos| < 2e-3 AU, no catapult (r < 0.5)
    nk = _nk()
    g = load_golden("frame_sundiver_8d.npz")
    sim = nk.NBodyCuda(0)
    st = sim.load_state(g["x"], g["y"], g["vx"], g["vy"], g["mass"], g["vis"], g["is_ast"])
    out = sim.step(st, float(g["dt"]))
    n1 = len(g["x"])
    dp = np.max(np.hypot(out[0:n1] - g["rx"], out[n1:2 * n1] - g["ry"]))
    r_now = np.hypot(out[1:n1] - out[0], out[n1 + 1:2 * n1] - out[n1])
    assert dp < 2e-3 and r_now.max() < 0.5


@pytest.mark.parametrize("massive_ast", [False, True])
@pytest.mark.parametrize("dim", [2, 3])
def test_matches_frame_oracle(massive_ast, dim):
    nk = _nk()
    x, y, vx, vy, mass, vis, is_ast = diver_scene()
    n = len(x)
    z = vz = None
    if dim == 3:
        rng = np.random.default_rng(9)
        z = rng.normal(0, 0.02, n); z[0] = 0.0
        vz = rng.normal(0, 0.05, n); vz[0] = 0.0
    if massive_ast:
        mass = mass.copy()
        mass[is_ast != 0] = 1e-7
    rr = np.zeros(n); rr[0] = 0.00465          # solar radius: some divers touch it
    vis = vis.copy(); vis[7] = 0               # a frozen asteroid
    K, dt = 3, 1.0 / 365.25
    ost, a, m = oracle_state(x, y, vx, vy, mass, vis, is_ast, rr, z, vz)
    res = of.frame_launch(ost, dt, K, m_sub=8)
    sim = nk.NBodyCuda(0, m_sub=8)
    st = sim.load_state(x, y, vx, vy, mass, vis, is_ast, rr, z=z, vz=vz)
    out = sim.step_batch(st, dt, K)
    ref = full_order(ost, a, m, n)
    f = sim.export_f64(st)
    scale = np.abs(ref).max()
    assert np.abs(f - ref).max() <= 1e-9 * scale
    # snapshot rows: f32 images of the oracle's states
    for ks in range(K):
        row = np.empty(2 * dim * n)
        for c in range(2 * dim):
            row[c * n + a] = res["snap"][ks, c]
            row[c * n + m] = res["snapM"][ks, c]
        assert np.allclose(out[ks], row.astype(np.float32), rtol=3e-7, atol=1e-7)
    # sub-samples of hot asteroids and contacts
    for ks in range(K):
        idx, pos = st["sub"][ks]
        want = a[res["subN"][ks] == 8]
        assert sorted(idx.tolist()) == sorted(want.tolist())
        for col, body in enumerate(idx):
            i = int(np.flatnonzero(a == body)[0])
            assert np.allclose(pos[:, :, col], res["subPos"][ks, :, :, i], rtol=1e-6, atol=1e-6)
    hi, ht, hm = st["hits"]
    want = a[res["hitT"] >= 0]
    assert sorted(hi.tolist()) == sorted(want.tolist())
    for body, t, partner in zip(hi, ht, hm):
        i = int(np.flatnonzero(a == body)[0])
        assert abs(t - res["hitT"][i]) <= 1e-6 * max(1.0, abs(res["hitT"][i]))
        assert partner == m[res["hitM"][i]]


def test_batch_equals_single_steps():
    # test_kernel.py:157-167: K=4 in one launch == 4 single steps, < 1e-6
    nk = _nk()
    state = make_system(500)
    sim = nk.NBodyCuda(0)
    st1 = sim.load_state(*state)
    st2 = sim.load_state(*state)
    raster = 0.5 / 365.25
    batch = sim.step_batch(st1, raster, 4)
    singles = [sim.step(st2, raster) for _ in range(4)]
    assert max(np.max(np.abs(batch[i] - singles[i])) for i in range(4)) < 1e-6


def test_updates_hit_the_right_slots():
    # test_kernel.py:146-155
    nk = _nk()
    state = make_system(5)
    sim = nk.NBodyCuda(0)
    st = sim.load_state(*state)
    n = len(state[0])
    idx = np.array([12, 2], dtype=np.int64)
    vals = np.array([[9.0, -9.0, 0.0, 0.0], [4.0, 4.5, 0.0, 0.0]])
    sim.apply_updates(st, idx, vals)
    out = sim.step(st, 1e-9)
    assert abs(out[12] - 9.0) < 1e-4 and abs(out[n + 12] + 9.0) < 1e-4
    assert abs(out[2] - 4.0) < 1e-4 and abs(out[n + 2] - 4.5) < 1e-4
    # additive deltas, body state, radius, deactivate, export
    f0 = sim.export_f64(st)
    sim.apply_deltas(st, np.array([12, 5]), np.array([[0.5, 0.0, 0.1, 0.0], [0.0, -0.25, 0.0, 0.2]]))
    f1 = sim.export_f64(st)
    assert f1[12] == f0[12] + 0.5 and f1[2 * n + 12] == f0[2 * n + 12] + 0.1
    assert f1[n + 5] == f0[n + 5] - 0.25 and f1[3 * n + 5] == f0[3 * n + 5] + 0.2
    sim.apply_body_state(st, 1, 1.5, 0.0, 0.0, 5.0, 2e-6)
    f2 = sim.export_f64(st)
    assert (f2[1], f2[n + 1], f2[2 * n + 1], f2[3 * n + 1]) == (1.5, 0.0, 0.0, 5.0)
    sim.set_radius(st, 0, 0.01)
    sim.deactivate_body(st, 13)
    before = sim.export_f64(st)
    sim.step(st, 1.0 / 365.25)
    after = sim.export_f64(st)
    assert after[13] == before[13] and after[n + 13] == before[n + 13]
    with pytest.raises(ValueError):
        sim.apply_deltas(st, np.array([12, 12]), np.zeros((2, 4)))


def test_resident_one_year_matches_oracle():
    # test_kernel.py:133-144: 73 x 5-day steps without re-upload
    nk = _nk()
    state = make_system(0)
    sim = nk.NBodyCuda(0)
    st = sim.load_state(*state)
    ost, a, m = oracle_state(*state)
    for _ in range(73):
        out = sim.step(st, 5 / 365.25)
        of.frame_launch(ost, 5 / 365.25, 1)
    n = len(state[0])
    ref = full_order(ost, a, m, n)
    assert np.abs(sim.export_f64(st) - ref).max() < 1e-9 * np.abs(ref).max()
    assert abs(np.hypot(out[3] - out[0], out[n + 3] - out[n]) - 3.0) < 0.1   # frozen planet at 3 AU


def _fine_vv(px, py, pvx, pvy, mu, sx, sy, svx, svy, dt, steps):
    """Fine velocity-Verlet of test particles around a uniformly moving
    point mass (test_subsamples.py:20-42, test_bewegter_stern.py:27-50),
    vectorised over cases; returns the path at every step if asked."""
    h = dt / steps

    def acc(t, px, py):
        dx = (sx + svx * t) - px
        dy = (sy + svy * t) - py
        r2 = dx * dx + dy * dy + of.SOFTENING
        f = mu / (r2 * np.sqrt(r2))
        return f * dx, f * dy

    t = 0.0
    ax, ay = acc(t, px, py)
    path = []
    for _ in range(steps):
        px = px + pvx * h + 0.5 * ax * h * h
        py = py + pvy * h + 0.5 * ay * h * h
        t += h
        nax, nay = acc(t, px, py)
        pvx = pvx + 0.5 * (ax + nax) * h
        pvy = pvy + 0.5 * (ay + nay) * h
        ax, ay = nax, nay
        path.append((px, py))
    return px, py, path


def test_subsamples_lie_on_the_true_orbit():
    # test_subsamples.py: diver hot, far asteroid calm, sub-samples < 1e-4 AU
    nk = _nk()
    ms = nk.SUB_SAMPLES
    sim = nk.NBodyCuda(0, m_sub=ms)
    taucher = (0.15, 0.004, -160.0, 0.0)
    fern = (3.0, 0.0, 0.0, np.sqrt(nk.G_AU / 3.0))
    x = np.array([0.0, taucher[0], fern[0]]); y = np.array([0.0, taucher[1], fern[1]])
    vx = np.array([0.0, taucher[2], fern[2]]); vy = np.array([0.0, taucher[3], fern[3]])
    mass = np.array([1.0, 0.0, 0.0])
    dt_raster = 0.5 / 365.25
    st = sim.load_state(x, y, vx, vy, mass, np.ones(3, np.uint8), np.array([0, 1, 1], np.uint8))
    sim.step_batch(st, dt_raster, 1)
    idx, pos = st["sub"][0]
    assert 1 in idx.tolist() and 2 not in idx.tolist()
    assert pos.shape[0] == ms and pos.shape[1] == 2
    col = idx.tolist().index(1)
    steps = 200_000
    _, _, path = _fine_vv(np.array(taucher[0]), np.array(taucher[1]), np.array(taucher[2]),
                          np.array(taucher[3]), nk.G_AU, 0.0, 0.0, 0.0, 0.0, dt_raster, steps)
    worst = 0.0
    for j in range(ms):
        rx, ry = path[int(round((j + 1) / ms * steps)) - 1]
        worst = max(worst, float(np.hypot(pos[j, 0, col] - rx, pos[j, 1, col] - ry)))
    assert worst < 1e-4


def test_close_pass_of_a_moving_star():
    # test_bewegter_stern.py: < 1e-3 AU for star speeds 0, 0.5, 2, 5 AU/yr
    nk = _nk()
    speeds = np.array([0.0, 0.5, 2.0, 5.0])
    dt = 0.5 / 365.25
    gpu = []
    for v_star in speeds:
        sim = nk.NBodyCuda(0, m_sub=nk.SUB_SAMPLES)
        st = sim.load_state(np.array([0.0, -0.6]), np.array([0.0, -0.25]), np.array([v_star, 11.0]),
                            np.array([0.0, 3.0]), np.array([1.0, 0.0]), np.ones(2, np.uint8),
                            np.array([0, 1], np.uint8))
        out = sim.step_batch(st, dt, 16)
        gpu.append((float(out[-1][1]), float(out[-1][3])))
    n = len(speeds)
    rx, ry, _ = _fine_vv(np.full(n, -0.6), np.full(n, -0.25), np.full(n, 11.0), np.full(n, 3.0), nk.G_AU,
                         0.0, 0.0, speeds, 0.0, dt * 16, 400_000)
    for k in range(n):
        assert np.hypot(gpu[k][0] - rx[k], gpu[k][1] - ry[k]) < 1e-3


def test_argument_errors():
    nk = _nk()
    sim = nk.NBodyCuda(0)
    n = 70
    with pytest.raises(ValueError, match="zu viele massive"):
        sim.load_state(np.arange(n, dtype=float), np.zeros(n), np.zeros(n), np.zeros(n), np.ones(n),
                       np.ones(n, np.uint8), np.zeros(n, np.uint8))
    st = sim.load_state(*make_system(3))
    with pytest.raises(ValueError):
        sim.step_batch(st, 0.01, 0)
    with pytest.raises(ValueError):
        sim.step_batch(st, 0.01, nk.K_MAX + 1)
    with pytest.raises(ValueError):
        nk.NBodyCuda(0, m_sub=nk.SUB_SAMPLES_MAX + 1)


def test_f32_pair_forces_on_the_asteroid_clouds():
    """pair_f32 (FP32 pair forces, FP64 state) on the asteroid-cloud
    configuration's bodies (star, 7 planets, 5 clouds): the accelerations
    against the f64 path within 1e-6 median and 1e-4 maximum relative error,
    and one 0.5-day raster of positions within 1e-9 AU."""
    from solarsystemsimulator_b200 import workloads
    nk = _nk()
    w = workloads.asteroid_clouds(n_per_cloud=4000)
    x, y = w["pos"][0], w["pos"][1]
    vx, vy = w["vel"][0] * 365.25, w["vel"][1] * 365.25
    vis = np.ones(len(x), np.uint8)
    args = (x, y, vx, vy, w["mass"], vis, w["is_ast"], w["radius"])
    sims = [nk.NBodyCuda([0]), nk.NBodyCuda([0], pair_f32=True)]
    sts = [s.load_state(*args) for s in sims]
    for s, st in zip(sims, sts):
        s.step_batch(st, 0.0, 1)                        # no step: the accelerations at the loaded positions
    a64, a32 = (st["aacc"][:, :st["n_ast"]].cpu().numpy() for st in sts)
    rel = np.linalg.norm(a32 - a64, axis=0) / np.linalg.norm(a64, axis=0)
    assert np.median(rel) <= 1e-6 and rel.max() <= 1e-4
    outs = [s.step_batch(st, 0.5 / 365.25, 1) for s, st in zip(sims, sts)]
    f64s = [s.export_f64(st) for s, st in zip(sims, sts)]
    n = len(x)
    assert np.abs(f64s[1][:2 * n] - f64s[0][:2 * n]).max() <= 1e-9
    assert outs[0].shape == outs[1].shape
