"""GPU parity of the all-pairs self-gravity path against the CPU oracle.

Tolerances:
* f64 path: per component |a - a_ref| <= 1e-12 * max(|a_ref_c|, |a_ref|)
  (the plain-f64 parity bar), golden fixtures and oracle alike.
* mixed path: median relative force error <= 1e-5 against the f64 oracle.
Mirrors the reference's own test_selfgrav.py questions A (circular orbit),
B (energy), C (determinism), F (tracers).
"""
import numpy as np
import pytest
import torch

from oracle import selfgrav as osg

pytestmark = pytest.mark.gpu

PARITY = 1e-12


def _sg():
    from solarsystemsimulator_b200 import selfgrav_kernel as sg
    return sg


def parity_ok(a, ref, dim):
    scale = np.linalg.norm(ref[:, :dim], axis=1)
    err = np.abs(a[:, :dim] - ref[:, :dim])
    bound = PARITY * np.maximum(np.abs(ref[:, :dim]), scale[:, None])
    return bool(np.all(err <= bound)), float((err / np.maximum(bound / PARITY, 1e-300)).max())


def cloud(n, dim, seed, box=1.0):
    rng = np.random.default_rng(seed)
    rec = np.zeros((n, 4))
    rec[:, :dim] = rng.uniform(-box / 2, box / 2, (n, dim))
    rec[:, 3] = rng.uniform(0.5, 1.5, n) / n
    return rec


def test_library_loads_on_gpu():
    from solarsystemsimulator_b200 import _lib
    lib = _lib.load()
    assert lib.sss_abi_version() == 1
    assert _lib.context(0).num_sms > 0


@pytest.mark.parametrize("name", ["selfgrav_accel_n256.npz", "selfgrav_accel_n1000.npz"])
def test_f64_accel_matches_reference_golden(load_golden, name):
    sg = _sg()
    g = load_golden(name)
    rec = osg.records(g["x"], g["y"], None, g["G"] * g["m"])
    t = torch.from_numpy(rec).cuda()
    a = sg.allpairs_accel(t, t, float(g["eps2"]), dim=2, precision="f64").cpu().numpy()
    ref = np.stack([g["ax"], g["ay"], np.zeros_like(g["ax"]), np.zeros_like(g["ax"])], 1)
    ok, worst = parity_ok(a, ref, 2)
    assert ok, worst


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("n_src,n_tgt", [(1, 1), (2, 7), (511, 513), (1025, 300), (4096, 4096),
                                         (20000, 20000)])
def test_f64_accel_parity_with_oracle(dim, n_src, n_tgt):
    sg = _sg()
    src = cloud(n_src, dim, seed=n_src)
    tgt = cloud(n_tgt, dim, seed=n_tgt + 1)
    tgt[: min(n_src, n_tgt)] = src[: min(n_src, n_tgt)]   # include self terms
    eps2 = 1e-4
    ref = osg.accel(src, tgt, eps2, dim=dim)
    a = sg.allpairs_accel(torch.from_numpy(src).cuda(), torch.from_numpy(tgt).cuda(), eps2,
                          dim=dim, precision="f64").cpu().numpy()
    ok, worst = parity_ok(a, ref, dim)
    assert ok, worst
    assert np.all(a[:, 3] == 0.0)


@pytest.mark.parametrize("precision,tol", [("f64", None), ("mixed", 1e-5)])
def test_equal_mass_tiles_and_mixed_tiles(precision, tol):
    # equal-mass tiles take the mass-factored loop, others the general loop
    sg = _sg()
    rng = np.random.default_rng(21)
    n = 9000
    src = np.zeros((n, 4))
    src[:, :3] = rng.uniform(-0.5, 0.5, (n, 3))
    src[:, 3] = 1.0 / n
    src[600:700, 3] *= rng.uniform(0.5, 2.0, 100)      # tile 1 (f64) / tile 1 (mixed)
    src[5000, 3] = 3.0 / n                               # one odd mass in a later tile
    ref = osg.accel(src, src, 1e-4, dim=3)
    t = torch.from_numpy(src).cuda()
    a = sg.allpairs_accel(t, t, 1e-4, dim=3, precision=precision).cpu().numpy()
    if tol is None:
        ok, worst = parity_ok(a, ref, 3)
        assert ok, worst
    else:
        rel = np.linalg.norm(a[:, :3] - ref[:, :3], axis=1) / np.linalg.norm(ref[:, :3], axis=1)
        assert np.median(rel) <= tol


def test_f64_accel_is_deterministic():
    sg = _sg()
    src = torch.from_numpy(cloud(30000, 3, 5)).cuda()
    a1 = sg.allpairs_accel(src, src, 1e-6, dim=3).cpu().numpy()
    a2 = sg.allpairs_accel(src, src, 1e-6, dim=3).cpu().numpy()
    assert np.array_equal(a1, a2)


def test_zero_targets_and_bad_args():
    sg = _sg()
    src = torch.from_numpy(cloud(10, 3, 1)).cuda()
    empty = torch.zeros((0, 4), dtype=torch.float64, device="cuda")
    out = sg.allpairs_accel(src, empty, 1e-4)
    assert out.shape == (0, 4)
    with pytest.raises(ValueError):
        sg.allpairs_accel(src, src, 1e-4, dim=4)
    with pytest.raises(ValueError):
        sg.allpairs_accel(src.float(), src, 1e-4)


@pytest.mark.parametrize("dim", [2, 3])
def test_mixed_accel_error_below_1e5(dim):
    sg = _sg()
    # a clustered cloud (close pairs) and a lattice-like one
    rng = np.random.default_rng(11)
    n = 30000
    rec = np.zeros((n, 4))
    cen = rng.uniform(-0.5, 0.5, (30, dim))
    rec[:, :dim] = cen[rng.integers(0, 30, n)] + rng.normal(0, 0.02, (n, dim))
    rec[:, 3] = 1.0 / n
    eps2 = 1e-6
    t = torch.from_numpy(rec).cuda()
    a64 = sg.allpairs_accel(t, t, eps2, dim=dim, precision="f64").cpu().numpy()[:, :dim]
    amx = sg.allpairs_accel(t, t, eps2, dim=dim, precision="mixed").cpu().numpy()[:, :dim]
    rel = np.linalg.norm(amx - a64, axis=1) / np.linalg.norm(a64, axis=1)
    assert np.median(rel) <= 1e-5, np.median(rel)
    assert np.percentile(rel, 99) <= 1e-3


def test_potential_matches_oracle():
    sg = _sg()
    src = cloud(3000, 3, 9)
    ref = osg.potential(src, src, 1e-4, dim=3)
    t = torch.from_numpy(src).cuda()
    phi = sg.allpairs_potential(t, t, 1e-4, dim=3).cpu().numpy()
    assert np.allclose(phi, ref, rtol=1e-12, atol=0)


def test_kdk_trajectory_matches_reference_golden(load_golden):
    sg = _sg()
    g = load_golden("selfgrav_kdk_n128.npz")
    sim = sg.NBodySelfGrav(0, softening_au=float(np.sqrt(g["eps2"])), kraft_f32=False)
    st = sim.load_state(g["x"], g["y"], g["vx"], g["vy"], g["m"])
    out = sim.step_batch(st, float(g["dt"]), int(g["steps"]))
    n = len(g["x"])
    assert out.shape == (int(g["steps"]), 4 * n) and out.dtype == np.float32
    f = sim.export_f64(st)
    scale = np.abs(g["rx"]).max()
    assert np.abs(f[:n] - g["rx"]).max() < 1e-10 * scale
    assert np.abs(f[n:2 * n] - g["ry"]).max() < 1e-10 * scale
    vs = np.abs(g["rvx"]).max()
    assert np.abs(f[2 * n:3 * n] - g["rvx"]).max() < 1e-8 * vs
    # last snapshot row is the f32 image of the f64 state
    assert np.array_equal(out[-1], f.astype(np.float32))


@pytest.mark.parametrize("integrator", ["kdk", "yoshida4"])
def test_integrator_matches_oracle_3d_with_tracers(integrator):
    sg = _sg()
    rng = np.random.default_rng(3)
    n, T, dim = 700, 300, 3
    pos = rng.uniform(-0.5, 0.5, (n + T, 3))
    vel = rng.normal(0, 0.1, (n + T, 3))
    m = np.full(n, 1.0 / n)
    eps = 1e-2
    dt, steps = 1e-3, 4
    w = (1.0,) if integrator == "kdk" else (osg.YOSHIDA_W1, osg.YOSHIDA_W0, osg.YOSHIDA_W1)
    rp, rv, _, snaps = osg.integrate(pos, vel, m, eps * eps, dt, steps, dim=3, n_src=n,
                                     weights=w, snapshots=True)
    sim = sg.NBodySelfGrav(0, softening_au=eps, G=1.0, integrator=integrator, precision="f64")
    st = sim.load_state(pos[:n, 0], pos[:n, 1], vel[:n, 0], vel[:n, 1], m, z=pos[:n, 2],
                        vz=vel[:n, 2], tracer=(pos[n:, 0], pos[n:, 1], vel[n:, 0], vel[n:, 1]),
                        tracer_z=(pos[n:, 2], vel[n:, 2]))
    out = sim.step_batch(st, dt, steps)
    assert out.shape == (steps, 6 * n + 3 * T)
    f = sim.export_f64(st).reshape(6, n)
    ft = sim.export_tracers_f64(st).reshape(6, T)
    for k in range(3):
        assert np.abs(f[k] - rp[:n, k]).max() < 1e-12
        assert np.abs(f[3 + k] - rv[:n, k]).max() < 1e-10
        assert np.abs(ft[k] - rp[n:, k]).max() < 1e-12
    assert np.abs(out - snaps).max() < 1e-6


def test_two_body_circular_orbit_closes():
    # reference question A (test_selfgrav.py:101-123)
    sg = _sg()
    G = sg.G_AU
    m, r = 1.0, 1.0
    v = np.sqrt(G * m / (4 * r))
    periode = 2 * np.pi * r / v
    steps = 20000
    sim = sg.NBodySelfGrav(0, softening_au=1e-4, kraft_f32=False)
    st = sim.load_state(np.array([-r, r]), np.zeros(2), np.zeros(2), np.array([-v, v]),
                        np.array([m, m]))
    for _ in range(10):
        sim.step_batch_device(st, periode / steps, steps // 10, snapshots=False)
    z = sim.export_f64(st)
    assert np.hypot(z[0] + r, z[2]) < 1e-4 * 2 * r


@pytest.mark.parametrize("kraft_f32", [False, True])
def test_energy_conservation_n400(kraft_f32):
    # reference question B (test_selfgrav.py:126-152): |dE/E| < 5e-4
    sg = _sg()
    rng = np.random.default_rng(7)
    n, steps, dt = 400, 8000, 0.0055
    BOX, M, EPS = 100_000.0, 1.12e7, 100.0
    x = rng.uniform(-BOX / 2, BOX / 2, n)
    y = rng.uniform(-BOX / 2, BOX / 2, n)
    mass = np.full(n, M)
    v_typ = np.sqrt(sg.G_AU * mass.sum() / (BOX / 2))
    th = rng.uniform(0, 2 * np.pi, n)
    vx, vy = v_typ * 0.4 * np.cos(th), v_typ * 0.4 * np.sin(th)
    sim = sg.NBodySelfGrav(0, softening_au=EPS, kraft_f32=kraft_f32)
    st = sim.load_state(x, y, vx, vy, mass)
    e0 = sim.energy(st)
    for _ in range(4):
        sim.step_batch_device(st, dt, steps // 4, snapshots=False)
    e1 = sim.energy(st)
    assert abs((e1 - e0) / e0) < 5e-4


def test_tracer_follows_field_without_back_reaction():
    # reference question F (test_selfgrav.py:227-258)
    sg = _sg()
    G = sg.G_AU
    m, r = 1.0, 5.0
    v = np.sqrt(G * m / r)
    periode = 2 * np.pi * r / v
    steps = 20000
    sim = sg.NBodySelfGrav(0, softening_au=1e-4)
    st = sim.load_state(np.array([0.0]), np.array([0.0]), np.array([0.0]), np.array([0.0]),
                        np.array([m]), tracer=(np.array([r]), np.array([0.0]), np.array([0.0]),
                                               np.array([v])))
    out = sim.step_batch(st, periode / steps, steps)
    n, mt = st["N"], st["T"]
    tx, ty = float(out[-1][4 * n]), float(out[-1][4 * n + mt])
    assert np.hypot(tx - r, ty) < 1e-3 * r
    assert abs(float(out[-1][0])) + abs(float(out[-1][n])) == 0.0


def test_batches_equal_one_long_batch():
    sg = _sg()
    rng = np.random.default_rng(1)
    n = 2000
    x, y = rng.normal(size=n), rng.normal(size=n)
    vx, vy = rng.normal(0, 0.1, n), rng.normal(0, 0.1, n)
    m = np.full(n, 1.0 / n)
    sim = sg.NBodySelfGrav(0, softening_au=0.05, G=1.0, integrator="yoshida4", precision="f64")
    s1 = sim.load_state(x, y, vx, vy, m)
    s2 = sim.load_state(x, y, vx, vy, m)
    a = sim.step_batch(s1, 1e-3, 6)
    b = np.concatenate([sim.step_batch(s2, 1e-3, 2) for _ in range(3)])
    assert np.array_equal(a, b)
    assert np.array_equal(sim.export_f64(s1), sim.export_f64(s2))


def test_step_batch_argument_errors():
    sg = _sg()
    sim = sg.NBodySelfGrav(0, softening_au=0.1)
    with pytest.raises(ValueError):
        sim.load_state(np.zeros(0), np.zeros(0), np.zeros(0), np.zeros(0), np.zeros(0))
    st = sim.load_state(np.zeros(2), np.array([0.0, 1.0]), np.zeros(2), np.zeros(2), np.ones(2))
    with pytest.raises(ValueError):
        sim.step_batch(st, 0.01, 0)
    with pytest.raises(ValueError):
        sim.step_batch(None, 0.01, 1)
    with pytest.raises(ValueError):
        sg.NBodySelfGrav(0, softening_au=0.0)
