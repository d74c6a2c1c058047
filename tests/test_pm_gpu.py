"""GPU 2-D particle mesh against the reference's pm_kernel outputs and the
reference's own statistical PM tests (test_pm.py).

Parity tolerances: density rtol 1e-12 (atomic deposit order); forces
|d| <= 1e-10 * max|a| (cuFFT vs the reference's FFT rounding); 5 KDK steps:
f64 state within 1e-9 of the state scale, f32 rows within 1e-6 relative.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _pk():
    from solarsystemsimulator_b200 import pm_kernel as pk
    return pk


def test_grid_density_and_forces_match_reference(load_golden):
    pk = _pk()
    g = load_golden("pm2d_n2000_g128.npz")
    n = int(g["grid_n"])
    x0, y0, h = pk.grid_fuer(g["x"], g["y"], n)
    assert (x0, y0, h) == (float(g["x0"]), float(g["y0"]), float(g["h"]))
    rho = pk._cic_deposit(g["x"], g["y"], g["m"], n, x0, y0, h).cpu().numpy()
    assert np.allclose(rho, g["rho"], rtol=1e-12, atol=1e-12 * np.abs(g["rho"]).max())
    ax, ay = pk.pm_accelerations(g["x"], g["y"], g["m"], n, x0, y0, h, float(g["eps2"]))
    scale = max(np.abs(g["ax"]).max(), np.abs(g["ay"]).max())
    assert np.abs(ax.cpu().numpy() - g["ax"]).max() <= 1e-10 * scale
    assert np.abs(ay.cpu().numpy() - g["ay"]).max() <= 1e-10 * scale
    fx, fy = pk.pm_force_field(g["x"], g["y"], g["m"], n, x0, y0, h, float(g["eps2"]))
    assert fx.shape == (n, n) and fy.shape == (n, n)


def test_cic_gather_drop_in(load_golden):
    """_cic_gather(feld, gx, gy, grid_n, x0, y0, h) (pm_kernel.py:93-107) on a
    field the caller holds: bit-identical to the oracle's restatement on a
    random field (points inside the grid, on its clip edges and outside it),
    and on the force field the same values gather_accel returns."""
    from oracle import pm as opm
    pk = _pk()
    rng = np.random.default_rng(17)
    n, x0, y0, h = 96, -3.0, 2.0, 0.05
    feld = rng.normal(0, 1, (n, n))
    px = x0 + rng.uniform(-0.5, n + 0.5, 5000) * h
    py = y0 + rng.uniform(-0.5, n + 0.5, 5000) * h
    px[:4] = [x0, x0 + (n - 1) * h, x0 + (n - 2) * h, x0 + 10.25 * h]
    got = pk._cic_gather(feld, px, py, n, x0, y0, h).cpu().numpy()
    assert np.array_equal(got, opm.cic_gather(feld, px, py, n, x0, y0, h))
    # a non-contiguous field (a crop) is accepted too
    big = rng.normal(0, 1, (n + 8, n + 8))
    got = pk._cic_gather(torch.as_tensor(big).cuda()[:n, :n], px, py, n, x0, y0, h).cpu().numpy()
    assert np.array_equal(got, opm.cic_gather(big[:n, :n], px, py, n, x0, y0, h))
    g = load_golden("pm2d_n2000_g128.npz")
    m = int(g["grid_n"])
    x0, y0, h = float(g["x0"]), float(g["y0"]), float(g["h"])
    fx, fy = pk.pm_force_field(g["x"], g["y"], g["m"], m, x0, y0, h, float(g["eps2"]))
    ax, ay = pk.gather_accel(fx, fy, g["x"], g["y"], m, x0, y0, h)
    assert torch.equal(pk._cic_gather(fx, g["x"], g["y"], m, x0, y0, h), ax)
    assert torch.equal(pk._cic_gather(fy, g["x"], g["y"], m, x0, y0, h), ay)


def test_kdk_matches_reference(load_golden):
    pk = _pk()
    g = load_golden("pm2d_kdk_n1500.npz")
    sim = pk.NBodyPM([0], grid_n=int(g["grid_n"]), softening_zellen=float(g["soft_cells"]))
    st = sim.load_state(g["x"], g["y"], g["vx"], g["vy"], g["m"], tracer=(g["tx"], g["ty"], g["tvx"], g["tvy"]))
    out = sim.step_batch(st, float(g["dt"]), int(g["steps"]))
    assert out.shape == g["out"].shape and out.dtype == np.float32
    f = sim.export_f64(st)
    assert np.abs(f - g["f64"]).max() <= 1e-9 * np.abs(g["f64"]).max()
    assert np.allclose(out, g["out"], rtol=1e-6, atol=1e-6 * np.abs(g["out"]).max())


def _allpairs(x, y, m, eps2, G):
    from solarsystemsimulator_b200 import selfgrav_kernel as sg
    rec = np.zeros((len(x), 4))
    rec[:, 0], rec[:, 1], rec[:, 3] = x, y, G * m
    t = torch.from_numpy(rec).cuda()
    a = sg.allpairs_accel(t, t, eps2, dim=2, precision="f64").cpu().numpy()
    return a[:, 0], a[:, 1]


def test_momentum_conservation():
    # test_pm.py:44-58
    pk = _pk()
    rng = np.random.default_rng(42)
    n = 5000
    x = rng.uniform(-40000, 40000, n); y = rng.uniform(-40000, 40000, n); m = rng.uniform(1e6, 2e7, n)
    x0, y0, h = pk.grid_fuer(x, y, 512)
    ax, ay = (a.cpu().numpy() for a in pk.pm_accelerations(x, y, m, 512, x0, y0, h, (2 * h) ** 2))
    rel = np.hypot(np.sum(m * ax), np.sum(m * ay)) / np.sum(m * np.hypot(ax, ay))
    assert rel < 1e-3


def test_far_pair_matches_newton():
    # test_pm.py:61-78: within 2 % of G m / r^2
    pk = _pk()
    grid_n, h = 512, 100.0
    r = 60 * h
    cx = grid_n * h / 2
    x = np.array([cx - r / 2, cx + r / 2]); y = np.array([cx, cx]); m = np.array([1e10, 1e10])
    ax, _ = pk.pm_accelerations(x, y, m, grid_n, 0.0, 0.0, h, (2 * h) ** 2)
    analytic = pk.G_AU * 1e10 / (r * r)
    assert abs(abs(float(ax[0])) - analytic) / analytic < 0.02


@pytest.mark.parametrize("eps_in_h,bound", [(4.0, 0.03), (1.0, 0.12)])
def test_cloud_against_all_pairs(eps_in_h, bound):
    # test_pm.py:81-100: median relative error below 3 % (eps = 4h) / 12 % (eps = h)
    pk = _pk()
    rng = np.random.default_rng(43)
    n = 4000
    x = rng.uniform(-40000, 40000, n); y = rng.uniform(-40000, 40000, n); m = rng.uniform(1e6, 2e7, n)
    x0, y0, h = pk.grid_fuer(x, y, 512)
    eps2 = (eps_in_h * h) ** 2
    ax, ay = (a.cpu().numpy() for a in pk.pm_accelerations(x, y, m, 512, x0, y0, h, eps2))
    rx, ry = _allpairs(x, y, m, eps2, pk.G_AU)
    rel = np.hypot(ax - rx, ay - ry) / np.maximum(np.hypot(rx, ry), 1e-30)
    assert np.median(rel) < bound


def test_dynamics_conserve_energy_and_momentum():
    # test_pm.py:121-159: 100 KDK steps, energy drift < 3 %, momentum < 1e-6
    pk = _pk()
    from solarsystemsimulator_b200 import selfgrav_kernel as sg
    rng = np.random.default_rng(44)
    n, R, Mtot = 10000, 30000.0, 5.6e9
    r = R * np.sqrt(rng.uniform(0, 1, n)); th = rng.uniform(0, 2 * np.pi, n)
    x = r * np.cos(th); y = r * np.sin(th)
    m = np.full(n, Mtot / n)
    vvir = np.sqrt(pk.G_AU * Mtot / R)
    ang = rng.uniform(0, 2 * np.pi, n)
    vx = 0.7 * vvir * np.cos(ang); vy = 0.7 * vvir * np.sin(ang)
    vx -= np.sum(m * vx) / Mtot; vy -= np.sum(m * vy) / Mtot
    _, _, h = pk.grid_fuer(x, y, 2048, 4.0)
    eps2 = (1.5 * h) ** 2

    def energy(x, y, vx, vy):
        rec = np.zeros((n, 4)); rec[:, 0], rec[:, 1], rec[:, 3] = x, y, pk.G_AU * m
        t = torch.from_numpy(rec).cuda()
        phi = sg.allpairs_potential(t, t, eps2, dim=2).cpu().numpy()
        pot = 0.5 * np.sum(m * phi) + 0.5 * pk.G_AU * np.sum(m * m) / np.sqrt(eps2)
        return 0.5 * np.sum(m * (vx * vx + vy * vy)) + pot

    e0 = energy(x, y, vx, vy)
    sim = pk.NBodyPM([0], grid_n=2048, softening_zellen=1.5)
    st = sim.load_state(x, y, vx, vy, m)
    sim.step_batch(st, (R / vvir) / 1000.0, 100)
    f = sim.export_f64(st)
    e1 = energy(f[:n], f[n:2 * n], f[2 * n:3 * n], f[3 * n:])
    p_rel = np.hypot(np.sum(m * f[2 * n:3 * n]), np.sum(m * f[3 * n:])) / np.hypot(np.sum(m * np.abs(vx)),
                                                                                     np.sum(m * np.abs(vy)))
    assert abs(e1 - e0) / abs(e0) < 0.03 and p_rel < 1e-6
