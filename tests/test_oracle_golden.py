"""The CPU oracle against the reference's own outputs (golden fixtures).

Pins oracle/ before any GPU result is compared with it.
"""
import numpy as np
import pytest

from oracle import selfgrav as osg


@pytest.mark.parametrize("name", ["selfgrav_accel_n256.npz", "selfgrav_accel_n1000.npz"])
def test_allpairs_accel_matches_reference(load_golden, name):
    g = load_golden(name)
    rec = osg.records(g["x"], g["y"], None, g["G"] * g["m"])
    a = osg.accel(rec, rec, float(g["eps2"]), dim=2)
    scale = np.hypot(g["ax"], g["ay"])
    for k, ref in ((0, g["ax"]), (1, g["ay"])):
        err = np.abs(a[:, k] - ref)
        # the reference sums pairwise (NumPy .sum), the oracle sequentially
        assert np.all(err <= 1e-12 * np.maximum(np.abs(ref), scale)), err.max()


def test_kdk_matches_reference(load_golden):
    g = load_golden("selfgrav_kdk_n128.npz")
    n = len(g["x"])
    pos = np.zeros((n, 3)); vel = np.zeros((n, 3))
    pos[:, 0], pos[:, 1] = g["x"], g["y"]
    vel[:, 0], vel[:, 1] = g["vx"], g["vy"]
    p, v, _ = osg.integrate(pos, vel, g["G"] * g["m"], float(g["eps2"]), float(g["dt"]),
                            int(g["steps"]), dim=2)
    scale_p = np.abs(g["rx"]).max()
    assert np.abs(p[:, 0] - g["rx"]).max() < 1e-11 * scale_p
    assert np.abs(p[:, 1] - g["ry"]).max() < 1e-11 * scale_p
    scale_v = np.abs(g["rvx"]).max()
    assert np.abs(v[:, 0] - g["rvx"]).max() < 1e-9 * scale_v
    assert np.abs(v[:, 1] - g["rvy"]).max() < 1e-9 * scale_v


def test_energy_matches_reference(load_golden):
    g = load_golden("selfgrav_kdk_n128.npz")
    n = len(g["x"])
    pos = np.zeros((n, 3)); vel = np.zeros((n, 3))
    pos[:, 0], pos[:, 1] = g["x"], g["y"]
    vel[:, 0], vel[:, 1] = g["vx"], g["vy"]
    e0 = osg.energy(pos, vel, g["m"], float(g["G"]), float(g["eps2"]), dim=2)
    assert abs(e0 - float(g["e0"])) <= 1e-12 * abs(float(g["e0"]))


def test_3d_reduces_to_2d():
    rng = np.random.default_rng(1)
    n = 300
    rec = osg.records(rng.normal(size=n), rng.normal(size=n), np.zeros(n), rng.uniform(1, 2, n))
    a2 = osg.accel(rec, rec, 1e-2, dim=2)
    a3 = osg.accel(rec, rec, 1e-2, dim=3)
    assert np.array_equal(a2[:, :2], a3[:, :2])
    assert np.all(a3[:, 2] == 0.0)


def test_momentum_conservation_of_oracle():
    rng = np.random.default_rng(2)
    n = 500
    m = rng.uniform(1, 3, n)
    rec = osg.records(rng.normal(size=n), rng.normal(size=n), rng.normal(size=n), m)
    a = osg.accel(rec, rec, 1e-3, dim=3)
    p = (m[:, None] * a[:, :3]).sum(0)
    assert np.abs(p).max() < 1e-12 * (m[:, None] * np.abs(a[:, :3])).sum()


def test_batched_oracle_matches_reference_advance(load_golden):
    """oracle/batched.py's fixed-step Yoshida-4 against the reference's own
    test_kernel.reference_advance (test_kernel.py:16-81) on all-massive
    planetary systems of 3, 7 and 12 bodies whose substep stays at
    MAX_SUB_DT_YEARS: 400 steps, within 1e-13 of the scale (rounding order
    only: the reference's position-Verlet form against kick-drift-kick)."""
    from oracle import batched as ob
    g = load_golden("batched_reference_advance.npz")
    for s in range(3):
        pos = np.stack([g[f"x{s}"], g[f"y{s}"]])
        vel = np.stack([g[f"vx{s}"], g[f"vy{s}"]])
        p, v = ob.yoshida(pos, vel, g[f"m{s}"], float(g["G"]), float(g["dt"]), int(g["steps"]),
                          eps2=float(g["eps2"]))
        rp = np.stack([g[f"rx{s}"], g[f"ry{s}"]])
        rv = np.stack([g[f"rvx{s}"], g[f"rvy{s}"]])
        assert np.abs(p - rp).max() <= 1e-13 * np.abs(rp).max()
        assert np.abs(v - rv).max() <= 1e-13 * np.abs(rv).max()
        assert np.abs(rp - pos).max() > 0.5                     # the systems really moved
