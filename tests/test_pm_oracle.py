"""The 2-D PM oracle against the reference's own pm_kernel outputs."""
import numpy as np

from oracle import pm as opm


def test_force_and_density_match_reference(load_golden):
    g = load_golden("pm2d_n2000_g128.npz")
    n = int(g["grid_n"])
    x0, y0, h = opm.grid_fuer(g["x"], g["y"], n)
    assert (x0, y0, h) == (float(g["x0"]), float(g["y0"]), float(g["h"]))
    rho = opm.cic_deposit(g["x"], g["y"], g["m"], n, x0, y0, h)
    assert np.array_equal(rho, g["rho"])
    ax, ay = opm.pm_accelerations(g["x"], g["y"], g["m"], n, x0, y0, h, float(g["eps2"]))
    assert np.array_equal(ax, g["ax"]) and np.array_equal(ay, g["ay"])


def test_kdk_matches_reference(load_golden):
    g = load_golden("pm2d_kdk_n1500.npz")
    rows, f64 = opm.kdk(g["x"], g["y"], g["vx"], g["vy"], g["m"], (g["tx"], g["ty"], g["tvx"], g["tvy"]),
                        float(g["dt"]), int(g["steps"]), int(g["grid_n"]))
    assert np.array_equal(rows, g["out"]) and np.array_equal(f64, g["f64"])
