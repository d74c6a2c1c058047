"""The few-massive-body oracle against the reference's own NumPy oracle.

oracle/frame.py restates `frame_kernel` (hierarchical steps + hot fine loop)
and the reference's `reference_advance` (all bodies on one adaptive step).
The golden fixtures hold reference_advance outputs computed by the
reference's own code; the tolerances are the reference's GPU-test bars
(test_kernel.py:116-131, :190-219).
"""
import numpy as np

from oracle import frame as of


def _state(g):
    x, y, vx, vy = g["x"], g["y"], g["vx"], g["vy"]
    ast = g["is_ast"] != 0
    a, m = np.flatnonzero(ast), np.flatnonzero(~ast)
    return of.FrameState(np.stack([x[a], y[a]]), np.stack([vx[a], vy[a]]), g["mass"][a], g["vis"][a] != 0,
                         np.zeros(len(a)), np.stack([x[m], y[m]]), np.stack([vx[m], vy[m]]), g["mass"][m],
                         g["vis"][m] != 0, np.zeros(len(m))), a, m


def test_reference_advance_restatement_is_exact(load_golden):
    g = load_golden("frame_system200_5d.npz")
    rx, ry, rvx, rvy = of.reference_advance(float(g["dt"]), g["x"], g["y"], g["vx"], g["vy"], g["mass"],
                                            g["vis"], g["is_ast"])
    for mine, ref in ((rx, g["rx"]), (ry, g["ry"]), (rvx, g["rvx"]), (rvy, g["rvy"])):
        assert np.array_equal(mine, ref)


def test_frame_restatement_matches_reference_calm(load_golden):
    g = load_golden("frame_system200_5d.npz")
    st, a, m = _state(g)
    of.frame_launch(st, float(g["dt"]), 1)
    x = np.empty(len(g["x"])); y = np.empty_like(x); vx = np.empty_like(x); vy = np.empty_like(x)
    x[a], y[a], vx[a], vy[a] = st.ax[0], st.ax[1], st.av[0], st.av[1]
    x[m], y[m], vx[m], vy[m] = st.mx[0], st.mx[1], st.mv[0], st.mv[1]
    err_p = max(np.abs(x - g["rx"]).max(), np.abs(y - g["ry"]).max())
    err_v = max(np.abs(vx - g["rvx"]).max(), np.abs(vy - g["rvy"]).max())
    assert err_p < 5e-6 and err_v < 5e-6
    # the frozen planet (visible[3] = 0) stays put
    assert x[3] == g["x"][3] and y[3] == g["y"][3]


def test_frame_restatement_sun_diver(load_golden):
    g = load_golden("frame_sundiver_8d.npz")
    st, a, m = _state(g)
    of.frame_launch(st, float(g["dt"]), 1)
    x = np.empty(len(g["x"])); y = np.empty_like(x)
    x[a], y[a] = st.ax[0], st.ax[1]
    x[m], y[m] = st.mx[0], st.mx[1]
    dp = np.max(np.hypot(x - g["rx"], y - g["ry"]))
    r_now = np.hypot(x[1:] - x[0], y[1:] - y[0])
    assert dp < 2e-3 and r_now.max() < 0.5
