"""The stream-frame oracle (oracle/frames.py) reproduces the golden frames of
the reference's own build_frame bit for bit (index lists and u16
coordinates of both samples, the box)."""
import numpy as np
import pytest

from oracle import frames as ofr

SCENES = ["wolken", "massenwolke", "autobox_log", "klein_tot"]


@pytest.mark.parametrize("scene", SCENES)
def test_oracle_reproduces_reference_frames(load_golden, scene):
    g = load_golden(f"server_frame_{scene}.npz")
    log_zoom = bool(g["log_zoom"])
    qx0, qy0 = ofr.display_coords(g["x0"], g["y0"], log_zoom)
    box = ofr.make_box(qx0, qy0, tuple(g["view"]))
    assert np.array_equal(np.array(box), g["box"])
    a = g["is_ast"] != 0
    inj = g["injected"] != 0
    for k in range(2):
        t_i = float(g["t0"]) + (k + 1) * float(g["raster_days"])
        alive = g["kill_t"] > t_i - float(g["raster_days"])
        sel, qx, qy = ofr.sample_frame(g[f"x{k}"], g[f"y{k}"], alive, a, inj, box, log_zoom, int(g["budget"]))
        assert np.array_equal(sel, g[f"sel{k}"]) and np.array_equal(qx, g[f"qx{k}"]) and np.array_equal(qy, g[f"qy{k}"])
