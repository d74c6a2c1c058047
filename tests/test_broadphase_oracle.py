"""The broadphase oracle against the reference's own `_hits` outputs."""
import numpy as np
import pytest

from oracle import broadphase as obp

SCENES = ["wolke", "klumpen", "zwei_wolken", "auf_der_grenze"]


@pytest.mark.parametrize("scene", SCENES)
def test_oracle_hits_are_the_reference_hits(load_golden, scene):
    g = load_golden(f"broadphase_{scene}.npz")
    res, cand = obp.hits(g["x"], g["y"], g["vx"], g["vy"], g["rr"], float(g["dt_y"]), float(g["h"]),
                         float(g["halo"]))
    assert cand == int(g["n_cand"])
    assert res is not None
    assert np.array_equal(res[0], g["hit_i"]) and np.array_equal(res[1], g["hit_j"])


@pytest.mark.parametrize("scene", SCENES)
def test_oracle_stripes_union_is_the_full_set(load_golden, scene):
    g = load_golden(f"broadphase_{scene}.npz")
    full = set(zip(g["hit_i"].tolist(), g["hit_j"].tolist()))
    for k in (2, 3, 5):
        got, count = set(), 0
        for lo, hi in g[f"stripes{k}_bounds"]:
            res, _ = obp.hits(g["x"], g["y"], g["vx"], g["vy"], g["rr"], float(g["dt_y"]), float(g["h"]),
                              float(g["halo"]), lo=lo, hi=hi)
            if res is not None:
                part = set(zip(res[0].tolist(), res[1].tolist()))
                assert not (got & part)
                got |= part
                count += len(res[0])
        assert got == full and count == int(g[f"stripes{k}_count"])
