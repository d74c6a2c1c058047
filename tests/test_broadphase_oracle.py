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


@pytest.mark.parametrize("scene", ["wolke", "klumpen", "zwei_wolken", "auf_der_grenze"])
def test_c_oracle_matches_reference_golden(load_golden, scene):
    """oracle/broadphase.c (the multithreaded restatement) against the
    reference's own _hits outputs, full line and stripes."""
    g = load_golden(f"broadphase_{scene}.npz")
    args = (g["x"], g["y"], g["vx"], g["vy"], g["rr"], float(g["dt_y"]), float(g["h"]), float(g["halo"]))
    res, cand = obp.hits_c(*args)
    assert cand == int(g["n_cand"])
    assert (res is None and len(g["hit_i"]) == 0) or (np.array_equal(res[0], g["hit_i"])
                                                     and np.array_equal(res[1], g["hit_j"]))
    for k in (2, 3, 5):
        tot = 0
        for lo, hi in g[f"stripes{k}_bounds"]:
            r, _ = obp.hits_c(*args, lo=lo, hi=hi)
            tot += 0 if r is None else len(r[0])
        assert tot == int(g[f"stripes{k}_count"])


def test_c_oracle_on_the_asteroid_clouds(load_golden):
    """The configured 200,000-asteroid cloud scene (3.1e9 candidates): the C
    restatement reproduces the reference's hit list and candidate count."""
    import hashlib
    from solarsystemsimulator_b200 import workloads
    g = load_golden("broadphase_asteroid_clouds_200k.npz")
    w = workloads.asteroid_clouds(n_per_cloud=int(g["n_per_cloud"]))
    a = np.flatnonzero(w["is_ast"] != 0)
    f = [np.ascontiguousarray(v, dtype=np.float32) for v in
         (w["pos"][0, a], w["pos"][1, a], w["vel"][0, a], w["vel"][1, a], w["radius"][a])]
    d = hashlib.sha256()
    for v in f:
        d.update(v.tobytes())
    assert d.hexdigest() == str(g["digest"])
    res, cand = obp.hits_c(*f, float(g["dt"]), float(g["h"]), float(g["halo"]))
    assert cand == int(g["n_cand"])
    assert np.array_equal(res[0], g["hit_i"]) and np.array_equal(res[1], g["hit_j"])
