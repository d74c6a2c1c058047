"""Batched small systems against the per-system f64 oracle.

Tolerances: positions and velocities within 1e-9 of their scale after 50
steps (f64, different rsqrt/FMA rounding only); every team mapping, the
graph replay and one-launch-per-system give bit-identical states (each body
sums its partners in the same order in all of them); the block-per-system
mappings (partial sums over source chunks) agree to 1e-12 of the scale.
"""
import numpy as np
import pytest
import torch

from oracle import batched as ob

pytestmark = pytest.mark.gpu


def _ens(n=240, f8=24, seed=3):
    from solarsystemsimulator_b200 import workloads
    return workloads.batched_ensemble(n, f8, seed)


def test_matches_oracle_per_system():
    from solarsystemsimulator_b200 import batched
    systems = _ens()
    ens = batched.BatchedSystems(systems, device=0)
    steps = 50
    ens.run(steps)
    out = ens.export()
    for s, (p, v) in zip(systems, out):
        rp, rv = ob.yoshida(s["pos"], s["vel"], s["mass"], s["G"], s["dt"], steps)
        assert np.abs(p - rp).max() <= 1e-9 * max(np.abs(rp).max(), 1e-30)
        assert np.abs(v - rv).max() <= 1e-9 * max(np.abs(rv).max(), 1e-30)


def _state(ens):
    return np.concatenate([np.concatenate([p, v], 1) for p, v in ens.export()], 1)


def test_mappings_graph_and_single_launches_agree():
    """Team mappings (shuffles, one lane per target), the graph replay and
    one launch per system sum every body's partners in the same order:
    bit-identical states. The block-per-system mappings add the partial sums
    of their source chunks, and the autotuner may pick them: within 1e-12 of
    the scale."""
    from solarsystemsimulator_b200 import batched
    systems = _ens(120, 12, seed=5)
    steps = 30

    def run(variant, maps=None):
        ens = batched.BatchedSystems(systems, device=0, autotune=(variant == "tuned"))
        if maps is not None:
            for g in ens.groups:
                g["map"] = maps(g)
        if variant == "graph":
            ens.capture(steps)
            ens.replay()
        elif variant == "single":
            ens.run_one_launch_per_system(steps)
        else:
            ens.run(steps)
        torch.cuda.synchronize()
        return _state(ens)

    base = run("default")
    widest_team = lambda g: [m for m in batched.candidates(g["max_n"]) if m[0] <= 32][-1]
    for r in (run("default", widest_team), run("graph"), run("single")):
        assert np.array_equal(r, base)
    scale = np.abs(base).max(axis=0, keepdims=True)
    for k in range(3):
        def blocks(g, k=k):
            if g["max_n"] <= 8:
                return g["map"]
            maps = batched.BLOCK_MAPS[batched.block_bucket(g["max_n"])]
            return maps[k % len(maps)]
        r = run("default", blocks)
        assert np.all(np.abs(r - base) <= 1e-12 * np.maximum(scale, 1e-30))
    r = run("tuned")
    assert np.all(np.abs(r - base) <= 1e-12 * np.maximum(scale, 1e-30))


def test_figure8_conserves_energy_over_a_period():
    from solarsystemsimulator_b200 import batched, workloads
    pos, vel, m = workloads.figure8()
    sysd = {"pos": pos, "vel": vel, "mass": m, "G": 1.0, "dt": 1e-3 * workloads.FIGURE8_PERIOD}
    ens = batched.BatchedSystems([sysd] * 8, device=0)
    e0 = ob.energy(pos, vel, m, 1.0)
    ens.run(1000)
    p, v = ens.export()[0]
    assert abs((ob.energy(p, v, m, 1.0) - e0) / e0) < 1e-10
    # after one period the choreography closes on itself
    assert np.abs(p - pos).max() < 1e-4


def test_rejects_oversized_systems():
    from solarsystemsimulator_b200 import batched
    big = {"pos": np.zeros((3, 65)), "vel": np.zeros((3, 65)), "mass": np.ones(65), "G": 1.0, "dt": 1e-3}
    with pytest.raises(ValueError):
        batched.BatchedSystems([big], device=0)


def test_matches_reference_advance_golden(load_golden):
    """The batched kernel against the reference's own reference_advance
    (test_kernel.py:16-81) on all-massive systems whose substep stays at
    MAX_SUB_DT_YEARS (fixture by tests/golden/make_golden.py): 400 Yoshida-4
    steps, 2-D, each system also repeated so every size group holds many."""
    from solarsystemsimulator_b200 import batched
    g = load_golden("batched_reference_advance.npz")
    base = []
    for s in range(3):
        base.append({"pos": np.stack([g[f"x{s}"], g[f"y{s}"]]), "vel": np.stack([g[f"vx{s}"], g[f"vy{s}"]]),
                     "mass": g[f"m{s}"], "G": float(g["G"]), "dt": float(g["dt"])})
    systems = [base[k % 3] for k in range(300)]
    ens = batched.BatchedSystems(systems, device=0, eps2=float(g["eps2"]), dim=2)
    ens.run(int(g["steps"]))
    for k, (p, v) in enumerate(ens.export()):
        s = k % 3
        rp = np.stack([g[f"rx{s}"], g[f"ry{s}"]])
        rv = np.stack([g[f"rvx{s}"], g[f"rvy{s}"]])
        assert np.abs(p - rp).max() <= 1e-12 * np.abs(rp).max()
        assert np.abs(v - rv).max() <= 1e-12 * np.abs(rv).max()
