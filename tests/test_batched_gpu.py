"""Batched small systems against the per-system f64 oracle.

Tolerances: positions and velocities within 1e-9 of their scale after 50
steps (f64, different rsqrt/FMA rounding only); every team mapping, the
graph replay and one-launch-per-system give bit-identical states (each body
sums its partners in the same order in all of them).
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


def test_mappings_graph_and_single_launches_agree():
    from solarsystemsimulator_b200 import batched
    systems = _ens(120, 12, seed=5)
    runs = []
    for variant in range(4):
        ens = batched.BatchedSystems(systems, device=0, autotune=(variant == 0))
        if variant == 1:
            for g in ens.groups:
                g["map"] = batched.candidates(g["max_n"])[-1]        # largest team
        if variant == 2:
            ens.capture(30)
            ens.replay()
        elif variant == 3:
            ens.run_one_launch_per_system(30)
        else:
            ens.run(30)
        torch.cuda.synchronize()
        runs.append(np.concatenate([np.concatenate([p, v], 1) for p, v in ens.export()], 1))
    for r in runs[1:]:
        assert np.array_equal(r, runs[0])


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
