"""Failure detection without a GPU fault: step guards that run out, bounded
waits that give up, and the checkpoint round trip.

* Guards (nbody_kernel.py:248-250 substeps per raster, :424 the fine loop's
  8000 iterations): the reference stops the interval where a guard runs out
  and goes on silently; this build keeps that behaviour and records
  SSS_ERR_GUARD, which NBodyCuda turns into a RuntimeWarning (or an SSSError
  with strict_guard=True). A guard of 1 forces it.
* Bounded waits: sss_selftest_wait runs the mbarrier wait and the two grid
  barriers with a wait that nothing completes and a 10 ms limit; each gives
  up, the status reads SSS_ERR_TIMEOUT once, and the context stays usable.
* Checkpoint: export_f64 -> load_state -> N steps equals N uninterrupted
  steps bit for bit (the producer's dump, film_producer.py:670-675).
"""
import ctypes
import warnings

import numpy as np
import pytest
import torch

from oracle import frame as of

pytestmark = pytest.mark.gpu


def _calm(n_ast=300, seed=7):
    rng = np.random.default_rng(seed)
    n = 10 + n_ast
    x = np.zeros(n); y = np.zeros(n); vx = np.zeros(n); vy = np.zeros(n)
    mass = np.full(n, 1e-6); mass[0] = 1.0
    is_ast = np.zeros(n, np.uint8); is_ast[10:] = 1
    vis = np.ones(n, np.uint8)
    rp = np.arange(1, 10, dtype=np.float64)
    x[1:10] = rp
    vy[1:10] = np.sqrt(of.G_AU / rp)
    r = 2 + 2 * rng.random(n_ast)
    th = rng.random(n_ast) * 2 * np.pi
    x[10:] = r * np.cos(th); y[10:] = r * np.sin(th)
    v = np.sqrt(of.G_AU / r)
    vx[10:] = -v * np.sin(th); vy[10:] = v * np.cos(th)
    mass[10:] = 0.0
    return x, y, vx, vy, mass, vis, is_ast


def test_substep_guard_runs_out():
    from solarsystemsimulator_b200 import _lib
    from solarsystemsimulator_b200.nbody_kernel import MAX_SUB_DT_YEARS, NBodyCuda
    state = _calm()
    # one raster of two maximal substeps with a guard of one substep
    sim = NBodyCuda([0], max_sub_steps=1)
    st = sim.load_state(*state)
    with pytest.warns(RuntimeWarning, match="guard"):
        out = sim.step_batch(st, 2 * MAX_SUB_DT_YEARS, 1)
    assert st["guard_exhausted"] == 1
    # ... it stopped after that one substep, as the reference does
    ref = NBodyCuda([0])
    st_ref = ref.load_state(*state)
    with warnings.catch_warnings():
        warnings.simplefilter("error")
        out_ref = ref.step_batch(st_ref, MAX_SUB_DT_YEARS, 1)
    assert np.array_equal(out, out_ref)
    assert np.array_equal(sim.export_f64(st), ref.export_f64(st_ref))
    # strict: an error with the status code
    strict = NBodyCuda([0], max_sub_steps=1, strict_guard=True)
    st2 = strict.load_state(*state)
    with pytest.raises(_lib.SSSError) as e:
        strict.step_batch(st2, 2 * MAX_SUB_DT_YEARS, 1)
    assert e.value.code == _lib.SSS_ERR_GUARD
    # the context goes on: a raster the guard allows runs clean
    with warnings.catch_warnings():
        warnings.simplefilter("error")
        strict.step_batch(st2, MAX_SUB_DT_YEARS, 1)


def test_fine_loop_guard_runs_out():
    from solarsystemsimulator_b200 import _lib
    from solarsystemsimulator_b200.nbody_kernel import NBodyCuda
    from test_frame_gpu import diver_scene
    scene = diver_scene()
    raster = 0.5 / 365.25
    with warnings.catch_warnings():
        warnings.simplefilter("error")                  # the divers need fine steps, but far fewer than 8000
        full = NBodyCuda([0])
        full.step_batch(full.load_state(*scene), raster, 2)
    sim = NBodyCuda([0], max_fine_steps=1, strict_guard=True)
    with pytest.raises(_lib.SSSError) as e:
        sim.step_batch(sim.load_state(*scene), raster, 2)
    assert e.value.code == _lib.SSS_ERR_GUARD
    with pytest.raises(ValueError):
        NBodyCuda([0], max_fine_steps=0)


@pytest.mark.parametrize("which", [0, 1, 2])
def test_bounded_waits_give_up(which):
    """0: the mbarrier wait of the bulk-copy / tensor-core kernels, 1: the
    frame kernel's grid barrier, 2: the stream-frame kernel's grid barrier."""
    from solarsystemsimulator_b200 import _lib
    ctx = _lib.context(0)
    s = ctypes.c_void_p(_lib.stream_handle(0))
    assert ctx.lib.sss_device_status(ctx.ptr, s) == _lib.SSS_OK
    assert ctx.lib.sss_selftest_wait(ctx.ptr, which, 0.01, s) == _lib.SSS_OK
    assert ctx.lib.sss_device_status(ctx.ptr, s) == _lib.SSS_ERR_TIMEOUT
    assert ctx.lib.sss_device_status(ctx.ptr, s) == _lib.SSS_OK         # read once, then cleared
    assert ctx.lib.sss_selftest_wait(ctx.ptr, 3, 0.01, s) == _lib.SSS_ERR_ARG
    assert ctx.lib.sss_selftest_wait(ctx.ptr, 0, 0.0, s) == _lib.SSS_ERR_ARG
    # the context is still usable
    from solarsystemsimulator_b200 import selfgrav_kernel as sg
    rng = np.random.default_rng(1)
    b = torch.as_tensor(np.concatenate([rng.uniform(-1, 1, (500, 3)), np.full((500, 1), 1e-3)], 1)).cuda()
    acc = sg.allpairs_accel(b, b, 1e-4)
    assert ctx.lib.sss_device_status(ctx.ptr, s) == _lib.SSS_OK
    assert torch.isfinite(acc).all() and acc.abs().max() > 0


def test_checkpoint_round_trip_frame():
    """NBodyCuda: export_f64 after 3 rasters, a fresh load_state from it, 3
    more rasters == 6 uninterrupted rasters, bit for bit."""
    from solarsystemsimulator_b200.nbody_kernel import NBodyCuda
    from test_frame_gpu import diver_scene
    x, y, vx, vy, mass, vis, is_ast = diver_scene()
    raster = 0.5 / 365.25
    sim = NBodyCuda([0])
    st = sim.load_state(x, y, vx, vy, mass, vis, is_ast)
    whole = [sim.step_batch(st, raster, 3), sim.step_batch(st, raster, 3)]
    sim2 = NBodyCuda([0])
    st2 = sim2.load_state(x, y, vx, vy, mass, vis, is_ast)
    first = sim2.step_batch(st2, raster, 3)
    f = sim2.export_f64(st2)
    n = len(x)
    sim3 = NBodyCuda([0])
    st3 = sim3.load_state(f[0:n], f[n:2 * n], f[2 * n:3 * n], f[3 * n:4 * n], mass, vis, is_ast)
    second = sim3.step_batch(st3, raster, 3)
    assert np.array_equal(first, whole[0]) and np.array_equal(second, whole[1])
    assert np.array_equal(sim3.export_f64(st3), sim.export_f64(st))


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_checkpoint_round_trip_selfgrav(precision):
    """NBodySelfGrav: export_f64 -> load_state -> steps == uninterrupted
    steps, bit for bit (the starting accelerations are recomputed from the
    positions by the same force kernel)."""
    from solarsystemsimulator_b200 import selfgrav_kernel as sg
    rng = np.random.default_rng(4)
    n = 3000
    x, y = rng.normal(0, 1, n), rng.normal(0, 1, n)
    vx, vy = rng.normal(0, 0.1, n), rng.normal(0, 0.1, n)
    m = np.full(n, 1.0 / n)
    kw = dict(softening_au=0.05, G=1.0, integrator="yoshida4", precision=precision)
    a = sg.NBodySelfGrav(0, **kw)
    st = a.load_state(x, y, vx, vy, m)
    a.step_batch(st, 1e-3, 10)
    b = sg.NBodySelfGrav(0, **kw)
    st_b = b.load_state(x, y, vx, vy, m)
    b.step_batch(st_b, 1e-3, 5)
    f = b.export_f64(st_b)
    c = sg.NBodySelfGrav(0, **kw)
    st_c = c.load_state(f[0:n], f[n:2 * n], f[2 * n:3 * n], f[3 * n:4 * n], m)
    c.step_batch(st_c, 1e-3, 5)
    assert np.array_equal(c.export_f64(st_c), a.export_f64(st))


def test_checkpoint_round_trip_pm():
    """NBodyPM: the same round trip (the grid geometry and the force are
    recomputed from the positions at load_state). The deposit adds f64
    masses with atomics, as CuPy's bincount does, so two runs of the same
    steps differ in the last bits: the bar is the PM parity bar, 1e-9 of the
    state scale."""
    from solarsystemsimulator_b200 import pm_kernel as pk
    rng = np.random.default_rng(5)
    n = 2000
    x, y = rng.normal(0, 1e4, n), rng.normal(0, 1e4, n)
    vx, vy = rng.normal(0, 10, n), rng.normal(0, 10, n)
    m = np.full(n, 1e6)
    a = pk.NBodyPM([0], grid_n=256)
    st = a.load_state(x, y, vx, vy, m)
    a.step_batch(st, 0.01, 6)
    b = pk.NBodyPM([0], grid_n=256)
    st_b = b.load_state(x, y, vx, vy, m)
    b.step_batch(st_b, 0.01, 3)
    f = b.export_f64(st_b)
    c = pk.NBodyPM([0], grid_n=256)
    st_c = c.load_state(f[0:n], f[n:2 * n], f[2 * n:3 * n], f[3 * n:4 * n], m)
    c.step_batch(st_c, 0.01, 3)
    ref = a.export_f64(st)
    got = c.export_f64(st_c)
    for q in range(4):
        part = slice(q * n, (q + 1) * n)
        assert np.abs(got[part] - ref[part]).max() <= 1e-9 * np.abs(ref[part]).max()
