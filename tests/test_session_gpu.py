"""The C-ABI sessions (sss_sg_*, sss_nbody_*) against the Python classes.

A host without torch drives the library through these sessions with plain
host arrays. They run the same kernels on the same inputs as NBodySelfGrav
and NBodyCuda, so every result must be bit-identical to the classes':
snapshots, exported f64 state, contacts, sub-sample chains, and the state
after point updates. Error paths return the reference's messages.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lib():
    from solarsystemsimulator_b200 import _lib
    return _lib


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else ctypes.c_void_p(0)


def _cloud(n, T, dim, seed):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-0.5, 0.5, (n + T, 3))
    vel = rng.normal(0, 0.05, (n + T, 3))
    if dim == 2:
        pos[:, 2] = 0.0
        vel[:, 2] = 0.0
    m = rng.uniform(0.5, 1.5, n) / n
    return pos, vel, m


@pytest.mark.parametrize("precision,dim", [("f64", 3), ("mixed", 3), ("mixed_tc", 3), ("f64", 2)])
def test_selfgrav_session_equals_class(precision, dim):
    from solarsystemsimulator_b200 import selfgrav_kernel as sg
    L = _lib()
    ctx = L.context(0)
    lib = ctx.lib
    n, T, steps, dt = 900, 400, 4, 1e-3
    pos, vel, m = _cloud(n, T, dim, 11)
    sim = sg.NBodySelfGrav(0, softening_au=1e-2, G=1.0, integrator="yoshida4", precision=precision)
    kw = dict(tracer=(pos[n:, 0], pos[n:, 1], vel[n:, 0], vel[n:, 1]))
    if dim == 3:
        kw.update(z=pos[:n, 2], vz=vel[:n, 2], tracer_z=(pos[n:, 2], vel[n:, 2]))
    st = sim.load_state(pos[:n, 0], pos[:n, 1], vel[:n, 0], vel[:n, 1], m, **kw)
    ref = sim.step_batch(st, dt, steps)
    ref_f = sim.export_f64(st)

    s = ctypes.c_void_p()
    ctx.check(lib.sss_sg_create(ctx.ptr, sg._PRECISIONS[precision], L.INT_YOSHIDA4, 1.0, 1e-2, ctypes.byref(s)))
    try:
        soa = np.ascontiguousarray(np.concatenate([pos[:n, :dim].T, vel[:n, :dim].T]).ravel())
        tsoa = np.ascontiguousarray(np.concatenate([pos[n:, :dim].T, vel[n:, :dim].T]).ravel())
        assert lib.sss_sg_row_width(s) == 0
        ctx.check(lib.sss_sg_load(s, dim, n, _ptr(soa), _ptr(m), T, _ptr(tsoa)))
        row = lib.sss_sg_row_width(s)
        assert row == 2 * dim * n + dim * T == ref.shape[1]
        snap = np.empty((steps, row), np.float32)
        ctx.check(lib.sss_sg_step_batch(s, dt, steps, _ptr(snap)))
        out = np.empty(2 * dim * n)
        ctx.check(lib.sss_sg_export_f64(s, _ptr(out)))
        assert np.array_equal(snap, ref)
        assert np.array_equal(out, ref_f)
        # a batch without snapshots advances the same way
        ref2 = sim.step_batch(st, dt, 2)
        ctx.check(lib.sss_sg_step_batch(s, dt, 1, None))
        snap1 = np.empty((1, row), np.float32)
        ctx.check(lib.sss_sg_step_batch(s, dt, 1, _ptr(snap1)))
        assert np.array_equal(snap1[0], ref2[1])
    finally:
        lib.sss_sg_destroy(s)


def test_selfgrav_session_errors():
    L = _lib()
    ctx = L.context(0)
    lib = ctx.lib
    s = ctypes.c_void_p()
    assert lib.sss_sg_create(ctx.ptr, L.PREC_F64, L.INT_KDK, 1.0, 0.0, ctypes.byref(s)) == L.SSS_ERR_ARG
    assert b"Softening muss positiv sein" in lib.sss_last_error(ctx.ptr)
    ctx.check(lib.sss_sg_create(ctx.ptr, L.PREC_F64, L.INT_KDK, 1.0, 0.1, ctypes.byref(s)))
    try:
        assert lib.sss_sg_step_batch(s, 1e-3, 1, None) == L.SSS_ERR_ARG
        assert b"kein Zustand geladen" in lib.sss_last_error(ctx.ptr)
        one = np.zeros(4)
        assert lib.sss_sg_load(s, 2, 0, _ptr(one), _ptr(one), 0, None) == L.SSS_ERR_ARG
        assert b"leerer Zustand" in lib.sss_last_error(ctx.ptr)
        soa = np.array([0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0])   # two bodies, 2-D
        ctx.check(lib.sss_sg_load(s, 2, 2, _ptr(soa), _ptr(np.ones(2)), 0, None))
        assert lib.sss_sg_step_batch(s, 1e-3, 0, None) == L.SSS_ERR_ARG
        assert b"steps muss >= 1 sein" in lib.sss_last_error(ctx.ptr)
    finally:
        lib.sss_sg_destroy(s)


def _diver_scene(dim):
    """Sun (with a contact radius) + 3 planets + asteroids diving at the sun
    (hot, sub-samples, contacts) + a calm belt; optional 3-D tilt."""
    rng = np.random.default_rng(3)
    G = 4 * np.pi ** 2
    x, y, z, vx, vy, vz, mass, is_ast, rr = [0.0], [0.0], [0.0], [0.0], [0.0], [0.0], [1.0], [0], [0.00465]
    for r in (0.7, 1.5, 5.2):
        x.append(r); y.append(0.0); z.append(0.0); vx.append(0.0); vy.append(np.sqrt(G / r)); vz.append(0.0)
        mass.append(3e-6); is_ast.append(0); rr.append(3e-5)
    for k in range(14):
        t = rng.random() * 2 * np.pi
        r0 = 0.05 + 0.05 * rng.random()
        b = 0.01 * rng.random()
        sp = 20.0 + 20.0 * rng.random()
        ux, uy = -np.cos(t), -np.sin(t)
        x.append(r0 * np.cos(t) - b * uy); y.append(r0 * np.sin(t) + b * ux); z.append(0.0)
        vx.append(sp * ux); vy.append(sp * uy); vz.append(0.0)
        mass.append(0.0); is_ast.append(1); rr.append(1e-7)
    for k in range(40):
        r = 2.2 + 0.02 * k
        t = 0.37 * k
        v = np.sqrt(G / r)
        x.append(r * np.cos(t)); y.append(r * np.sin(t)); z.append(0.01 * np.sin(k) if dim == 3 else 0.0)
        vx.append(-v * np.sin(t)); vy.append(v * np.cos(t)); vz.append(0.0)
        mass.append(1e-12 if k % 5 == 0 else 0.0); is_ast.append(1); rr.append(1e-7)
    a = [np.array(q, np.float64) for q in (x, y, z, vx, vy, vz, mass, rr)]
    vis = np.ones(len(x), np.uint8)
    vis[5] = 0
    return a + [vis, np.array(is_ast, np.uint8)]


def _class_and_session(dim, k):
    from solarsystemsimulator_b200 import nbody_kernel as nk
    L = _lib()
    ctx = L.context(0)
    lib = ctx.lib
    x, y, z, vx, vy, vz, mass, rr, vis, is_ast = _diver_scene(dim)
    n = len(x)
    sim = nk.NBodyCuda(0, m_sub=8)
    kw = dict(z=z, vz=vz) if dim == 3 else {}
    st = sim.load_state(x, y, vx, vy, mass, vis, is_ast, rr, **kw)
    s = ctypes.c_void_p()
    ctx.check(lib.sss_nbody_create(ctx.ptr, None, ctypes.byref(s)))
    P = [x, y] + ([z] if dim == 3 else [])
    V = [vx, vy] + ([vz] if dim == 3 else [])
    soa = np.ascontiguousarray(np.concatenate(P + V))
    ctx.check(lib.sss_nbody_load(s, dim, n, _ptr(soa), _ptr(mass), _ptr(vis), _ptr(is_ast), _ptr(rr)))
    return sim, st, s, n, ctx, lib


def _session_batch(ctx, lib, s, dim, n, k, dt):
    snap = np.empty((k, 2 * dim * n), np.float32)
    ctx.check(lib.sss_nbody_step_batch(s, dt, k, _ptr(snap)))
    nh = ctypes.c_int64()
    ctx.check(lib.sss_nbody_hits(s, ctypes.byref(nh), None, None, None, 0))
    hi = np.empty(max(nh.value, 1), np.int64)
    ht = np.empty(max(nh.value, 1), np.float32)
    hm = np.empty(max(nh.value, 1), np.int64)
    ctx.check(lib.sss_nbody_hits(s, ctypes.byref(nh), _ptr(hi), _ptr(ht), _ptr(hm), nh.value))
    subs = []
    for q in range(k):
        c = ctypes.c_int64()
        ctx.check(lib.sss_nbody_sub(s, q, ctypes.byref(c), None, None, 0))
        idx = np.empty(max(c.value, 1), np.int64)
        pos = np.empty(max(8 * dim * c.value, 1), np.float32)
        ctx.check(lib.sss_nbody_sub(s, q, ctypes.byref(c), _ptr(idx), _ptr(pos), c.value))
        subs.append((idx[:c.value], pos[:8 * dim * c.value].reshape(8, dim, c.value)))
    return snap, (hi[:nh.value], ht[:nh.value], hm[:nh.value]), subs


def _assert_batch_equal(out, st, snap, hits, subs):
    assert np.array_equal(snap, out)
    for a, b in zip(st["hits"], hits):
        assert np.array_equal(np.asarray(a), b)
    assert len(st["sub"]) == len(subs)
    for (ai, ap), (bi, bp) in zip(st["sub"], subs):
        assert np.array_equal(ai, bi)
        assert np.array_equal(ap, bp)


@pytest.mark.parametrize("dim", [2, 3])
def test_nbody_session_equals_class(dim):
    k, dt = 4, 1.5e-3
    sim, st, s, n, ctx, lib = _class_and_session(dim, k)
    try:
        out = sim.step_batch(st, dt, k)
        snap, hits, subs = _session_batch(ctx, lib, s, dim, n, k, dt)
        _assert_batch_equal(out, st, snap, hits, subs)
        assert len(hits[0]) > 0 and sum(len(i) for i, _ in subs) > 0   # the scene exercises both
        ref_f = sim.export_f64(st)
        f = np.empty(2 * dim * n)
        ctx.check(lib.sss_nbody_export_f64(s, _ptr(f)))
        assert np.array_equal(f, ref_f)

        # point updates: absolute, additive, full body state; radius; deactivation
        w = 2 * dim
        idx0 = np.array([2, 30, 40], np.int64)
        v0 = np.ascontiguousarray(ref_f.reshape(w, n)[:, idx0].T * 1.001)
        sim.apply_updates(st, idx0, v0)
        ctx.check(lib.sss_nbody_scatter(s, _ptr(idx0), _ptr(v0), 3, 0))
        idx1 = np.array([41, 3], np.int64)
        d1 = np.full((2, w), 1e-6)
        sim.apply_deltas(st, idx1, d1)
        ctx.check(lib.sss_nbody_scatter(s, _ptr(idx1), _ptr(np.ascontiguousarray(d1)), 2, 1))
        idx2 = np.array([45], np.int64)
        v2 = np.ascontiguousarray(np.append(ref_f.reshape(w, n)[:, 45], 1e-9)[None, :])
        bs = [float(q) for q in v2[0]]
        if dim == 3:
            sim.apply_body_state(st, 45, bs[0], bs[1], bs[3], bs[4], bs[6], z=bs[2], vz=bs[5])
        else:
            sim.apply_body_state(st, 45, *bs)
        ctx.check(lib.sss_nbody_scatter(s, _ptr(idx2), _ptr(v2), 1, 2))
        sim.set_radius(st, 1, 0.01)
        ctx.check(lib.sss_nbody_set_radius(s, 1, 0.01))
        sim.deactivate_body(st, 50)
        ctx.check(lib.sss_nbody_deactivate(s, 50))
        sim.deactivate_body(st, 4)
        ctx.check(lib.sss_nbody_deactivate(s, 4))
        out = sim.step_batch(st, dt, k)
        snap, hits, subs = _session_batch(ctx, lib, s, dim, n, k, dt)
        _assert_batch_equal(out, st, snap, hits, subs)
        ctx.check(lib.sss_nbody_export_f64(s, _ptr(f)))
        assert np.array_equal(f, sim.export_f64(st))
    finally:
        lib.sss_nbody_destroy(s)


def test_nbody_session_errors():
    L = _lib()
    ctx = L.context(0)
    lib = ctx.lib
    s = ctypes.c_void_p()
    bad = L.NBodyCfg(4 * np.pi ** 2, 1e-6, 0.5 / 365.25, 100000, 8000, 33, 0)
    assert lib.sss_nbody_create(ctx.ptr, ctypes.byref(bad), ctypes.byref(s)) == L.SSS_ERR_ARG
    assert b"m_sub ausserhalb" in lib.sss_last_error(ctx.ptr)
    ctx.check(lib.sss_nbody_create(ctx.ptr, None, ctypes.byref(s)))
    try:
        assert lib.sss_nbody_step_batch(s, 1e-3, 1, None) == L.SSS_ERR_ARG
        assert b"kein Zustand geladen" in lib.sss_last_error(ctx.ptr)
        n = 70                                      # 65 massive bodies: one too many
        soa = np.zeros(4 * n)
        soa[:n] = np.arange(n)
        mass = np.full(n, 1e-6)
        vis = np.ones(n, np.uint8)
        is_ast = np.zeros(n, np.uint8)
        is_ast[65:] = 1
        rc = lib.sss_nbody_load(s, 2, n, _ptr(soa), _ptr(mass), _ptr(vis), _ptr(is_ast), None)
        assert rc == L.SSS_ERR_TOO_MANY_MASSIVE
        assert b"zu viele massive Koerper" in lib.sss_last_error(ctx.ptr)
        is_ast[60:] = 1
        ctx.check(lib.sss_nbody_load(s, 2, n, _ptr(soa), _ptr(mass), _ptr(vis), _ptr(is_ast), None))
        assert lib.sss_nbody_step_batch(s, 1e-3, 17, None) == L.SSS_ERR_ARG
        assert b"k ausserhalb" in lib.sss_last_error(ctx.ptr)
        idx = np.array([62, 62], np.int64)
        assert lib.sss_nbody_scatter(s, _ptr(idx), _ptr(np.zeros(8)), 2, 1) == L.SSS_ERR_ARG
        assert b"idx must be unique" in lib.sss_last_error(ctx.ptr)
        assert lib.sss_nbody_set_radius(s, n, 1.0) == L.SSS_ERR_ARG
    finally:
        lib.sss_nbody_destroy(s)
