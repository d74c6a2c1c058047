"""CPU checks of the 3-D periodic PM / Ewald / MLP oracle (oracle/pm3d.py).

The reference has no 3-D or periodic solver (its mesh plan is TODO.md:
225-253, its code 2-D isolated, backend/pm_kernel.py), so the restatement
is pinned by properties the exact answers have: the Ewald sum does not
depend on the splitting parameter alpha, a symmetric lattice feels no
force, the mesh force conserves momentum and agrees with the direct sum on
a smooth density, and the MLP gradient matches finite differences.
"""
import math

import numpy as np
import pytest
import torch

from oracle import pm3d as o


def test_ewald_independent_of_alpha():
    rng = np.random.default_rng(1)
    n = 512
    src = rng.uniform(0, 1, (n, 3))
    m = rng.uniform(0.5, 1.5, n) / n
    si = np.arange(6)
    a1 = o.ewald_accel(src, m, src[:6], alpha=10, r_cut=0.46, h_max=17, self_index=si)
    a2 = o.ewald_accel(src, m, src[:6], alpha=6, r_cut=0.78, h_max=11, images=1, self_index=si)
    a3 = o.ewald_accel(src, m, src[:6], alpha=14, r_cut=0.33, h_max=24, self_index=si)
    scale = np.abs(a1).max()
    assert np.abs(a1 - a2).max() <= 1e-9 * scale
    assert np.abs(a1 - a3).max() <= 1e-9 * scale


def test_ewald_lattice_feels_no_force():
    g = (np.arange(4) + 0.5) / 4
    q = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    m = np.full(len(q), 1.0 / len(q))
    a = o.ewald_accel(q, m, q[:5], self_index=np.arange(5))
    # scale: one neighbour at the lattice spacing
    assert np.abs(a).max() <= 1e-10 * (m[0] / 0.25 ** 2)


def test_ewald_softening_is_the_plummer_correction_of_every_pair():
    src = np.array([[0.5, 0.5, 0.5], [0.5005, 0.5, 0.5], [0.1, 0.2, 0.3], [0.95, 0.45, 0.52]])
    m = np.array([1e-3, 2e-3, 3e-3, 4e-3])
    a0 = o.ewald_accel(src, m, src[:1], self_index=np.array([0]))
    eps = 1e-3
    a1 = o.ewald_accel(src, m, src[:1], eps=eps, self_index=np.array([0]))
    d = src[0] - src[1:]
    d -= np.rint(d)
    r2 = (d * d).sum(1)
    expect = -((m[1:] * ((r2 + eps * eps) ** -1.5 - r2 ** -1.5))[:, None] * d).sum(0)
    assert np.allclose(a1 - a0, expect[None], rtol=1e-9, atol=0)
    # independent of alpha with softening too
    a2 = o.ewald_accel(src, m, src[:1], eps=eps, alpha=14, r_cut=0.33, h_max=24, self_index=np.array([0]))
    assert np.abs(a2 - a1).max() <= 1e-9 * np.abs(a1).max()


def test_pm_conserves_momentum():
    rng = np.random.default_rng(2)
    pos = rng.uniform(0, 1, (3000, 3))
    m = rng.uniform(0.5, 1.5, 3000) / 3000
    a = o.pm_accel(pos, m, 16)
    p = (m[:, None] * a).sum(0)
    assert np.abs(p).max() <= 1e-12 * (m[:, None] * np.abs(a)).sum()


def test_pm_matches_ewald_on_a_displaced_lattice():
    # 16^3 lattice displaced by long longitudinal modes, mesh 32^3 (two cells
    # per particle spacing, as the 1M-particle workload on 256^3): the
    # deconvolved, Gaussian-filtered mesh force is within a few per cent of
    # the direct sum, the unfiltered W^-2 one is not
    g = (np.arange(16) + 0.5) / 16
    q = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    pos = o.wrap(q + 0.01 * np.sin(2 * np.pi * q) + 0.004 * np.sin(6 * np.pi * q[:, [1, 2, 0]]))
    m = np.full(len(pos), 1.0 / len(pos))
    sel = np.arange(0, len(pos), 97)
    a_ew = o.ewald_accel(pos, m, pos[sel], alpha=6, r_cut=0.78, h_max=11, images=1, self_index=sel)
    err = o.median_rel_err(o.pm_accel(pos, m, 32)[sel], a_ew)
    raw = o.median_rel_err(o.pm_accel(pos, m, 32, r_split=0.0)[sel], a_ew)
    assert err < 0.1 and raw > 2 * err, (err, raw)


def test_pm_single_mode_matches_the_analytic_field():
    # density 1 + A cos(2 pi x) on the mesh: a_x = -(2 G A) sin(2 pi x) (G = 1, rho_mean = 1)
    n = 32
    x = np.arange(n) / n
    rho = np.broadcast_to((1.0 + 0.3 * np.cos(2 * np.pi * x))[:, None, None], (n, n, n)).copy()
    acc = o.force_meshes(rho, deconv=0)
    expect = -2.0 * 0.3 * np.sin(2 * np.pi * x)
    assert np.allclose(acc[0][:, 3, 5], expect, atol=1e-12)
    assert np.abs(acc[1]).max() < 1e-12 and np.abs(acc[2]).max() < 1e-12


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.normal(0, 1, 5000), rng.normal(0, 1e-3, 5000), [0.0, -0.0, 1.0, 3.0e38]])
    ref = torch.tensor(x, dtype=torch.float32).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(o.bf16(x), ref)


def test_mlp_gradient_matches_finite_differences():
    rng = np.random.default_rng(4)
    p = o.init_params(5)
    X = np.zeros((12, o.K1))
    X[:, :o.N_IN] = rng.normal(0, 1, (12, o.N_IN))
    T = rng.normal(0, 1, (12, 3))
    Y, cache = o.forward(p, X, emulate=False)
    g = o.backward(p, cache, T, emulate=False)
    sel = np.concatenate([rng.choice(np.arange(0, 67 * 128), 8), [o.K1 * o.HID + 3],
                          o.K1 * o.HID + o.HID + rng.choice(o.HID * o.HID, 8),
                          [o.N_PARAMS - o.K3 - o.HID * o.K3 + 5 * o.K3 + 1, o.N_PARAMS - o.K3 + 2]])
    for i in sel:
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (o.loss(o.forward(pp, X, False)[0], T) - o.loss(o.forward(pm, X, False)[0], T)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1e-3, abs(g[i])), (i, fd, g[i])
    # padded rows / columns get no gradient
    d = o.unpack(g)
    assert np.all(d["W1"][o.N_IN:] == 0.0) and np.all(d["W3"][:, 3:] == 0.0) and np.all(d["b3"][3:] == 0.0)


def test_emulated_gradient_close_to_exact():
    rng = np.random.default_rng(5)
    p = o.init_params(6)
    X = np.zeros((256, o.K1))
    X[:, :o.N_IN] = rng.normal(0, 1, (256, o.N_IN))
    T = rng.normal(0, 1, (256, 3))
    g0 = o.backward(p, o.forward(p, X, False)[1], T, False)
    g1 = o.backward(p, o.forward(p, X, True)[1], T, True)
    assert np.linalg.norm(g1 - g0) <= 0.05 * np.linalg.norm(g0)


def test_features_layout():
    n = 8
    rho = np.arange(n ** 3, dtype=np.float64).reshape(n, n, n)
    pos = np.array([[0.3 / n, 7.6 / n, 2.25 / n]])
    X = o.features(pos, rho, rho_mean=1.0)
    # cell (0, 7, 2), patch cells (i-1 .. i+2) wrapped
    c = 0
    for a in range(4):
        for b in range(4):
            for e in range(4):
                ix, iy, iz = (0 + a - 1) % n, (7 + b - 1) % n, (2 + e - 1) % n
                assert X[0, c] == np.log1p(rho[ix, iy, iz])
                c += 1
    assert np.allclose(X[0, 64:67], [0.3 - 0.5, 0.6 - 0.5, 0.25 - 0.5])
    assert np.all(X[0, 67:] == 0.0)


def test_judge_rule():
    from solarsystemsimulator_b200.pm3d import CorrectionJudge
    j = CorrectionJudge()
    assert j.accept(0.02, 0.015) and not j.accept(0.02, 0.021)
    j = CorrectionJudge(tol=1e-3)
    assert j.accept(0.5, 9e-4) and not j.accept(0.5, 2e-3)


def test_adam_restatement():
    p = np.array([1.0, -2.0])
    g = np.array([0.5, -0.25])
    m = np.zeros(2)
    v = np.zeros(2)
    p1, m1, v1 = o.adam(p, g, m, v, 1, 0.1)
    # first step of Adam moves every parameter by lr against its gradient's sign
    assert np.allclose(p1, p - 0.1 * np.sign(g), rtol=0, atol=1e-6)


def test_p3m_pair_term_two_bodies():
    """Two bodies 0.01 apart, across the periodic boundary: the pair term is
    G m (erfc(x) + 2x e^{-x^2}/sqrt(pi) + (1 + eps^2/r^2)^{-3/2} - 1) / r^2
    towards the other body; nothing beyond r_cut."""
    from oracle import pm3d as opm
    alpha, eps = 32.0, 2e-3
    pos = np.array([[0.995, 0.3, 0.7], [0.005, 0.3, 0.7]])
    a = opm.p3m_short(pos, np.array([2.0, 3.0]), pos, alpha, 0.1, eps=eps, self_index=np.array([0, 1]))
    r, x = 0.01, alpha * 0.01
    g = math.erfc(x) + 2.0 / math.sqrt(math.pi) * x * math.exp(-x * x) + (1.0 + eps * eps / (r * r)) ** -1.5 - 1.0
    assert a[0, 0] == pytest.approx(3.0 * g / r ** 2, rel=1e-12)
    assert a[1, 0] == pytest.approx(-2.0 * g / r ** 2, rel=1e-12)
    assert np.abs(a[:, 1:]).max() == 0.0
    far = opm.p3m_short(pos, np.array([2.0, 3.0]), pos, alpha, 0.009, eps=eps, self_index=np.array([0, 1]))
    assert np.abs(far).max() == 0.0


def test_p3m_pair_term_is_the_ewald_real_space_part():
    """With softening and r_cut inside the nearest image, the pair term is
    the real-space part of the Ewald sum (no k vectors) wherever the
    softening correction beyond r_cut is negligible."""
    from oracle import pm3d as opm
    rng = np.random.default_rng(4)
    src = rng.uniform(0, 1, (300, 3))
    m = rng.uniform(0.5, 1.5, 300)
    tgt = src[:5]
    alpha, r_cut, eps = 8.0, 0.33, 1e-6
    real = opm.ewald_accel(src, m, tgt, alpha=alpha, r_cut=r_cut, h_max=0, eps=eps, self_index=np.arange(5))
    pair = opm.p3m_short(src, m, tgt, alpha, r_cut, eps=eps, self_index=np.arange(5))
    assert np.allclose(pair, real, rtol=1e-9, atol=1e-9 * np.abs(real).max())


def test_deposit_in_a_plane_is_the_reference_2d_deposit(load_golden):
    """With z on a mesh plane the 3-D CIC stencil reduces to the 2-D one: the
    oracle's deposit of the reference's own 2-D case (pm_kernel._cic_deposit,
    pm_kernel.py:63-90, fixture pm2d_n2000_g128.npz) in plane z = 0 of a
    periodic box of the same cells, times h^3, is the reference's mass grid.
    The bodies sit inside the grid's margin, so its clipping never acts and
    the periodic wrap never reaches them."""
    g = load_golden("pm2d_n2000_g128.npz")
    n, h = int(g["grid_n"]), float(g["h"])
    pos = np.stack([g["x"] - float(g["x0"]), g["y"] - float(g["y0"]), np.zeros(len(g["x"]))], 1)
    rho3 = o.cic_deposit(pos, g["m"], n, L=n * h)
    plane = rho3[:, :, 0] * h ** 3
    assert np.abs(rho3[:, :, 1:]).max() == 0.0
    assert np.abs(plane - g["rho"]).max() <= 1e-12 * np.abs(g["rho"]).max()


def test_gather_of_a_z_constant_field_is_the_reference_2d_gather(load_golden):
    """A mesh whose planes are all equal reduces the 3-D trilinear stencil to
    the 2-D bilinear one: the oracle's 3-D gather of the reference's 2-D force
    field (pm_force_field of the reference's case, fixture pm2d_n2000_g128.npz,
    which the 2-D oracle reproduces bit for bit) stacked along z, at the
    bodies' positions in the same cells, is the reference's own gathered
    acceleration (pm_kernel._cic_gather, pm_kernel.py:93-107), up to the order
    of the eight weighted terms. The bodies sit inside the grid's margin, so
    neither the 2-D clipping nor the periodic wrap acts."""
    from oracle import pm as opm2
    g = load_golden("pm2d_n2000_g128.npz")
    n, h = int(g["grid_n"]), float(g["h"])
    x0, y0 = float(g["x0"]), float(g["y0"])
    fx, fy = opm2.pm_force_field(g["x"], g["y"], g["m"], n, x0, y0, h, float(g["eps2"]))
    meshes = np.zeros((3, n, n, n))
    meshes[0] = fx[:, :, None]
    meshes[1] = fy[:, :, None]
    for z in (0.0, 0.37 * h, 0.999 * h):            # on a plane and between two equal planes
        pos = np.stack([g["x"] - x0, g["y"] - y0, np.full(len(g["x"]), 17 * h + z)], 1)
        a = o.cic_gather(meshes, pos, L=n * h)
        scale = max(np.abs(g["ax"]).max(), np.abs(g["ay"]).max())
        assert np.abs(a[:, 0] - g["ax"]).max() <= 1e-12 * scale
        assert np.abs(a[:, 1] - g["ay"]).max() <= 1e-12 * scale
        assert np.abs(a[:, 2]).max() == 0.0
