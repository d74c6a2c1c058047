"""GPU parity of the 3-D periodic PM, the f64 Ewald judge and the learned
correction (sss_pm3_*, sss_ewald_*, sss_mlp_*) against oracle/pm3d.py.

Tolerances: the mesh is f32 (deposit by f32 atomics, cuFFT f32), so mesh
values and mesh forces agree with the f64 oracle to ~1e-6 of their scale
(bar 2e-5); the Ewald sum is f64 on both sides (bar 1e-10 of the force
scale); the MLP runs bf16 operands with f32 sums, compared against an f64
restatement that rounds at the same points (bars per check below).
"""
import numpy as np
import pytest
import torch

from oracle import pm3d as o

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mods():
    from solarsystemsimulator_b200 import _lib, pm3d, mlp, ewald
    return _lib, pm3d, mlp, ewald


def _cloud(n, seed, clump=False):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0, 1, (n, 3))
    if clump:
        # a third of the particles inside one mesh cell region: warp groups collide
        k = n // 3
        pos[:k] = 0.5 + rng.uniform(0, 0.01, (k, 3))
    vel = rng.normal(0, 0.05, (n, 3))
    m = rng.uniform(0.5, 1.5, n) / n
    return pos, vel, m


@pytest.mark.parametrize("clump", [False, True])
def test_deposit_matches_oracle(mods, clump):
    _lib, pm3d, _, _ = mods
    pos, vel, m = _cloud(20000, 1, clump)
    pm = pm3d.PMPeriodic3D(32, 1.0, 1.0)
    st = pm.load_state(pos, vel, m)
    pm.mesh_forces(st)
    rho = pm.rho.double().cpu().numpy()
    ref = o.cic_deposit(pos, m, 32)
    assert np.abs(rho - ref).max() <= 2e-6 * ref.max()
    assert abs(rho.sum() - ref.sum()) <= 1e-5 * ref.sum()


def test_deposit_in_a_plane_is_the_reference_2d_deposit(mods, load_golden):
    """k_deposit3 with every body on the plane z = 0 against the reference's
    own 2-D deposit (pm_kernel._cic_deposit, fixture pm2d_n2000_g128.npz):
    the plane times h^3 is its mass grid to f32 rounding, the other planes
    stay empty."""
    _lib, pm3d, _, _ = mods
    g = load_golden("pm2d_n2000_g128.npz")
    n, h = int(g["grid_n"]), float(g["h"])
    pos = np.stack([g["x"] - float(g["x0"]), g["y"] - float(g["y0"]), np.zeros(len(g["x"]))], 1)
    pm = pm3d.PMPeriodic3D(n, n * h, 1.0)
    st = pm.load_state(pos, np.zeros_like(pos), g["m"])
    pm.mesh_forces(st)
    rho = pm.rho.double().cpu().numpy().reshape(n, n, n)
    assert np.abs(rho[:, :, 1:]).max() == 0.0
    assert np.abs(rho[:, :, 0] * h ** 3 - g["rho"]).max() <= 2e-6 * np.abs(g["rho"]).max()


def test_gather_of_a_z_constant_field_is_the_reference_2d_gather(mods, load_golden):
    """k_gather3 on acceleration meshes whose planes all hold the reference's
    2-D force field (pm_force_field of the reference's case, fixture
    pm2d_n2000_g128.npz, reproduced bit for bit by the 2-D oracle) gives the
    reference's own gathered accelerations (pm_kernel._cic_gather,
    pm_kernel.py:93-107) to the f32 rounding of the mesh values; the z
    component stays zero."""
    _lib, pm3d, _, _ = mods
    from oracle import pm as opm2
    g = load_golden("pm2d_n2000_g128.npz")
    n, h = int(g["grid_n"]), float(g["h"])
    x0, y0 = float(g["x0"]), float(g["y0"])
    fx, fy = opm2.pm_force_field(g["x"], g["y"], g["m"], n, x0, y0, h, float(g["eps2"]))
    pm = pm3d.PMPeriodic3D(n, n * h, 1.0)
    pos = np.stack([g["x"] - x0, g["y"] - y0, np.full(len(g["x"]), 17.37 * h)], 1)
    st = pm.load_state(pos, np.zeros_like(pos), g["m"])
    mesh = torch.zeros((3, n, n, n), dtype=torch.float32)
    mesh[0] = torch.from_numpy(fx.astype(np.float32))[:, :, None]
    mesh[1] = torch.from_numpy(fy.astype(np.float32))[:, :, None]
    pm.acc_mesh.copy_(mesh.to(pm.acc_mesh.device))
    pm.gather(st)
    a = st["buf"][6:9].cpu().numpy().T
    scale = max(np.abs(g["ax"]).max(), np.abs(g["ay"]).max())
    assert np.abs(a[:, 0] - g["ax"]).max() <= 1e-6 * scale
    assert np.abs(a[:, 1] - g["ay"]).max() <= 1e-6 * scale
    assert np.abs(a[:, 2]).max() == 0.0


@pytest.mark.parametrize("mesh,deconv,rs", [(32, 2, 0.6), (64, 2, 0.6), (32, 0, 0.0), (48, 1, 1.0)])
def test_forces_match_oracle(mods, mesh, deconv, rs):
    _lib, pm3d, _, _ = mods
    pos, vel, m = _cloud(20000, 2)
    pm = pm3d.PMPeriodic3D(mesh, 1.0, 1.0, deconv=deconv, r_split_cells=rs)
    st = pm.load_state(pos, vel, m)
    a = pm.forces(st).cpu().numpy().T
    ref = o.pm_accel(pos, m, mesh, deconv=deconv, r_split=rs / mesh)
    scale = np.abs(ref).max()
    assert np.abs(a - ref).max() <= 2e-5 * scale
    # momentum: the mesh force sums to zero
    assert np.abs((m[:, None] * a).sum(0)).max() <= 1e-5 * (m[:, None] * np.abs(a)).sum()


def test_kdk_steps_match_oracle(mods):
    _lib, pm3d, _, _ = mods
    pos, vel, m = _cloud(8000, 3)
    pm = pm3d.PMPeriodic3D(32, 1.0, 1.0)
    st = pm.load_state(pos, vel, m)
    snaps = pm.step_batch(st, 0.01, 6, snapshots=True)
    x, v = pm.export_f64(st)
    a0 = o.pm_accel(pos, m, 32)
    xr, vr, _ = o.kdk(pos, vel, a0, m, 0.01, 6, 32)
    dx = x - xr
    dx -= np.rint(dx)
    assert np.abs(dx).max() <= 1e-8
    assert np.abs(v - vr).max() <= 1e-6 * np.abs(vr).max()
    last = snaps[-1].reshape(6, -1)
    assert np.allclose(last[0:3].T, x, atol=1e-6) and np.allclose(last[3:6].T, v, rtol=1e-6, atol=1e-9)
    assert np.all((x >= 0) & (x < 1))


def test_ewald_matches_oracle(mods):
    _lib, pm3d, _, ewald = mods
    pos, vel, m = _cloud(3000, 4)
    pm = pm3d.PMPeriodic3D(16, 1.0, 1.0)
    st = pm.load_state(pos, vel, m)
    ew = ewald.EwaldDirect(1.0, 1.0, softening=1e-3)
    idx = torch.arange(0, 3000, 47, device="cuda")
    a = ew.accel(st["parts"], st["buf"][0:3, idx].contiguous(), idx).cpu().numpy().T
    sel = idx.cpu().numpy()
    ref = o.ewald_accel(pos, m, pos[sel], alpha=ew.alpha, r_cut=ew.r_cut, h_max=ew.h_max, eps=1e-3,
                        self_index=sel)
    assert np.abs(a - ref).max() <= 1e-10 * np.abs(ref).max()


def test_ewald_independent_of_alpha_on_gpu(mods):
    _lib, pm3d, _, ewald = mods
    pos, vel, m = _cloud(40000, 5)
    pm = pm3d.PMPeriodic3D(16, 1.0, 1.0)
    st = pm.load_state(pos, vel, m)
    idx = torch.arange(0, 40000, 131, device="cuda")
    t = st["buf"][0:3, idx].contiguous()
    a1 = ewald.EwaldDirect(1.0, 1.0, 1e-3, alpha=10.0).accel(st["parts"], t, idx)
    a2 = ewald.EwaldDirect(1.0, 1.0, 1e-3, alpha=13.0).accel(st["parts"], t, idx)
    assert float((a1 - a2).abs().max()) <= 1e-9 * float(a1.abs().max())


def test_features_match_oracle(mods):
    _lib, pm3d, mlp, _ = mods
    pos, vel, m = _cloud(20000, 6, clump=True)
    pm = pm3d.PMPeriodic3D(32, 1.0, 1.0)
    st = pm.load_state(pos, vel, m)
    pm.mesh_forces(st)
    net = mlp.ShortRangeMLP(0, seed=1)
    idx = torch.arange(0, 20000, 7, device="cuda")
    X = net.features(pm, st["parts"], idx, st["rho_mean"])
    xb = X.cpu().numpy().view(np.uint16).astype(np.uint32) << 16
    xg = xb.view(np.float32).astype(np.float64)
    rho = pm.rho.double().cpu().numpy()
    ref = o.bf16(o.features(pos[idx.cpu().numpy()], rho, st["rho_mean"]))
    diff = np.abs(xg - ref)
    # log1pf vs log1p may round to the neighbouring bf16 value, nothing more
    assert np.all(diff <= 2.0 ** -7 * np.maximum(np.abs(ref), 2.0 ** -126))
    assert np.mean(diff > 0) < 2e-3


def _x_to_f64(X):
    return (X.cpu().numpy().view(np.uint16).astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def _rand_inputs(rows, seed):
    rng = np.random.default_rng(seed)
    X = np.zeros((rows, o.K1))
    X[:, :64] = np.log1p(rng.exponential(1.0, (rows, 64)))
    X[:, 64:67] = rng.uniform(-0.5, 0.5, (rows, 3))
    Xb = o.bf16(X).astype(np.float32).view(np.uint32) >> 16
    return torch.as_tensor(Xb.astype(np.uint16).view(np.int16)).cuda(), X


def test_forward_matches_oracle(mods):
    _lib, pm3d, mlp, _ = mods
    net = mlp.ShortRangeMLP(0, seed=2)
    X, _ = _rand_inputs(1000, 7)
    Y = net.forward(X).double().cpu().numpy()
    ref, _ = o.forward(net.params.double().cpu().numpy(), _x_to_f64(X))
    err = np.abs(Y - ref)
    scale = np.sqrt(np.mean(ref ** 2))
    assert np.median(err) <= 1e-4 * scale
    assert err.max() <= 2e-2 * scale


def test_gradients_match_oracle(mods):
    _lib, pm3d, mlp, _ = mods
    net = mlp.ShortRangeMLP(0, seed=3)
    X, _ = _rand_inputs(1000, 8)
    T = torch.randn((1000, 3), generator=torch.Generator().manual_seed(9)).float().cuda()
    g, loss = net.grad(X, T)
    g = g.double().cpu().numpy()
    p = net.params.double().cpu().numpy()
    Y, cache = o.forward(p, _x_to_f64(X))
    Tn = T.double().cpu().numpy()
    ref = o.backward(p, cache, Tn)
    assert abs(float(loss) - o.loss(Y, Tn)) <= 1e-3 * o.loss(Y, Tn)
    gd, rd = o.unpack(g), o.unpack(ref)
    for k in rd:
        assert np.linalg.norm(gd[k] - rd[k]) <= 1e-2 * np.linalg.norm(rd[k]), k
    assert np.all(gd["W1"][o.N_IN:] == 0.0) and np.all(gd["W3"][:, 3:] == 0.0)
    # a row subset through idx equals the compacted rows
    idx = torch.arange(3, 1000, 3, dtype=torch.int32, device="cuda")
    g1 = net.grad(X, T, idx)[0].clone()
    g2 = net.grad(X[idx.long()].contiguous(), T[idx.long()].contiguous())[0].clone()
    assert torch.equal(g1, g2)


def test_adam_matches_oracle(mods):
    _lib, pm3d, mlp, _ = mods
    net = mlp.ShortRangeMLP(0, seed=4)
    p0 = net.params.double().cpu().numpy()
    rng = np.random.default_rng(10)
    gs = [rng.normal(0, 1e-2, p0.size) for _ in range(3)]
    m = np.zeros_like(p0)
    v = np.zeros_like(p0)
    p = p0.copy()
    for t, gr in enumerate(gs, 1):
        net.adam_step(torch.as_tensor(gr, dtype=torch.float32).cuda(), 1e-3)
        p, m, v = o.adam(p, gr.astype(np.float32).astype(np.float64), m, v, t, 1e-3)
    assert np.abs(net.params.double().cpu().numpy() - p).max() <= 1e-6


@pytest.mark.parametrize("n", [10000, 128 * 37])
def test_correction_pass_adds_the_network_output(mods, n):
    # the correction pass (tcgen05, one particle per TMEM lane) against the
    # mma.sync forward on the same inputs: both round at the same points
    # (bf16 inputs, weights, hidden activations; f32 sums) but sum in a
    # different order, so a hidden value may round to its bf16 neighbour
    _lib, pm3d, mlp, _ = mods
    pos, vel, m = _cloud(n, 11)
    pm = pm3d.PMPeriodic3D(32, 1.0, 1.0)
    st = pm.load_state(pos, vel, m)
    net = mlp.ShortRangeMLP(0, seed=5)
    net.out_scale = 0.25
    a_pm = pm.forces(st).clone()
    a = pm.forces(st, net).clone()
    X = net.features(pm, st["parts"], torch.arange(n, device="cuda"), st["rho_mean"])
    y = net.forward(X).double().T * 0.25
    err = (a - a_pm - y).abs()
    rms = float(torch.sqrt(torch.mean(y * y)))
    assert float(err.median()) <= 1e-4 * rms
    assert float(err.max()) <= 2e-2 * rms
    ref, _ = o.forward(net.params.double().cpu().numpy(), _x_to_f64(X))
    e2 = np.abs((a - a_pm).cpu().numpy().T / 0.25 - ref)
    assert np.median(e2) <= 1e-4 * rms / 0.25 and e2.max() <= 2e-2 * rms / 0.25


def test_training_reduces_the_loss(mods):
    _lib, pm3d, mlp, _ = mods
    net = mlp.ShortRangeMLP(0, seed=6)
    X, Xf = _rand_inputs(8192, 12)
    # a smooth target of the inputs
    T = np.stack([np.tanh(Xf[:, 64] * 3) * Xf[:, :8].mean(1), Xf[:, 65] ** 2, Xf[:, 10] - Xf[:, 50]], 1)
    Tt = torch.as_tensor(T, dtype=torch.float32).cuda()
    losses = net.train(X, Tt, 300, 1024, 3e-3, np.random.default_rng(0))
    assert np.mean(losses[-20:]) < 0.2 * np.mean(losses[:5])


def test_learned_run_gains_and_judge_reverts(mods):
    _lib, pm3d, mlp, _ = mods
    from solarsystemsimulator_b200.workloads import periodic_structure
    w = periodic_structure(n_side=32, mesh_n=64, seed=21, fcc=False)
    sim = pm3d.NBodyPMLearned(0, mesh_n=64, softening=w["softening"], check_every=10, samples=4096,
                              iters=400, batch=1024, lr=2e-3, seed=1)
    st = sim.load_state(w["pos"], w["vel"], w["mass"])
    recs = sim.run(st, 2e-3, 30)
    assert len(recs) == 4
    judged = [r for r in recs if r.err_corr is not None]
    # the trained network lowers the median force error on fresh particles
    assert all(r.err_corr < r.err_mesh for r in judged[1:]), [(r.err_mesh, r.err_corr) for r in judged]
    assert all(r.accepted for r in judged[1:])
    # planted mistake: a network whose output is scaled up 50x must be
    # rejected, and the block replayed with the last accepted network
    good = sim.accepted
    assert good is not None
    sim.net.out_scale *= 50.0
    buf0 = st["buf"].clone()
    sim._steps(st, 2e-3, 5)
    rec = sim.check(st, 2e-3, block_start=(buf0, 5))
    assert rec.reverted and rec.accepted is False
    x_after = st["buf"][0:3].clone()
    net2 = mlp.ShortRangeMLP(0)
    net2.restore(good)
    st["buf"].copy_(buf0)
    sim.pm.forces(st, net2)
    sim.pm.step_batch(st, 2e-3, 5, net2)
    # the deposit adds f32 weights by atomics in no fixed order, so two replays
    # agree to rounding (~1e-12 here); the mesh-only force or the rejected
    # network would move the particles by 5e-7 .. 1e-5 over these 5 steps
    d = (x_after - st["buf"][0:3]).abs()
    assert float(torch.minimum(d, 1.0 - d).max()) <= 1e-9


def test_learned_gain_over_the_p3m_method(mods):
    """The method the configured row uses, scaled down: mesh filtered at
    r_split = 2.25 cells + the P3M pair term cut at 3 / alpha, 32^3
    particles on 64^3, 60 steps, a check every 10. The network, trained on
    the residual direct - method, lowers the median force error on fresh
    particles below the method's at most checks, and the training loss
    stays of order one at every check (targets renormalised per check)."""
    _lib, pm3d, _, _ = mods
    from solarsystemsimulator_b200.workloads import periodic_structure
    w = periodic_structure(n_side=32, mesh_n=64, seed=21, fcc=False)
    sim = pm3d.NBodyPMLearned(0, mesh_n=64, softening=w["softening"], check_every=10, samples=4096, iters=200,
                              batch=2048, lr=2e-3, seed=1, short_range=True, r_split_cells=2.25, x_cut=3.0,
                              window=4)
    st = sim.load_state(w["pos"], w["vel"], w["mass"])
    recs = sim.run(st, 2e-3, 60)
    judged = [r for r in recs if r.err_corr is not None]
    assert len(judged) == 6
    gains = [r.err_corr < r.err_mesh for r in judged]
    assert sum(gains) >= 4, [(r.err_mesh, r.err_corr) for r in judged]
    assert all(r.loss_last < 1.5 for r in recs), [r.loss_last for r in recs]


def test_output_rescale_keeps_the_force(mods):
    """rescale_output(f) with out_scale / f is the same force, to the bf16
    rounding of the rescaled output layer."""
    _lib, pm3d, mlp, _ = mods
    rng = np.random.default_rng(3)
    net = mlp.ShortRangeMLP(0, seed=4)
    X = torch.as_tensor((rng.normal(0, 1, (512, mlp.K1)).astype(np.float32)).view(np.int32) >> 16).to(
        torch.int16).cuda()
    net.out_scale = 2.0
    y0 = net.forward(X).double() * net.out_scale
    net.rescale_output(0.37)
    net.out_scale = 2.0 / 0.37
    y1 = net.forward(X).double() * net.out_scale
    assert float((y1 - y0).abs().max()) <= 1e-2 * float(y0.abs().max())


def test_learned_run_on_the_p3m_force(mods):
    """The learned model over the mesh + P3M pair term (32^3 particles on
    64^3, r_split 1 cell, r_cut 3 / alpha): the judge accepts exactly the
    checks where the corrected force is no worse than the method's, and on
    the evolved state the method's force is far better than the mesh's."""
    _lib, pm3d, _, _ = mods
    from solarsystemsimulator_b200.workloads import periodic_structure
    w = periodic_structure(n_side=32, mesh_n=64, seed=21, fcc=False)
    sim = pm3d.NBodyPMLearned(0, mesh_n=64, softening=w["softening"], check_every=10, samples=4096, iters=200,
                              batch=1024, lr=2e-3, seed=1, short_range=True, r_split_cells=1.0, x_cut=3.0)
    st = sim.load_state(w["pos"], w["vel"], w["mass"])
    recs = sim.run(st, 2e-3, 30)
    assert len(recs) == 4
    judged = [r for r in recs if r.err_corr is not None]
    assert judged and all((r.err_corr <= r.err_mesh) == bool(r.accepted) for r in judged)
    assert all(r.reverted == (not r.accepted) for r in judged)
    plain = pm3d.PMPeriodic3D(64, 1.0, 1.0, 0, 2, 0.6)
    pos, vel = sim.pm.export_f64(st)
    stp = plain.load_state(pos, vel, w["mass"])
    idx = torch.arange(0, st["n"], 7, device=st["buf"].device)
    ref = sim.ewald.accel(stp["parts"], stp["buf"][0:3, idx].contiguous(), idx)
    plain.forces(stp)
    e_mesh = pm3d.median_rel_err(stp["buf"][6:9, idx], ref)
    sim.pm.method_forces(st)
    e_p3m = pm3d.median_rel_err(st["buf"][6:9, idx], ref)
    assert e_p3m < 0.2 * e_mesh, (e_p3m, e_mesh)
