"""P3M pair term (sss_pm3_short): parity with the oracle's restatement,
the two-body closed form, and the accuracy it adds to the mesh force
against the f64 Ewald direct sum."""
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _clustered(n, seed):
    rng = np.random.default_rng(seed)
    cen = rng.uniform(0, 1, (6, 3))
    lab = rng.integers(0, 6, n)
    pos = cen[lab] + rng.normal(0, 1, (n, 3)) * rng.uniform(0.01, 0.08, 6)[lab, None]
    pos = np.concatenate([pos[: n // 2], rng.uniform(0, 1, (n - n // 2, 3))])
    return np.mod(pos, 1.0), rng.uniform(0.5, 1.5, n) / n


def _pair_only(pm, st):
    st["buf"][6:9] = 0.0
    pm.short(st)
    torch.cuda.synchronize()
    return st["buf"][6:9].cpu().numpy().T


@pytest.mark.parametrize("mesh_n,rs,eps", [(64, 1.0, 0.0), (64, 1.25, 2e-3), (128, 0.6, 1e-3)])
def test_pair_term_matches_oracle(mesh_n, rs, eps):
    from oracle import pm3d as opm
    from solarsystemsimulator_b200 import pm3d
    pos, mass = _clustered(20_000, mesh_n)
    pm = pm3d.PMPeriodic3D(mesh_n, 1.0, 1.0, 0, 2, rs, short_range=True, softening=eps)
    st = pm.load_state(pos, np.zeros_like(pos), mass)
    a = _pair_only(pm, st)
    sel = np.random.default_rng(1).choice(len(pos), 400, replace=False)
    ref = opm.p3m_short(pos, mass, pos[sel], pm.alpha, pm.r_cut, eps=eps, self_index=sel)
    err = np.linalg.norm(a[sel] - ref, axis=1) / np.maximum(np.linalg.norm(ref, axis=1), 1e-30)
    assert np.median(err) < 1e-5, np.median(err)
    assert np.quantile(err, 0.99) < 1e-3, np.quantile(err, 0.99)


def test_two_bodies_closed_form():
    """Two particles 0.01 apart (and across the periodic boundary): the
    term is G m g(alpha r) / r^2 towards the other."""
    from solarsystemsimulator_b200 import pm3d
    pm = pm3d.PMPeriodic3D(64, 1.0, 1.0, 0, 2, 1.0, short_range=True)
    for x0 in (0.5, 0.995):
        pos = np.array([[x0, 0.3, 0.7], [x0 + 0.01, 0.3, 0.7]])
        st = pm.load_state(pos, np.zeros_like(pos), np.array([2.0, 3.0]))
        a = _pair_only(pm, st)
        x = pm.alpha * 0.01
        g = math.erfc(x) + 2.0 / math.sqrt(math.pi) * x * math.exp(-x * x)
        assert a[0, 0] == pytest.approx(3.0 * g / 1e-4, rel=2e-5)
        assert a[1, 0] == pytest.approx(-2.0 * g / 1e-4, rel=2e-5)
        assert np.abs(a[:, 1:]).max() < 1e-6 * abs(a[0, 0])


def test_pair_term_improves_on_the_mesh():
    """32,768 clustered particles on a 64^3 mesh: the median relative error
    against the f64 Ewald sum drops well below the mesh force's."""
    from solarsystemsimulator_b200 import pm3d
    from solarsystemsimulator_b200.ewald import EwaldDirect
    pos, mass = _clustered(32_768, 7)
    ew = EwaldDirect(1.0, 1.0, 1e-3)
    errs = {}
    for short in (False, True):
        pm = pm3d.PMPeriodic3D(64, 1.0, 1.0, 0, 2, 1.25, short_range=short, softening=1e-3)
        st = pm.load_state(pos, np.zeros_like(pos), mass)
        idx = torch.arange(0, len(pos), 16, device=st["buf"].device)
        ref = ew.accel(st["parts"], st["buf"][0:3, idx].contiguous(), idx)
        pm.method_forces(st)
        a = st["buf"][6:9, idx]
        errs[short] = pm3d.median_rel_err(a, ref)
    assert errs[True] < 0.2 * errs[False], errs


def test_bad_arguments():
    from solarsystemsimulator_b200 import pm3d
    with pytest.raises(ValueError):
        pm3d.PMPeriodic3D(8, 1.0, 1.0, 0, 2, 1.0, short_range=True)        # r_cut > box / 3
