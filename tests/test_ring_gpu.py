"""GPU ring slots and row reorder (sss_ring_slot, sss_ring_reorder) against
oracle/ring.py, the restatement of the reference's schreibe_slot and
self-gravity reorder (film_producer.py:79-123, :1245-1261): byte-exact."""
import struct

import numpy as np
import pytest
import torch

from oracle import ring as orng

pytestmark = pytest.mark.gpu

G_AU = 4 * np.pi * np.pi


def _divers(n_div=16, n_calm=40, seed=5):
    """Sun, three planets, asteroids diving at the sun (hot: gap-free
    sub-sample chains) and calm belt asteroids."""
    rng = np.random.default_rng(seed)
    x = [0.0]; y = [0.0]; vx = [0.0]; vy = [0.0]; mass = [1.0]; is_ast = [0]
    for r in (0.7, 1.5, 5.2):
        x.append(r); y.append(0.0); vx.append(0.0); vy.append(np.sqrt(G_AU / r)); mass.append(3e-6); is_ast.append(0)
    for k in range(n_calm + n_div):
        if k % 3 == 1 and k // 3 < n_div:
            t = rng.random() * 2 * np.pi
            r = 0.05 + 0.05 * rng.random()
            sp = 20.0 + 20.0 * rng.random()
            x.append(r * np.cos(t)); y.append(r * np.sin(t))
            vx.append(-sp * np.cos(t)); vy.append(-sp * np.sin(t))
        else:
            r = 2.5 + 0.01 * k
            t = 0.3 * k
            v = np.sqrt(G_AU / r)
            x.append(r * np.cos(t)); y.append(r * np.sin(t)); vx.append(-v * np.sin(t)); vy.append(v * np.cos(t))
        mass.append(0.0); is_ast.append(1)
    n = len(x)
    return (np.array(x), np.array(y), np.array(vx), np.array(vy), np.array(mass), np.ones(n, np.uint8),
            np.array(is_ast, np.uint8))


def _defined(buf, n, m_sub, sub_max):
    """The bytes a slot defines: x|y, the count, the first count indices and chains."""
    b = bytes(buf)
    (nh,) = struct.unpack_from("<I", b, 8 * n)
    idx0 = 8 * n + 4
    ch0 = idx0 + 4 * sub_max
    return b[:8 * n + 4] + b[idx0:idx0 + 4 * nh] + b[ch0:ch0 + 8 * m_sub * nh], nh


@pytest.mark.parametrize("sub_max", [2048, 3])
def test_slots_match_oracle(sub_max):
    from solarsystemsimulator_b200 import ring
    from solarsystemsimulator_b200.nbody_kernel import NBodyCuda
    sim = NBodyCuda([0])
    st = sim.load_state(*_divers())
    n = st["N"]
    K = 4
    rows = sim.step_batch(st, 0.5 / 365.25, K)
    slot = torch.zeros(orng.slot_bytes(n, sim.m_sub, sub_max), dtype=torch.uint8, device="cuda")
    seen_hot = 0
    for ks in range(K):
        over = ring.write_slot(sim, st, ks, slot, sub_max)
        ref, ref_over = orng.write_slot(n, sim.m_sub, sub_max, rows[ks], st["sub"][ks])
        got, nh = _defined(slot.cpu().numpy(), n, sim.m_sub, sub_max)
        want, nh_ref = _defined(np.frombuffer(ref, np.uint8), n, sim.m_sub, sub_max)
        assert nh == nh_ref and got == want
        assert over == ref_over
        seen_hot += nh
    assert seen_hot > 0
    if sub_max == 3:
        assert any(len(s[0]) > 3 for s in st["sub"])


def test_reorder_matches_oracle():
    from solarsystemsimulator_b200 import ring
    rng = np.random.default_rng(9)
    n, nm = 1000, 300
    perm = rng.permutation(n)
    sg_m, sg_t = np.sort(perm[:nm]), np.sort(perm[nm:])
    K = 3
    outs = rng.normal(0, 1, (K, 4 * nm + 2 * (n - nm))).astype(np.float32)
    got = ring.reorder_selfgrav(torch.as_tensor(outs).cuda(), sg_m, sg_t, n).cpu().numpy()
    assert np.array_equal(got, orng.reorder_selfgrav(outs, sg_m, sg_t, n))


@pytest.mark.parametrize("case", ["few", "overflow"])
def test_slot_matches_reference_golden(load_golden, case):
    """sss_ring_slot against the bytes the reference's own schreibe_slot
    wrote (tests/golden/make_golden.py): the golden hot bodies become gap-free
    sub-sample chains in the frame kernel's layout [m_sub][2][n_ast]."""
    import ctypes
    from solarsystemsimulator_b200 import _lib
    g = load_golden("ring_slots.npz")
    n, m_sub, sub_max = int(g["n"]), int(g["m_sub"]), int(g[f"{case}_sub_max"])
    idx, pos = g[f"{case}_idx"], g[f"{case}_pos"]
    sub_pos = np.zeros((m_sub, 2, n), np.float32)
    sub_pos[:, :, idx] = pos
    sub_n = np.zeros(n, np.uint8)
    sub_n[idx] = m_sub
    sub_n[np.setdiff1d(np.arange(0, n, 7), idx)] = m_sub - 1      # chains with a gap are not hot
    d = {k: torch.as_tensor(v).cuda() for k, v in
         (("row", g["out_i"]), ("pos", sub_pos), ("sn", sub_n), ("ai", np.arange(n, dtype=np.int64)))}
    slot = torch.zeros(orng.slot_bytes(n, m_sub, sub_max), dtype=torch.uint8, device="cuda")
    hot = ctypes.c_int64()
    ctx = _lib.context(0)
    ctx.check(ctx.lib.sss_ring_slot(ctx.ptr, d["row"].data_ptr(), n, d["pos"].data_ptr(), d["sn"].data_ptr(),
                                    d["ai"].data_ptr(), n, m_sub, 2, sub_max, slot.data_ptr(), ctypes.byref(hot),
                                    ctypes.c_void_p(_lib.stream_handle(0))))
    got, nh = _defined(slot.cpu().numpy(), n, m_sub, sub_max)
    want, nh_ref = _defined(g[f"{case}_slot"], n, m_sub, sub_max)
    assert nh == nh_ref and got == want
    assert (hot.value > sub_max) == bool(g[f"{case}_overflow"])


def test_reorder_matches_reference_golden(load_golden):
    from solarsystemsimulator_b200 import ring
    g = load_golden("ring_slots.npz")
    got = ring.reorder_selfgrav(torch.as_tensor(g["sg_outs"]).cuda(), g["sg_m"], g["sg_t"], int(g["sg_n"]))
    assert np.array_equal(got.cpu().numpy(), g["sg_full"])
