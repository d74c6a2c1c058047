"""Host-side bookkeeping of the collision response (no GPU): the free-slot
list kept across samples and the batched merge response with its runaways
in one array operation, against a recount and against the reference's
per-body call sequence (film_producer.py:781-861) on a recording stand-in
for the simulation."""
import copy

import numpy as np
import pytest

from solarsystemsimulator_b200.collide import CollisionResponse

N, M = 2000, 8


def _response(rng):
    """A CollisionResponse with host mirrors only (the device side is not
    touched by apply_merges without a device sample)."""
    cr = CollisionResponse.__new__(CollisionResponse)
    cr.n = N
    cr.mass = np.concatenate([rng.uniform(1e-6, 1e-3, M), rng.uniform(0, 1e-12, N - M)])
    cr.real_r = rng.uniform(1e-6, 1e-4, N)
    cr.vis = (rng.random(N) > 0.1).astype(np.uint8)
    cr.is_ast = np.arange(N) >= M
    cr.is_star_bh = np.zeros(N, bool)
    cr.pending = np.zeros(N, bool)
    cr.G = 4 * np.pi ** 2
    cr.shatter = False
    cr._free = None
    cr.changed = np.zeros(0, np.int64)
    return cr


class _Recorder:
    """The simulation's point updates, recorded in call order."""

    def __init__(self):
        self.removed, self.states, self.radii = [], {}, {}

    def apply_body_state(self, st, a, x, y, vx, vy, m):
        self.states[int(a)] = (float(x), float(y), float(vx), float(vy), float(m))

    def deactivate_body(self, st, b):
        self.removed.append(int(b))

    def set_radius(self, st, a, r):
        self.radii[int(a)] = float(r)

    def apply_body_states(self, st, idx, rows):
        for i, r in zip(idx, rows):
            self.states[int(i)] = tuple(float(v) for v in r)

    def set_radii(self, st, idx, r):
        for i, v in zip(idx, r):
            self.radii[int(i)] = float(v)

    def deactivate_bodies(self, st, idx):
        self.removed += [int(i) for i in idx]


def _merge_inputs(rng):
    sample = rng.normal(0, 1, 4 * N).astype(np.float32)
    pairs = [(int(rng.integers(0, M)), int(rng.integers(M, N)), 0.5) for _ in range(int(rng.integers(0, 6)))]
    pairs += [(int(rng.integers(0, N)), int(rng.integers(0, N)), 0.1) for _ in range(int(rng.integers(0, 3)))]
    run = rng.integers(0, N, int(rng.integers(0, 40)))
    if len(run) > 2 and rng.random() < 0.5:
        run[1] = run[0]                                  # a repeated index acts once
    return sample, pairs, run


@pytest.mark.parametrize("seed", range(4))
def test_batched_merges_and_runaways_follow_the_reference_sequence(seed):
    rng = np.random.default_rng(seed)
    for _ in range(60):
        base = _response(rng)
        sample, pairs, run = _merge_inputs(rng)
        out = []
        for batched in (False, True):
            cr = copy.deepcopy(base)
            sim = _Recorder()
            ev, sh = cr.apply_merges(sim, {"dim": 2}, sample, pairs, run.copy(), batched=batched)
            out.append((ev, sh, cr.mass, cr.vis, cr.real_r, cr.changed, sim))
        (ev0, sh0, m0, v0, r0, c0, s0), (ev1, sh1, m1, v1, r1, c1, s1) = out
        assert ev0 == ev1 and sh0 == sh1
        for a, b in ((m0, m1), (v0, v1), (r0, r1), (c0, c1)):
            assert np.array_equal(a, b)
        assert s0.removed == s1.removed and s0.states == s1.states and s0.radii == s1.radii
        cr = copy.deepcopy(base)                         # no simulation: the mirrors alone
        ev2, _ = cr.apply_merges(None, None, sample, pairs, run.copy())
        assert ev2 == ev0 and np.array_equal(cr.vis, v0) and np.array_equal(cr.mass, m0)


def test_free_slot_list_equals_a_recount():
    """Hidden asteroids (absorbed, runaways) join the ascending free-slot
    list as merges happen; fragments take slots from its front and become
    visible later. After every step the kept list equals a recount."""
    rng = np.random.default_rng(3)
    cr = _response(rng)
    kept = 0
    for _ in range(300):
        if cr._free is None or rng.random() < 0.3:       # fragments placed in the lowest free slots
            f = cr._free_slots()
            k = int(rng.integers(0, min(len(f), 30) + 1))
            cr.pending[f[:k]] = True
            cr._free = f[k:]
        if rng.random() < 0.2:                           # ... and activated with the next batch
            idx = np.flatnonzero(cr.pending)
            cr.vis[idx] = 1
            cr.pending[idx] = False
        sample, pairs, run = _merge_inputs(rng)
        cr.apply_merges(None, None, sample, pairs, run)
        inc = cr._free
        cr._free = None
        if inc is not None:
            assert np.array_equal(inc, cr._free_slots())
            kept += 1
    assert kept > 200
