"""Collision response of the asteroid films on one B200: the per-sample
analysis of the reference's film producer with its array parts on the device.

    cr = CollisionResponse(mass, real_r, vis, is_ast, is_star_bh, m_idx)
    pairs, runaways = cr.analyze_merge(g, dt_y)          # analyze_merge, film_producer.py:707-779
    res = cr.bounce_deltas(g, hits_dev, n_hits, dt_y)    # bounce_deltas, :916-1019
    events, shatter = cr.apply_merges(sim, st, sample, pairs, runaways, k_ev)   # apply_merges, :781-861
    cr.apply_bounce(sim, st, res)                        # apply_bounce, :1021-1040 (deltas on the device)
    parents, frags = cr.fragment(g, res, FRAG_V_ESC, seed)  # fast impacts break up (no reference counterpart)
    cr.apply_fragments(sim, st, parents, frags)
    cr.activate_fragments(g0)                            # after the next batch's integration (g0: its first sample)

`g` is the sample on the device as f32 rows (4, n) [x|y|vx|vy] (the row the
detection card holds); `sample` the same row on the host (f32, 4n). The
host mirrors mass / real_r / vis are updated by apply_merges exactly as the
reference's are; `refresh()` copies them to the device mirrors (the
reference's stammdaten_laden, :636-643), which the caller does after a batch
whose merges changed them.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib

G_AU = 4 * np.pi * np.pi
BOUNCE_E = 0.6            # restitution (film_producer.py:47)
SHATTER_V_ESC = 1.5       # body x body impacts at >= 1.5 v_esc stop the film for the client's shatter
N_FRAG = 5                # fragments of a fragmenting impact (the client's shatter(), index.html:7705-7745)
FRAG_V_ESC = 5.0          # asteroid x asteroid impacts at >= 5 v_esc fragment (the asteroid-cloud configuration)


class CollisionResponse:
    def __init__(self, mass, real_r, vis, is_ast, is_star_bh=None, m_idx=None, device: int = 0, G: float = G_AU,
                 bounce_e: float = BOUNCE_E, shatter: bool = True):
        self.device = int(device)
        self.ctx = _lib.context(device)
        self.dev = torch.device("cuda", self.device)
        self.mass = np.array(mass, dtype=np.float64, copy=True)
        self.real_r = np.array(real_r, dtype=np.float64, copy=True)
        self.vis = np.array(vis, dtype=np.uint8, copy=True)
        self.is_ast = np.asarray(is_ast) != 0
        self.n = len(self.mass)
        self.is_star_bh = (np.zeros(self.n, bool) if is_star_bh is None else np.asarray(is_star_bh) != 0)
        self.pending = np.zeros(self.n, bool)   # fragment slots placed, visible from the next batch
        self.m_idx = np.flatnonzero(~self.is_ast) if m_idx is None else np.asarray(m_idx, np.int64)
        if len(self.m_idx) > 64:
            raise ValueError(f"zu viele massive Koerper: {len(self.m_idx)} > 64")
        self.G = float(G)
        self.e = float(bounce_e)
        self.shatter = bool(shatter)
        self.prev = None                # (px, py) device f32 of the previous analysed sample
        self.d_ast = torch.as_tensor(self.is_ast.astype(np.uint8)).to(self.dev)
        self.d_midx = torch.as_tensor(self.m_idx.astype(np.int64)).to(self.dev)
        self.changed = np.zeros(0, np.int64)   # bodies whose host mirrors the last apply_merges changed
        self._free = None                      # free asteroid slots, ascending (None: recompute)
        self.refresh()

    def refresh(self, idx=None) -> None:
        """Copy the host mirrors (vis, radii, masses) to the device: all of
        them (the reference's stammdaten_laden, film_producer.py:636-643), or
        only the bodies idx (e.g. `self.changed` after apply_merges)."""
        if idx is None:
            self.d_vis = torch.as_tensor(self.vis).to(self.dev)
            self.d_rr32 = torch.as_tensor(self.real_r.astype(np.float32)).to(self.dev)
            self.d_rr = torch.as_tensor(self.real_r).to(self.dev)
            self.d_mass = torch.as_tensor(self.mass).to(self.dev)
            self._free = None
            return
        idx = np.asarray(idx, np.int64).ravel()
        if len(idx) == 0:
            return
        # one transfer: index, vis, radius, mass as f64 rows (exact: indices < 2^53, vis 0/1);
        # the f32 radius is the f64 one rounded to nearest on the device, as astype(float32)
        pk = np.empty((4, len(idx)))
        pk[0], pk[1], pk[2], pk[3] = idx, self.vis[idx], self.real_r[idx], self.mass[idx]
        d = torch.as_tensor(pk).to(self.dev)
        i_t = d[0].long()
        self.d_vis[i_t] = d[1].to(torch.uint8)
        self.d_rr32[i_t] = d[2].float()
        self.d_rr[i_t] = d[2]
        self.d_mass[i_t] = d[3]

    def _free_slots(self) -> np.ndarray:
        """Hidden asteroid slots not yet taken by a fragment, ascending."""
        if self._free is None:
            self._free = np.flatnonzero((self.vis == 0) & self.is_ast & ~self.pending)
        return self._free

    def _s(self):
        return ctypes.c_void_p(_lib.stream_handle(self.device))

    # ---------------------------------------------------------- analysis
    def analyze_merge(self, g: torch.Tensor, dt_y: float, cap: int = 65536):
        """Merge candidates [(massive, body, frac)] and runaways (int64
        array or None) of the sample g (device f32 (4, n))."""
        g = g.contiguous()
        n = self.n
        px, py = (g[0], g[1]) if self.prev is None else self.prev
        pairs = torch.empty((cap, 3), dtype=torch.int32, device=self.dev)
        run = torch.empty(max(n, 1), dtype=torch.int32, device=self.dev)
        npair, nrun = ctypes.c_int64(), ctypes.c_int64()
        with torch.cuda.device(self.device):
            rc = self.ctx.lib.sss_collide_sweep(
                self.ctx.ptr, n, g[0].data_ptr(), g[1].data_ptr(), g[2].data_ptr(), g[3].data_ptr(),
                px.data_ptr(), py.data_ptr(), self.d_rr32.data_ptr(), self.d_vis.data_ptr(), self.d_ast.data_ptr(),
                self.d_mass.data_ptr(), self.d_midx.data_ptr(), len(self.m_idx), float(dt_y), self.G,
                pairs.data_ptr(), cap, run.data_ptr(), n, ctypes.byref(npair), ctypes.byref(nrun), self._s())
        self.ctx.check(rc)
        self.prev = (g[0].clone(), g[1].clone())
        k = npair.value
        out = []
        if k:
            p = pairs[:k].cpu().numpy()
            fr = p[:, 2].copy().view(np.float32)
            out = [(int(a), int(b), float(f)) for a, b, f in zip(p[:, 0], p[:, 1], fr)]
        runaways = run[:nrun.value].cpu().numpy().astype(np.int64) if nrun.value else None
        return out, runaways

    def bounce_deltas(self, g: torch.Tensor, hits: torch.Tensor, n_hits: int, dt_y: float):
        """None or (hi, hj, touched, deltas) as device tensors: the active
        hits in order (int32), the touched bodies ascending (int64) and their
        (dx, dy, dvx, dvy) (f64)."""
        if n_hits <= 0:
            return None
        g = g.contiguous()
        n = self.n
        pairs = torch.empty((n_hits, 2), dtype=torch.int32, device=self.dev)
        cap_t = min(n, 2 * n_hits)
        touched = torch.empty(cap_t, dtype=torch.int64, device=self.dev)
        deltas = torch.empty((cap_t, 4), dtype=torch.float64, device=self.dev)
        na, nt = ctypes.c_int64(), ctypes.c_int64()
        with torch.cuda.device(self.device):
            rc = self.ctx.lib.sss_collide_bounce(
                self.ctx.ptr, n, g[0].data_ptr(), g[1].data_ptr(), g[2].data_ptr(), g[3].data_ptr(),
                self.d_rr.data_ptr(), self.d_mass.data_ptr(), hits.data_ptr(), int(n_hits), float(dt_y), self.e,
                pairs.data_ptr(), touched.data_ptr(), deltas.data_ptr(), ctypes.byref(na), ctypes.byref(nt),
                self._s())
        self.ctx.check(rc)
        if na.value == 0:
            return None
        return pairs[:na.value, 0], pairs[:na.value, 1], touched[:nt.value], deltas[:nt.value]

    # ---------------------------------------------------------- application
    def apply_merges(self, sim, st, sample, pairs, runaways, k_ev: int = 0, contact: dict | None = None,
                     batched: bool = False):
        """Apply merges and runaway removals in order (apply_merges,
        film_producer.py:781-861) to the simulation and the host mirrors.
        Returns (events, shatter): events (a, b, new_mass, kind, frac, x, y),
        kind 0 merge / 2 runaway; shatter (a, b, frac) when a body x body
        impact at >= 1.5 v_esc stopped the processing (the reference freezes
        the film there and leaves the fragments to its client).

        `sample` is the sample as host f32 (4n), or the device tensor (4, n):
        then only the columns of the bodies named in `pairs` and `runaways`
        come to the host. By default each merge and removal reaches the
        simulation at once, through the reference's calls in the reference's
        order (apply_body_state, deactivate_body, set_radius). With
        batched=True (a simulation with apply_body_states, set_radii and
        deactivate_bodies, as NBodyCuda) they are applied in one go after the
        loop (each body's last state, then the removals); the loop reads host
        data only, so the simulation ends in the same state. `self.changed`
        lists the bodies whose host mirrors changed (for refresh(self.changed))."""
        n = self.n
        if isinstance(sample, torch.Tensor):
            need = {int(a) for a, _, _ in pairs} | {int(b) for _, b, _ in pairs}
            if runaways is not None:
                need |= {int(j) for j in runaways}
            sx, sy, svx, svy = (np.empty(n, np.float32) for _ in range(4))
            if need:
                ni = np.fromiter(sorted(need), np.int64, len(need))
                cols = sample.reshape(4, n)[:, torch.as_tensor(ni).to(sample.device)].cpu().numpy()
                sx[ni], sy[ni], svx[ni], svy[ni] = cols[0], cols[1], cols[2], cols[3]
        else:
            sx, sy = sample[0:n], sample[n:2 * n]
            svx, svy = sample[2 * n:3 * n], sample[3 * n:4 * n]
        mass, vis, rr = self.mass, self.vis, self.real_r
        events = []
        contact = {} if contact is None else contact
        states, radii, removed = {}, {}, []     # batched simulation updates, in the loop's order
        changed = []

        def flush():
            if sim is None or not batched:
                return
            if states:
                d = st["dim"]
                rows = [[v[0], v[1], 0.0, v[2], v[3], 0.0, v[4]] if d == 3 else list(v) for v in states.values()]
                sim.apply_body_states(st, list(states), rows)
            if radii:
                sim.set_radii(st, list(radii), list(radii.values()))
            if removed:
                sim.deactivate_bodies(st, removed)

        def finish(shatter):
            flush()
            self.changed = np.unique(np.asarray(changed, np.int64))
            c = self.changed
            hid = c[self.is_ast[c] & (self.vis[c] == 0) & ~self.pending[c]]
            if len(hid) and self._free is not None:
                # hidden asteroids are free slots now: insert them into the ascending list
                free = self._free
                pos = np.searchsorted(free, hid)
                there = free[np.minimum(pos, len(free) - 1)] == hid if len(free) else np.zeros(len(hid), bool)
                self._free = np.insert(free, pos[~there], hid[~there])
            return events, shatter

        for mi, j, frac in pairs:
            tk = contact.pop(j, None)
            if tk is not None:
                f_kern = tk - (k_ev + 1)
                if -1.0 <= f_kern <= 1.0:
                    frac = f_kern
            if (self.shatter and not self.is_ast[mi] and not self.is_ast[j] and not self.is_star_bh[mi]
                    and not self.is_star_bh[j] and vis[mi] and vis[j] and mass[mi] > 0 and mass[j] > 0):
                v_imp = float(np.hypot(svx[j] - svx[mi], svy[j] - svy[mi]))
                touch = max(1e-12, rr[mi] + rr[j])
                v_esc = float(np.sqrt(2.0 * self.G * (mass[mi] + mass[j]) / touch))
                if v_imp >= SHATTER_V_ESC * v_esc:
                    return finish((int(mi), int(j), frac))
            if not vis[mi] or not vis[j] or mass[mi] <= 0:
                continue
            a, b = (mi, j) if mass[mi] >= mass[j] else (j, mi)
            m_a, m_b = mass[a], mass[b]
            m_ges = m_a + m_b
            if m_ges <= 0:
                continue
            nx = (sx[a] * m_a + sx[b] * m_b) / m_ges
            ny = (sy[a] * m_a + sy[b] * m_b) / m_ges
            nvx = (svx[a] * m_a + svx[b] * m_b) / m_ges
            nvy = (svy[a] * m_a + svy[b] * m_b) / m_ges
            if sim is not None:
                if batched:
                    states[int(a)] = (float(nx), float(ny), float(nvx), float(nvy), float(m_ges))
                    removed.append(int(b))
                else:
                    sim.apply_body_state(st, a, nx, ny, nvx, nvy, m_ges)
                    sim.deactivate_body(st, b)
            mass[a] = m_ges
            mass[b] = 0.0
            vis[b] = 0
            rr[a] = (rr[a] ** 3 + rr[b] ** 3) ** (1.0 / 3.0)
            changed += [int(a), int(b)]
            if sim is not None:
                if batched:
                    radii[int(a)] = float(rr[a])
                else:
                    sim.set_radius(st, a, float(rr[a]))
            events.append((int(a), int(b), float(m_ges), 0, float(frac), float(nx), float(ny)))
        if runaways is not None and (sim is None or batched):
            # the loop below without its per-body simulation calls: the visible runaways in order
            # (a repeated index acts once)
            run = np.asarray(runaways, np.int64).ravel()
            run = run[vis[run] != 0]
            if len(run):
                first = np.unique(run, return_index=True)[1]
                if len(first) < len(run):
                    run = run[np.sort(first)]
                if sim is not None:
                    removed.extend(run.tolist())
                mass[run] = 0.0
                vis[run] = 0
                changed += run.tolist()
                events += [(0xFFFFFFFF, j, 0.0, 2, 0.0, x, y)
                           for j, x, y in zip(run.tolist(), sx[run].tolist(), sy[run].tolist())]
        elif runaways is not None:
            for j in runaways:
                j = int(j)
                if not vis[j]:
                    continue
                if sim is not None:
                    if batched:
                        removed.append(j)
                    else:
                        sim.deactivate_body(st, j)
                mass[j] = 0.0
                vis[j] = 0
                changed.append(j)
                events.append((0xFFFFFFFF, j, 0.0, 2, 0.0, float(sx[j]), float(sy[j])))
        return finish(None)

    def fragment(self, g: torch.Tensor, res, factor: float, seed: int, n_frag: int = N_FRAG):
        """Fragmenting impacts among the active bounce pairs `res` (the
        result of bounce_deltas): impact speed >= factor x the pair's escape
        speed (sss_collide_fragment). Returns (parents int64 (E, 2), fragments
        f64 (E, n_frag, 6) of x, y, vx, vy, m, r) as host arrays."""
        empty = (np.zeros((0, 2), np.int64), np.zeros((0, n_frag, 6)))
        if res is None or factor <= 0:
            return empty
        hi, hj = res[0], res[1]
        k = int(hi.numel())
        if k == 0:
            return empty
        g = g.contiguous()
        pairs = torch.stack([hi, hj], 1).to(torch.int32).contiguous()
        parents = torch.empty((k, 2), dtype=torch.int32, device=self.dev)
        frags = torch.empty((k, n_frag, 6), dtype=torch.float64, device=self.dev)
        ne = ctypes.c_int64()
        with torch.cuda.device(self.device):
            rc = self.ctx.lib.sss_collide_fragment(
                self.ctx.ptr, self.n, g[0].data_ptr(), g[1].data_ptr(), g[2].data_ptr(), g[3].data_ptr(),
                self.d_rr.data_ptr(), self.d_mass.data_ptr(), pairs.data_ptr(), k, self.G, float(factor),
                int(n_frag), int(seed) & ((1 << 64) - 1), parents.data_ptr(), frags.data_ptr(), k,
                ctypes.byref(ne), self._s())
        self.ctx.check(rc)
        e = ne.value
        return parents[:e].cpu().numpy().astype(np.int64), frags[:e].cpu().numpy()

    def apply_fragments(self, sim, st, parents, frags):
        """Replace each fragmenting pair by its fragments (after the bounce
        deltas of the sample were applied: the parents' states are set anew).
        Fragments 0 and 1 take the parents' slots, the others free asteroid
        slots (hidden asteroids, lowest index first). A body can sit in
        several active bounce pairs; only the first event (in pair order)
        that names a body fragments it, and a later event sharing a parent
        with an earlier one is left out, as is an event with a parent hidden
        by a merge of the same sample and an event without enough free slots
        (the bounce of a left-out event stands). Returns (events (a, b,
        fragment mass, 3, 0.0, x, y), slots used per event, events left out).

        The samples of a batch are integrated before they are analysed, so
        the rest of the batch still shows the free slots where they were; the
        new slots join the analysis (vis) with the next batch, when
        activate_fragments() is called after its integration. The simulation
        integrates them from now on."""
        if len(parents) == 0:
            return [], [], 0
        n_events = len(parents)
        # a parent hidden since the broadphase ran (absorbed by a merge of the
        # same sample) does not fragment; neither does a body twice
        flat = parents.reshape(-1)
        if len(np.unique(flat)) == len(flat):      # disjoint (the one-hit-per-body bounce pairs)
            keep = np.flatnonzero((self.vis[parents[:, 0]] != 0) & (self.vis[parents[:, 1]] != 0))
        else:
            used, keep = set(), []
            for q, (a, b) in enumerate(parents):
                if self.vis[a] and self.vis[b] and int(a) not in used and int(b) not in used:
                    keep.append(q)
                    used.update((int(a), int(b)))
        parents, frags = parents[keep], frags[keep]
        n_frag = frags.shape[1]
        if len(parents) == 0:
            return [], [], n_events
        free = self._free_slots()                                             # ascending
        e = min(len(parents), len(free) // (n_frag - 2))                      # events with room, in order
        skipped = n_events - e
        if e == 0:
            return [], [], skipped
        slots = np.concatenate([parents[:e], free[:e * (n_frag - 2)].reshape(e, n_frag - 2)], 1)
        f = frags[:e].reshape(e * n_frag, 6)
        idx = slots.reshape(-1)
        if st["dim"] == 2:
            vals = f[:, 0:5]
        else:
            z = np.zeros((len(f), 1))
            vals = np.concatenate([f[:, 0:2], z, f[:, 2:4], z, f[:, 4:5]], 1)
        sim.set_asteroids(st, idx, vals, f[:, 5])
        self.mass[idx] = f[:, 4]
        self.real_r[idx] = f[:, 5]
        self.pending[slots[:, 2:].reshape(-1)] = True
        self._free = free[e * (n_frag - 2):]
        if self.prev is not None:          # fragments 0 and 1: their sweep segments start where they are placed
            p_idx = torch.as_tensor(slots[:, :2].reshape(-1)).to(self.dev)
            f01 = frags[:e, :2].reshape(2 * e, 6)
            self.prev[0][p_idx] = torch.as_tensor(f01[:, 0].astype(np.float32)).to(self.dev)
            self.prev[1][p_idx] = torch.as_tensor(f01[:, 1].astype(np.float32)).to(self.dev)
        self.refresh(idx)
        fr = frags[:e]
        # the event's place: the mean of its fragments' positions (summed in fragment order)
        events = [(a, b, m, 3, 0.0, x, y) for (a, b), m, x, y in
                  zip(parents[:e].tolist(), fr[:, 0, 4].tolist(), fr[:, :, 0].mean(axis=1).tolist(),
                      fr[:, :, 1].mean(axis=1).tolist())]
        return events, slots.tolist(), skipped

    def activate_fragments(self, g0: torch.Tensor | None = None) -> np.ndarray:
        """Make the fragments placed in free slots visible to the analysis
        (call after the integration of the next batch, with g0 its first
        sample (4, n) on the device: the new bodies' first sweep segments
        start there, as a body without a previous sample); returns their
        indices."""
        idx = np.flatnonzero(self.pending)
        if len(idx):
            self.vis[idx] = 1
            self.pending[idx] = False
            if self.prev is not None and g0 is not None:
                p_idx = torch.as_tensor(idx).to(self.dev)
                self.prev[0][p_idx] = g0[0][p_idx]
                self.prev[1][p_idx] = g0[1][p_idx]
            self.refresh(idx)
        return idx

    def apply_bounce(self, sim, st, res) -> int:
        """Add the bounce deltas to the simulation on the device (apply_bounce,
        film_producer.py:1021-1040); returns the number of bounces."""
        if res is None:
            return 0
        hi, hj, touched, deltas = res
        sim.apply_deltas_device(st, touched, deltas, int(touched.numel()))
        return int(hi.numel())
