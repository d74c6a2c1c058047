"""Thousands of small independent N-body systems on one B200.

    ens = BatchedSystems(systems, device=0)      # list of {pos, vel, mass, G, dt}
    ens.run(steps)                                # f64 Yoshida-4, all systems
    pos, vel = ens.export()                       # per system

Systems are grouped by body count (<= 4, <= 8, <= 16, <= 32, <= 64); each
group runs in one persistent kernel (sss_batched_launch) with the team
mapping that `autotune` measured fastest on this device: a team of T <= 32
lanes with B bodies per lane (positions by warp shuffles), or for the larger
groups a block of T threads per system that splits each body's sources
over T / 16, T / 32 or T / 64 threads. `run` launches every group concurrently, and
`capture(steps)` records those launches once into a CUDA graph that `replay`
re-launches with one call.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib

BUCKETS = (4, 8, 16, 32, 64)
TEAMS = (1, 2, 4, 8, 16, 32)
PER_LANE = (1, 2, 4, 8)
SUPPORTED = {(1, 1), (1, 2), (1, 4), (1, 8), (2, 1), (2, 2), (2, 4), (2, 8), (4, 1), (4, 2), (4, 4), (4, 8),
             (8, 1), (8, 2), (8, 4), (8, 8), (16, 1), (16, 2), (16, 4), (32, 1), (32, 2)}
# a block per system (T > 32 threads, B = 1): 16, 32 or 64 targets x T / 16, T / 32 or T / 64 source chunks
BLOCK_MAPS = {16: ((64, 1), (128, 1)), 32: ((64, 1), (128, 1), (256, 1)), 64: ((128, 1), (256, 1), (512, 1))}


def block_bucket(max_n: int) -> int:
    return 16 if max_n <= 16 else (32 if max_n <= 32 else 64)

_tuned: dict = {}


def candidates(max_n: int):
    """Team mappings that hold max_n bodies, smallest team first."""
    out = []
    for t in TEAMS:
        for b in PER_LANE:
            if (t, b) in SUPPORTED and t * b >= max_n and (t * b) // 2 < max_n:
                out.append((t, b))
    if max_n > 8:
        out.extend(BLOCK_MAPS[block_bucket(max_n)])
    return out


class BatchedSystems:
    def __init__(self, systems, device: int = 0, eps2: float = 0.0, dim: int = 3, autotune: bool = True):
        self.device = int(device)
        self.dim = int(dim)
        self.eps2 = float(eps2)
        self.ctx = _lib.context(self.device)
        dev = torch.device("cuda", self.device)
        sizes = np.array([len(s["mass"]) for s in systems])
        if sizes.max() > 64 or sizes.min() < 1:
            raise ValueError("systems must have 1..64 bodies")
        off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        self.n_sys = len(systems)
        self.sizes = sizes
        self.off_h = off
        X = np.concatenate([s["pos"][:dim] for s in systems], 1)
        V = np.concatenate([s["vel"][:dim] for s in systems], 1)
        self.x = torch.from_numpy(np.ascontiguousarray(X)).to(dev)
        self.v = torch.from_numpy(np.ascontiguousarray(V)).to(dev)
        self.m = torch.from_numpy(np.concatenate([s["mass"] for s in systems]).astype(np.float64)).to(dev)
        self.off = torch.from_numpy(off).to(dev)
        self.G = torch.tensor([float(s["G"]) for s in systems], dtype=torch.float64, device=dev)
        self.dt = torch.tensor([float(s["dt"]) for s in systems], dtype=torch.float64, device=dev)
        self.groups = []
        lo = 0
        for hi in BUCKETS:
            idx = np.flatnonzero((sizes > lo) & (sizes <= hi))
            lo = hi
            if len(idx) == 0:
                continue
            # heaviest systems first: teams that take a second system take light ones
            idx = idx[np.argsort(-sizes[idx], kind="stable")].astype(np.int32)
            self.groups.append({"max_n": int(sizes[idx].max()), "list": torch.from_numpy(idx).to(dev),
                                "n": len(idx), "map": candidates(int(sizes[idx].max()))[0]})
        self._graph = None
        if autotune:
            self.autotune()

    # ---------------------------------------------------------- launches
    def _ptrs(self, t):
        arr = (ctypes.c_void_p * 3)()
        for c in range(self.dim):
            arr[c] = t[c].data_ptr()
        return arr

    def _launch(self, g, steps, stream, mapping=None, sys_list=None, n_list=None):
        t, b = mapping or g["map"]
        lst = g["list"] if sys_list is None else sys_list
        n = g["n"] if n_list is None else n_list
        rc = self.ctx.lib.sss_batched_launch(
            self.ctx.ptr, self.dim, self._ptrs(self.x), self._ptrs(self.v), self.m.data_ptr(),
            self.off.data_ptr(), self.G.data_ptr(), self.dt.data_ptr(), lst.data_ptr(), n, g["max_n"], t, b,
            self.eps2, int(steps), 0, ctypes.c_void_p(stream))
        self.ctx.check(rc)

    def run(self, steps: int) -> None:
        """`steps` Yoshida steps of every system; the groups run concurrently."""
        main = torch.cuda.current_stream(self.device)
        if len(self.groups) == 1:
            self._launch(self.groups[0], steps, main.cuda_stream)
            return
        side = [torch.cuda.Stream(self.device) for _ in self.groups]
        for s, g in zip(side, self.groups):
            s.wait_stream(main)
            self._launch(g, steps, s.cuda_stream)
        for s in side:
            main.wait_stream(s)

    def run_one_launch_per_system(self, steps: int, systems=None) -> None:
        """The comparison: the same kernel launched once per system (serially)."""
        stream = torch.cuda.current_stream(self.device).cuda_stream
        for g in self.groups:
            lst = g["list"].cpu().numpy()
            for s in lst if systems is None else [x for x in lst if x in systems]:
                one = torch.tensor([s], dtype=torch.int32, device=self.x.device)
                self._launch(g, steps, stream, sys_list=one, n_list=1)

    def capture(self, steps: int) -> None:
        """Record `run(steps)` once into a CUDA graph (one launch per replay).
        The state is unchanged by the capture itself."""
        x0, v0 = self.x.clone(), self.v.clone()
        self.run(1)                                   # warm-up outside the capture
        torch.cuda.synchronize(self.device)
        self.x.copy_(x0)
        self.v.copy_(v0)
        self._graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self._graph):
            self.run(steps)

    def replay(self) -> None:
        if self._graph is None:
            raise RuntimeError("capture(steps) first")
        self._graph.replay()

    # ---------------------------------------------------------- autotune
    def autotune(self, probe_steps: int = 20, reps: int = 2) -> dict:
        """Per group, time every team mapping that holds the group on a copy
        of the state and keep the fastest (cached per device and group shape)."""
        name = torch.cuda.get_device_name(self.device)
        x0, v0 = self.x.clone(), self.v.clone()
        stream = torch.cuda.current_stream(self.device)
        report = {}
        for g in self.groups:
            key = (name, self.dim, g["max_n"], g["n"])
            if key in _tuned:
                g["map"] = _tuned[key]
                continue
            best, best_t = None, None
            for mapping in candidates(g["max_n"]):
                self._launch(g, 1, stream.cuda_stream, mapping)           # warm-up / load
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                for _ in range(reps):
                    self._launch(g, probe_steps, stream.cuda_stream, mapping)
                e1.record(stream)
                e1.synchronize()
                t = e0.elapsed_time(e1)
                report[(g["max_n"],) + mapping] = t
                if best_t is None or t < best_t:
                    best, best_t = mapping, t
            g["map"] = best
            _tuned[key] = best
        self.x.copy_(x0)
        self.v.copy_(v0)
        return report

    # ---------------------------------------------------------- results
    def export(self):
        X, V = self.x.cpu().numpy(), self.v.cpu().numpy()
        return [(X[:, a:b], V[:, a:b]) for a, b in zip(self.off_h[:-1], self.off_h[1:])]

    def pairs_per_step(self) -> int:
        return int(3 * np.sum(self.sizes * (self.sizes - 1)))
