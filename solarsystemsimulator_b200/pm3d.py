"""3-D periodic particle mesh with a learned short-range correction, on one
B200.

The reference's PM cycle (TODO.md:225-253: CIC deposit, Poisson solve in
Fourier space with the k = 0 term removed, CIC interpolation with the
deposit's stencil; the 2-D isolated code is backend/pm_kernel.py) in a
periodic cube, KDK leapfrog as the reference's NBodyPM (pm_kernel.py:
247-281):

    pm = PMPeriodic3D(mesh_n=256, box=1.0, G=1.0)
    st = pm.load_state(pos, vel, mass)          # (N, 3), (N, 3), (N,) or scalar
    snaps = pm.step_batch(st, dt, steps, snapshots=True)   # f32 (steps, 6N)
    x, v = pm.export_f64(st)

and the learned correction with its judge (NBodyPMLearned): a per-particle
MLP adds the short-range force the mesh cannot resolve; every
`check_every` steps the f64 Ewald direct sum on fresh random particles
judges the corrected force, the steps since the last check are reverted
and replayed when it fails, and the network is trained online on the
residuals (direct - mesh) of those particles.
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .ewald import EwaldDirect
from .mlp import ShortRangeMLP


class _CudaArray:
    """__cuda_array_interface__ wrapper of a library-owned device buffer."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


class PMPeriodic3D:
    """Mesh solver of one mesh size (an sss_pm3 plan) and the KDK stepper."""

    def __init__(self, mesh_n: int = 256, box: float = 1.0, G: float = 1.0, device: int = 0, deconv: int = 2,
                 r_split_cells: float = 0.6, short_range: bool = False, softening: float = 0.0,
                 x_cut: float = 3.5):
        """Green's function -4 pi G / k^2 * W_CIC(k)^-deconv *
        exp(-k^2 r_split^2), r_split = r_split_cells mesh cells.

        short_range adds the P3M pair term every force pass: the exact
        complement of that mesh force (erfc split with alpha = 1 / (2
        r_split)) and the Plummer softening, for pairs closer than r_cut =
        x_cut / alpha (sss_pm3_short)."""
        self.device = int(device)
        self.ctx = _lib.context(device)
        self.mesh_n = int(mesh_n)
        self.box = float(box)
        self.G = float(G)
        self.deconv = int(deconv)
        self.r_split = float(r_split_cells) * self.box / self.mesh_n
        self.short_range = bool(short_range)
        self.softening = float(softening)
        self.alpha = 0.5 / self.r_split if self.r_split > 0.0 else 0.0
        self.r_cut = float(x_cut) / self.alpha if self.alpha > 0.0 else 0.0
        if self.short_range and not (self.r_split > 0.0 and 3.0 * self.r_cut <= self.box):
            raise ValueError("short_range needs r_split > 0 and r_cut <= box / 3")
        ptr = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            self.ctx.check(self.ctx.lib.sss_pm3_create(self.ctx.ptr, self.mesh_n, self.box, ctypes.byref(ptr)))
        self.ptr = ptr
        rho, acc = _lib._dp(), _lib._dp()
        self.ctx.check(self.ctx.lib.sss_pm3_meshes(self.ptr, ctypes.byref(rho), ctypes.byref(acc)))
        n = self.mesh_n
        dev = torch.device("cuda", self.device)
        self.rho = torch.as_tensor(_CudaArray(rho.value, (n, n, n), "<f4"), device=dev)
        self.acc_mesh = torch.as_tensor(_CudaArray(acc.value, (3, n, n, n), "<f4"), device=dev)

    def __del__(self):
        try:
            if getattr(self, "ptr", None):
                self.rho = self.acc_mesh = None
                self.ctx.lib.sss_pm3_destroy(self.ptr)
                self.ptr = None
        except Exception:
            pass

    def name(self) -> str:
        return f"B200 periodic PM {self.mesh_n}^3"

    def _s(self):
        return ctypes.c_void_p(_lib.stream_handle(self.device))

    def _call(self, name, *args):
        with torch.cuda.device(self.device):
            self.ctx.check(getattr(self.ctx.lib, name)(self.ptr, *args, self._s()))

    # ---- state
    def load_state(self, pos, vel, mass) -> dict:
        """Particle state on the device: pos, vel (N, 3) (positions wrapped
        into [0, box)), mass (N,) or one scalar for every particle."""
        dev = torch.device("cuda", self.device)
        pos = np.asarray(pos, np.float64)
        vel = np.asarray(vel, np.float64)
        if pos.ndim != 2 or pos.shape[1] != 3 or vel.shape != pos.shape:
            raise ValueError("pos and vel must be (N, 3)")
        n = len(pos)
        if n < 1:
            raise ValueError("leerer Zustand")
        buf = torch.zeros((9, n), dtype=torch.float64, device=dev)
        p = pos - self.box * np.floor(pos / self.box)
        buf[0:3] = torch.as_tensor(np.ascontiguousarray(p.T)).to(dev)
        buf[3:6] = torch.as_tensor(np.ascontiguousarray(vel.T)).to(dev)
        if np.ndim(mass) == 0:
            m, mc, total = None, float(mass), float(mass) * n
        else:
            mm = np.asarray(mass, np.float64)
            if mm.shape != (n,):
                raise ValueError("mass must be (N,) or a scalar")
            m, mc, total = torch.as_tensor(mm).to(dev), 0.0, float(mm.sum())
        st = {"buf": buf, "mass": m, "mass_const": mc, "n": n, "acc_valid": False,
              "rho_mean": total / self.box ** 3}
        st["parts"] = self._parts(st)
        return st

    def _parts(self, st) -> _lib.Pm3Particles:
        b = st["buf"]
        s = _lib.Pm3Particles()
        s.n = st["n"]
        for c in range(3):
            s.x[c] = b[c].data_ptr()
            s.v[c] = b[3 + c].data_ptr()
            s.a[c] = b[6 + c].data_ptr()
        s.m = st["mass"].data_ptr() if st["mass"] is not None else None
        s.mass_const = st["mass_const"]
        return s

    def export_f64(self, st):
        """(pos, vel) as f64 (N, 3) host arrays."""
        b = st["buf"].cpu().numpy()
        return b[0:3].T.copy(), b[3:6].T.copy()

    # ---- passes
    def mesh_forces(self, st) -> None:
        """Deposit and solve: the acceleration meshes of the current positions."""
        self._call("sss_pm3_density", ctypes.byref(st["parts"]))
        self._call("sss_pm3_solve", self.G, self.deconv, self.r_split)

    def gather(self, st, mode=_lib.PM3_FORCE, hdt=0.0, dt=0.0, snap=None) -> None:
        self._call("sss_pm3_gather", ctypes.byref(st["parts"]), int(mode), float(hdt), float(dt),
                   snap.data_ptr() if snap is not None else None)

    def kick_drift(self, st, hdt: float, dt: float) -> None:
        self._call("sss_pm3_kick_drift", ctypes.byref(st["parts"]), float(hdt), float(dt))

    def short(self, st, mode=_lib.PM3_FORCE, hdt=0.0, dt=0.0, snap=None) -> None:
        """Add the P3M pair term to the mesh force in the state, then the
        epilogue `mode`."""
        self._call("sss_pm3_short", ctypes.byref(st["parts"]), self.G, self.alpha, self.r_cut, self.softening,
                   int(mode), float(hdt), float(dt), snap.data_ptr() if snap is not None else None)

    def method_forces(self, st, mode=_lib.PM3_FORCE, hdt=0.0, dt=0.0, snap=None) -> None:
        """The force without the network (mesh, and the pair term when
        short_range) with the epilogue `mode`."""
        self.mesh_forces(st)
        if self.short_range:
            self.gather(st)
            self.short(st, mode, hdt, dt, snap)
        else:
            self.gather(st, mode, hdt, dt, snap)

    def forces(self, st, net: ShortRangeMLP | None = None) -> torch.Tensor:
        """Accelerations at the current positions into the state (3, N)."""
        self.method_forces(st)
        if net is not None:
            net_correct(net, self, st, _lib.PM3_FORCE, 0.0, 0.0, None)
        st["acc_valid"] = True
        return st["buf"][6:9]

    def step_batch(self, st, dt: float, steps: int, net: ShortRangeMLP | None = None, snapshots: bool = False):
        """`steps` KDK steps (each: one deposit, one solve, one fused
        gather [+ correction] pass). Returns f32 (steps, 6N) rows
        [x|y|z|vx|vy|vz] when snapshots is set."""
        if steps < 1:
            raise ValueError("steps muss >= 1 sein")
        if not st["acc_valid"]:
            self.forces(st, net)
        n = st["n"]
        snap = torch.empty((steps, 6 * n), dtype=torch.float32, device=st["buf"].device) if snapshots else None
        hdt = 0.5 * dt
        self.kick_drift(st, hdt, dt)
        for s in range(steps):
            mode = _lib.PM3_KICK_DRIFT if s < steps - 1 else _lib.PM3_KICK
            row = snap[s] if snap is not None else None
            if net is None:
                self.method_forces(st, mode, hdt, dt, row)
            else:
                self.method_forces(st)
                net_correct(net, self, st, mode, hdt, dt, row)
        return snap.cpu().numpy() if snap is not None else None


def net_correct(net: ShortRangeMLP, pm: PMPeriodic3D, st, mode, hdt, dt, snap) -> None:
    """a += out_scale * MLP(inputs) for every particle, then the epilogue."""
    with torch.cuda.device(net.device):
        net.ctx.check(net.ctx.lib.sss_mlp_correct(
            net.ctx.ptr, pm.ptr, ctypes.byref(st["parts"]), net.params.data_ptr(), net.frags.data_ptr(),
            float(st["rho_mean"]), float(net.out_scale), int(mode), float(hdt), float(dt),
            snap.data_ptr() if snap is not None else None, ctypes.c_void_p(_lib.stream_handle(net.device))))


def median_rel_err(a: torch.Tensor, ref: torch.Tensor) -> float:
    """Median over particles of |a - ref| / |ref| ((3, T) tensors)."""
    e = torch.linalg.vector_norm(a - ref, dim=0) / torch.linalg.vector_norm(ref, dim=0)
    return float(torch.median(e))


class CorrectionJudge:
    """Accept / revert rule of the learned correction.

    The corrected force on fresh particles must stay within `tol` (median
    relative error against the direct sum); tol None means "no worse than
    the mesh force alone on the same particles"."""

    def __init__(self, tol: float | None = None):
        self.tol = tol

    def limit(self, err_mesh: float) -> float:
        return err_mesh if self.tol is None else float(self.tol)

    def accept(self, err_mesh: float, err_corr: float) -> bool:
        return bool(err_corr <= self.limit(err_mesh))


@dataclass
class CheckRecord:
    step: int
    err_mesh: float
    err_corr: float | None
    accepted: bool | None
    reverted: bool
    loss_first: float | None = None
    loss_last: float | None = None
    seconds: dict = field(default_factory=dict)


class NBodyPMLearned:
    """PM + learned correction + direct-sum judge (see the module doc)."""

    def __init__(self, device: int = 0, mesh_n: int = 256, box: float = 1.0, G: float = 1.0,
                 softening: float = 1e-3, check_every: int = 50, samples: int = 16384, tol: float | None = None,
                 iters: int = 200, batch: int = 2048, lr: float = 1e-3, seed: int = 0, fallback: str = "mesh",
                 learned: bool = True, deconv: int = 2, r_split_cells: float = 0.6, short_range: bool = False,
                 x_cut: float = 3.5, window: int = 4):
        if fallback not in ("mesh", "direct"):
            raise ValueError("fallback must be 'mesh' or 'direct'")
        self.pm = PMPeriodic3D(mesh_n, box, G, device, deconv, r_split_cells, short_range, softening, x_cut)
        self.net = ShortRangeMLP(device, seed) if learned else None
        self.ewald = EwaldDirect(box, G, softening, device=device)
        self.judge = CorrectionJudge(tol)
        self.check_every = int(check_every)
        self.samples = int(samples)
        self.iters, self.batch, self.lr = int(iters), int(batch), float(lr)
        self.rng = np.random.default_rng(seed)
        self.fallback = fallback
        self.active = False             # network in use for the force
        self.accepted = None            # snapshot of the last accepted network
        self.window = int(window)       # checks whose samples form the training set
        self.X = None                   # training inputs (rows, 80) bf16 bits
        self.R = None                   # residuals direct - mesh (rows, 3) f64
        self._rows: list[int] = []      # rows contributed by each check in the window
        self.records: list[CheckRecord] = []
        self.steps_done = 0

    def name(self) -> str:
        return self.pm.name() + (" + learned correction" if self.net is not None else "")

    def load_state(self, pos, vel, mass) -> dict:
        st = self.pm.load_state(pos, vel, mass)
        self.steps_done = 0
        return st

    # ---- the pieces of a check
    def _sample(self, st):
        n = st["n"]
        k = min(self.samples, n)
        idx = np.sort(self.rng.choice(n, size=k, replace=False))
        return torch.as_tensor(idx.astype(np.int64)).to(st["buf"].device)

    def _direct(self, st, idx):
        tgt = st["buf"][0:3, idx].contiguous()
        return self.ewald.accel(st["parts"], tgt, idx)

    def _mesh_at(self, st, idx):
        """The force without the network (mesh, and the P3M pair term when
        short_range) of all particles into the state; returns it at idx."""
        self.pm.method_forces(st)
        return st["buf"][6:9, idx].clone()

    def _full_force(self, st):
        """The force the stepper uses, at the current positions (state a)."""
        self.pm.forces(st, self.net if self.active else None)

    def _snapshot_state(self, st):
        return st["buf"].clone()

    def _steps(self, st, dt, k):
        if self.fallback == "direct" and not self.active and self.accepted is None and self._replaying:
            self._direct_steps(st, dt, k)
        else:
            self.pm.step_batch(st, dt, k, self.net if self.active else None)

    def _direct_steps(self, st, dt, k):
        """KDK steps with the Ewald direct sum of every particle as the force."""
        hdt = 0.5 * dt
        allidx = torch.arange(st["n"], device=st["buf"].device)
        for _ in range(k):
            self.pm.kick_drift(st, hdt, dt)
            st["buf"][6:9] = self._direct(st, allidx)
            self.pm.kick_drift(st, hdt, 0.0)

    def check(self, st, dt: float | None = None, block_start=None) -> CheckRecord:
        """Judge the force used since the last check on fresh particles
        (revert and replay the block if it fails), then train on them."""
        t0 = time.perf_counter()
        idx = self._sample(st)
        a_mesh = self._mesh_at(st, idx)
        a_dir = self._direct(st, idx)
        err_mesh = median_rel_err(a_mesh, a_dir)
        err_corr, accepted, reverted = None, None, False
        X = None
        if self.net is not None:
            X = self.net.features(self.pm, st["parts"], idx, st["rho_mean"])
        if self.active:
            y = self.net.forward(X).double().T * self.net.out_scale
            err_corr = median_rel_err(a_mesh + y, a_dir)
            accepted = self.judge.accept(err_mesh, err_corr)
            if accepted:
                self.accepted = self.net.snapshot()
            elif block_start is not None:
                # revert the block and replay it with the last accepted network
                # (or the fallback force), then sample afresh at the new positions
                reverted = True
                buf0, k = block_start
                st["buf"].copy_(buf0)
                if self.accepted is not None:
                    self.net.restore(self.accepted)
                else:
                    self.active = False
                self._replaying = True
                self._full_force(st)
                self._steps(st, dt, k)
                self._replaying = False
                idx = self._sample(st)
                a_mesh = self._mesh_at(st, idx)
                a_dir = self._direct(st, idx)
                err_mesh = median_rel_err(a_mesh, a_dir)
                X = self.net.features(self.pm, st["parts"], idx, st["rho_mean"])
        t1 = time.perf_counter()
        rec = CheckRecord(self.steps_done, err_mesh, err_corr, accepted, reverted)
        if self.net is not None:
            # training set: the samples of the last `window` checks; targets in
            # units of their current rms (the residuals grow as halos collapse),
            # the output layer rescaled so the network's force is unchanged
            R = (a_dir - a_mesh).T.contiguous()
            if self.X is None:
                self.X, self.R = X, R
            else:
                self.X = torch.cat([self.X, X])
                self.R = torch.cat([self.R, R])
            self._rows.append(int(R.shape[0]))
            if len(self._rows) > self.window:
                drop = self._rows.pop(0)
                self.X, self.R = self.X[drop:], self.R[drop:]
            scale = float(torch.sqrt(torch.mean(self.R * self.R)))
            if len(self._rows) > 1 and scale > 0.0:
                self.net.rescale_output(self.net.out_scale / scale)
            self.net.out_scale = scale
            T = (self.R / scale).float()
            losses = self.net.train(self.X, T, self.iters, self.batch, self.lr, self.rng)
            rec.loss_first, rec.loss_last = losses[0], losses[-1]
            self.active = True
        self._full_force(st)
        torch.cuda.synchronize(self.pm.device)
        rec.seconds = {"judge": t1 - t0, "train": time.perf_counter() - t1}
        self.records.append(rec)
        return rec

    _replaying = False

    def run(self, st, dt: float, steps: int) -> list[CheckRecord]:
        """`steps` KDK steps with a check (judge + training) at the start and
        after every `check_every` steps."""
        self.check(st, dt)
        done = 0
        while done < steps:
            k = min(self.check_every, steps - done)
            start = (self._snapshot_state(st), k)
            self._steps(st, dt, k)
            done += k
            self.steps_done += k
            self.check(st, dt, block_start=start)
        return self.records
