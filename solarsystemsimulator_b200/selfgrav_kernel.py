"""Self-gravitating bodies on one B200: tiled all-pairs Plummer gravity.

Drop-in for the reference's `backend/selfgrav_kernel.py` (Kernel A: massive
bodies, Kernel B: massless tracers). Same call surface:

    sim = NBodySelfGrav(devices, softening_au, kraft_f32=True)
    st = sim.load_state(x, y, vx, vy, mass, tracer=(tx, ty, tvx, tvy))
    out = sim.step_batch(st, dt, steps)   # f32 (steps, 4N + 2T)
    f64 = sim.export_f64(st)              # '<f8' (4N,) [x|y|vx|vy]

Additive keyword arguments (absent in the reference): `G` (default G_AU, the
reference's AU/year/Msun constant), `integrator` ("kdk" = the reference's
leapfrog, "yoshida4"), `precision` ("f64", "mixed" or "mixed_tc", the
mixed pair terms formed on the tensor cores; by default kraft_f32=True
selects "mixed", kraft_f32=False "f64"), and for 3-D states
`z=`, `vz=` in load_state plus `tracer_z=(tz, tvz)`. With z given the
snapshot rows are [x|y|z|vx|vy|vz | tx|ty|tz] (6N + 3T).

The state stays resident in HBM as torch tensors between calls; the work is
done by libsss (include/sss.h) — there is no CPU path.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib

BLOCK = 256                       # reference tile width (selfgrav_kernel.py:75)
G_AU = 4 * np.pi * np.pi          # AU^3 / (Msun yr^2), nbody_kernel.py:60
G_MAX = 8                         # reference multi-GPU limit (gpu_verbund.py:30)

_INTEGRATORS = {"kdk": _lib.INT_KDK, "leapfrog": _lib.INT_KDK,
                "yoshida4": _lib.INT_YOSHIDA4, "yoshida": _lib.INT_YOSHIDA4}
_PRECISIONS = {"f64": _lib.PREC_F64, "mixed": _lib.PREC_MIXED, "mixed_tc": _lib.PREC_MIXED_TC}


def _dev(device: int) -> torch.device:
    return torch.device("cuda", int(device))


def pack_bodies(x, y, z, gm, device) -> torch.Tensor:
    """(n, 4) float64 device tensor of {x, y, z, Gm} records."""
    n = len(x)
    h = np.empty((n, 4), np.float64)
    h[:, 0] = np.asarray(x, np.float64)
    h[:, 1] = np.asarray(y, np.float64)
    h[:, 2] = 0.0 if z is None else np.asarray(z, np.float64)
    h[:, 3] = 0.0 if gm is None else np.asarray(gm, np.float64)
    return torch.from_numpy(h).to(_dev(device))


def allpairs_accel(src4: torch.Tensor, tgt4: torch.Tensor, eps2: float, dim: int = 3,
                   precision: str = "f64", out: torch.Tensor | None = None) -> torch.Tensor:
    """a_t = sum_s Gm_s (r_s - r_t)/(|r_s - r_t|^2 + eps2)^1.5 on the GPU.

    src4, tgt4: contiguous (n, 4) float64 CUDA tensors {x, y, z, Gm}.
    Returns (n_tgt, 4) float64 {ax, ay, az, 0}. Same formula as the
    reference's `beschleunigung` (selfgrav_kernel.py:222-260)."""
    for t in (src4, tgt4):
        if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous() and t.dim() == 2
                and t.shape[1] == 4):
            raise ValueError("bodies must be contiguous (n, 4) float64 CUDA tensors")
    dev = src4.device.index
    if out is None:
        out = torch.empty((tgt4.shape[0], 4), dtype=torch.float64, device=src4.device)
    ctx = _lib.context(dev)
    rc = ctx.lib.sss_allpairs_accel(ctx.ptr, int(dim), _PRECISIONS[precision], src4.data_ptr(),
                                    src4.shape[0], tgt4.data_ptr(), tgt4.shape[0], out.data_ptr(),
                                    float(eps2), ctypes.c_void_p(_lib.stream_handle(dev)))
    ctx.check(rc)
    return out


def allpairs_potential(src4: torch.Tensor, tgt4: torch.Tensor, eps2: float, dim: int = 3,
                       out: torch.Tensor | None = None) -> torch.Tensor:
    """phi_t = -sum_s Gm_s / sqrt(|d|^2 + eps2) (self term included), f64."""
    dev = src4.device.index
    if out is None:
        out = torch.empty((tgt4.shape[0],), dtype=torch.float64, device=src4.device)
    ctx = _lib.context(dev)
    rc = ctx.lib.sss_allpairs_potential(ctx.ptr, int(dim), src4.data_ptr(), src4.shape[0],
                                        tgt4.data_ptr(), tgt4.shape[0], out.data_ptr(),
                                        float(eps2), ctypes.c_void_p(_lib.stream_handle(dev)))
    ctx.check(rc)
    return out


def segmentiere(n: int, gewichte: list[float]) -> list[tuple[int, int]]:
    """Split n bodies into contiguous segments proportional to `gewichte`.

    Same contract as the reference (selfgrav_kernel.py:156-178): gap-free,
    non-overlapping, covering [0, n), one (start, length) per weight; bounds
    kept monotone when n is tiny."""
    ges = float(sum(gewichte))
    grenzen = [0]
    lauf = 0.0
    for w in gewichte[:-1]:
        lauf += w
        grenzen.append(int(round(n * lauf / ges)))
    grenzen.append(n)
    for i in range(1, len(grenzen)):
        grenzen[i] = max(grenzen[i], grenzen[i - 1])
    return [(grenzen[i], grenzen[i + 1] - grenzen[i]) for i in range(len(gewichte))]


def waehle_karten(kraft_f32: bool = True, mindest_anteil: float = 0.25) -> list[int]:
    """Devices for the self-gravity kernel. One GPU per process here: [0]."""
    if not torch.cuda.is_available():
        raise RuntimeError("no CUDA device")
    return [torch.cuda.current_device()]


def miss_gewicht(device: int, kraft_f32: bool = True) -> float:
    """Relative device weight; a single-device build weighs every card 1."""
    return 1.0


class NBodySelfGrav:
    """Self-gravitating bodies (+ massless tracers) resident on one GPU."""

    def __init__(self, devices, softening_au: float, kraft_f32: bool = True, *,
                 G: float = G_AU, integrator: str = "kdk", precision: str | None = None):
        if isinstance(devices, int):
            devices = [devices]
        if not devices or len(devices) > G_MAX:
            raise ValueError(f"1..{G_MAX} Devices erwartet: {devices}")
        if not softening_au > 0:
            raise ValueError(f"Softening muss positiv sein: {softening_au}")
        if len(devices) > 1:
            raise ValueError("this build runs on one GPU; pass a single device")
        if integrator not in _INTEGRATORS:
            raise ValueError(f"unknown integrator {integrator!r}")
        if precision is None:
            precision = "mixed" if kraft_f32 else "f64"
        if precision not in _PRECISIONS:
            raise ValueError(f"unknown precision {precision!r}")
        self.devices = [int(devices[0])]
        self.device = self.devices[0]
        self.eps2 = float(softening_au) ** 2
        self.kraft_f32 = bool(kraft_f32)
        self.G = float(G)
        self.integrator = integrator
        self.precision = precision
        self._ctx = _lib.context(self.device)

    def name(self) -> str:
        return torch.cuda.get_device_name(self.device)

    # ------------------------------------------------------------ state
    def load_state(self, x, y, vx, vy, mass, *_egal, tracer=None, z=None, vz=None,
                   tracer_z=None, **_auch_egal) -> dict:
        """Take over the full state; it stays resident on the GPU.

        Extra positional arguments of `NBodyCuda.load_state` (visibility,
        asteroid flags, radii) are accepted and ignored, as in the reference
        (selfgrav_kernel.py:467-481)."""
        n = len(x)
        if n < 1:
            raise ValueError("leerer Zustand")
        dim = 3 if z is not None else 2
        T = 0
        if tracer is not None and len(tracer[0]):
            T = len(tracer[0])
        dev = _dev(self.device)
        h = np.zeros((n + T, 4), np.float64)
        hv = np.zeros((n + T, 4), np.float64)
        h[:n, 0] = np.asarray(x, np.float64)
        h[:n, 1] = np.asarray(y, np.float64)
        hv[:n, 0] = np.asarray(vx, np.float64)
        hv[:n, 1] = np.asarray(vy, np.float64)
        if dim == 3:
            h[:n, 2] = np.asarray(z, np.float64)
            hv[:n, 2] = 0.0 if vz is None else np.asarray(vz, np.float64)
        h[:n, 3] = self.G * np.asarray(mass, np.float64)
        if T:
            h[n:, 0] = np.asarray(tracer[0], np.float64)
            h[n:, 1] = np.asarray(tracer[1], np.float64)
            hv[n:, 0] = np.asarray(tracer[2], np.float64)
            hv[n:, 1] = np.asarray(tracer[3], np.float64)
            if dim == 3 and tracer_z is not None:
                h[n:, 2] = np.asarray(tracer_z[0], np.float64)
                hv[n:, 2] = np.asarray(tracer_z[1], np.float64)
        pos = torch.empty((2, n + T, 4), dtype=torch.float64, device=dev)
        pos[0].copy_(torch.from_numpy(h))
        pos[1].copy_(pos[0])
        vel = torch.from_numpy(hv).to(dev)
        acc = torch.zeros((n + T, 4), dtype=torch.float64, device=dev)
        cs = _lib.SelfGravState()
        cs.dim = dim
        cs.precision = _PRECISIONS[self.precision]
        cs.n_src = n
        cs.n_tracer = T
        cs.pos4[0] = pos[0].data_ptr()
        cs.pos4[1] = pos[1].data_ptr()
        cs.vel4 = vel.data_ptr()
        cs.acc4 = acc.data_ptr()
        cs.cur = 0
        cs.eps2 = self.eps2
        st = {"N": n, "T": T, "dim": dim, "pos": pos, "vel": vel, "acc": acc, "c": cs,
              "snap": None, "host": None, "mass": np.asarray(mass, np.float64).copy()}
        self._call(self._ctx.lib.sss_selfgrav_init_accel, ctypes.byref(cs))
        return st

    def _call(self, fn, *args):
        stream = _lib.stream_handle(self.device)
        with torch.cuda.device(self.device):
            rc = fn(self._ctx.ptr, *args, ctypes.c_void_p(stream))
        self._ctx.check(rc)

    def row_width(self, st: dict) -> int:
        d = st["dim"]
        return 2 * d * st["N"] + d * st["T"]

    def step_batch_device(self, st: dict, dt_years: float, steps: int,
                          snapshots: bool = True) -> torch.Tensor | None:
        """Advance `steps` steps; snapshots stay on the device (or none)."""
        if st is None:
            raise ValueError("kein Zustand geladen")
        if steps < 1:
            raise ValueError(f"steps muss >= 1 sein: {steps}")
        snap = None
        if snapshots:
            need = steps * self.row_width(st)
            buf = st["snap"]
            if buf is None or buf.numel() < need:
                buf = torch.empty(need, dtype=torch.float32, device=_dev(self.device))
                st["snap"] = buf
            snap = buf[:need].view(steps, self.row_width(st))
        self._call(self._ctx.lib.sss_selfgrav_step_batch, ctypes.byref(st["c"]),
                   _INTEGRATORS[self.integrator], float(dt_years), int(steps),
                   ctypes.c_void_p(snap.data_ptr() if snap is not None else 0))
        return snap

    def step_batch(self, st: dict, dt_years: float, steps: int) -> np.ndarray:
        """`steps` integrator steps; f32 (steps, 4N+2T) [x|y|vx|vy|tx|ty] in
        original order (selfgrav_kernel.py:558-627)."""
        snap = self.step_batch_device(st, dt_years, steps, snapshots=True)
        host = st["host"]
        if host is None or host.numel() < snap.numel():
            host = torch.empty(snap.numel(), dtype=torch.float32, pin_memory=True)
            st["host"] = host
        h = host[:snap.numel()].view(snap.shape)
        h.copy_(snap, non_blocking=True)
        torch.cuda.current_stream(self.device).synchronize()
        self._ctx.status(_lib.stream_handle(self.device))
        return h.numpy().copy()

    def export_f64(self, st: dict) -> np.ndarray:
        """Exact f64 state [x|y|(z)|vx|vy|(vz)] of the massive bodies."""
        n, d = st["N"], st["dim"]
        pos = st["pos"][st["c"].cur][:n, :d].cpu().numpy()
        vel = st["vel"][:n, :d].cpu().numpy()
        out = np.empty(2 * d * n, dtype="<f8")
        for k in range(d):
            out[k * n:(k + 1) * n] = pos[:, k]
            out[(d + k) * n:(d + k + 1) * n] = vel[:, k]
        return out

    def export_tracers_f64(self, st: dict) -> np.ndarray:
        """f64 tracer state [tx|ty|(tz)|tvx|tvy|(tvz)] (additive API)."""
        n, t, d = st["N"], st["T"], st["dim"]
        pos = st["pos"][st["c"].cur][n:n + t, :d].cpu().numpy()
        vel = st["vel"][n:n + t, :d].cpu().numpy()
        out = np.empty(2 * d * t, dtype="<f8")
        for k in range(d):
            out[k * t:(k + 1) * t] = pos[:, k]
            out[(d + k) * t:(d + k + 1) * t] = vel[:, k]
        return out

    def accelerations(self, st: dict) -> np.ndarray:
        """Current accelerations (n+T, dim) f64 (additive API)."""
        return st["acc"][:, :st["dim"]].cpu().numpy()

    def energy(self, st: dict) -> float:
        """Total energy of the massive bodies (kinetic + Plummer potential,
        self terms removed) in f64 on the GPU, as test_selfgrav.energie."""
        n, d = st["N"], st["dim"]
        pos = st["pos"][st["c"].cur][:n].contiguous()
        m = torch.from_numpy(st["mass"]).to(pos.device)
        phi = allpairs_potential(pos, pos, self.eps2, dim=d)
        v = st["vel"][:n, :d]
        kin = 0.5 * float((m * (v * v).sum(1)).sum())
        # phi_i includes the self term -G m_i / eps; remove it
        pot = 0.5 * float((m * phi).sum()) + 0.5 * self.G * float((m * m).sum()) / np.sqrt(self.eps2)
        return kin + pot
