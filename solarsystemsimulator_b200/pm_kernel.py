"""Particle-mesh gravity on one B200: drop-in for backend/pm_kernel.py.

2-D isolated PM of the reference (Hockney-James zero padding, convolution
with the softened 3-D force kernel in the plane, cloud-in-cell deposit and
gather, adaptive grid geometry, KDK):

    sim = NBodyPM(devices, softening_au=0.0, kraft_f32=True, grid_n=4096,
                  softening_zellen=1.5, rand_zellen=4.0)
    st = sim.load_state(x, y, vx, vy, mass, tracer=(tx, ty, tvx, tvy))
    out = sim.step_batch(st, dt, steps)     # f32 (steps, 4N+2T)
    f64 = sim.export_f64(st)

and the module functions build_force_kernels, grid_fuer, pm_force_field,
gather_accel, pm_accelerations, _cic_deposit, _cic_gather on CUDA tensors.
The work runs in libsss (sss_pm2d_*); cuFFT does the transforms only.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib

G_AU = 4 * np.pi * np.pi


def _f64(a, dev) -> torch.Tensor:
    if isinstance(a, torch.Tensor):
        return a.to(device=dev, dtype=torch.float64).contiguous()
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64)).to(dev)


class PMPlan:
    """cuFFT plans and grids of one grid size (an sss_pm2d object)."""

    def __init__(self, grid_n: int, device: int = 0):
        self.ctx = _lib.context(device)
        self.device = device
        self.grid_n = int(grid_n)
        ptr = ctypes.c_void_p()
        with torch.cuda.device(device):
            self.ctx.check(self.ctx.lib.sss_pm2d_create(self.ctx.ptr, self.grid_n, ctypes.byref(ptr)))
        self.ptr = ptr
        self.kernel_key = None

    def __del__(self):
        try:
            if getattr(self, "ptr", None):
                self.ctx.lib.sss_pm2d_destroy(self.ptr)
                self.ptr = None
        except Exception:
            pass

    def _s(self):
        return ctypes.c_void_p(_lib.stream_handle(self.device))

    def call(self, name, *args):
        with torch.cuda.device(self.device):
            self.ctx.check(getattr(self.ctx.lib, name)(self.ptr, *args, self._s()))


_plans: dict[tuple[int, int], PMPlan] = {}


def plan_for(grid_n: int, device: int = 0) -> PMPlan:
    key = (int(device), int(grid_n))
    if key not in _plans:
        _plans[key] = PMPlan(grid_n, device)
    return _plans[key]


def grid_fuer(gx, gy, grid_n: int, rand_zellen: float = 3.0, device: int = 0):
    """Origin (x0, y0) and cell size h so that all points fit with
    `rand_zellen` cells of margin (pm_kernel.py:110-124). The bounding box is
    reduced on the device; one 32-byte read returns it."""
    dev = torch.device("cuda", device)
    x, y = _f64(gx, dev), _f64(gy, dev)
    p = plan_for(grid_n, device)
    bb = torch.empty(4, dtype=torch.float64, device=dev)
    p.call("sss_pm2d_bbox", x.data_ptr(), y.data_ptr(), x.numel(), bb.data_ptr())
    xmin, xmax, ymin, ymax = bb.cpu().tolist()
    spanne = max(xmax - xmin, ymax - ymin, 1e-30)
    h = spanne / (grid_n - 2 * rand_zellen)
    return xmin - rand_zellen * h, ymin - rand_zellen * h, h


class ForceKernels:
    """Handle for the transforms of K_x, K_y held by a plan (build_force_kernels)."""

    def __init__(self, plan: PMPlan, h: float, eps2: float, G: float):
        self.plan, self.key = plan, (float(h), float(eps2), float(G))


def build_force_kernels(grid_n: int, h: float, eps2: float, G: float = G_AU, device: int = 0) -> ForceKernels:
    """Transforms of the softened force kernels on the 2N x 2N padded grid
    (pm_kernel.py:34-60), kept on the device."""
    p = plan_for(grid_n, device)
    if p.kernel_key != (float(h), float(eps2), float(G)):
        p.call("sss_pm2d_build_kernels", float(h), float(eps2), float(G))
        p.kernel_key = (float(h), float(eps2), float(G))
    return ForceKernels(p, h, eps2, G)


def pm_force_field(gx, gy, gm, grid_n, x0, y0, h, eps2, G: float = G_AU, kernels=None, device: int = 0):
    """The acceleration field on the N x N grid (pm_kernel.py:127-147).
    Returns (ax_grid, ay_grid) as (N, N) float64 CUDA tensors."""
    dev = torch.device("cuda", device)
    p = plan_for(grid_n, device)
    if kernels is None or kernels.plan is not p or p.kernel_key != kernels.key:
        kernels = build_force_kernels(grid_n, h, eps2, G, device)
    x, y, m = _f64(gx, dev), _f64(gy, dev), _f64(gm, dev)
    p.call("sss_pm2d_field", x.data_ptr(), y.data_ptr(), m.data_ptr(), x.numel(), float(x0), float(y0), float(h))
    return _crop_fields(p, dev)


def _crop_fields(p: PMPlan, dev):
    n = p.grid_n
    ax = torch.empty((n, n), dtype=torch.float64, device=dev)
    ay = torch.empty((n, n), dtype=torch.float64, device=dev)
    p.call("sss_pm2d_fields", ax.data_ptr(), ay.data_ptr())
    return ax, ay


def gather_accel(ax_grid, ay_grid, px, py, grid_n, x0, y0, h, device: int = 0):
    """Field read at (px, py) from the plan's last field (pm_kernel.py:150-154).
    ax_grid/ay_grid must be the fields pm_force_field returned last."""
    dev = torch.device("cuda", device)
    p = plan_for(grid_n, device)
    x, y = _f64(px, dev), _f64(py, dev)
    ax = torch.empty_like(x)
    ay = torch.empty_like(x)
    p.call("sss_pm2d_gather", x.data_ptr(), y.data_ptr(), x.numel(), float(x0), float(y0), float(h),
           ax.data_ptr(), ay.data_ptr())
    return ax, ay


def _cic_gather(feld, gx, gy, grid_n, x0, y0, h, device: int = 0):
    """The value of the (grid_n, grid_n) field `feld` at (gx, gy) with the
    deposit's bilinear stencil (pm_kernel.py:93-107). Returns an f64 device
    tensor."""
    dev = torch.device("cuda", device)
    f = _f64(feld, dev)
    if f.dim() != 2 or f.shape[0] != grid_n or f.shape[1] != grid_n:
        raise ValueError(f"feld must be ({grid_n}, {grid_n})")
    x, y = _f64(gx, dev), _f64(gy, dev)
    if x.numel() != y.numel():
        raise ValueError("gx and gy must have the same length")
    out = torch.empty_like(x)
    ctx = _lib.context(device)
    with torch.cuda.device(device):
        ctx.check(ctx.lib.sss_pm2d_gather_field(ctx.ptr, f.data_ptr(), int(grid_n), f.stride(0), x.data_ptr(),
                                                y.data_ptr(), x.numel(), float(x0), float(y0), float(h),
                                                out.data_ptr(), ctypes.c_void_p(_lib.stream_handle(device))))
    return out


def pm_accelerations(gx, gy, gm, grid_n, x0, y0, h, eps2, G: float = G_AU, kernels=None, device: int = 0):
    """Acceleration of each mass via PM (pm_kernel.py:157-163)."""
    dev = torch.device("cuda", device)
    p = plan_for(grid_n, device)
    if kernels is None or kernels.plan is not p or p.kernel_key != kernels.key:
        build_force_kernels(grid_n, h, eps2, G, device)
    x, y, m = _f64(gx, dev), _f64(gy, dev), _f64(gm, dev)
    p.call("sss_pm2d_field", x.data_ptr(), y.data_ptr(), m.data_ptr(), x.numel(), float(x0), float(y0), float(h))
    ax, ay = torch.empty_like(x), torch.empty_like(x)
    p.call("sss_pm2d_gather", x.data_ptr(), y.data_ptr(), x.numel(), float(x0), float(y0), float(h),
           ax.data_ptr(), ay.data_ptr())
    return ax, ay


def _cic_deposit(gx, gy, gm, grid_n, x0, y0, h, device: int = 0):
    """Cloud-in-cell mass grid (N, N) (pm_kernel.py:63-90)."""
    dev = torch.device("cuda", device)
    p = plan_for(grid_n, device)
    if p.kernel_key is None:
        build_force_kernels(grid_n, h, (2 * h) ** 2, G_AU, device)
    x, y, m = _f64(gx, dev), _f64(gy, dev), _f64(gm, dev)
    p.call("sss_pm2d_field", x.data_ptr(), y.data_ptr(), m.data_ptr(), x.numel(), float(x0), float(y0), float(h))
    rho = torch.empty((grid_n, grid_n), dtype=torch.float64, device=dev)
    p.call("sss_pm2d_density", rho.data_ptr())
    return rho


class NBodyPM:
    """Self-gravitating bodies via particle-mesh on ONE card (pm_kernel.py:166-293)."""

    def __init__(self, devices, softening_au: float = 0.0, kraft_f32: bool = True, grid_n: int = 4096,
                 softening_zellen: float = 1.5, rand_zellen: float = 4.0, *, G: float = G_AU):
        if isinstance(devices, int):
            devices = [devices]
        self.device = int(devices[0])
        self.devices = [self.device]
        self.grid_n = int(grid_n)
        self.softening_zellen = float(softening_zellen)
        self.rand_zellen = float(rand_zellen)
        self.softening_floor = float(softening_au)
        self.kraft_f32 = bool(kraft_f32)
        self.G = float(G)
        self._plan = plan_for(self.grid_n, self.device)
        self._kernel_h = None

    def name(self) -> str:
        return torch.cuda.get_device_name(self.device) + " (PM)"

    def _accel_into(self, st):
        """Field from the masses, read at masses and tracers (pm_kernel.py:212-229)."""
        p = self._plan
        x0, y0, h = grid_fuer(st["x"], st["y"], self.grid_n, self.rand_zellen, self.device)
        eps = max(self.softening_zellen * h, self.softening_floor)
        eps2 = eps * eps
        if self._kernel_h is None or abs(h - self._kernel_h) > 1e-6 * h:
            p.call("sss_pm2d_build_kernels", float(h), float(eps2), self.G)
            p.kernel_key = (float(h), float(eps2), self.G)
            self._kernel_h = h
        x, y, m = st["x"], st["y"], st["m"]
        p.call("sss_pm2d_field", x.data_ptr(), y.data_ptr(), m.data_ptr(), st["N"], x0, y0, h)
        p.call("sss_pm2d_gather", x.data_ptr(), y.data_ptr(), st["N"], x0, y0, h, st["ax"].data_ptr(),
               st["ay"].data_ptr())
        if st["T"]:
            p.call("sss_pm2d_gather", st["tx"].data_ptr(), st["ty"].data_ptr(), st["T"], x0, y0, h,
                   st["tax"].data_ptr(), st["tay"].data_ptr())

    def load_state(self, x, y, vx, vy, mass, *_egal, tracer=None, **_auch_egal) -> dict:
        dev = torch.device("cuda", self.device)
        st = {"x": _f64(x, dev), "y": _f64(y, dev), "vx": _f64(vx, dev), "vy": _f64(vy, dev),
              "m": _f64(mass, dev), "N": len(x)}
        st["ax"] = torch.zeros_like(st["x"])
        st["ay"] = torch.zeros_like(st["x"])
        if tracer is not None and len(tracer[0]):
            st["tx"], st["ty"] = _f64(tracer[0], dev), _f64(tracer[1], dev)
            st["tvx"], st["tvy"] = _f64(tracer[2], dev), _f64(tracer[3], dev)
            st["T"] = len(tracer[0])
            st["tax"] = torch.zeros_like(st["tx"])
            st["tay"] = torch.zeros_like(st["tx"])
        else:
            st["tx"] = st["ty"] = st["tvx"] = st["tvy"] = None
            st["T"] = 0
        self._accel_into(st)
        return st

    def step_batch(self, st: dict, dt_years: float, steps: int) -> np.ndarray:
        """`steps` KDK steps; f32 (steps, 4N+2T) [x|y|vx|vy | tx|ty] (pm_kernel.py:246-280)."""
        if steps < 1:
            raise ValueError(f"steps muss >= 1 sein: {steps}")
        n, t = st["N"], st["T"]
        dt = float(dt_years)
        hdt = 0.5 * dt
        p = self._plan
        dev = torch.device("cuda", self.device)
        snap = torch.empty((steps, 4 * n + 2 * t), dtype=torch.float32, device=dev)

        def kd(xk, yk, vxk, vyk, axk, ayk, cnt, drift):
            p.call("sss_pm2d_kick_drift", st[xk].data_ptr(), st[yk].data_ptr(), st[vxk].data_ptr(),
                   st[vyk].data_ptr(), st[axk].data_ptr(), st[ayk].data_ptr(), cnt, hdt, dt, drift)

        for s in range(steps):
            kd("x", "y", "vx", "vy", "ax", "ay", n, 1)
            if t:
                kd("tx", "ty", "tvx", "tvy", "tax", "tay", t, 1)
            self._accel_into(st)
            kd("x", "y", "vx", "vy", "ax", "ay", n, 0)
            if t:
                kd("tx", "ty", "tvx", "tvy", "tax", "tay", t, 0)
            row = snap[s]
            for k, key in enumerate(("x", "y", "vx", "vy")):
                p.call("sss_pm2d_to_f32", st[key].data_ptr(), n, row[k * n:(k + 1) * n].data_ptr())
            if t:
                p.call("sss_pm2d_to_f32", st["tx"].data_ptr(), t, row[4 * n:4 * n + t].data_ptr())
                p.call("sss_pm2d_to_f32", st["ty"].data_ptr(), t, row[4 * n + t:].data_ptr())
        return snap.cpu().numpy()

    def export_f64(self, st: dict) -> np.ndarray:
        """Exact f64 state [x|y|vx|vy] (4N) of the masses (pm_kernel.py:282-293)."""
        return torch.cat([st["x"], st["y"], st["vx"], st["vy"]]).cpu().numpy().astype("<f8")
