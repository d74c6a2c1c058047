"""f64 Ewald direct sum on one B200: the exact periodic force of point masses
(Plummer-softened on the nearest image) at chosen target positions.

It is the judge of the 3-D mesh force and the source of the training
targets of the learned correction (the role the all-pairs reference sum
plays for the reference's mesh code, test_selfgrav.py:66-88, made
periodic). The defaults (alpha = 10 / box, r_cut = 0.46 box, |h| <= 17)
truncate both sums below 1e-9 of the force.

    ew = EwaldDirect(box=1.0, G=1.0, softening=1e-3)
    a = ew.accel(src_particles, targets, self_idx)   # torch f64 (3, T)
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib


def hvectors(h_max: int) -> np.ndarray:
    """Half-space integer vectors 0 < |h| <= h_max (one of each +-h pair),
    int32 (nk, 3)."""
    r = np.arange(-h_max, h_max + 1)
    hx, hy, hz = np.meshgrid(r, r, r, indexing="ij")
    h = np.stack([hx.ravel(), hy.ravel(), hz.ravel()], 1)
    h2 = (h * h).sum(1)
    half = (h[:, 0] > 0) | ((h[:, 0] == 0) & (h[:, 1] > 0)) | ((h[:, 0] == 0) & (h[:, 1] == 0) & (h[:, 2] > 0))
    return h[half & (h2 <= h_max * h_max)].astype(np.int32)


class EwaldDirect:
    def __init__(self, box: float = 1.0, G: float = 1.0, softening: float = 0.0, alpha: float | None = None,
                 r_cut: float | None = None, h_max: int | None = None, device: int = 0):
        self.box = float(box)
        self.G = float(G)
        self.eps2 = float(softening) ** 2
        self.alpha = float(alpha) if alpha is not None else 10.0 / self.box
        self.r_cut = float(r_cut) if r_cut is not None else min(4.6 / self.alpha, 0.5 * self.box)
        if h_max is None:
            h_max = int(math.ceil(5.3 * self.alpha * self.box / math.pi))
        self.h_max = int(h_max)
        self.device = int(device)
        self.ctx = _lib.context(device)
        h = hvectors(self.h_max)
        k2 = ((2.0 * np.pi / self.box) ** 2) * (h.astype(np.float64) ** 2).sum(1)
        coef = 2.0 * 4.0 * np.pi / self.box ** 3 * np.exp(-k2 / (4.0 * self.alpha ** 2)) / k2
        dev = torch.device("cuda", self.device)
        self.nk = len(h)
        self.hvec = torch.as_tensor(h.ravel()).to(dev)
        self.coef = torch.as_tensor(coef).to(dev)
        self.sc = torch.empty(2 * self.nk, dtype=torch.float64, device=dev)

    def _s(self):
        return ctypes.c_void_p(_lib.stream_handle(self.device))

    def structure(self, parts: "_lib.Pm3Particles") -> None:
        """Structure factors of the sources (kept for accel calls)."""
        with torch.cuda.device(self.device):
            self.ctx.check(self.ctx.lib.sss_ewald_structure(
                self.ctx.ptr, ctypes.byref(parts), self.box, self.hvec.data_ptr(), self.nk, self.h_max,
                self.sc.data_ptr(), self._s()))

    def accel(self, parts: "_lib.Pm3Particles", targets: torch.Tensor, self_idx: torch.Tensor | None = None,
              structure: bool = True) -> torch.Tensor:
        """Accelerations (3, T) f64 at targets (3, T) f64 (device tensors).
        self_idx (int64, T): the source index each target is, skipped."""
        if structure:
            self.structure(parts)
        t = targets.contiguous()
        T = t.shape[1]
        out = torch.empty((3, T), dtype=torch.float64, device=t.device)
        tp = (_lib._dp * 3)(t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr())
        op = (_lib._dp * 3)(out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr())
        si = self_idx.contiguous() if self_idx is not None else None
        with torch.cuda.device(self.device):
            self.ctx.check(self.ctx.lib.sss_ewald_accel(
                self.ctx.ptr, ctypes.byref(parts), tp, si.data_ptr() if si is not None else None, T, self.G,
                self.box, self.alpha, self.r_cut, self.eps2, self.hvec.data_ptr(), self.coef.data_ptr(),
                self.sc.data_ptr(), self.nk, op, self._s()))
        return out
