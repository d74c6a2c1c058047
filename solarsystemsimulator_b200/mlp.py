"""The learned short-range correction of the 3-D mesh force: a per-particle
MLP 67 -> 128 -> 128 -> 3 (SiLU) with bf16 weights on the tensor cores
(tcgen05, f32 accumulators in tensor memory), trained online by the
library's own forward, backward and weight-gradient kernels (sss_mlp_*).

    net = ShortRangeMLP(device=0, seed=0)
    X = net.features(pm, parts, idx, rho_mean)    # uint16 (rows, 80) bf16 bits
    Y = net.forward(X)                            # f32 (rows, 3)
    g, loss = net.grad(X, T)                      # f32 (N_PARAMS,), float
    net.adam_step(g, lr)

Inputs: log1p(rho / rho_mean) on the 4x4x4 mesh cells around the particle's
cell and its sub-cell offset - 1/2. Output: the correction in units of
`out_scale` (set from the first training targets).
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib

N_IN = 67
K1 = _lib.MLP_IN_PAD
HID = 128
K3 = 8
SHAPES = (("W1", (K1, HID)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)),
          ("W3", (HID, K3)), ("b3", (K3,)))


def init_params(seed: int = 0) -> np.ndarray:
    """He-style uniform initial parameters (f32, flat layout of sss.h);
    padded rows of W1 and columns of W3 are zero (and stay zero: their
    gradients vanish)."""
    rng = np.random.default_rng(seed)
    w1 = np.zeros((K1, HID))
    w1[:N_IN] = rng.uniform(-1, 1, (N_IN, HID)) * math.sqrt(6.0 / N_IN)
    w2 = rng.uniform(-1, 1, (HID, HID)) * math.sqrt(6.0 / HID)
    w3 = np.zeros((HID, K3))
    w3[:, :3] = rng.uniform(-1, 1, (HID, 3)) * math.sqrt(1.0 / HID)
    flat = np.concatenate([w1.ravel(), np.zeros(HID), w2.ravel(), np.zeros(HID), w3.ravel(), np.zeros(K3)])
    assert flat.size == _lib.MLP_N_PARAMS
    return flat.astype(np.float32)


class ShortRangeMLP:
    def __init__(self, device: int = 0, seed: int = 0, params: np.ndarray | None = None):
        self.device = int(device)
        self.ctx = _lib.context(device)
        dev = torch.device("cuda", self.device)
        p = init_params(seed) if params is None else np.asarray(params, np.float32)
        self.params = torch.as_tensor(p.copy()).to(dev)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.frags = torch.empty(_lib.MLP_N_FRAGS, dtype=torch.int32, device=dev)
        self.grads = torch.empty_like(self.params)
        self.loss_dev = torch.zeros(1, dtype=torch.float32, device=dev)
        self.t = 0
        self.out_scale = 1.0
        self.pack()

    def _s(self):
        return ctypes.c_void_p(_lib.stream_handle(self.device))

    def _call(self, name, *args):
        with torch.cuda.device(self.device):
            self.ctx.check(getattr(self.ctx.lib, name)(self.ctx.ptr, *args, self._s()))

    # ---- state
    def pack(self) -> None:
        """Rebuild the bf16 operand images from the f32 parameters."""
        self._call("sss_mlp_pack", self.params.data_ptr(), self.frags.data_ptr())

    def snapshot(self) -> dict:
        return {"params": self.params.clone(), "m": self.m.clone(), "v": self.v.clone(), "t": self.t,
                "out_scale": self.out_scale}

    def restore(self, snap: dict) -> None:
        self.params.copy_(snap["params"])
        self.m.copy_(snap["m"])
        self.v.copy_(snap["v"])
        self.t = snap["t"]
        self.out_scale = snap["out_scale"]
        self.pack()

    def rescale_output(self, factor: float) -> None:
        """Multiply the output layer (W3, b3) by `factor`, with Adam's
        moments to match (m by factor, v by factor^2): the network's output
        in units of out_scale / factor is the same function as before."""
        off = 0
        for name, shape in SHAPES:
            size = int(np.prod(shape))
            if name in ("W3", "b3"):
                self.params[off:off + size] *= factor
                self.m[off:off + size] *= factor
                self.v[off:off + size] *= factor * factor
            off += size
        self.pack()

    # ---- compute
    def features(self, pm, parts, idx: torch.Tensor | None, rho_mean: float, rows: int | None = None) -> torch.Tensor:
        """bf16 inputs (rows, 80) of particles idx (int64 device tensor) from
        the density mesh of `pm` (a PMPeriodic3D after its deposit)."""
        n = int(idx.numel()) if idx is not None else int(rows)
        X = torch.empty((n, K1), dtype=torch.int16, device=torch.device("cuda", self.device))
        ii = idx.contiguous() if idx is not None else None
        self._call("sss_mlp_features", pm.ptr, ctypes.byref(parts), ii.data_ptr() if ii is not None else None, n,
                   float(rho_mean), X.data_ptr())
        return X

    def forward(self, X: torch.Tensor) -> torch.Tensor:
        rows = X.shape[0]
        Y = torch.empty((rows, 3), dtype=torch.float32, device=X.device)
        self._call("sss_mlp_forward", self.params.data_ptr(), self.frags.data_ptr(), X.data_ptr(), rows, Y.data_ptr())
        return Y

    def grad(self, X: torch.Tensor, T: torch.Tensor, idx: torch.Tensor | None = None, loss: bool = True):
        """Gradient of mean((Y - T)^2) over the rows idx (int32) of X, T."""
        rows = int(idx.numel()) if idx is not None else X.shape[0]
        if T.shape[0] != X.shape[0]:
            raise ValueError("X and T must have the same rows")
        self._call("sss_mlp_grad", self.params.data_ptr(), self.frags.data_ptr(), X.data_ptr(),
                   T.contiguous().data_ptr(), X.shape[0], idx.data_ptr() if idx is not None else None, rows,
                   self.grads.data_ptr(), self.loss_dev.data_ptr() if loss else None)
        return self.grads, self.loss_dev

    def adam_step(self, grads: torch.Tensor, lr: float, beta1: float = 0.9, beta2: float = 0.999,
                  eps: float = 1e-8) -> None:
        self.t += 1
        self._call("sss_mlp_adam", self.params.data_ptr(), grads.data_ptr(), self.m.data_ptr(), self.v.data_ptr(),
                   self.params.numel(), self.t, lr, beta1, beta2, eps)
        self.pack()

    def train(self, X: torch.Tensor, T: torch.Tensor, iters: int, batch: int, lr: float,
              rng: np.random.Generator) -> list[float]:
        """`iters` Adam steps on minibatches of `batch` rows drawn from
        (X, T); returns the minibatch losses (read back once at the end)."""
        n = X.shape[0]
        dev = X.device
        losses = torch.empty(iters, dtype=torch.float32, device=dev)
        draws = rng.integers(0, n, size=(iters, min(batch, n)), dtype=np.int32)
        idx_all = torch.as_tensor(draws).to(dev)
        for it in range(iters):
            self.grad(X, T, idx_all[it])
            losses[it:it + 1].copy_(self.loss_dev)
            self.adam_step(self.grads, lr)
        return losses.cpu().tolist()
