"""The server's per-sample stream core on one B200 (reference
backend/server.py: FilmSession.build_frame with _anzeige_koords,
_lod_auswahl, _dichte_filter and _index_hash): culling by box and kill time,
the density LOD and the u16 quantisation of a sample, bit-exact against the
reference (linear display coordinates; the log zoom evaluates hypot and
log1p on the device).

    sf = StreamFrames(is_ast, injected, visible)
    box = sf.box(x_dev, y_dev, view, log_zoom)              # the session's box rule
    sel, qx, qy = sf.sample(x_dev, y_dev, t_i, raster_days, box, log_zoom, budget)
    sf.kill(idx, t)                                         # the event stream's kill times
    frame = sf.sample_batch([x0, x1], [y0, y1], [t0, t1], raster_days, box, log_zoom, budget)

The frame bytes around it (header, events, sub-sample chains, the unchanged
index list flag) stay with the server's own packing code.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib

LOD_MAX = 120_000        # server.py build_frame: the client's decode limit per sample


def lod_budget(setting: int, bandwidth: float) -> int:
    """Points per sample (build_frame's lod_max)."""
    return setting or min(LOD_MAX, max(20000, int(bandwidth * 0.7 / 20.0 / 8.0)))


class StreamFrames:
    def __init__(self, is_ast, injected=None, visible=None, device: int = 0):
        self.device = int(device)
        self.dev = torch.device("cuda", self.device)
        self.ctx = _lib.context(device)
        is_ast = np.asarray(is_ast) != 0
        self.n = len(is_ast)
        self.d_ast = torch.as_tensor(is_ast.astype(np.uint8)).to(self.dev)
        self.d_inj = (torch.as_tensor((np.asarray(injected) != 0).astype(np.uint8)).to(self.dev)
                      if injected is not None else None)
        vis = np.ones(self.n, bool) if visible is None else np.asarray(visible) != 0
        self.kill_t = torch.as_tensor(np.where(vis, np.inf, -np.inf)).to(self.dev)
        self.sel = torch.empty(self.n, dtype=torch.int32, device=self.dev)
        self.qx = torch.empty(self.n, dtype=torch.int16, device=self.dev)
        self.qy = torch.empty(self.n, dtype=torch.int16, device=self.dev)
        self._bsel = self._bqx = self._bqy = None       # batch outputs, grown on demand

    def _s(self):
        return ctypes.c_void_p(_lib.stream_handle(self.device))

    def kill(self, idx, t: float) -> None:
        """Kill time of bodies (min with the known one), as the event stream sets it."""
        i = torch.as_tensor(np.asarray(idx, np.int64)).to(self.dev)
        self.kill_t[i] = torch.minimum(self.kill_t[i], torch.full_like(self.kill_t[i], float(t)))

    def display(self, x, y):
        """Log-zoom display coordinates of f32 device tensors x, y
        (_anzeige_koords with log_zoom, server.py:99-111): new tensors."""
        x = x.to(device=self.dev, dtype=torch.float32).contiguous()
        y = y.to(device=self.dev, dtype=torch.float32).contiguous()
        if x.numel() != y.numel():
            raise ValueError("display: x and y must have the same length")
        qx, qy = torch.empty_like(x), torch.empty_like(y)
        with torch.cuda.device(self.device):
            self.ctx.check(self.ctx.lib.sss_stream_display(self.ctx.ptr, x.numel(), x.data_ptr(), y.data_ptr(),
                                                           qx.data_ptr(), qy.data_ptr(), self._s()))
        return qx, qy

    def box(self, x, y, view, log_zoom: bool):
        """The reference box: 2x the viewport about the camera, or before
        the client reported one, the whole distribution plus 5 %."""
        cx, cy, hw, hh = (float(v) for v in view)
        if hw > 0 and hh > 0:
            return (cx - 2 * hw, cy - 2 * hh, max(4 * hw, 1e-6), max(4 * hh, 1e-6))
        out = (ctypes.c_float * 4)()
        with torch.cuda.device(self.device):
            self.ctx.check(self.ctx.lib.sss_stream_minmax(self.ctx.ptr, self.n, x.data_ptr(), y.data_ptr(),
                                                          int(bool(log_zoom)), out, self._s()))
        bx0, bx1, by0, by1 = (float(v) for v in out)
        mx = 0.05 * max(bx1 - bx0, 1e-6)
        my = 0.05 * max(by1 - by0, 1e-6)
        return (bx0 - mx, by0 - my, max(bx1 - bx0 + 2 * mx, 1e-6), max(by1 - by0 + 2 * my, 1e-6))

    def sample(self, x, y, t_i: float, raster_days: float, box, log_zoom: bool, budget: int):
        """(sel u32, qx u16, qy u16) views of one sample (device tensors,
        valid until the next call)."""
        x = x.contiguous()
        y = y.contiguous()
        for v in (x, y):
            if v.numel() != self.n or v.dtype != torch.float32 or v.device != self.dev:
                raise ValueError(f"sample: x and y must be f32 tensors of {self.n} bodies on {self.dev}")
        b = (ctypes.c_double * 4)(*(float(v) for v in box))
        cnt = ctypes.c_int64()
        args = (self.ctx.ptr, self.n, x.data_ptr(), y.data_ptr(), self.kill_t.data_ptr(), float(t_i - raster_days),
                self.d_ast.data_ptr(), self.d_inj.data_ptr() if self.d_inj is not None else None, b,
                int(bool(log_zoom)), int(budget), self.sel.data_ptr(), self.qx.data_ptr(), self.qy.data_ptr(),
                ctypes.byref(cnt))
        if torch.cuda.current_device() == self.device:
            self.ctx.check(self.ctx.lib.sss_stream_sample(*args, self._s()))
        else:
            with torch.cuda.device(self.device):
                self.ctx.check(self.ctx.lib.sss_stream_sample(*args, self._s()))
        m = cnt.value
        return self.sel[:m], self.qx[:m], self.qy[:m]

    def sample_batch(self, xs, ys, t_is, raster_days: float, box, log_zoom: bool, budget: int):
        """The samples of one frame at once (build_frame's list of ring
        slots): xs, ys sequences of f32 device tensors, t_is their sample
        times. A list of (sel u32, qx u16, qy u16) device views per sample,
        valid until the next batch call."""
        k = len(xs)
        if len(ys) != k or len(t_is) != k:
            raise ValueError("sample_batch: xs, ys and t_is must have the same length")
        if k == 0:
            return []
        xs = [x.contiguous() for x in xs]
        ys = [y.contiguous() for y in ys]
        for v in xs + ys:
            if v.numel() != self.n or v.dtype != torch.float32 or v.device != self.dev:
                raise ValueError(f"sample_batch: samples must be f32 tensors of {self.n} bodies on {self.dev}")
        if self._bsel is None or self._bsel.numel() < k * self.n:
            self._bsel = torch.empty(k * self.n, dtype=torch.int32, device=self.dev)
            self._bqx = torch.empty(k * self.n, dtype=torch.int16, device=self.dev)
            self._bqy = torch.empty(k * self.n, dtype=torch.int16, device=self.dev)
        px = (ctypes.c_void_p * k)(*(x.data_ptr() for x in xs))
        py = (ctypes.c_void_p * k)(*(y.data_ptr() for y in ys))
        tc = (ctypes.c_double * k)(*(float(t) - float(raster_days) for t in t_is))
        b = (ctypes.c_double * 4)(*(float(v) for v in box))
        cnt = (ctypes.c_int64 * k)()
        args = (self.ctx.ptr, self.n, k, px, py, self.kill_t.data_ptr(), tc, self.d_ast.data_ptr(),
                self.d_inj.data_ptr() if self.d_inj is not None else None, b, int(bool(log_zoom)), int(budget),
                self._bsel.data_ptr(), self._bqx.data_ptr(), self._bqy.data_ptr(), cnt)
        with torch.cuda.device(self.device):
            self.ctx.check(self.ctx.lib.sss_stream_sample_batch(*args, self._s()))
        out = []
        for i in range(k):
            o = i * self.n
            m = cnt[i]
            out.append((self._bsel[o:o + m], self._bqx[o:o + m], self._bqy[o:o + m]))
        return out
