"""The film producer's ring slots, written on the device (reference
backend/film_producer.py:60-123 SUB_MAX_*, sub_max_fuer, slot_bytes,
schreibe_slot) and the self-gravity row reorder (:1245-1261).

    slot = torch.empty(slot_bytes(n, m_sub, sub_max), dtype=torch.uint8, device="cuda")
    overflow = write_slot(sim, st, ks, slot, sub_max)   # sample ks of the last step_batch
    rows = reorder_selfgrav(outs_dev, sg_m, sg_t, n)    # (K, 4n) f32 on the device

The slot can then go to the shared-memory ring with one device-to-host
copy (or be written by a mapped pointer of that ring).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib

SUB_MAX_ANTEIL = 32      # film_producer.py:63
SUB_MAX_MIN = 2048       # film_producer.py:64


def sub_max_fuer(n: int) -> int:
    return min(n, max(SUB_MAX_MIN, n // SUB_MAX_ANTEIL))


def slot_bytes(n: int, m_sub: int, sub_max: int) -> int:
    return 8 * n + 4 + sub_max * (4 + 8 * m_sub)


def write_slot(sim, st: dict, ks: int, slot: torch.Tensor, sub_max: int) -> bool:
    """Ring slot of sample ks of the last NBodyCuda.step_batch(_device)
    into the device byte tensor `slot`. Returns True when more hot bodies
    occurred than the slot holds (schreibe_slot's overflow flag)."""
    n, na, d = st["N"], st["n_ast"], st["dim"]
    need = slot_bytes(n, sim.m_sub, sub_max)
    if slot.numel() < need or slot.dtype != torch.uint8:
        raise ValueError(f"slot must be a uint8 tensor of >= {need} bytes")
    if "a_idx_d" not in st:
        st["a_idx_d"] = torch.as_tensor(st["a_idx_h"].astype(np.int64)).to(torch.device("cuda", sim.device))
    row = st["snap"][ks]
    ctx = _lib.context(sim.device)
    hot = ctypes.c_int64()
    sub_pos = st["subpos"][ks] if na and sim.m_sub else None
    sub_n = st["subn"][ks] if na and sim.m_sub else None
    with torch.cuda.device(sim.device):
        rc = ctx.lib.sss_ring_slot(ctx.ptr, row.data_ptr(), n,
                                   sub_pos.data_ptr() if sub_pos is not None else None,
                                   sub_n.data_ptr() if sub_n is not None else None,
                                   st["a_idx_d"].data_ptr(), na, sim.m_sub, d, sub_max, slot.data_ptr(),
                                   ctypes.byref(hot), ctypes.c_void_p(_lib.stream_handle(sim.device)))
    ctx.check(rc)
    return hot.value > sub_max


def reorder_selfgrav(outs: torch.Tensor, sg_m, sg_t, n: int, device: int = 0) -> torch.Tensor:
    """(K, 4nm + 2nt) rows of NBodySelfGrav.step_batch_device ->
    (K, 4n) [x|y|vx|vy] in the client's order (tracer velocities 0)."""
    dev = torch.device("cuda", device)
    outs = outs.to(device=dev, dtype=torch.float32).contiguous()
    m = torch.as_tensor(np.asarray(sg_m, np.int64)).to(dev)
    t = torch.as_tensor(np.asarray(sg_t, np.int64)).to(dev)
    K = outs.shape[0]
    out = torch.empty((K, 4 * n), dtype=torch.float32, device=dev)
    ctx = _lib.context(device)
    with torch.cuda.device(device):
        rc = ctx.lib.sss_ring_reorder(ctx.ptr, outs.data_ptr(), K, m.data_ptr(), m.numel(), t.data_ptr(),
                                      t.numel(), n, out.data_ptr(), ctypes.c_void_p(_lib.stream_handle(device)))
    ctx.check(rc)
    return out
