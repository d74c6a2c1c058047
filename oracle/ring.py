"""CPU oracle (test infrastructure only) of the film producer's ring-slot
format and the self-gravity row reorder (reference backend/film_producer.py:
79-123 `slot_bytes` / `schreibe_slot`, :1245-1261 the tracer reorder).

A slot is x|y f32 (8n bytes) | u32 count | u32 indices (a fixed field of
sub_max entries) | f32 sub-samples (nh, mSub, 2), the hot bodies' indices
ascending (at most sub_max kept), their sub-sample chains stored body by
body.
"""
from __future__ import annotations

import struct

import numpy as np


def slot_bytes(n: int, m_sub: int, sub_max: int) -> int:
    return 8 * n + 4 + sub_max * (4 + 8 * m_sub)


def write_slot(n: int, m_sub: int, sub_max: int, out_i, sub_i):
    """(slot bytes, overflow) for kernel output row out_i (f32, [x|y|...])
    and sub_i = (idx, pos (mSub, d, nh)) or None."""
    buf = bytearray(slot_bytes(n, m_sub, sub_max))
    out_i = np.asarray(out_i, np.float32)
    buf[0:8 * n] = out_i[0:2 * n].tobytes()
    off = 8 * n
    if sub_i is None or not sub_max:
        buf[off:off + 4] = struct.pack("<I", 0)
        return bytes(buf), False
    idx, pos = sub_i
    idx = np.asarray(idx)
    overflow = len(idx) > sub_max
    order = np.argsort(idx, kind="stable")[:sub_max]
    nh = len(order)
    buf[off:off + 4] = struct.pack("<I", nh)
    off += 4
    buf[off:off + 4 * nh] = idx[order].astype("<u4").tobytes()
    off += 4 * sub_max
    if nh:
        chains = np.ascontiguousarray(np.asarray(pos)[:, 0:2, order].transpose(2, 0, 1)).astype("<f4")
        buf[off:off + chains.nbytes] = chains.tobytes()
    return bytes(buf), overflow


def reorder_selfgrav(outs, sg_m, sg_t, n):
    """Rows [x_m|y_m|vx_m|vy_m|x_t|y_t] -> [x|y|vx|vy] in original order,
    tracer velocities zero (film_producer.py:1245-1261)."""
    outs = np.asarray(outs, np.float32)
    nm, nt = len(sg_m), len(sg_t)
    full = np.zeros((outs.shape[0], 4 * n), np.float32)
    full[:, sg_m] = outs[:, 0:nm]
    full[:, n + sg_m] = outs[:, nm:2 * nm]
    full[:, 2 * n + sg_m] = outs[:, 2 * nm:3 * nm]
    full[:, 3 * n + sg_m] = outs[:, 3 * nm:4 * nm]
    if nt:
        full[:, sg_t] = outs[:, 4 * nm:4 * nm + nt]
        full[:, n + sg_t] = outs[:, 4 * nm + nt:4 * nm + 2 * nt]
    return full
