"""Golden stream frames from the reference's own server code.

Runs the reference's FilmSession.build_frame (backend/server.py:378-537, with
_lod_auswahl :629-684, _dichte_filter :686-747, _anzeige_koords :99-111,
_index_hash :117-131) unmodified on CPU: the session object is created
without its producer process and given only the attributes build_frame
reads (a ring of two f32 samples, no events, no sub-samples). CuPy is
replaced by NumPy through cupy_shim. Writes server_frame_<scene>.npz with
the inputs and, per sample, the culled/thinned index list, the u16
coordinates and the box.

    python tests/golden/make_golden_frames.py /path/to/reference/backend

NumPy runs with its SIMD dispatch switched off (NPY_DISABLE_CPU_FEATURES,
read when NumPy is imported), so float32 log1p and hypot are the C
library's: on CPUs with AVX512_SKX NumPy would otherwise take float32 log1p
from a SIMD kernel that differs from the C library in the last bit or two
for about 10 % of the inputs, and the log-zoom frame would depend on the
CPU that wrote it.
"""
from __future__ import annotations

import os
import struct
import sys

os.environ["NPY_DISABLE_CPU_FEATURES"] = ("AVX512F AVX512CD AVX512_SKX AVX512_CLX AVX512_CNL AVX512_ICL "
                                          "AVX512_SPR AVX2 FMA3 F16C AVX")

import numpy as np  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


class _Val:
    def __init__(self, v):
        self.value = v


def _session(server, n, samples, is_ast, injected, kill_t, view, log_zoom, budget):
    S = object.__new__(server.FilmSession)
    S.n = n
    S.ev_count_val = _Val(0)
    S.sent_ev = 0
    S.ev_cap = 1024
    S.ev_verworfen = 0
    S._kill_t = kill_t
    S.view = view
    S.m_sub = 0
    S.t0 = 0.0
    S.raster_days = 0.5
    S.log_zoom = log_zoom
    S.lod_budget = budget
    S._bw = 1e9
    S._letzte_sel = None
    S.head_val = _Val(len(samples))
    S.capacity = 64
    S._is_ast = is_ast
    S._injiziert = injected
    S.slot_pos = lambda i: samples[i]
    return S


def _parse(frame, n_samples):
    typ, n, k, ev_n = struct.unpack_from("<IIII", frame, 0)
    meta = struct.unpack_from("<9d", frame, 16)
    off = 16 + 72 + 8 * k
    out = []
    last = None
    for _ in range(k):
        (kopf,) = struct.unpack_from("<I", frame, off)
        off += 4
        m = kopf & 0x7FFF_FFFF
        if kopf & 0x8000_0000:
            sel = last
        else:
            sel = np.frombuffer(frame, "<u4", m, off).copy()
            off += 4 * m
        qx = np.frombuffer(frame, "<u2", m, off).copy()
        off += 2 * m
        qy = np.frombuffer(frame, "<u2", m, off).copy()
        off += 2 * m
        (ns,) = struct.unpack_from("<I", frame, off)
        off += 4
        off += (-off) % 4
        out.append((sel, qx, qy, bool(kopf & 0x8000_0000)))
        last = sel
    return meta, out


def _clouds(rng, n_mass, n_ast, n_inj, spread=1.0):
    n = n_mass + n_ast + n_inj
    x = np.zeros(n)
    y = np.zeros(n)
    x[:n_mass] = rng.uniform(-5, 5, n_mass)
    y[:n_mass] = rng.uniform(-5, 5, n_mass)
    cen = rng.uniform(-3, 3, (6, 2))
    lab = rng.integers(0, 6, n_ast + n_inj)
    sig = 10 ** rng.uniform(-2.5, -0.5, 6) * spread
    x[n_mass:] = cen[lab, 0] + rng.normal(0, 1, n_ast + n_inj) * sig[lab]
    y[n_mass:] = cen[lab, 1] + rng.normal(0, 1, n_ast + n_inj) * sig[lab]
    is_ast = np.zeros(n, bool)
    is_ast[n_mass:] = True
    inj = np.zeros(n, bool)
    inj[n_mass + n_ast:] = True
    return x, y, is_ast, inj


def scenes():
    rng = np.random.default_rng(20261203)
    out = {}
    # asteroid clouds, view box on part of the scene, budget forcing the density LOD
    x, y, a, inj = _clouds(rng, 12, 16000, 4000)
    out["wolken"] = (x, y, a, inj, (0.5, -0.5, 2.5, 2.0), False, 4000)
    # many massive bodies (self-gravity cloud): the masses' own share of the budget
    x, y, a, inj = _clouds(rng, 3000, 2000, 0, spread=2.0)
    out["massenwolke"] = (x, y, a, inj, (0.0, 0.0, 4.0, 4.0), False, 1500)
    # no view reported (auto box over all bodies), log zoom, LOD
    x, y, a, inj = _clouds(rng, 9, 20000, 0)
    out["autobox_log"] = (x, y, a, inj, (0.0, 0.0, -1.0, -1.0), True, 4000)
    # small scene under the budget: culling only, some bodies dead
    x, y, a, inj = _clouds(rng, 5, 3000, 500)
    out["klein_tot"] = (x, y, a, inj, (0.0, 0.0, 3.0, 3.0), False, 100000)
    return out


def main(backend: str) -> None:
    sys.path.insert(0, HERE)
    import cupy_shim
    cupy_shim.install()
    sys.path.insert(0, backend)
    import server
    rng = np.random.default_rng(7)
    for name, (x, y, a, inj, view, log_zoom, budget) in scenes().items():
        n = len(x)
        kill_t = np.full(n, np.inf)
        if name == "klein_tot":
            dead = rng.choice(n, 300, replace=False)
            kill_t[dead[:150]] = -np.inf               # dead before the film
            kill_t[dead[150:]] = 0.3                   # dies between the samples
        # two samples: the second moved a little (its index list usually changes)
        s0 = np.concatenate([x, y]).astype("<f4")
        s1 = np.concatenate([x + rng.normal(0, 1e-3, n), y + rng.normal(0, 1e-3, n)]).astype("<f4")
        S = _session(server, n, {0: s0, 1: s1}, a, inj, kill_t, view, log_zoom, budget)
        frame = S.build_frame([0, 1])
        meta, blocks = _parse(frame, 2)
        rec = {"x0": s0[:n], "y0": s0[n:], "x1": s1[:n], "y1": s1[n:], "is_ast": a.astype(np.uint8),
               "injected": inj.astype(np.uint8), "kill_t": kill_t, "view": np.array(view), "log_zoom": log_zoom,
               "budget": budget, "raster_days": 0.5, "t0": 0.0, "box": np.array(meta[2:6])}
        for k, (sel, qx, qy, same) in enumerate(blocks):
            rec[f"sel{k}"] = sel
            rec[f"qx{k}"] = qx
            rec[f"qy{k}"] = qy
            rec[f"same{k}"] = same
        np.savez_compressed(os.path.join(HERE, f"server_frame_{name}.npz"), **rec)
        print(name, n, [len(b[0]) for b in blocks], meta[2:6])


if __name__ == "__main__":
    if len(sys.argv) < 2 or not os.path.isfile(os.path.join(sys.argv[1], "server.py")):
        sys.exit("usage: make_golden_frames.py REFERENCE_CHECKOUT/backend")
    main(sys.argv[1])
