"""Few massive bodies + many asteroids on one B200 (f64, Yoshida-4).

Drop-in for the reference's `backend/nbody_kernel.py` (`NBodyCuda`):

    sim = NBodyCuda(devices, m_sub=SUB_SAMPLES)
    st = sim.load_state(x, y, vx, vy, mass, visible, is_ast, real_r=None)
    out = sim.step_batch(st, dt_raster_years, k)   # f32 (k, 4n) [x|y|vx|vy]
    st["sub"], st["hits"]                          # sub-samples, contacts
    sim.apply_updates / apply_deltas / apply_body_state / set_radius /
    deactivate_body / export_f64

Additive keyword arguments: 3-D states (`z=`, `vz=` in load_state; rows
become [x|y|z|vx|vy|vz], update values [x,y,z,vx,vy,vz]), and the physical
constants `G`, `softening`, `max_sub_dt` of the constructor (defaults: the
reference's AU/year/Msun values).

The state stays resident in HBM (torch tensors); the integration runs in
libsss (`sss_frame_launch`), with no CPU path.
"""
from __future__ import annotations

import ctypes
import warnings

import numpy as np
import torch

from . import _lib

M_MAX = 64
K_MAX = 16
G_AU = 4 * np.pi * np.pi
SOFTENING = 1e-6
MAX_SUB_DT_YEARS = 0.5 / 365.25
MAX_SUB_STEPS_PER_FRAME = 100_000
FINE_STEPS_MAX = 8000          # iteration guard of the hot asteroids' fine loop (nbody_kernel.py:424)
YOSHIDA_W1 = 1.0 / (2.0 - 2.0 ** (1.0 / 3.0))
YOSHIDA_W0 = -(2.0 ** (1.0 / 3.0)) / (2.0 - 2.0 ** (1.0 / 3.0))
SUB_SAMPLES = 8
SUB_SAMPLES_MAX = 32
G_MAX = 8


def f64_score(i: int) -> float:
    """Relative f64 throughput of device i (SMs x clock x f64 ratio)."""
    p = torch.cuda.get_device_properties(i)
    ratio = 0.5 if p.major in (6, 7, 8, 9, 10) and p.minor == 0 else 1 / 32
    return p.multi_processor_count * ratio


def pick_device() -> int:
    """The physics GPU (single-device build: the current device)."""
    if not torch.cuda.is_available():
        raise RuntimeError("no CUDA device")
    return torch.cuda.current_device()


def pick_devices() -> list[int]:
    return [pick_device()]


def pick_detect_devices(exclude, rank: int = 0, count: int = 1) -> list[int]:
    """GPUs outside the physics cards for collision detection. One GPU per
    process here, so none: detection runs on the physics card (the
    reference's fallback when no card is free, nbody_kernel.py:591-614)."""
    return []


FrameState = _lib.FrameState


class NBodyCuda:
    """Few massive + many asteroid bodies, resident on one GPU."""

    def __init__(self, devices, m_sub=SUB_SAMPLES, *, G: float = G_AU, softening: float = SOFTENING,
                 max_sub_dt: float = MAX_SUB_DT_YEARS, max_sub_steps: int = MAX_SUB_STEPS_PER_FRAME,
                 max_fine_steps: int = FINE_STEPS_MAX, strict_guard: bool = False, pair_f32: bool = False):
        """Additive keywords beyond the reference's: max_fine_steps is the
        iteration guard of a hot asteroid's fine loop (the reference's fixed
        8000); strict_guard=True turns a guard that ran out into an SSSError
        (SSS_ERR_GUARD) instead of a RuntimeWarning; pair_f32=True evaluates
        the asteroid x massive pair forces of calm asteroids and the
        back-reaction in f32 (f64 state, f64 sums; hot asteroids and the
        massive bodies' mutual forces stay f64)."""
        if isinstance(devices, int):
            devices = [devices]
        if not devices or len(devices) > G_MAX:
            raise ValueError(f"1..{G_MAX} Devices erwartet: {devices}")
        if not 0 <= m_sub <= SUB_SAMPLES_MAX:
            raise ValueError(f"m_sub ausserhalb 0..{SUB_SAMPLES_MAX}: {m_sub}")
        if len(devices) > 1:
            raise ValueError("this build runs on one GPU; pass a single device")
        self.m_sub = int(m_sub)
        self.devices = [int(devices[0])]
        self.device = self.devices[0]
        self.G = float(G)
        self.softening = float(softening)
        self.max_sub_dt = float(max_sub_dt)
        self.max_sub_steps = int(max_sub_steps)
        if max_fine_steps < 1:
            raise ValueError("max_fine_steps must be >= 1")
        self.max_fine_steps = int(max_fine_steps)
        self.strict_guard = bool(strict_guard)
        self.pair_f32 = bool(pair_f32)
        self._ctx = _lib.context(self.device)

    def name(self) -> str:
        return torch.cuda.get_device_name(self.device)

    # ------------------------------------------------------------ state
    def load_state(self, x, y, vx, vy, mass, visible, is_ast, real_r=None, *, z=None, vz=None) -> dict:
        """Take over the full state (resident afterwards). Massive bodies are
        those with is_ast == 0 (at most M_MAX), the rest asteroids
        (nbody_kernel.py:659-780)."""
        ast = np.asarray(is_ast) != 0
        m_idx = np.flatnonzero(~ast)
        a_idx = np.flatnonzero(ast)
        m = len(m_idx)
        if m > M_MAX:
            raise ValueError(f"zu viele massive Koerper: {m} > {M_MAX}")
        n = len(x)
        dim = 3 if z is not None else 2
        dev = torch.device("cuda", self.device)
        pos = [np.asarray(x, np.float64), np.asarray(y, np.float64)]
        vel = [np.asarray(vx, np.float64), np.asarray(vy, np.float64)]
        if dim == 3:
            pos.append(np.asarray(z, np.float64))
            vel.append(np.zeros(n) if vz is None else np.asarray(vz, np.float64))
        mass = np.asarray(mass, np.float64)
        vis = (np.asarray(visible) != 0).astype(np.uint8)
        rr = np.zeros(n) if real_r is None else np.asarray(real_r, np.float64)
        na = len(a_idx)

        def t(a, dtype=torch.float64):
            return torch.as_tensor(np.ascontiguousarray(a)).to(device=dev, dtype=dtype)

        st = {
            "N": n, "m": m, "n_ast": na, "dim": dim,
            "m_idx_h": m_idx, "a_idx_h": a_idx,
            "ax": t(np.stack([p[a_idx] for p in pos]) if na else np.zeros((dim, 1))),
            "av": t(np.stack([v[a_idx] for v in vel]) if na else np.zeros((dim, 1))),
            "aacc": torch.zeros((dim, max(na, 1)), dtype=torch.float64, device=dev),
            "am": t(mass[a_idx] if na else np.zeros(1)),
            "avis": t(vis[a_idx] if na else np.zeros(1, np.uint8), torch.uint8),
            "ar": t(rr[a_idx] if na else np.zeros(1)),
            "aidx": t(a_idx if na else np.zeros(1, np.int64), torch.int64),
            "hot": torch.zeros(max(na, 1), dtype=torch.uint8, device=dev),
            "mx": t(np.stack([p[m_idx] for p in pos]) if m else np.zeros((dim, 1))),
            "mv": t(np.stack([v[m_idx] for v in vel]) if m else np.zeros((dim, 1))),
            "mm": t(mass[m_idx] if m else np.zeros(1)),
            "mvis": t(vis[m_idx] if m else np.zeros(1, np.uint8), torch.uint8),
            "mr": t(rr[m_idx] if m else np.zeros(1)),
            "midx": t(m_idx if m else np.zeros(1, np.int64), torch.int64),
            "snap": torch.empty((K_MAX, 2 * dim, n), dtype=torch.float32, device=dev),
            "subpos": torch.zeros((K_MAX, max(self.m_sub, 1), dim, max(na, 1)), dtype=torch.float32,
                                  device=dev),
            "subn": torch.zeros((K_MAX, max(na, 1)), dtype=torch.uint8, device=dev),
            "hitt": torch.full((max(na, 1),), -1.0, dtype=torch.float32, device=dev),
            "hitm": torch.zeros(max(na, 1), dtype=torch.int32, device=dev),
            "guard": torch.zeros(1, dtype=torch.int32, device=dev),
            # host mirrors: masses and visibility decide the massless mode
            "am_h": mass[a_idx].copy(), "avis_h": vis[a_idx].copy(),
        }
        inv_kind = np.zeros(n, np.int8)          # 1 = asteroid, -1 = massive
        inv_pos = np.zeros(n, np.int64)
        inv_kind[a_idx] = 1
        inv_pos[a_idx] = np.arange(na)
        inv_kind[m_idx] = -1
        inv_pos[m_idx] = np.arange(m)
        st["inv_kind"], st["inv_pos"] = inv_kind, inv_pos
        st["c"] = self._make_struct(st)
        return st

    def _make_struct(self, st) -> FrameState:
        c = FrameState()
        d = st["dim"]
        c.dim = d
        c.n_ast = st["n_ast"]
        c.M = st["m"]
        for k in range(d):
            c.ast_x[k] = st["ax"][k].data_ptr()
            c.ast_v[k] = st["av"][k].data_ptr()
            c.ast_acc[k] = st["aacc"][k].data_ptr()
            c.mas_x[k] = st["mx"][k].data_ptr()
            c.mas_v[k] = st["mv"][k].data_ptr()
        c.ast_m = st["am"].data_ptr()
        c.ast_vis = st["avis"].data_ptr()
        c.ast_r = st["ar"].data_ptr()
        c.ast_idx = st["aidx"].data_ptr()
        c.ast_hot = st["hot"].data_ptr()
        c.mas_m = st["mm"].data_ptr()
        c.mas_vis = st["mvis"].data_ptr()
        c.mas_r = st["mr"].data_ptr()
        c.mas_idx = st["midx"].data_ptr()
        c.G = self.G
        c.softening = self.softening
        c.max_sub_dt = self.max_sub_dt
        c.max_sub_steps = self.max_sub_steps
        c.fine_guard = self.max_fine_steps
        c.pair_f32 = int(self.pair_f32)
        c.w1 = YOSHIDA_W1
        c.w0 = YOSHIDA_W0
        return c

    def _stream(self) -> ctypes.c_void_p:
        return ctypes.c_void_p(_lib.stream_handle(self.device))

    # ------------------------------------------------------------ step
    def step_batch_device(self, st: dict, dt_raster_years: float, k: int) -> torch.Tensor:
        """k raster samples in one launch; snapshots stay on the device."""
        if st is None:
            raise ValueError("kein Zustand geladen — FULL-Frame noetig")
        if not 1 <= k <= K_MAX:
            raise ValueError(f"k ausserhalb 1..{K_MAX}: {k}")
        c = st["c"]
        c.massless_asteroids = int(not np.any((st["am_h"] != 0) & (st["avis_h"] != 0)))
        st["hitt"].fill_(-1.0)
        with torch.cuda.device(self.device):
            rc = self._ctx.lib.sss_frame_launch(
                self._ctx.ptr, ctypes.byref(c), float(dt_raster_years), int(k), self.m_sub,
                st["snap"].data_ptr(), st["subpos"].data_ptr(), st["subn"].data_ptr(),
                st["hitt"].data_ptr(), st["hitm"].data_ptr(), st["guard"].data_ptr(), self._stream())
        self._ctx.check(rc)
        return st["snap"][:k]

    def step_batch(self, st: dict, dt_raster_years: float, k: int) -> np.ndarray:
        """k raster samples in ONE launch; f32 (k, 4n) [x|y|vx|vy] in original
        order; st["sub"] and st["hits"] as the reference
        (nbody_kernel.py:783-934)."""
        snap = self.step_batch_device(st, dt_raster_years, k)
        out = snap.reshape(k, -1).cpu().numpy()
        rc = self._ctx.status_code(_lib.stream_handle(self.device))
        if rc == _lib.SSS_ERR_GUARD:
            # the reference stops the interval where its guard runs out and goes on
            # (nbody_kernel.py:248-250, :424); this build reports it
            st["guard_exhausted"] = st.get("guard_exhausted", 0) + 1
            msg = ("a step guard ran out (MAX_SUB_STEPS_PER_FRAME or the fine-loop limit): "
                   "the batch did not cover its interval")
            if self.strict_guard:
                raise _lib.SSSError(rc, msg)
            warnings.warn(msg, RuntimeWarning)
        else:
            self._ctx.check(rc)
        st["sub"] = self._collect_sub(st, k)
        st["hits"] = self._collect_hits(st)
        return out

    def step(self, st: dict, dt_years: float) -> np.ndarray:
        """A single sample (the live path of the server)."""
        return self.step_batch(st, dt_years, 1)[0]

    def _collect_hits(self, st):
        na = st["n_ast"]
        if not na:
            return (np.empty(0, np.int64), np.empty(0, np.float32), np.empty(0, np.int64))
        ht = st["hitt"][:na].cpu().numpy()
        sel = np.flatnonzero(ht >= 0.0)
        if sel.size == 0:
            return (np.empty(0, np.int64), np.empty(0, np.float32), np.empty(0, np.int64))
        hm = st["hitm"][:na].cpu().numpy()
        return (st["a_idx_h"][sel], ht[sel], st["m_idx_h"][hm[sel]])

    def _collect_sub(self, st, k):
        if self.m_sub <= 0:
            return None
        ms, na, d = self.m_sub, st["n_ast"], st["dim"]
        frames = []
        if not na:
            return [(np.empty(0, np.int64), np.empty((ms, d, 0), np.float32)) for _ in range(k)]
        subn = st["subn"][:k, :na]
        for ks in range(k):
            sel = torch.nonzero(subn[ks] == ms).flatten()
            if sel.numel() == 0:
                frames.append((np.empty(0, np.int64), np.empty((ms, d, 0), np.float32)))
                continue
            pos = st["subpos"][ks, :ms, :, :na][:, :, sel].cpu().numpy()
            frames.append((st["a_idx_h"][sel.cpu().numpy()], pos))
        return frames

    # ------------------------------------------------------- point updates
    def _scatter(self, st, idx, vals, mode):
        idx = np.asarray(idx, np.int64).ravel()
        vals = np.asarray(vals, np.float64).reshape(len(idx), -1)
        d = st["dim"]
        want = 2 * d + (1 if mode == 2 else 0)
        if vals.shape[1] != want:
            raise ValueError(f"expected {want} values per body, got {vals.shape[1]}")
        kind = st["inv_kind"][idx]
        pos = st["inv_pos"][idx]
        slot = np.where(kind > 0, pos, -pos - 1).astype(np.int64)
        dev = torch.device("cuda", self.device)
        s_t = torch.from_numpy(slot).to(dev)
        v_t = torch.from_numpy(np.ascontiguousarray(vals)).to(dev)
        with torch.cuda.device(self.device):
            rc = self._ctx.lib.sss_frame_scatter(self._ctx.ptr, ctypes.byref(st["c"]), s_t.data_ptr(),
                                                 v_t.data_ptr(), len(idx), mode, self._stream())
        self._ctx.check(rc)
        torch.cuda.current_stream(self.device).synchronize()

    def apply_updates(self, st: dict, idx, vals) -> None:
        """Set x/y/vx/vy absolutely at original indices (nbody_kernel.py:947-950)."""
        self._scatter(st, idx, vals, 0)

    def apply_deltas(self, st: dict, idx, deltas) -> None:
        """Add x/y/vx/vy corrections; idx must be unique (nbody_kernel.py:952-956)."""
        idx = np.asarray(idx, np.int64)
        if len(np.unique(idx)) != len(idx):
            raise ValueError("apply_deltas: idx must be unique")
        self._scatter(st, idx, deltas, 1)

    def apply_deltas_device(self, st: dict, idx, deltas, m: int) -> None:
        """apply_deltas for device arrays (idx int64 [m] unique original
        indices, deltas f64 [m][2*dim]) without a host round trip."""
        if m <= 0:
            return
        if "slot_d" not in st:
            slot = np.where(st["inv_kind"] > 0, st["inv_pos"], -st["inv_pos"] - 1).astype(np.int64)
            st["slot_d"] = torch.as_tensor(slot).to(torch.device("cuda", self.device))
        s_t = st["slot_d"][idx[:m]].contiguous()
        v_t = deltas[:m].contiguous()
        if v_t.shape[1] != 2 * st["dim"]:
            raise ValueError(f"expected {2 * st['dim']} values per body, got {v_t.shape[1]}")
        with torch.cuda.device(self.device):
            rc = self._ctx.lib.sss_frame_scatter(self._ctx.ptr, ctypes.byref(st["c"]), s_t.data_ptr(),
                                                 v_t.data_ptr(), int(m), 1, self._stream())
        self._ctx.check(rc)

    def apply_body_state(self, st: dict, idx: int, x: float, y: float, vx: float, vy: float,
                         mass: float, *, z: float = 0.0, vz: float = 0.0) -> None:
        """Set one body completely (x, y, vx, vy, mass) (nbody_kernel.py:990-1010)."""
        d = st["dim"]
        vals = [x, y, z, vx, vy, vz, mass] if d == 3 else [x, y, vx, vy, mass]
        self._scatter(st, [idx], [vals], 2)
        if st["inv_kind"][idx] > 0:
            st["am_h"][st["inv_pos"][idx]] = mass

    def apply_body_states(self, st: dict, idx, vals) -> None:
        """apply_body_state for several bodies in one scatter: vals [m][2*dim+1]
        (x, y, (z), vx, vy, (vz), mass) at unique original indices idx (the
        batched form of nbody_kernel.py:990-1010; additive API)."""
        idx = np.asarray(idx, np.int64).ravel()
        if len(idx) == 0:
            return
        if len(np.unique(idx)) != len(idx):
            raise ValueError("apply_body_states: idx must be unique")
        vals = np.asarray(vals, np.float64).reshape(len(idx), -1)
        self._scatter(st, idx, vals, 2)
        ast = st["inv_kind"][idx] > 0
        st["am_h"][st["inv_pos"][idx[ast]]] = vals[ast, -1]

    def set_radii(self, st: dict, idx, radii) -> None:
        """set_radius for several bodies at once (additive API)."""
        idx = np.asarray(idx, np.int64).ravel()
        if len(idx) == 0:
            return
        r = np.asarray(radii, np.float64).ravel()
        dev = torch.device("cuda", self.device)
        ast = st["inv_kind"][idx] > 0
        for sel, key in ((ast, "ar"), (~ast, "mr")):
            if sel.any():
                p_t = torch.as_tensor(st["inv_pos"][idx[sel]]).to(dev)
                st[key][p_t] = torch.as_tensor(r[sel]).to(dev)

    def deactivate_bodies(self, st: dict, idx) -> None:
        """deactivate_body for several bodies at once: mass 0, not visible
        (additive API)."""
        idx = np.asarray(idx, np.int64).ravel()
        if len(idx) == 0:
            return
        dev = torch.device("cuda", self.device)
        ast = st["inv_kind"][idx] > 0
        if ast.any():
            pos = st["inv_pos"][idx[ast]]
            p_t = torch.as_tensor(pos).to(dev)
            st["am"][p_t] = 0.0
            st["avis"][p_t] = 0
            st["am_h"][pos] = 0.0
            st["avis_h"][pos] = 0
        if (~ast).any():
            p_t = torch.as_tensor(st["inv_pos"][idx[~ast]]).to(dev)
            st["mm"][p_t] = 0.0
            st["mvis"][p_t] = 0

    def set_asteroids(self, st: dict, idx, vals, radii) -> None:
        """Set asteroids completely and make them visible: vals [m][2*dim+1]
        (x, y, (z), vx, vy, (vz), mass) and contact radii [m] at original
        indices idx (unique asteroids), in one scatter. The fragments of a
        fragmenting impact take their parents' and free slots this way (no
        reference counterpart: its client creates fragment bodies)."""
        idx = np.asarray(idx, np.int64).ravel()
        if len(idx) == 0:
            return
        if len(np.unique(idx)) != len(idx) or np.any(st["inv_kind"][idx] <= 0):
            raise ValueError("set_asteroids: idx must be unique asteroid indices")
        self._scatter(st, idx, vals, 2)
        pos = st["inv_pos"][idx]
        dev = torch.device("cuda", self.device)
        p_t = torch.from_numpy(pos).to(dev)
        st["ar"][p_t] = torch.from_numpy(np.asarray(radii, np.float64)).to(dev)
        st["avis"][p_t] = 1
        st["am_h"][pos] = np.asarray(vals, np.float64).reshape(len(idx), -1)[:, -1]
        st["avis_h"][pos] = 1

    def set_radius(self, st: dict, idx: int, wert: float) -> None:
        """Contact radius of one body (nbody_kernel.py:1012-1025)."""
        p = int(st["inv_pos"][idx])
        (st["ar"] if st["inv_kind"][idx] > 0 else st["mr"])[p] = float(wert)

    def deactivate_body(self, st: dict, idx: int) -> None:
        """Freeze a body and make it force-free: mass 0, visible 0 (:1027-1040)."""
        p = int(st["inv_pos"][idx])
        if st["inv_kind"][idx] > 0:
            st["am"][p] = 0.0
            st["avis"][p] = 0
            st["am_h"][p] = 0.0
            st["avis_h"][p] = 0
        else:
            st["mm"][p] = 0.0
            st["mvis"][p] = 0

    def export_f64(self, st: dict) -> np.ndarray:
        """Exact f64 state [x|y|(z)|vx|vy|(vz)] in original order (:1042-1060)."""
        n, d = st["N"], st["dim"]
        out = np.empty(2 * d * n, dtype="<f8")
        a, m = st["a_idx_h"], st["m_idx_h"]
        ax, av = st["ax"].cpu().numpy(), st["av"].cpu().numpy()
        mx, mv = st["mx"].cpu().numpy(), st["mv"].cpu().numpy()
        for c in range(d):
            out[c * n + a] = ax[c, :len(a)]
            out[(d + c) * n + a] = av[c, :len(a)]
            out[c * n + m] = mx[c, :len(m)]
            out[(d + c) * n + m] = mv[c, :len(m)]
        return out
