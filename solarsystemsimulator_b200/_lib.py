"""ctypes binding of libsss.so (the C ABI declared in include/sss.h).

The library is the only compute path: if it is missing or no CUDA device is
present, every entry point raises — there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsss.so")

SSS_OK = 0
SSS_ERR_ARG = 1
SSS_ERR_TOO_MANY_MASSIVE = 2
SSS_ERR_GUARD = 3
SSS_ERR_TIMEOUT = 4
SSS_ERR_CUDA = 5
SSS_ERR_CAPACITY = 6

PREC_F64 = 0
PREC_MIXED = 1
PREC_MIXED_TC = 2
INT_KDK = 0
INT_YOSHIDA4 = 1

_c_i64 = ctypes.c_int64
_vp = ctypes.c_void_p
_dp = ctypes.c_void_p   # device pointers travel as integers


class SelfGravState(ctypes.Structure):
    """Mirror of sss_selfgrav_state."""
    _fields_ = [
        ("dim", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("n_src", _c_i64),
        ("n_tracer", _c_i64),
        ("pos4", _dp * 2),
        ("vel4", _dp),
        ("acc4", _dp),
        ("cur", ctypes.c_int),
        ("eps2", ctypes.c_double),
    ]


class FrameState(ctypes.Structure):
    """Mirror of sss_frame_state."""
    _fields_ = [
        ("dim", ctypes.c_int), ("n_ast", _c_i64), ("M", ctypes.c_int),
        ("ast_x", _dp * 3), ("ast_v", _dp * 3), ("ast_acc", _dp * 3),
        ("ast_m", _dp), ("ast_vis", _dp), ("ast_r", _dp), ("ast_idx", _dp), ("ast_hot", _dp),
        ("mas_x", _dp * 3), ("mas_v", _dp * 3),
        ("mas_m", _dp), ("mas_vis", _dp), ("mas_r", _dp), ("mas_idx", _dp),
        ("G", ctypes.c_double), ("softening", ctypes.c_double), ("max_sub_dt", ctypes.c_double),
        ("max_sub_steps", ctypes.c_int), ("w1", ctypes.c_double), ("w0", ctypes.c_double),
        ("massless_asteroids", ctypes.c_int),
        ("fine_guard", ctypes.c_int), ("pair_f32", ctypes.c_int),
    ]


class NBodyCfg(ctypes.Structure):
    """sss_nbody_cfg (include/sss.h)."""
    _fields_ = [("G", ctypes.c_double), ("softening", ctypes.c_double), ("max_sub_dt", ctypes.c_double),
                ("max_sub_steps", ctypes.c_int), ("fine_guard", ctypes.c_int), ("m_sub", ctypes.c_int),
                ("pair_f32", ctypes.c_int)]


class Pm3Particles(ctypes.Structure):
    """Mirror of sss_pm3_particles."""
    _fields_ = [
        ("n", _c_i64), ("x", _dp * 3), ("v", _dp * 3), ("a", _dp * 3),
        ("m", _dp), ("mass_const", ctypes.c_double),
    ]


PM3_FORCE = 0
PM3_KICK = 1
PM3_KICK_DRIFT = 2
MLP_N_PARAMS = 27912
MLP_N_FRAGS = 22016
MLP_IN_PAD = 80
COLLIDE_MAX_BODIES = 1600000

# name -> (restype, argtypes); every symbol include/sss.h declares
SIGNATURES = {
    "sss_abi_version": (ctypes.c_int, []),
    "sss_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_vp)]),
    "sss_destroy": (None, [_vp]),
    "sss_last_error": (ctypes.c_char_p, [_vp]),
    "sss_device_status": (ctypes.c_int, [_vp, _vp]),
    "sss_num_sms": (ctypes.c_int, [_vp]),
    "sss_allpairs_accel": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _dp, _c_i64, _dp, _c_i64,
                                          _dp, ctypes.c_double, _vp]),
    "sss_allpairs_potential": (ctypes.c_int, [_vp, ctypes.c_int, _dp, _c_i64, _dp, _c_i64, _dp,
                                              ctypes.c_double, _vp]),
    "sss_selfgrav_init_accel": (ctypes.c_int, [_vp, ctypes.POINTER(SelfGravState), _vp]),
    "sss_selfgrav_step_batch": (ctypes.c_int, [_vp, ctypes.POINTER(SelfGravState), ctypes.c_int,
                                               ctypes.c_double, ctypes.c_int, _dp, _vp]),
    "sss_frame_launch": (ctypes.c_int, [_vp, ctypes.POINTER(FrameState), ctypes.c_double, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp,
                                        _dp, _dp, _dp, _vp]),
    "sss_frame_scatter": (ctypes.c_int, [_vp, ctypes.POINTER(FrameState), _dp, _dp, ctypes.c_int, ctypes.c_int, _vp]),
    "sss_broadphase": (ctypes.c_int, [_vp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _c_i64, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_double, ctypes.c_float, ctypes.c_float, _dp,
                                      _c_i64, ctypes.POINTER(_c_i64), ctypes.POINTER(_c_i64), _vp]),
    "sss_broadphase_order": (ctypes.c_int, [_vp, _dp, _c_i64, _c_i64, _vp]),
    "sss_pm2d_create": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(_vp)]),
    "sss_pm2d_destroy": (None, [_vp]),
    "sss_pm2d_bbox": (ctypes.c_int, [_vp, _dp, _dp, _c_i64, _dp, _vp]),
    "sss_pm2d_build_kernels": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, _vp]),
    "sss_pm2d_field": (ctypes.c_int, [_vp, _dp, _dp, _dp, _c_i64, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, _vp]),
    "sss_pm2d_gather_field": (ctypes.c_int, [_vp, _dp, ctypes.c_int, _c_i64, _dp, _dp, _c_i64, ctypes.c_double,
                                             ctypes.c_double, ctypes.c_double, _dp, _vp]),
    "sss_pm2d_gather": (ctypes.c_int, [_vp, _dp, _dp, _c_i64, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                       _dp, _dp, _vp]),
    "sss_pm2d_density": (ctypes.c_int, [_vp, _dp, _vp]),
    "sss_pm2d_fields": (ctypes.c_int, [_vp, _dp, _dp, _vp]),
    "sss_pm2d_kick_drift": (ctypes.c_int, [_vp, _dp, _dp, _dp, _dp, _dp, _dp, _c_i64, ctypes.c_double,
                                           ctypes.c_double, ctypes.c_int, _vp]),
    "sss_pm2d_to_f32": (ctypes.c_int, [_vp, _dp, _c_i64, _dp, _vp]),
    "sss_batched_launch": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(_dp), ctypes.POINTER(_dp), _dp, _dp,
                                          _dp, _dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_double, ctypes.c_int, ctypes.c_int, _vp]),
    "sss_collide_sweep": (ctypes.c_int, [_vp, _c_i64, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp,
                                         ctypes.c_int, ctypes.c_double, ctypes.c_double, _dp, _c_i64, _dp, _c_i64,
                                         ctypes.POINTER(_c_i64), ctypes.POINTER(_c_i64), _vp]),
    "sss_collide_fragment": (ctypes.c_int, [_vp, _c_i64, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _c_i64, ctypes.c_double,
                                            ctypes.c_double, ctypes.c_int, ctypes.c_uint64, _dp, _dp, _c_i64,
                                            ctypes.POINTER(_c_i64), _vp]),
    "sss_collide_bounce": (ctypes.c_int, [_vp, _c_i64, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _c_i64, ctypes.c_double,
                                          ctypes.c_double, _dp, _dp, _dp, ctypes.POINTER(_c_i64),
                                          ctypes.POINTER(_c_i64), _vp]),
    "sss_ring_slot": (ctypes.c_int, [_vp, _dp, _c_i64, _dp, _dp, _dp, _c_i64, ctypes.c_int, ctypes.c_int, _c_i64,
                                     _dp, ctypes.POINTER(_c_i64), _vp]),
    "sss_ring_reorder": (ctypes.c_int, [_vp, _dp, ctypes.c_int, _dp, _c_i64, _dp, _c_i64, _c_i64, _dp, _vp]),
    "sss_stream_sample": (ctypes.c_int, [_vp, _c_i64, _dp, _dp, _dp, ctypes.c_double, _dp, _dp,
                                         ctypes.POINTER(ctypes.c_double), ctypes.c_int, _c_i64, _dp, _dp, _dp,
                                         ctypes.POINTER(_c_i64), _vp]),
    "sss_stream_sample_batch": (ctypes.c_int, [_vp, _c_i64, ctypes.c_int, ctypes.POINTER(_dp), ctypes.POINTER(_dp),
                                               _dp, ctypes.POINTER(ctypes.c_double), _dp, _dp,
                                               ctypes.POINTER(ctypes.c_double), ctypes.c_int, _c_i64, _dp, _dp, _dp,
                                               ctypes.POINTER(_c_i64), _vp]),
    "sss_stream_minmax": (ctypes.c_int, [_vp, _c_i64, _dp, _dp, ctypes.c_int, ctypes.POINTER(ctypes.c_float), _vp]),
    "sss_stream_display": (ctypes.c_int, [_vp, _c_i64, _dp, _dp, _dp, _dp, _vp]),
    "sss_pm3_create": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, ctypes.POINTER(_vp)]),
    "sss_pm3_destroy": (None, [_vp]),
    "sss_pm3_meshes": (ctypes.c_int, [_vp, ctypes.POINTER(_dp), ctypes.POINTER(_dp)]),
    "sss_pm3_density": (ctypes.c_int, [_vp, ctypes.POINTER(Pm3Particles), _vp]),
    "sss_pm3_solve": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_int, ctypes.c_double, _vp]),
    "sss_pm3_gather": (ctypes.c_int, [_vp, ctypes.POINTER(Pm3Particles), ctypes.c_int, ctypes.c_double,
                                      ctypes.c_double, _dp, _vp]),
    "sss_pm3_kick_drift": (ctypes.c_int, [_vp, ctypes.POINTER(Pm3Particles), ctypes.c_double, ctypes.c_double,
                                          _vp]),
    "sss_pm3_short": (ctypes.c_int, [_vp, ctypes.POINTER(Pm3Particles), ctypes.c_double, ctypes.c_double,
                                     ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                     ctypes.c_double, _dp, _vp]),
    "sss_ewald_structure": (ctypes.c_int, [_vp, ctypes.POINTER(Pm3Particles), ctypes.c_double, _dp, ctypes.c_int,
                                           ctypes.c_int, _dp, _vp]),
    "sss_ewald_accel": (ctypes.c_int, [_vp, ctypes.POINTER(Pm3Particles), ctypes.POINTER(_dp), _dp, _c_i64,
                                       ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_double, _dp, _dp, _dp, ctypes.c_int, ctypes.POINTER(_dp), _vp]),
    "sss_ewald_gtab": (ctypes.c_int, [_dp, _c_i64, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)]),
    "sss_mlp_pack": (ctypes.c_int, [_vp, _dp, _dp, _vp]),
    "sss_mlp_features": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(Pm3Particles), _dp, _c_i64, ctypes.c_double,
                                        _dp, _vp]),
    "sss_mlp_forward": (ctypes.c_int, [_vp, _dp, _dp, _dp, _c_i64, _dp, _vp]),
    "sss_mlp_grad": (ctypes.c_int, [_vp, _dp, _dp, _dp, _dp, _c_i64, _dp, _c_i64, _dp, _dp, _vp]),
    "sss_mlp_adam": (ctypes.c_int, [_vp, _dp, _dp, _dp, _dp, _c_i64, ctypes.c_int, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_double, ctypes.c_double, _vp]),
    "sss_mlp_correct": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(Pm3Particles), _dp, _dp, ctypes.c_double,
                                       ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double, _dp, _vp]),
    "sss_selftest_wait": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, _vp]),
    "sss_probe_fma": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
    "sss_allpairs_accel_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _c_i64,
                                                  _dp, _c_i64, _dp, ctypes.c_double, _dp, _vp,
                                                  ctypes.c_char_p, ctypes.c_size_t]),
    # sessions (host arrays; no torch on the caller's side)
    "sss_sg_create": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                     ctypes.POINTER(_vp)]),
    "sss_sg_destroy": (None, [_vp]),
    "sss_sg_load": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int64, _vp, _vp, ctypes.c_int64, _vp]),
    "sss_sg_row_width": (ctypes.c_int64, [_vp]),
    "sss_sg_step_batch": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_int, _vp]),
    "sss_sg_export_f64": (ctypes.c_int, [_vp, _vp]),
    "sss_nbody_create": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(_vp)]),
    "sss_nbody_destroy": (None, [_vp]),
    "sss_nbody_load": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int64, _vp, _vp, _vp, _vp, _vp]),
    "sss_nbody_step_batch": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_int, _vp]),
    "sss_nbody_hits": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, ctypes.c_int64]),
    "sss_nbody_sub": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _vp, ctypes.c_int64]),
    "sss_nbody_export_f64": (ctypes.c_int, [_vp, _vp]),
    "sss_nbody_scatter": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int]),
    "sss_nbody_set_radius": (ctypes.c_int, [_vp, ctypes.c_int64, ctypes.c_double]),
    "sss_nbody_deactivate": (ctypes.c_int, [_vp, ctypes.c_int64]),
}

_lib = None
_lock = threading.Lock()


class SSSError(RuntimeError):
    """A libsss call failed (status code in .code)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"libsss error {code}: {msg}")
        self.code = code


def load() -> ctypes.CDLL:
    """Load libsss.so once and declare its signatures."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is not built; run `python -m solarsystemsimulator_b200.build` "
                "(nvcc, sm_100a). There is no CPU fallback.")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


class Context:
    """One sss_ctx on one CUDA device."""

    def __init__(self, device: int):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("no CUDA device: the B200 kernels have no CPU fallback")
        self.lib = load()
        self.device = int(device)
        ptr = _vp()
        rc = self.lib.sss_create(self.device, ctypes.byref(ptr))
        if rc != SSS_OK:
            raise SSSError(rc, f"sss_create(device={device}) failed")
        self.ptr = ptr

    def __del__(self):
        try:
            if getattr(self, "ptr", None):
                self.lib.sss_destroy(self.ptr)
                self.ptr = None
        except Exception:
            pass

    def last_error(self) -> str:
        return self.lib.sss_last_error(self.ptr).decode(errors="replace")

    def check(self, rc: int) -> None:
        if rc == SSS_OK:
            return
        msg = self.last_error()
        if rc == SSS_ERR_ARG:
            raise ValueError(msg)
        raise SSSError(rc, msg)

    def status(self, stream: int) -> None:
        self.check(self.lib.sss_device_status(self.ptr, _vp(stream)))

    def status_code(self, stream: int) -> int:
        """Synchronise the stream, read and clear the device status word."""
        return int(self.lib.sss_device_status(self.ptr, _vp(stream)))

    @property
    def num_sms(self) -> int:
        return int(self.lib.sss_num_sms(self.ptr))


_contexts: dict[int, Context] = {}


def context(device: int) -> Context:
    """Process-wide context per device (created on first use)."""
    with _lock:
        c = _contexts.get(int(device))
    if c is None:
        c = Context(device)
        with _lock:
            _contexts[int(device)] = c
    return c


def stream_handle(device: int) -> int:
    import torch
    return int(torch.cuda.current_stream(device).cuda_stream)
