"""The stream-frame oracle (oracle/frames.py) reproduces the golden frames of
the reference's own build_frame bit for bit (index lists and u16
coordinates of both samples, the box)."""
import numpy as np
import pytest

from oracle import frames as ofr

SCENES = ["wolken", "massenwolke", "autobox_log", "klein_tot"]


@pytest.mark.parametrize("scene", SCENES)
def test_oracle_reproduces_reference_frames(load_golden, scene):
    g = load_golden(f"server_frame_{scene}.npz")
    log_zoom = bool(g["log_zoom"])
    qx0, qy0 = ofr.display_coords(g["x0"], g["y0"], log_zoom)
    box = ofr.make_box(qx0, qy0, tuple(g["view"]))
    assert np.array_equal(np.array(box), g["box"])
    a = g["is_ast"] != 0
    inj = g["injected"] != 0
    for k in range(2):
        t_i = float(g["t0"]) + (k + 1) * float(g["raster_days"])
        alive = g["kill_t"] > t_i - float(g["raster_days"])
        sel, qx, qy = ofr.sample_frame(g[f"x{k}"], g[f"y{k}"], alive, a, inj, box, log_zoom, int(g["budget"]))
        assert np.array_equal(sel, g[f"sel{k}"]) and np.array_equal(qx, g[f"qx{k}"]) and np.array_equal(qy, g[f"qy{k}"])


def _glibc_version():
    import ctypes
    try:
        libc = ctypes.CDLL("libc.so.6")
        libc.gnu_get_libc_version.restype = ctypes.c_char_p
        return tuple(int(v) for v in libc.gnu_get_libc_version().decode().split(".")[:2])
    except (OSError, AttributeError, ValueError):
        return None


def test_log1p_f32_is_the_c_library_log1pf():
    """The oracle's f32 log1p is the C library's log1pf bit for bit (the
    function NumPy calls for float32 log1p with its SIMD dispatch off), on
    display radii from 1e-10 to 1e6 AU and the reduction's branch points."""
    import ctypes
    ver = _glibc_version()
    if ver is None or ver > (2, 40):
        pytest.skip("the C library's log1pf here is not the fdlibm reduction")
    libm = ctypes.CDLL("libm.so.6")
    libm.log1pf.restype = ctypes.c_float
    libm.log1pf.argtypes = [ctypes.c_float]
    rng = np.random.default_rng(5)
    x = np.exp(rng.uniform(np.log(1e-10), np.log(1e6), 60_000)).astype(np.float32)
    edge = np.arange(0x3ED413D0, 0x3ED413E0, dtype=np.int32).view(np.float32)
    x = np.concatenate([x, edge, np.float32([0.0, 1e-9, 2e-9, 2.0**-29, 0.41421, 1.0, 3.0])])
    want = np.array([libm.log1pf(float(v)) for v in x], np.float32)
    assert np.array_equal(ofr.log1p_f32(x).view(np.int32), want.view(np.int32))


def test_hypot_f32_is_numpys():
    rng = np.random.default_rng(6)
    x = (rng.normal(0, 1, 200_000) * 10.0 ** rng.uniform(-9, 4, 200_000)).astype(np.float32)
    y = (rng.normal(0, 1, 200_000) * 10.0 ** rng.uniform(-9, 4, 200_000)).astype(np.float32)
    assert np.array_equal(ofr.hypot_f32(x, y), np.hypot(x, y))
