"""A cupy -> numpy import shim, used ONLY by make_golden.py.

The reference's array-level code (backend/pm_kernel.py, the broadphase in
backend/film_producer.py, the NumPy oracles in backend/test_*.py) imports
cupy. With this shim installed as sys.modules["cupy"] it runs unmodified on
the CPU in f64 NumPy. Differences to CuPy that matter are pinned here:
argsort is stable (CuPy sorts stably), and asarray always copies (CuPy's
asarray of a host array is a device copy, so in-place updates on the
"device" array must not reach the caller's array).
"""
from __future__ import annotations

import sys
import types

import numpy as np


class _Device:
    def __init__(self, dev=0):
        self.id = dev

    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False

    def use(self):
        return self

    def synchronize(self):
        return None


class _Stream:
    def synchronize(self):
        return None


def install() -> types.ModuleType:
    cp = types.ModuleType("cupy")
    for name in dir(np):
        if not name.startswith("__"):
            setattr(cp, name, getattr(np, name))
    cp.asnumpy = lambda a, *args, **kw: np.asarray(a)
    cp.asarray = lambda a, dtype=None: np.array(a, dtype=dtype, copy=True)

    def argsort(a, axis=-1, *args, **kw):
        return np.argsort(a, axis=axis, kind="stable")

    cp.argsort = argsort
    cuda = types.ModuleType("cupy.cuda")
    cuda.Device = _Device
    cuda.Stream = types.SimpleNamespace(null=_Stream())
    runtime = types.ModuleType("cupy.cuda.runtime")
    runtime.getDeviceCount = lambda: 1
    runtime.getDeviceProperties = lambda d: {"name": b"cpu-shim", "major": 7, "minor": 0,
                                             "multiProcessorCount": 1, "clockRate": 1}
    cuda.runtime = runtime
    compiler = types.ModuleType("cupy.cuda.compiler")
    cuda.compiler = compiler
    cp.cuda = cuda
    sys.modules["cupy"] = cp
    sys.modules["cupy.cuda"] = cuda
    sys.modules["cupy.cuda.runtime"] = runtime
    sys.modules["cupy.cuda.compiler"] = compiler
    return cp
