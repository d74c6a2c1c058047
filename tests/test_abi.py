"""The C ABI library loads and exports every symbol include/sss.h declares.

No compute call is made (no GPU needed).
"""
import ctypes
import os
import re

from solarsystemsimulator_b200 import _lib
from solarsystemsimulator_b200 import build as sss_build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "sss.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sss_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_api():
    syms = declared_symbols()
    assert "sss_create" in syms and "sss_allpairs_accel" in syms


def test_library_exports_every_declared_symbol():
    sss_build.build()
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(declared_symbols()) == set(_lib.SIGNATURES)


def test_abi_version():
    lib = _lib.load()
    assert lib.sss_abi_version() == 1


def test_library_built_for_sm100a():
    # the build flags pin the architecture; nvcc refuses an unknown arch
    assert "arch=compute_100a,code=sm_100a" in " ".join(sss_build.ARCH_FLAGS)
