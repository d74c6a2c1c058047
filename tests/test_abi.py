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


def test_c_host_compiles_links_and_calls_without_gpu(tmp_path):
    """A plain C99 host (what a cgo or JNI binding compiles against) includes
    include/sss.h, links libsss.so and calls entry points that need no GPU;
    sss_create fails cleanly when no device is visible."""
    import shutil
    import subprocess
    cc = shutil.which("gcc")
    if cc is None:
        import pytest
        pytest.skip("no C compiler")
    sss_build.build()
    src = tmp_path / "host.c"
    src.write_text(
        '#include <stdio.h>\n#include "sss.h"\n'
        "int main(void) {\n"
        "    sss_ctx* ctx = 0;\n"
        "    int rc = sss_create(0, &ctx);\n"
        "    if (rc == SSS_OK) sss_destroy(ctx);\n"
        '    printf("%d %d %s\\n", sss_abi_version(), rc == SSS_OK || rc == SSS_ERR_CUDA || rc == SSS_ERR_ARG,\n'
        "           sss_last_error(0));\n"
        "    return 0;\n}\n")
    exe = tmp_path / "host"
    libdir = os.path.dirname(_lib.LIB_PATH)
    subprocess.run([cc, "-std=c99", "-Wall", "-Werror", "-pedantic", f"-I{os.path.join(ROOT, 'include')}",
                    str(src), f"-L{libdir}", "-lsss", f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True, timeout=120).stdout.split()
    assert out[0] == "1" and out[1] == "1" and " ".join(out[2:]) == "NULL context"
