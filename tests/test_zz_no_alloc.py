"""The no-allocation all-pairs entry point against the context entry point.

sss_allpairs_accel_noalloc serves callers that may not allocate device
memory (an application that owns the device-memory budget and passes the
library only pre-sized buffers, or a loop that cannot afford the blocking
cudaMalloc/cudaFree). It keeps its scratch in a fixed file-scope device
array. This test calls it through the C ABI twice in a row — the second call
finds the first call's leftovers in the shared array — and checks both
results against sss_allpairs_accel within the plain-f64 parity tolerance
(1e-12 per component of the force scale) and, in mixed precision, within
the same bound relative to the mixed result of the context path. It also
checks that sizes above the documented maximum are rejected.

The file is named to be collected last, so a run that stops at the first
failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _cloud(n, dim, seed):
    rng = np.random.default_rng(seed)
    rec = np.zeros((n, 4))
    rec[:, :dim] = rng.uniform(-0.5, 0.5, (n, dim))
    rec[:, 3] = rng.uniform(0.5, 1.5, n) / n
    return torch.from_numpy(rec).cuda()


def _close(a, ref, dim):
    a, ref = a[:, :dim], ref[:, :dim]
    scale = np.linalg.norm(ref, axis=1)[:, None]
    bound = TOL * np.maximum(np.abs(ref), scale)
    return bool(np.all(np.abs(a - ref) <= bound))


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("n_src,n_tgt", [(3000, 2000), (40000, 50000)])
def test_noalloc_matches_context_entry_point(precision, dim, n_src, n_tgt):
    from solarsystemsimulator_b200 import _lib
    lib = _lib.load()
    ctx = _lib.context(0)
    src = _cloud(n_src, dim, 1)
    tgt = _cloud(n_tgt, dim, 2)
    tgt[: min(n_src, n_tgt)] = src[: min(n_src, n_tgt)]
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    ref = torch.empty((n_tgt, 4), dtype=torch.float64, device="cuda")
    ctx.check(lib.sss_allpairs_accel(ctx.ptr, dim, precision, src.data_ptr(), n_src, tgt.data_ptr(),
                                     n_tgt, ref.data_ptr(), 1e-4, stream))
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    err = ctypes.create_string_buffer(256)
    outs = []
    for _ in range(2):
        out = torch.full((n_tgt, 4), float("nan"), dtype=torch.float64, device="cuda")
        rc = lib.sss_allpairs_accel_noalloc(0, dim, precision, src.data_ptr(), n_src, tgt.data_ptr(),
                                            n_tgt, out.data_ptr(), 1e-4, status.data_ptr(), stream,
                                            err, len(err))
        assert rc == 0, err.value.decode()
        outs.append(out)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    r = ref.cpu().numpy()
    for out in outs:
        assert _close(out.cpu().numpy(), r, dim)


def test_noalloc_rejects_sizes_beyond_maximum():
    from solarsystemsimulator_b200 import _lib
    lib = _lib.load()
    n_max = 1044480   # SSS_NOALLOC_MAX_MIXED_SOURCES
    src = torch.zeros((n_max + 1, 4), dtype=torch.float64, device="cuda")
    tgt = torch.zeros((4, 4), dtype=torch.float64, device="cuda")
    out = torch.zeros((4, 4), dtype=torch.float64, device="cuda")
    err = ctypes.create_string_buffer(256)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.sss_allpairs_accel_noalloc(0, 3, 1, src.data_ptr(), n_max + 1, tgt.data_ptr(), 4,
                                        out.data_ptr(), 1e-4, None, stream, err, len(err))
    assert rc == _lib.SSS_ERR_CAPACITY
    assert b"no-allocation scratch" in err.value
    # at the maximum it is accepted
    rc = lib.sss_allpairs_accel_noalloc(0, 3, 1, src.data_ptr(), n_max, tgt.data_ptr(), 4,
                                        out.data_ptr(), 1e-4, None, stream, err, len(err))
    assert rc == 0, err.value.decode()
    torch.cuda.synchronize()
