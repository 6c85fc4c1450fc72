"""The allocation-free timestep reduction against the context-based one.

``mhd_timestep_noalloc`` exists for callers that cannot let the library
allocate device memory: code being captured into a CUDA graph (where
cudaMalloc is not allowed), embedders that own every device allocation
themselves, and real-time loops that must not enter the driver's allocator.
It keeps its scratch in a fixed file-scope device array instead of a
context's workspace, so it must give exactly the result of ``mhd_timestep``
(a minimum is exact), call after call, since every call reuses that array.

The file is named to be collected last: a failure here leaves every other
test already run.
"""

import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _ctx(lib, _abi, n_max):
    p = _abi.make_params(3, "cubic", 1.2, 5.0 / 3.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, [0, 0, 0], [1, 1, 1],
                         [True] * 3)
    ctx = ctypes.c_void_p()
    _abi.check(lib.mhd_ctx_create(ctypes.byref(p), n_max, ctypes.byref(ctx)))
    return ctx


def _with_context(lib, _abi, ctx, dt_adapt, t, tf):
    """dt from the existing entry point (the context's tf is set to ``tf``)."""
    p = _abi.make_params(3, "cubic", 1.2, 5.0 / 3.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, tf, [0, 0, 0], [1, 1, 1],
                         [True] * 3)
    _abi.check(lib.mhd_ctx_set_params(ctx, ctypes.byref(p)), ctx)
    s = _abi.state_type()()
    s.dt_adapt = ctypes.c_void_p(dt_adapt.data_ptr())
    dt = ctypes.c_double()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _abi.check(lib.mhd_timestep(ctx, ctypes.byref(s), dt_adapt.numel(), t, ctypes.byref(dt), stream), ctx)
    return dt.value


def _without_allocation(lib, dt_adapt, t, tf):
    out = torch.full((1,), -1.0, dtype=torch.float64, device=dt_adapt.device)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.mhd_timestep_noalloc(ctypes.c_void_p(dt_adapt.data_ptr()), dt_adapt.numel(), t, tf,
                                  ctypes.c_void_p(out.data_ptr()), stream)
    assert rc == 0, lib.mhd_last_error(None)
    return float(out.item())


def test_noalloc_timestep_matches_context_timestep_on_consecutive_calls():
    from src import _abi

    lib = _abi.load()
    torch.cuda.set_device(0)
    gen = torch.Generator(device="cuda").manual_seed(7)
    ctx = _ctx(lib, _abi, 1 << 21)
    try:
        # call 1: two million values, no clip
        a = torch.rand(2_000_003, dtype=torch.float64, device="cuda", generator=gen) * 1e-3 + 1e-6
        ref1 = _with_context(lib, _abi, ctx, a, 0.0, 1e30)
        got1 = _without_allocation(lib, a, 0.0, 1e30)
        assert got1 == ref1 == float(a.min())
        # call 2 on the same scratch: fewer blocks than call 1, and the tf clip applies
        b = torch.rand(4099, dtype=torch.float64, device="cuda", generator=gen) * 1e-2 + 1e-4
        tf = 1.0
        t = tf - 0.5 * float(b.min())
        ref2 = _with_context(lib, _abi, ctx, b, t, tf)
        got2 = _without_allocation(lib, b, t, tf)
        assert got2 == ref2 == tf - t
    finally:
        lib.mhd_ctx_destroy(ctx)


def test_noalloc_timestep_rejects_oversize_and_flags_invalid_steps():
    from src import _abi

    lib = _abi.load()
    dummy = torch.ones(4, dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = lib.mhd_timestep_noalloc(ctypes.c_void_p(dummy.data_ptr()), _abi.NOALLOC_MAX_N + 1, 0.0, 1.0,
                                  ctypes.c_void_p(out.data_ptr()), None)
    assert rc == -1 and b"MHD_NOALLOC_MAX_N" in lib.mhd_last_error(None)
    bad = torch.tensor([1e-3, 0.0, 2e-3], dtype=torch.float64, device="cuda")
    assert np.isnan(_without_allocation(lib, bad, 0.0, 1.0))


_FRESH_PROCESS = r"""
import ctypes, sys
import torch
sys.path[:0] = sys.argv[1:]
from src import _abi
lib = _abi.load()
torch.cuda.set_device(0)
gen = torch.Generator(device="cuda").manual_seed(11)
side = torch.cuda.Stream()  # non-blocking with respect to the legacy default stream
out = torch.full((2,), -1.0, dtype=torch.float64, device="cuda")
with torch.cuda.stream(side):
    a = torch.rand(3_000_017, dtype=torch.float64, device="cuda", generator=gen) + 1e-3
    b = torch.rand(70_001, dtype=torch.float64, device="cuda", generator=gen) + 1e-3
    st = ctypes.c_void_p(side.cuda_stream)
    for k, v in enumerate((a, b)):
        rc = lib.mhd_timestep_noalloc(ctypes.c_void_p(v.data_ptr()), v.numel(), 0.0, 1e30,
                                      ctypes.c_void_p(out[k:].data_ptr()), st)
        assert rc == 0, lib.mhd_last_error(None)
side.synchronize()
assert float(out[0]) == float(a.min()) and float(out[1]) == float(b.min()), (out.tolist(), float(a.min()), float(b.min()))
print("FRESH_OK")
"""


def test_noalloc_first_calls_on_a_nonblocking_stream_in_a_fresh_process():
    """The first two calls of a process, both on a stream that does not wait
    for the legacy default stream: the scratch needs no set-up work ordered
    before them."""
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    res = subprocess.run([sys.executable, "-c", _FRESH_PROCESS, root, os.path.join(root, "pysph-mhd_b200")],
                         capture_output=True, text=True, timeout=300)
    assert res.returncode == 0 and "FRESH_OK" in res.stdout, res.stdout + res.stderr


def test_noalloc_timestep_large_input_with_ragged_tail():
    """About 10^7 values (610 blocks, the last one partly filled), twice in a
    row, against torch's own minimum."""
    from src import _abi

    lib = _abi.load()
    gen = torch.Generator(device="cuda").manual_seed(5)
    n = 10_000_019
    assert n % 16384 and n // 16384 < 4096
    for _ in range(2):
        a = torch.rand(n, dtype=torch.float64, device="cuda", generator=gen) + 1e-4
        a[n - 3] = 1e-6  # the minimum in the ragged tail
        assert _without_allocation(lib, a, 0.0, 1e30) == float(a.min()) == 1e-6
