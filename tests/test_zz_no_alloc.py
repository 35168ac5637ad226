"""les_op_expand_noalloc: expand() for callers that cannot allocate device
memory (memory reserved up front, allocation-free regions, allocator
policies banning hidden allocations).  Its scratch is a static 16 MiB device
array; this checks, through the C ABI, that two calls in a row give the same
planes as les_op_expand (which allocates its scratch per call), that calls at
99.6% of the static capacity work and one plane more is refused instead of
overrunning it, and -- in a fresh process under lazy module loading -- that
after a first call the host may reserve all free device memory and later
calls still run without taking any.

Collected last (file name) so a stop-at-first-failure run has already run
every other test."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bind(L):
    f = L.les_op_expand_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                  ctypes.c_void_p]
    return f


def _expand(L, fn, a, nx, ny, howmany, rb):
    import torch
    out = torch.zeros((howmany, 3 * ny // 2, 3 * nx // 2), dtype=a.dtype, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    rc = fn(a.data_ptr(), out.data_ptr(), nx, ny, howmany, rb, s)
    assert rc == 0, L.les_op_last_error().decode()
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("rb", [8, 4])
def test_noalloc_expand_matches_allocating_expand_twice(gpu_lib, rb):
    import torch
    L = gpu_lib
    f = _bind(L)
    dt = torch.float64 if rb == 8 else torch.float32
    tol = 1e-12 if rb == 8 else 2e-5  # the tolerances of the expand parity tests
    rng = np.random.default_rng(rb)
    for (nx, ny, howmany) in ((64, 32, 3), (128, 128, 2)):  # two calls in a row, different shapes
        a = torch.tensor(rng.standard_normal((howmany, ny, nx)), dtype=dt, device="cuda")
        ref = _expand(L, L.les_op_expand, a, nx, ny, howmany, rb)
        got = _expand(L, f, a, nx, ny, howmany, rb)
        assert np.abs(got - ref).max() <= tol * np.abs(ref).max()


def test_noalloc_expand_refuses_oversize(gpu_lib):
    import torch
    L = gpu_lib
    f = _bind(L)
    # 512x512x8 planes need 8*256*(512+768)*16 B = 40 MiB > 16 MiB
    a = torch.zeros((1,), dtype=torch.float64, device="cuda")
    rc = f(a.data_ptr(), a.data_ptr(), 512, 512, 8, 8, None)
    assert rc == 1
    assert b"16 MiB" in L.les_op_last_error()


@pytest.mark.parametrize("rb", [8, 4])
def test_noalloc_expand_at_the_capacity_limit(gpu_lib, rb):
    """128x128 planes need (64*(128+192)) complex values each: 51 planes
    (rb 8) or 102 (rb 4) fill 99.6% of the 16 MiB, one more is refused."""
    import torch
    L = gpu_lib
    f = _bind(L)
    dt = torch.float64 if rb == 8 else torch.float32
    tol = 1e-12 if rb == 8 else 2e-5
    fit = 51 if rb == 8 else 102
    rng = np.random.default_rng(10 + rb)
    a = torch.tensor(rng.standard_normal((fit, 128, 128)), dtype=dt, device="cuda")
    ref = _expand(L, L.les_op_expand, a, 128, 128, fit, rb)
    for _ in range(2):
        got = _expand(L, f, a, 128, 128, fit, rb)
        assert np.abs(got - ref).max() <= tol * np.abs(ref).max()
    b = torch.zeros((fit + 1, 128, 128), dtype=dt, device="cuda")
    out = torch.zeros((fit + 1, 192, 192), dtype=dt, device="cuda")
    assert f(b.data_ptr(), out.data_ptr(), 128, 128, fit + 1, rb, None) == 1
    assert b"16 MiB" in L.les_op_last_error()


_RESERVE_SCRIPT = r"""
import ctypes, json, sys
import numpy as np
import torch
import importlib.util
spec = importlib.util.spec_from_file_location("les_gpu_host", %(root)r + "/paes-channelflow_b200/les_gpu.py")
P = importlib.util.module_from_spec(spec)
spec.loader.exec_module(P)
L = P.lib()
f = L.les_op_expand_noalloc
f.restype = ctypes.c_int
f.argtypes = [ctypes.c_void_p] * 2 + [ctypes.c_int] * 4 + [ctypes.c_void_p]
torch.cuda.init()
s = torch.cuda.current_stream().cuda_stream
# 1. the first call on this device, before any memory is reserved: it loads
#    the library's allocation-free module (scratch array and tables)
a0 = torch.zeros((1, 32, 32), dtype=torch.float64, device="cuda")
o0 = torch.zeros((1, 48, 48), dtype=torch.float64, device="cuda")
assert f(a0.data_ptr(), o0.data_ptr(), 32, 32, 1, 8, s) == 0
rng = np.random.default_rng(3)
a = torch.tensor(rng.standard_normal((51, 128, 128)), dtype=torch.float64, device="cuda")
out = torch.zeros((51, 192, 192), dtype=torch.float64, device="cuda")
torch.cuda.synchronize()
# 2. the host reserves all but 256 MiB of the free device memory
free0, total = torch.cuda.mem_get_info()
hold = torch.empty(max(free0 - (256 << 20), 0), dtype=torch.uint8, device="cuda")
torch.cuda.synchronize()
free1 = torch.cuda.mem_get_info()[0]
# 3. two calls at 99.6%% of the capacity run without taking device memory
rcs = []
for _ in range(2):
    rcs.append(f(a.data_ptr(), out.data_ptr(), 128, 128, 51, 8, s))
    torch.cuda.synchronize()
free2 = torch.cuda.mem_get_info()[0]
got = out.cpu().numpy()
del hold
torch.cuda.synchronize()
torch.cuda.empty_cache()
ref = torch.zeros_like(out)
assert L.les_op_expand(a.data_ptr(), ref.data_ptr(), 128, 128, 51, 8, s) == 0
torch.cuda.synchronize()
ref = ref.cpu().numpy()
print(json.dumps(dict(rcs=rcs, free_reserved=free1, free_after=free2,
                      err=float(np.abs(got - ref).max() / np.abs(ref).max()))))
"""


def test_noalloc_first_call_then_reserve_all_memory(gpu_lib):
    """In a fresh process: the first call, then the host reserves all free
    device memory but 256 MiB, then calls at the capacity limit still run,
    match les_op_expand and leave the free device memory unchanged."""
    import json
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ)
    env.pop("CUDA_MODULE_LOADING", None)  # the default: lazy loading
    r = subprocess.run([sys.executable, "-c", _RESERVE_SCRIPT % {"root": root}], capture_output=True, text=True,
                       timeout=600, env=env, cwd=root)
    assert r.returncode == 0, r.stderr[-2000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert res["rcs"] == [0, 0], res
    assert res["free_after"] == res["free_reserved"], res
    assert res["err"] <= 1e-12, res
