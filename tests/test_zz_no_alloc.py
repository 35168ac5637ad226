"""les_op_expand_noalloc: expand() for callers that cannot allocate device
memory (memory reserved up front, allocation-free regions, allocator
policies banning hidden allocations).  Its scratch is a static 16 MiB device
array; this checks, through the C ABI, that two calls in a row give the same
planes as les_op_expand (which allocates its scratch per call), and that a
call beyond the static capacity is refused instead of overrunning it.

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
