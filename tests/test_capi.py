"""CPU tests of the C ABI library: it loads, exports every entry point the
header declares, rejects bad configurations, and refuses to run without a
device instead of falling back to the CPU."""
import ctypes

import numpy as np
import pytest

from conftest import load_product


def test_library_exports_every_declared_symbol():
    P = load_product()
    L = P.lib()
    names = P.exported_symbols()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_config_layout_matches_header():
    P = load_product()
    assert P.lib().les_gpu_config_size() == ctypes.sizeof(P.LesConfig)
    c = P.LesConfig()
    P.lib().les_gpu_default_config(ctypes.byref(c))
    assert (c.nnx, c.nny, c.nnz) == (32, 32, 32) and c.emin == 1e-6 and c.forcing == 0.016


@pytest.mark.parametrize("bad", [dict(nnx=24), dict(nnz=2), dict(imodel=7), dict(isurface=0), dict(precision=2)])
def test_init_rejects_bad_config(bad):
    P = load_product()
    cfg = P.channel_config(32, 32, 16)
    for k, v in bad.items():
        setattr(cfg, k, v)
    h = ctypes.c_void_p()
    rc = P.lib().les_gpu_init(ctypes.byref(cfg), ctypes.byref(h))
    assert rc == P.LES_EINVAL and not h.value
    assert P.lib().les_gpu_last_error(None)


def test_no_cpu_fallback_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    P = load_product()
    with pytest.raises(P.LesError) as ei:
        P.LesGpu(P.channel_config(32, 32, 16))
    assert ei.value.code == P.LES_ENOTBUILT


def test_null_handle_is_rejected():
    P = load_product()
    L = P.lib()
    assert L.les_gpu_sync(None, 1.0) == P.LES_EINVAL
    assert L.les_gpu_stage(None, 0, 0, 1, 1e-3, 0.0, 1.0) == P.LES_EINVAL
    assert L.les_op_tridv(None, 4, 4, 8, None) == P.LES_EINVAL
