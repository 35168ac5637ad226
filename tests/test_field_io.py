"""Restart files in the reference's .field layout (read_write.f90:16-40,
les.F90:69-82 and 331-351).  CPU: the numpy restatement's byte layout is
pinned by hand-computed record lengths and round-trips; the C-ABI header
reader agrees with it.  GPU: files written by the library read back with
numpy equal the handle's state, and files written with numpy load into a
handle, in both real widths, synchronously and from the background writer."""
import struct

import numpy as np
import pytest

from oracle import field_io as F
from oracle import oracle as O


def _fields(nx, ny, nz, seed):
    rng = np.random.default_rng(seed)
    return {k: rng.standard_normal((nz, ny, nx)) for k in "uvwep"}


HDR = dict(time=12.5, xl=2 * np.pi, yl=np.pi, zl=2.0, dt=1e-3, z0=3e-4, utau=0.12)


@pytest.mark.parametrize("rb", [4, 8])
def test_layout_and_round_trip(tmp_path, rb):
    nx, ny, nz = 8, 6, 3
    f = _fields(nx, ny, nz, 1)
    path = str(tmp_path / "a.field")
    F.write_field(path, f, HDR, real_bytes=rb)
    raw = open(path, "rb").read()
    # record 1: real + 3 integers + 3 reals, framed by its length twice
    n1 = 4 * rb + 12
    assert struct.unpack_from("<i", raw, 0)[0] == n1 and struct.unpack_from("<i", raw, 4 + n1)[0] == n1
    assert struct.unpack_from("<3i", raw, 4 + rb) == (nx, ny, nz)
    lvl = 5 * nx * ny * rb
    total = (8 + n1) + (8 + 3 * rb) + (8 + 6 * rb) + nz * (8 + lvl)
    assert len(raw) == total
    h, g = F.read_field(path, real_bytes=rb)
    assert (h["nnx"], h["nny"], h["nnz"]) == (nx, ny, nz)
    for k in HDR:
        assert h[k] == pytest.approx(HDR[k], rel=1e-7 if rb == 4 else 0)
    for k in "uvwep":
        np.testing.assert_array_equal(g[k], f[k].astype(np.float32 if rb == 4 else np.float64))


def test_header_reader_of_the_library(tmp_path, product):
    path = str(tmp_path / "b.field")
    F.write_field(path, _fields(16, 8, 4, 2), HDR, real_bytes=8)
    dims, h = product.field_header(path, 8)
    assert dims == (16, 8, 4)
    for k in HDR:
        assert h[k] == HDR[k]
    with pytest.raises(product.LesError):
        product.field_header(path, 4)  # wrong real width: record lengths do not match


@pytest.mark.gpu
@pytest.mark.parametrize("rb,background", [(8, False), (8, True), (4, False)])
def test_gpu_write_then_numpy_read(gpu_lib, product, tmp_path, rb, background):
    cfg = product.channel_config(32, 16, 8, dt=2e-3, re_tau=180.0)
    cfg.ugal, cfg.vgal = 0.25, -0.125  # the Galilean shift the header must carry
    g = product.LesGpu(cfg)
    g.make_ic(seed=4, amp=0.3, re_tau=180.0)
    for it in range(2):
        g.step(it=it, mnout=False)
    path = str(tmp_path / "c.field")
    d = g.download(dtype=np.float64 if rb == 8 else np.float32)  # the state the file must hold
    g.write_field(path, time=3.0, real_bytes=rb, background=background)
    if background:
        g.step(it=2, mnout=False)  # keeps running while the file is written
        g.field_wait()
    h, f = F.read_field(path, real_bytes=rb)
    assert (h["nnx"], h["nny"], h["nnz"]) == (32, 16, 8) and h["time"] == 3.0
    assert h["dt"] == pytest.approx(2e-3, rel=1e-7) and h["utau"] > 0
    # the post-processing programs' shift formula (calc_pdf.f90:99-100)
    ugal = (max(0.0, max(h["ugtop"], h["ugbot"])) + min(0.0, min(h["ugtop"], h["ugbot"]))) * 0.5
    vgal = (max(0.0, max(h["vgtop"], h["vgbot"])) + min(0.0, min(h["vgtop"], h["vgbot"]))) * 0.5
    assert ugal == pytest.approx(0.25) and vgal == pytest.approx(-0.125)
    for k in "uvwep":
        np.testing.assert_array_equal(f[k], d[k])
    g.close()


@pytest.mark.gpu
def test_numpy_write_then_gpu_read(gpu_lib, product, tmp_path):
    o = O.Oracle(O.make_config(32, 16, 8, dt=2e-3))
    o.make_ic(seed=5, amp=0.3)
    f = o.get_fields()  # a dealiased field, as restart files hold
    path = str(tmp_path / "d.field")
    F.write_field(path, f, HDR, real_bytes=8)
    g = product.LesGpu(product.channel_config(32, 16, 8, dt=2e-3))
    assert g.read_field(path, 8) == HDR["time"]
    d = g.download()
    for k in "uvwe":
        np.testing.assert_allclose(d[k], f[k], rtol=0, atol=1e-12 * np.abs(f[k]).max())
    with pytest.raises(product.LesError):
        product.LesGpu(product.channel_config(16, 16, 8)).read_field(path, 8)  # other grid
