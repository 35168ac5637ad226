"""The C++ host replay of les.F90 (tests/replay/les_replay.cpp): it calls
the library's C ABI in the order les.F90:146-357 calls the routines the
library replaces (init, initial field, per stage lower / upper / comp1 /
comprhs / press / comp2, compmn at mnout steps, restart files, finalize).

CPU: the driver compiles and links against include/ and libles_gpu.so.
GPU: its restart file after N steps equals, bit for bit, the state of the
Python host stepping the same split entry points, and matches the oracle
stepped from the same initial field."""
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import field_io as F
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "paes-channelflow_b200")
SRC = os.path.join(ROOT, "tests", "replay", "les_replay.cpp")
CUDA_LIB = "/usr/local/cuda/lib64"


def build(tmp):
    exe = os.path.join(str(tmp), "les_replay")
    cmd = ["/usr/bin/g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe,
           "-L", PKG, "-lles_gpu", "-Wl,-rpath," + PKG, "-L", CUDA_LIB, "-Wl,-rpath-link," + CUDA_LIB]
    subprocess.check_call(cmd)
    return exe


def test_replay_driver_builds_against_the_c_abi(tmp_path):
    if not os.path.exists(os.path.join(PKG, "libles_gpu.so")):
        pytest.skip("libles_gpu.so not built")
    exe = build(tmp_path)
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_replay_matches_python_host_and_oracle(gpu_lib, product, tmp_path):
    nx, ny, nz, re_tau, nsteps = 32, 32, 16, 180.0, 6
    exe = build(tmp_path)
    prefix = os.path.join(str(tmp_path), "rp")
    out = subprocess.run([exe, str(nx), str(ny), str(nz), str(re_tau), str(nsteps), "2", "3", prefix],
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    lines = out.stdout.strip().splitlines()
    dt = float(lines[-1].split()[1])
    stats = [list(map(float, l.split())) for l in lines[:-1]]
    assert [int(s[0]) for s in stats] == [0, 2, 4]
    assert all(s[3] < 1e-20 for s in stats)  # divz (squared divergence) at round-off
    h, f = F.read_field(prefix + "%d.field" % nsteps, real_bytes=8)
    assert (h["nnx"], h["nny"], h["nnz"]) == (nx, ny, nz)
    assert h["dt"] == dt
    # the Python host through the same split entry points
    g = product.LesGpu(product.channel_config(nx, ny, nz, dt=dt, re_tau=re_tau))
    g.make_ic(seed=12345, amp=0.1, re_tau=re_tau)
    assert g.cfl_dt(0.5) == dt
    for it in range(nsteps):
        for s in (1, 2, 3):
            g.stage_split(it, it % 2 == 0, s, dt=dt)
    d = g.download()
    for k in "uvwep":
        assert np.array_equal(f[k], d[k]), k
    # and the oracle from the same initial field
    o = O.Oracle(O.make_config(nx, ny, nz, dt=dt, re_tau=re_tau))
    o.make_ic(seed=12345, amp=0.1, re_tau=re_tau)
    o.set_dt(dt)
    o.step(0, nsteps, 2)
    fo = o.get_fields()
    scale = np.abs(fo["u"]).max()
    for k in "uvw":
        assert np.abs(f[k] - fo[k]).max() <= 1e-9 * scale, k
