"""TMA geometry of the L2 prefetches (csrc/les_tma.cuh), checked on the CPU.

k_y_inverse and k_y_forward prefetch column tiles with
cp.async.bulk.prefetch.tensor through 2-D tensor maps of real elements; a
tiled TMA copy whose innermost coordinate is not 16-byte aligned raises an
illegal instruction on B200, and a box holds at most 256 rows.  The tile's
column offset is cg*TC complex values, so TC complex values must be a
multiple of 16 bytes.  The test compiles tests/tma_geometry/geom.cu against
the kernels' own launch shapes (ColCfg, ColBox) and checks every grid length
the library dispatches in both precisions.  k_row_fused's row prefetch
(cp.async.bulk.prefetch.L2) wants 16-byte aligned rows of a multiple of 16
bytes: KX = NX/2 complex values."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "tma_geometry", "geom.cu")
CSRC = os.path.join(ROOT, "paes-channelflow_b200", "csrc")
NVCC = "/usr/local/cuda/bin/nvcc"
SIZES = [16, 32, 64, 96, 128, 192, 256, 384, 512]


def test_tma_prefetch_boxes_follow_the_alignment_rules(tmp_path):
    exe = os.path.join(str(tmp_path), "geom")
    subprocess.check_call([NVCC, "-std=c++17", "--expt-relaxed-constexpr", "-ccbin", "/usr/bin/g++",
                           "-gencode", "arch=compute_100a,code=sm_100a", "-I", CSRC, SRC, "-o", exe])
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    rows = [l.split() for l in out if l.strip()]
    assert len(rows) == 2 * 2 * len(SIZES)
    seen = set()
    for real, ns, which, tc, nb, br, ok, cxb in rows:
        real, ns, tc, nb, br, ok, cxb = map(int, (real, ns, tc, nb, br, ok, cxb))
        seen.add((real, ns, which))
        nrows = ns if which == "inverse" else 3 * ns // 2
        # every dispatched grid prefetches (ok), so the rules below apply to all
        assert ok == 1, (real, ns, which)
        assert nb * br == nrows and br <= 256, (real, ns, which, nb, br)
        assert (tc * cxb) % 16 == 0, (real, ns, which, tc)  # innermost coordinate 16-byte aligned
        assert 2 * tc <= 256  # box width in real elements
        assert (nb * br * tc * cxb) >= 64  # a non-empty tile
    assert seen == {(r, n, w) for r in (4, 8) for n in SIZES for w in ("inverse", "forward")}


def test_fused_row_prefetch_rows_are_16_byte_multiples():
    for nx in SIZES:
        kx = nx // 2
        for cxb in (8, 16):
            assert (kx * cxb) % 16 == 0, (nx, cxb)
