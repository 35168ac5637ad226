"""Small profiling case for ncu: one handle, the seeded initial field and a
few eager stages (no CUDA graph), so that every stage kernel appears as its
own launch.

    python paes-channelflow_b200/profile_case.py [precision=8|4] [n=256] [nz=32] [stages=2]
"""
import importlib.util
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    spec = importlib.util.spec_from_file_location("les_gpu_host", os.path.join(HERE, "les_gpu.py"))
    P = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(P)
    a = sys.argv[1:] + [None] * 4
    prec = int(a[0] or 8)
    n = int(a[1] or 256)
    nz = int(a[2] or 32)
    stages = int(a[3] or 2)
    cfg = P.channel_config(n, n, nz, dt=1e-3, re_tau=590.0, precision=prec)
    g = P.LesGpu(cfg)
    g.make_ic(seed=12345, amp=0.1, re_tau=590.0)
    for s in range(stages):
        g.stage(0, False, s % 3 + 1)
    g.sync()
    print("ok")


if __name__ == "__main__":
    main()
