"""Small profiling case for ncu: one handle, the seeded initial field and a
few eager stages (no CUDA graph), so that every stage kernel appears as its
own launch.

    python paes-channelflow_b200/profile_case.py [precision=8|4] [n=256] [nz=32] [stages=2] [learned=0|1]

With learned=1 the handle uses the learned closure (imodel 5) with the
network in paes-channelflow_b200/weights/sgs_c4.npz (a seeded untrained
network if the file is absent), so the tensor-core kernel k_mlp_infer and
the other learned-stage kernels are launched too.  Prints the per-kernel
CUDA-event times of the last stage.
"""
import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    spec = importlib.util.spec_from_file_location("les_gpu_host", os.path.join(HERE, "les_gpu.py"))
    P = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(P)
    a = sys.argv[1:] + [None] * 5
    prec = int(a[0] or 8)
    n = int(a[1] or 256)
    nz = int(a[2] or 32)
    stages = int(a[3] or 2)
    learned = int(a[4] or 0)
    cfg = P.channel_config(n, n, nz, dt=1e-3, re_tau=590.0, precision=prec,
                           imodel=P.SGS_LEARNED if learned else P.SGS_DEARDORFF)
    g = P.LesGpu(cfg)
    m = None
    if learned:
        w = os.path.join(HERE, "weights", "sgs_c4.npz")
        if os.path.exists(w):
            z = np.load(w)
            m = P.Mlp(z["params"], z["norm"])
        else:
            rng = np.random.default_rng(0)
            shapes = [(64, 11), (64,), (64, 64), (64,), (64, 64), (64,), (6, 64), (6,)]
            p = np.concatenate([rng.standard_normal(sh).ravel() / np.sqrt(sh[-1]) if len(sh) == 2
                                else np.zeros(sh) for sh in shapes])
            m = P.Mlp(p)
        g.set_mlp(m, 590.0)
    g.make_ic(seed=12345, amp=0.1, re_tau=590.0)
    for s in range(stages):
        g.stage(0, False, s % 3 + 1)
    g.sync()
    for name, ms in g.profile_stage(2):
        print("%-40s %8.4f ms" % (name, ms))
    g.close()
    print("ok")


if __name__ == "__main__":
    main()
