"""A-posteriori comparison at the production grid: the FP64 Deardorff run, the
mixed-precision Deardorff run and the mixed-precision learned-closure run
from the same seeded initial field (512x512x256, Re_tau 590, isurface 6,
fixed dt from CFL 0.5 of the initial field), with the mean-velocity profile,
<u'w'> and u_rms of the mixed forms compared with the FP64 run every
`every` steps.

    python paes-channelflow_b200/aposteriori_c5.py [steps=1500] [every=250] [out=aposteriori_c5.json]

Writes one JSON file: per checkpoint step, for each mixed form, the largest
|U - U_fp64| over U_b, the largest <u'w'> and u_rms differences over their
FP64 maxima, and for the learned forms (default fallback test, and the sign
test only) the last stage's (flag, network dissipation, Deardorff
dissipation).
"""
import importlib.util
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NX = NY = 512
NZ = 256
RE_TAU = 590.0


def load():
    spec = importlib.util.spec_from_file_location("les_gpu_host", os.path.join(HERE, "les_gpu.py"))
    P = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(P)
    return P


def run(P, precision, imodel, steps, every, dt=None, mlp=None, guard=None):
    """Mean-profile rows (U, <u'w'>, u_rms) at every checkpoint of one form;
    guard: the learned closure's fallback factor (None: the default)."""
    cfg = P.channel_config(NX, NY, NZ, dt=1e-3, re_tau=RE_TAU, precision=precision, imodel=imodel)
    g = P.LesGpu(cfg)
    if mlp is not None:
        g.set_mlp(mlp, RE_TAU)
        if guard is not None:
            g.set_learned_guard(guard)
    g.make_ic(seed=12345, amp=0.1, re_tau=RE_TAU)
    if dt is None:
        dt = g.cfl_dt(0.5)
    out, used = {}, {}
    for it in range(1, steps + 1):
        mn = (it % every == 0)
        g.step(it=it, mnout=mn, dt=dt)
        if mn:
            mb, _ = g.stats()
            out[it] = (mb[3].copy(), mb[9].copy(), np.sqrt(np.maximum(mb[6], 0)))
            if mlp is not None:
                u_, d_ = g.learned_status()
                used[it] = (u_, d_, g.learned_deardorff())
    g.sync()
    g.close()
    return out, used, dt


def main():
    a = sys.argv[1:] + [None] * 3
    steps = int(a[0] or 1500)
    every = int(a[1] or 250)
    path = a[2] or "aposteriori_c5.json"
    P = load()
    z = np.load(os.path.join(HERE, "weights", "sgs_c4.npz"))
    mlp = P.Mlp(z["params"], z["norm"])
    ref, _, dt = run(P, P.PREC_FP64, P.SGS_DEARDORFF, steps, every)
    forms = {"mixed_deardorff": run(P, P.PREC_MIXED, P.SGS_DEARDORFF, steps, every, dt),
             "learned_mixed": run(P, P.PREC_MIXED, P.SGS_LEARNED, steps, every, dt, mlp),
             "learned_mixed_sign_test_only": run(P, P.PREC_MIXED, P.SGS_LEARNED, steps, every, dt, mlp, 0.0)}
    res = {"grid": [NX, NY, NZ], "re_tau": RE_TAU, "dt": dt, "steps": steps, "every": every, "forms": {}}
    for name, (prof, used, _) in forms.items():
        rows = []
        for it in sorted(prof):
            U, uw, ur = prof[it]
            U0, uw0, ur0 = ref[it]
            ub = float(np.mean(U0))
            rows.append({"step": it, "time": it * dt,
                         "mean_u_max_err_over_ub": float(np.abs(U - U0).max() / ub),
                         "uw_max_err_over_max": float(np.abs(uw - uw0).max() / max(np.abs(uw0).max(), 1e-300)),
                         "u_rms_max_err_over_max": float(np.abs(ur - ur0).max() / max(ur0.max(), 1e-300)),
                         "learned_used": used.get(it)})
        res["forms"][name] = rows
    with open(path, "w") as f:
        json.dump(res, f, indent=1)
    for name, rows in res["forms"].items():
        for r in rows:
            print(name, r["step"], "%.4g %.4g %.4g" % (r["mean_u_max_err_over_ub"], r["uw_max_err_over_max"],
                                                       r["u_rms_max_err_over_max"]), r["learned_used"])


if __name__ == "__main__":
    main()
