"""A-posteriori comparison of the precision forms and closures against the
FP64 Deardorff run on one grid, from the same seeded initial field
(make_ic: parabolic mean plus uniform(-0.1, 0.1) u_tau perturbations,
projected), isurface 6, fixed dt from CFL 0.5 of the initial field.

    python paes-channelflow_b200/aposteriori.py --grid 512 512 256 --re-tau 590 --steps 5000 --every 500
        [--forms mixed,learned,learned_sign_only] [--weights paes-channelflow_b200/weights/sgs_c4.npz]
        [--out aposteriori.json]

Forms (each against the FP64 Deardorff run):
  mixed              FP32 transforms / advection / SGS, FP64 pressure,
                     mean modes and reductions, Deardorff closure;
  learned            the mixed form with the learned closure and the
                     library's default fallback test (sign, and a factor 4
                     of the Smagorinsky estimate);
  learned_sign_only  the same with the sign test only.
With --ref-production the FP64 reference and the mixed form add the TKE
shear production the shipped Deardorff model lacks (a physically complete
Deardorff LES); the learned forms keep the shipped TKE equation.
At every checkpoint: the largest |U - U_fp64| over U_b, the largest <u'w'>
and u_rms differences over their FP64 maxima, the largest relative
difference of the u x-spectra (spectra2.f90:24-32) over the resolved band
kx = 1..nx/3 at the levels nearest z+ = 15 and 100, and for the learned
forms the fraction of stages so far that used the network.
"""
import argparse
import importlib.util
import json
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def load():
    spec = importlib.util.spec_from_file_location("les_gpu_host", os.path.join(HERE, "les_gpu.py"))
    P = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(P)
    return P


def spec_levels(nz, re_tau, zl=2.0):
    return sorted({max(1, int(round(zp / (zl / nz * re_tau) + 0.5))) for zp in (15.0, 100.0)})


def run(P, grid, re_tau, precision, imodel, steps, every, dt=None, mlp=None, guard=None, log=print, production=0):
    """Checkpoints of one form: {step: (U, <u'w'>, u_rms, {level: u x-spectrum})}
    and the learned closure's (stages, used) counters per checkpoint."""
    nx, ny, nz = grid
    cfg = P.channel_config(nx, ny, nz, dt=1e-3, re_tau=re_tau, precision=precision, imodel=imodel,
                           tke_production=production)
    g = P.LesGpu(cfg)
    if mlp is not None:
        g.set_mlp(mlp, re_tau)
        if guard is not None:
            g.set_learned_guard(guard)
    g.make_ic(seed=12345, amp=0.1, re_tau=re_tau)
    if dt is None:
        dt = g.cfl_dt(0.5)
    levels = spec_levels(nz, re_tau)
    out, counts = {}, {}
    t0 = time.time()
    for it in range(1, steps + 1):
        mn = (it % every == 0)
        g.step(it=it, mnout=mn, dt=dt)
        if mn:
            mb, _ = g.stats()
            out[it] = (mb[3].copy(), mb[9].copy(), np.sqrt(np.maximum(mb[6], 0)),
                       {iz: g.spectra(0, iz)[0] for iz in levels})
            if mlp is not None:
                counts[it] = g.learned_counts() + (g.learned_status()[1], g.learned_reference())
            log("  step %d (%.0f s)%s" % (it, time.time() - t0, "" if mlp is None else " counts %s" % (counts[it],)))
    g.sync()
    g.close()
    return out, counts, dt


def averaged(prof, ref, steps):
    """Profiles averaged over the checkpoints of the second half of the run
    (a statistical comparison: the instantaneous fields of two turbulent
    runs decorrelate once round-off differences have grown)."""
    keys = [it for it in sorted(prof) if it > steps // 2 and it in ref]
    if not keys:
        return {}
    avg = lambda d, j: np.mean([d[it][j] for it in keys], axis=0)
    U, uw, ur = avg(prof, 0), avg(prof, 1), avg(prof, 2)
    U0, uw0, ur0 = avg(ref, 0), avg(ref, 1), avg(ref, 2)
    ub = float(np.mean(U0))
    return {"checkpoints": len(keys), "from_step": keys[0], "to_step": keys[-1],
            "mean_u_max_err_over_ub": float(np.abs(U - U0).max() / ub),
            "uw_max_err_over_max": float(np.abs(uw - uw0).max() / max(np.abs(uw0).max(), 1e-300)),
            "u_rms_max_err_over_max": float(np.abs(ur - ur0).max() / max(ur0.max(), 1e-300))}


def compare(prof, ref, counts, dt, nx):
    rows = []
    kmax = nx // 3
    for it in sorted(prof):
        U, uw, ur, sp = prof[it]
        U0, uw0, ur0, sp0 = ref[it]
        ub = float(np.mean(U0))
        spec = {}
        for iz, s in sp.items():
            s0 = sp0[iz]
            spec["u_xspec_level%d" % iz] = float(np.max(np.abs(s[1:kmax] - s0[1:kmax]) /
                                                        np.maximum(s0[1:kmax], 1e-300)))
        r = {"step": it, "time": it * dt, "mean_u_max_err_over_ub": float(np.abs(U - U0).max() / ub),
             "uw_max_err_over_max": float(np.abs(uw - uw0).max() / max(np.abs(uw0).max(), 1e-300)),
             "u_rms_max_err_over_max": float(np.abs(ur - ur0).max() / max(ur0.max(), 1e-300)), **spec}
        if it in counts:
            st, used, dis, dref = counts[it]
            r.update(stages=st, stages_used=used, used_fraction=used / max(st, 1),
                     last_network_dissipation=dis, last_reference_dissipation=dref)
        rows.append(r)
    return rows


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", type=int, nargs=3, default=[512, 512, 256])
    ap.add_argument("--re-tau", type=float, default=590.0)
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--every", type=int, default=500)
    ap.add_argument("--forms", default="mixed,learned,learned_sign_only",
                    help="comma list of mixed, learned, learned_sign_only, learned_guard<factor>")
    ap.add_argument("--weights", default=os.path.join(HERE, "weights", "sgs_c4.npz"))
    ap.add_argument("--out", default="aposteriori.json")
    ap.add_argument("--ref-production", action="store_true",
                    help="the FP64 Deardorff reference (and the mixed form) with the TKE shear production "
                         "term the shipped model lacks (tke_production = 1); the learned forms keep the "
                         "shipped TKE equation")
    a = ap.parse_args(argv)
    P = load()
    forms = a.forms.split(",")
    mlp = None
    if any(f.startswith("learned") for f in forms):
        z = np.load(a.weights)
        mlp = P.Mlp(z["params"], z["norm"])
    print("fp64 Deardorff")
    ref, _, dt = run(P, a.grid, a.re_tau, P.PREC_FP64, P.SGS_DEARDORFF, a.steps, a.every,
                     production=int(a.ref_production))
    res = {"grid": a.grid, "re_tau": a.re_tau, "dt": dt, "steps": a.steps, "every": a.every,
           "reference_tke_production": int(a.ref_production),
           "spectrum_levels": spec_levels(a.grid[2], a.re_tau), "weights": os.path.basename(a.weights),
           "forms": {}}
    for name in forms:
        print(name)
        try:
            if name == "mixed":
                r = run(P, a.grid, a.re_tau, P.PREC_MIXED, P.SGS_DEARDORFF, a.steps, a.every, dt,
                        production=int(a.ref_production))
            elif name == "learned":
                r = run(P, a.grid, a.re_tau, P.PREC_MIXED, P.SGS_LEARNED, a.steps, a.every, dt, mlp)
            elif name == "learned_sign_only":
                r = run(P, a.grid, a.re_tau, P.PREC_MIXED, P.SGS_LEARNED, a.steps, a.every, dt, mlp, 0.0)
            elif name.startswith("learned_guard"):
                r = run(P, a.grid, a.re_tau, P.PREC_MIXED, P.SGS_LEARNED, a.steps, a.every, dt, mlp,
                        float(name[len("learned_guard"):]))
            else:
                raise ValueError(name)
            res["forms"][name] = compare(r[0], ref, r[1], dt, a.grid[0])
            res.setdefault("second_half_average", {})[name] = averaged(r[0], ref, a.steps)
        except P.LesError as e:  # e.g. a run that blew up (LES_ENAN): recorded, the others still run
            res["forms"][name] = {"failed": str(e)}
        with open(a.out, "w") as f:
            json.dump(res, f, indent=1)
    for name, rows in res["forms"].items():
        for r in (rows if isinstance(rows, list) else [rows]):
            print(name, json.dumps(r))
    for name, r in res.get("second_half_average", {}).items():
        print("second-half average", name, json.dumps(r))


if __name__ == "__main__":
    main()
