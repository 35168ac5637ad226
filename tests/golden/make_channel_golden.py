"""Generates the channel parity fixtures from the oracle (oracle/, the CPU
restatement of the reference's RK3 stage) on the host cores.

    python tests/golden/make_channel_golden.py c1      # 64^3, 100 steps (~2 min)
    python tests/golden/make_channel_golden.py c2      # 128x128x96, 1000 steps (~1.5 h on 8 cores)

Cases (the channel of every configuration: Lx = 2 pi, Ly = pi, walls at
z = 0, 2, forcing 0.016, Deardorff SGS (imodel 3), wall model isurface 6,
tke_production off, FP64):
  c1: 64 x 64 x 64, Re_tau 180; snapshots after 10 and 100 steps.
  c2: 128 x 128 x 96, Re_tau 395; snapshots after 10, 100 and 1000 steps.
Initial field: the oracle's make_ic (parabolic mean of the log-law bulk
velocity plus seeded uniform(-0.1, 0.1) u_tau perturbations, e = 1e-4,
dealiased and projected), seed 12345; dt from the advective CFL 0.5 of that
field (les.F90:205-208), fixed for the run.  mnout at it = 0 and every 10th
step, as the GPU tests replay it.  Each snapshot holds channel_golden's
fingerprint, compmn's meanbuf and scalars and the u x-spectra of the sampled
levels; every step's post-projection divergence ratio is recorded.

Writes tests/golden/<case>.npz.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import channel_golden as G  # noqa: E402
from oracle import oracle as O  # noqa: E402

CASES = {
    "c1": dict(nx=64, ny=64, nz=64, re_tau=180.0, snaps=(10, 100)),
    "c2": dict(nx=128, ny=128, nz=96, re_tau=395.0, snaps=(10, 100, 1000)),
}
SEED, AMP, CFL, MNOUT_EVERY = 12345, 0.1, 0.5, 10


def run(case):
    c = CASES[case]
    cfg = O.make_config(c["nx"], c["ny"], c["nz"], dt=1e-3, re_tau=c["re_tau"])
    o = O.Oracle(cfg)
    o.make_ic(seed=SEED, amp=AMP, re_tau=c["re_tau"])
    dt = o.cfl_dt(CFL)
    o.set_dt(dt)
    f0 = o.get_fields()
    out = dict(dt=dt, re_tau=c["re_tau"], grid=np.array([c["nx"], c["ny"], c["nz"]]),
               ic_sum=np.array([f0[k].sum() for k in "uvwe"]),
               ic_sumsq=np.array([(f0[k] ** 2).sum() for k in "uvwe"]),
               snaps=np.array(c["snaps"]), mnout_every=MNOUT_EVERY, seed=SEED, amp=AMP)
    div = []
    t0 = time.time()
    for it in range(max(c["snaps"])):
        o.step(it, 1, MNOUT_EVERY)
        f = o.get_fields()
        div.append(G.divergence_ratio(f, cfg.xl, cfg.yl, cfg.zl))
        n = it + 1
        if n in c["snaps"]:
            fp = G.fingerprint(f)
            for k, a in fp.items():
                out["s%d_%s" % (n, k)] = a
            o.compmn()
            mb, sc = o.stats()
            out["s%d_meanbuf" % n] = mb
            out["s%d_scalars" % n] = sc
            out["s%d_xspec_u" % n] = np.array([G.xspectrum(f["u"][z]) for z in G.sample_levels(c["nz"])])
            print("%s: %d steps, %.1f s, max div ratio %.3e" % (case, n, time.time() - t0, max(div)), flush=True)
    out["div_ratio"] = np.array(div)
    np.savez_compressed(os.path.join(HERE, case + ".npz"), **out)


if __name__ == "__main__":
    for case in sys.argv[1:] or ["c1"]:
        run(case)
