"""Training of the learned sub-grid closure on one GPU.

    python paes-channelflow_b200/train_closure.py [--fine 384 384 192] [--factor 4 2]
        [--re-tau 395] [--snapshots 200] [--spinup 14000] [--every 40] [--epochs 20]
        [--aposteriori 4000] [--out paes-channelflow_b200/weights/sgs_c4]

1. A fine run of this solver (Deardorff closure) from the log-law mean
   profile of the wall model plus random perturbations (small-scale noise
   and large structures, which make the flow transition within a few eddy
   turnovers); the spin-up runs in the mixed form, then the state moves to
   an FP64 handle for the data.
2. After the spin-up, every `every` steps: les_gpu_learn_filter onto the
   coarse grid (box filter: `fxy` fine cells in x, y and `fz` in z) gives
   the filtered u, v, w and tau_ij = filt(u_i u_j) - filt(u_i) filt(u_j)
   plus (by default) the filtered Deardorff stress of the fine run itself,
   i.e. the total sub-filter stress the coarse grid misses (without it the
   targets lack the momentum flux the fine run's model carries near the
   walls, and coarse runs with the network lose their near-wall velocity);
   the filtered fields are loaded into a coarse handle whose
   les_gpu_learned_features computes the network inputs with the same
   kernels the learned stage uses.
3. Normalisation (mean / standard deviation per input and output) from the
   training snapshots; the last `holdout` fraction of snapshots is held out.
4. Adam (lr 1e-3, batch 65536, f32 master weights) on the tensor-core
   kernels (les_mlp_adam_step), shuffled batches, `epochs` passes.
5. A-priori evaluation on the held-out snapshots: per-component
   correlation coefficient and normalised MSE of the deviatoric stresses,
   for the network and for the Deardorff eddy viscosity
   tau_ij^dev = -2 (0.1 Delta sqrt(e)) S_ij with the filtered e = tau_kk / 2.
6. A-posteriori (optional): coarse runs from the first filtered snapshot
   with the Deardorff closure and with the network; mean U(z) against the
   filtered fine run's mean profile.
7. Writes <out>.npz (params, norm, re_tau, grids), <out>.json (report) and
   <out>_eval.npz (the first filtered snapshot and the filtered fine run's
   mean profile; --evaluate repeats step 6 from it).
"""
import argparse
import importlib.util
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _host():
    name = "les_gpu_host"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(HERE, "les_gpu.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def loglaw_field(cfg, amp, seed, large=0.0, utau=float(np.sqrt(0.016)), kappa=0.4, kmax=4):
    """Initial field of the training run: the log-law mean profile of the
    wall model, U = (u_tau / kappa) ln(z_wall / z0), plus uniform(-amp,
    amp) u_tau noise on u, v, w, plus (large > 0) a random field of the
    modes |kx|, |ky| <= kmax with standard deviation large * U_bulk times
    sin(pi z / zl) on each component; w = 0 on the top level.  The first
    projection of the run makes the field solenoidal."""
    nx, ny, nz = cfg.nnx, cfg.nny, cfg.nnz
    dz = cfg.zl / nz
    zc = (np.arange(nz) + 0.5) * dz
    zw = np.minimum(zc, cfg.zl - zc)
    U = utau / kappa * np.log(np.maximum(zw / cfg.z0, 1.0))
    rng = np.random.default_rng(seed)
    noise = lambda: rng.uniform(-amp, amp, (nz, ny, nx)) * utau
    u = U[:, None, None] + noise()
    v = noise()
    w = noise()
    if large > 0:
        env = np.sin(np.pi * zc / cfg.zl)[:, None, None]
        kx = np.arange(nx // 2 + 1)[None, None, :]
        ky = np.abs(np.fft.fftfreq(ny, 1.0 / ny))[None, :, None]
        keep = (kx <= kmax) & (ky <= kmax)
        for a in (u, v, w):
            f = np.fft.irfft2(np.fft.rfft2(rng.standard_normal((nz, ny, nx))) * keep, s=(ny, nx))
            a += large * U.mean() * env * f / f.std()
    w[-1] = 0.0
    e = np.full((nz, ny, nx), 1e-4)
    return u, v, w, e


def collect(fine=(384, 384, 192), factor=(4, 2), re_tau=395.0, snapshots=200, spinup=14000, every=40, amp=1.0,
            large=0.3, seed=12345, cfl=0.5, spinup_precision=4, with_model=True, log=print):
    """Run the fine case and return (features f32 (S, Nc, 16), targets f64
    (S, Nc, 6), info, first filtered (u, v, w)) with the sample arrays as
    CUDA tensors."""
    import torch
    P = _host()
    nx, ny, nz = fine
    fxy, fz = factor
    t0 = time.time()
    cfg = P.channel_config(nx, ny, nz, dt=1e-3, re_tau=re_tau, precision=spinup_precision)
    g = P.LesGpu(cfg)
    u, v, w, e = loglaw_field(cfg, amp, seed, large)
    g.upload(u, v, w, e, None)
    del u, v, w, e
    dt = g.cfl_dt(cfl)
    state = {"it": 0}
    hist = []

    def monitor(h, tag):
        mb, sc = h.stats()
        it = state["it"]
        rec = dict(step=it, t=it * dt, utau=float(sc[0]), u_rms_max=float(np.sqrt(np.maximum(mb[6], 0.0)).max()),
                   uw_quarter=float(mb[9][nz // 8]), uw_half=float(mb[9][nz // 4]))
        hist.append(rec)
        log("%s step %d t=%.1f (%.0f s): utau %.4f, max u_rms %.4f, <u'w'>(z=.25) %.5f" %
            (tag, it, it * dt, time.time() - t0, rec["utau"], rec["u_rms_max"], rec["uw_quarter"]))

    nmon = max(1, spinup // 10)
    for _ in range(spinup):
        g.step(it=state["it"], mnout=False, dt=dt)
        state["it"] += 1
        if state["it"] % nmon == 0:
            monitor(g, "spin-up")
    if spinup_precision != 8:
        f = g.download()
        g.close()
        cfg = P.channel_config(nx, ny, nz, dt=dt, re_tau=re_tau, precision=8)
        g = P.LesGpu(cfg)
        g.upload(f["u"], f["v"], f["w"], f["e"], f["p"])
        del f
    ccfg = P.channel_config(nx // fxy, ny // fxy, nz // fz, dt=dt, re_tau=re_tau, precision=8)
    ccfg.z0 = cfg.z0
    c = P.LesGpu(ccfg)
    nc = (nx // fxy) * (ny // fxy) * (nz // fz)
    feats = torch.empty((snapshots, nc, 16), dtype=torch.float32, device="cuda")
    targs = torch.empty((snapshots, nc, 6), dtype=torch.float64, device="cuda")
    fine_means = []
    first = None
    for s in range(snapshots):
        if s > 0:
            for _ in range(every):
                g.step(it=state["it"], mnout=False, dt=dt)
                state["it"] += 1
        out = g.learn_filter(fxy, fz, with_model=with_model)
        uvw = out[:3].cpu().numpy()
        if first is None:
            first = uvw.copy()
        c.upload(uvw[0], uvw[1], uvw[2], np.full_like(uvw[0], 1e-4), None)
        feats[s] = c.learned_features(re_tau)
        targs[s] = out[3:].reshape(6, nc).t()
        fine_means.append(uvw[0].mean(axis=(1, 2)))
        if s == 0 or (s + 1) % max(1, snapshots // 10) == 0:
            monitor(g, "snapshot %d/%d" % (s + 1, snapshots))
    g.sync()
    info = dict(fine=list(fine), factor=list(factor), re_tau=re_tau, snapshots=snapshots, spinup=spinup,
                spinup_precision=spinup_precision, every=every, amp=amp, large=large, seed=seed, dt=dt,
                targets="filtered total sub-filter stress" if with_model else "filtered minus resolved products",
                steps=state["it"], coarse=[nx // fxy, ny // fxy, nz // fz], history=hist,
                collect_seconds=time.time() - t0, filtered_mean_u=np.mean(fine_means, axis=0).tolist(), z0=cfg.z0)
    g.close()
    c.close()
    return feats, targs, info, first


def normalisation(feats, targs):
    """in_shift, in_scale per input, out_scale, out_shift per output (34
    floats); a constant input (the filter width on one grid) gets scale 0."""
    import torch
    f = feats.reshape(-1, 16)[:, :11].double()
    t = targs.reshape(-1, 6)
    fm, fs = f.mean(0), f.std(0)
    tm, ts = t.mean(0), t.std(0)
    in_scale = torch.where(fs > 1e-6 * (fm.abs() + 1e-30), 1.0 / fs, torch.zeros_like(fs))
    norm = np.concatenate([fm.cpu().numpy(), in_scale.cpu().numpy(), ts.cpu().numpy(), tm.cpu().numpy()])
    return norm.astype(np.float32)


def to_training(feats, targs, norm):
    """bf16 normalised features (N, 16) and f32 normalised targets (N, 8)."""
    import torch
    n = torch.from_numpy(norm.astype(np.float64)).to(feats.device)
    f = feats.reshape(-1, 16).double()
    x = torch.zeros_like(f)
    x[:, :11] = (f[:, :11] - n[:11]) * n[11:22]
    t = targs.reshape(-1, 6)
    y = torch.zeros((t.shape[0], 8), dtype=torch.float32, device=t.device)
    y[:, :6] = ((t - n[28:34]) / n[22:28]).float()
    return x.to(torch.bfloat16).contiguous(), y.contiguous()


def init_params(seed=0):
    """Seeded initial parameters: weights N(0, 1/fan_in), biases 0."""
    rng = np.random.default_rng(seed)
    shapes = [(64, 11), (64,), (64, 64), (64,), (64, 64), (64,), (6, 64), (6,)]
    out = []
    for sh in shapes:
        if len(sh) == 2:
            out.append(rng.standard_normal(sh).ravel() / np.sqrt(sh[1]))
        else:
            out.append(np.zeros(sh))
    p = np.concatenate(out).astype(np.float32)
    assert p.size == 9478
    return p


def train(mlp, x, y, epochs=20, batch=65536, lr=1e-3, seed=0, log=print):
    import torch
    gen = torch.Generator(device=x.device)
    gen.manual_seed(seed)
    n = x.shape[0]
    nb = max(1, n // batch)
    hist = []
    step = 0
    t0 = time.time()
    for ep in range(epochs):
        perm = torch.randperm(n, device=x.device, generator=gen)
        for b in range(nb):
            idx = perm[b * batch:(b + 1) * batch]
            want = (b == nb - 1) or (b % 200 == 0)
            loss = mlp.adam_step(x[idx].contiguous(), y[idx].contiguous(), lr=lr, want_loss=want)
            if want:
                hist.append((step, loss))
            step += 1
        log("epoch %d: loss %.5f (%d steps, %.1f s)" % (ep + 1, hist[-1][1], step, time.time() - t0))
    torch.cuda.synchronize()
    return hist, step, time.time() - t0


def deviatoric(t):
    """(N, 6) stresses -> deviatoric (trace removed from the diagonal)."""
    d = t.clone()
    tr = (t[:, 0] + t[:, 1] + t[:, 2]) / 3.0
    for i in range(3):
        d[:, i] = t[:, i] - tr
    return d


def apriori(mlp, feats, targs, norm, delta):
    """Correlation coefficient and normalised MSE per deviatoric component,
    network vs Deardorff's eddy viscosity, on (S, Nc, ...) held-out data."""
    import torch
    x, _ = to_training(feats, targs, norm)
    yhat = mlp.forward(x)[:, :6].double()
    n = torch.from_numpy(norm.astype(np.float64)).to(yhat.device)
    tau_net = yhat * n[22:28] + n[28:34]
    tau = targs.reshape(-1, 6)
    f = feats.reshape(-1, 16).double()
    g = f[:, :9] / delta  # (ux, vx, wx, uy, vy, wy, uz, vz, wz)
    S = torch.stack([g[:, 0], g[:, 4], g[:, 8], 0.5 * (g[:, 3] + g[:, 1]), 0.5 * (g[:, 6] + g[:, 2]),
                     0.5 * (g[:, 7] + g[:, 5])], dim=1)
    e = torch.clamp(0.5 * (tau[:, 0] + tau[:, 1] + tau[:, 2]), min=0.0)
    nut = 0.1 * delta * torch.sqrt(e)
    tau_dd = -2.0 * nut[:, None] * S
    td, nd, dd = deviatoric(tau), deviatoric(tau_net), deviatoric(tau_dd)
    names = ["tau11", "tau22", "tau33", "tau12", "tau13", "tau23"]
    rep = {}
    for i, nm in enumerate(names):
        a = td[:, i]
        var = float(((a - a.mean()) ** 2).mean())
        r = {}
        for lab, p in (("network", nd[:, i]), ("deardorff", dd[:, i])):
            rho = float(torch.corrcoef(torch.stack([a, p]))[0, 1])
            mse = float(((p - a) ** 2).mean()) / max(var, 1e-300)
            r[lab] = dict(rho=rho, nmse=mse)
        rep[nm] = r
    w = torch.tensor([1.0, 1.0, 1.0, 2.0, 2.0, 2.0], dtype=torch.float64, device=S.device)
    rep["dissipation"] = dict(network=float((-(tau_net * S * w).sum(1)).mean()),
                              filtered=float((-(tau * S * w).sum(1)).mean()))
    return rep


def aposteriori(first, info, params, norm, nsteps, log=print, guard=0.0):
    """Coarse runs from the first filtered snapshot with the Deardorff
    closure and with the trained network; time-averaged mean U(z) over the
    second half against the filtered fine run's mean profile.  guard: the
    factor of the fallback test against the Deardorff dissipation for the
    learned run (0: the sign test only, so the network itself is judged)."""
    P = _host()
    nxc, nyc, nzc = info["coarse"]
    re_tau = info["re_tau"]
    ref = np.array(info["filtered_mean_u"])
    ub = float(ref.mean())
    out = {}
    for name, imodel in (("deardorff", 3), ("learned", 5)):
        cfg = P.channel_config(nxc, nyc, nzc, dt=1e-3, re_tau=re_tau, imodel=imodel, precision=8)
        cfg.z0 = info["z0"]
        g = P.LesGpu(cfg)
        g.upload(first[0], first[1], first[2], np.full_like(first[0], 1e-4), None)
        m = None
        if imodel == 5:
            m = P.Mlp(params, norm)
            g.set_mlp(m, re_tau)
            g.set_learned_guard(guard)
        dt = g.cfl_dt(0.5)
        prof, used, nstat = [], 0, 0
        t0 = time.time()
        for it in range(nsteps):
            g.step(it=it, mnout=False, dt=dt)
            if it >= nsteps // 2 and it % 10 == 0:
                mb, _ = g.stats()
                prof.append(mb[3].copy())
                if m is not None:
                    used += g.learned_status()[0]
                nstat += 1
        g.sync()
        U = np.mean(prof, axis=0)
        err = np.abs(U - ref).max() / ub
        out[name] = dict(mean_u=U.tolist(), max_err_vs_filtered_over_ub=float(err),
                         used_fraction=(used / nstat if m is not None else None), seconds=time.time() - t0,
                         steps=nsteps, dt=dt)
        log("a posteriori %s: max |U - U_filtered| / U_b = %.4f" % (name, err))
        g.close()
        if m is not None:
            m.close()
    out["filtered_mean_u"] = ref.tolist()
    return out


def run(args, log=print):
    import torch
    P = _host()
    t_all = time.time()
    feats, targs, info, first = collect(tuple(args.fine), tuple(args.factor), args.re_tau, args.snapshots,
                                        args.spinup, args.every, args.amp, args.large, args.seed,
                                        spinup_precision=args.spinup_precision,
                                        with_model=not getattr(args, "resolved_only", False), log=log)
    S = feats.shape[0]
    nho = max(1, int(round(S * args.holdout)))
    ftr, ttr = feats[:S - nho], targs[:S - nho]
    fho, tho = feats[S - nho:], targs[S - nho:]
    norm = normalisation(ftr, ttr)
    x, y = to_training(ftr, ttr, norm)
    log("training samples %d, held-out snapshots %d" % (x.shape[0], nho))
    mlp = P.Mlp(init_params(args.seed), norm)
    hist, steps, secs = train(mlp, x, y, args.epochs, args.batch, args.lr, seed=args.seed, log=log)
    del x, y
    torch.cuda.empty_cache()
    nxc, nyc, nzc = info["coarse"]
    xl, yl, zl = 2 * np.pi, np.pi, 2.0
    delta = (xl / nxc * yl / nyc * zl / nzc) ** (1.0 / 3.0)
    rep_ho = apriori(mlp, fho, tho, norm, delta)
    params, _ = mlp.get_params()
    mlp.close()
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    # what the a-posteriori runs need, for evaluating later closures without a new fine run
    ev = dict(coarse=info["coarse"], re_tau=info["re_tau"], z0=info["z0"], filtered_mean_u=info["filtered_mean_u"])
    np.savez(args.out + "_eval.npz", first=first, meta=json.dumps(ev))
    apost = None
    if args.aposteriori:
        apost = aposteriori(first, info, params, norm, args.aposteriori, log, getattr(args, "guard", 0.0))
    np.savez(args.out + ".npz", params=params, norm=norm, re_tau=np.float64(args.re_tau),
             coarse=np.array(info["coarse"]), fine=np.array(info["fine"]), factor=np.array(info["factor"]))
    report = dict(data=info, training=dict(steps=steps, seconds=secs, batch=args.batch, lr=args.lr,
                                           epochs=args.epochs, samples=int(ftr.shape[0] * ftr.shape[1]),
                                           samples_per_s=steps * args.batch / max(secs, 1e-9),
                                           loss=hist[::max(1, len(hist) // 50)] + hist[-1:]),
                  apriori_heldout=rep_ho, aposteriori=apost, total_seconds=time.time() - t_all)
    with open(args.out + ".json", "w") as fh:
        json.dump(report, fh, indent=1)
    log(json.dumps(rep_ho, indent=1))
    return report


def evaluate(args, log=print):
    """A-posteriori runs only, from <out>.npz (network) and <out>_eval.npz
    (first filtered snapshot and the filtered fine run's mean profile);
    updates the 'aposteriori' entry of <out>.json."""
    z = np.load(args.out + ".npz")
    ev = np.load(args.out + "_eval.npz")
    info = json.loads(str(ev["meta"]))
    apost = aposteriori(ev["first"], info, z["params"], z["norm"], args.aposteriori or 4000, log,
                        getattr(args, "guard", 0.0))
    rp = args.out + ".json"
    rep_ = json.load(open(rp)) if os.path.exists(rp) else {}
    rep_["aposteriori"] = apost
    with open(rp, "w") as fh:
        json.dump(rep_, fh, indent=1)
    return apost


def main(argv=None):
    ap = argparse.ArgumentParser(description="Train the learned SGS closure on one GPU.")
    ap.add_argument("--fine", type=int, nargs=3, default=[384, 384, 192])
    ap.add_argument("--factor", type=int, nargs=2, default=[4, 2])
    ap.add_argument("--re-tau", type=float, default=395.0)
    ap.add_argument("--snapshots", type=int, default=200)
    ap.add_argument("--spinup", type=int, default=14000)
    ap.add_argument("--spinup-precision", type=int, choices=[4, 8], default=4)
    ap.add_argument("--every", type=int, default=40)
    ap.add_argument("--amp", type=float, default=1.0)
    ap.add_argument("--large", type=float, default=0.3)
    ap.add_argument("--seed", type=int, default=12345)
    ap.add_argument("--holdout", type=float, default=0.1)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--aposteriori", type=int, default=0, help="coarse steps of the a-posteriori runs (0 = skip)")
    ap.add_argument("--guard", type=float, default=0.0,
                    help="fallback factor against the Deardorff dissipation in the a-posteriori learned run "
                         "(0 = sign test only: the network itself is judged)")
    ap.add_argument("--resolved-only", action="store_true",
                    help="targets without the fine run's own model stress")
    ap.add_argument("--out", default=os.path.join(HERE, "weights", "sgs_c4"))
    ap.add_argument("--evaluate", action="store_true",
                    help="only the a-posteriori runs, from <out>.npz and <out>_eval.npz")
    args = ap.parse_args(argv)
    if args.evaluate:
        evaluate(args)
    else:
        run(args)


if __name__ == "__main__":
    main()
