"""Training of the learned sub-grid closure on one GPU.

    python paes-channelflow_b200/train_closure.py [--fine 384 384 192] [--factors 2 4]
        [--re-tau 395] [--snapshots 100] [--spinup 14000] [--every 60] [--epochs 12]
        [--out paes-channelflow_b200/weights/sgs_c4]

The closure is dimensionless (les_mlp.h): inputs g/|G| (the nine resolved
velocity gradients over their Frobenius norm), min(z_w/Delta, 16) and z_w/h,
outputs c with tau_ij = (Delta |G|)^2 c_ij.  Trained on several filter
widths Delta of the same fine run, it learns the stress per (Delta |G|)^2 as
a function of the local flow geometry and the wall distance in filter
widths, which is what carries it from the training grids to others.

1. A fine run of this solver (Deardorff closure) from the log-law mean
   profile of the wall model plus random perturbations (small-scale noise
   and large structures, which make the flow transition within a few eddy
   turnovers); the spin-up runs in the mixed form, then the state moves to
   an FP64 handle for the data.
2. After the spin-up, every `every` steps and for every filter factor f:
   les_gpu_learn_filter onto the grid (nx/f, ny/f, nz/f) (box filter of f
   fine cells in x, y and z, so the coarse cells keep the fine cells' aspect
   ratio) gives the filtered u, v, w and tau_ij = filt(u_i u_j) -
   filt(u_i) filt(u_j) plus (by default) the filtered Deardorff stress of
   the fine run itself, i.e. the total sub-filter stress the coarse grid
   misses; the filtered fields are loaded into a coarse handle whose
   les_gpu_learned_features computes the network inputs (and Delta |G|)
   with the same kernels the learned stage uses.
3. Targets: the deviatoric stress over (Delta |G|)^2, clipped to the
   training set's 99.9th percentile of |c| per component (points where |G|
   is tiny carry stresses the local gradients cannot explain); normalisation
   (mean / standard deviation per input and output) from the training
   snapshots; the last `holdout` fraction of snapshots is held out.
4. Adam (lr 1e-3, batch 65536, f32 master weights) on the tensor-core
   kernels (les_mlp_adam_step), shuffled batches over all filter widths.
5. A-priori evaluation per filter width on the held-out snapshots: per
   component correlation and normalised MSE of the deviatoric stresses for
   the network, for the Deardorff eddy viscosity -2 (0.1 Delta sqrt(e)) S
   with the filtered e = tau_kk / 2, and for Smagorinsky -2 (0.1 Delta)^2
   |S| S; the network as the solver applies it (local backscatter removed
   along S) and raw; mean dissipations of the network, the filtered truth
   and the Smagorinsky estimate (Lilly's C_s = 0.17) the runtime fallback
   test compares with.
6. Writes <out>.npz (params, norm, grids) and <out>.json (report).
"""
import argparse
import importlib.util
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
COMPONENTS = ("tau11", "tau22", "tau33", "tau12", "tau13", "tau23")


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


def delta_of(grid, xl=2 * np.pi, yl=np.pi, zl=2.0):
    nx, ny, nz = grid
    return (xl / nx * yl / ny * zl / nz) ** (1.0 / 3.0)


def collect(fine=(384, 384, 192), factors=(2, 4), re_tau=395.0, snapshots=100, spinup=14000, every=60, amp=1.0,
            large=0.3, seed=12345, cfl=0.5, spinup_precision=4, with_model=True, log=print):
    """Run the fine case; returns ({factor: (features f32 (S, Nc, 16), stresses
    f32 (S, Nc, 6))} as CUDA tensors, info)."""
    import torch
    P = _host()
    nx, ny, nz = fine
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
    coarse, data = {}, {}
    for fac in factors:
        ccfg = P.channel_config(nx // fac, ny // fac, nz // fac, dt=dt, re_tau=re_tau, precision=8)
        ccfg.z0 = cfg.z0
        nc = (nx // fac) * (ny // fac) * (nz // fac)
        coarse[fac] = P.LesGpu(ccfg)
        data[fac] = (torch.empty((snapshots, nc, 16), dtype=torch.float32, device="cuda"),
                     torch.empty((snapshots, nc, 6), dtype=torch.float32, device="cuda"))
    for s in range(snapshots):
        if s > 0:
            for _ in range(every):
                g.step(it=state["it"], mnout=False, dt=dt)
                state["it"] += 1
        for fac in factors:
            out = g.learn_filter(fac, fac, with_model=with_model)
            uvw = out[:3].cpu().numpy()
            c = coarse[fac]
            c.upload(uvw[0], uvw[1], uvw[2], np.full_like(uvw[0], 1e-4), None)
            data[fac][0][s] = c.learned_features()
            data[fac][1][s] = out[3:].reshape(6, -1).t().float()
        if s == 0 or (s + 1) % max(1, snapshots // 10) == 0:
            monitor(g, "snapshot %d/%d" % (s + 1, snapshots))
    g.sync()
    info = dict(fine=list(fine), factors=list(factors), re_tau=re_tau, snapshots=snapshots, spinup=spinup,
                spinup_precision=spinup_precision, every=every, amp=amp, large=large, seed=seed, dt=dt,
                targets="filtered total sub-filter stress" if with_model else "filtered minus resolved products",
                steps=state["it"], coarse={str(f): [nx // f, ny // f, nz // f] for f in factors}, history=hist,
                collect_seconds=time.time() - t0, z0=cfg.z0)
    g.close()
    for c in coarse.values():
        c.close()
    return data, info


def deviatoric(t):
    """(N, 6) stresses -> deviatoric (trace removed from the diagonal)."""
    d = t.clone()
    tr = (t[:, 0] + t[:, 1] + t[:, 2]) / 3.0
    for i in range(3):
        d[:, i] = t[:, i] - tr
    return d


def targets(feats, tau, clip=None):
    """c = tau_dev / (Delta |G|)^2 of (N, 16) raw features and (N, 6)
    stresses (float64); clip: per-component bound on |c| (None: none)."""
    import torch
    s2 = feats[:, 11].double() ** 2
    c = deviatoric(tau.double()) / torch.where(s2 > 0, s2, torch.ones_like(s2))[:, None]
    c[s2 <= 0] = 0.0
    if clip is not None:
        c = torch.maximum(torch.minimum(c, clip[None, :]), -clip[None, :])
    return c


def clip_bounds(data, train_snaps, q=0.999, sample=4_000_000):
    """99.9th percentile of |c| per component over a sample of the training
    points of every filter width."""
    import torch
    gen = torch.Generator(device="cuda")
    gen.manual_seed(0)
    cs = []
    for fac, (f, t) in data.items():
        ff = f[:train_snaps].reshape(-1, 16)
        tt = t[:train_snaps].reshape(-1, 6)
        idx = torch.randint(0, ff.shape[0], (min(sample, ff.shape[0]),), device="cuda", generator=gen)
        cs.append(targets(ff[idx], tt[idx]).abs())
    return torch.quantile(torch.cat(cs), q, dim=0)


def normalisation(data, train_snaps, clip):
    """in_shift, in_scale per input, out_scale, out_shift per output (34
    floats) from the training snapshots of every filter width."""
    import torch
    n = 0
    s1 = torch.zeros(11, dtype=torch.float64, device="cuda")
    s2 = torch.zeros(11, dtype=torch.float64, device="cuda")
    t1 = torch.zeros(6, dtype=torch.float64, device="cuda")
    t2 = torch.zeros(6, dtype=torch.float64, device="cuda")
    for fac, (f, t) in data.items():
        for s in range(train_snaps):
            x = f[s][:, :11].double()
            c = targets(f[s], t[s], clip)
            s1 += x.sum(0); s2 += (x * x).sum(0)
            t1 += c.sum(0); t2 += (c * c).sum(0)
            n += x.shape[0]
    fm, tm = s1 / n, t1 / n
    fs = torch.sqrt(torch.clamp(s2 / n - fm * fm, min=0.0))
    ts = torch.sqrt(torch.clamp(t2 / n - tm * tm, min=1e-30))
    in_scale = torch.where(fs > 1e-6 * (fm.abs() + 1e-30), 1.0 / fs, torch.zeros_like(fs))
    norm = torch.cat([fm, in_scale, ts, tm]).cpu().numpy()
    return norm.astype(np.float32)


def to_training(feats, tau, norm, clip):
    """bf16 normalised features (N, 16) and f32 normalised targets (N, 8)
    of (N, 16) raw features and (N, 6) stresses."""
    import torch
    n = torch.from_numpy(norm.astype(np.float64)).to(feats.device)
    x = torch.zeros((feats.shape[0], 16), dtype=torch.float64, device=feats.device)
    x[:, :11] = (feats[:, :11].double() - n[:11]) * n[11:22]
    c = targets(feats, tau, clip)
    y = torch.zeros((feats.shape[0], 8), dtype=torch.float32, device=feats.device)
    y[:, :6] = ((c - n[28:34]) / n[22:28]).float()
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


def train(mlp, x, y, epochs=12, batch=65536, lr=1e-3, seed=0, log=print):
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


def apriori(mlp, feats, tau, norm, clip, delta):
    """Per deviatoric component: correlation and normalised MSE of the
    network's stresses, of Deardorff's eddy viscosity (filtered e) and of
    Smagorinsky's, against the filtered truth; mean dissipations.  feats
    (N, 16) raw features, tau (N, 6) stresses of held-out snapshots."""
    import torch
    x, _ = to_training(feats, tau, norm, clip)
    y = mlp.forward(x)[:, :6].double()
    n = torch.from_numpy(norm.astype(np.float64)).to(y.device)
    s = feats[:, 11].double()
    tau_raw = (y * n[22:28] + n[28:34]) * (s * s)[:, None]
    t = tau.double()
    g = feats[:, :9].double() * (s / delta)[:, None]  # (ux, vx, wx, uy, vy, wy, uz, vz, wz)
    S = torch.stack([g[:, 0], g[:, 4], g[:, 8], 0.5 * (g[:, 3] + g[:, 1]), 0.5 * (g[:, 6] + g[:, 2]),
                     0.5 * (g[:, 7] + g[:, 5])], dim=1)
    w = torch.tensor([1.0, 1.0, 1.0, 2.0, 2.0, 2.0], dtype=torch.float64, device=S.device)
    # the stress the solver applies: local backscatter (tau:S > 0) removed along S
    ts, ss = (tau_raw * S * w).sum(1), (S * S * w).sum(1)
    a = torch.where((ts > 0) & (ss > 0), -ts / torch.where(ss > 0, ss, torch.ones_like(ss)), torch.zeros_like(ts))
    tau_net = tau_raw + a[:, None] * S
    smag = torch.sqrt(2.0 * (S * S * w).sum(1))
    e = torch.clamp(0.5 * (t[:, 0] + t[:, 1] + t[:, 2]), min=0.0)
    tau_dd = -2.0 * (0.1 * delta * torch.sqrt(e))[:, None] * S
    tau_sm = -2.0 * ((0.1 * delta) ** 2 * smag)[:, None] * S
    td = deviatoric(t)
    rep = {}
    for i, nm in enumerate(COMPONENTS):
        a = td[:, i]
        var = float(((a - a.mean()) ** 2).mean())
        r = {}
        for lab, p in (("network", deviatoric(tau_net)[:, i]), ("network_raw", deviatoric(tau_raw)[:, i]),
                       ("deardorff", deviatoric(tau_dd)[:, i]), ("smagorinsky", deviatoric(tau_sm)[:, i])):
            rho = float(torch.corrcoef(torch.stack([a, p]))[0, 1])
            mse = float(((p - a) ** 2).mean()) / max(var, 1e-300)
            r[lab] = dict(rho=rho, nmse=mse)
        rep[nm] = r
    dis = lambda tt: float((-(tt * S * w).sum(1)).mean())
    rep["dissipation"] = dict(network=dis(tau_net), network_raw=dis(tau_raw), filtered=dis(t), deardorff=dis(tau_dd),
                              smagorinsky_reference=float((0.17 ** 2 * delta ** 2 * smag ** 3).mean()))
    rep["dissipation"]["network_over_reference"] = rep["dissipation"]["network"] / rep["dissipation"][
        "smagorinsky_reference"]
    return rep


def run(args, log=print):
    import torch
    P = _host()
    t_all = time.time()
    data, info = collect(tuple(args.fine), tuple(args.factors), args.re_tau, args.snapshots, args.spinup,
                         args.every, args.amp, args.large, args.seed, spinup_precision=args.spinup_precision,
                         with_model=not getattr(args, "resolved_only", False), log=log)
    S = args.snapshots
    nho = max(1, int(round(S * args.holdout)))
    ntr = S - nho
    clip = clip_bounds(data, ntr)
    norm = normalisation(data, ntr, clip)
    xs, ys = [], []
    for fac, (f, t) in data.items():
        x, y = to_training(f[:ntr].reshape(-1, 16), t[:ntr].reshape(-1, 6), norm, clip)
        xs.append(x)
        ys.append(y)
    x, y = torch.cat(xs), torch.cat(ys)
    del xs, ys
    log("training samples %d, held-out snapshots %d per filter width" % (x.shape[0], nho))
    mlp = P.Mlp(init_params(args.seed), norm)
    hist, steps, secs = train(mlp, x, y, args.epochs, args.batch, args.lr, seed=args.seed, log=log)
    nsamples = int(x.shape[0])
    del x, y
    torch.cuda.empty_cache()
    rep_ho = {}
    for fac, (f, t) in data.items():
        grid = info["coarse"][str(fac)]
        rep_ho[str(fac)] = apriori(mlp, f[ntr:].reshape(-1, 16), t[ntr:].reshape(-1, 6), norm, clip,
                                   delta_of(grid))
        rep_ho[str(fac)]["grid"] = grid
        rep_ho[str(fac)]["delta"] = delta_of(grid)
    params, _ = mlp.get_params()
    mlp.close()
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    np.savez(args.out + ".npz", params=params, norm=norm, re_tau=np.float64(args.re_tau),
             factors=np.array(args.factors), fine=np.array(info["fine"]), clip=clip.cpu().numpy())
    report = dict(closure="dimensionless: x = (g/|G|, min(z_w/Delta, 16), z_w/h), tau = (Delta |G|)^2 c",
                  data=info, clip=clip.cpu().numpy().tolist(),
                  training=dict(steps=steps, seconds=secs, batch=args.batch, lr=args.lr, epochs=args.epochs,
                                samples=nsamples, samples_per_s=steps * args.batch / max(secs, 1e-9),
                                loss=hist[::max(1, len(hist) // 50)] + hist[-1:]),
                  apriori_heldout=rep_ho, total_seconds=time.time() - t_all)
    with open(args.out + ".json", "w") as fh:
        json.dump(report, fh, indent=1)
    log(json.dumps(rep_ho, indent=1))
    return report


def main(argv=None):
    ap = argparse.ArgumentParser(description="Train the learned SGS closure on one GPU.")
    ap.add_argument("--fine", type=int, nargs=3, default=[384, 384, 192])
    ap.add_argument("--factors", type=int, nargs="+", default=[2, 4],
                    help="filter factors f: coarse grids (nx/f, ny/f, nz/f); f = 1 or even")
    ap.add_argument("--re-tau", type=float, default=395.0)
    ap.add_argument("--snapshots", type=int, default=100)
    ap.add_argument("--spinup", type=int, default=14000)
    ap.add_argument("--spinup-precision", type=int, choices=[4, 8], default=4)
    ap.add_argument("--every", type=int, default=60)
    ap.add_argument("--amp", type=float, default=1.0)
    ap.add_argument("--large", type=float, default=0.3)
    ap.add_argument("--seed", type=int, default=12345)
    ap.add_argument("--holdout", type=float, default=0.1)
    ap.add_argument("--epochs", type=int, default=12)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--resolved-only", action="store_true",
                    help="targets without the fine run's own model stress")
    ap.add_argument("--out", default=os.path.join(HERE, "weights", "sgs_c4"))
    run(ap.parse_args(argv))


if __name__ == "__main__":
    main()
