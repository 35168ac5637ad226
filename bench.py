"""Benchmark of the LES RK3 hot path (one JSON line on rank 0).

Workload: the production channel grid nx=ny=512, nz=256 (67.1 M points,
3/2-padded planes of 768x768), Re_tau=590, wall model isurface=6, seeded
synthetic initial field (parabolic mean + uniform perturbations, projected
divergence-free) built on the device, fixed dt at CFL 0.5.  A step is one
full RK3 step (three stages of comp1 + comprhs + press + comp2) of the
whole domain; metric = nx*ny*nz*steps / seconds.

Three forms run the same steps from the same initial field:
  fp64          plain FP64 drop-in, Deardorff TKE closure;
  mixed         FP32 transforms/advection/SGS, FP64 pressure, mean modes and
                reductions, Deardorff closure;
  learned_mixed the mixed form with the learned closure (bf16 network on
                the tensor cores, weights from paes-channelflow_b200/weights,
                Deardorff fallback when its mean dissipation is negative).
`value` is learned_mixed with the library's default fallback test (the
metric compares it with fp64: `forms`, which also reports the fraction of
timed stages that used the network and, as a separate key, the rate with
the sign test only), with the state resident in HBM; `errors` states its
mean-profile, Reynolds-stress, rms and divergence differences from the fp64
run after the timed steps.  `e2e` is the learned_mixed metric through the C
ABI a host program uses, as a device-resident drop-in runs: the state is
uploaded once from pinned host memory inside the timed region, then every
step ends with les_gpu_stats (statistics read back to the host).

--impl reference times the CPU restatement of the reference (oracle/, FP64,
OpenMP on all host cores) on a 512x512x4 slab of the same grid (the cost
per point depends on nx, ny, not nz), one RK3 step per timed step.

Multi-GPU (torchrun): the domain is not decomposed (single-GPU tier, no MPI
decomposition): each rank runs an independent replica; value = points*steps
of all ranks / max-over-ranks time ("weak" scaling, replicas only).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NX = NY = 512
NZ = 256
RE_TAU = 590.0
SLAB_NZ = 4
# The learned form is timed with the library's default fallback test (the
# network's mean dissipation must be >= 0 and within a factor 4 of the
# Smagorinsky estimate); the line reports the fraction of timed stages that
# used the network.
LEARNED_FALLBACK = "library default: sign test and factor 4 of the Smagorinsky dissipation"
# levels (1-based) of the stated x-spectrum errors: nearest z+ = 15 and z+ = 100
SPEC_LEVELS = tuple(int(round(zp / (2.0 / NZ * RE_TAU) + 0.5)) for zp in (15.0, 100.0))
METRIC = "RK3 Mpoint-steps/s"


def load_product():
    import importlib.util
    name = "les_gpu_host"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(ROOT, "paes-channelflow_b200", "les_gpu.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def bf16_peak_tflops():
    """Sustained bf16 GEMM rate (the network kernel runs inside a long step)."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops_sustained"]), "measured sustained"
    except Exception:
        return 1400.0, "fallback sustained"


def algorithmic_bytes(kernel, nx, ny, nz, tb, learned=False):
    """Compulsory HBM bytes of one launch (one stage over all levels) of the
    stage kernels: every array the kernel must read once and write once.
    With the learned closure the fused row kernel leaves the UY and WY
    inputs unread (only ux and vy of the gradients are transformed)."""
    mx, my, kx = 3 * nx // 2, 3 * ny // 2, nx // 2
    pad = mx * my * tb            # padded physical plane
    mix = my * kx * 2 * tb        # x-spectral, y-physical plane on the padded y grid
    spec = ny * kx * 2 * tb       # small spectrum plane
    small = nx * ny * tb
    L, Lw = nz, nz - 1            # levels of u, v | w, e
    nm = ny * kx
    table = {
        "k_y_inverse": (2 * L + 2 * Lw) * spec + (4 * L + 4 * Lw) * mix,
        "k_x_inverse": (4 * L + 4 * Lw) * mix + (6 * L + 6 * Lw) * pad,
        "k_flux": (6 * L + 6 * Lw) * pad + (5 * L + 6 * Lw) * pad,
        "k_x_forward": (5 * L + 6 * Lw) * pad + (4 * L + 4 * Lw) * mix,
        "k_y_forward": (4 * L + 4 * Lw) * mix + (2 * L + Lw) * spec + Lw * spec,
        "k_clip_y": Lw * pad * 2,
        "k_clip_x": Lw * pad * 4,
        "k_e_prep": Lw * (3 * small + spec),
        "k_e_update": Lw * (spec + 3 * small),
        "k_press": nz * (9 * spec + 2 * 24 * nm + 16 * nm),
        "k_update": nz * (15 * spec + 16 * nm),
        # fused row kernel: reads the 8 mixed inputs, writes the 8 mixed outputs
        "k_row_fused": ((3 * L + 3 * Lw) if learned else (4 * L + 4 * Lw)) * mix + (4 * L + 4 * Lw) * mix,
    }
    return table.get(kernel)


WEIGHTS = os.path.join(ROOT, "paes-channelflow_b200", "weights", "sgs_c4.npz")


def load_network(P, dev):
    """The trained closure (weights file), else a seeded untrained network."""
    if os.path.exists(WEIGHTS):
        z = np.load(WEIGHTS)
        return P.Mlp(z["params"], z["norm"], device=dev), "trained (%s)" % os.path.relpath(WEIGHTS, ROOT)
    rng = np.random.default_rng(0)
    shapes = [(64, 11), (64,), (64, 64), (64,), (64, 64), (64,), (6, 64), (6,)]
    p = np.concatenate([rng.standard_normal(sh).ravel() / np.sqrt(sh[-1]) if len(sh) == 2 else np.zeros(sh)
                        for sh in shapes]).astype(np.float32)
    norm = np.concatenate([np.zeros(11), np.full(9, 30.0), [1.0 / RE_TAU, 0.0], np.full(6, 1e-3), np.zeros(6)])
    return P.Mlp(p, norm, device=dev), "untrained (seeded)"


def run_form(P, precision, steps, warmup, dev, want_profile, imodel=3, mlp=None, guard=None):
    import torch
    cfg = P.channel_config(NX, NY, NZ, dt=1e-3, re_tau=RE_TAU, precision=precision, device=dev, imodel=imodel)
    g = P.LesGpu(cfg)
    if mlp is not None:
        g.set_mlp(mlp, RE_TAU)
        if guard is not None:
            g.set_learned_guard(guard)
    g.make_ic(seed=12345, amp=0.1, re_tau=RE_TAU)
    dt = g.cfl_dt(0.5)
    g.cfg.dt = dt
    for i in range(warmup):
        g.step(it=i + 1, mnout=False, dt=dt)
    g.sync()
    stream = torch.cuda.ExternalStream(g.stream_handle(), device=torch.device("cuda", dev))
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n0 = g.kernel_launches()
    c0 = g.learned_counts() if mlp is not None else (0, 0)
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev) as clk:
        ev0.record(stream)
        for i in range(steps):
            g.step(it=warmup + i + 1, mnout=False, dt=dt)
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = ev0.elapsed_time(ev1)
    launches = g.kernel_launches() - n0
    g.sync()
    out = {"ms": ms, "launches": launches, "clocks": clk.summary(), "dt": dt}
    if mlp is not None:
        c1 = g.learned_counts()
        out["stages_timed"], out["stages_used"] = c1[0] - c0[0], c1[1] - c0[1]
    if want_profile:
        # per-kernel CUDA-event times of one eager stage, the minimum over
        # three repeats (kernel by kernel, in launch order)
        runs = [g.profile_stage(2, dt) for _ in range(3)]
        out["profile"] = [(runs[0][i][0], min(r[i][1] for r in runs)) for i in range(len(runs[0]))]
    mb, sc = g.stats()
    out["utau"] = float(sc[0])
    out["divz_max"] = float(np.max(mb[2]))
    out["meanbuf"] = mb
    # 1D x-spectra of u and w at the levels nearest z+ = 15 and 100
    out["spectra"] = {(f, iz): g.spectra(f, iz)[0] for f in (0, 2) for iz in SPEC_LEVELS}
    if mlp is not None:
        out["learned_status"] = g.learned_status()
        out["learned_reference"] = g.learned_reference()
    out["handle"] = g
    return out


def run_e2e(P, steps, dev, precision, imodel=3, mlp=None):
    """Through the C ABI with host buffers: upload the state from pinned host
    memory, then steps x (les_gpu_step + les_gpu_stats read-back).  The host
    arrays hold the form's own reals: 8 bytes for the FP64 form, 4 for the
    mixed forms (the reference as shipped keeps u, v, w, e, p in 4-byte
    reals; FP64 is its -fdefault-real-8 build)."""
    import torch
    cfg = P.channel_config(NX, NY, NZ, dt=1e-3, re_tau=RE_TAU, precision=precision, device=dev, imodel=imodel)
    g = P.LesGpu(cfg)
    if mlp is not None:
        g.set_mlp(mlp, RE_TAU)
    g.make_ic(seed=12345, amp=0.1, re_tau=RE_TAU)
    dt = g.cfl_dt(0.5)
    shape = (NZ, NY, NX)
    hdt = torch.float64 if precision == 8 else torch.float32
    host = {k: torch.empty(shape, dtype=hdt, pin_memory=True) for k in "uvwep"}
    g.download_into(*[host[k] for k in "uvwep"])
    g.step(it=1, mnout=False, dt=dt)  # build the step graph outside the timed region
    g.stats()
    g.sync()
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    g.upload(*[host[k] for k in "uvwep"])
    for i in range(steps):
        g.step(it=i + 2, mnout=False, dt=dt)
        g.stats()
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    barrier()
    h2d = sum(t.numel() * t.element_size() for t in host.values())
    d2h = (19 * NZ + 5) * 8
    g.close()
    return el, h2d / steps, d2h


_pg = None


def barrier():
    if _pg is not None:
        import torch.distributed as dist
        dist.barrier()


def init_dist(backend, timeout_s=120):
    """One process group over all ranks (env:// rendezvous: MASTER_ADDR,
    MASTER_PORT, RANK, WORLD_SIZE); a short timeout so that ranks waiting for
    a rank that died end with an error."""
    global _pg
    import datetime
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    _pg = dist.group.WORLD


def max_over_ranks(x):
    if _pg is None:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(points_per_rank, steps, ms_local):
    """Whole-job rate of independent replicas (one per rank): the points of
    all ranks times steps over the max-over-ranks time, in Mpoint-steps/s;
    returns (rate, max ms)."""
    world = 1
    if _pg is not None:
        import torch.distributed as dist
        world = dist.get_world_size()
    ms = max_over_ranks(ms_local)
    return world * points_per_rank * steps / (ms / 1e3) / 1e6, ms


def cpu_baseline(steps=1, warmup=1, nz=SLAB_NZ):
    """The oracle (CPU restatement of the reference, FP64, OpenMP on all host
    cores) on a 512x512xnz slab of the grid: `warmup` untimed RK3 steps, then
    `steps` timed ones.  Returns (Mpoint-steps/s, threads, seconds)."""
    from oracle import oracle as O
    lib = O.lib()
    cfg = O.make_config(NX, NY, nz, dt=1e-3, re_tau=RE_TAU)
    o = O.Oracle(cfg)
    o.make_ic(seed=12345, amp=0.1, re_tau=RE_TAU)
    o.set_dt(o.cfl_dt(0.5))
    if warmup > 0:
        o.step(0, warmup, 0)
    t0 = time.perf_counter()
    o.step(warmup, steps, 0)
    el = time.perf_counter() - t0
    pts = NX * NY * nz * steps
    return pts / el / 1e6, lib.orc_threads(), el


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-full-step", action="store_true",
                    help="time one oracle RK3 step on the full 512x512x256 grid beside the slab (CPU only)")
    args = ap.parse_args()
    rank, local_rank, world = dist_env()

    if args.cpu_full_step:
        # one RK3 step of the oracle on the whole 512x512x256 grid beside the
        # slab's rate: the check that the slab's cost per point stands for the
        # full grid's (a few minutes of CPU; not part of the default run)
        vf, cores, elf = cpu_baseline(1, warmup=0, nz=NZ)
        vs, _, els = cpu_baseline(args.steps, warmup=args.warmup)
        print(json.dumps({"cpu_full_grid_step": {"value": vf, "seconds": elf, "cores": cores},
                          "cpu_slab": {"value": vs, "seconds": els, "steps": args.steps, "warmup": args.warmup},
                          "unit": "Mpoint-steps/s", "full_over_slab": vf / vs}))
        return

    if args.impl == "reference":
        if rank != 0:
            return
        val, cores, el = cpu_baseline(args.steps, warmup=args.warmup)
        line = {"metric": METRIC, "value": val, "unit": "Mpoint-steps/s", "impl": "reference", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": "channel 512x512x256 Re_tau=590 Deardorff isurface=6, sampled as a 512x512x4 slab",
                           "global_batch": NX * NY * SLAB_NZ, "parallelism": "cpu-openmp"},
                "cpu_baseline": {"value": val, "unit": "Mpoint-steps/s", "cores": cores, "kind": "port",
                                 "sample": "512x512x4 slab of the 512x512x256 grid, %d warm-up + %d timed RK3 steps, "
                                           "FP64 oracle" % (args.warmup, args.steps)},
                "e2e": {"value": val, "unit": "Mpoint-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    if world > 1:
        torch.cuda.set_device(local_rank)
        init_dist("nccl")
    dev = local_rank if world > 1 else 0
    torch.cuda.set_device(dev)
    P = load_product()

    r64 = run_form(P, P.PREC_FP64, args.steps, args.warmup, dev, want_profile=True)
    prof64 = r64.pop("profile")
    r64.pop("handle").close()
    r32 = run_form(P, P.PREC_MIXED, args.steps, args.warmup, dev, want_profile=True)
    prof32 = r32.pop("profile")
    r32.pop("handle").close()
    torch.cuda.empty_cache()
    mlp, weights = load_network(P, dev)
    rl = run_form(P, P.PREC_MIXED, args.steps, args.warmup, dev, want_profile=True, imodel=P.SGS_LEARNED, mlp=mlp)
    prof = rl.pop("profile")
    rl.pop("handle").close()
    torch.cuda.empty_cache()
    # the same form with the sign test only: every stage runs the network's
    # whole path (a separate key; the headline uses the default test)
    rs = run_form(P, P.PREC_MIXED, args.steps, args.warmup, dev, want_profile=False, imodel=P.SGS_LEARNED, mlp=mlp,
                  guard=0.0)
    rs.pop("handle").close()
    torch.cuda.empty_cache()
    e2e_s, h2d, d2h = run_e2e(P, args.steps, dev, P.PREC_MIXED, imodel=P.SGS_LEARNED, mlp=mlp)
    mlp.close()

    pts = NX * NY * NZ
    fp64, ms64 = replica_rate(pts, args.steps, r64["ms"])
    mixed, ms32 = replica_rate(pts, args.steps, r32["ms"])
    value, msl = replica_rate(pts, args.steps, rl["ms"])
    sign_only, mss = replica_rate(pts, args.steps, rs["ms"])
    e2e, _ = replica_rate(pts, args.steps, 1e3 * e2e_s)

    # stated errors of the learned mixed (and mixed Deardorff) form against fp64
    def errors(r):
        a, b = r["meanbuf"], r64["meanbuf"]
        ub = float(np.mean(b[3]))
        rms = lambda m: np.sqrt(np.maximum(m[6], 0))
        spec = {}
        for (f, iz), sa in r["spectra"].items():
            sb = r64["spectra"][(f, iz)]
            key = "spectrum_%s_zplus%d_max_rel_err" % ("uw"[f // 2], round((iz - 0.5) * 2.0 / NZ * RE_TAU))
            # over the resolved band, relative to each wavenumber's FP64 energy
            spec[key] = float(np.max(np.abs(sa[1:NX // 3] - sb[1:NX // 3]) / np.maximum(sb[1:NX // 3], 1e-300)))
        return {"mean_u_max_err_over_ub": float(np.abs(a[3] - b[3]).max() / ub),
                "uw_max_err_over_max": float(np.abs(a[9] - b[9]).max() / max(np.abs(b[9]).max(), 1e-300)),
                "u_rms_max_err_over_max": float(np.abs(rms(a) - rms(b)).max() / max(rms(b).max(), 1e-300)),
                "divz_max": float(np.max(a[2])), "divz_max_fp64": float(np.max(b[2])), **spec,
                "after_steps": args.warmup + args.steps, "plus_profiled_stages": 3}

    # roofline of the dominant kernel (per-kernel CUDA events on the handle's stream)
    agg = {}
    for name, t in prof:
        base = name.split("<")[0]
        agg.setdefault(base, [name, 0.0])
        agg[base][1] += t
    top = max(agg.items(), key=lambda kv: kv[1][1])
    kname, (kfull, kms) = top[0], top[1]
    peak, peak_kind = peaks()
    ab = algorithmic_bytes(kname, NX, NY, NZ, 4, learned=True)
    achieved = ab / (kms / 1e3) / 1e9 if ab else None
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "traffic_k_row_fused_512x512x256.txt")
    if os.path.exists(tfile):
        for ln in open(tfile):
            f = ln.split()
            if len(f) >= 3 and f[0] == kname:
                traffic = float(f[2])
    stage_ms = sum(t for _, t in prof)
    # compute roof of the fused row kernel: its transform and pointwise flops
    # (12 complex transforms of 3nx/2 points at 5 N log2 N -- 10 with the
    # learned closure, whose phase I skips UY+iVY and WX+iWY -- and ~150 flops
    # per point of the pointwise rows) per padded row and level, against the
    # device's FP32 / FP64 FMA rate from the library's probe kernel
    mxp = 3 * NX // 2
    def fused_flops(transforms):
        return 3 * NY // 2 * NZ * (transforms * 5.0 * mxp * np.log2(mxp) + 150.0 * mxp)
    fma32, fma64 = P.fma_rate(4, dev), P.fma_rate(8, dev)
    def compute_roof(profile, peak, transforms=12):
        row_flops = fused_flops(transforms)
        ms = sum(t for n, t in profile if n.startswith("k_row_fused"))
        return {"kernel": "k_row_fused", "transforms_per_row": transforms, "flops_per_launch": row_flops, "kernel_ms": ms,
                "achieved_tflops": row_flops / (ms / 1e3) / 1e12, "peak_tflops": peak / 1e12,
                "frac": row_flops / (ms / 1e3) / peak, "peak_source": "les_probe_fma_rate (measured FMA rate)"}
    # the network's tensor-core kernel: 2*(11*64 + 2*64*64 + 64*6) flops per point
    fpp = 2 * (11 * 64 + 2 * 64 * 64 + 64 * 6)
    mlp_ms = sum(t for n, t in prof if n.startswith("k_mlp_infer"))
    mlp_tf = (fpp * pts / (mlp_ms / 1e3) / 1e12) if mlp_ms else None
    bf16_peak, bf16_kind = bf16_peak_tflops()

    line = {
        "metric": METRIC, "value": value, "unit": "Mpoint-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": msl / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "mixed: f32 transforms/advection/SGS, bf16 network, f64 pressure/reductions",
        "data": "synthetic",
        "config": {"workload": "channel 512x512x256 (3/2-padded 768x768), Re_tau=590, learned SGS closure with "
                               "Deardorff fallback, mixed precision, isurface=6, RK3 at CFL 0.5, seeded projected "
                               "random IC", "network": weights,
                   "learned_fallback": LEARNED_FALLBACK,
                   "global_batch": pts * world, "seq_len": None, "parallelism": "replicas%d" % world,
                   "l2": "working set (tens of GB) >> 126 MB L2; no flush needed"},
        "forms": {"learned_mixed": value, "fp64": fp64, "mixed": mixed,
                  "learned_mixed_vs_fp64": value / fp64, "mixed_vs_fp64": mixed / fp64,
                  "fp64_ms_per_step": ms64 / args.steps, "mixed_ms_per_step": ms32 / args.steps,
                  "learned_mixed_ms_per_step": msl / args.steps,
                  "learned_timed_stages": rl["stages_timed"], "learned_timed_stages_used": rl["stages_used"],
                  "learned_used_fraction": rl["stages_used"] / max(rl["stages_timed"], 1),
                  "learned_used_last_stage": rl["learned_status"][0],
                  "learned_dissipation_last_stage": rl["learned_status"][1],
                  "reference_dissipation_last_stage": rl["learned_reference"],
                  "learned_mixed_sign_test_only": sign_only,
                  "learned_mixed_sign_test_only_ms_per_step": mss / args.steps,
                  "learned_mixed_sign_test_only_used_fraction": rs["stages_used"] / max(rs["stages_timed"], 1)},
        "errors": {"learned_mixed_vs_fp64": errors(rl), "mixed_vs_fp64": errors(r32)},
        "e2e": {"value": e2e, "unit": "Mpoint-steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "mode": "device-resident drop-in: state (4-byte host reals, as the shipped reference keeps them) "
                        "uploaded once inside the timed region, statistics read back every step"},
        "gpu_launches": rl["launches"],
        "clocks": rl["clocks"],
        "roofline": {"bound": "hbm", "kernel": kfull, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                     "peak_source": peak_kind, "kernel_ms": kms, "stage_ms": stage_ms,
                     "algorithmic_bytes": ab},
        "roofline_network": {"bound": "tensor", "kernel": "k_mlp_infer", "achieved": mlp_tf, "peak": bf16_peak,
                             "unit": "TFLOP/s", "frac": (mlp_tf / bf16_peak) if mlp_tf else None,
                             "kernel_ms": mlp_ms, "flops_per_point": fpp, "peak_source": bf16_kind},
        "roofline_compute": {"learned_mixed_f32": compute_roof(prof, fma32, transforms=10), "mixed_f32": compute_roof(prof32, fma32),
                             "fp64": compute_roof(prof64, fma64)},
        "kernels_ms_stage2_learned_mixed": {n: round(t, 4) for n, t in prof},
        "kernels_ms_stage2_fp64": {n: round(t, 4) for n, t in prof64},
        "kernels_ms_stage2_mixed": {n: round(t, 4) for n, t in prof32},
        "physics": {"utau": rl["utau"], "divz_max": rl["divz_max"], "dt": rl["dt"]},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the same sample, warm-up and repeats as the reference arm
        v, cores, el = cpu_baseline(args.steps, warmup=args.warmup)
        line["cpu_baseline"] = {"value": v, "unit": "Mpoint-steps/s", "cores": cores, "kind": "port",
                                "sample": "512x512x4 slab of the 512x512x256 grid, %d warm-up + %d timed RK3 steps, "
                                          "FP64 oracle, %.1f s timed" % (args.warmup, args.steps, el)}
    if rank == 0:
        print(json.dumps(line))
    if _pg is not None:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
