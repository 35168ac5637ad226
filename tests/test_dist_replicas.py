"""The host side of bench.py on CPU: two ranks over gloo (127.0.0.1) run
the replica aggregation the GPU runs use over NCCL (a barrier, the
max-over-ranks time and the whole-job rate: all ranks' points over the
slowest rank's time); a rank other than 0 of the reference arm exits without
output; rank 0 of the reference arm prints the contract's JSON line."""
import importlib.util
import multiprocessing as mp
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, ms, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist
    b = _bench()
    b.init_dist("gloo", timeout_s=60)
    b.barrier()
    rate, mx = b.replica_rate(1000, 5, ms[rank])
    q.put((rank, rate, mx))
    b.barrier()
    dist.destroy_process_group()


def test_replica_rate_two_ranks_gloo():
    ms = [10.0, 25.0]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, ms, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, rate, mx in res:
        assert mx == max(ms)
        assert rate == pytest.approx(2 * 1000 * 5 / (max(ms) / 1e3) / 1e6)


def test_single_rank_rate_needs_no_group():
    b = _bench()
    rate, mx = b.replica_rate(1000, 5, 10.0)
    assert mx == 10.0 and rate == pytest.approx(1000 * 5 / 0.01 / 1e6)


def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2", MASTER_ADDR="127.0.0.1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_reference_arm_line_contract():
    """Rank 0 of the reference arm prints one JSON line with the contract's
    keys; its e2e moves no host-device bytes (the oracle port runs on CPU)."""
    import json
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e", "impl"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert "workload" in d["config"]
