"""bench.py's replica bookkeeping with two gloo ranks on the CPU: every rank sees the slowest
rank's time, and the whole-job rate counts all ranks' cells (weak scaling)."""
from __future__ import annotations

import importlib.util
import os
import socket
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        b = _bench()
        ms = b.max_over_ranks(10.0 * (rank + 1))  # rank 1 is twice as slow
        out[rank] = (ms, b.replica_rate(1_000_000, 30, ms, world))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_agree_on_the_slowest():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0] == res[1]
    ms, rate = res[0]
    assert ms == 20.0
    assert rate == 2 * 1_000_000 * 30 / 0.020 / 1e6


def test_single_process_is_its_own_max():
    b = _bench()
    assert b.max_over_ranks(7.5) == 7.5
    assert b.replica_rate(100, 3, 1.0, 1) == 100 * 3 / 1e-3 / 1e6


def test_gpus_flag_self_launches_gloo_ranks():
    """`bench.py --gpus 2` without torchrun starts two ranks itself (torch.distributed.run on
    127.0.0.1).  The reference arm needs no GPU: its ranks meet in a gloo group, rank 0 alone
    runs the oracle and prints one line with the N it ran under."""
    import json
    import subprocess
    import sys
    env = {k: v for k, v in os.environ.items()
           if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT")}
    env["OMP_NUM_THREADS"] = "2"
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus",
                        "2", "--workload", "tgv64", "--steps", "1", "--warmup", "3"],
                       capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(ln) for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["value"] > 0 and line["config"]["step"].startswith("one RK3 step")


def test_relaunch_command_is_torchrun_on_localhost():
    b = _bench()
    cmd = b.relaunch_cmd(4, ["--steps", "2"], port=29555)
    assert cmd[1:3] == ["-m", "torch.distributed.run"]
    assert "--nproc-per-node=4" in cmd and "--master-addr=127.0.0.1" in cmd
    assert "--master-port=29555" in cmd and cmd[-2:] == ["--steps", "2"]
