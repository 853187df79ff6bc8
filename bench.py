"""Benchmark of the RK3 stage on B200: one JSON line per run (rank 0).

Workload (default): the curvilinear shock case — 256 x 128 x 128 cells on the wavy periodic
mapping, Ma 1.5 round jet, single-species ideal air, plain FP64 — advanced with the fused
one-launch-per-stage kernel.  A "step" is one SSP-RK3 step (three stages).

  value  Mcell-stage/s with the state resident in HBM, device-timed with CUDA events over K
         steps (max over ranks; N ranks run N independent replicas: weak scaling)
  e2e    the same metric through the public host-buffer call (DeviceCase.advance_from_host):
         every step uploads the ghosted Q and rho_i from pinned memory and downloads them
  roofline  one RK3 stage (the unit the algorithmic bytes are defined for: one fused launch in
         configurations 0-2, the prep pass and three pencil sweeps in configuration 3) against
         the measured HBM copy bandwidth, with B_alg = 8 (41 + 3 Ns + [Ns >= 2] Ns) bytes per
         interior cell-stage; `traffic` is the DRAM bytes per stage from an ncu capture
  cpu_baseline  the oracle (C++ FP64 restatement, OpenMP over all host cores) on a bounded
         sample of the same workload

  fp64 (in roofline)  the same stage against the measured FP64 FMA peak (libflame3d_probe.so):
         FP64 FLOPs per cell-stage from the ncu instruction counts in profiles/ncu_fp64.json

On one GPU the default (jet) run also measures, in the same JSON line: the reference's own
launch sequence of 1:1 kernels on the jet (`launch_sequence`), the mixed-precision stage on the
jet with its error against the FP64 stage after a bounded number of steps (`mixed`), and the
batched mixed-precision ensemble of 64 cases against the plain FP64 paths one case at a time,
with step p50/p99 and a bounded error check (`ensemble64`): the "batched mixed-prec" half of
the metric.  `--no-extras` skips them.

`--gpus N` without torchrun launches itself under torch.distributed.run with N ranks (one
process per GPU, replicas; rendezvous on 127.0.0.1).

`--impl reference` times the reference path's CPU implementation instead (the oracle port:
the reference's RHS exists only as Julia CUDA.jl kernels and Julia is not installed).
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
METRIC = "Mcell-stage/s plain FP64 vs batched mixed-prec; p50/p99 step latency at err"
UNIT = "Mcell-stage/s"
PEAKS = ROOT / "MEASURED_PEAKS.json"
E2E_LANES = 3  # cases / streams the end-to-end calls rotate over
TRAFFIC = ROOT / "profiles" / "ncu_traffic.json"
FP64_COUNTS = ROOT / "profiles" / "ncu_fp64.json"


def _package():
    if "flame3d_b200" in sys.modules:
        return sys.modules["flame3d_b200"]
    pkg = ROOT / "flame3d.jl_b200"
    spec = importlib.util.spec_from_file_location("flame3d_b200", pkg / "__init__.py",
                                                  submodule_search_locations=[str(pkg)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["flame3d_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def b_alg(ns: int, precision: int = 0) -> int:
    """Algorithmic bytes per interior cell-stage of a perfectly fused stage: Q read 7 +
    metrics 10 + mu, lambda 2 + U read 5 + Un 5 + U write 5 + Q write 7 = 41 words, plus
    3 Ns (rho_i read, rho_n, rho_i write) and Ns for D when Ns >= 2.  Mixed precision stores
    Q, mu, lambda, D in 4 bytes."""
    d = ns if ns >= 2 else 0
    if precision == 0:
        return 8 * (41 + 3 * ns + d)
    return 4 * (7 + 2 + 7 + d) + 8 * (10 + 15 + 3 * ns)


WORKLOADS = {
    "jet256x128x128": dict(kind="jet", nx=256, ny=128, nz=128),
    "jet128x64x64": dict(kind="jet", nx=128, ny=64, nz=64),
    "tgv64": dict(kind="tgv", n=64),
    "mix192_ns9": dict(kind="mixing", n=192, ns=9),
    # the reference's own transport: mixture-averaged (thermo.jl:289-369) with seeded fits
    "mix96_ns9_law2": dict(kind="mixing", n=96, ns=9, law2=True),
    "ensemble64": dict(kind="ensemble"),
    "serve": dict(kind="serve"),
    "precision": dict(kind="precision"),
}


def make_case(f3d, name: str, nz_override: int | None = None):
    w = dict(WORKLOADS[name])
    kind = w.pop("kind")
    if kind == "jet":
        if nz_override:
            w["nz"] = nz_override
        return f3d.curvilinear_jet(**w)
    if kind == "tgv":
        return f3d.taylor_green(**w)
    law2 = w.pop("law2", False)
    case = f3d.mixing_layer(**w)
    if law2:
        case.transport = f3d.cases.mixture_averaged_transport(case.thermo, seed=3)
    return case


# ------------------------------------------------------------------------------ clocks
class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons of one GPU every 100 ms."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str | None):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines: list[str] = []
        self.t = None

    def start(self):
        try:
            cmd = ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                   "-lms", "100"]
            if self.gpu_id:
                cmd += ["-i", self.gpu_id]
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                         text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, ValueError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict | None:
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.t:
            self.t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax),
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------------------ CPU side
def cpu_sample(f3d, workload: str, stages: int):
    """Times the oracle on a bounded sample of the workload: `stages` RK3 stages on a
    256 x 128 x 16 slab of the same mapping and flow (1/8 of the cells)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    lib = oracle.load()
    w = WORKLOADS[workload]
    nz = 16 if w["kind"] == "jet" else None
    case = make_case(f3d, workload, nz_override=nz) if nz else make_case(f3d, workload)
    oc = oracle.OracleCase(case)
    oc.stage(1)  # warm-up (page faults, thread pool)
    t0 = time.perf_counter()
    for s in range(stages):
        oc.stage(1 + (s % 3))
    dt = time.perf_counter() - t0
    value = case.cells * stages / dt / 1e6
    return value, lib.oracle_num_threads(), case, dt


def run_reference(args, f3d):
    """The reference path's CPU implementation (the oracle port, all host threads) on a bounded
    sample of the workload: each step is one full RK3 step (three stages) of a 1/8 slab.  Under
    N ranks only rank 0 works; the ranks meet in a gloo process group so that every rank takes
    the same collective steps, and rank 0 prints the line with the N it ran under."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("gloo", timeout=timedelta(seconds=600))
    line = None
    if rank == 0:
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle
        lib = oracle.load()
        if WORKLOADS[args.workload]["kind"] not in ("jet", "tgv", "mixing"):
            args.workload = "jet256x128x128"  # case-set workloads: the reference RHS on the jet
        w = WORKLOADS[args.workload]
        nz = 16 if w["kind"] == "jet" else None
        case = make_case(f3d, args.workload, nz_override=nz) if nz else make_case(f3d, args.workload)
        oc = oracle.OracleCase(case)
        for _ in range(args.warmup):
            oc.step()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            oc.step()
        dt = time.perf_counter() - t0
        value = case.cells * 3 * args.steps / dt / 1e6
        sample = (f"each step = one RK3 step (3 stages) of the oracle (C++ FP64 restatement of "
                  f"the reference RHS) on a {case.nx}x{case.ny}x{case.nz} slab of the workload")
        line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": args.workload, "sample_cells": case.cells,
                           "step": "one RK3 step of the sample slab"},
                "cpu_baseline": {"value": value, "unit": UNIT, "cores": lib.oracle_num_threads(),
                                 "kind": "port", "sample": sample},
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)
    return 0


def _free_port() -> int:
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def relaunch_cmd(n: int, argv: list[str], port: int | None = None) -> list[str]:
    """The torch.distributed.run command that runs this script with n ranks on this node."""
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
            f"--nproc-per-node={n}", "--master-addr=127.0.0.1",
            f"--master-port={port or _free_port()}", str(Path(__file__).resolve()), *argv]


def relaunch(n: int, argv: list[str]) -> int:
    """--gpus N > 1 without torchrun: run N ranks of this script (one process per GPU) and
    return the launcher's status; rank 0's JSON line reaches stdout."""
    return subprocess.run(relaunch_cmd(n, argv)).returncode


# ------------------------------------------------------------------------------ ensemble
def _pct(xs, q):
    xs = sorted(xs)
    return xs[min(len(xs) - 1, int(round(q / 100 * (len(xs) - 1))))]


def ensemble_record(f3d, dev, k: int, warm: int = 3, check_steps: int = 20) -> dict:
    """64 independent periodic cases (sizes 32^3-128^3, 1-9 species): the batched
    mixed-precision path (one graph replay per RK3 step for all cases; persistent kernels as
    the other mode) against the plain FP64 paths advancing one case at a time (FIFO): the fused
    pencil stage and the reference launch sequence of 1:1 kernels.  Device-timed with CUDA
    events.  Error check: four cases (the smallest and largest, fewest and most species)
    advanced `check_steps` RK3 steps in a mixed-precision graph batch against the plain FP64
    stage from the same state, relative L2 of rho, rho*u, rho*E."""
    import torch
    S, B = f3d.solver_module(), f3d.batch_module()
    cases = f3d.cases.ensemble(64, seed=4)
    cells = sum(c.cells for c in cases)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def fifo(precision, fused, n):
        tot = 0.0
        for c in cases:
            dc = S.DeviceCase(c, device=dev, precision=precision, tile="auto" if fused else 3,
                              sequence_buffers=not fused)
            dc.step(fused)
            torch.cuda.synchronize(dev)
            e0.record()
            for _ in range(n):
                dc.step(fused)
            e1.record()
            torch.cuda.synchronize(dev)
            tot += e0.elapsed_time(e1)
            del dc
            torch.cuda.empty_cache()
        return cells * 3 * n / (tot / 1e3) / 1e6, tot / n

    plain, plain_ms = fifo(0, True, 3)
    seq, seq_ms = fifo(0, False, 1)
    pencil = [S.DeviceCase(c, device=dev, precision=1, tile=3) for c in cases]
    tuned = [S.DeviceCase(c, device=dev, precision=1, tile="auto") for c in cases]
    modes = {}
    for mode, dcs, nst in (("graph", tuned, 16), ("graph_s32", tuned, 32),
                           ("graph_pencil", pencil, 16), ("persistent", pencil, 16),
                           ("hybrid", pencil, 16)):
        batch = B.Batch(dcs, device=dev, mode=mode.split("_")[0], streams=nst)
        batch.capture()
        for _ in range(warm):
            batch.step()
        torch.cuda.synchronize(dev)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(k + 1)]
        ev[0].record()
        for i in range(k):
            batch.step()
            ev[i + 1].record()
        torch.cuda.synchronize(dev)
        per_step = [ev[i].elapsed_time(ev[i + 1]) for i in range(k)]
        ms = ev[0].elapsed_time(ev[k])
        modes[mode] = (cells * 3 * k / (ms / 1e3) / 1e6, ms, per_step)
        batch.close()
    best = max(modes, key=lambda m: modes[m][0])
    value, ms, per_step = modes[best]

    def persistent_launches(dcs):  # per step: two kernels per chunk and stage, four for law 2
        groups = {}
        for d in dcs:
            key = (d.case.ns, d.transport.law == 2)
            groups[key] = groups.get(key, 0) + 1
        return 3 * sum(((n + 19) // 20) * (4 if law2 else 2) for (_, law2), n in groups.items())

    small = [d for d in pencil if d.case.cells <= B.SMALL_CELLS]
    launches = (3 * sum(d.launches_per_stage() for d in tuned) if best in ("graph", "graph_s32")
                else 3 * sum(d.launches_per_stage() for d in pencil) if best == "graph_pencil"
                else persistent_launches(pencil) if best == "persistent"
                else persistent_launches(small)
                + 3 * sum(d.launches_per_stage() for d in pencil if d.case.cells > B.SMALL_CELLS))
    del pencil, tuned
    torch.cuda.empty_cache()
    # bounded error check
    pick = sorted(range(len(cases)), key=lambda i: (cases[i].cells, cases[i].ns))
    pick = sorted({pick[0], pick[-1], min(range(len(cases)), key=lambda i: cases[i].ns),
                   max(range(len(cases)), key=lambda i: cases[i].ns)})
    mixed = [S.DeviceCase(cases[i], device=dev, precision=1, tile="auto") for i in pick]
    batch = B.Batch(mixed, device=dev, mode="graph")
    for _ in range(check_steps):
        batch.step()
    batch.close()
    errs = {}
    for dc, i in zip(mixed, pick):
        ref = S.DeviceCase(cases[i], device=dev, precision=0, tile="auto")
        for _ in range(check_steps):
            ref.step()
        errs[cases[i].name] = _conserved_errors(dc.conserved(), ref.conserved(),
                                                lambda a: a[..., 4:-4, 4:-4, 4:-4])
        del ref
    del mixed
    torch.cuda.empty_cache()
    worst = {f: max(e[f] for e in errs.values()) for f in ("rho", "rhou", "rhoE")}
    return {"value": value, "unit": UNIT, "steps": k, "warmup": warm, "ms_per_step": ms / k,
            "dtype": "f32/f64", "cases": len(cases), "cells": cells,
            "path": f"batched stages ({best} mode), mixed precision, CUDA graph per step",
            "modes": {m: v[0] for m, v in modes.items()},
            "launches_per_step": launches,
            "step_latency_ms": {"p50": _pct(per_step, 50), "p99": _pct(per_step, 99)},
            "plain_fp64_fused_fifo": {"value": plain, "unit": UNIT,
                                      "ms_per_step_all_cases": plain_ms},
            "plain_fp64_launch_sequence_fifo": {"value": seq, "unit": UNIT,
                                                "ms_per_step_all_cases": seq_ms},
            "speedup_vs_plain_fp64_fused": value / plain,
            "speedup_vs_launch_sequence": value / seq,
            "error_check": {"steps": check_steps, "cases": errs, "max_rel_l2": worst,
                            "against": "plain FP64 fused stage from the same state"}}


def run_ensemble(args, f3d) -> int:
    """--workload ensemble64: the ensemble record as the JSON line."""
    import torch
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    r = ensemble_record(f3d, dev, max(args.steps // 10, 10), max(args.warmup, 3))
    out = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": 1, "steps": r["steps"],
           "warmup": r["warmup"], "ms_per_step": r["ms_per_step"], "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64",
           "data": "synthetic (seeded Taylor-Green ensemble with Fourier perturbations)",
           "config": {"workload": "ensemble64", "cases": r["cases"], "cells": r["cells"],
                      "path": r["path"], "modes": r["modes"],
                      "launches_per_step": r["launches_per_step"]},
           **{key: r[key] for key in ("step_latency_ms", "plain_fp64_fused_fifo",
                                     "plain_fp64_launch_sequence_fifo",
                                     "speedup_vs_plain_fp64_fused", "speedup_vs_launch_sequence",
                                     "error_check")}}
    print(json.dumps(out), flush=True)
    return 0


def _conserved_errors(U, Uref, interior) -> dict:
    """Relative L2 of ρ, ρu (the momentum vector field) and ρE."""
    import numpy as np
    I = interior
    rel = lambda a, b, n: float(np.linalg.norm((I(a) - I(b)).ravel()) / n)  # noqa: E731
    mom = np.linalg.norm(I(Uref[1:4]).ravel())
    return {"rho": rel(U[0], Uref[0], np.linalg.norm(I(Uref[0]).ravel())),
            "rhou": rel(U[1:4], Uref[1:4], mom),
            "rhoE": rel(U[4], Uref[4], np.linalg.norm(I(Uref[4]).ravel()))}


def run_precision(args, f3d) -> int:
    """Error of the mixed-precision path after 1000 RK3 steps.  Full-size configurations: mixed
    against the plain FP64 path on the GPU (itself within 1e-12 of the oracle in the parity
    tests).  Small cases: both GPU paths against the FP64 oracle on the host cores."""
    import numpy as np

    import torch
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    S = f3d.solver_module()
    steps = args.precision_steps
    I = oracle.interior
    out = {"steps": steps, "full_size": {}, "vs_oracle": {}}
    full = [("tgv64", f3d.taylor_green(n=64)), ("jet256x128x128", f3d.curvilinear_jet()),
            ("mix192_ns9", f3d.mixing_layer(n=192, ns=9))]
    for name, case in full:
        res = {}
        for prec in (0, 1):
            dc = S.DeviceCase(case, device=dev, precision=prec, tile=3)
            t0 = time.perf_counter()
            for _ in range(steps):
                dc.step()
            torch.cuda.synchronize(dev)
            res[prec] = (dc.conserved(), time.perf_counter() - t0)
            del dc
            torch.cuda.empty_cache()
        entry = {"mixed_vs_fp64": _conserved_errors(res[1][0], res[0][0], I),
                 "finite": bool(np.isfinite(res[1][0]).all()),
                 "seconds": {"fp64": res[0][1], "mixed": res[1][1]}}
        if name.startswith("jet"):
            # the flow's own sensitivity: plain FP64 from the initial state rounded to FP32
            import copy
            rounded = copy.copy(case)
            rounded.Q = case.Q.astype(np.float32).astype(np.float64)
            dc = S.DeviceCase(rounded, device=dev, precision=0, tile=3)
            for _ in range(steps):
                dc.step()
            entry["fp64_from_fp32_rounded_start_vs_fp64"] = _conserved_errors(
                dc.conserved(), res[0][0], I)
            del dc
            torch.cuda.empty_cache()
        out["full_size"][name] = entry
        print(json.dumps({name: out["full_size"][name]}), flush=True)
    small = [("tgv32", f3d.taylor_green(n=32)),
             ("jet64x32x32", f3d.curvilinear_jet(nx=64, ny=32, nz=32)),
             ("mix32_ns9", f3d.mixing_layer(n=32, ns=9))]
    for name, case in small:
        oc = oracle.OracleCase(case)
        t0 = time.perf_counter()
        for _ in range(steps):
            oc.step()
        t_or = time.perf_counter() - t0
        errs = {}
        for prec, label in ((0, "fp64"), (1, "mixed")):
            dc = S.DeviceCase(case, device=dev, precision=prec, tile=3)
            for _ in range(steps):
                dc.step()
            errs[label] = _conserved_errors(dc.conserved(), oc.U, I)
            del dc
        out["vs_oracle"][name] = {**errs, "oracle_seconds": t_or}
        print(json.dumps({name: out["vs_oracle"][name]}), flush=True)
    print(json.dumps({"workload": "precision", **out}), flush=True)
    return 0


def run_serve(args, f3d) -> int:
    """The serving stream: seeded Poisson arrivals (λ = 20/s) of solve requests with n
    log-uniform over 32-256, Cartesian or curvilinear, 1-9 species, Re 400-3200, Ma 0.1-1.5
    and 200-2000 RK3 steps scaled by --step-scale, admitted against a 150 GB HBM budget and
    served with continuous batching in mixed precision; against the same requests one at a time
    in arrival order with the plain FP64 stage.  Wall-clock makespan from the first arrival to
    the last completion (case construction on the device and result download included)."""
    import importlib

    import torch
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    S = importlib.import_module(f3d.__name__ + ".serving")
    reqs = S.request_stream(args.requests, rate=20.0, seed=5, step_scale=args.step_scale)
    warm = S.request_stream(3, rate=1000.0, seed=6, n_range=(16, 24), steps_range=(2, 3))
    S.fifo(warm, dev, precision=0)  # module loads, allocator, graph pools
    S.Server(dev, precision=1).run(warm)
    t_tune = time.perf_counter()
    tuned = S.pretune(reqs, dev)  # the autotuner's cache for every key of the stream
    t_tune = time.perf_counter() - t_tune
    torch.cuda.synchronize(dev)
    props = torch.cuda.get_device_properties(dev)
    uuid = getattr(props, "uuid", None)
    clk = ClockSampler(f"GPU-{uuid}" if uuid else None)
    clk.start()
    time.sleep(0.3)
    base = S.fifo(reqs, dev, precision=0)
    torch.cuda.empty_cache()
    seq = S.fifo(reqs, dev, precision=0, fused=False) if args.serve_sequence else None
    torch.cuda.empty_cache()
    srv = S.Server(dev, precision=1, hbm_budget=150e9)
    rep = srv.run(reqs)
    clocks = clk.stop()
    if args.serve_log:
        with open(args.serve_log, "w") as fh:
            for arm, r in (("fifo_fp64", base), ("fifo_fp64_sequence", seq),
                           ("serving_mixed", rep)):
                if r is None:
                    continue
                for pr in r["per_request"]:
                    fh.write(json.dumps({"arm": arm, **pr}) + "\n")
    drop = ("per_request",)
    summ = lambda r: {k: v for k, v in r.items() if k not in drop}  # noqa: E731
    value = rep["mcell_stage_per_s"]
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1,
           "steps": rep["step_latency_ms"]["steps"], "warmup": 3,
           "ms_per_step": rep["step_latency_ms"]["p50"], "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64",
           "data": "synthetic (seeded Poisson request stream, Taylor-Green initial states "
                   "built on the device)",
           "config": {"workload": "serve", "requests": len(reqs), "rate_per_s": 20.0,
                      "seed": 5, "step_scale": args.step_scale, "hbm_budget_bytes": 150e9,
                      "cell_stages": sum(r.cell_stages for r in reqs),
                      "path": "continuous batching, graph-mode batch, mixed precision, "
                              "autotuned stage configurations (both arms)",
                      "autotune": {"keys_tuned_before_serving": tuned, "seconds": t_tune},
                      "l2": "inputs of the large cases exceed L2; no flush between steps"},
           "step_latency_ms": rep["step_latency_ms"],
           "completion_latency_s": rep["completion_latency_s"],
           "serving": summ(rep), "plain_fp64_fifo": summ(base),
           "speedup_vs_plain_fp64_fifo": value / base["mcell_stage_per_s"],
           "plain_fp64_launch_sequence_fifo": summ(seq) if seq else None,
           "speedup_vs_launch_sequence_fifo": (value / seq["mcell_stage_per_s"]) if seq else None,
           "clocks": clocks}
    print(json.dumps(out), flush=True)
    return 0


# ------------------------------------------------------------------------------ FP64 roof
def fp64_peak_tflops(f3d, dev) -> float | None:
    """Measured FP64 FMA throughput of this GPU in TFLOP/s: the project's probe kernel
    (csrc/probe/fp64_peak.cu, eight independent FMA chains per thread, 8 blocks of 256 threads
    per SM), CUDA events over five launches after two warm-ups."""
    import ctypes as C
    import importlib

    import torch
    try:
        path = importlib.import_module(f3d.__name__ + ".build").build_probe()
    except (RuntimeError, OSError):
        return None
    lib = C.CDLL(str(path))
    fn = lib.flame_probe_fp64_fma
    fn.restype, fn.argtypes = C.c_double, [C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    blocks = 8 * torch.cuda.get_device_properties(dev).multi_processor_count
    out = torch.empty(blocks * 256, dtype=torch.float64, device=dev)
    s = torch.cuda.current_stream(dev)
    for _ in range(2):
        fn(blocks, 4000, out.data_ptr(), s.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    flops = sum(fn(blocks, 10000, out.data_ptr(), s.cuda_stream) for _ in range(5))
    e1.record(s)
    torch.cuda.synchronize(dev)
    return flops / (e0.elapsed_time(e1) / 1e3) / 1e12 if flops > 0 else None


# ------------------------------------------------------------------------------ extras
def _device_rate(dc, steps: int, warm: int = 1, fused: bool = True):
    """Mcell-stage/s of `steps` RK3 steps of one DeviceCase, CUDA events on its stream."""
    import torch
    for _ in range(warm):
        dc.step(fused)
    st = torch.cuda.current_stream(dc.device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dc.device)
    e0.record(st)
    for _ in range(steps):
        dc.step(fused)
    e1.record(st)
    torch.cuda.synchronize(dc.device)
    ms = e0.elapsed_time(e1)
    return dc.case.cells * 3 * steps / (ms / 1e3) / 1e6, ms / steps


def launch_sequence_record(f3d, case, dev, steps: int = 2) -> dict:
    """The reference's own kernel structure on the same GPU: solver.jl:298-326 as ~30 launches
    of the 1:1 entry points per stage (plain FP64), the literal drop-in."""
    import torch
    dc = f3d.solver_module().DeviceCase(case, device=dev, sequence_buffers=True)
    rate, ms = _device_rate(dc, steps, fused=False)
    del dc
    torch.cuda.empty_cache()
    return {"value": rate, "unit": UNIT, "ms_per_step": ms, "steps": steps,
            "path": "1:1 entry points, the reference's launch sequence (solver.jl:298-326)"}


def mixed_record(f3d, case, dev, steps: int) -> dict:
    """Mixed precision on the same workload: its device-timed rate, and after `steps` RK3 steps
    from the same initial state its relative L2 error in rho, rho*u, rho*E against the plain
    FP64 stage (itself within 1e-12 of the oracle per stage in the parity tests)."""
    import numpy as np
    import torch
    S = f3d.solver_module()
    mixed = S.DeviceCase(case, device=dev, precision=1, tile="auto")
    fp64 = S.DeviceCase(case, device=dev, precision=0, tile="auto")
    for _ in range(steps):
        mixed.step()
        fp64.step()
    U, Uref = mixed.conserved(), fp64.conserved()
    err = _conserved_errors(U, Uref, lambda a: a[..., 4:-4, 4:-4, 4:-4])
    rate, ms = _device_rate(mixed, 10)
    out = {"value": rate, "unit": UNIT, "ms_per_step": ms, "stage_config": mixed.launched_config,
           "error_vs_fp64_after_steps": steps, "rel_l2": err,
           "finite": bool(np.isfinite(U).all())}
    del mixed, fp64
    torch.cuda.empty_cache()
    return out


# ------------------------------------------------------------------------------ replicas
def max_over_ranks(ms: float, device=None) -> float:
    """The slowest rank's time: N replicas are done when the last one is (all_reduce MAX; on
    one process the time itself).  `device` is where the collective's tensor lives (the rank's
    GPU under NCCL, the CPU under gloo)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(ms)
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(cells: int, stages: int, ms_max: float, world: int) -> float:
    """Whole-job Mcell-stage/s of `world` replicas that each ran `stages` stages of `cells`
    cells, finished when the slowest did (weak scaling: per-rank work fixed)."""
    return world * cells * stages / (ms_max / 1e3) / 1e6


# ------------------------------------------------------------------------------ GPU side
def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="jet256x128x128", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--cpu-stages", type=int, default=3)
    ap.add_argument("--tile", type=lambda v: v if v == "auto" else int(v), default="auto",
                    help="stage configuration (0-3); default: the autotuner's choice")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--requests", type=int, default=48, help="serve: requests in the stream")
    ap.add_argument("--step-scale", type=float, default=0.05,
                    help="serve: factor on the requested 200-2000 steps")
    ap.add_argument("--serve-log", default=None, help="serve: per-request JSON lines to this file")
    ap.add_argument("--serve-sequence", action="store_true",
                    help="serve: also time the 1:1 launch-sequence FIFO (about a minute more)")
    ap.add_argument("--precision-steps", type=int, default=1000,
                    help="precision: RK3 steps before the errors are measured")
    ap.add_argument("--no-extras", action="store_true",
                    help="jet workload: skip the launch-sequence, mixed and ensemble records")
    ap.add_argument("--mixed-check-steps", type=int, default=100,
                    help="jet workload: RK3 steps before the mixed-vs-FP64 error is taken")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return relaunch(args.gpus, sys.argv[1:])
    f3d = _package()
    if args.impl == "reference":
        return run_reference(args, f3d)
    if args.workload == "ensemble64":
        return run_ensemble(args, f3d)
    if args.workload == "serve":
        return run_serve(args, f3d)
    if args.workload == "precision":
        return run_precision(args, f3d)

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    # under torchrun the ranks always form an NCCL group, one rank included, so that the
    # barriers and the max-over-ranks reduction run the same calls at every N
    distributed = "WORLD_SIZE" in os.environ
    if distributed:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=dev)
    prec = 0 if args.precision == "fp64" else 1
    case = make_case(f3d, args.workload)
    dc = f3d.solver_module().DeviceCase(case, device=dev, precision=prec, tile=args.tile)
    stream = torch.cuda.current_stream(dev)

    def barrier():
        if distributed:
            dist.barrier()
        torch.cuda.synchronize(dev)

    for _ in range(args.warmup):
        dc.step()
    barrier()
    props = torch.cuda.get_device_properties(dev)
    uuid = getattr(props, "uuid", None)
    clk = ClockSampler(f"GPU-{uuid}" if uuid else None)
    clk.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record(stream)
    for _ in range(args.steps):
        dc.step()
    e1.record(stream)
    barrier()
    clocks = clk.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), dev)
    stages = 3 * args.steps
    cells = case.cells
    launches_per_stage = dc.launches_per_stage()
    stage_path, stage_config = dc.stage_kernels(), dc.launched_config
    value = replica_rate(cells, stages, ms, world)
    stage_ms = ms / stages  # device time of one stage (all of its launches)

    # ---- end to end through the host-buffer API (pinned host memory, copies timed).  Each
    # step is one call: upload Q, rho_i from pinned host memory, prim2c, one RK3 step, download
    # Q, rho_i.  Serial: one call after the other on one stream.  Pipelined (reported as e2e):
    # independent calls rotate over three cases on three streams, so while one call computes the
    # others upload and download (PCIe is full duplex; a call's two copies together take about
    # as long as its step, so two lanes leave the GPU idle between steps); every step still
    # makes its own copies.
    ns = case.ns
    Qh = torch.from_numpy(case.Q).pin_memory()
    rh = torch.from_numpy(case.rhoi).pin_memory()
    Qo = [torch.empty_like(Qh).pin_memory() for _ in range(E2E_LANES)]
    ro = [torch.empty_like(rh).pin_memory() for _ in range(E2E_LANES)]
    # at least ten calls per lane: the pipeline's first upload and last download (about two
    # steps' worth of copies) are not overlapped, and over fewer calls they would weigh as a
    # throughput loss that a continuously running caller does not have
    e2e_steps = E2E_LANES * max(10, min(args.steps, 60) // E2E_LANES)
    for _ in range(2):
        dc.advance_from_host(Qh, rh, 1, Qo[0], ro[0])
    barrier()
    e0.record(stream)
    for _ in range(e2e_steps):
        dc.advance_from_host(Qh, rh, 1, Qo[0], ro[0])
    e1.record(stream)
    barrier()
    ms_serial = max_over_ranks(e0.elapsed_time(e1), dev)
    dcs = [dc] + [dc.clone() for _ in range(E2E_LANES - 1)]
    lanes = [torch.cuda.Stream(dev) for _ in range(E2E_LANES)]
    for k in range(E2E_LANES):  # warm the other cases and every stream
        with torch.cuda.stream(lanes[k]):
            dcs[k].advance_from_host(Qh, rh, 1, Qo[k], ro[k])
    barrier()
    e0.record(stream)
    for i in range(e2e_steps):
        k = i % E2E_LANES
        lanes[k].wait_event(e0)
        with torch.cuda.stream(lanes[k]):
            dcs[k].advance_from_host(Qh, rh, 1, Qo[k], ro[k])
    for ln in lanes:
        stream.wait_stream(ln)
    e1.record(stream)
    barrier()
    ms_e2e = max_over_ranks(e0.elapsed_time(e1), dev)
    e2e_value = replica_rate(cells, 3 * e2e_steps, ms_e2e, world)
    e2e_serial = replica_rate(cells, 3 * e2e_steps, ms_serial, world)
    del dcs
    h2d = (Qh.numel() * Qh.element_size() + rh.numel() * rh.element_size())
    d2h = (Qo[0].numel() * Qo[0].element_size() + ro[0].numel() * ro[0].element_size())

    if rank != 0:
        if distributed:
            dist.destroy_process_group()
        return 0

    # ---- roofline of one stage
    peaks = json.loads(PEAKS.read_text()) if PEAKS.exists() else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    balg = b_alg(ns, prec)
    achieved = balg * cells / (stage_ms / 1e3) / 1e9
    traffic = None
    if TRAFFIC.exists():
        tr = json.loads(TRAFFIC.read_text()).get(f"{args.workload}:{args.precision}:{stage_config}")
        if tr:
            traffic = tr.get("bytes_per_stage")
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": traffic,
            "peak_source": "measured" if PEAKS.exists() else "fallback",
            "kernel": stage_path, "b_alg_bytes_per_cell": balg,
            "stage_ms": stage_ms}
    # the compute roof of the plain FP64 stage: FP64 FLOPs per cell-stage (ncu instruction
    # counts, committed under profiles/) at the measured rate, against the measured FP64 peak
    counts = json.loads(FP64_COUNTS.read_text()) if FP64_COUNTS.exists() else {}
    fc = counts.get(f"{args.workload}:{args.precision}")
    if fc and prec == 0:
        fpk = fp64_peak_tflops(f3d, dev)
        fach = fc["flop_per_cell_stage"] * cells / (stage_ms / 1e3) / 1e12
        roof["fp64"] = {"achieved": fach, "peak": fpk, "unit": "TFLOP/s",
                        "frac": fach / fpk if fpk else None,
                        "flop_per_cell_stage": fc["flop_per_cell_stage"],
                        "peak_source": "measured (csrc/probe/fp64_peak.cu, this run)",
                        "counts_source": counts.get("source")}
        roof["limiter"] = ("neither roof: FP64 issue and latency at 24 of 64 warps per SM on "
                           "the y and z sweeps (profiles/pencil_stage_traffic_jet128x64x64.md)")

    cpu = None
    if not args.no_cpu:
        cv, cores, cc, secs = cpu_sample(f3d, args.workload, args.cpu_stages)
        cpu = {"value": cv, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{args.cpu_stages} RK3 stages of the oracle on a "
                         f"{cc.nx}x{cc.ny}x{cc.nz} slab of the workload ({secs:.1f} s)"}

    extras = {}
    if world == 1 and args.workload == "jet256x128x128" and not args.no_extras:
        del dc
        torch.cuda.empty_cache()
        extras["launch_sequence"] = launch_sequence_record(f3d, case, dev)
        if prec == 0:
            extras["mixed"] = mixed_record(f3d, case, dev, args.mixed_check_steps)
        extras["ensemble64"] = ensemble_record(f3d, dev, 10)
        extras["extras_note"] = (
            "launch_sequence: the reference's ~30 launches per stage of 1:1 kernels on this jet; "
            "mixed: the same jet in mixed precision; ensemble64: BASELINE config 4, batched "
            "mixed precision vs the plain FP64 paths one case at a time")

    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f64" if prec == 0 else "f32/f64",
           "data": "synthetic (seeded jet on the wavy periodic mapping)",
           "config": {"workload": args.workload, "cells": cells, "species": ns,
                      "precision": args.precision, "path": stage_path, "stage_config": stage_config,
                      "l2": "inputs larger than L2 (state ~%.1f GB per replica)" % (
                          (35 + 3 * ns) * case.Q[0].size * 8 / 1e9),
                      "parallelism": f"replicas x{world}"},
           "roofline": roof, "cpu_baseline": cpu, "clocks": clocks,
           "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                   "d2h_bytes_per_step": d2h, "steps": e2e_steps,
                   "calls": "DeviceCase.advance_from_host, one RK3 step per call, independent "
                            f"calls rotating over {E2E_LANES} cases on {E2E_LANES} streams",
                   "serial_one_stream": e2e_serial},
           "gpu_launches": stages * launches_per_stage, **extras}
    print(json.dumps(out), flush=True)
    if distributed:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
