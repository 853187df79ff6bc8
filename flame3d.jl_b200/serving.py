"""Serving: a request loop over resident simulations with continuous batching.

A client sends solve requests (grid size, Cartesian or curvilinear, species count, Re, Ma and a
number of RK3 steps).  The server

* builds each admitted case's initial state and metrics directly on the GPU (torch operations on
  the device; the same formulas as the numpy generators in `cases`),
* admits requests in arrival order while their resident bytes fit the HBM budget and a slot is
  free, and keeps every admitted case's state, metrics and scratch on the device until it
  completes,
* advances all admitted cases together one RK3 step at a time (a graph-mode `Batch`: every
  case's launch chain on one of several streams, so their work overlaps on the device), and
  changes the batch only at step boundaries: finished cases leave, waiting requests join,
* downloads a case's primitive state when its last step is done.

It records per-request admit / first-step / finish times and the latency of each batched step,
and reports p50 / p99 per-step and completion latency beside the aggregate Mcell-stage/s.
`fifo` is the baseline: the same requests one at a time in arrival order on the same GPU.

The reference has no serving layer: its driver (solver.jl:58-510) runs one case per process.
A case's result does not depend on the cases it shares the GPU with: each case has its own
kernels, buffers and reduction order, and no kernel reads another case's memory.
"""
from __future__ import annotations

import math
import queue as _queue
import time
from collections import deque
from concurrent.futures import ThreadPoolExecutor
from dataclasses import asdict, dataclass, field

import numpy as np
import torch

from . import abi
from .batch import Batch
from .cases import (NG, Case, Transport, cartesian_metrics, ghosted, ideal_air,
                    metrics_from_mapping, periodic_fill, synthetic_species, wavy_mapping)
from .solver import DeviceCase


# ------------------------------------------------------------------------------------ requests
@dataclass
class SolveRequest:
    rid: int
    arrival: float          # seconds after the stream opens
    n: int                  # cells per direction (cube)
    curvilinear: bool       # the wavy mapping (scaled to [0, 2π)) instead of a uniform grid
    ns: int                 # species, 1..9
    Re: float
    Ma: float
    steps: int              # RK3 steps to run
    seed: int

    @property
    def cells(self) -> int:
        return self.n ** 3

    @property
    def cell_stages(self) -> int:
        return 3 * self.steps * self.cells


def request_stream(count: int, rate: float = 20.0, seed: int = 5, n_range=(32, 256),
                   steps_range=(200, 2000), step_scale: float = 1.0, ns_range=(1, 9),
                   Re_range=(400.0, 3200.0), Ma_range=(0.1, 1.5),
                   curvilinear_fraction: float = 0.5) -> list[SolveRequest]:
    """Seeded Poisson stream: exponential inter-arrival times of mean 1/rate, n log-uniform over
    n_range (rounded to an integer), Cartesian or curvilinear with the given odds, species,
    Re, Ma uniform over their ranges, steps uniform over steps_range then multiplied by
    step_scale (at least 1)."""
    rng = np.random.default_rng(seed)
    out, t = [], 0.0
    lo, hi = math.log(n_range[0]), math.log(n_range[1])
    for i in range(count):
        t += float(rng.exponential(1.0 / rate))
        n = int(round(math.exp(rng.uniform(lo, hi))))
        curv = bool(rng.random() < curvilinear_fraction)
        ns = int(rng.integers(ns_range[0], ns_range[1] + 1))
        Re = float(rng.uniform(*Re_range))
        Ma = float(rng.uniform(*Ma_range))
        steps = int(rng.integers(steps_range[0], steps_range[1] + 1))
        steps = max(1, int(round(steps * step_scale)))
        out.append(SolveRequest(i, t, n, curv, ns, Re, Ma, steps, seed * 100003 + i))
    return out


# ------------------------------------------------------------------- initial state on a device
def _noise_axis(rng, x, kmax=8, nmodes=24):
    """Random-phase modes with integer wavenumbers |k| <= kmax on a cube whose three axes are
    the 1-D coordinate `x`: the same draws and sums as cases._fourier_noise."""
    n = x.shape[0]
    acc = torch.zeros((n, n, n), dtype=torch.float64, device=x.device)
    for _ in range(nmodes):
        while True:
            k = rng.integers(-kmax, kmax + 1, 3)
            if 0 < np.linalg.norm(k) <= kmax:
                break
        ph = float(rng.uniform(0, 2 * math.pi))
        ex = torch.exp(1j * float(k[0]) * x)
        ey = torch.exp(1j * float(k[1]) * x)
        ez = torch.exp(1j * (float(k[2]) * x + ph))
        acc += (ez[:, None, None] * ey[None, :, None] * ex[None, None, :]).imag
    return acc / nmodes


def _cfl_dt(Q, metrics, n, cfl):
    """cases.cfl_dt on the device: flame_cfl_max (strict IEEE, the host rule's operation order)
    for CUDA tensors, torch operations otherwise."""
    if Q.is_cuda:
        import ctypes as C
        lib = abi.load_library()
        out = torch.empty(1, dtype=torch.float64, device=Q.device)
        cm = abi.FlameMetrics(**{k: v.data_ptr() for k, v in metrics.items()})
        g = abi.FlameGrid(n, n, n, NG, 1, 7)
        rc = lib.flame_cfl_max(C.byref(g), C.c_void_p(torch.cuda.current_stream(Q.device).cuda_stream),
                               Q.data_ptr(), C.byref(cm), out.data_ptr())
        abi.check(lib, rc)
        return float(cfl / out.item())
    sl = (slice(NG, NG + n),) * 3
    rho, u, v, w, p, e = (Q[k][sl] for k in (0, 1, 2, 3, 4, 6))
    c = torch.sqrt((p / e + 1) * p / rho)
    J = metrics["J"][sl]
    tot = torch.zeros_like(rho)
    for a, b, cc in (("dxidx", "dxidy", "dxidz"), ("detadx", "detady", "detadz"),
                     ("dzetadx", "dzetady", "dzetadz")):
        mx, my, mz = metrics[a][sl], metrics[b][sl], metrics[cc][sl]
        tot += J * ((mx * u + my * v + mz * w).abs() + c * torch.sqrt(mx * mx + my * my + mz * mz))
    return float(cfl / tot.max().item())


def build_request_case(req: SolveRequest, device="cuda", species_seed: int = 3,
                       perturb: float = 0.02, cfl: float = 0.5) -> Case:
    """The request's initial state, built on `device` (a `Case` whose Q, rhoi and metrics are
    torch tensors there).

    A Taylor-Green vortex on [0, 2π)^3 (cases.taylor_green: T0 = 300 K, p0 = 101325 Pa,
    U0 = Ma sqrt(γ R T0), μ = ρ0 U0 / Re, uniform random mixture of the first ns synthetic
    species, `perturb` relative random-phase modes with |k| <= 8 on u, v, w), on a uniform grid
    or on the wavy curvilinear mapping scaled to [0, 2π).  Above Ma ≈ 1.38 the TGV pressure
    field p0 + ρ0 U0²/16 (cos 2x + cos 2y)(cos 2z + 2) goes negative, so its fluctuation is
    scaled to keep p >= 0.2 p0 (a factor min(1, 0.8 / (6 γ Ma² / 16)); 1 below Ma 1.23).
    On a Cartesian request it reproduces cases.taylor_green(n, Re, Ma, ns, perturb, seed)."""
    n, ns = req.n, req.ns
    dev = torch.device(device)
    thermo = ideal_air() if ns == 1 else synthetic_species(9, species_seed).subset(ns)
    rng = np.random.default_rng(req.seed)
    Y = np.ones(1) if ns == 1 else rng.dirichlet(np.ones(ns))
    h = 2 * math.pi / n
    if req.curvilinear:
        xyz = wavy_mapping(n, n, n, amp=0.1, scale=2 * math.pi)
        metrics = metrics_from_mapping(xyz, n, n, n, device=dev)
    else:
        xyz = lambda i, j, k: (i * h, j * h, k * h)  # noqa: E731
        metrics = cartesian_metrics(n, n, n, h, h, h, device=dev)
    ar = torch.arange(0, n, dtype=torch.float64, device=dev)
    K, Jg, I = torch.meshgrid(ar, ar, ar, indexing="ij")
    X, Yg, Z = xyz(I, Jg, K)
    del K, Jg, I
    T0, p0 = 300.0, 101325.0
    Wmix = 1.0 / np.sum(Y / thermo.mw)
    R = thermo.Ru / Wmix
    cp = float(thermo.cp_mass(np.array([T0]), Y[:, None])[0])
    gam = cp / (cp - R)
    U0 = req.Ma * math.sqrt(gam * R * T0)
    rho0 = p0 / (R * T0)
    u = U0 * torch.sin(X) * torch.cos(Yg) * torch.cos(Z)
    v = -U0 * torch.cos(X) * torch.sin(Yg) * torch.cos(Z)
    w = torch.zeros_like(u)
    if perturb > 0:
        xs = ar * h  # modes in index space, periodic on either grid
        for comp in (u, v, w):
            comp += perturb * U0 * _noise_axis(rng, xs)
    damp = min(1.0, 0.8 / (6.0 * gam * req.Ma ** 2 / 16.0))
    p = p0 + damp * rho0 * U0 ** 2 / 16 * (torch.cos(2 * X) + torch.cos(2 * Yg)) * \
        (torch.cos(2 * Z) + 2)
    del X, Yg, Z
    rho = p / (R * T0)
    # _finish: p and e recomputed from T and rho_i with the thermo formulas (thermo.jl:20-26,
    # 219-228), in the operation order of Thermo.pressure / Thermo.internal_energy
    Tt = np.array([T0])
    rhoi_int = [rho * float(Y[k]) for k in range(ns)]
    yow = torch.zeros_like(rho)
    for k in range(ns):
        yow = yow + rhoi_int[k] / float(thermo.mw[k])
    p = thermo.Ru * T0 * yow
    e = torch.zeros_like(rho)
    for k, ek in enumerate(thermo.species_energy(Tt)):
        e = e + rhoi_int[k] * float(ek[0]) / float(thermo.mw[k])
    e = e * thermo.Ru
    tx, ty, tz = ghosted(n, n, n)
    Q = torch.zeros((7, tz, ty, tx), dtype=torch.float64, device=dev)
    rhoi = torch.zeros((ns, tz, ty, tx), dtype=torch.float64, device=dev)
    sl = (slice(NG, NG + n),) * 3
    for k, f in enumerate((rho, u, v, w, p, None, e)):
        if f is None:
            Q[(5,) + sl] = T0
        else:
            Q[(k,) + sl] = f
    for k in range(ns):
        rhoi[(k,) + sl] = rhoi_int[k]
    del rho, u, v, w, p, e, yow, rhoi_int
    periodic_fill(Q, n, n, n)
    periodic_fill(rhoi, n, n, n)
    mu = rho0 * U0 * 1.0 / req.Re
    tr = Transport(law=0, mu_ref=mu, Pr=0.71, lambda_ref=cp * mu / 0.71,
                   D_ref=cp * mu / 0.71 / (rho0 * cp))
    name = f"req{req.rid:04d}_{'curv' if req.curvilinear else 'cart'}{n}_ns{ns}"
    info = {"Re": req.Re, "Ma": req.Ma, "U0": U0, "rho0": rho0, "seed": req.seed, "h": h,
            "cfl": cfl}
    c = Case(name, n, n, n, thermo, tr, metrics, Q, rhoi, 0.0, req.steps, 7, info)
    c.dt = _cfl_dt(Q, metrics, n, cfl)
    return c


def case_to_host(c: Case) -> Case:
    """A numpy copy of a device-built case (for the oracle)."""
    cpu = lambda t: t.detach().cpu().numpy()  # noqa: E731
    return Case(c.name, c.nx, c.ny, c.nz, c.thermo, c.transport,
                {k: cpu(v) for k, v in c.metrics.items()}, cpu(c.Q), cpu(c.rhoi), c.dt,
                c.steps, c.periodic, dict(c.info))


def resident_bytes(req: SolveRequest, precision: int, lib=None) -> int:
    """Device bytes a DeviceCase of this request holds while it is resident: metrics (10 FP64),
    Q in/out (7 each), transport in/out (3 each) in the storage type, rho_i in/out, rho_n, U, Un
    in FP64, and the pencil configuration's scratch (flame_stage_scratch_bytes)."""
    import ctypes as C
    lib = lib or abi.load_library()
    tx, ty, tz = ghosted(req.n, req.n, req.n)
    P = tx * ty * tz
    q = 8 if precision == 0 else 4
    g = abi.FlameGrid(req.n, req.n, req.n, NG, req.ns, 7)
    scratch = int(lib.flame_stage_scratch_bytes(C.byref(g), precision))
    return P * (8 * (10 + 10 + 3 * req.ns) + q * (14 + 6)) + scratch


# -------------------------------------------------------------------------------------- server
def admissions(queue: deque, nbytes, used: int, budget: int, free_slots: int):
    """Admission at a step boundary, first come first served: pops from the head of `queue`
    the requests that fit in the budget's remainder and the free slots, stopping at the first
    one that does not fit (later requests wait behind it), and pops requests that could never
    fit (more than the whole budget).  Returns (admitted, rejected)."""
    admit, reject = [], []
    while queue and len(admit) < free_slots:
        b = nbytes(queue[0])
        if b > budget:
            reject.append(queue.popleft())
            continue
        if used + b > budget:
            break
        used += b
        admit.append(queue.popleft())
    return admit, reject


def _pct(xs, q):
    return float(np.percentile(np.asarray(xs, dtype=np.float64), q)) if len(xs) else None


@dataclass
class RequestRecord:
    rid: int
    name: str
    cells: int
    steps: int
    bytes: int
    arrival: float
    admitted: float = math.nan
    first_step: float = math.nan
    finished: float = math.nan
    rejected: str | None = None
    failed: str | None = None   # stopped early: the NaN check found a non-finite state
    finite: bool = True
    step_ms: list = field(default_factory=list, repr=False)

    def summary(self) -> dict:
        d = {k: v for k, v in asdict(self).items() if k != "step_ms"}
        d["completion_latency_s"] = self.finished - self.arrival
        d["queue_wait_s"] = self.admitted - self.arrival
        d["step_ms_p50"] = _pct(self.step_ms, 50)
        d["step_ms_p99"] = _pct(self.step_ms, 99)
        run = self.finished - self.first_step
        d["mcell_stage_per_s"] = 3 * self.steps * self.cells / run / 1e6 if run > 0 else None
        return d


@dataclass(eq=False)
class _Slot:
    req: SolveRequest
    rec: RequestRecord
    dc: DeviceCase
    remaining: int
    done_steps: int = 0


class Server:
    """Continuous-batching server on one GPU.

    precision: 1 = mixed (FP32 storage and bulk arithmetic, FP64 accumulation), 0 = FP64.
    hbm_budget: bytes of resident case state admitted at once (resident_bytes per request).
    max_slots: cases advanced together at most.
    capture: replay a batch composition's step as CUDA graphs when that pays (_should_capture).
    check_every: every that many steps each case's U is checked for NaN / inf (the reference's
        check, solver.jl:388-391, every 10 steps); a failing case stops early, its result is
        copied out for inspection and its slot and bytes are freed.
    keep_results: keep each finished case's (Q, rho_i) on the host in `results`.
    """

    def __init__(self, device="cuda", precision: int = 1, hbm_budget: float = 150e9,
                 max_slots: int = 64, streams: int = 16, capture: bool = True,
                 keep_results: bool = False, builder=build_request_case,
                 capture_min_steps: int = 8, tile="auto", check_every: int = 10):
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise abi.FlameError(1, "the server needs a CUDA device")
        self.lib = abi.load_library()
        self.precision = precision
        self.budget = int(hbm_budget)
        self.max_slots = max_slots
        self.streams = streams
        self.capture = capture
        self.capture_min_steps = capture_min_steps
        self.tile = tile
        self.check_every = check_every
        self.keep_results = keep_results
        self.builder = builder
        self.results: dict[int, tuple[np.ndarray, np.ndarray]] = {}
        self.trace: list[tuple[float, int, int]] = []  # (time, active cases, resident bytes)
        self.build_stream = torch.cuda.Stream(self.device)
        self.copy_stream = torch.cuda.Stream(self.device)

    def _admit(self, req: SolveRequest, rec: RequestRecord, now: float) -> _Slot:
        """Builds the case on the build stream (overlapping the batch step in flight); the
        main stream waits for it before the next step."""
        rec.admitted = now
        with torch.cuda.stream(self.build_stream):
            case = self.builder(req, self.device)
            dc = DeviceCase(case, self.device, precision=self.precision, tile=self.tile)
        case.Q = case.rhoi = None  # the DeviceCase holds the state now
        case.metrics = {}
        torch.cuda.current_stream(self.device).wait_stream(self.build_stream)
        return _Slot(req, rec, dc, req.steps)

    def _download(self, s: _Slot, ready: torch.cuda.Event) -> None:
        """Worker thread: copies a finished case's primitive state (storage precision) to the
        host on the copy stream once `ready` (the end of its last step) has passed."""
        td = time.perf_counter()
        try:
            with torch.cuda.device(self.device), torch.cuda.stream(self.copy_stream):
                self.copy_stream.wait_event(ready)
                i = s.dc.cur
                finite = torch.isfinite(s.dc.Q[i]).all() & torch.isfinite(s.dc.rhoi[i]).all()
                Q, r = s.dc.Q[i].cpu().numpy(), s.dc.rhoi[i].cpu().numpy()
            s.rec.finite = bool(finite)
            if self.keep_results:
                self.results[s.req.rid] = (Q, r)
            s.rec.finished = time.perf_counter() - self._t0
        finally:
            self._download_s += time.perf_counter() - td
            self._done.put(s)

    def run(self, requests: list[SolveRequest]) -> dict:
        """Serves the stream in real time (arrival times from now on) and returns the report."""
        t0 = self._t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0  # noqa: E731
        future = deque(sorted(requests, key=lambda r: r.arrival))
        queue: deque = deque()
        active: list[_Slot] = []
        leaving: list = []  # finished cases whose results are being copied out
        self._done = _queue.Queue()
        self._download_s = 0.0
        pool = ThreadPoolExecutor(max_workers=1)
        jobs = []
        records: dict[int, RequestRecord] = {}
        st = {"used": 0, "busy_ms": 0.0, "build_s": 0.0, "download_s": 0.0, "capture_s": 0.0,
              "rebuilds": 0, "captures": 0, "peak_active": 0, "peak_bytes": 0, "steps": 0}
        batch, stable, pending = None, 0, None
        step_ms: list[float] = []
        launch_s = 0.0  # host time of the last eager batch.step()
        main = torch.cuda.current_stream(self.device)
        while future or queue or active or leaving:
            while not self._done.empty():  # downloads that completed: their memory is free
                s = self._done.get()
                st["used"] -= s.rec.bytes
                leaving = [x for x in leaving if x is not s]
                del s
            for j in jobs:
                if j.done() and j.exception() is not None:
                    pool.shutdown(wait=True)
                    raise j.exception()
            t = now()
            while future and future[0].arrival <= t:
                r = future.popleft()
                records[r.rid] = RequestRecord(r.rid, "", r.cells, r.steps,
                                               resident_bytes(r, self.precision, self.lib),
                                               r.arrival)
                queue.append(r)
            admit, reject = admissions(queue, lambda r: records[r.rid].bytes, st["used"],
                                       self.budget, self.max_slots - len(active))
            for r in reject:
                records[r.rid].rejected = (f"needs {records[r.rid].bytes} B, more than the "
                                           f"{self.budget} B budget")
            for r in admit:
                rec = records[r.rid]
                tb = time.perf_counter()
                s = self._admit(r, rec, now())
                st["build_s"] += time.perf_counter() - tb
                rec.name = s.dc.case.name
                active.append(s)
                st["used"] += rec.bytes
            if not active:
                if leaving:
                    time.sleep(1e-3)
                elif future:
                    time.sleep(max(0.0, future[0].arrival - now()))
                continue
            if admit or batch is None:
                if batch is not None:
                    batch.close()
                batch = Batch([s.dc for s in active], self.device, mode="graph",
                              streams=self.streams)
                st["rebuilds"] += 1
                stable = 0
            elif self._should_capture(batch, stable, active, future, step_ms, launch_s, now()):
                tc = time.perf_counter()
                batch.capture()
                st["capture_s"] += time.perf_counter() - tc
                st["captures"] += 1
            st["peak_active"] = max(st["peak_active"], len(active))
            st["peak_bytes"] = max(st["peak_bytes"], st["used"])
            self.trace.append((now(), len(active), st["used"]))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            tl = time.perf_counter()
            e0.record(main)
            batch.step()
            e1.record(main)
            if not batch.graphs:
                launch_s = time.perf_counter() - tl
            stable += 1
            # keep one step in flight: wait for the previous step, then account for it
            if pending is not None:
                st["busy_ms"] += self._account(pending, step_ms)
            pending = (e0, e1, [s.rec for s in active])
            for s in active:
                if math.isnan(s.rec.first_step):
                    s.rec.first_step = now()
                s.remaining -= 1
                s.done_steps += 1
            st["steps"] += 1
            if self.check_every and st["steps"] % self.check_every == 0:
                counts = [(s, s.dc.nonfinite_launch()) for s in active]
                for s, c in counts:
                    if s.remaining > 0 and int(c.item()) > 0:
                        s.rec.failed = f"non-finite state after {s.done_steps} steps"
                        s.remaining = 0
            done = [s for s in active if s.remaining == 0]
            if done:
                ready = torch.cuda.Event()
                ready.record(main)
                for s in done:
                    leaving.append(s)
                    jobs.append(pool.submit(self._download, s, ready))
                active = [s for s in active if s.remaining > 0]
                batch.close()
                batch = None
                del done, s
        if pending is not None:
            st["busy_ms"] += self._account(pending, step_ms)
        if batch is not None:
            batch.close()
        pool.shutdown(wait=True)
        st["download_s"] = self._download_s
        return _report(records, step_ms, st)

    def _should_capture(self, batch, stable, active, future, step_ms, launch_s, t) -> bool:
        """Capture the current composition's step as graphs when it pays: the batch ran one
        eager step, it will stay unchanged for at least capture_min_steps more steps (the
        nearest completion, and the next arrival at the last step's pace), and the GPU waits
        on the launches (the last step's device time under twice its host launch time)."""
        if not self.capture or batch.graphs or stable < 1 or not step_ms:
            return False
        last_s = step_ms[-1] / 1e3
        steps_left = min(s.remaining for s in active)
        if future:
            steps_left = min(steps_left, (future[0].arrival - t) / max(last_s, 1e-6))
        return steps_left >= self.capture_min_steps and last_s < 2 * launch_s

    @staticmethod
    def _account(ev, step_ms) -> float:
        e0, e1, recs = ev
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        step_ms.append(ms)
        for r in recs:
            r.step_ms.append(ms)
        return ms


def _report(records, step_ms, st) -> dict:
    busy_ms = st["busy_ms"]
    done = [r for r in records.values()
            if r.rejected is None and r.failed is None and not math.isnan(r.finished)]
    cs = sum(3 * r.steps * r.cells for r in done)
    first = min((r.arrival for r in records.values()), default=0.0)
    last = max((r.finished for r in done), default=first)
    lat = [r.finished - r.arrival for r in done]
    wait = [r.admitted - r.arrival for r in done]
    return {
        "requests": len(records), "completed": len(done),
        "rejected": sum(r.rejected is not None for r in records.values()),
        "failed": sum(r.failed is not None for r in records.values()),
        "nonfinite": sum(not r.finite for r in done),
        "cell_stages": cs,
        "makespan_s": last - first,
        "mcell_stage_per_s": cs / (last - first) / 1e6 if last > first else None,
        "busy_s": busy_ms / 1e3,
        "busy_mcell_stage_per_s": cs / (busy_ms / 1e3) / 1e6 if busy_ms > 0 else None,
        "step_latency_ms": {"p50": _pct(step_ms, 50), "p99": _pct(step_ms, 99),
                            "steps": len(step_ms)},
        "completion_latency_s": {"p50": _pct(lat, 50), "p99": _pct(lat, 99),
                                 "mean": float(np.mean(lat)) if lat else None},
        "queue_wait_s": {"p50": _pct(wait, 50), "p99": _pct(wait, 99)},
        "peak_active": st["peak_active"], "peak_resident_bytes": st["peak_bytes"],
        "batch_rebuilds": st["rebuilds"], "graph_captures": st["captures"],
        "graph_capture_s": st["capture_s"], "build_s": st["build_s"],
        "download_s": st["download_s"],
        "per_request": [r.summary() for r in sorted(records.values(), key=lambda r: r.rid)],
    }


def pretune(requests: list[SolveRequest], device="cuda", precisions=(0, 1),
            builder=build_request_case) -> int:
    """Fills the autotuner's cache for every (precision, species, size class) the requests
    need, ahead of serving; returns the number of configurations tuned."""
    from . import autotune
    tuner = autotune.default()
    gpu = tuner.gpu_name(torch.device(device))
    todo = {}
    for r in requests:
        for p in precisions:
            todo.setdefault(autotune.key(gpu, p, r.ns, r.cells), (r, p))
    n = 0
    for k, (r, p) in todo.items():
        if k in tuner.table:
            continue
        dc = DeviceCase(builder(r, device), device, precision=p, tile="auto")
        del dc
        n += 1
    torch.cuda.empty_cache()
    return n


def fifo(requests: list[SolveRequest], device="cuda", precision: int = 0,
         keep_results: bool = False, builder=build_request_case, tile="auto",
         fused: bool = True) -> dict:
    """The baseline: one case at a time in arrival order (plain stage launches, no batching,
    no graphs), same arrival times, same GPU, same report.  fused=False runs each stage as the
    reference's own launch sequence of 1:1 kernels (the literal drop-in; FP64 only)."""
    dev = torch.device(device)
    main = torch.cuda.current_stream(dev)
    t0 = time.perf_counter()
    now = lambda: time.perf_counter() - t0  # noqa: E731
    records, step_ms, busy = {}, [], 0.0
    results = {}
    st = {"build_s": 0.0, "download_s": 0.0, "capture_s": 0.0, "rebuilds": 0, "captures": 0}
    for r in sorted(requests, key=lambda r: r.arrival):
        wait = r.arrival - now()
        if wait > 0:
            time.sleep(wait)
        rec = RequestRecord(r.rid, "", r.cells, r.steps, resident_bytes(r, precision), r.arrival)
        records[r.rid] = rec
        rec.admitted = now()
        tb = time.perf_counter()
        case = builder(r, dev)
        dc = DeviceCase(case, dev, precision=precision, tile=tile if fused else 3,
                        sequence_buffers=not fused)
        case.Q = case.rhoi = None
        case.metrics = {}
        rec.name = case.name
        st["build_s"] += time.perf_counter() - tb
        evs = []
        rec.first_step = now()
        for _ in range(r.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(main)
            dc.step(fused)
            e1.record(main)
            evs.append((e0, e1))
        main.synchronize()
        td = time.perf_counter()
        for e0, e1 in evs:
            ms = e0.elapsed_time(e1)
            rec.step_ms.append(ms)
            step_ms.append(ms)
            busy += ms
        Q, rh = dc.primitives()
        rec.finite = bool(np.isfinite(Q).all() and np.isfinite(rh).all())
        if keep_results:
            results[r.rid] = (Q, rh)
        rec.finished = now()
        st["download_s"] += time.perf_counter() - td
        del dc
    st.update(busy_ms=busy, peak_active=1,
              peak_bytes=max((x.bytes for x in records.values()), default=0))
    rep = _report(records, step_ms, st)
    if keep_results:
        rep["results"] = results
    return rep


# ------------------------------------------------------------------------------- replicas
def route(requests: list[SolveRequest], n_replicas: int, cost=None) -> list[list[SolveRequest]]:
    """Assigns each request, in arrival order, to the replica (GPU) with the least work assigned
    so far (cost: cell-stages by default; ties to the lowest index).  Deterministic; every
    request goes to exactly one replica and keeps its arrival order there."""
    cost = cost or (lambda r: r.cell_stages)
    loads = [0.0] * n_replicas
    out: list[list[SolveRequest]] = [[] for _ in range(n_replicas)]
    for r in sorted(requests, key=lambda r: r.arrival):
        k = min(range(n_replicas), key=lambda i: (loads[i], i))
        out[k].append(r)
        loads[k] += cost(r)
    return out


class MultiServer:
    """One Server per GPU; replicas share nothing (no data-path collective), each runs its own
    stream of arrivals in its own host thread.  Requests are assigned by `route` before the
    replicas start: an online rule (a request's replica depends only on the requests that
    arrived before it, never on later ones), so it is the assignment a router that sees each
    request at its arrival would make, but it does not look at how far each replica has got."""

    def __init__(self, devices, **server_kwargs):
        self.servers = [Server(d, **server_kwargs) for d in devices]

    def run(self, requests: list[SolveRequest]) -> dict:
        parts = route(requests, len(self.servers))
        reports: list = [None] * len(self.servers)

        def work(i):
            with torch.cuda.device(self.servers[i].device):
                reports[i] = self.servers[i].run(parts[i]) if parts[i] else None

        with ThreadPoolExecutor(max_workers=len(self.servers)) as pool:
            for f in [pool.submit(work, i) for i in range(len(self.servers))]:
                f.result()
        done = [r for r in reports if r]
        cs = sum(r["cell_stages"] for r in done)
        first = min((p["arrival"] for r in done for p in r["per_request"]), default=0.0)
        last = max((p["finished"] for r in done for p in r["per_request"]
                    if not math.isnan(p["finished"])), default=first)
        return {"replicas": len(self.servers), "requests": len(requests),
                "completed": sum(r["completed"] for r in done), "cell_stages": cs,
                "makespan_s": last - first,
                "mcell_stage_per_s": cs / (last - first) / 1e6 if last > first else None,
                "per_replica": [{k: v for k, v in r.items() if k != "per_request"} if r else None
                                for r in reports]}
