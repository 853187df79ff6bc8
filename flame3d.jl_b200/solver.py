"""Host-side mirror of solver.jl's stage loop over the libflame3d_b200 C ABI.

`DeviceCase` keeps one case's state and metrics resident on a GPU (torch tensors are only the
allocator and the stream; every computation is a call into the sm_100a library):

  * `stage_sequence(s)` issues the reference's own launch sequence for one RK3 stage
    (solver.jl:298-326: mixture, shockSensor, specAdvance, flowAdvance, linComb, c2Prim and the
    ghost fill) through the 1:1 entry points;
  * `stage_fused(s)` is the same stage as one `flame_rk_stage` launch.

Both take the primitive state Q, rho_i (ghosts filled) to the next stage's Q, rho_i.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import abi
from .abi import FlameMetrics, FlameStageBuffers, METRIC_NAMES
from .cases import Case

RK3 = {2: (0.25, 0.75), 3: (2.0 / 3.0, 1.0 / 3.0)}


def _p(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


class DeviceCase:
    """One case resident on one GPU."""

    def __init__(self, case: Case, device: str | torch.device = "cuda", precision: int = 0,
                 sequence_buffers: bool = False, tile: int | None = None):
        self.lib = abi.load_library()
        self.case = case
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise abi.FlameError(1, "DeviceCase needs a CUDA device; there is no CPU path")
        self.precision = precision
        self.grid = case.grid()
        self.thermo = case.thermo.to_c()
        self.poly = None  # law 2: the transport fits, on the device
        if case.transport.law == 2:
            self.poly = torch.as_tensor(case.transport.poly, dtype=torch.float64).to(self.device)
            self.transport = case.transport.to_c(self.poly.data_ptr())
        else:
            self.transport = case.transport.to_c()
        self.dt = case.dt
        dev = self.device
        f64 = dict(dtype=torch.float64, device=dev)
        qdt = torch.float64 if precision == 0 else torch.float32

        def up(a, dtype=torch.float64):
            if isinstance(a, torch.Tensor):  # built on the device: adopted when dtype matches
                return a.to(device=dev, dtype=dtype).contiguous()
            return torch.from_numpy(np.ascontiguousarray(a)).to(device=dev, dtype=dtype)

        self.metrics = {k: up(case.metrics[k]) for k in METRIC_NAMES}
        self.cmetrics = FlameMetrics(**{k: v.data_ptr() for k, v in self.metrics.items()})
        # mixed precision: the metrics rounded to FP32 once (FlameStageBuffers.metrics_lo)
        self.metrics_lo = (torch.stack([self.metrics[k] for k in METRIC_NAMES]).float()
                           .contiguous() if precision == 1 else None)
        shp = case.Q.shape[1:]
        ns = case.ns
        self.Q = [up(case.Q, qdt), torch.empty((7,) + shp, dtype=qdt, device=dev)]
        self.rhoi = [up(case.rhoi), torch.empty((ns,) + shp, **f64)]
        self.Q[1].copy_(self.Q[0])
        self.rhoi[1].copy_(self.rhoi[0])
        self.cur = 0
        self.U = torch.empty((5,) + shp, **f64)
        self.Un = torch.empty((5,) + shp, **f64)
        self.rhon = torch.empty((ns,) + shp, **f64)
        # μ, λ, D of the state, recomputed by every fused stage for the next one; with the
        # mixture-averaged law (law 2) one D per species: μ, λ, D_0 .. D_{ns-1}
        nt = 2 + ns if case.transport.law == 2 else 3
        self.T = [torch.empty((nt,) + shp, dtype=qdt, device=dev) for _ in range(2)]
        if precision == 0:
            self._call("flame_prim2c", _p(self.U), _p(self.Q[0]))
        elif isinstance(case.Q, torch.Tensor):  # U from the FP64 primitives, before rounding
            self._call("flame_prim2c", _p(self.U), _p(up(case.Q)))
        else:
            self.U.copy_(torch.from_numpy(case.U()).to(dev))
        self.scratch = None
        self.seq = None
        # the reference's own boundary conditions (not periodic): inflow / zero-gradient fills
        # after every stage, as solver.jl:321-325 runs them after c2Prim
        self.Yi = None
        self.inflow = None
        if case.periodic != 7:
            if case.periodic != 0 or precision != 0:
                raise abi.FlameError(5, "DeviceCase runs the reference's fills on grids periodic "
                                        "on no axis, in FP64 (the fill kernels are FP64)")
            from .cases import reference_inflow
            self.inflow = case.inflow if case.inflow is not None else reference_inflow(ns)
            self.Yi = torch.zeros((ns,) + shp, **f64)
            self._fill(0)  # solver.jl:192-200: prim2c, then fillGhost and fillSpec
        self._transport()
        # tile: a configuration of flame_rk_stage_tiled, "auto" for the autotuner's choice, or
        # None for the pencil sweeps (configuration 3; with law 2 the library runs the pencil
        # configurations as 6)
        self.set_tile(3 if tile is None or tile == "auto" else tile)
        if tile == "auto":
            from . import autotune
            self.set_tile(autotune.default().choose(self))
        if sequence_buffers:
            self._alloc_sequence()

    def _fill(self, cur: int) -> None:
        """The reference's ghost fills of state `cur` (boundary.jl:180-191): fillGhost on Q, U,
        rho_i, then fillSpec on rho_i (one GPU: x-slab rank 0 of 1)."""
        Q, r = self.Q[cur], self.rhoi[cur]
        self._call("flame_fillGhost", _p(Q), _p(self.U), _p(r), _p(self.Yi), C.byref(self.thermo),
                   C.byref(self.inflow), 0, 1)
        self._call("flame_fillSpec", _p(r))

    def nonfinite_launch(self) -> torch.Tensor:
        """Queues flame_check_finite over U (solver.jl:388-391) and returns the device counter
        it writes; read it after the stream has passed (`int(counter.item())`)."""
        if getattr(self, "_nf", None) is None:
            self._nf = torch.zeros(1, dtype=torch.int32, device=self.device)
        self._call("flame_check_finite", _p(self.U), 5, _p(self._nf))
        return self._nf

    def check_finite(self) -> None:
        """The reference's NaN check: raises FLAME_ENONFINITE when U holds NaN or inf."""
        n = int(self.nonfinite_launch().item())
        if n:
            raise abi.FlameError(4, f"{self.case.name}: {n} non-finite conserved values")

    def restore_conserved(self, q64: torch.Tensor) -> None:
        """After the primitive state was replaced (a restart): U from the FP64 primitives
        (prim2c, utils.jl:71-92) and the transport of the state for the fused stage."""
        self._call("flame_prim2c", _p(self.U), _p(q64.contiguous()))
        self._transport()

    def set_tile(self, tile: int) -> None:
        """Switches the fused stage's configuration (the pencil ones need scratch)."""
        self.tile = int(tile)
        if self.tile in (3, 4, 5, 6):
            if self.scratch is None:
                nbytes = self.lib.flame_stage_scratch_bytes(C.byref(self.grid), self.precision)
                self.scratch = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        else:
            self.scratch = None

    def clone(self, tile: int | None = None) -> "DeviceCase":
        """A copy of the current state on the same device (metrics shared: no kernel writes
        them), optionally with another configuration."""
        c = DeviceCase.__new__(DeviceCase)
        for a in ("lib", "case", "device", "precision", "grid", "thermo", "transport", "dt",
                  "metrics", "cmetrics", "cur", "poly", "metrics_lo", "inflow"):
            setattr(c, a, getattr(self, a))
        c.Yi = None if self.Yi is None else self.Yi.clone()
        c.Q = [q.clone() for q in self.Q]
        c.rhoi = [r.clone() for r in self.rhoi]
        c.T = [t.clone() for t in self.T]
        c.U, c.Un, c.rhon = self.U.clone(), self.Un.clone(), self.rhon.clone()
        c.scratch = None
        c.seq = None
        c.set_tile(self.tile if tile is None else tile)
        return c

    # ------------------------------------------------------------------ plumbing
    @property
    def stream(self) -> int:
        return torch.cuda.current_stream(self.device).cuda_stream

    def _call(self, name: str, *args):
        fn = getattr(self.lib, name)
        rc = fn(C.byref(self.grid), C.c_void_p(self.stream), *args)
        abi.check(self.lib, rc)

    def _transport(self) -> None:
        self._call("flame_transport", _p(self.Q[self.cur]), _p(self.rhoi[self.cur]),
                   _p(self.T[self.cur]), C.byref(self.thermo), C.byref(self.transport),
                   self.precision)

    def _alloc_sequence(self):
        c = self.case
        shp = c.Q.shape[1:]
        ns = c.ns
        nx, ny, nz = c.nx, c.ny, c.nz
        f64 = dict(dtype=torch.float64, device=self.device)
        fx, fy, fz = (nz, ny, nx + 1), (nz, ny + 1, nx), (nz + 1, ny, nx)
        z = torch.zeros
        self.seq = dict(
            Yi=z((ns,) + shp, **f64), lam=z(shp, **f64), mu=z(shp, **f64), D=z((ns,) + shp, **f64),
            phi=z(shp, **f64), Fp=z((5,) + shp, **f64), Fm=z((5,) + shp, **f64),
            Fpi=z((ns,) + shp, **f64), Fmi=z((ns,) + shp, **f64),
            Fx=z((5,) + fx, **f64), Fy=z((5,) + fy, **f64), Fz=z((5,) + fz, **f64),
            Fvx=z((4,) + fx, **f64), Fvy=z((4,) + fy, **f64), Fvz=z((4,) + fz, **f64),
            Fxi=z((ns,) + fx, **f64), Fyi=z((ns,) + fy, **f64), Fzi=z((ns,) + fz, **f64),
            Fdx=z((ns,) + fx, **f64), Fdy=z((ns,) + fy, **f64), Fdz=z((ns,) + fz, **f64),
            Fhx=z((3,) + fx, **f64), Fhy=z((3,) + fy, **f64), Fhz=z((3,) + fz, **f64),
        )

    # ------------------------------------------------------------------ stages
    def stage_sequence(self, stage: int) -> None:
        """solver.jl:298-326 through the 1:1 entry points (plain FP64 only)."""
        if self.precision != 0:
            raise abi.FlameError(5, "the launch sequence is FP64 only")
        if self.seq is None:
            self._alloc_sequence()
        w = self.seq
        Q, ri = self.Q[self.cur], self.rhoi[self.cur]
        g = C.byref
        dt = C.c_double(self.dt)
        if stage == 1:
            self.Un.copy_(self.U)
            self.rhon.copy_(ri)
        self._call("flame_mixture", _p(Q), _p(ri), _p(w["Yi"]), _p(w["lam"]), _p(w["mu"]),
                   _p(w["D"]), g(self.thermo), g(self.transport), None)
        self._call("flame_shockSensor", _p(w["phi"]), _p(Q))
        self._call("flame_specAdvance", _p(ri), _p(Q), _p(w["Yi"]), _p(w["Fpi"]), _p(w["Fmi"]),
                   _p(w["Fxi"]), _p(w["Fyi"]), _p(w["Fzi"]), _p(w["Fdx"]), _p(w["Fdy"]),
                   _p(w["Fdz"]), *self.cmetrics.args(), dt, _p(w["phi"]), _p(w["D"]), _p(w["Fhx"]),
                   _p(w["Fhy"]), _p(w["Fhz"]), g(self.thermo), None)
        self._call("flame_flowAdvance", _p(self.U), _p(Q), _p(w["Fp"]), _p(w["Fm"]), _p(w["Fx"]),
                   _p(w["Fy"]), _p(w["Fz"]), _p(w["Fvx"]), _p(w["Fvy"]), _p(w["Fvz"]),
                   *self.cmetrics.args(), dt, _p(w["phi"]), _p(w["lam"]), _p(w["mu"]), _p(w["Fhx"]),
                   _p(w["Fhy"]), _p(w["Fhz"]), None)
        if stage in RK3:
            a, b = RK3[stage]
            self._call("flame_linComb", _p(self.U), _p(self.Un), 5, a, b, None)
            self._call("flame_linComb", _p(ri), _p(self.rhon), self.case.ns, a, b, None)
        self._call("flame_c2Prim", _p(self.U), _p(Q), _p(ri), g(self.thermo), None)
        if self.inflow is not None:  # solver.jl:321-325
            self._fill(self.cur)
        else:
            self._call("flame_fill_periodic", _p(Q), 7)
            self._call("flame_fill_periodic", _p(ri), self.case.ns)

    def stage_fused(self, stage: int) -> None:
        """The same stage as one flame_rk_stage launch (ping-pong of Q and rho_i)."""
        i, o = self.cur, 1 - self.cur
        b = FlameStageBuffers(_p(self.U), _p(self.Un), _p(self.Q[i]), _p(self.Q[o]),
                              _p(self.rhoi[i]), _p(self.rhoi[o]), _p(self.rhon),
                              _p(self.T[i]), _p(self.T[o]), _p(self.scratch),
                              _p(self.metrics_lo))
        rc = self.lib.flame_rk_stage_tiled(C.byref(self.grid), C.c_void_p(self.stream), stage,
                                           self.dt, C.byref(b), C.byref(self.cmetrics),
                                           C.byref(self.thermo), C.byref(self.transport),
                                           self.precision, self.tile)
        abi.check(self.lib, rc)
        self.cur = o
        if self.inflow is not None:  # the ghosts of the result, then their transport
            self._fill(o)
            self._call("flame_transport_boundary", _p(self.Q[o]), _p(self.rhoi[o]), _p(self.T[o]),
                       C.byref(self.thermo), C.byref(self.transport), self.precision)

    @property
    def launched_config(self) -> int:
        """The configuration the library runs: the pencil configurations take the mixture-
        averaged law (law 2) as configuration 6."""
        if self.transport.law == 2 and self.tile in (3, 4, 5, 6):
            return 6
        return self.tile

    def launches_per_stage(self) -> int:
        """Kernels one fused stage launches: 4 for the pencil sweeps, one more with the
        separate finish (4, 6) and two more with split species sweeps (5, 6); 1 for a tile
        kernel."""
        return {3: 4, 4: 5, 5: 6, 6: 7}.get(self.launched_config, 1)

    def stage_kernels(self) -> str:
        t = self.launched_config
        if t in (3, 4, 5, 6):
            yz = ("k_pencil_staged<z> + k_pencil_staged<y>" if t < 5 else
                  "k_pencil_staged<z, flow> + k_pencil_staged<z, species> + "
                  "k_pencil_staged<y, flow> + k_pencil_staged<y, species>")
            fin = " + k_finish" if t in (4, 6) else ""
            return f"pencil::k_prep + {yz} + k_pencil_x{fin}"
        return "fused::k_stage<tile %d>" % t

    def step(self, fused: bool = True) -> None:
        torch.cuda.nvtx.range_push(f"step {self.case.name}")
        for s in (1, 2, 3):
            (self.stage_fused if fused else self.stage_sequence)(s)
        torch.cuda.nvtx.range_pop()

    def advance_from_host(self, Q_host: torch.Tensor, rhoi_host: torch.Tensor, nsteps: int,
                          Q_out: torch.Tensor, rhoi_out: torch.Tensor) -> None:
        """End-to-end call with host buffers: uploads the primitive state (ghosted Q, rho_i in
        FP64, ideally pinned), rebuilds U (prim2c, utils.jl:71-92), advances `nsteps` RK3 steps
        with the fused stage and downloads the resulting Q, rho_i (Q_out may be FP64 or the
        storage type).  Asynchronous on the current stream; synchronize before reading."""
        Q, r = self.Q[self.cur], self.rhoi[self.cur]
        if self.precision == 0:
            Q.copy_(Q_host, non_blocking=True)
            q64 = Q
        else:  # FP64 host state: U from the FP64 primitives, Q stored rounded to FP32
            if getattr(self, "_q64", None) is None:
                self._q64 = torch.empty(Q.shape, dtype=torch.float64, device=self.device)
            q64 = self._q64
            q64.copy_(Q_host, non_blocking=True)
            Q.copy_(q64)
        r.copy_(rhoi_host, non_blocking=True)
        self._call("flame_prim2c", _p(self.U), _p(q64))
        self._transport()
        for _ in range(nsteps):
            self.step()
        Q_out.copy_(self.Q[self.cur], non_blocking=True)
        rhoi_out.copy_(self.rhoi[self.cur], non_blocking=True)

    # ------------------------------------------------------------------ results
    def primitives(self) -> tuple[np.ndarray, np.ndarray]:
        return (self.Q[self.cur].double().cpu().numpy(), self.rhoi[self.cur].cpu().numpy())

    def conserved(self) -> np.ndarray:
        return self.U.cpu().numpy()
