"""Batched stages: many resident cases advanced together.

A `Batch` groups `DeviceCase`s that use the pencil configuration (each owns its state, metrics
and scratch).  Three modes:

* "persistent": flame_batch_* in the C ABI; one stage is two persistent launches per chunk
  of up to 20 cases of one species count and transport family (four for the mixture-averaged
  law 2), over a (case, block) work list of every phase of every case (device counters order a
  case's prep before its sweeps; `status()` reports a wait that ran out);
* "graph": every case's own launch chain (prep, z, y, x sweeps per stage) on one of several
  streams, forked and joined inside one CUDA graph, so the chains of small cases run side by
  side on the GPU and every kernel keeps its parameters in the constant bank;
* "hybrid": the cases of at most `small_cells` cells (configuration 3) in a persistent batch on
  a stream of their own, every other case in a graph-mode batch, both forked from the caller's
  stream and joined back in the same step (the persistent kernels are ahead of the stand-alone
  chains where a case is too small to fill the GPU between launches, behind on large cases).

`capture()` records one RK3 step per in/out parity as CUDA graphs, so the serving loop replays a
whole step of every case with one graph launch.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import abi
from .abi import FlameCaseDesc, FlameStageBuffers


def _p(t):
    return None if t is None else t.data_ptr()


SMALL_CELLS = 48 ** 3  # hybrid mode: cases up to this size run in the persistent part


class Batch:
    def __init__(self, cases: list, device: str | torch.device = "cuda", mode: str = "graph",
                 streams: int = 16, small_cells: int = SMALL_CELLS):
        if not cases:
            raise abi.FlameError(1, "a batch needs at least one case")
        self.lib = abi.load_library()
        self.cases = list(cases)
        self.device = torch.device(device)
        prec = {dc.precision for dc in self.cases}
        if len(prec) != 1:
            raise abi.FlameError(1, "all cases of a batch share one precision")
        self.precision = prec.pop()
        if mode == "persistent" and any(dc.tile != 3 or dc.scratch is None for dc in self.cases):
            raise abi.FlameError(1, "the persistent batch runs the pencil configuration (tile=3)")
        self.mode = mode
        self.parity = 0
        self.graphs: dict[int, torch.cuda.CUDAGraph] = {}
        self.handle = None
        if mode == "hybrid":
            small = [dc for dc in self.cases if dc.case.cells <= small_cells and dc.tile == 3
                     and dc.scratch is not None]
            rest = [dc for dc in self.cases if not any(dc is x for x in small)]
            self.parts = [Batch(small, self.device, "persistent")] if small else []
            if rest:
                self.parts.append(Batch(rest, self.device, "graph", streams))
            self.pstream = torch.cuda.Stream(self.device)
            return
        if mode == "graph":
            # largest cases first, dealt round-robin over the streams
            self.order = sorted(range(len(self.cases)), key=lambda k: -self.cases[k].case.cells)
            self.side = [torch.cuda.Stream(self.device) for _ in range(min(streams, len(cases)))]
            return
        if mode != "persistent":
            raise abi.FlameError(1, f"unknown batch mode {mode!r}")
        n = len(self.cases)
        descs = (FlameCaseDesc * n)()
        for k, dc in enumerate(self.cases):
            i, o = dc.cur, 1 - dc.cur
            d = descs[k]
            d.grid = dc.grid
            d.dt = dc.dt
            d.buf = FlameStageBuffers(_p(dc.U), _p(dc.Un), _p(dc.Q[i]), _p(dc.Q[o]),
                                      _p(dc.rhoi[i]), _p(dc.rhoi[o]), _p(dc.rhon),
                                      _p(dc.T[i]), _p(dc.T[o]), _p(dc.scratch),
                                      _p(dc.metrics_lo))
            d.metrics = dc.cmetrics
            d.thermo = dc.thermo
            d.transport = dc.transport
        self._descs = descs
        nbytes = self.lib.flame_batch_workspace_bytes(descs, n, self.precision)
        self.workspace = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=self.device)
        h = C.c_void_p()
        rc = self.lib.flame_batch_create(C.byref(h), descs, n, self.precision,
                                         _p(self.workspace), nbytes, C.c_void_p(self.stream))
        abi.check(self.lib, rc)
        self.handle = h

    @property
    def stream(self) -> int:
        return torch.cuda.current_stream(self.device).cuda_stream

    @property
    def cells(self) -> int:
        return sum(dc.case.cells for dc in self.cases)

    def _launch(self, stage: int, parity: int) -> None:
        rc = self.lib.flame_batch_stage(self.handle, C.c_void_p(self.stream), stage, parity)
        abi.check(self.lib, rc)

    def _hybrid_step(self, parity: int) -> None:
        """One RK3 step of both parts: the persistent part's three stages (from `parity`) on its
        own stream, the graph part's chains on theirs, all joined back to the current stream.
        Flips the graph part's cases (as DeviceCase.step does), not the persistent part's."""
        main = torch.cuda.current_stream(self.device)
        parts = list(self.parts)
        if parts and parts[0].mode == "persistent":
            pers = parts.pop(0)
            ev = torch.cuda.Event()
            ev.record(main)
            self.pstream.wait_event(ev)
            with torch.cuda.stream(self.pstream):
                p = parity
                for s in (1, 2, 3):
                    pers._launch(s, p)
                    p ^= 1
        for part in parts:  # the graph part forks from and joins back to `main` itself
            part._fork_step()
        main.wait_stream(self.pstream)

    def _hybrid_flip(self) -> None:
        """The bookkeeping of one step: the persistent part's three stage flips (its graph
        part's cases were flipped by their DeviceCase.step)."""
        for part in self.parts:
            if part.mode == "persistent":
                for _ in range(3):
                    part._flip()
            else:
                part.parity ^= 1
        self.parity ^= 1

    def _fork_step(self) -> None:
        """One RK3 step of every case, each case's chain on a side stream (flips every cur)."""
        main = torch.cuda.current_stream(self.device)
        ev = torch.cuda.Event()
        ev.record(main)
        for j, k in enumerate(self.order):
            st = self.side[j % len(self.side)]
            st.wait_event(ev)
            with torch.cuda.stream(st):
                self.cases[k].step()
        for st in self.side:
            main.wait_stream(st)

    def _flip(self) -> None:
        self.parity ^= 1
        for dc in self.cases:
            dc.cur = 1 - dc.cur

    def stage(self, stage: int) -> None:
        if self.mode == "hybrid":
            for part in self.parts:
                part.stage(stage)
            self.parity ^= 1
            return
        if self.mode == "graph":
            main = torch.cuda.current_stream(self.device)
            ev = torch.cuda.Event()
            ev.record(main)
            for j, k in enumerate(self.order):
                st = self.side[j % len(self.side)]
                st.wait_event(ev)
                with torch.cuda.stream(st):
                    self.cases[k].stage_fused(stage)  # flips the case's cur
            for st in self.side:
                main.wait_stream(st)
            self.parity ^= 1
            return
        self._launch(stage, self.parity)
        self._flip()

    def step(self) -> None:
        """One RK3 step of every case; replays the captured graph when there is one."""
        g = self.graphs.get(self.parity)
        if self.mode == "hybrid":
            if g is not None:
                g.replay()
                for part in self.parts:  # a replay flips nothing: the graph part's cases too
                    if part.mode == "graph":
                        for dc in part.cases:
                            dc.cur = 1 - dc.cur
            else:
                self._hybrid_step(self._persistent_parity())
            self._hybrid_flip()
            return
        if g is not None:
            g.replay()
            for _ in range(3):
                self._flip()
            return
        if self.mode == "graph":
            self._fork_step()  # DeviceCase.step flips each case's cur
            self.parity ^= 1
            return
        for s in (1, 2, 3):
            self.stage(s)

    def capture(self) -> None:
        """Records one RK3 step for each starting parity as a CUDA graph."""
        torch.cuda.synchronize(self.device)
        if self.mode == "hybrid":
            # one graph per starting parity of the whole batch; the persistent part's stage
            # parities are explicit arguments, the graph part's pointers are its cases' current
            # ones, flipped by the capture and flipped back by the second one
            start, pstart = self.parity, self._persistent_parity()
            for k, par in enumerate((start, start ^ 1)):
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, capture_error_mode="thread_local"):
                    self._hybrid_step(pstart ^ k)
                self.graphs[par] = g
            torch.cuda.synchronize(self.device)
            return
        if self.mode == "graph":
            start = self.parity
            for par in (start, start ^ 1):
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, capture_error_mode="thread_local"):
                    self._fork_step()  # records the pointers of this parity, flips every cur
                self.parity ^= 1
                self.graphs[par] = g
            # capturing launched nothing: both flips are undone, the state is unchanged
            torch.cuda.synchronize(self.device)
            return
        for par in (0, 1):
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, capture_error_mode="thread_local"):
                p = par
                for s in (1, 2, 3):
                    self._launch(s, p)
                    p ^= 1
            self.graphs[par] = g
        torch.cuda.synchronize(self.device)

    def _persistent_parity(self) -> int:
        return next((p.parity for p in self.parts if p.mode == "persistent"), 0)

    def status(self) -> None:
        """Raises FlameError(FLAME_ETIMEOUT) if a persistent stage's bounded wait ran out since
        the last call (synchronizes the stream); nothing to check in graph mode."""
        if self.mode == "hybrid":
            for part in self.parts:
                part.status()
            return
        if self.handle:
            abi.check(self.lib, self.lib.flame_batch_status(self.handle, C.c_void_p(self.stream)))

    def close(self) -> None:
        self.graphs.clear()
        for part in getattr(self, "parts", []):
            part.close()
        if self.handle:
            self.lib.flame_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
