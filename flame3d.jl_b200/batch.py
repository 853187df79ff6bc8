"""Batched stages: many resident cases advanced together (flame_batch_* in the C ABI).

A `Batch` groups `DeviceCase`s that use the pencil configuration (each owns its state, metrics
and scratch).  One stage is a few persistent launches per species-count group, whatever the
number of cases; `capture()` records one RK3 step per in/out parity as CUDA graphs so the
serving loop replays a whole step with one graph launch.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import abi
from .abi import FlameCaseDesc, FlameStageBuffers


def _p(t):
    return None if t is None else t.data_ptr()


class Batch:
    def __init__(self, cases: list, device: str | torch.device = "cuda"):
        if not cases:
            raise abi.FlameError(1, "a batch needs at least one case")
        self.lib = abi.load_library()
        self.cases = list(cases)
        self.device = torch.device(device)
        prec = {dc.precision for dc in self.cases}
        if len(prec) != 1:
            raise abi.FlameError(1, "all cases of a batch share one precision")
        self.precision = prec.pop()
        for dc in self.cases:
            if dc.tile != 3 or dc.scratch is None:
                raise abi.FlameError(1, "batched cases use the pencil configuration (tile=3)")
        n = len(self.cases)
        descs = (FlameCaseDesc * n)()
        for k, dc in enumerate(self.cases):
            i, o = dc.cur, 1 - dc.cur
            d = descs[k]
            d.grid = dc.grid
            d.dt = dc.dt
            d.buf = FlameStageBuffers(_p(dc.U), _p(dc.Un), _p(dc.Q[i]), _p(dc.Q[o]),
                                      _p(dc.rhoi[i]), _p(dc.rhoi[o]), _p(dc.rhon),
                                      _p(dc.T[i]), _p(dc.T[o]), _p(dc.scratch))
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
        self.parity = 0
        self.graphs: dict[int, torch.cuda.CUDAGraph] = {}

    @property
    def stream(self) -> int:
        return torch.cuda.current_stream(self.device).cuda_stream

    @property
    def cells(self) -> int:
        return sum(dc.case.cells for dc in self.cases)

    def _launch(self, stage: int, parity: int) -> None:
        rc = self.lib.flame_batch_stage(self.handle, C.c_void_p(self.stream), stage, parity)
        abi.check(self.lib, rc)

    def _flip(self) -> None:
        self.parity ^= 1
        for dc in self.cases:
            dc.cur = 1 - dc.cur

    def stage(self, stage: int) -> None:
        self._launch(stage, self.parity)
        self._flip()

    def step(self) -> None:
        """One RK3 step of every case; replays the captured graph when there is one."""
        g = self.graphs.get(self.parity)
        if g is not None:
            g.replay()
            for _ in range(3):
                self._flip()
            return
        for s in (1, 2, 3):
            self.stage(s)

    def capture(self) -> None:
        """Records one RK3 step for each starting parity as a CUDA graph."""
        torch.cuda.synchronize(self.device)
        for par in (0, 1):
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, capture_error_mode="thread_local"):
                p = par
                for s in (1, 2, 3):
                    self._launch(s, p)
                    p ^= 1
            self.graphs[par] = g
        torch.cuda.synchronize(self.device)

    def close(self) -> None:
        self.graphs.clear()
        if self.handle:
            self.lib.flame_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
