"""Autotuner: picks the stage configuration per (GPU, precision, species count, grid size).

Configurations (flame_rk_stage_tiled): 0, 1, 2 = one tile kernel per stage (16x8x8 with one or
two CTAs per SM, 8x8x8); 3 = prep + z, y, x pencil sweeps, the x sweep finishing the stage;
4 = the same sweeps with the finish in its own per-cell launch; 5, 6 = 3, 4 with each y / z
sweep split into a flow sweep and a species sweep.  The mixture-averaged transport (law 2) runs
on the pencil configurations only (as 6); the tile configurations refuse it and are skipped.  Which is fastest depends on
the species count (registers and shared memory per point grow with it), on the grid size (the
tile kernels launch once per stage, which matters for small grids) and on the precision.

The tuner times every candidate on a device-side clone of the case being set up (its own
fields, so the hybrid scheme's branch mix is the real one), a warm-up step and then `steps`
timed RK3 steps with CUDA events, and keeps the fastest.  Choices are cached in a JSON file
(FLAME3D_B200_CACHE, else ~/.cache/flame3d_b200/autotune.json) under a key naming the GPU,
precision, species count and the grid's size class (log2 of the cell count).
"""
from __future__ import annotations

import json
import math
import os
import threading
from pathlib import Path

CANDIDATES = (0, 1, 2, 3, 4, 5, 6)


def cache_path() -> Path:
    base = os.environ.get("FLAME3D_B200_CACHE")
    root = Path(base) if base else Path.home() / ".cache" / "flame3d_b200"
    return root / "autotune.json"


def size_class(cells: int) -> int:
    return int(round(math.log2(max(cells, 1))))


def key(gpu: str, precision: int, ns: int, cells: int, law: int = 1) -> str:
    """The cache key; the mixture-averaged transport (law 2) is tuned apart (its candidates and
    its costs differ)."""
    return f"{gpu}|p{precision}|ns{ns}|c{size_class(cells)}" + ("|law2" if law == 2 else "")


class Autotuner:
    """`choose(dc)` returns the configuration for DeviceCase `dc` (tuning on a miss).

    `measure(dc, tile) -> ms per step` may be replaced (tests use a fake timer)."""

    def __init__(self, path: Path | None = None, candidates=CANDIDATES, steps: int = 2,
                 measure=None):
        self.path = Path(path) if path else cache_path()
        self.candidates = tuple(candidates)
        self.steps = steps
        self.measure = measure or self._measure
        self._lock = threading.Lock()
        self.table: dict[str, dict] = self._load()

    def _load(self) -> dict:
        try:
            return json.loads(self.path.read_text())
        except (OSError, ValueError):
            return {}

    def _save(self) -> None:
        try:
            self.path.parent.mkdir(parents=True, exist_ok=True)
            merged = self._load()
            merged.update(self.table)
            tmp = self.path.with_suffix(".tmp")
            tmp.write_text(json.dumps(merged, indent=1, sort_keys=True))
            tmp.replace(self.path)
        except OSError:
            pass  # a read-only home: the choice still holds for this process

    @staticmethod
    def gpu_name(device) -> str:
        import torch
        p = torch.cuda.get_device_properties(device)
        return f"{p.name} sm{p.multi_processor_count}".replace(" ", "_")

    def choose(self, dc, gpu: str | None = None) -> int:
        gpu = gpu or self.gpu_name(dc.device)
        law = getattr(getattr(dc, "transport", None), "law", 1)
        k = key(gpu, dc.precision, dc.case.ns, dc.case.cells, law)
        with self._lock:
            hit = self.table.get(k)
            if hit is not None:
                return int(hit["tile"])
            times = {}
            for t in self.candidates:
                try:
                    times[t] = float(self.measure(dc, t))
                except Exception:  # a configuration that cannot run this case is skipped
                    continue
            if not times:
                return 3
            best = min(times, key=times.get)
            self.table[k] = {"tile": best, "ms_per_step": {str(t): v for t, v in times.items()}}
            self._save()
            return best

    def _measure(self, dc, tile: int) -> float:
        import torch
        c = dc.clone(tile=tile)
        try:
            c.step()  # warm-up: module load, shared-memory attributes, caches
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(self.steps):
                c.step()
            e1.record()
            e1.synchronize()
            return e0.elapsed_time(e1) / self.steps
        finally:
            del c


_DEFAULT: Autotuner | None = None


def default() -> Autotuner:
    global _DEFAULT
    if _DEFAULT is None:
        _DEFAULT = Autotuner()
    return _DEFAULT
