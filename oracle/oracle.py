"""Python binding of the oracle (liboracle.so) — TEST INFRASTRUCTURE ONLY.

The oracle is the CPU FP64 restatement of the reference hot path (flame_oracle.cpp).  Only the
tests, __graft_entry__.smoke() and bench.py's CPU baseline / reference arm use it, and only as
the checker or the timed CPU baseline; the product library never calls it.
"""
from __future__ import annotations

import ctypes as C
import importlib.util
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
LIB = HERE / "liboracle.so"
LIB_FMA = HERE / "liboracle_fma.so"


def _pkg():
    if "flame3d_b200" in sys.modules:
        return sys.modules["flame3d_b200"]
    root = ROOT / "flame3d.jl_b200"
    spec = importlib.util.spec_from_file_location("flame3d_b200", root / "__init__.py",
                                                  submodule_search_locations=[str(root)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["flame3d_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


abi = _pkg().abi

P = C.c_void_p
G = C.POINTER(abi.FlameGrid)
M = C.POINTER(abi.FlameMetrics)
TH = C.POINTER(abi.FlameThermo)
TR = C.POINTER(abi.FlameTransport)
D = C.c_double
I = C.c_int

SIGS = {
    "oracle_shockSensor": [G, P, P],
    "oracle_fluxSplit": [G, P, P, P, P, P, P, P],
    "oracle_split": [G, P, P, P, P, P, P, P, P],
    "oracle_WENO": [G, I, P, P, P, P, I, P],
    "oracle_viscousFlux": [G, I, P, P, M, P, P, P, P],
    "oracle_specViscousFlux": [G, I, P, P, P, M, P, P, TH, P],
    "oracle_div": [G, P, P, P, P, P, P, P, D, P, P],
    "oracle_divSpecs": [G, P, P, P, P, P, P, P, D, P, P],
    "oracle_linComb": [G, P, P, I, D, D, P],
    "oracle_c2Prim": [G, P, P, P, TH, P],
    "oracle_prim2c": [G, P, P],
    "oracle_mixture": [G, P, P, P, P, P, P, TH, TR, P],
    "oracle_fill_periodic": [G, P, I],
    "oracle_fill_x": [G, P, P, P, P, TH, C.POINTER(abi.FlameInflow), I, I],
    "oracle_fill_y": [G, P, P, P],
    "oracle_fill_z": [G, P, P, P, P, TH, C.POINTER(abi.FlameInflow)],
    "oracle_fill_z_s": [G, P],
    "oracle_fill_ib": [G, P, P, P, P, P, P, P, P, P, TH, D],
    "oracle_mixture_properties": [D, D, P, TH, P, I, P, P, P],
    "oracle_production_rate": [P, P, P, D, TH, C.POINTER(abi.FlameReactions), I],
    "oracle_solve": [P, P, P, I],
    "oracle_eval_chem": [G, I, P, P, P, D, TH, C.POINTER(abi.FlameReactions), P, D, I],
    "oracle_rk_stage_seq": [G, I, D, P, P, P, P, P, M, TH, TR],
    "oracle_h_specs": [P, D, TH, I],
    "oracle_up7": [P],
}
RESTYPES = {"oracle_GetT": (D, [D, P, TH, I]), "oracle_InternalEnergy": (D, [D, P, TH, I]),
            "oracle_CP": (D, [D, P, TH, I]), "oracle_num_threads": (C.c_int, []),
            "oracle_cfl_max": (D, [G, P, M])}

_cache: dict[str, C.CDLL] = {}


def build() -> None:
    """Compiles the oracle with its Makefile (g++, no GPU needed)."""
    r = subprocess.run(["make", "-s", "-C", str(HERE)], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")


def load(fma: bool = False) -> C.CDLL:
    path = LIB_FMA if fma else LIB
    key = str(path)
    if key in _cache:
        return _cache[key]
    if not path.exists():
        build()
    lib = C.CDLL(key)
    for n, a in SIGS.items():
        f = getattr(lib, n)
        f.argtypes, f.restype = a, None
    for n, (r, a) in RESTYPES.items():
        f = getattr(lib, n)
        f.argtypes, f.restype = a, r
    _cache[key] = lib
    return lib


def ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"] and a.dtype == np.float64
    return a.ctypes.data_as(C.c_void_p)


def metrics_struct(metrics: dict) -> "abi.FlameMetrics":
    return abi.FlameMetrics(**{k: metrics[k].ctypes.data for k in abi.METRIC_NAMES})


class OracleCase:
    """A case advanced by the oracle's restatement of solver.jl:298-326 (host arrays)."""

    def __init__(self, case, fma: bool = False):
        self.lib = load(fma)
        self.case = case
        self.grid = case.grid()
        self.th = case.thermo.to_c()
        self.tr = case.transport.to_c()
        self.metrics = {k: np.ascontiguousarray(v) for k, v in case.metrics.items()}
        self.cm = metrics_struct(self.metrics)
        self.Q = case.Q.copy()
        self.rhoi = case.rhoi.copy()
        self.U = np.empty((5,) + self.Q.shape[1:])
        self.lib.oracle_prim2c(C.byref(self.grid), ptr(self.U), ptr(self.Q))
        self.Un = np.empty_like(self.U)
        self.rhon = np.empty_like(self.rhoi)
        self.dt = case.dt
        # not periodic: the reference's fills after prim2c and after every stage
        # (solver.jl:192-200, 321-325); the stage's periodic fill then does nothing
        self.inflow = None
        if case.periodic != 7:
            self.inflow = getattr(case, "inflow", None)
            self.Yi = np.zeros_like(self.rhoi)
            self.fill()

    def fill(self) -> None:
        """fillGhost (fill_x, fill_y, fill_z) and fillSpec (fill_y_s, fill_z_s),
        boundary.jl:180-191, on rank 0 of 1."""
        g, th, P = C.byref(self.grid), C.byref(self.th), ptr
        self.lib.oracle_fill_x(g, P(self.Q), P(self.U), P(self.rhoi), P(self.Yi), th,
                               C.byref(self.inflow), 0, 1)
        self.lib.oracle_fill_y(g, P(self.Q), P(self.U), None)
        self.lib.oracle_fill_z(g, P(self.Q), P(self.U), P(self.rhoi), P(self.Yi), th,
                               C.byref(self.inflow))
        self.lib.oracle_fill_y(g, None, None, P(self.rhoi))
        self.lib.oracle_fill_z_s(g, P(self.rhoi))

    def stage(self, s: int) -> None:
        self.lib.oracle_rk_stage_seq(C.byref(self.grid), s, self.dt, ptr(self.U), ptr(self.Un),
                                     ptr(self.Q), ptr(self.rhoi), ptr(self.rhon),
                                     C.byref(self.cm), C.byref(self.th), C.byref(self.tr))
        if self.inflow is not None:
            self.fill()

    def step(self) -> None:
        for s in (1, 2, 3):
            self.stage(s)


def rel_l2(x: np.ndarray, ref: np.ndarray) -> float:
    """‖x − ref‖₂ / ‖ref‖₂ (0 when both vanish)."""
    d = np.linalg.norm((x - ref).ravel())
    n = np.linalg.norm(ref.ravel())
    return float(d / n) if n > 0 else float(d)


def interior(a: np.ndarray, ng: int = 4) -> np.ndarray:
    return a[..., ng:-ng, ng:-ng, ng:-ng]
