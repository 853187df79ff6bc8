"""ctypes view of the C ABI in include/flame3d_b200.h and the loader of libflame3d_b200.so.

The structures here are field-for-field copies of the C structs; the function table gives every
exported entry point its argument types so a wrong call fails in Python, not on the device.
"""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libflame3d_b200.so"
HEADER = HERE.parent / "include" / "flame3d_b200.h"

FLAME_NG = 4
FLAME_MAX_NS = 16

ERRORS = {0: "FLAME_OK", 1: "FLAME_EINVAL", 2: "FLAME_ELAUNCH", 3: "FLAME_ETIMEOUT",
          4: "FLAME_ENONFINITE", 5: "FLAME_EUNSUPPORTED"}


class FlameError(RuntimeError):
    """A libflame3d_b200 call returned a non-zero status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"{ERRORS.get(code, code)}: {message}")
        self.code = code


class FlameGrid(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("ng", C.c_int32),
                ("ns", C.c_int32), ("periodic", C.c_int32)]


class FlameThermo(C.Structure):
    _fields_ = [("Ru", C.c_double), ("min_temp", C.c_double), ("max_temp", C.c_double),
                ("ns", C.c_int32), ("pad", C.c_int32),
                ("mw", C.c_double * FLAME_MAX_NS), ("coeffs_sep", C.c_double * FLAME_MAX_NS),
                ("coeffs_lo", C.c_double * (7 * FLAME_MAX_NS)),
                ("coeffs_hi", C.c_double * (7 * FLAME_MAX_NS))]


class FlameTransport(C.Structure):
    _fields_ = [("law", C.c_int32), ("pad", C.c_int32), ("mu_ref", C.c_double),
                ("T_ref", C.c_double), ("exponent", C.c_double), ("Pr", C.c_double),
                ("lambda_ref", C.c_double), ("D_ref", C.c_double), ("poly", C.c_void_p)]


METRIC_NAMES = ("dxidx", "dxidy", "dxidz", "detadx", "detady", "detadz",
                "dzetadx", "dzetady", "dzetadz", "J")


class FlameInflow(C.Structure):
    _fields_ = [("P", C.c_double), ("T", C.c_double), ("u", C.c_double), ("v", C.c_double),
                ("w", C.c_double), ("Y", C.c_double * FLAME_MAX_NS)]


class FlameReactions(C.Structure):
    _fields_ = [("nreacs", C.c_int32), ("pad", C.c_int32), ("atm", C.c_double),
                ("reaction_type", C.c_void_p), ("sgm", C.c_void_p), ("vf", C.c_void_p),
                ("vr", C.c_void_p), ("Arr", C.c_void_p), ("ef", C.c_void_p), ("loP", C.c_void_p),
                ("Troe", C.c_void_p)]


class FlameMetrics(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in METRIC_NAMES]

    def args(self) -> tuple:
        """The ten pointers in the reference's argument order (dξdx … dζdz, J), for the entry
        points that take them as separate arguments."""
        return tuple(getattr(self, n) for n in METRIC_NAMES)


class FlameStageBuffers(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("U", "Un", "Q_in", "Q_out", "rhoi_in", "rhoi_out",
                                          "rhon", "trans_in", "trans_out", "scratch",
                                          "metrics_lo")]


class FlameCaseDesc(C.Structure):
    _fields_ = [("grid", FlameGrid), ("dt", C.c_double), ("buf", FlameStageBuffers),
                ("metrics", FlameMetrics), ("thermo", FlameThermo),
                ("transport", FlameTransport)]


P = C.c_void_p
G = C.POINTER(FlameGrid)
S = C.c_void_p  # cudaStream_t
M = C.POINTER(FlameMetrics)
TH = C.POINTER(FlameThermo)
TR = C.POINTER(FlameTransport)
I = C.c_int
D = C.c_double
MET10 = [P] * 10  # the nine metric cofactors and J as separate arrays (viscous.jl:1, 430)

SIGNATURES = {
    "flame_shockSensor": [G, S, P, P],
    "flame_fluxSplit": [G, S, P, P, P, P, P, P, P],
    "flame_split": [G, S, P, P, P, P, P, P, P, P],
    "flame_WENO_x": [G, S, P, P, P, P, I, P],
    "flame_WENO_y": [G, S, P, P, P, P, I, P],
    "flame_WENO_z": [G, S, P, P, P, P, I, P],
    "flame_viscousFlux_x": [G, S, P, P, *MET10, P, P, P, P],
    "flame_viscousFlux_y": [G, S, P, P, *MET10, P, P, P, P],
    "flame_viscousFlux_z": [G, S, P, P, *MET10, P, P, P, P],
    "flame_specViscousFlux_x": [G, S, P, P, P, *MET10, P, P, TH, P],
    "flame_specViscousFlux_y": [G, S, P, P, P, *MET10, P, P, TH, P],
    "flame_specViscousFlux_z": [G, S, P, P, P, *MET10, P, P, TH, P],
    "flame_div": [G, S, P, P, P, P, P, P, P, D, P, P],
    "flame_divSpecs": [G, S, P, P, P, P, P, P, P, D, P, P],
    "flame_linComb": [G, S, P, P, I, D, D, P],
    "flame_c2Prim": [G, S, P, P, P, TH, P],
    "flame_prim2c": [G, S, P, P],
    "flame_mixture": [G, S, P, P, P, P, P, P, TH, TR, P],
    "flame_fill_periodic": [G, S, P, I],
    "flame_fill_x": [G, S, P, P, P, P, TH, C.POINTER(FlameInflow), I, I],
    "flame_fill_y": [G, S, P, P],
    "flame_fill_z": [G, S, P, P, P, P, TH, C.POINTER(FlameInflow)],
    "flame_fill_y_s": [G, S, P],
    "flame_fill_z_s": [G, S, P],
    "flame_fillGhost": [G, S, P, P, P, P, TH, C.POINTER(FlameInflow), I, I],
    "flame_fillSpec": [G, S, P],
    "flame_fillIB": [G, S, P, P, P, P, P, P, P, P, P, TH, D],
    "flame_cfl_max": [G, S, P, M, P],
    "flame_check_finite": [G, S, P, I, P],
    "flame_eval_gpu": [G, S, P, P, P, D, TH, C.POINTER(FlameReactions), P, D],
    "flame_eval_gpu_stiff": [G, S, P, P, P, D, TH, C.POINTER(FlameReactions), P, D, I],
    "flame_flowAdvance": [G, S, *[P] * 10, *MET10, D, P, P, P, P, P, P, P],
    "flame_specAdvance": [G, S, *[P] * 11, *MET10, D, P, P, P, P, P, TH, P],
    "flame_rk_stage": [G, S, I, D, C.POINTER(FlameStageBuffers), M, TH, TR, I],
    "flame_rk_stage_tiled": [G, S, I, D, C.POINTER(FlameStageBuffers), M, TH, TR, I, I],
    "flame_rk_stage_noalloc": [G, S, I, D, C.POINTER(FlameStageBuffers), M, TH, TR, I],
    "flame_transport": [G, S, P, P, P, TH, TR, I],
    "flame_transport_boundary": [G, S, P, P, P, TH, TR, I],
    "flame_stage_scratch_bytes": [G, I],
    "flame_batch_workspace_bytes": [C.POINTER(FlameCaseDesc), I, I],
    "flame_batch_create": [C.POINTER(C.c_void_p), C.POINTER(FlameCaseDesc), I, I, P, C.c_size_t,
                           S],
    "flame_batch_stage": [P, S, I, I],
    "flame_batch_status": [P, S],
    "flame_batch_test_stall": [P, I],
    "flame_batch_destroy": [P],
    "flame_last_error": [C.c_char_p, C.c_size_t],
    "flame_version": [],
}


def header_symbols(path: Path = HEADER) -> list[str]:
    """Every `flame_*` function the public header declares."""
    text = path.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(?:int|size_t)\s+(flame_\w+)\s*\(", text)))


_LIB: C.CDLL | None = None


def load_library(path: Path = LIB_PATH) -> C.CDLL:
    """Loads the in-tree library (built by build.py); raises if it is missing."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not path.exists():
        raise FlameError(1, f"{path} is missing: build it with `python {HERE/'build.py'}`")
    lib = C.CDLL(str(path))
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = C.c_size_t if name.endswith("_bytes") else C.c_int
    _LIB = lib
    return lib


def last_error(lib: C.CDLL) -> str:
    buf = C.create_string_buffer(512)
    lib.flame_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(lib: C.CDLL, rc: int) -> None:
    if rc != 0:
        raise FlameError(rc, last_error(lib))
