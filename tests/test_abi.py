"""The C ABI library without a GPU: it builds, loads, exports every declared symbol, its structs
match the header byte for byte, and argument errors are reported before any CUDA call."""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def lib(f3d):
    import importlib
    build = importlib.import_module("flame3d_b200.build")
    build.build()
    return f3d.load_library()


def test_exports_every_header_symbol(f3d, lib):
    syms = f3d.header_symbols()
    assert len(syms) >= 27
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    # and the ctypes table covers the whole header
    assert set(syms) <= set(f3d.abi.SIGNATURES), set(syms) - set(f3d.abi.SIGNATURES)


def test_struct_layout_matches_header(f3d, tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(r'''
#include <stdio.h>
#include <stddef.h>
#include "flame3d_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu\n", sizeof(FlameGrid), sizeof(FlameThermo),
         sizeof(FlameTransport), sizeof(FlameMetrics), sizeof(FlameStageBuffers),
         offsetof(FlameThermo, coeffs_hi));
  return 0;
}''')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = list(map(int, subprocess.run([str(exe)], capture_output=True, text=True,
                                       check=True).stdout.split()))
    a = f3d.abi
    want = [C.sizeof(a.FlameGrid), C.sizeof(a.FlameThermo), C.sizeof(a.FlameTransport),
            C.sizeof(a.FlameMetrics), C.sizeof(a.FlameStageBuffers),
            a.FlameThermo.coeffs_hi.offset]
    assert got == want


def test_argument_errors_need_no_gpu(f3d, lib):
    g = f3d.FlameGrid(8, 8, 8, 3, 1, 7)  # ng must be 4
    rc = lib.flame_fluxSplit(C.byref(g), None, 1, 1, 1, 1, 1, 1, None)
    assert rc == 1 and "ng=3" in f3d.abi.last_error(lib)
    assert lib.flame_shockSensor(None, None, 1, 1) == 1
    g = f3d.FlameGrid(8, 8, 8, 4, 0, 7)
    assert lib.flame_split(C.byref(g), None, 1, 1, 1, 1, 1, 1, 1, None) == 1
    assert "ns=0" in f3d.abi.last_error(lib)
    # the fused stage refuses non-periodic grids and unknown precisions before launching
    g = f3d.FlameGrid(8, 8, 8, 4, 1, 3)
    b = f3d.FlameStageBuffers(1, 2, 3, 4, 5, 6, 7, 8, 9)
    m = f3d.FlameMetrics(*([1] * 10))
    th, tr = f3d.FlameThermo(), f3d.FlameTransport()
    rc = lib.flame_rk_stage(C.byref(g), None, 1, 1e-3, C.byref(b), C.byref(m), C.byref(th),
                            C.byref(tr), 0)
    assert rc == 5 and "periodic" in f3d.abi.last_error(lib)
    g = f3d.FlameGrid(8, 8, 8, 4, 1, 7)
    rc = lib.flame_rk_stage(C.byref(g), None, 4, 1e-3, C.byref(b), C.byref(m), C.byref(th),
                            C.byref(tr), 0)
    assert rc == 1 and "stage" in f3d.abi.last_error(lib)
    b2 = f3d.FlameStageBuffers(1, 2, 3, 3, 5, 6, 7, 8, 9)
    rc = lib.flame_rk_stage(C.byref(g), None, 1, 1e-3, C.byref(b2), C.byref(m), C.byref(th),
                            C.byref(tr), 0)
    assert rc == 1 and "differ" in f3d.abi.last_error(lib)
    assert lib.flame_version() >= 10000


def test_python_raises_flame_error(f3d, lib):
    with pytest.raises(f3d.FlameError) as e:
        f3d.abi.check(lib, lib.flame_prim2c(None, None, 1, 1))
    assert e.value.code == 1
