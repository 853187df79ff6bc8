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
    # the fused stage refuses unknown precisions, stages and aliased buffers before launching
    g = f3d.FlameGrid(8, 8, 8, 4, 1, 3)
    b = f3d.FlameStageBuffers(1, 2, 3, 4, 5, 6, 7, 8, 9)
    m = f3d.FlameMetrics(*([1] * 10))
    th, tr = f3d.FlameThermo(), f3d.FlameTransport()
    rc = lib.flame_rk_stage(C.byref(g), None, 1, 1e-3, C.byref(b), C.byref(m), C.byref(th),
                            C.byref(tr), 2)
    assert rc == 1 and "precision" in f3d.abi.last_error(lib)
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


def test_signature_arity_matches_header(f3d):
    """Every declaration's parameter count equals the ctypes table's, so a call made from Python
    (or a Julia ccall written from the header) passes the arguments the library reads."""
    import re
    text = re.sub(r"/\*.*?\*/", "", f3d.abi.HEADER.read_text(), flags=re.S)
    decls = re.findall(r"\b(?:int|size_t)\s+(flame_\w+)\s*\(([^)]*)\)\s*;", text)
    assert decls
    for name, params in decls:
        n = 0 if params.strip() in ("", "void") else params.count(",") + 1
        assert n == len(f3d.abi.SIGNATURES[name]), (name, n, len(f3d.abi.SIGNATURES[name]))


def test_viscous_entry_points_take_the_reference_argument_list(f3d):
    """viscousFlux_x(Fv_x, Q, dξdx, dξdy, dξdz, dηdx, dηdy, dηdz, dζdx, dζdy, dζdz, J, λ, μ, Fh,
    tag) (viscous.jl:1) and specViscousFlux_x(Fd, Q, Yi, 9 metrics, J, D, Fh, thermo, tag)
    (viscous.jl:430): the metrics are ten separate arrays after (grid, stream)."""
    import re
    text = re.sub(r"/\*.*?\*/", "", f3d.abi.HEADER.read_text(), flags=re.S)
    metric = ["dxidx", "dxidy", "dxidz", "detadx", "detady", "detadz", "dzetadx", "dzetady",
              "dzetadz", "J"]
    want = {"flame_viscousFlux": ["Fv", "Q", *metric, "lambda", "mu", "Fh", "tag"],
            "flame_specViscousFlux": ["Fd", "Q", "Yi", *metric, "D", "Fh", "thermo", "tag"],
            "flame_flowAdvance": ["U", "Q", "Fp", "Fm", "Fx", "Fy", "Fz", "Fv_x", "Fv_y", "Fv_z",
                                  *metric, "dt", "phi", "lambda", "mu", "Fhx", "Fhy", "Fhz",
                                  "tag"],
            "flame_specAdvance": ["rhoi", "Q", "Yi", "Fp_i", "Fm_i", "Fx_i", "Fy_i", "Fz_i",
                                  "Fd_x", "Fd_y", "Fd_z", *metric, "dt", "phi", "D", "Fhx",
                                  "Fhy", "Fhz", "thermo", "tag"]}
    for stem, names in want.items():
        sfx = ["_x", "_y", "_z"] if "Flux" in stem else [""]
        for s in sfx:
            m = re.search(rf"\b{stem}{s}\s*\(([^)]*)\)", text)
            got = [re.findall(r"(\w+)\s*$", a.strip())[0] for a in m.group(1).split(",")][2:]
            assert got == names, (stem + s, got)


def test_size_queries_do_not_wrap(f3d, lib):
    """flame_stage_scratch_bytes saturates instead of wrapping, and the stage's size check
    rejects extents whose point count would overflow, before any CUDA call."""
    big = f3d.FlameGrid(2**31 - 9, 2**31 - 9, 2**31 - 9, 4, 1, 7)
    assert lib.flame_stage_scratch_bytes(C.byref(big), 0) == 2**64 - 1
    g = f3d.FlameGrid(64, 32, 32, 4, 1, 7)
    assert lib.flame_stage_scratch_bytes(C.byref(g), 0) == 72 * 40 * 40 * (2 * 6 * 8 + 2 * 8)
    b = f3d.FlameStageBuffers(1, 2, 3, 4, 5, 6, 7, 8, 9)
    m = f3d.FlameMetrics(*([1] * 10))
    for ext in ((1 << 21,) * 3, (2**31 - 9,) * 3, (100000, 100000, 4)):
        g = f3d.FlameGrid(*ext, 4, 1, 7)
        rc = lib.flame_rk_stage(C.byref(g), None, 1, 1e-3, C.byref(b), C.byref(m),
                                C.byref(f3d.FlameThermo()), C.byref(f3d.FlameTransport()), 0)
        assert rc == 1 and "2^31" in f3d.abi.last_error(lib), ext


def test_batch_planning_needs_no_gpu(f3d, lib):
    """flame_batch_workspace_bytes plans on the host: it takes transport laws 0, 1 and 2 (a
    law-2 case adds the species-sweep and finish phases to its chunk's work list, so its plan
    is larger than the same grid's under law 1), and refuses an unknown law, a grid that is
    not periodic, more than nine species and a NULL buffer (size 0)."""
    def desc(law=1, ns=2, periodic=7, n=16, buf=True):
        d = f3d.abi.FlameCaseDesc()
        d.grid = f3d.FlameGrid(n, n, n, 4, ns, periodic)
        d.dt = 1e-6
        d.buf = f3d.FlameStageBuffers(*([4096 if buf else 0] * 10))
        d.metrics = f3d.FlameMetrics(*([4096] * 10))
        d.transport.law = law
        return d

    def plan(*descs, precision=0):
        arr = (f3d.abi.FlameCaseDesc * len(descs))(*descs)
        return lib.flame_batch_workspace_bytes(arr, len(descs), precision)

    for precision in (0, 1):
        one, two = plan(desc(1), precision=precision), plan(desc(2), precision=precision)
        assert one > 0 and two > one, (precision, one, two)
        assert plan(desc(0), desc(2), desc(1, ns=5), precision=precision) > 0
    assert plan(desc(3)) == 0
    assert plan(desc(periodic=3)) == 0
    assert plan(desc(ns=10)) == 0
    assert plan(desc(buf=False)) == 0


def test_fused_stage_refuses_extents_below_the_ghost_width(f3d, lib):
    """The fused stage (and the no-alloc entry, which runs through it) needs every extent >= 4
    (a stencil reaches 3 cells past a face and the periodic images are single copies); smaller
    grids are refused before any CUDA call, on every configuration."""
    b = f3d.FlameStageBuffers(1, 2, 3, 4, 5, 6, 7, 8, 9)
    m = f3d.FlameMetrics(*([1] * 10))
    th, tr = f3d.FlameThermo(), f3d.FlameTransport()
    for ext in ((3, 8, 8), (8, 1, 8), (8, 8, 2)):
        g = f3d.FlameGrid(*ext, 4, 1, 7)
        for tile in range(7):
            rc = lib.flame_rk_stage_tiled(C.byref(g), None, 1, 1e-3, C.byref(b), C.byref(m),
                                          C.byref(th), C.byref(tr), 0, tile)
            assert rc == 1 and "extents must be >= 4" in f3d.abi.last_error(lib), (ext, tile)
        rc = lib.flame_rk_stage_noalloc(C.byref(g), None, 1, 1e-3, C.byref(b), C.byref(m),
                                        C.byref(th), C.byref(tr), 0)
        assert rc == 1 and "extents must be >= 4" in f3d.abi.last_error(lib), ext
