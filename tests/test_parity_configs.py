"""Parity with the oracle at the benchmark configurations' full sizes (solver.jl:297-326).

The other stage tests run grids of 12-32 cells per axis; these run the configurations the
benchmarks quote, so an indexing error that only shows on large grids (all indices inside the
fused kernels are 32-bit) cannot hide:

* Taylor-Green vortex 64^3, plain FP64 with the autotuned configuration: every field within
  1e-12 relative L2 of the oracle after stages 1, 2 and 3, and after 100 steps;
* the curvilinear Ma 1.5 jet 256x128x128, plain FP64: one full RK3 step, 1e-12 per stage;
* the mixing layer 192^3 with 9 species, plain FP64: one stage, 1e-12;
* Taylor-Green 64^3 in mixed precision after 1000 steps: rho, rho*u and rho*E within 1e-5 of
  the oracle's FP64 run (the FP64 path's own error after 1000 steps is printed beside it).

The oracle runs on all host cores; the whole module takes a few minutes, most of it the
oracle's 1000 Taylor-Green steps.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ["rho", "rhou", "rhov", "rhow", "E"]


def _rel(x, ref, scale=None):
    d = np.linalg.norm((x - ref).ravel())
    n = np.linalg.norm(ref.ravel()) if scale is None else scale
    return float(d / n) if n > 0 else float(d)


def _errors(dc, oc, oracle) -> dict:
    """Relative L2 per field over interior cells; momentum and velocity components against the
    norm of the whole vector field.  Ghost cells of the primitive state are compared too."""
    I = oracle.interior
    U = dc.conserved()
    Q, r = dc.primitives()
    mom = np.linalg.norm(I(oc.U[1:4]).ravel())
    vel = np.linalg.norm(I(oc.Q[1:4]).ravel())
    e = {f: _rel(I(U[n]), I(oc.U[n]), mom if 1 <= n <= 3 else None) for n, f in enumerate(FIELDS)}
    e["Q"] = max(_rel(I(Q[n]), I(oc.Q[n]), vel if 1 <= n <= 3 else None) for n in range(7))
    e["rhoi"] = max(_rel(I(r[n]), I(oc.rhoi[n])) for n in range(r.shape[0]))
    e["Q_ghosts"] = max(_rel(Q[n], oc.Q[n], vel if 1 <= n <= 3 else None) for n in range(7))
    return e


def _conserved(U, Uref, oracle) -> dict:
    """rho, the momentum vector field and rho*E, relative L2 over interior cells."""
    I = oracle.interior
    mom = np.linalg.norm(I(Uref[1:4]).ravel())
    return {"rho": _rel(I(U[0]), I(Uref[0])), "rhou": _rel(I(U[1:4]), I(Uref[1:4]), mom),
            "rhoE": _rel(I(U[4]), I(Uref[4]))}


@pytest.fixture(scope="module")
def tgv64_oracle(f3d, oracle):
    """The oracle's Taylor-Green 64^3 run: conserved state after 100 and after 1000 steps."""
    case = f3d.taylor_green(n=64)
    oc = oracle.OracleCase(case)
    snaps = {}
    for step in range(1, 1001):
        oc.step()
        if step in (100, 1000):
            snaps[step] = oc.U.copy()
    return case, snaps


def test_tgv64_fp64_stages(f3d, oracle, cuda_ok):
    case = f3d.taylor_green(n=64)
    dc = f3d.solver_module().DeviceCase(case, tile="auto")
    oc = oracle.OracleCase(case)
    for s in (1, 2, 3):
        dc.stage_fused(s)
        oc.stage(s)
        e = _errors(dc, oc, oracle)
        assert max(e.values()) <= 1e-12, (dc.launched_config, s, e)


def test_tgv64_fp64_100_steps(f3d, oracle, cuda_ok, tgv64_oracle):
    case, snaps = tgv64_oracle
    dc = f3d.solver_module().DeviceCase(case, tile="auto")
    for _ in range(100):
        dc.step()
    e = _conserved(dc.conserved(), snaps[100], oracle)
    print(f"TGV 64^3 FP64 (configuration {dc.launched_config}) after 100 steps: {e}")
    assert max(e.values()) <= 1e-12, e


@pytest.mark.parametrize("tile", ["auto", 3])
def test_tgv64_mixed_1000_steps(f3d, oracle, cuda_ok, tgv64_oracle, tile):
    case, snaps = tgv64_oracle
    S = f3d.solver_module()
    mixed = S.DeviceCase(case, precision=1, tile=tile)
    fp64 = S.DeviceCase(case, precision=0, tile=tile)
    for _ in range(1000):
        mixed.step()
        fp64.step()
    e = _conserved(mixed.conserved(), snaps[1000], oracle)
    e64 = _conserved(fp64.conserved(), snaps[1000], oracle)
    print(f"TGV 64^3 after 1000 steps against the oracle: mixed (configuration "
          f"{mixed.launched_config}) {e}; FP64 {e64}")
    assert np.isfinite(mixed.conserved()).all()
    assert max(e.values()) <= 1e-5, e
    assert max(e64.values()) <= 1e-11, e64


def test_jet256x128x128_fp64_one_step(f3d, oracle, cuda_ok):
    case = f3d.curvilinear_jet()
    dc = f3d.solver_module().DeviceCase(case, tile="auto")
    oc = oracle.OracleCase(case)
    for s in (1, 2, 3):
        dc.stage_fused(s)
        oc.stage(s)
        e = _errors(dc, oc, oracle)
        assert max(e.values()) <= 1e-12, (dc.launched_config, s, e)


def test_mix192_ns9_fp64_one_stage(f3d, oracle, cuda_ok):
    case = f3d.mixing_layer(n=192, ns=9)
    dc = f3d.solver_module().DeviceCase(case, tile="auto")
    oc = oracle.OracleCase(case)
    dc.stage_fused(1)
    oc.stage(1)
    e = _errors(dc, oc, oracle)
    assert max(e.values()) <= 1e-12, (dc.launched_config, e)
