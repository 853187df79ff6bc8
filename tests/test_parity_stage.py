"""Parity of whole RK3 stages and steps with the oracle's restatement of solver.jl:298-326.

* launch sequence (1:1 kernels, -fmad=false): agrees with the oracle to 1e-14 relative L2
  (only pow() in the transport law differs from libm);
* fused one-launch stage, plain FP64: ≤ 1e-12 relative L2 per field (the bound the fused
  path is held to);
* fused stage, mixed precision: ≤ 1e-5 relative L2 in ρ, ρu, ρE after several steps.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ["rho", "rhou", "rhov", "rhow", "E"]


def _cases(f3d):
    return {
        "tgv24": lambda: f3d.taylor_green(n=24),
        "rand_ns1": lambda: f3d.random_curvilinear(n=12, ns=1, seed=41),
        "rand_ns3": lambda: f3d.random_curvilinear(n=12, ns=3, seed=42),
        "mix_ns9": lambda: f3d.mixing_layer(n=16, ns=9),
        "jet": lambda: f3d.curvilinear_jet(nx=32, ny=16, nz=16, pressure_noise=0.02),
    }


def _rel(x, ref, scale=None):
    d = np.linalg.norm((x - ref).ravel())
    n = np.linalg.norm(ref.ravel()) if scale is None else scale
    return float(d / n) if n > 0 else float(d)


def _errors(dc, oc, oracle):
    """Relative L2 per field over interior cells.  A momentum or velocity component is measured
    against the norm of the whole vector field, so a component that starts at zero (w in the
    mixing layer) is not divided by its own round-off."""
    I = oracle.interior
    U = dc.conserved()
    Q, r = dc.primitives()
    mom = np.linalg.norm(I(oc.U[1:4]).ravel())
    vel = np.linalg.norm(I(oc.Q[1:4]).ravel())
    e = {}
    for n, f in enumerate(FIELDS):
        e[f] = _rel(I(U[n]), I(oc.U[n]), mom if 1 <= n <= 3 else None)
    e["Q"] = max(_rel(I(Q[n]), I(oc.Q[n]), vel if 1 <= n <= 3 else None) for n in range(7))
    e["rhoi"] = max(_rel(I(r[n]), I(oc.rhoi[n])) for n in range(r.shape[0]))
    # ghosts of the primitive state are filled identically
    e["Q_ghosts"] = max(_rel(Q[n], oc.Q[n], vel if 1 <= n <= 3 else None) for n in range(7))
    return e


@pytest.mark.parametrize("name", ["tgv24", "rand_ns1", "rand_ns3", "mix_ns9", "jet"])
def test_sequence_matches_oracle(f3d, oracle, cuda_ok, name):
    case = _cases(f3d)[name]()
    solver = f3d.solver_module()
    dc = solver.DeviceCase(case, sequence_buffers=True)
    oc = oracle.OracleCase(case)
    for s in (1, 2, 3):
        dc.stage_sequence(s)
        oc.stage(s)
    e = _errors(dc, oc, oracle)
    assert max(e.values()) <= 1e-14, e


TILES = [0, 1, 2, 3, 4, 5, 6]


@pytest.mark.parametrize("tile", TILES)
@pytest.mark.parametrize("name", ["tgv24", "rand_ns1", "rand_ns3", "mix_ns9", "jet"])
def test_fused_fp64_matches_oracle(f3d, oracle, cuda_ok, name, tile):
    case = _cases(f3d)[name]()
    dc = f3d.solver_module().DeviceCase(case, tile=tile)
    oc = oracle.OracleCase(case)
    for s in (1, 2, 3):
        dc.stage_fused(s)
        oc.stage(s)
        e = _errors(dc, oc, oracle)
        assert max(e.values()) <= 1e-12, (s, e)


@pytest.mark.parametrize("tile", [0, 3])
def test_fused_fp64_ten_steps_tgv(f3d, oracle, cuda_ok, tile):
    case = f3d.taylor_green(n=32)
    dc = f3d.solver_module().DeviceCase(case, tile=tile)
    oc = oracle.OracleCase(case)
    for _ in range(10):
        dc.step()
        oc.step()
    e = _errors(dc, oc, oracle)
    assert max(e.values()) <= 1e-12, e


@pytest.mark.parametrize("tile", [1, 3])
def test_fused_fp64_five_steps_jet_branches(f3d, oracle, cuda_ok, tile):
    """Curvilinear supersonic jet with pressure noise: all hybrid branches active."""
    case = f3d.curvilinear_jet(nx=32, ny=24, nz=16, pressure_noise=0.05)
    dc = f3d.solver_module().DeviceCase(case, tile=tile)
    oc = oracle.OracleCase(case)
    for _ in range(5):
        dc.step()
        oc.step()
    e = _errors(dc, oc, oracle)
    assert max(e.values()) <= 1e-12, e


@pytest.mark.parametrize("tile", [1, 3])
@pytest.mark.parametrize("name", ["tgv24", "rand_ns3", "mix_ns9"])
def test_fused_mixed_precision_error(f3d, oracle, cuda_ok, name, tile):
    case = _cases(f3d)[name]()
    dc = f3d.solver_module().DeviceCase(case, precision=1, tile=tile)
    oc = oracle.OracleCase(case)
    for _ in range(5):
        dc.step()
        oc.step()
    e = _errors(dc, oc, oracle)
    for f in ("rho", "rhou", "E"):
        assert e[f] <= 1e-5, (f, e)


@pytest.mark.parametrize("precision", [0, 1])
def test_split_finish_is_bit_identical(f3d, cuda_ok, precision):
    """Configuration 4 (finish in its own launch) rounds R + rhs once, like configuration 3."""
    S = f3d.solver_module()
    case = f3d.random_curvilinear(n=12, ns=3, seed=61)
    a = S.DeviceCase(case, precision=precision, tile=3)
    b = a.clone(tile=4)
    for _ in range(2):
        a.step()
        b.step()
    for x, y in zip(a.primitives() + (a.conserved(),), b.primitives() + (b.conserved(),)):
        assert np.array_equal(x, y)


def test_autotuned_case_matches_fixed_configuration(f3d, cuda_ok, tmp_path, monkeypatch):
    monkeypatch.setenv("FLAME3D_B200_CACHE", str(tmp_path))
    S = f3d.solver_module()
    import importlib
    A = importlib.import_module(f3d.__name__ + ".autotune")
    monkeypatch.setattr(A, "_DEFAULT", None)
    case = f3d.random_curvilinear(n=12, ns=2, seed=62)
    auto = S.DeviceCase(case, tile="auto")
    assert auto.tile in A.CANDIDATES
    assert (tmp_path / "autotune.json").exists()
    fixed = S.DeviceCase(case, tile=3)
    auto.step()
    fixed.step()
    Ua, Uf = auto.conserved(), fixed.conserved()
    mom = np.linalg.norm(Uf[1:4].ravel())
    for n in range(5):
        scale = mom if 1 <= n <= 3 else np.linalg.norm(Uf[n].ravel())
        assert np.linalg.norm((Ua[n] - Uf[n]).ravel()) <= 1e-12 * scale


@pytest.mark.parametrize("n", [6, 7, 27, 31])
@pytest.mark.parametrize("tile", [0, 3, 4, 5])
def test_fused_odd_extents(f3d, oracle, cuda_ok, n, tile):
    """Extents that divide neither the pencil (26 owned cells), the 16-column blocks nor the
    tiles, down to 4 cells on an axis (random_curvilinear uses n+4, n, n-2)."""
    S = f3d.solver_module()
    case = f3d.random_curvilinear(n=n, ns=2, seed=90 + n)
    dc = S.DeviceCase(case, tile=tile)
    oc = oracle.OracleCase(case)
    for s in (1, 2, 3):
        dc.stage_fused(s)
        oc.stage(s)
    U = dc.conserved()
    I = oracle.interior
    mom = np.linalg.norm(I(oc.U[1:4]).ravel())
    for k in range(5):
        ref = I(oc.U[k])
        scale = mom if 1 <= k <= 3 else np.linalg.norm(ref.ravel())
        assert np.linalg.norm((I(U[k]) - ref).ravel()) <= 1e-12 * scale, (n, tile, k)
    Q, r = dc.primitives()
    assert np.array_equal(Q[:, :, :, :4], Q[:, :, :, case.nx:case.nx + 4])  # periodic ghosts
