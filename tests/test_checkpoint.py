"""Checkpoints in the reference's restart layout (raw files; solver.jl:69-79, 438-466)."""
from __future__ import annotations

import json

import numpy as np
import pytest


def _ck(f3d):
    import importlib
    return importlib.import_module(f3d.__name__ + ".checkpoint")


def test_round_trip_and_julia_layout(f3d, tmp_path):
    ck = _ck(f3d)
    case = f3d.random_curvilinear(n=8, ns=3, seed=71)
    d = ck.save(tmp_path / "chk12.f3d", case.Q, case.rhoi, step=12, dt=case.dt)
    Q, r, meta = ck.load(d)
    assert np.array_equal(Q, case.Q) and np.array_equal(r, case.rhoi)
    assert meta["step"] == 12 and meta["dt"] == case.dt
    tx, ty, tz = case.nx + 8, case.ny + 8, case.nz + 8
    assert meta["datasets"]["Q_h"]["shape"] == [tx, ty, tz, 7, 1]
    assert meta["datasets"]["ρi_h"]["shape"] == [tx, ty, tz, 3, 1]
    raw = np.fromfile(d / "Q_h.bin", "<f8")
    i, j, k, n = 3, 5, 2, 4   # Julia Q_h[i+1, j+1, k+1, n+1, 1]
    assert raw[i + tx * (j + ty * (k + tz * n))] == case.Q[n, k, j, i]


def test_rejects_foreign_and_truncated(f3d, tmp_path):
    ck = _ck(f3d)
    case = f3d.random_curvilinear(n=8, ns=1, seed=72)
    d = ck.save(tmp_path / "c", case.Q, case.rhoi)
    (d / "Q_h.bin").write_bytes((d / "Q_h.bin").read_bytes()[:-8])
    with pytest.raises(ValueError):
        ck.load(d)
    meta = json.loads((d / "meta.json").read_text())
    meta["format"] = "something else"
    (d / "meta.json").write_text(json.dumps(meta))
    with pytest.raises(ValueError):
        ck.load(d)
    with pytest.raises(ValueError):
        ck.save(tmp_path / "bad", case.Q[:5], case.rhoi)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_restart_continues_bitwise(f3d, cuda_ok, tmp_path, precision):
    """Run 2 steps, checkpoint, run 2 more; a fresh case restored from the checkpoint and run
    2 steps ends in the same state.  A restart rebuilds U from the stored primitives (prim2c),
    as the reference's does, so FP64 agrees to round-off (1e-12) and mixed precision, whose
    checkpoint holds the FP32 primitives widened, to 1e-6."""
    ck = _ck(f3d)
    S = f3d.solver_module()
    case = f3d.random_curvilinear(n=12, ns=2, seed=73)
    a = S.DeviceCase(case, precision=precision, tile=3)
    for _ in range(2):
        a.step()
    d = ck.save_case(tmp_path / "chk2.f3d", a, step=2)
    b = S.DeviceCase(case, precision=precision, tile=3)
    meta = ck.restore_case(d, b)
    assert meta["step"] == 2
    for _ in range(2):
        a.step()
        b.step()
    (Qa, ra), (Qb, rb) = a.primitives(), b.primitives()
    tol = 1e-12 if precision == 0 else 1e-6
    vel = np.linalg.norm(Qa[1:4].ravel())
    for n, (x, y) in enumerate(list(zip(Qa, Qb)) + list(zip(ra, rb))):
        scale = vel if 1 <= n <= 3 else np.linalg.norm(x.ravel())
        assert np.linalg.norm((x - y).ravel()) <= tol * scale, n
