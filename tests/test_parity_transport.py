"""GPU parity of the mixture-averaged transport (law 2, thermo.jl:289-403) on the per-kernel
path: flame_mixture against the oracle, and the reference launch sequence over two stages.
log() and sqrt() come from different math libraries on the two sides, so the bound is a
relative 1e-13 rather than bit equality."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(f3d, ns=5, seed=41):
    case = f3d.random_curvilinear(n=12, ns=ns, seed=seed)
    case.transport = f3d.cases.mixture_averaged_transport(case.thermo, seed=seed)
    return case


def test_mixture_law2_matches_oracle(f3d, oracle, cuda_ok):
    import torch
    case = _case(f3d)
    ns, shp = case.ns, case.Q.shape[1:]
    dQ = torch.from_numpy(case.Q).cuda()
    dr = torch.from_numpy(case.rhoi).cuda()
    dpoly = torch.from_numpy(case.transport.poly).cuda()
    out = {k: torch.zeros(n, *shp, dtype=torch.float64, device="cuda")
           for k, n in (("Yi", ns), ("lam", 1), ("mu", 1), ("D", ns))}
    lib = f3d.load_library()
    tr = case.transport.to_c(dpoly.data_ptr())
    rc = lib.flame_mixture(C.byref(case.grid()), C.c_void_p(torch.cuda.current_stream().cuda_stream),
                           dQ.data_ptr(), dr.data_ptr(), out["Yi"].data_ptr(),
                           out["lam"].data_ptr(), out["mu"].data_ptr(), out["D"].data_ptr(),
                           C.byref(case.thermo.to_c()), C.byref(tr), None)
    f3d.abi.check(lib, rc)
    torch.cuda.synchronize()
    ref = {k: np.zeros((n,) + shp) for k, n in (("Yi", ns), ("lam", 1), ("mu", 1), ("D", ns))}
    P = oracle.ptr
    oracle.load().oracle_mixture(C.byref(case.grid()), P(case.Q), P(case.rhoi), P(ref["Yi"]),
                                 P(ref["lam"]), P(ref["mu"]), P(ref["D"]),
                                 C.byref(case.thermo.to_c()), C.byref(case.transport.to_c()), None)
    assert np.array_equal(out["Yi"].cpu().numpy(), ref["Yi"])
    for k in ("lam", "mu", "D"):
        np.testing.assert_allclose(out[k].cpu().numpy(), ref[k], rtol=1e-13, atol=0)
    D = ref["D"]
    assert np.isfinite(D).all() and (D > 0).all()
    assert len(np.unique(np.round(D[:, 6, 6, 6] / D[0, 6, 6, 6], 6))) == ns  # per species


def test_launch_sequence_law2_matches_oracle(f3d, oracle, cuda_ok):
    S = f3d.solver_module()
    case = _case(f3d, ns=6, seed=42)
    dc = S.DeviceCase(case, sequence_buffers=True)
    oc = oracle.OracleCase(case)
    for s in (1, 2):
        dc.stage_sequence(s)
        oc.stage(s)
    U = dc.conserved()
    I = oracle.interior
    mom = np.linalg.norm(I(oc.U[1:4]).ravel())
    for n in range(5):
        ref = I(oc.U[n])
        scale = mom if 1 <= n <= 3 else np.linalg.norm(ref.ravel())
        assert np.linalg.norm((I(U[n]) - ref).ravel()) <= 1e-12 * scale, n
    _, r = dc.primitives()
    assert np.linalg.norm((I(r) - I(oc.rhoi)).ravel()) <= 1e-12 * np.linalg.norm(I(oc.rhoi).ravel())


def test_fused_stage_refuses_law2(f3d, cuda_ok):
    S = f3d.solver_module()
    case = _case(f3d, ns=3, seed=43)
    dc = S.DeviceCase(case)
    assert dc.tile is None
    lib = f3d.load_library()
    b = f3d.FlameStageBuffers(*([1] * 10))
    rc = lib.flame_rk_stage_tiled(C.byref(dc.grid), None, 1, 1e-6, C.byref(b),
                                  C.byref(dc.cmetrics), C.byref(dc.thermo),
                                  C.byref(dc.transport), 0, 3)
    assert rc == 5 and "law 2" in f3d.abi.last_error(lib)
