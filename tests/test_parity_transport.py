"""GPU parity of the mixture-averaged transport (law 2, thermo.jl:289-403): flame_mixture
against the oracle, the reference launch sequence over two stages, and the fused stage's pencil
configurations (per-species D_k in the sweeps, the mixture rule in the finish) over two steps.
log() and sqrt() come from different math libraries on the two sides, so the bound on the
transport fields is a relative 1e-13 rather than bit equality, and 1e-12 on the stages."""
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


def test_tile_configs_refuse_law2(f3d, cuda_ok):
    """The tile kernels hold one D per point; law 2 is refused there with FLAME_EUNSUPPORTED
    (before any launch) and runs on the pencil configurations as configuration 6."""
    S = f3d.solver_module()
    case = _case(f3d, ns=3, seed=43)
    dc = S.DeviceCase(case)
    assert dc.tile == 3 and dc.launched_config == 6 and dc.T[0].shape[0] == 2 + 3
    lib = f3d.load_library()
    b = f3d.FlameStageBuffers(*([1] * 10))
    for tile in (0, 1, 2):
        rc = lib.flame_rk_stage_tiled(C.byref(dc.grid), None, 1, 1e-6, C.byref(b),
                                      C.byref(dc.cmetrics), C.byref(dc.thermo),
                                      C.byref(dc.transport), 0, tile)
        assert rc == 5 and "law 2" in f3d.abi.last_error(lib)


def _stage_errors(dc, oc, oracle):
    I = oracle.interior
    U = dc.conserved()
    mom = np.linalg.norm(I(oc.U[1:4]).ravel())
    e = {}
    for n in range(5):
        ref = I(oc.U[n])
        scale = mom if 1 <= n <= 3 else np.linalg.norm(ref.ravel())
        e[f"U{n}"] = float(np.linalg.norm((I(U[n]) - ref).ravel()) / scale)
    _, r = dc.primitives()
    e["rhoi"] = oracle.rel_l2(I(r), I(oc.rhoi))
    return e


@pytest.mark.parametrize("tile", [3, 4, 6])
@pytest.mark.parametrize("ns", [2, 5, 9])
def test_fused_law2_matches_oracle(f3d, oracle, cuda_ok, ns, tile):
    """Two RK3 steps of the fused stage with mixture-averaged transport against the oracle's
    launch sequence (mixture kernel first in every stage): 1e-12 relative L2."""
    S = f3d.solver_module()
    case = _case(f3d, ns=ns, seed=50 + ns)
    dc = S.DeviceCase(case, tile=tile)
    oc = oracle.OracleCase(case)
    for _ in range(2):
        dc.step()
        oc.step()
    e = _stage_errors(dc, oc, oracle)
    assert max(e.values()) <= 1e-12, e
    assert np.isfinite(dc.conserved()).all()


def test_fused_law2_transport_fields(f3d, oracle, cuda_ok):
    """The transport fields the stage leaves for the next one: μ, λ and one D_k per species,
    equal to the oracle's mixture kernel on the stage's own output state."""
    import torch
    S = f3d.solver_module()
    case = _case(f3d, ns=5, seed=57)
    dc = S.DeviceCase(case, tile=4)
    dc.stage_fused(1)
    torch.cuda.synchronize()
    Q, r = dc.primitives()
    T = dc.T[dc.cur].cpu().numpy()
    shp, ns = Q.shape[1:], case.ns
    ref = {k: np.zeros((n,) + shp) for k, n in (("Yi", ns), ("lam", 1), ("mu", 1), ("D", ns))}
    P = oracle.ptr
    Qc, rc = np.ascontiguousarray(Q), np.ascontiguousarray(r)
    oracle.load().oracle_mixture(C.byref(case.grid()), P(Qc), P(rc), P(ref["Yi"]),
                                 P(ref["lam"]), P(ref["mu"]), P(ref["D"]),
                                 C.byref(case.thermo.to_c()), C.byref(case.transport.to_c()), None)
    np.testing.assert_allclose(T[0], ref["mu"][0], rtol=1e-13, atol=0)
    np.testing.assert_allclose(T[1], ref["lam"][0], rtol=1e-13, atol=0)
    np.testing.assert_allclose(T[2:], ref["D"], rtol=1e-13, atol=0)


def test_fused_law2_mixed_precision(f3d, oracle, cuda_ok):
    """Mixed precision with law 2 (D_k stored in FP32): within the mixed path's 1e-5 bound of
    the oracle after two steps."""
    S = f3d.solver_module()
    case = _case(f3d, ns=5, seed=58)
    dc = S.DeviceCase(case, precision=1, tile=6)
    oc = oracle.OracleCase(case)
    for _ in range(2):
        dc.step()
        oc.step()
    e = _stage_errors(dc, oc, oracle)
    assert max(e["U0"], e["U4"], e["U1"]) <= 1e-5, e


def test_fused_law2_odd_extents(f3d, oracle, cuda_ok):
    """Odd, unequal extents (15 x 11 x 9): the per-species D_k loads of the sweeps follow the
    pencils' strides, and the finish writes every ghost image."""
    S = f3d.solver_module()
    case = f3d.random_curvilinear(n=11, ns=3, seed=59)
    case.transport = f3d.cases.mixture_averaged_transport(case.thermo, seed=59)
    dc = S.DeviceCase(case, tile=6)
    oc = oracle.OracleCase(case)
    for _ in range(2):
        dc.step()
        oc.step()
    e = _stage_errors(dc, oc, oracle)
    assert max(e.values()) <= 1e-12, e
