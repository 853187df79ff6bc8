"""flame_rk_stage_noalloc: the RK3 stage for callers that cannot allocate device memory.

A Julia program whose device memory all belongs to CUDA.jl's pool, or a serving process that has
already committed its HBM budget, cannot hand the library a scratch buffer for the pencil-sweep
stage.  This entry point uses a fixed array the library keeps in device memory instead.  Here it
is called through the C ABI twice in a row (stage 1, then stage 2 on the result) next to
flame_rk_stage_tiled with a caller-owned scratch buffer on identical inputs; both must agree to
the 1e-12 relative L2 bound of the other parity tests.  The file is named so pytest runs it last.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(x, ref):
    n = np.linalg.norm(ref.ravel())
    d = np.linalg.norm((x - ref).ravel())
    return float(d / n) if n > 0 else float(d)


def _noalloc_stage(f3d, dc, stage):
    """One stage of `dc` through flame_rk_stage_noalloc (dc's own scratch is not passed)."""
    i, o = dc.cur, 1 - dc.cur
    p = lambda t: t.data_ptr()
    b = f3d.FlameStageBuffers(p(dc.U), p(dc.Un), p(dc.Q[i]), p(dc.Q[o]), p(dc.rhoi[i]),
                              p(dc.rhoi[o]), p(dc.rhon), p(dc.T[i]), p(dc.T[o]), None)
    rc = dc.lib.flame_rk_stage_noalloc(C.byref(dc.grid), C.c_void_p(dc.stream), stage, dc.dt,
                                       C.byref(b), C.byref(dc.cmetrics), C.byref(dc.thermo),
                                       C.byref(dc.transport), dc.precision)
    f3d.abi.check(dc.lib, rc)
    dc.cur = o


def _case(f3d, law):
    case = f3d.random_curvilinear(n=12, ns=2 if law == 1 else 3, seed=7)
    if law == 2:  # the mixture-averaged law: the stage runs configuration 6's launches
        case.transport = f3d.cases.mixture_averaged_transport(case.thermo, seed=3)
    return case


@pytest.mark.parametrize("law", [1, 2])
@pytest.mark.parametrize("precision", [0, 1])
def test_noalloc_matches_caller_scratch_two_calls(f3d, cuda_ok, precision, law):
    import torch
    S = f3d.solver_module()
    case = _case(f3d, law)
    ref = S.DeviceCase(case, precision=precision, tile=3)
    new = S.DeviceCase(case, precision=precision, tile=3)
    for stage in (1, 2):
        ref.stage_fused(stage)
        _noalloc_stage(f3d, new, stage)
        torch.cuda.synchronize()
        Ur, Un = ref.conserved(), new.conserved()
        (Qr, rr), (Qn, rn) = ref.primitives(), new.primitives()
        errs = {"U": max(_rel(Un[k], Ur[k]) for k in range(5)),
                "Q": max(_rel(Qn[k], Qr[k]) for k in (0, 4, 5, 6)),
                "rhoi": max(_rel(rn[k], rr[k]) for k in range(rr.shape[0])),
                "trans": _rel(new.T[new.cur].double().cpu().numpy(),
                              ref.T[ref.cur].double().cpu().numpy())}
        assert max(errs.values()) <= 1e-12, (stage, errs)
        assert np.isfinite(Un).all()


@pytest.mark.parametrize("ext", [(512, 512, 256), (1 << 21, 1 << 21, 1 << 21),
                                 (2**31 - 9, 2**31 - 9, 2**31 - 9)])
def test_noalloc_rejects_grids_beyond_its_scratch(f3d, cuda_ok, ext):
    """Too large for the library's array, including extents whose scratch size would wrap a
    64-bit product: rejected before any launch."""
    lib = f3d.load_library()
    g = f3d.FlameGrid(*ext, 4, 1, 7)
    assert lib.flame_stage_scratch_bytes(C.byref(g), 0) > (64 << 20)
    b = f3d.FlameStageBuffers(*([1] * 10))
    m = f3d.FlameMetrics(*([1] * 10))
    rc = lib.flame_rk_stage_noalloc(C.byref(g), None, 1, 1e-3, C.byref(b), C.byref(m),
                                    C.byref(f3d.FlameThermo()), C.byref(f3d.FlameTransport()), 0)
    assert rc == 1 and "scratch" in f3d.abi.last_error(lib)
