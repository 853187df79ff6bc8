"""GPU parity of the reference's ghost fills (boundary.jl:1-191) and the CFL reduction.

The kernels are in the -fmad=false translation unit, so they must equal the oracle bit for bit:
fillGhost (fill_x, fill_y, fill_z) then fillSpec (fill_y_s, fill_z_s) on random states with the
reference's inflow, every x-slab rank position, and the CFL rate on three kinds of grid."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("rank,nprocs", [(0, 1), (0, 2), (1, 2), (1, 3)])
def test_fillghost_fillspec_bit_identical(f3d, oracle, cuda_ok, rank, nprocs):
    import torch
    case = f3d.random_curvilinear(n=10, ns=6, seed=31 + rank)
    Q, rhoi = case.Q.copy(), case.rhoi.copy()
    U = case.U()
    Yi = np.random.default_rng(7).uniform(0, 1, rhoi.shape)
    th, inflow = case.thermo.to_c(), f3d.cases.reference_inflow(case.ns)
    g = case.grid()
    dQ, dU, dr, dY = (_dev(a) for a in (Q, U, rhoi, Yi))
    lib = f3d.load_library()
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    f3d.abi.check(lib, lib.flame_fillGhost(C.byref(g), s, dQ.data_ptr(), dU.data_ptr(),
                                           dr.data_ptr(), dY.data_ptr(), C.byref(th),
                                           C.byref(inflow), rank, nprocs))
    f3d.abi.check(lib, lib.flame_fillSpec(C.byref(g), s, dr.data_ptr()))
    torch.cuda.synchronize()
    o, P = oracle.load(), oracle.ptr
    hQ, hU, hr, hY = (np.ascontiguousarray(a) for a in (Q, U, rhoi, Yi))
    o.oracle_fill_x(C.byref(g), P(hQ), P(hU), P(hr), P(hY), C.byref(th), C.byref(inflow), rank,
                    nprocs)
    o.oracle_fill_y(C.byref(g), P(hQ), P(hU), None)
    o.oracle_fill_z(C.byref(g), P(hQ), P(hU), P(hr), P(hY), C.byref(th), C.byref(inflow))
    o.oracle_fill_y(C.byref(g), None, None, P(hr))
    o.oracle_fill_z_s(C.byref(g), P(hr))
    for d, h in ((dQ, hQ), (dU, hU), (dr, hr), (dY, hY)):
        assert np.array_equal(d.cpu().numpy(), h)


def test_fills_reject_tiny_grids(f3d, cuda_ok):
    lib = f3d.load_library()
    g = f3d.FlameGrid(2, 8, 8, 4, 1, 0)
    rc = lib.flame_fill_y(C.byref(g), None, C.c_void_p(1), C.c_void_p(1))
    assert rc == 1 and "3 cells" in f3d.abi.last_error(lib)


@pytest.mark.parametrize("maker", ["jet", "rand", "tgv"])
def test_cfl_max_bit_identical(f3d, oracle, cuda_ok, maker):
    import torch
    case = {"jet": lambda: f3d.curvilinear_jet(nx=40, ny=24, nz=20, pressure_noise=0.02),
            "rand": lambda: f3d.random_curvilinear(n=14, ns=4, seed=33),
            "tgv": lambda: f3d.taylor_green(n=24, Ma=0.9)}[maker]()
    dm = {k: _dev(v) for k, v in case.metrics.items()}
    cm = f3d.FlameMetrics(**{k: v.data_ptr() for k, v in dm.items()})
    dQ = _dev(case.Q)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    lib = f3d.load_library()
    f3d.abi.check(lib, lib.flame_cfl_max(C.byref(case.grid()),
                                         C.c_void_p(torch.cuda.current_stream().cuda_stream),
                                         dQ.data_ptr(), C.byref(cm), out.data_ptr()))
    m = {k: np.ascontiguousarray(v) for k, v in case.metrics.items()}
    ref = oracle.load().oracle_cfl_max(C.byref(case.grid()), oracle.ptr(np.ascontiguousarray(case.Q)),
                                       C.byref(oracle.metrics_struct(m)))
    assert out.item() == ref
    assert case.info["cfl"] / out.item() == case.dt


def test_fill_ib_bit_identical(f3d, oracle, cuda_ok):
    import importlib

    import torch
    tb = importlib.import_module("test_oracle_boundary")
    case = f3d.random_curvilinear(n=12, ns=4, seed=42)
    Q, r = case.Q.copy(), case.rhoi.copy()
    U = np.ascontiguousarray(case.U())
    tag, ni, nj, nk, cd, cn, _ = tb._ib_setup(case, seed=5, nghost=40)
    cd[cd != 0] *= np.random.default_rng(6).uniform(0.5, 1.5, np.count_nonzero(cd))
    cn[cn != 0] *= np.random.default_rng(7).uniform(0.5, 1.5, np.count_nonzero(cn))
    d = {k: _dev(v) for k, v in dict(Q=Q, U=U, r=r, ni=ni, nj=nj, nk=nk, cd=cd, cn=cn,
                                     tag=tag).items()}
    lib = f3d.load_library()
    th = case.thermo.to_c()
    f3d.abi.check(lib, lib.flame_fillIB(C.byref(case.grid()),
                                        C.c_void_p(torch.cuda.current_stream().cuda_stream),
                                        *(d[k].data_ptr() for k in ("Q", "U", "r", "ni", "nj",
                                                                    "nk", "cd", "cn", "tag")),
                                        C.byref(th), 300.0))
    torch.cuda.synchronize()
    P = oracle.ptr
    I64 = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    oracle.load().oracle_fill_ib(C.byref(case.grid()), P(Q), P(U), P(r), I64(ni), I64(nj),
                                 I64(nk), P(cd), P(cn), I64(tag), C.byref(th), 300.0)
    for k, h in (("Q", Q), ("U", U), ("r", r)):
        assert np.array_equal(d[k].cpu().numpy(), h), k
