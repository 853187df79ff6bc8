"""The oracle's restatement of the reference's ghost fills (boundary.jl:1-191) and of the CFL
rate reduction, checked against their definitions on the host (no GPU)."""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import pytest


def _state(f3d, ns=5, seed=21):
    case = f3d.random_curvilinear(n=10, ns=ns, seed=seed)
    Q = np.ascontiguousarray(case.Q.copy())
    rhoi = np.ascontiguousarray(case.rhoi.copy())
    U = np.ascontiguousarray(case.U())
    Yi = np.ascontiguousarray(np.random.default_rng(seed).uniform(0, 1, rhoi.shape))
    return case, Q, U, rhoi, Yi


def test_fill_x_inflow_and_outlet(f3d, oracle):
    case, Q, U, rhoi, Yi = _state(f3d)
    Q0, U0, r0 = Q.copy(), U.copy(), rhoi.copy()
    th = case.thermo.to_c()
    inflow = f3d.cases.reference_inflow(case.ns)
    lib = oracle.load()
    P = oracle.ptr
    lib.oracle_fill_x(C.byref(case.grid()), P(Q), P(U), P(rhoi), P(Yi), C.byref(th),
                      C.byref(inflow), 0, 1)
    NG, nx = f3d.FLAME_NG, case.nx
    W = case.thermo.mw
    Y = np.zeros(case.ns)
    Y[1], Y[4] = 0.233, 0.767
    rho = 79.8 / (case.thermo.Ru * 270.65 * np.sum(Y / W))
    e = case.thermo.internal_energy(np.array([270.65]), (Y * rho)[:, None])[0]
    inl = Q[:, :, :, :NG + 1]                       # i <= NG+1 (1-based)
    assert np.allclose(inl[0], rho, rtol=1e-15) and np.all(inl[1] == 1000.0)
    assert np.all(inl[2] == 0) and np.all(inl[3] == 0) and np.all(inl[4] == 79.8)
    assert np.all(inl[5] == 270.65) and np.allclose(inl[6], e, rtol=1e-14)
    assert np.allclose(U[4, :, :, :NG + 1], e + 0.5 * rho * 1e6, rtol=1e-14)
    assert np.allclose(rhoi[:, :, :, 0], (Y * rho)[:, None, None], rtol=1e-15)
    assert np.all(Yi[:, :, :, 0] == Y[:, None, None])
    src = nx + NG - 2                               # Nxp+NG-1 (1-based)
    for a, a0 in ((Q, Q0), (U, U0), (rhoi, r0)):
        assert np.array_equal(a[..., nx + NG - 1:], np.repeat(a0[..., src:src + 1], NG + 1, -1))
        assert np.array_equal(a[..., NG + 1:src + 1], a0[..., NG + 1:src + 1])  # untouched


def test_fill_x_ranks(f3d, oracle):
    """Middle ranks of an x-slab decomposition fill nothing; the last one only the outlet."""
    case, Q, U, rhoi, Yi = _state(f3d)
    Q0 = Q.copy()
    th, inflow = case.thermo.to_c(), f3d.cases.reference_inflow(case.ns)
    lib, P = oracle.load(), oracle.ptr
    lib.oracle_fill_x(C.byref(case.grid()), P(Q), P(U), P(rhoi), P(Yi), C.byref(th),
                      C.byref(inflow), 1, 3)
    assert np.array_equal(Q, Q0)
    lib.oracle_fill_x(C.byref(case.grid()), P(Q), P(U), P(rhoi), P(Yi), C.byref(th),
                      C.byref(inflow), 2, 3)
    NG = f3d.FLAME_NG
    assert np.array_equal(Q[..., :NG + 1], Q0[..., :NG + 1])  # no inflow off rank 0


def test_fill_y_and_z_zero_gradient(f3d, oracle):
    case, Q, U, rhoi, Yi = _state(f3d, seed=22)
    Q0, U0, r0 = Q.copy(), U.copy(), rhoi.copy()
    lib, P, g = oracle.load(), oracle.ptr, C.byref(case.grid())
    NG, ny, nz = f3d.FLAME_NG, case.ny, case.nz
    lib.oracle_fill_y(g, P(Q), P(U), None)
    for a, a0 in ((Q, Q0), (U, U0)):
        assert np.array_equal(a[:, :, :NG + 1, :], np.repeat(a0[:, :, NG + 1:NG + 2, :], NG + 1, 2))
        s = ny + NG - 2
        assert np.array_equal(a[:, :, ny + NG - 1:, :], np.repeat(a0[:, :, s:s + 1, :], NG + 1, 2))
    assert np.array_equal(rhoi, r0)  # fill_y leaves ρi to fill_y_s
    lib.oracle_fill_y(g, None, None, P(rhoi))
    assert np.array_equal(rhoi[:, :, :NG + 1, :], np.repeat(r0[:, :, NG + 1:NG + 2, :], NG + 1, 2))
    r1 = rhoi.copy()
    lib.oracle_fill_z_s(g, P(rhoi))
    s = nz + NG - 2
    assert np.array_equal(rhoi[:, nz + NG - 1:], np.repeat(r1[:, s:s + 1], NG + 1, 1))
    assert np.array_equal(rhoi[:, :nz + NG - 1], r1[:, :nz + NG - 1])


def test_fill_z_inflow(f3d, oracle):
    case, Q, U, rhoi, Yi = _state(f3d, seed=23)
    Q0 = Q.copy()
    th, inflow = case.thermo.to_c(), f3d.cases.reference_inflow(case.ns)
    lib, P = oracle.load(), oracle.ptr
    lib.oracle_fill_z(C.byref(case.grid()), P(Q), P(U), P(rhoi), P(Yi), C.byref(th),
                      C.byref(inflow))
    NG, nz = f3d.FLAME_NG, case.nz
    assert np.all(Q[1, :NG + 1] == 1000.0) and np.all(Q[4, :NG + 1] == 79.8)
    s = nz + NG - 2
    assert np.array_equal(Q[:, nz + NG - 1:], np.repeat(Q0[:, s:s + 1], NG + 1, 1))


def test_reference_inflow_needs_five_species(f3d):
    with pytest.raises(ValueError):
        f3d.cases.reference_inflow(3)


@pytest.mark.parametrize("maker", ["jet", "rand", "tgv"])
def test_cfl_max_matches_host_rule(f3d, oracle, maker):
    case = {"jet": lambda: f3d.curvilinear_jet(nx=24, ny=16, nz=12),
            "rand": lambda: f3d.random_curvilinear(n=12, ns=3, seed=24),
            "tgv": lambda: f3d.taylor_green(n=16, Ma=0.4)}[maker]()
    m = {k: np.ascontiguousarray(v) for k, v in case.metrics.items()}
    rate = oracle.load().oracle_cfl_max(C.byref(case.grid()), oracle.ptr(np.ascontiguousarray(case.Q)),
                                        C.byref(oracle.metrics_struct(m)))
    cfl = case.info.get("cfl", 0.5)
    assert cfl / rate == case.dt  # the same rule, the same operation order, bit for bit
    assert math.isfinite(rate) and rate > 0


def _ib_setup(case, seed=3, nghost=12):
    """Immersed-boundary arrays in the reference's layout: tag (Tx, Ty, Tz) with a few ghost
    points (3), each with a 15-point stencil of fluid points (1-based Julia indices) and
    averaging coefficients (Y and p zero gradient, velocity mirrored)."""
    rng = np.random.default_rng(seed)
    sh = case.Q.shape[1:]                       # (Tz, Ty, Tx)
    tz, ty, tx = sh
    np_ = tz * ty * tx
    tag = np.zeros(sh, dtype=np.int64)
    flat = rng.choice(np_, size=nghost, replace=False)
    tag.ravel()[flat] = 3
    fluid = np.flatnonzero(tag.ravel() == 0)
    ni = np.ones((np_, 15), dtype=np.int64)     # Julia (15, Tx, Ty, Tz): point-major rows
    nj, nk = ni.copy(), ni.copy()
    cd = np.zeros((np_, 16))
    cn = np.zeros((np_, 16))
    for p in flat:
        pts = rng.choice(fluid, size=15, replace=False)
        x, y, z = pts % tx, (pts // tx) % ty, pts // (tx * ty)
        ni[p], nj[p], nk[p] = x + 1, y + 1, z + 1
        cn[p, 0], cn[p, 1:] = -1.0, 1.0 / 15
        cd[p, 0], cd[p, 1:] = 1.0, 1.0 / 15
    return tag, ni, nj, nk, cd, cn, flat


def test_fill_ib_averages_and_mirrors(f3d, oracle):
    case = f3d.random_curvilinear(n=10, ns=3, seed=41)
    Q, r = case.Q.copy(), case.rhoi.copy()
    U = np.ascontiguousarray(case.U())
    tag, ni, nj, nk, cd, cn, flat = _ib_setup(case)
    P = oracle.ptr
    I64 = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    oracle.load().oracle_fill_ib(C.byref(case.grid()), P(Q), P(U), P(r), I64(ni), I64(nj),
                                 I64(nk), P(cd), P(cn), I64(tag), C.byref(case.thermo.to_c()),
                                 300.0)
    th = case.thermo
    Qf, rf = case.Q.reshape(7, -1), case.rhoi.reshape(case.ns, -1)
    for p in flat:
        pts = (ni[p] - 1) + case.Q.shape[3] * ((nj[p] - 1) + case.Q.shape[2] * (nk[p] - 1))
        Y = (rf[:, pts] / Qf[0, pts]).mean(axis=1)
        pg = Qf[4, pts].mean()
        rho = pg / (th.Ru * 300.0 * np.sum(Y / th.mw))
        q = Q.reshape(7, -1)[:, p]
        np.testing.assert_allclose(q[[1, 2, 3]], -Qf[1:4, pts].mean(axis=1), rtol=1e-13)
        assert q[4] == pytest.approx(pg, rel=1e-14) and q[5] == 300.0
        assert q[0] == pytest.approx(rho, rel=1e-13)
        np.testing.assert_allclose(r.reshape(case.ns, -1)[:, p], Y * rho, rtol=1e-13)
        e = th.internal_energy(np.array([300.0]), (Y * rho)[:, None])[0]
        assert q[6] == pytest.approx(e, rel=1e-13)
    keep = tag.ravel() != 3
    assert np.array_equal(Q.reshape(7, -1)[:, keep], Qf[:, keep])  # only ghost points change


def test_inflow_case_has_reference_boundaries_and_all_branches(f3d, oracle):
    """cases.inflow_jet on the oracle: the reference's fills put the inflow state on the x-low
    planes (boundary.jl:9-41), and the sensor spans all three hybrid branches (schemes.jl:86-437:
    UP7 below 1e-3, WENO-Z below 0.1, minmod above), so the GPU parity test on this case
    exercises every branch next to the non-periodic boundaries."""
    import ctypes as C
    import numpy as np
    case = f3d.inflow_jet(nx=32, ny=16, nz=16, ns=5)
    oc = oracle.OracleCase(case)
    ng = 4
    assert np.allclose(oc.Q[1, :, :, :ng + 1], 1000.0)
    assert np.allclose(oc.Q[5, :, :, :ng + 1], 270.65)
    phi = np.zeros(oc.Q.shape[1:])
    oracle.load().oracle_shockSensor(C.byref(oc.grid), oracle.ptr(phi), oracle.ptr(oc.Q))
    inner = oracle.interior(phi)
    assert (inner < 1e-3).any() and ((inner >= 1e-3) & (inner < 0.1)).any() and (inner >= 0.1).any()
    oc.step()
    assert np.isfinite(oc.U).all()

