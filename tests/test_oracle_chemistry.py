"""The oracle's restatement of the reference's finite-rate chemistry (reactions.jl:187-504) on a
seeded synthetic mechanism, checked against conservation laws and independent computations."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest


def _mech(f3d):
    import importlib
    return importlib.import_module(f3d.__name__ + ".mechanism")


def _rates(oracle, mech, sc, T, jac=False):
    ns = mech.thermo.ns
    w = np.zeros(ns)
    A = np.zeros(ns * ns) if jac else None
    oracle.load().oracle_production_rate(oracle.ptr(w), oracle.ptr(np.ascontiguousarray(sc)),
                                         oracle.ptr(A) if jac else None, T,
                                         C.byref(mech.thermo.to_c()), C.byref(mech.to_c()), ns)
    return (w, A.reshape(ns, ns).T) if jac else w   # A[l, m] = d wdot_l / d sc_m


@pytest.mark.parametrize("T", [900.0, 1500.0, 2600.0])
def test_mass_and_elements_conserved(f3d, oracle, T):
    M = _mech(f3d)
    mech = M.synthetic_mechanism()
    sc = np.random.default_rng(1).uniform(1e-8, 1e-5, mech.thermo.ns)  # mol/cm^3
    w = _rates(oracle, mech, sc, T)
    assert np.abs(w).max() > 0
    scale = np.abs(w * mech.thermo.mw).sum()
    assert abs(np.sum(w * mech.thermo.mw)) <= 1e-13 * scale
    for e in range(3):
        col = M.ATOMS[:, e]
        assert abs(np.sum(w * col)) <= 1e-13 * np.abs(w * col).sum() + 1e-300


def test_jacobian_matches_finite_differences_for_arrhenius(f3d, oracle):
    """For plain Arrhenius reactions the reference's Jacobian (Σ ν q / sc) is exact."""
    M = _mech(f3d)
    mech = M.synthetic_mechanism()
    keep = mech.reaction_type == 1
    sub = M.Mechanism(mech.thermo, mech.reaction_type[keep], mech.sgm[keep], mech.vf[keep],
                      mech.vr[keep], mech.Arr[keep], mech.ef[keep], mech.loP[keep],
                      mech.Troe[keep])
    sc = np.random.default_rng(2).uniform(1e-7, 1e-5, mech.thermo.ns)
    w, A = _rates(oracle, sub, sc, 1800.0, jac=True)
    for m in range(mech.thermo.ns):
        h = 1e-4 * sc[m]  # smaller steps lose the small columns to cancellation
        sp, sm = sc.copy(), sc.copy()
        sp[m] += h
        sm[m] -= h
        fd = (_rates(oracle, sub, sp, 1800.0) - _rates(oracle, sub, sm, 1800.0)) / (2 * h)
        np.testing.assert_allclose(A[:, m], fd, rtol=1e-5, atol=1e-9 * np.abs(fd).max())


def test_solve_matches_numpy(f3d, oracle):
    rng = np.random.default_rng(3)
    for n in (1, 3, 8):
        a = rng.normal(size=(n, n)) + n * np.eye(n)
        a[[0, -1]] = a[[-1, 0]]  # something for the pivoting to do
        b = rng.normal(size=n)
        x = np.zeros(n)
        ac = np.ascontiguousarray(a.T)  # column-major
        oracle.load().oracle_solve(oracle.ptr(x), oracle.ptr(ac), oracle.ptr(b.copy()), n)
        np.testing.assert_allclose(x, np.linalg.solve(a, b), rtol=1e-12, atol=1e-14)


def _reacting_case(f3d, seed=5):
    M = _mech(f3d)
    mech = M.synthetic_mechanism()
    case = f3d.random_curvilinear(n=8, ns=8, seed=seed, T_range=(400.0, 2600.0))
    Q, r = M.reacting_state(mech, case)
    return M, mech, case, Q, r


@pytest.mark.parametrize("stiff", [0, 1])
def test_chemistry_step_conserves_and_respects_threshold(f3d, oracle, stiff):
    M, mech, case, Q, r = _reacting_case(f3d)
    U = np.ascontiguousarray(case.U())
    Q0, r0 = Q.copy(), r.copy()
    Tcrit = 1200.0
    oracle.load().oracle_eval_chem(C.byref(case.grid()), stiff, oracle.ptr(U), oracle.ptr(Q),
                                   oracle.ptr(r), 1e-12, C.byref(mech.thermo.to_c()),
                                   C.byref(mech.to_c()), None, Tcrit, 0)
    I = oracle.interior
    cold = I(Q0[5]) <= Tcrit
    assert cold.any() and (~cold).any()
    assert np.array_equal(I(r)[:, cold], I(r0)[:, cold])      # below T_criteria: untouched
    hot = ~cold
    assert not np.array_equal(I(r)[:, hot], I(r0)[:, hot])    # above: reacted
    np.testing.assert_allclose(I(r).sum(axis=0), I(Q0[0]), rtol=1e-14)  # rho_i sums to rho
    e0, e1 = M.element_totals(mech, I(r0)), M.element_totals(mech, I(r))
    np.testing.assert_allclose(e1[:2], e0[:2], rtol=1e-12)    # H and O atoms (no clipping)
    assert np.isfinite(Q).all() and (I(Q[5]) > 0).all()


@pytest.mark.parametrize("transposed", [0, 1])
def test_stiff_step_solves_the_linearised_system(f3d, oracle, transposed):
    """At a hot cell the point-implicit step is (I - A W_n / W_l dt) Δρ = ẇ W 1e6 dt, solved
    here with numpy from the oracle's own ẇ and Jacobian; then Δei from the formation
    coefficients (coeffs_lo[6, n], or the reference's transposed read [n, 6]), the clip and the
    rescale to ρ."""
    M, mech, case, Q, r = _reacting_case(f3d, seed=6)
    th = mech.thermo
    ns = th.ns
    dt = 1e-8
    U = np.ascontiguousarray(case.U())
    U0, r0 = U.copy(), r.copy()
    oracle.load().oracle_eval_chem(C.byref(case.grid()), 1, oracle.ptr(U), oracle.ptr(Q),
                                   oracle.ptr(r), dt, C.byref(th.to_c()), C.byref(mech.to_c()),
                                   None, 500.0, transposed)
    NG = f3d.FLAME_NG
    T0 = case.Q[5]
    k, j, i = [int(v) for v in np.argwhere(T0[NG:-NG, NG:-NG, NG:-NG] > 1500.0)[0] + NG]
    rc = r0[:, k, j, i]
    sc = rc / th.mw * 1e-6
    w, A = _rates(oracle, mech, sc, float(T0[k, j, i]), jac=True)
    A1 = np.eye(ns) - A * th.mw[:, None] / th.mw[None, :] * dt
    d = np.linalg.solve(A1, w * th.mw * 1e6 * dt)
    lo = th.to_c().coeffs_lo
    a6 = np.array([lo[n + 35] if transposed else lo[5 + 7 * n] for n in range(ns)])
    dei = np.sum(-a6 * d * th.Ru / th.mw)
    new = np.maximum(rc + d, 0.0)
    new *= case.Q[0, k, j, i] / new.sum()
    np.testing.assert_allclose(r[:, k, j, i], new, rtol=1e-10, atol=1e-14 * new.max())
    assert U[4, k, j, i] - U0[4, k, j, i] == pytest.approx(dei, rel=1e-9)
