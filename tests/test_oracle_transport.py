"""The oracle's mixture-averaged transport (law 2, mixtureProperties thermo.jl:289-369) against
its defining formulas on the host, and against limits with closed forms."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest


def _props(oracle, T, P, X, thermo, tr):
    ns = thermo.ns
    th = thermo.to_c()
    Dk = np.zeros(ns)
    lam, mu = C.c_double(), C.c_double()
    Xa = np.ascontiguousarray(X, dtype=np.float64)
    oracle.load().oracle_mixture_properties(T, P, oracle.ptr(Xa), C.byref(th),
                                            oracle.ptr(tr.poly), ns, oracle.ptr(Dk),
                                            C.byref(lam), C.byref(mu))
    return lam.value, mu.value, Dk


def _numpy_props(T, P, X, thermo, poly):
    """The same definitions written independently with numpy."""
    ns = thermo.ns
    visc = poly[:5 * ns].reshape(ns, 5)
    cond = poly[5 * ns:10 * ns].reshape(ns, 5)
    binc = poly[10 * ns:].reshape(ns, ns, 5)
    L = np.log(T) ** np.arange(5)
    lam_k = np.sqrt(T) * cond @ L
    lam = 0.5 * (np.sum(X * lam_k) + 1 / np.sum(X / lam_k))
    mu_k = (T ** 0.25 * visc @ L) ** 2
    W = thermo.mw
    phi = (1 + np.sqrt(mu_k[:, None] / mu_k[None, :]) * (W[None, :] / W[:, None]) ** 0.25) ** 2 \
        / np.sqrt(8 * (1 + W[:, None] / W[None, :]))
    mu = np.sum(X * mu_k / (phi @ X))
    Djk = T ** 1.5 * binc @ L  # symmetric
    Dk = np.array([(1 - X[k]) / (P * sum(X[j] / Djk[k, j] for j in range(ns) if j != k)
                                 + 2.220446049250313e-16) for k in range(ns)])
    return lam, mu, Dk


@pytest.mark.parametrize("ns", [2, 5, 9])
def test_matches_numpy_restatement(f3d, oracle, ns):
    thermo = f3d.synthetic_species(9, 3).subset(ns)
    tr = f3d.cases.mixture_averaged_transport(thermo, seed=ns)
    rng = np.random.default_rng(ns)
    for T in (300.0, 1234.5, 2900.0):
        X = rng.dirichlet(np.ones(ns))
        P = 101325.0 * rng.uniform(0.5, 2)
        lam, mu, Dk = _props(oracle, T, P, X, thermo, tr)
        rl, rm, rd = _numpy_props(T, P, X, thermo, tr.poly)
        assert lam == pytest.approx(rl, rel=1e-13)
        assert mu == pytest.approx(rm, rel=1e-13)
        np.testing.assert_allclose(Dk, rd, rtol=1e-13)


def test_single_species_limit(f3d, oracle):
    thermo = f3d.synthetic_species(9, 3).subset(1)
    tr = f3d.cases.mixture_averaged_transport(thermo, seed=4)
    for T in (250.0, 800.0, 2500.0):
        lam, mu, Dk = _props(oracle, T, 1e5, np.ones(1), thermo, tr)
        L = np.log(T) ** np.arange(5)
        assert mu == pytest.approx((T ** 0.25 * tr.poly[:5] @ L) ** 2, rel=1e-13)
        assert lam == pytest.approx(np.sqrt(T) * tr.poly[5:10] @ L, rel=1e-13)
        assert Dk[0] == 0.0  # (1 - X) / (0 + eps)


def test_identical_species_limit(f3d, oracle):
    """Two copies of one species: Wilke's φ = 1, so μ and λ are the pure values and
    D_k = D_12 / P."""
    one = f3d.synthetic_species(9, 3).subset(1)
    thermo = f3d.Thermo(np.repeat(one.mw, 2), np.repeat(one.lo, 2, 0), np.repeat(one.hi, 2, 0),
                        np.repeat(one.sep, 2), one.min_temp, one.max_temp, one.Ru)
    tr1 = f3d.cases.mixture_averaged_transport(one, seed=5)
    v, c, b = tr1.poly[:5], tr1.poly[5:10], tr1.poly[10:15]
    poly = np.concatenate([v, v, c, c, b, b, b, b])
    tr = f3d.Transport(law=2, poly=poly)
    T, P = 900.0, 2e5
    lam, mu, Dk = _props(oracle, T, P, np.array([0.3, 0.7]), thermo, tr)
    L = np.log(T) ** np.arange(5)
    assert mu == pytest.approx((T ** 0.25 * v @ L) ** 2, rel=1e-14)
    assert lam == pytest.approx(np.sqrt(T) * c @ L, rel=1e-14)
    np.testing.assert_allclose(Dk, T ** 1.5 * (b @ L) / P, rtol=1e-14)


def test_fits_reproduce_their_laws(f3d):
    thermo = f3d.synthetic_species(9, 3).subset(3)
    tr = f3d.cases.mixture_averaged_transport(thermo, seed=6)
    rng = np.random.default_rng(6)
    mu0 = rng.uniform(1e-5, 3e-5, 3)
    T = np.array([300.0, 1000.0, 2500.0])
    L = np.log(T)[:, None] ** np.arange(5)
    mu = (T ** 0.25 * (L @ tr.poly[:5])) ** 2
    np.testing.assert_allclose(mu, mu0[0] * (T / 300) ** 0.7, rtol=1e-3)
