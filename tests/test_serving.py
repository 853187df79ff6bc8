"""Serving: request stream, initial states built on the device, admission, continuous batching.

CPU tests cover the request generator, the device-side builder (run with torch on the CPU
against the numpy generators) and the admission rule.  GPU tests run the server on small
streams: every request completes, resident bytes stay within the budget, each result is
bitwise the same served alone and in the mix, and results agree with the FP64 oracle.
"""
from __future__ import annotations

import math
from collections import deque

import numpy as np
import pytest


def _serving(f3d):
    import importlib
    return importlib.import_module(f3d.__name__ + ".serving")


def test_request_stream_is_seeded_poisson(f3d):
    S = _serving(f3d)
    a = S.request_stream(2000, rate=20.0, seed=5)
    b = S.request_stream(2000, rate=20.0, seed=5)
    assert [(r.arrival, r.n, r.ns, r.steps) for r in a] == [(r.arrival, r.n, r.ns, r.steps)
                                                            for r in b]
    t = np.array([r.arrival for r in a])
    gaps = np.diff(np.concatenate([[0.0], t]))
    assert (gaps > 0).all()
    assert abs(gaps.mean() - 1 / 20) < 0.1 / 20          # mean 1/λ
    assert abs(gaps.std() / gaps.mean() - 1) < 0.1       # exponential: CV = 1
    n = np.array([r.n for r in a])
    assert n.min() >= 32 and n.max() <= 256
    ln = np.log(n)                                       # log-uniform: median near sqrt(32*256)
    assert abs(np.median(ln) - math.log(math.sqrt(32 * 256))) < 0.1
    assert {r.ns for r in a} == set(range(1, 10))
    assert 0.4 < np.mean([r.curvilinear for r in a]) < 0.6
    assert min(r.Ma for r in a) >= 0.1 and max(r.Ma for r in a) <= 1.5
    assert min(r.steps for r in a) >= 200 and max(r.steps for r in a) <= 2000
    c = S.request_stream(50, step_scale=0.05, seed=5)
    assert all(1 <= r.steps <= 100 for r in c)


@pytest.mark.parametrize("ns,Ma", [(1, 0.3), (4, 0.8)])
def test_device_builder_matches_numpy_taylor_green(f3d, ns, Ma):
    """On a Cartesian request the torch builder reproduces cases.taylor_green."""
    S = _serving(f3d)
    req = S.SolveRequest(0, 0.0, 12, False, ns, 1000.0, Ma, 5, 77)
    c = S.build_request_case(req, device="cpu")
    ref = f3d.taylor_green(n=12, Re=1000.0, Ma=Ma, ns=ns, perturb=0.02, seed=77)
    for name in ref.metrics:
        np.testing.assert_allclose(c.metrics[name].numpy(), ref.metrics[name], rtol=1e-14,
                                   atol=0)
    for k in range(7):
        scale = np.abs(ref.Q[k]).max() or 1.0
        assert np.abs(c.Q[k].numpy() - ref.Q[k]).max() <= 1e-13 * scale, k
    np.testing.assert_allclose(c.rhoi.numpy(), ref.rhoi, rtol=1e-13, atol=0)
    assert abs(c.dt - ref.dt) <= 1e-13 * ref.dt
    assert c.transport.mu_ref == pytest.approx(ref.transport.mu_ref, rel=1e-14)


def test_device_builder_curvilinear(f3d):
    """The wavy mapping scaled to [0, 2π): periodic metrics, positive pressure at Ma 1.5."""
    S = _serving(f3d)
    req = S.SolveRequest(0, 0.0, 10, True, 3, 800.0, 1.5, 5, 78)
    c = S.build_request_case(req, device="cpu")
    xyz = f3d.cases.wavy_mapping(10, 10, 10, amp=0.1, scale=2 * math.pi)
    ref = f3d.cases.metrics_from_mapping(xyz, 10, 10, 10)
    for name in ref:
        np.testing.assert_allclose(c.metrics[name].numpy(), ref[name], rtol=1e-13,
                                   atol=1e-13 * np.abs(ref[name]).max())
    Q = c.Q.numpy()
    NG = f3d.FLAME_NG
    inner = Q[:, NG:-NG, NG:-NG, NG:-NG]
    assert inner[4].min() >= 0.2 * 101325.0 * (1 - 1e-12)
    assert np.isfinite(Q).all() and (Q[0] > 0).all()
    np.testing.assert_array_equal(Q[:, :, :, :NG], Q[:, :, :, 10:10 + NG])  # periodic ghosts
    assert c.dt > 0


def test_admission_is_first_come_first_served(f3d):
    S = _serving(f3d)
    size = {0: 40, 1: 30, 2: 200, 3: 10, 4: 20}
    q = deque([0, 1, 2, 3, 4])
    admit, reject = S.admissions(q, size.get, used=0, budget=100, free_slots=8)
    assert admit == [0, 1, 3, 4] and reject == [2]    # 2 can never fit: rejected, not blocking
    assert list(q) == []
    q = deque([0, 1, 3, 4])
    admit, reject = S.admissions(q, size.get, used=50, budget=100, free_slots=8)
    assert admit == [0] and reject == [] and list(q) == [1, 3, 4]  # 1 blocks 3 and 4
    q = deque([3, 4, 0])
    admit, _ = S.admissions(q, size.get, used=0, budget=100, free_slots=1)
    assert admit == [3] and list(q) == [4, 0]          # slots bound too


def test_resident_bytes_formula(f3d):
    """Resident bytes grow with the ghosted points and species; mixed precision holds less."""
    S = _serving(f3d)
    r1 = S.SolveRequest(0, 0.0, 32, False, 1, 1000.0, 0.3, 5, 1)
    r9 = S.SolveRequest(0, 0.0, 32, False, 9, 1000.0, 0.3, 5, 1)
    P = 40 ** 3
    b0, b1 = S.resident_bytes(r1, 0), S.resident_bytes(r1, 1)
    assert b1 < b0
    assert b0 >= P * 8 * (10 + 10 + 3 + 14 + 6)
    assert S.resident_bytes(r9, 0) - b0 >= P * 8 * 3 * 8


# ---------------------------------------------------------------------------------------- GPU
def _conserved(Q):
    """ρ, ρu, ρv, ρw, ρE from the primitives (prim2c, utils.jl:71-92)."""
    rho, u, v, w, e = Q[0], Q[1], Q[2], Q[3], Q[6]
    return np.stack([rho, rho * u, rho * v, rho * w, e + 0.5 * rho * (u * u + v * v + w * w)])


def _small_stream(S, count=8, seed=9):
    reqs = S.request_stream(count, rate=400.0, seed=seed, n_range=(12, 20),
                            steps_range=(2, 7), Ma_range=(0.1, 1.5))
    return reqs


@pytest.mark.gpu
def test_server_completes_within_budget_and_equals_alone(f3d, cuda_ok):
    S = _serving(f3d)
    reqs = _small_stream(S)
    sizes = sorted(S.resident_bytes(r, 1) for r in reqs)
    budget = sum(sizes[-3:])  # about three cases at a time: requests wait, join and leave
    srv = S.Server(precision=1, hbm_budget=budget, keep_results=True)
    rep = srv.run(reqs)
    assert rep["completed"] == len(reqs) and rep["rejected"] == 0 and rep["nonfinite"] == 0
    assert rep["peak_resident_bytes"] <= budget
    assert rep["batch_rebuilds"] >= 2  # the batch changed while it ran
    assert max(a for _, a, _ in srv.trace) >= 2  # cases really shared the GPU
    for pr in rep["per_request"]:
        assert pr["admitted"] >= pr["arrival"] and pr["finished"] > pr["first_step"]
    for r in reqs:
        alone = S.Server(precision=1, keep_results=True)
        r0 = S.SolveRequest(**{**r.__dict__, "arrival": 0.0})
        alone.run([r0])
        Qa, ra = alone.results[r.rid]
        Qm, rm = srv.results[r.rid]
        assert np.array_equal(Qa, Qm) and np.array_equal(ra, rm), r


@pytest.mark.gpu
def test_server_rejects_what_never_fits(f3d, cuda_ok):
    S = _serving(f3d)
    reqs = _small_stream(S, count=4, seed=10)
    big = max(reqs, key=lambda r: S.resident_bytes(r, 1))
    budget = S.resident_bytes(big, 1) - 1
    others = [r for r in reqs if r is not big]
    assert all(S.resident_bytes(r, 1) <= budget for r in others)
    rep = S.Server(precision=1, hbm_budget=budget).run(reqs)
    assert rep["rejected"] == 1 and rep["completed"] == len(reqs) - 1


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [(0, 1e-12), (1, 1e-5)])
def test_served_results_match_oracle(f3d, oracle, cuda_ok, precision, tol):
    """Each served result against the FP64 oracle run from the same (device-built) initial
    state: FP64 within 1e-12, mixed within 1e-5 relative L2 in ρ, ρu, ρE."""
    S = _serving(f3d)
    reqs = _small_stream(S, count=3, seed=11)
    srv = S.Server(precision=precision, keep_results=True)
    rep = srv.run(reqs)
    assert rep["completed"] == 3
    I = oracle.interior
    for r in reqs:
        host = S.case_to_host(S.build_request_case(r, "cuda"))
        oc = oracle.OracleCase(host)
        for _ in range(r.steps):
            oc.step()
        Q, _ = srv.results[r.rid]
        U, Uo = _conserved(Q), _conserved(oc.Q)
        mom = np.linalg.norm(I(Uo[1:4]).ravel())
        for k in range(5):
            ref = I(Uo[k])
            scale = mom if 1 <= k <= 3 else np.linalg.norm(ref.ravel())
            err = np.linalg.norm((I(U[k]) - ref).ravel()) / scale
            assert err <= tol, (r.rid, k, err)


@pytest.mark.gpu
def test_fifo_baseline_matches_server_fp64(f3d, cuda_ok):
    S = _serving(f3d)
    reqs = _small_stream(S, count=3, seed=12)
    base = S.fifo(reqs, precision=0, keep_results=True)
    srv = S.Server(precision=0, keep_results=True)
    rep = srv.run(reqs)
    assert base["completed"] == rep["completed"] == 3
    for r in reqs:
        Qf, rf = base["results"][r.rid]
        Qs, rs = srv.results[r.rid]
        assert np.array_equal(Qf, Qs) and np.array_equal(rf, rs)


def test_route_balances_and_keeps_order(f3d):
    S = _serving(f3d)
    reqs = S.request_stream(200, seed=21)
    parts = S.route(reqs, 4)
    got = sorted(r.rid for p in parts for r in p)
    assert got == [r.rid for r in reqs]                       # each request exactly once
    for p in parts:
        assert [r.arrival for r in p] == sorted(r.arrival for r in p)
    loads = [sum(r.cell_stages for r in p) for p in parts]
    assert max(loads) - min(loads) <= max(r.cell_stages for r in reqs)  # greedy bound
    assert S.route(reqs, 4) == parts                          # deterministic
    assert S.route(reqs, 1) == [sorted(reqs, key=lambda r: r.arrival)]


@pytest.mark.gpu
def test_multiserver_on_one_gpu_equals_server(f3d, cuda_ok):
    S = _serving(f3d)
    reqs = _small_stream(S, count=4, seed=14)
    ms = S.MultiServer(["cuda:0"], precision=1, keep_results=True)
    rep = ms.run(reqs)
    assert rep["completed"] == 4 and rep["replicas"] == 1
    alone = S.Server(precision=1, keep_results=True)
    alone.run(reqs)
    for r in reqs:
        for a, b in zip(ms.servers[0].results[r.rid], alone.results[r.rid]):
            assert np.array_equal(a, b)
