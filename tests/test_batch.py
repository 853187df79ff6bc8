"""Batched stages (flame_batch_*): parity with the oracle, alone-vs-mix equality, graph replay."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mix(f3d):
    return [f3d.taylor_green(n=16),
            f3d.random_curvilinear(n=12, ns=2, seed=51),
            f3d.random_curvilinear(n=10, ns=1, seed=52),
            f3d.taylor_green(n=12, ns=3, perturb=0.02, seed=53),
            f3d.curvilinear_jet(nx=24, ny=16, nz=12, pressure_noise=0.02)]


def _state(dc):
    U = dc.conserved()
    Q, r = dc.primitives()
    return U, Q, r


MODES = ["persistent", "graph", "hybrid"]


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("precision", [0, 1])
def test_batch_matches_oracle(f3d, oracle, cuda_ok, precision, mode):
    S = f3d.solver_module()
    B = f3d.batch_module()
    cases = _mix(f3d)
    dcs = [S.DeviceCase(c, precision=precision, tile=3) for c in cases]
    batch = B.Batch(dcs, mode=mode)
    ocs = [oracle.OracleCase(c) for c in cases]
    for _ in range(2):
        batch.step()
        for oc in ocs:
            oc.step()
    tol = 1e-12 if precision == 0 else 1e-5
    I = oracle.interior
    for dc, oc, c in zip(dcs, ocs, cases):
        U = dc.conserved()
        mom = np.linalg.norm(I(oc.U[1:4]).ravel())
        for n in range(5):
            ref = I(oc.U[n])
            scale = mom if 1 <= n <= 3 else np.linalg.norm(ref.ravel())
            err = np.linalg.norm((I(U[n]) - ref).ravel()) / scale
            assert err <= tol, (c.name, n, err)
    batch.close()


@pytest.mark.parametrize("mode", MODES)
def test_alone_equals_in_mix_bitwise(f3d, cuda_ok, mode):
    """A case's result does not depend on the other cases of its batch."""
    S = f3d.solver_module()
    B = f3d.batch_module()
    cases = _mix(f3d)
    alone = S.DeviceCase(cases[1], precision=1, tile=3)
    b1 = B.Batch([alone], mode=mode)
    mixed = [S.DeviceCase(c, precision=1, tile=3) for c in cases]
    b2 = B.Batch(mixed, mode=mode)
    b2.capture()
    for _ in range(3):
        b1.step()
        b2.step()
    for a, m in zip(_state(alone), _state(mixed[1])):
        assert np.array_equal(a, m)
    b1.close()
    b2.close()


@pytest.mark.parametrize("mode", MODES)
def test_graph_replay_equals_launches(f3d, cuda_ok, mode):
    S = f3d.solver_module()
    B = f3d.batch_module()
    cases = _mix(f3d)
    d1 = [S.DeviceCase(c, tile=3) for c in cases]
    d2 = [S.DeviceCase(c, tile=3) for c in cases]
    b1, b2 = B.Batch(d1, mode=mode), B.Batch(d2, mode=mode)
    b1.stage(1)  # a single stage first, so the graphs start from the odd parity
    b2.stage(1)
    b2.capture()
    for _ in range(3):  # both parities of the captured graphs
        b1.step()
        b2.step()
    for x, y in zip(d1, d2):
        for a, b in zip(_state(x), _state(y)):
            assert np.array_equal(a, b)
    b1.close()
    b2.close()


def test_batch_agrees_with_single_case_path(f3d, cuda_ok):
    S = f3d.solver_module()
    B = f3d.batch_module()
    case = f3d.random_curvilinear(n=12, ns=3, seed=54)
    single = S.DeviceCase(case, tile=3)
    batched = S.DeviceCase(case, tile=3)
    b = B.Batch([batched])
    single.step()
    b.step()
    for a, c in zip(_state(single), _state(batched)):
        n = np.linalg.norm(a.ravel())
        assert np.linalg.norm((a - c).ravel()) <= 1e-13 * n
    b.close()


def test_graph_batch_with_mixed_configurations(f3d, cuda_ok):
    """Autotuned cases each keep their own configuration inside one graph-mode batch; every
    case ends bit for bit where it ends when run alone with that configuration."""
    S = f3d.solver_module()
    B = f3d.batch_module()
    cases = _mix(f3d)
    tiles = [0, 3, 4, 5, 6]
    batched = [S.DeviceCase(c, precision=1, tile=t) for c, t in zip(cases, tiles)]
    alone = [S.DeviceCase(c, precision=1, tile=t) for c, t in zip(cases, tiles)]
    b = B.Batch(batched, mode="graph")
    b.capture()
    for _ in range(2):
        b.step()
        for dc in alone:
            dc.step()
    for x, y in zip(batched, alone):
        for a, c in zip(_state(x), _state(y)):
            assert np.array_equal(a, c)
    b.close()


def _law2(f3d, ns, seed, n=12):
    case = f3d.random_curvilinear(n=n, ns=ns, seed=seed)
    case.transport = f3d.cases.mixture_averaged_transport(case.thermo, seed=seed)
    return case


@pytest.mark.parametrize("mode", MODES)
def test_batch_with_law2_cases(f3d, cuda_ok, mode):
    """Cases with mixture-averaged transport (law 2, configuration 6's shape: flow and species
    sweeps, the x sweep, the finish with the mixture rule) batched with law-1 cases of the same
    and other species counts: each law-2 case ends bit for bit where it ends alone in a batch
    of its own, and (the persistent launches being other kernels than the stand-alone ones)
    within 1e-12 of the stand-alone stage."""
    S = f3d.solver_module()
    B = f3d.batch_module()
    law2 = [_law2(f3d, 4, 55), _law2(f3d, 2, 56, n=10)]
    cases = _mix(f3d)[:3] + law2 + [f3d.random_curvilinear(n=10, ns=4, seed=58)]
    batched = [S.DeviceCase(c, tile=3) for c in cases]
    solo = [S.DeviceCase(c, tile=3) for c in law2]
    ref = [S.DeviceCase(c, tile=3) for c in law2]
    b = B.Batch(batched, mode=mode)
    b.capture()
    b1 = [B.Batch([dc], mode=mode) for dc in solo]
    for _ in range(2):
        b.step()
        for x in b1:
            x.step()
        for dc in ref:
            dc.step()
    b.status()
    for k, (alone, r) in enumerate(zip(solo, ref)):
        mixed = batched[3 + k]
        for a, m in zip(_state(alone), _state(mixed)):
            assert np.array_equal(a, m), (mode, law2[k].name)
        for a, c in zip(_state(mixed), _state(r)):
            for f in range(a.shape[0]):
                n = np.linalg.norm(c[f].ravel())
                assert np.linalg.norm((a[f] - c[f]).ravel()) <= 1e-12 * n, (mode, law2[k].name, f)
    b.close()
    for x in b1:
        x.close()


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("ns", [2, 5, 9])
def test_persistent_law2_matches_oracle(f3d, oracle, cuda_ok, ns, precision):
    """The persistent law-2 launches over two RK3 steps against the oracle: 1e-12 relative L2
    per field (partial densities included) in FP64, 1e-5 on the conserved fields in mixed
    precision."""
    S = f3d.solver_module()
    B = f3d.batch_module()
    case = _law2(f3d, ns, 60 + ns)
    dc = S.DeviceCase(case, precision=precision, tile=3)
    b = B.Batch([dc], mode="persistent")
    oc = oracle.OracleCase(case)
    for _ in range(2):
        b.step()
        oc.step()
    b.status()
    I = oracle.interior
    U = dc.conserved()
    mom = np.linalg.norm(I(oc.U[1:4]).ravel())
    tol = 1e-12 if precision == 0 else 1e-5
    for n in range(5):
        ref = I(oc.U[n])
        scale = mom if 1 <= n <= 3 else np.linalg.norm(ref.ravel())
        assert np.linalg.norm((I(U[n]) - ref).ravel()) / scale <= tol, (n, precision)
    if precision == 0:
        _, r = dc.primitives()
        assert oracle.rel_l2(I(r), I(oc.rhoi)) <= tol
    b.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_persistent_batch_agrees_with_configuration_3(f3d, cuda_ok, precision):
    """The persistent kernels run configuration 3's prep, z, y and finishing x blocks from one
    work list; each case ends where the stand-alone configuration 3 puts it, up to the
    compiler's multiply-add contraction in a different kernel (1e-12 FP64, 1e-6 FP32, relative
    L2 per field; species counts 1-6)."""
    S = f3d.solver_module()
    B = f3d.batch_module()
    cases = _mix(f3d) + [f3d.taylor_green(n=12, ns=5, perturb=0.02, seed=56),
                         f3d.random_curvilinear(n=10, ns=6, seed=57)]
    batched = [S.DeviceCase(c, precision=precision, tile=3) for c in cases]
    alone = [S.DeviceCase(c, precision=precision, tile=3) for c in cases]
    b = B.Batch(batched, mode="persistent")
    b.capture()
    for _ in range(2):
        b.step()
        for dc in alone:
            dc.step()
    b.status()
    tol = 1e-12 if precision == 0 else 1e-6
    for x, y in zip(batched, alone):
        for a, c in zip(_state(x), _state(y)):
            for k in range(a.shape[0]):
                n = np.linalg.norm(c[k].ravel())
                assert np.linalg.norm((a[k] - c[k]).ravel()) <= tol * n, (x.case.name, k)
    b.close()


def test_persistent_batch_more_cases_than_one_chunk(f3d, cuda_ok):
    """More cases of one species count than the constant descriptor table holds (20): the
    batch runs them in chunks, and every case agrees with its stand-alone run."""
    S = f3d.solver_module()
    B = f3d.batch_module()
    cases = [f3d.taylor_green(n=8 + (i % 5), perturb=0.02, seed=100 + i) for i in range(23)]
    batched = [S.DeviceCase(c, tile=3) for c in cases]
    alone = [S.DeviceCase(c, tile=3) for c in cases]
    b = B.Batch(batched, mode="persistent")
    b.step()
    b.status()
    for dc in alone:
        dc.step()
    for x, y in zip(batched, alone):
        U, V = x.conserved(), y.conserved()
        assert np.linalg.norm((U - V).ravel()) <= 1e-12 * np.linalg.norm(V.ravel())
    b.close()


def test_persistent_wait_runs_out_and_reports(f3d, cuda_ok):
    """A completion that never comes (flame_batch_test_stall): the waits give up after their
    bound, the stage returns, flame_batch_status reports FLAME_ETIMEOUT once, and the batch and
    the GPU stay usable; nothing faults or hangs.  A law-2 case gives the batch a chunk of
    four launches too."""
    S = f3d.solver_module()
    B = f3d.batch_module()
    cases = _mix(f3d)[:3] + [_law2(f3d, 3, 61, n=10)]
    dcs = [S.DeviceCase(c, tile=3) for c in cases]
    b = B.Batch(dcs, mode="persistent")
    f3d.abi.check(b.lib, b.lib.flame_batch_test_stall(b.handle, 1))
    b.step()
    with pytest.raises(f3d.abi.FlameError) as e:
        b.status()
    assert e.value.code == 3
    b.status()  # reported once
    f3d.abi.check(b.lib, b.lib.flame_batch_test_stall(b.handle, 0))
    fresh = [S.DeviceCase(c, tile=3) for c in cases]
    alone = [S.DeviceCase(c, tile=3) for c in cases]
    b2 = B.Batch(fresh, mode="persistent")
    b2.step()
    b2.status()
    for dc in alone:
        dc.step()
    for x, y in zip(fresh, alone):
        for a, c in zip(_state(x), _state(y)):
            for k in range(a.shape[0]):
                n = np.linalg.norm(c[k].ravel())
                assert np.linalg.norm((a[k] - c[k]).ravel()) <= 1e-12 * n
    b.close()
    b2.close()


def test_hybrid_batch_splits_the_cases(f3d, oracle, cuda_ok):
    """Hybrid mode with the size limit between the mix's cases: the cases of at most 12^3
    cells run in the persistent part, the others in the graph part, both in one CUDA graph per
    step.  After two captured steps every case is within 1e-12 of the oracle, and the graph
    part's cases are bit for bit where they end when run alone."""
    S = f3d.solver_module()
    B = f3d.batch_module()
    cases = _mix(f3d)
    dcs = [S.DeviceCase(c, tile=3) for c in cases]
    b = B.Batch(dcs, mode="hybrid", small_cells=12 ** 3)
    assert [p.mode for p in b.parts] == ["persistent", "graph"]
    big = [dc for dc in b.parts[1].cases]
    assert all(dc.case.cells > 12 ** 3 for dc in big)
    assert all(dc.case.cells <= 12 ** 3 for dc in b.parts[0].cases)
    alone = {id(dc): S.DeviceCase(dc.case, tile=3) for dc in big}
    ocs = [oracle.OracleCase(c) for c in cases]
    b.capture()
    for _ in range(2):
        b.step()
        for oc in ocs:
            oc.step()
        for a in alone.values():
            a.step()
    b.status()
    I = oracle.interior
    for dc, oc, c in zip(dcs, ocs, cases):
        U = dc.conserved()
        mom = np.linalg.norm(I(oc.U[1:4]).ravel())
        for n in range(5):
            ref = I(oc.U[n])
            scale = mom if 1 <= n <= 3 else np.linalg.norm(ref.ravel())
            assert np.linalg.norm((I(U[n]) - ref).ravel()) / scale <= 1e-12, (c.name, n)
    for dc in big:
        for x, y in zip(_state(dc), _state(alone[id(dc)])):
            assert np.array_equal(x, y), dc.case.name
    b.close()
