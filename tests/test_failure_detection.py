"""The reference's NaN check (solver.jl:388-391) as flame_check_finite, and the serving loop
stopping a case whose state has gone non-finite.  The failure is planted in the data (a NaN in
an initial state), never in a kernel: nothing here faults or stalls the GPU."""
from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_check_finite_counts(f3d, cuda_ok):
    S = f3d.solver_module()
    dc = S.DeviceCase(f3d.random_curvilinear(n=10, ns=2, seed=81), tile=3)
    assert int(dc.nonfinite_launch().item()) == 0
    dc.check_finite()
    dc.U[0, 5, 5, 5] = float("nan")
    dc.U[4, 6, 7, 8] = float("inf")
    dc.U[2, 0, 0, 0] = float("-inf")   # a ghost point counts too, as in the reference
    assert int(dc.nonfinite_launch().item()) == 3
    with pytest.raises(f3d.FlameError) as e:
        dc.check_finite()
    assert e.value.code == 4


def test_server_stops_a_case_that_goes_nonfinite(f3d, cuda_ok):
    import importlib
    Sv = importlib.import_module(f3d.__name__ + ".serving")
    reqs = Sv.request_stream(4, rate=400.0, seed=13, n_range=(12, 16), steps_range=(8, 10),
                             Ma_range=(0.1, 0.5))
    bad = reqs[1].rid

    def builder(req, device):
        c = Sv.build_request_case(req, device)
        if req.rid == bad:
            c.Q[1, 8, 8, 8] = float("nan")
        return c

    srv = Sv.Server(precision=1, keep_results=True, builder=builder, check_every=2)
    rep = srv.run(reqs)
    recs = {r["rid"]: r for r in rep["per_request"]}
    assert recs[bad]["failed"] is not None and not recs[bad]["finite"]
    assert rep["failed"] == 1 and rep["completed"] == len(reqs) - 1
    assert int(recs[bad]["failed"].split()[-2]) <= 2  # caught at the first check
    for r in reqs:
        if r.rid == bad:
            continue
        assert recs[r.rid]["failed"] is None and recs[r.rid]["finite"]
        alone = Sv.Server(precision=1, keep_results=True)
        alone.run([Sv.SolveRequest(**{**r.__dict__, "arrival": 0.0})])
        for a, b in zip(alone.results[r.rid], srv.results[r.rid]):
            assert np.array_equal(a, b)  # the broken neighbour changed nothing
    assert not math.isnan(recs[bad]["finished"])
