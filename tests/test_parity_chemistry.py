"""GPU parity of the finite-rate chemistry step (reactions.jl eval_gpu / eval_gpu_stiff) with the
oracle on a seeded synthetic mechanism.  The kernels are strict IEEE like the other 1:1 kernels;
exp, log, log10 and pow come from the device and the host math libraries, hence 1e-12."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("stiff,transposed,dt", [(0, 0, 1e-9), (1, 0, 1e-7), (1, 1, 1e-7)])
def test_chemistry_step_matches_oracle(f3d, oracle, cuda_ok, stiff, transposed, dt):
    import importlib

    import torch
    M = importlib.import_module(f3d.__name__ + ".mechanism")
    mech = M.synthetic_mechanism()
    case = f3d.random_curvilinear(n=10, ns=8, seed=7, T_range=(400.0, 2600.0))
    Q, r = M.reacting_state(mech, case)
    U = np.ascontiguousarray(case.U())
    th = mech.thermo.to_c()
    arrays, rc = mech.to_device()
    dU, dQ, dr = (torch.from_numpy(a.copy()).cuda() for a in (U, Q, r))
    lib = f3d.load_library()
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    g = case.grid()
    if stiff:
        rc_ = lib.flame_eval_gpu_stiff(C.byref(g), s, dU.data_ptr(), dQ.data_ptr(), dr.data_ptr(),
                                       dt, C.byref(th), C.byref(rc), None, 500.0, transposed)
    else:
        rc_ = lib.flame_eval_gpu(C.byref(g), s, dU.data_ptr(), dQ.data_ptr(), dr.data_ptr(), dt,
                                 C.byref(th), C.byref(rc), None, 500.0)
    f3d.abi.check(lib, rc_)
    torch.cuda.synchronize()
    oracle.load().oracle_eval_chem(C.byref(g), stiff, oracle.ptr(U), oracle.ptr(Q), oracle.ptr(r),
                                   dt, C.byref(th), C.byref(mech.to_c()), None, 500.0, transposed)
    assert not np.array_equal(r, M.reacting_state(mech, case)[1])  # something reacted
    for d, h in ((dU, U), (dQ, Q), (dr, r)):
        got = d.cpu().numpy()
        np.testing.assert_allclose(got, h, rtol=1e-12, atol=1e-12 * np.abs(h).max())


def test_chemistry_rejects_bad_mechanism(f3d, cuda_ok):
    lib = f3d.load_library()
    g = f3d.FlameGrid(8, 8, 8, 4, 8, 7)
    rc = f3d.abi.FlameReactions()
    rc.nreacs = 0
    rc_ = lib.flame_eval_gpu(C.byref(g), None, C.c_void_p(1), C.c_void_p(1), C.c_void_p(1), 1e-9,
                             C.byref(f3d.FlameThermo()), C.byref(rc), None, 500.0)
    assert rc_ == 1  # NULL arrays
