"""Parity of every 1:1 kernel with the oracle on the GPU, through the C ABI.

The 1:1 kernels are built with -fmad=false, so apart from pow() in the transport law they must
agree with the strict-IEEE oracle bit for bit.  Inputs are seeded random curvilinear fields
whose pressure jumps put faces in all three hybrid branches."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


_KEEP: list = []


def _t(a):
    """Device copy of a host array.  The tensor is kept alive until the next test so its
    memory cannot be recycled by the caching allocator while a launch still reads it."""
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    _KEEP.append(t)
    return t


@pytest.fixture(autouse=True)
def _release():
    yield
    _KEEP.clear()


def _np(t):
    return t.cpu().numpy()


class Env:
    def __init__(self, f3d, oracle, ns, seed):
        import torch
        self.torch = torch
        self.f3d, self.o = f3d, oracle
        self.case = f3d.random_curvilinear(n=12, ns=ns, seed=seed)
        self.g = self.case.grid()
        self.lib = f3d.load_library()
        self.olib = oracle.load()
        self.th = self.case.thermo.to_c()
        self.tr = self.case.transport.to_c()
        self.m = {k: np.ascontiguousarray(v) for k, v in self.case.metrics.items()}
        self.dm = {k: _t(v) for k, v in self.m.items()}
        self.cm_host = oracle.metrics_struct(self.m)
        self.cm_dev = f3d.FlameMetrics(**{k: v.data_ptr() for k, v in self.dm.items()})
        self.Q = np.ascontiguousarray(self.case.Q)
        self.rhoi = np.ascontiguousarray(self.case.rhoi)
        self.shape = self.Q.shape[1:]
        self.ns = ns
        c = self.case
        self.fshape = [(c.nz, c.ny, c.nx + 1), (c.nz, c.ny + 1, c.nx), (c.nz + 1, c.ny, c.nx)]

    def gcall(self, name, *args):
        rc = getattr(self.lib, name)(C.byref(self.g), None, *args)
        self.f3d.abi.check(self.lib, rc)
        self.torch.cuda.synchronize()

    def ocall(self, name, *args):
        getattr(self.olib, name)(C.byref(self.g), *args)


def P(x):
    return x.data_ptr() if hasattr(x, "data_ptr") else x.ctypes.data


@pytest.fixture(scope="module", params=[(1, 31), (3, 32)], ids=["ns1", "ns3"])
def env(request, f3d, oracle, cuda_ok):
    return Env(f3d, oracle, *request.param)


def exact(a, b):
    assert a.shape == b.shape
    if not np.array_equal(a, b):
        d = np.abs(a - b)
        i = np.unravel_index(np.argmax(d), d.shape)
        raise AssertionError(f"max |diff| {d.max():.3e} at {i}: {a[i]!r} vs {b[i]!r}")


def test_shock_sensor(env):
    phi_h = np.zeros(env.shape)
    env.ocall("oracle_shockSensor", P(phi_h), P(env.Q))
    phi_d = _t(np.zeros(env.shape))
    env.gcall("flame_shockSensor", P(phi_d), P(_t(env.Q)))
    exact(_np(phi_d), phi_h)
    # the random case exercises all three hybrid branches
    inner = phi_h[3:-3, 3:-3, 3:-3]
    assert (inner < 1e-3).any() and ((inner >= 1e-3) & (inner < 0.1)).any() and (inner >= 0.1).any()


@pytest.mark.parametrize("d", [0, 1, 2])
def test_flux_split_and_species_split(env, d):
    A = [("dxidx", "dxidy", "dxidz"), ("detadx", "detady", "detadz"),
         ("dzetadx", "dzetady", "dzetadz")][d]
    Fp_h, Fm_h = np.zeros((5,) + env.shape), np.zeros((5,) + env.shape)
    env.ocall("oracle_fluxSplit", P(env.Q), P(Fp_h), P(Fm_h), *[P(env.m[a]) for a in A], None)
    Fp_d, Fm_d = _t(np.zeros((5,) + env.shape)), _t(np.zeros((5,) + env.shape))
    env.gcall("flame_fluxSplit", P(_t(env.Q)), P(Fp_d), P(Fm_d), *[P(env.dm[a]) for a in A], None)
    exact(_np(Fp_d), Fp_h)
    exact(_np(Fm_d), Fm_h)
    ns = env.ns
    Sp_h, Sm_h = np.zeros((ns,) + env.shape), np.zeros((ns,) + env.shape)
    env.ocall("oracle_split", P(env.rhoi), P(env.Q), P(Sp_h), P(Sm_h), *[P(env.m[a]) for a in A],
              None)
    Sp_d, Sm_d = _t(np.zeros((ns,) + env.shape)), _t(np.zeros((ns,) + env.shape))
    env.gcall("flame_split", P(_t(env.rhoi)), P(_t(env.Q)), P(Sp_d), P(Sm_d),
              *[P(env.dm[a]) for a in A], None)
    exact(_np(Sp_d), Sp_h)
    exact(_np(Sm_d), Sm_h)


@pytest.mark.parametrize("d", [0, 1, 2])
def test_weno_hybrid(env, d):
    rng = np.random.default_rng(d)
    NV = 5
    Fp = np.ascontiguousarray(rng.normal(size=(NV,) + env.shape))
    Fm = np.ascontiguousarray(rng.normal(size=(NV,) + env.shape))
    # sensor values spread over the three branches, including exact thresholds
    phi = np.ascontiguousarray(rng.choice([0.0, 5e-4, 1e-3, 0.05, 0.1, 0.3], size=env.shape))
    F_h = np.zeros((NV,) + env.fshape[d])
    env.olib.oracle_WENO(C.byref(env.g), d, P(F_h), P(phi), P(Fp), P(Fm), NV, None)
    F_d = _t(np.zeros((NV,) + env.fshape[d]))
    env.gcall(["flame_WENO_x", "flame_WENO_y", "flame_WENO_z"][d], P(F_d), P(_t(phi)),
              P(_t(Fp)), P(_t(Fm)), NV, None)
    exact(_np(F_d), F_h)


def _mixture(env):
    ns = env.ns
    Yi, D = np.zeros((ns,) + env.shape), np.zeros((ns,) + env.shape)
    lam, mu = np.zeros(env.shape), np.zeros(env.shape)
    env.ocall("oracle_mixture", P(env.Q), P(env.rhoi), P(Yi), P(lam), P(mu), P(D),
              C.byref(env.th), C.byref(env.tr), None)
    return Yi, lam, mu, D


def test_mixture(env):
    Yi, lam, mu, D = _mixture(env)
    ns = env.ns
    d = {k: _t(np.zeros(v.shape)) for k, v in dict(Yi=Yi, lam=lam, mu=mu, D=D).items()}
    env.gcall("flame_mixture", P(_t(env.Q)), P(_t(env.rhoi)), P(d["Yi"]), P(d["lam"]),
              P(d["mu"]), P(d["D"]), C.byref(env.th), C.byref(env.tr), None)
    exact(_np(d["Yi"]), Yi)
    # pow() differs between libm and CUDA by at most an ulp or two
    for k, ref in (("lam", lam), ("mu", mu), ("D", D)):
        np.testing.assert_allclose(_np(d[k]), ref, rtol=1e-15, atol=0)
    assert ns == Yi.shape[0]


@pytest.mark.parametrize("d", [0, 1, 2])
def test_viscous_and_species_diffusion(env, d):
    Yi, lam, mu, D = _mixture(env)
    ns = env.ns
    fs = env.fshape[d]
    Fd_h, Fh_h = np.zeros((ns,) + fs), np.zeros((3,) + fs)
    env.olib.oracle_specViscousFlux(C.byref(env.g), d, P(Fd_h), P(env.Q), P(Yi),
                                    C.byref(env.cm_host), P(D), P(Fh_h), C.byref(env.th), None)
    Fd_d, Fh_d = _t(np.zeros((ns,) + fs)), _t(np.zeros((3,) + fs))
    sfx = "xyz"[d]
    # the reference's argument list: the nine metric cofactors and J one by one
    env.gcall(f"flame_specViscousFlux_{sfx}", P(Fd_d), P(_t(env.Q)), P(_t(Yi)),
              *env.cm_dev.args(), P(_t(D)), P(Fh_d), C.byref(env.th), None)
    exact(_np(Fd_d), Fd_h)
    exact(_np(Fh_d), Fh_h)
    Fv_h = np.zeros((4,) + fs)
    env.olib.oracle_viscousFlux(C.byref(env.g), d, P(Fv_h), P(env.Q), C.byref(env.cm_host),
                                P(lam), P(mu), P(Fh_h), None)
    Fv_d = _t(np.zeros((4,) + fs))
    env.gcall(f"flame_viscousFlux_{sfx}", P(Fv_d), P(_t(env.Q)), *env.cm_dev.args(),
              P(_t(lam)), P(_t(mu)), P(Fh_d), None)
    exact(_np(Fv_d), Fv_h)


def test_div_divspecs_lincomb_c2prim(env):
    rng = np.random.default_rng(7)
    ns = env.ns
    U = np.ascontiguousarray(env.case.U())
    F = [np.ascontiguousarray(rng.normal(size=(5,) + s)) for s in env.fshape]
    Fv = [np.ascontiguousarray(rng.normal(size=(4,) + s)) for s in env.fshape]
    dt = 1e-3
    U_h = U.copy()
    env.ocall("oracle_div", P(U_h), *[P(a) for a in F], *[P(a) for a in Fv], dt, P(env.m["J"]),
              None)
    U_d = _t(U)
    env.gcall("flame_div", P(U_d), *[P(_t(a)) for a in F], *[P(_t(a)) for a in Fv], dt,
              P(env.dm["J"]), None)
    exact(_np(U_d), U_h)
    Fs = [np.ascontiguousarray(rng.normal(size=(ns,) + s)) for s in env.fshape]
    Fd = [np.ascontiguousarray(rng.normal(size=(ns,) + s)) for s in env.fshape]
    r_h = env.rhoi.copy()
    env.ocall("oracle_divSpecs", P(r_h), *[P(a) for a in Fs], *[P(a) for a in Fd], dt,
              P(env.m["J"]), None)
    r_d = _t(env.rhoi)
    env.gcall("flame_divSpecs", P(r_d), *[P(_t(a)) for a in Fs], *[P(_t(a)) for a in Fd], dt,
              P(env.dm["J"]), None)
    exact(_np(r_d), r_h)
    Un = np.ascontiguousarray(U * (1 + 1e-3 * rng.normal(size=U.shape)))
    env.ocall("oracle_linComb", P(U_h), P(Un), 5, 0.25, 0.75, None)
    env.gcall("flame_linComb", P(U_d), P(_t(Un)), 5, 0.25, 0.75, None)
    exact(_np(U_d), U_h)
    Q_h, ri_h = env.Q.copy(), env.rhoi.copy()
    env.ocall("oracle_c2Prim", P(U), P(Q_h), P(ri_h), C.byref(env.th), None)
    Q_d, ri_d = _t(env.Q), _t(env.rhoi)
    env.gcall("flame_c2Prim", P(_t(U)), P(Q_d), P(ri_d), C.byref(env.th), None)
    exact(_np(Q_d), Q_h)
    exact(_np(ri_d), ri_h)
    U2_h = np.zeros_like(U)
    env.ocall("oracle_prim2c", P(U2_h), P(env.Q))
    U2_d = _t(np.zeros_like(U))
    env.gcall("flame_prim2c", P(U2_d), P(_t(env.Q)))
    exact(_np(U2_d), U2_h)


def test_fill_periodic(env):
    rng = np.random.default_rng(3)
    A = np.ascontiguousarray(rng.normal(size=(2,) + env.shape))
    A_h = A.copy()
    env.ocall("oracle_fill_periodic", P(A_h), 2)
    A_d = _t(A)
    env.gcall("flame_fill_periodic", P(A_d), 2)
    exact(_np(A_d), A_h)
    c = env.case
    np.testing.assert_array_equal(A_h[:, 4:8, 4:-4, 4:-4], A_h[:, c.nz + 4:c.nz + 8, 4:-4, 4:-4])
