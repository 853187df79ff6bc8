"""Seeded synthetic cases: grids, curvilinear metrics, thermodynamics and initial fields.

Array convention: a field with `nv` variables on a ghosted grid is a C-contiguous numpy array
of shape (nv, Tz, Ty, Tx) (Tx = nx + 2*NG ...), i.e. exactly the memory of the reference's
Julia array of size (Tx, Ty, Tz, nv).

Metrics follow parse_mesh.jl:117-221: the 6th-order central difference CD6 of the coordinates
in index space, J = 1/det, and the J^-1-scaled cofactors dξ/dx ... dζ/dz.  For the periodic
benchmark grids the coordinates are evaluated analytically three cells beyond the interior so
CD6 applies at every interior point, and metric ghosts are exact periodic copies.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .abi import FLAME_NG, FlameGrid, FlameThermo, FlameTransport, METRIC_NAMES

RU = 8.314462618  # J/(mol K)
NG = FLAME_NG


# ----------------------------------------------------------------------------- thermodynamics
@dataclass
class Thermo:
    """NASA-7 species data in the layout of thermoProperty (run.jl:71-82)."""
    mw: np.ndarray          # (ns,) kg/mol
    lo: np.ndarray          # (ns, 7)
    hi: np.ndarray          # (ns, 7)
    sep: np.ndarray         # (ns,) K
    min_temp: float = 200.0
    max_temp: float = 6000.0
    Ru: float = RU

    @property
    def ns(self) -> int:
        return int(self.mw.shape[0])

    def to_c(self) -> FlameThermo:
        t = FlameThermo()
        t.Ru, t.min_temp, t.max_temp, t.ns = self.Ru, self.min_temp, self.max_temp, self.ns
        for n in range(self.ns):
            t.mw[n] = self.mw[n]
            t.coeffs_sep[n] = self.sep[n]
            for a in range(7):
                t.coeffs_lo[a + 7 * n] = self.lo[n, a]
                t.coeffs_hi[a + 7 * n] = self.hi[n, a]
        return t

    def subset(self, ns: int) -> "Thermo":
        return Thermo(self.mw[:ns].copy(), self.lo[:ns].copy(), self.hi[:ns].copy(),
                      self.sep[:ns].copy(), self.min_temp, self.max_temp, self.Ru)

    # Host evaluations with the reference's formulas (thermo.jl), vectorised over points.
    def species_energy(self, T: np.ndarray) -> list[np.ndarray]:
        """Per species e_n(T) R_u^-1 W_n (the polynomial of InternalEnergy, thermo.jl:219-228)."""
        T2 = 0.5 * T * T
        T3 = 2.0 / 3.0 * T2 * T
        T4 = T2 * T2
        T5 = 0.8 * T4 * T
        out = []
        for n in range(self.ns):
            lo, hi = self.lo[n], self.hi[n]
            e_lo = (lo[0] - 1) * T + lo[1] * T2 + lo[2] * T3 + lo[3] * T4 + lo[4] * T5
            e_hi = ((hi[0] - 1) * T + hi[1] * T2 + hi[2] * T3 + hi[3] * T4 + hi[4] * T5
                    + (hi[5] - lo[5]))
            out.append(np.where(T < self.sep[n], e_lo, e_hi))
        return out

    def internal_energy(self, T: np.ndarray, rhoi: np.ndarray) -> np.ndarray:
        """InternalEnergy (thermo.jl:219-228), J/m^3; rhoi has shape (ns, ...)."""
        r = np.zeros_like(T)
        for n, e in enumerate(self.species_energy(T)):
            r = r + rhoi[n] * e / self.mw[n]
        return r * self.Ru

    def cp_mass(self, T: np.ndarray, Y: np.ndarray) -> np.ndarray:
        """Mass-specific mixture cp, J/(kg K)."""
        T2 = T * T
        T3 = T2 * T
        T4 = T2 * T2
        r = np.zeros_like(T)
        for n in range(self.ns):
            lo, hi = self.lo[n], self.hi[n]
            c_lo = lo[0] + lo[1] * T + lo[2] * T2 + lo[3] * T3 + lo[4] * T4
            c_hi = hi[0] + hi[1] * T + hi[2] * T2 + hi[3] * T3 + hi[4] * T4
            r = r + np.where(T < self.sep[n], c_lo, c_hi) * Y[n] / self.mw[n]
        return r * self.Ru

    def pressure(self, T: np.ndarray, rhoi: np.ndarray) -> np.ndarray:
        yow = np.zeros_like(T)
        for n in range(self.ns):
            yow = yow + rhoi[n] / self.mw[n]
        return self.Ru * T * yow


def ideal_air() -> Thermo:
    """One species, W = 28.97 g/mol, cp/R = 3.5 in both ranges, so gamma = 1.4 exactly."""
    lo = np.zeros((1, 7))
    lo[0, 0] = 3.5
    return Thermo(mw=np.array([0.02897]), lo=lo, hi=lo.copy(), sep=np.array([1000.0]),
                  min_temp=200.0, max_temp=6000.0)


def synthetic_species(ns: int = 9, seed: int = 3) -> Thermo:
    """Seeded synthetic species: W ~ U[2, 32] g/mol; single-range NASA-7 with
    a1 ~ U[2.5, 3.5], a2 ~ U[0, (5 - a1)/3000], a3..a5 = 0, a6 ~ U[-1e3, 1e3], a7 = 0, so
    cp/R stays within [2.5, 5.0] over 200-3000 K."""
    rng = np.random.default_rng(seed)
    mw = rng.uniform(2.0, 32.0, ns) * 1e-3
    lo = np.zeros((ns, 7))
    lo[:, 0] = rng.uniform(2.5, 3.5, ns)
    lo[:, 1] = rng.uniform(0.0, 1.0, ns) * (5.0 - lo[:, 0]) / 3000.0
    lo[:, 5] = rng.uniform(-1e3, 1e3, ns)
    return Thermo(mw=mw, lo=lo, hi=lo.copy(), sep=np.full(ns, 1000.0), min_temp=200.0,
                  max_temp=3000.0)


@dataclass
class Transport:
    """law 0: constants; law 1: mu = mu_ref (T/T_ref)^exponent, lambda = cp mu / Pr,
    D = lambda / (rho cp) (unity Lewis); law 2: the reference's mixture-averaged properties
    (thermo.jl:289-369) from the log(T) fits in `poly` (visc (5, ns) | conduct (5, ns) |
    binarydiff (5, ns, ns), each column-major, flattened back to back)."""
    law: int = 1
    mu_ref: float = 1.8e-5
    T_ref: float = 300.0
    exponent: float = 0.7
    Pr: float = 0.71
    lambda_ref: float = 0.0
    D_ref: float = 0.0
    poly: np.ndarray | None = None

    def to_c(self, poly_ptr: int | None = None) -> FlameTransport:
        """The C struct; for law 2 `poly_ptr` is the address of `poly` where the callee reads
        it (a device copy for the GPU, the host array for the oracle)."""
        t = FlameTransport()
        t.law, t.mu_ref, t.T_ref, t.exponent = self.law, self.mu_ref, self.T_ref, self.exponent
        t.Pr, t.lambda_ref, t.D_ref = self.Pr, self.lambda_ref, self.D_ref
        if self.law == 2:
            if poly_ptr is None:
                poly_ptr = self.poly.ctypes.data  # host: the array itself
            t.poly = poly_ptr
        return t


def _fit_log_poly(T: np.ndarray, f: np.ndarray) -> np.ndarray:
    """Least-squares quartic in ln T, coefficients in ascending order (dot5, thermo.jl:284)."""
    return np.polynomial.polynomial.polyfit(np.log(T), f, 4)


def mixture_averaged_transport(thermo: Thermo, seed: int = 9) -> Transport:
    """Seeded log(T) fits in the form initThermo takes from Cantera (thermo.jl:405-436), for law
    2.  Per species μ_k = μ0_k (T/300)^0.7, μ0_k ~ U[1, 3]·1e-5 Pa s, fitted as sqrt(μ/√T);
    λ_k = λ0_k (T/300)^0.8, λ0_k ~ U[0.02, 0.2] W/(m K), fitted as λ/√T; binary diffusion
    P·D_jk = d_jk (T/300)^1.75, d_jk = d_kj ~ U[1, 4] Pa m²/s, fitted as P·D/T^1.5; all over
    200-3000 K."""
    ns = thermo.ns
    rng = np.random.default_rng(seed)
    T = np.linspace(200.0, 3000.0, 64)
    visc = np.zeros((ns, 5))
    cond = np.zeros((ns, 5))
    binc = np.zeros((ns, ns, 5))
    mu0 = rng.uniform(1e-5, 3e-5, ns)
    lam0 = rng.uniform(0.02, 0.2, ns)
    d0 = rng.uniform(1.0, 4.0, (ns, ns))
    d0 = 0.5 * (d0 + d0.T)
    for k in range(ns):
        mu = mu0[k] * (T / 300.0) ** 0.7
        visc[k] = _fit_log_poly(T, np.sqrt(mu / np.sqrt(T)))
        cond[k] = _fit_log_poly(T, lam0[k] * (T / 300.0) ** 0.8 / np.sqrt(T))
        for j in range(ns):
            binc[k, j] = _fit_log_poly(T, d0[j, k] * (T / 300.0) ** 1.75 / T ** 1.5)
    # column-major (5, ns) and (5, ns, ns): coefficient fastest, then the first species index
    poly = np.concatenate([visc.ravel(), cond.ravel(), binc.ravel()])
    return Transport(law=2, poly=np.ascontiguousarray(poly))


# ------------------------------------------------------------------------------------- grids
def ghosted(nx: int, ny: int, nz: int) -> tuple[int, int, int]:
    return nx + 2 * NG, ny + 2 * NG, nz + 2 * NG


def reference_inflow(ns: int):
    """The inflow state fill_x / fill_z hard-code (boundary.jl:17-25, 96-104): P = 79.8 Pa,
    T = 270.65 K, u = 1000 m/s, v = w = 0, Y(2) = 0.233 and Y(5) = 0.767 (1-based species
    indices, so ns >= 5), every other mass fraction zero."""
    from .abi import FlameInflow
    if ns < 5:
        raise ValueError("the reference inflow sets species 2 and 5: ns >= 5")
    f = FlameInflow()
    f.P, f.T, f.u, f.v, f.w = 79.8, 270.65, 1000.0, 0.0, 0.0
    f.Y[1], f.Y[4] = 0.233, 0.767
    return f


def periodic_fill(a: np.ndarray, nx: int, ny: int, nz: int) -> np.ndarray:
    """Copies every ghost of a (nv, Tz, Ty, Tx) array from its periodic image, in place
    (axis by axis, so edges and corners come from the images already filled)."""
    for ax, n in ((3, nx), (2, ny), (1, nz)):
        def sl(lo, hi):
            idx = [slice(None)] * 4
            idx[ax] = slice(lo, hi)
            return tuple(idx)
        a[sl(0, NG)] = a[sl(n, n + NG)]
        a[sl(n + NG, n + 2 * NG)] = a[sl(NG, 2 * NG)]
    return a


def _cd6(f: np.ndarray, axis: int, n: int) -> np.ndarray:
    """CD6 (parse_mesh.jl:117-120) at interior points of an array extended by 3 on `axis`."""
    def s(o):
        sl = [slice(None)] * f.ndim
        sl[axis] = slice(3 + o, 3 + o + n)
        return f[tuple(sl)]
    return 1 / 60 * (s(3) - s(-3)) - 3 / 20 * (s(2) - s(-2)) + 3 / 4 * (s(1) - s(-1))


def _sin(x):
    """np.sin for numpy arrays, torch.sin for torch tensors (the mappings serve both)."""
    return np.sin(x) if isinstance(x, (np.ndarray, float)) else x.sin()


def _array_ops(device):
    """(arange, meshgrid, zeros) in float64: numpy when `device` is None, else torch on it."""
    if device is None:
        return (lambda a, b: np.arange(a, b, dtype=np.float64), np.meshgrid,
                lambda s: np.zeros(s))
    import torch
    return (lambda a, b: torch.arange(a, b, dtype=torch.float64, device=device), torch.meshgrid,
            lambda s: torch.zeros(s, dtype=torch.float64, device=device))


def metrics_from_mapping(xyz, nx: int, ny: int, nz: int, device=None) -> dict:
    """Metrics of a periodic-in-index mapping; xyz(i, j, k) -> (x, y, z) for index arrays.

    Returns the ten ghosted (Tz, Ty, Tx) arrays named as in FlameMetrics: numpy arrays, or
    torch tensors built on `device` when one is given (same operations in the same order)."""
    arange, meshgrid, zeros = _array_ops(device)
    e = 3
    der = {}
    for ax, n in enumerate((nx, ny, nz)):
        # coordinates extended by 3 along this axis only, interior along the other two
        ii = arange(-e, nx + e) if ax == 0 else arange(0, nx)
        jj = arange(-e, ny + e) if ax == 1 else arange(0, ny)
        kk = arange(-e, nz + e) if ax == 2 else arange(0, nz)
        K, J, I = meshgrid(kk, jj, ii, indexing="ij")
        X, Y, Z = xyz(I, J, K)
        npax = 2 - ax  # numpy axis of i/j/k
        der["x", ax] = _cd6(X, npax, n)
        der["y", ax] = _cd6(Y, npax, n)
        der["z", ax] = _cd6(Z, npax, n)
    dxdxi, dxdeta, dxdzeta = der["x", 0], der["x", 1], der["x", 2]
    dydxi, dydeta, dydzeta = der["y", 0], der["y", 1], der["y", 2]
    dzdxi, dzdeta, dzdzeta = der["z", 0], der["z", 1], der["z", 2]
    # parse_mesh.jl:210-221
    Jm = 1 / (dxdxi * (dydeta * dzdzeta - dydzeta * dzdeta)
              - dxdeta * (dydxi * dzdzeta - dydzeta * dzdxi)
              + dxdzeta * (dydxi * dzdeta - dydeta * dzdxi))
    vals = {
        "dxidx": dydeta * dzdzeta - dydzeta * dzdeta,
        "dxidy": dxdzeta * dzdeta - dxdeta * dzdzeta,
        "dxidz": dxdeta * dydzeta - dxdzeta * dydeta,
        "detadx": dydzeta * dzdxi - dydxi * dzdzeta,
        "detady": dxdxi * dzdzeta - dxdzeta * dzdxi,
        "detadz": dxdzeta * dydxi - dxdxi * dydzeta,
        "dzetadx": dydxi * dzdeta - dydeta * dzdxi,
        "dzetady": dxdeta * dzdxi - dxdxi * dzdeta,
        "dzetadz": dxdxi * dydeta - dxdeta * dydxi,
        "J": Jm,
    }
    del der, dxdxi, dxdeta, dxdzeta, dydxi, dydeta, dydzeta, dzdxi, dzdeta, dzdzeta
    tx, ty, tz = ghosted(nx, ny, nz)
    out = {}
    for k in METRIC_NAMES:
        a = zeros((1, tz, ty, tx))
        a[0, NG:NG + nz, NG:NG + ny, NG:NG + nx] = vals.pop(k)
        periodic_fill(a, nx, ny, nz)
        out[k] = a[0]
    return out


def cartesian_metrics(nx, ny, nz, hx, hy, hz, device=None):
    return metrics_from_mapping(lambda i, j, k: (i * hx, j * hy, k * hz), nx, ny, nz, device)


def wavy_mapping(nx, ny, nz, amp=0.1, scale=1.0):
    """x = s (ξ + a sin2πη sin2πζ), y = s (η + a sin2πζ sin2πξ), z = s (ζ + a sin2πξ sin2πη)
    with ξ = i/nx, η = j/ny, ζ = k/nz (the curvilinear benchmark mapping, scaled by s)."""
    tp = 2 * math.pi

    def xyz(i, j, k):
        xi, eta, zeta = i / nx, j / ny, k / nz
        x = xi + amp * _sin(tp * eta) * _sin(tp * zeta)
        y = eta + amp * _sin(tp * zeta) * _sin(tp * xi)
        z = zeta + amp * _sin(tp * xi) * _sin(tp * eta)
        return (x, y, z) if scale == 1.0 else (scale * x, scale * y, scale * z)
    return xyz


def wavy_metrics(nx, ny, nz, amp=0.1):
    xyz = wavy_mapping(nx, ny, nz, amp)
    return metrics_from_mapping(xyz, nx, ny, nz), xyz


# -------------------------------------------------------------------------------------- cases
@dataclass
class Case:
    name: str
    nx: int
    ny: int
    nz: int
    thermo: Thermo
    transport: Transport
    metrics: dict
    Q: np.ndarray       # (7, Tz, Ty, Tx): rho u v w p T e
    rhoi: np.ndarray    # (ns, Tz, Ty, Tx)
    dt: float
    steps: int = 1
    periodic: int = 7
    info: dict = field(default_factory=dict)
    # non-periodic cases: the inflow state of the reference's fills (FlameInflow), used by
    # fill_x / fill_z at the x-low and z-low boundaries (boundary.jl:1-137)
    inflow: object = None

    @property
    def ns(self) -> int:
        return self.thermo.ns

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz

    def grid(self) -> FlameGrid:
        return FlameGrid(self.nx, self.ny, self.nz, NG, self.ns, self.periodic)

    def U(self) -> np.ndarray:
        """prim2c (utils.jl:71-92) on every ghosted point."""
        rho, u, v, w, e = self.Q[0], self.Q[1], self.Q[2], self.Q[3], self.Q[6]
        return np.stack([rho, u * rho, v * rho, w * rho, e + 0.5 * rho * (u * u + v * v + w * w)])


def _finish(name, nx, ny, nz, thermo, transport, metrics, rho, u, v, w, T, Y, cfl, steps,
            info) -> Case:
    """Assembles Q and rhoi from interior primitive fields, fills ghosts, picks dt."""
    tx, ty, tz = ghosted(nx, ny, nz)
    ns = thermo.ns
    rhoi_int = rho[None] * Y
    p = thermo.pressure(T, rhoi_int)
    e = thermo.internal_energy(T, rhoi_int)
    Q = np.zeros((7, tz, ty, tx))
    rhoi = np.zeros((ns, tz, ty, tx))
    sl = (slice(NG, NG + nz), slice(NG, NG + ny), slice(NG, NG + nx))
    for n, f in enumerate([rho, u, v, w, p, T, e]):
        Q[(n,) + sl] = f
    rhoi[(slice(None),) + sl] = rhoi_int
    periodic_fill(Q, nx, ny, nz)
    periodic_fill(rhoi, nx, ny, nz)
    c = Case(name, nx, ny, nz, thermo, transport, metrics, Q, rhoi, 0.0, steps, 7, info)
    c.dt = cfl_dt(c, cfl)
    c.info.setdefault("cfl", cfl)
    return c


def cfl_dt(case: Case, cfl: float = 0.5) -> float:
    """dt = cfl / max over cells of Σ_d J (|m_d·u| + c |m_d|), with m_d the stored metric rows
    and c = sqrt(γ p / ρ), γ = p/e + 1 (split.jl:40-41).  The reference uses a fixed dt
    (run.jl:30); this rule is this project's choice."""
    sl = (slice(NG, NG + case.nz), slice(NG, NG + case.ny), slice(NG, NG + case.nx))
    rho, u, v, w, p, e = (case.Q[n][sl] for n in (0, 1, 2, 3, 4, 6))
    gam = p / e + 1
    c = np.sqrt(gam * p / rho)
    m = case.metrics
    J = m["J"][sl]
    tot = np.zeros_like(rho)
    for a, b, cc in (("dxidx", "dxidy", "dxidz"), ("detadx", "detady", "detadz"),
                     ("dzetadx", "dzetady", "dzetadz")):
        mx, my, mz = m[a][sl], m[b][sl], m[cc][sl]
        tot += J * (np.abs(mx * u + my * v + mz * w) + c * np.sqrt(mx * mx + my * my + mz * mz))
    return float(cfl / tot.max())


def taylor_green(n: int = 64, Re: float = 1600.0, Ma: float = 0.1, ns: int = 1,
                 perturb: float = 0.0, seed: int = 4, species_seed: int = 3,
                 cfl: float = 0.5, steps: int = 100) -> Case:
    """Taylor-Green vortex on [0, 2π)^3, h = 2π/n, T0 = 300 K, p0 = 101325 Pa,
    U0 = Ma sqrt(γ R T0), ρ = p/(R T0), μ = ρ0 U0 L / Re (L = 1), λ = cp μ / Pr (Pr = 0.71).
    With ns > 1 the gas is a uniform random mixture of the synthetic species; `perturb` adds
    random-phase Fourier modes with |k| <= 8 of that relative amplitude to u, v, w."""
    thermo = ideal_air() if ns == 1 else synthetic_species(9, species_seed).subset(ns)
    rng = np.random.default_rng(seed)
    Y = np.ones(1) if ns == 1 else rng.dirichlet(np.ones(ns))
    h = 2 * math.pi / n
    metrics = cartesian_metrics(n, n, n, h, h, h)
    x = np.arange(n) * h
    Z, Yg, X = np.meshgrid(x, x, x, indexing="ij")
    T0, p0 = 300.0, 101325.0
    Wmix = 1.0 / np.sum(Y / thermo.mw)
    R = thermo.Ru / Wmix
    cp = float(thermo.cp_mass(np.array([T0]), Y[:, None])[0])
    gam = cp / (cp - R)
    U0 = Ma * math.sqrt(gam * R * T0)
    rho0 = p0 / (R * T0)
    u = U0 * np.sin(X) * np.cos(Yg) * np.cos(Z)
    v = -U0 * np.cos(X) * np.sin(Yg) * np.cos(Z)
    w = np.zeros_like(u)
    if perturb > 0:
        for comp in (u, v, w):
            comp += perturb * U0 * _fourier_noise(rng, X, Yg, Z, kmax=8)
    p = p0 + rho0 * U0 ** 2 / 16 * (np.cos(2 * X) + np.cos(2 * Yg)) * (np.cos(2 * Z) + 2)
    rho = p / (R * T0)
    T = np.full_like(rho, T0)
    mu = rho0 * U0 * 1.0 / Re
    tr = Transport(law=0, mu_ref=mu, Pr=0.71, lambda_ref=cp * mu / 0.71,
                   D_ref=cp * mu / 0.71 / (rho0 * cp))
    Yf = np.broadcast_to(Y[:, None, None, None], (ns,) + rho.shape)
    info = {"Re": Re, "Ma": Ma, "U0": U0, "rho0": rho0, "seed": seed, "h": h}
    return _finish(f"tgv{n}_ns{ns}", n, n, n, thermo, tr, metrics, rho, u, v, w, T, Yf, cfl,
                   steps, info)


def _fourier_noise(rng, X, Y, Z, kmax=8, nmodes=24):
    """Sum of random-phase modes with integer wavenumbers |k| <= kmax, unit max amplitude.
    X, Y, Z are the meshgrid of a uniform periodic axis; each mode is the imaginary part of an
    outer product of three 1-D complex exponentials."""
    x, y, z = X[0, 0, :], Y[0, :, 0], Z[:, 0, 0]
    acc = np.zeros_like(X)
    for _ in range(nmodes):
        while True:
            k = rng.integers(-kmax, kmax + 1, 3)
            if 0 < np.linalg.norm(k) <= kmax:
                break
        ph = rng.uniform(0, 2 * math.pi)
        ex, ey, ez = np.exp(1j * k[0] * x), np.exp(1j * k[1] * y), np.exp(1j * (k[2] * z + ph))
        acc += (ez[:, None, None] * ey[None, :, None] * ex[None, None, :]).imag
    return acc / nmodes


def ensemble(n_cases: int = 64, seed: int = 4, sizes=(32, 48, 64, 96, 128),
             species_seed: int = 3) -> list:
    """The batched benchmark ensemble: independent periodic Taylor-Green cases with sizes drawn
    uniformly from `sizes` (cubes), Re ~ U[400, 3200], Ma ~ U[0.1, 0.5], 1-9 species from the
    synthetic set, plus 2 % random-phase Fourier modes with |k| <= 8 (seeded per case)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_cases):
        n = int(rng.choice(sizes))
        Re = float(rng.uniform(400, 3200))
        Ma = float(rng.uniform(0.1, 0.5))
        ns = int(rng.integers(1, 10))
        c = taylor_green(n=n, Re=Re, Ma=Ma, ns=ns, perturb=0.02, seed=seed * 1000 + i,
                         species_seed=species_seed)
        c.name = f"ens{i:02d}_tgv{n}_ns{ns}"
        out.append(c)
    return out


def curvilinear_jet(nx: int = 256, ny: int = 128, nz: int = 128, seed: int = 1,
                    cfl: float = 0.5, steps: int = 500, amp: float = 0.1,
                    pressure_noise: float = 0.0) -> Case:
    """Ma 1.5 round jet on the wavy periodic mapping (diameter D = 0.25 centred in y, z; tanh
    shear layer of thickness 0.05 D; T 5000 K in the jet, 300 K outside; p = 3596 Pa; seeded
    1 % velocity perturbations).  `pressure_noise` > 0 adds relative random pressure noise,
    which drives the shock sensor into the WENO-Z and minmod branches (used by the tests)."""
    thermo = ideal_air()
    metrics, xyz = wavy_metrics(nx, ny, nz, amp)
    rng = np.random.default_rng(seed)
    kk, jj, ii = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    X, Y, Z = xyz(ii.astype(float), jj.astype(float), kk.astype(float))
    Dj, Tj, Ta, p0 = 0.25, 5000.0, 300.0, 3596.0
    R = thermo.Ru / thermo.mw[0]
    r = np.sqrt((Y - 0.5) ** 2 + (Z - 0.5) ** 2)
    f = 0.5 * (1 + np.tanh((Dj / 2 - r) / (2 * 0.05 * Dj)))
    Uj = 1.5 * math.sqrt(1.4 * R * Tj)
    T = Ta + (Tj - Ta) * f
    u = Uj * f + 0.01 * Uj * rng.uniform(-1, 1, f.shape)
    v = 0.01 * Uj * rng.uniform(-1, 1, f.shape)
    w = 0.01 * Uj * rng.uniform(-1, 1, f.shape)
    p = np.full_like(T, p0)
    if pressure_noise > 0:
        p = p * (1 + pressure_noise * rng.uniform(-1, 1, p.shape))
    rho = p / (R * T)
    tr = Transport(law=1, mu_ref=1.8e-5, T_ref=300.0, exponent=0.7, Pr=0.71)
    info = {"Uj": Uj, "seed": seed, "amp": amp, "pressure_noise": pressure_noise}
    return _finish(f"jet{nx}x{ny}x{nz}", nx, ny, nz, thermo, tr, metrics, rho, u, v, w, T,
                   np.ones((1,) + rho.shape), cfl, steps, info)


def mixing_layer(n: int = 192, ns: int = 9, seed: int = 2, species_seed: int = 3,
                 L: float = 0.01, cfl: float = 0.5, steps: int = 100) -> Case:
    """Cartesian periodic mixing layer with `ns` synthetic species.  A periodic double layer
    g(y) = ½[tanh((y − L/4)/δ) − tanh((y − 3L/4)/δ)], δ = L/20, blends T from 300 to 1500 K,
    the composition from Y_A to Y_B (Dirichlet(1), seeds `seed`, `seed`+1) and u = ΔU (g − ½)
    with ΔU = 0.3 c(300 K); p = 101325 Pa; μ = 1.8e-5 (T/300)^0.7, λ = cp μ/0.71, D = λ/(ρ cp)."""
    thermo = synthetic_species(ns, species_seed)
    h = L / n
    metrics = cartesian_metrics(n, n, n, h, h, h)
    x = (np.arange(n) + 0.5) * h
    Zg, Yg, Xg = np.meshgrid(x, x, x, indexing="ij")
    d = L / 20
    g = 0.5 * (np.tanh((Yg - L / 4) / d) - np.tanh((Yg - 3 * L / 4) / d))
    YA = np.random.default_rng(seed).dirichlet(np.ones(ns))
    YB = np.random.default_rng(seed + 1).dirichlet(np.ones(ns))
    Y = (1 - g)[None] * YA[:, None, None, None] + g[None] * YB[:, None, None, None]
    T = 300.0 + 1200.0 * g
    p0 = 101325.0
    Wmix = 1.0 / np.sum(Y / thermo.mw[:, None, None, None], axis=0)
    rho = p0 * Wmix / (thermo.Ru * T)
    cp300 = float(thermo.cp_mass(np.array([300.0]), YA[:, None])[0])
    R300 = thermo.Ru / (1.0 / np.sum(YA / thermo.mw))
    c0 = math.sqrt(cp300 / (cp300 - R300) * R300 * 300.0)
    u = 0.3 * c0 * (g - 0.5)
    v = 1e-3 * c0 * np.sin(2 * math.pi * Xg / L) * np.exp(-((Yg - L / 4) / (2 * d)) ** 2)
    w = np.zeros_like(u)
    tr = Transport(law=1, mu_ref=1.8e-5, T_ref=300.0, exponent=0.7, Pr=0.71)
    info = {"seed": seed, "species_seed": species_seed, "L": L, "c0": c0}
    return _finish(f"mix{n}_ns{ns}", n, n, n, thermo, tr, metrics, rho, u, v, w, T, Y, cfl,
                   steps, info)


def random_curvilinear(n: int = 16, ns: int = 1, seed: int = 11, amp: float = 0.1,
                       noise: float = 0.05, T_range=(300.0, 1500.0), cfl: float = 0.5) -> Case:
    """Small parity case: wavy mapping, random smooth-plus-noise fields with random pressure so
    all three hybrid branches (UP7, WENO-Z, minmod) occur.  Non-cubic extents catch index bugs."""
    nx, ny, nz = n + 4, n, n - 2
    thermo = ideal_air() if ns == 1 else synthetic_species(max(ns, 2), 3).subset(ns)
    metrics, xyz = wavy_metrics(nx, ny, nz, amp)
    rng = np.random.default_rng(seed)
    kk, jj, ii = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    X, Y, Z = xyz(ii.astype(float), jj.astype(float), kk.astype(float))
    tp = 2 * math.pi
    T = T_range[0] + (T_range[1] - T_range[0]) * (0.5 + 0.4 * np.sin(tp * X) * np.cos(tp * Y))
    T *= 1 + 0.05 * rng.uniform(-1, 1, T.shape)
    # smooth pressure in the first third of x (UP7 faces), noise in the middle third (WENO-Z)
    # and a 1.6x jump at two thirds (minmod faces)
    p = 1e5 * (1 + 0.3 * np.sin(tp * Z))
    mid = (ii >= nx // 3) & (ii < 2 * nx // 3)
    p = p * (1 + noise * rng.uniform(-1, 1, T.shape) * mid)
    p[:, :, 2 * nx // 3:] *= 1.6
    Ys = rng.dirichlet(np.ones(ns), size=T.shape).transpose(3, 0, 1, 2) if ns > 1 \
        else np.ones((1,) + T.shape)
    Wmix = 1.0 / np.sum(Ys / thermo.mw[:, None, None, None], axis=0)
    rho = p * Wmix / (thermo.Ru * T)
    c = np.sqrt(1.4 * p / rho)
    u = 0.5 * c * np.sin(tp * Y) + 0.05 * c * rng.uniform(-1, 1, T.shape)
    v = 0.3 * c * np.cos(tp * Z) + 0.05 * c * rng.uniform(-1, 1, T.shape)
    w = 0.2 * c * np.sin(tp * X) + 0.05 * c * rng.uniform(-1, 1, T.shape)
    tr = Transport(law=1, mu_ref=1.8e-3, T_ref=300.0, exponent=0.7, Pr=0.71)
    return _finish(f"rand{nx}x{ny}x{nz}_ns{ns}", nx, ny, nz, thermo, tr, metrics, rho, u, v, w,
                   T, Ys, cfl, 1, {"seed": seed})


def inflow_jet(nx: int = 32, ny: int = 16, nz: int = 16, ns: int = 5, seed: int = 12,
               amp: float = 0.1, cfl: float = 0.5) -> Case:
    """The reference's own boundary conditions (boundary.jl:1-191, solver.jl:321-325): not
    periodic; supersonic inflow at the x-low and z-low boundaries with the state fill_x / fill_z
    hard-code (79.8 Pa, 270.65 K, 1000 m/s along x, Y_2 = 0.233, Y_5 = 0.767), zero-gradient
    copies elsewhere.  The initial field is that free stream (boundary.jl:281-324) on the wavy
    mapping (scaled to a 1 m box), with a hot, fast round jet of species 1 along x through the
    middle (diameter 0.25, 900 K, u = 2000 m/s, Y_1 = 0.3), seeded 2 % velocity and pressure
    noise and a 1.6x pressure jump at two thirds of x, so all hybrid branches occur.  Synthetic species (`ns` >= 5).  Ghosts are given
    zero-gradient copies here; the device and the oracle replace them with the reference's
    fills before the first stage, as solver.jl:192-200 does."""
    thermo = synthetic_species(max(ns, 5), 3).subset(ns)
    inflow = reference_inflow(ns)
    metrics, xyz = wavy_metrics(nx, ny, nz, amp)
    rng = np.random.default_rng(seed)
    kk, jj, ii = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    X, Y, Z = xyz(ii.astype(float), jj.astype(float), kk.astype(float))
    r = np.sqrt((Y - 0.5) ** 2 + (Z - 0.5) ** 2)
    f = 0.5 * (1 + np.tanh((0.125 - r) / 0.02))
    Yair = np.array([inflow.Y[n] for n in range(ns)])
    Yjet = 0.7 * Yair
    Yjet[0] += 0.3
    Ys = (1 - f)[None] * Yair[:, None, None, None] + f[None] * Yjet[:, None, None, None]
    T = inflow.T + (900.0 - inflow.T) * f
    p = inflow.P * (1 + 0.02 * rng.uniform(-1, 1, T.shape))
    p[:, :, 2 * nx // 3:] *= 1.6  # a pressure jump across x = 2/3: minmod faces
    u = inflow.u + 1000.0 * f + 20.0 * rng.uniform(-1, 1, T.shape)
    v = 20.0 * rng.uniform(-1, 1, T.shape)
    w = 20.0 * rng.uniform(-1, 1, T.shape)
    Wmix = 1.0 / np.sum(Ys / thermo.mw[:, None, None, None], axis=0)
    rho = p * Wmix / (thermo.Ru * T)
    tr = Transport(law=1, mu_ref=1.8e-5, T_ref=300.0, exponent=0.7, Pr=0.71)
    c = _finish(f"inflowjet{nx}x{ny}x{nz}_ns{ns}", nx, ny, nz, thermo, tr, metrics, rho, u, v, w,
                T, Ys, cfl, 1, {"seed": seed, "bc": "reference inflow / zero gradient"})
    # zero-gradient ghosts in place of the periodic images _finish made
    sl = (slice(None), slice(NG, NG + nz), slice(NG, NG + ny), slice(NG, NG + nx))
    pad = ((0, 0), (NG, NG), (NG, NG), (NG, NG))
    c.Q = np.ascontiguousarray(np.pad(c.Q[sl], pad, mode="edge"))
    c.rhoi = np.ascontiguousarray(np.pad(c.rhoi[sl], pad, mode="edge"))
    c.periodic = 0
    c.inflow = inflow
    return c


def case_by_name(name: str, **kw) -> Case:
    table = {"tgv": taylor_green, "jet": curvilinear_jet, "mixing": mixing_layer,
             "random": random_curvilinear, "inflow": inflow_jet}
    return table[name](**kw)
