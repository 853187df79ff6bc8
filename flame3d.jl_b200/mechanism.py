"""A seeded synthetic reaction mechanism in the form reactionProperty holds (run.jl:84-94).

The reference takes its mechanism from Cantera (initReact, reactions.jl:506-575), which is not
installed here.  This one has eight species and eight reversible reactions of the three kinds
the reference supports (1 Arrhenius, 2 three-body, 3 falloff with the Troe form); the molar
masses are sums of atomic masses, so every reaction balances mass and elements exactly in real
arithmetic.  Rate parameters are drawn from a seeded generator in plausible ranges; the NASA-7
data are single-range with a1 (cp/R), a6 (formation enthalpy / R) and a7 (entropy constant
from a standard entropy at 298.15 K).  It is test and benchmark data, not a model of hydrogen
combustion.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .abi import FlameReactions
from .cases import RU, Thermo

SPECIES = ("H2", "O2", "H", "O", "OH", "H2O", "H2O2", "N2")
# atom counts (H, O, N)
ATOMS = np.array([[2, 0, 0], [0, 2, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0], [2, 1, 0], [2, 2, 0],
                  [0, 0, 2]])
ATOMIC_MASS = np.array([1.008e-3, 15.999e-3, 14.007e-3])  # kg/mol
# formation enthalpy / R [K] and standard entropy / R at 298.15 K (textbook magnitudes)
HF_R = np.array([0.0, 0.0, 26219.0, 29968.0, 4500.0, -29084.0, -16313.0, 0.0])
S298_R = np.array([15.70, 24.65, 13.82, 19.48, 22.13, 22.73, 28.43, 23.08])
CP_R = np.array([3.5, 3.7, 2.5, 2.5, 3.6, 4.2, 5.0, 3.6])

# (type, reactants, products); M (third body) is implied by the type
REACTIONS = (
    (1, {"H": 1, "O2": 1}, {"O": 1, "OH": 1}),
    (1, {"O": 1, "H2": 1}, {"H": 1, "OH": 1}),
    (1, {"OH": 1, "H2": 1}, {"H": 1, "H2O": 1}),
    (1, {"OH": 2}, {"O": 1, "H2O": 1}),
    (2, {"H": 2}, {"H2": 1}),
    (2, {"H": 1, "OH": 1}, {"H2O": 1}),
    (2, {"O": 2}, {"O2": 1}),
    (3, {"OH": 2}, {"H2O2": 1}),
)


@dataclass
class Mechanism:
    thermo: Thermo
    reaction_type: np.ndarray  # (nr,) int64
    sgm: np.ndarray            # (nr,) int64
    vf: np.ndarray             # Julia (ns, nr): numpy (nr, ns) C order, int64
    vr: np.ndarray
    Arr: np.ndarray            # Julia (3, nr): numpy (nr, 3)
    ef: np.ndarray             # Julia (ns, nr): numpy (nr, ns)
    loP: np.ndarray            # Julia (3, nr): numpy (nr, 3)
    Troe: np.ndarray           # Julia (4, nr): numpy (nr, 4)
    atm: float = 101325.0

    FIELDS = ("reaction_type", "sgm", "vf", "vr", "Arr", "ef", "loP", "Troe")

    @property
    def nreacs(self) -> int:
        return int(self.reaction_type.shape[0])

    def to_c(self, arrays: dict | None = None) -> FlameReactions:
        """The C struct over `arrays` (name -> object with .data_ptr() or a numpy array); by
        default this mechanism's own numpy arrays (for the oracle)."""
        src = arrays or {k: getattr(self, k) for k in self.FIELDS}
        ptr = {k: (v.data_ptr() if hasattr(v, "data_ptr") else v.ctypes.data)
               for k, v in src.items()}
        r = FlameReactions()
        r.nreacs, r.atm = self.nreacs, self.atm
        for k in self.FIELDS:
            setattr(r, k, ptr[k])
        return r

    def to_device(self, device="cuda"):
        """Device copies of the arrays and the struct pointing at them."""
        import torch
        arrays = {k: torch.from_numpy(np.ascontiguousarray(getattr(self, k))).to(device)
                  for k in self.FIELDS}
        return arrays, self.to_c(arrays)


def synthetic_mechanism(seed: int = 13) -> Mechanism:
    """The eight-species, eight-reaction mechanism with seeded rate parameters: A = 10^U[7, 11]
    (bimolecular, m^3/mol/s) or 10^U[3, 7] (three-body, m^6/mol^2/s), b ~ U[-1, 1],
    E/R ~ U[0, 9000] K; falloff low-pressure A = 10^U[9, 13]; Troe (a, T***, T*, T**) with
    a ~ U[0.4, 0.8], T*** ~ U[100, 500] K, T* ~ U[1000, 5000] K, T** = 1e30; third-body
    efficiencies 1 with H2O 6 and H2 2.5."""
    rng = np.random.default_rng(seed)
    ns, nr = len(SPECIES), len(REACTIONS)
    mw = ATOMS @ ATOMIC_MASS
    lo = np.zeros((ns, 7))
    lo[:, 0] = CP_R
    lo[:, 5] = HF_R - CP_R * 298.15
    lo[:, 6] = S298_R - CP_R * math.log(298.15)
    thermo = Thermo(mw=mw, lo=lo, hi=lo.copy(), sep=np.full(ns, 1000.0), min_temp=200.0,
                    max_temp=6000.0, Ru=RU)
    idx = {s: i for i, s in enumerate(SPECIES)}
    rtype = np.zeros(nr, dtype=np.int64)
    vf = np.zeros((nr, ns), dtype=np.int64)
    vr = np.zeros((nr, ns), dtype=np.int64)
    Arr = np.zeros((nr, 3))
    ef = np.zeros((nr, ns))
    loP = np.zeros((nr, 3))
    Troe = np.zeros((nr, 4))
    for j, (t, reac, prod) in enumerate(REACTIONS):
        rtype[j] = t
        for s, k in reac.items():
            vf[j, idx[s]] = k
        for s, k in prod.items():
            vr[j, idx[s]] = k
        Arr[j] = (10 ** rng.uniform(7, 11) if t != 2 else 10 ** rng.uniform(3, 7),
                  rng.uniform(-1, 1), rng.uniform(0, 9000))
        if t >= 2:
            ef[j] = 1.0
            ef[j, idx["H2O"]] = 6.0
            ef[j, idx["H2"]] = 2.5
        if t == 3:
            loP[j] = (10 ** rng.uniform(9, 13), rng.uniform(-1, 1), rng.uniform(0, 3000))
            Troe[j] = (rng.uniform(0.4, 0.8), rng.uniform(100, 500), rng.uniform(1000, 5000),
                       1e30)
    sgm = (vf - vr).sum(axis=1).astype(np.int64)
    return Mechanism(thermo, rtype, sgm, vf, vr, Arr, ef, loP, Troe)


def reacting_state(mech: Mechanism, case):
    """Q and rho_i of `case` re-expressed with the mechanism's thermodynamics: the same T and
    mixture fractions, rho_i rescaled to sum to rho, p and e recomputed (thermo.jl:20-26,
    219-228).  `case` must have len(SPECIES) species."""
    th = mech.thermo
    Q = case.Q.copy()
    r = case.rhoi.copy()
    r *= Q[0] / r.sum(axis=0)
    Q[4] = th.pressure(Q[5], r)
    Q[6] = th.internal_energy(Q[5], r)
    return np.ascontiguousarray(Q), np.ascontiguousarray(r)


def element_totals(mech: Mechanism, rhoi: np.ndarray) -> np.ndarray:
    """Moles of H, O, N per volume at every point, (3, ...)."""
    mol = rhoi / mech.thermo.mw.reshape((-1,) + (1,) * (rhoi.ndim - 1))
    return np.tensordot(ATOMS.T.astype(float), mol, axes=1)

