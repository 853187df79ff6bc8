"""Regenerates the committed fixtures in tests/golden/ (run in the development container).

up7_fdmcoeffs.json
    The reference's own coefficient generator, Utils/FDMcoeffs.py (imported from the read-only
    reference checkout), evaluated exactly as its last line does: the UP5 flux coefficients
    (fluxCoeff(6, -3)) blended 0.7 / 0.3 with the CD6 ones (fluxCoeff(7, -3)).  Prepending the
    zero weight of F[i-4] gives run.jl:57's UP7 constant.  This pins the reconstruction weights
    of the oracle and the kernels to reference code that actually runs here.

oracle_regression.json
    Oracle outputs (one RK3 stage) on three small seeded cases: input hashes plus per-field sums,
    norms and sampled values.  They are not reference outputs (the reference cannot run here);
    they freeze the oracle so an accidental edit of the restatement is caught.

    python tests/golden/make_golden.py --reference /path/to/Flame3D.jl
    (or FLAME3D_REFERENCE=/path/to/Flame3D.jl python tests/golden/make_golden.py)
"""
from __future__ import annotations

import argparse
import contextlib
import hashlib
import importlib.util
import io
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "tests"))
sys.path.insert(0, str(ROOT / "oracle"))


def up7_fixture(ref: Path) -> dict:
    spec = importlib.util.spec_from_file_location("FDMcoeffs", ref / "Utils" / "FDMcoeffs.py")
    mod = importlib.util.module_from_spec(spec)
    out = io.StringIO()
    with contextlib.redirect_stdout(out):
        spec.loader.exec_module(mod)
    a = mod.fluxCoeff(7, -3)
    b = np.append(mod.fluxCoeff(6, -3), 0)
    blend = b * 0.7 + 0.3 * a
    return {"source": "Utils/FDMcoeffs.py fluxCoeff(7,-3), fluxCoeff(6,-3), blend 0.7/0.3",
            "cd6_flux": a.tolist(), "up5_flux": b.tolist(), "blend": blend.tolist(),
            "printed": out.getvalue().strip()}


REG_CASES = [("random", dict(n=8, ns=1, seed=21)), ("random", dict(n=8, ns=3, seed=22)),
             ("tgv", dict(n=8, ns=1))]
SAMPLE = 48


def summarize(a: np.ndarray) -> dict:
    flat = a.reshape(a.shape[0], -1)
    rng = np.random.default_rng(0)
    idx = rng.choice(flat.shape[1], SAMPLE, replace=False)
    return {"sum": flat.sum(axis=1).tolist(), "l2": np.linalg.norm(flat, axis=1).tolist(),
            "idx": idx.tolist(), "vals": flat[:, idx].tolist()}


def input_hash(case) -> str:
    h = hashlib.sha256()
    for a in (case.Q, case.rhoi, *[case.metrics[k] for k in sorted(case.metrics)]):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def regression_fixture() -> dict:
    from conftest import load_package
    f3d = load_package()
    import oracle
    out = {}
    for name, kw in REG_CASES:
        case = f3d.cases.case_by_name(name, **kw)
        oc = oracle.OracleCase(case)
        oc.stage(1)
        key = f"{name}:{json.dumps(kw, sort_keys=True)}"
        out[key] = {"input_sha256": input_hash(case), "dt": case.dt, "U": summarize(oc.U),
                    "Q": summarize(oc.Q), "rhoi": summarize(oc.rhoi)}
    return out


if __name__ == "__main__":
    import os
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("FLAME3D_REFERENCE"),
                    help="checkout of Flame3D.jl (default: $FLAME3D_REFERENCE)")
    a = ap.parse_args()
    if not a.reference:
        ap.error("give the reference checkout: --reference PATH or FLAME3D_REFERENCE=PATH")
    (HERE / "up7_fdmcoeffs.json").write_text(json.dumps(up7_fixture(Path(a.reference)), indent=1))
    (HERE / "oracle_regression.json").write_text(json.dumps(regression_fixture(), indent=1))
    print("wrote", HERE / "up7_fdmcoeffs.json", HERE / "oracle_regression.json")
