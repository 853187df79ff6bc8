"""Checkpoints in the reference's restart layout, written as raw files (no HDF5 in this image).

The reference writes `CHK/chk<step>.h5` (solver.jl:438-466) with two Float64 datasets,
`Q_h` of size (Nx_tot, Ny_tot, Nz_tot, Nprim, Nprocs) and `ρi_h` of size
(Nx_tot, Ny_tot, Nz_tot, Nspecs, Nprocs), one slab per MPI rank, and restarts by reading slab
rank+1 of each (solver.jl:69-79).  Neither h5py nor libhdf5 is available here, so a checkpoint
is a directory `chk<step>.f3d/` holding

    Q_h.bin, rhoi_h.bin   the datasets' elements as little-endian float64 in Julia's
                          column-major order (i fastest, then j, k, variable, rank): exactly the
                          bytes of the in-memory arrays, for one rank (Nprocs = 1)
    meta.json             shapes (in Julia's order), dtype, dataset names, step, dt, grid

Converting to the reference's file where HDF5 exists is one call per dataset, e.g. with h5py:
`f.create_dataset("Q_h", data=np.fromfile("Q_h.bin", "<f8").reshape(shape[::-1]))` — h5py's
C-order shape is Julia's reversed, so HDF5.jl reads back (Nx_tot, Ny_tot, Nz_tot, Nprim, 1).
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

FORMAT = "flame3d-b200 raw checkpoint 1"


def _julia_shape(a: np.ndarray) -> list[int]:
    """(nv, Tz, Ty, Tx) C-order -> Julia (Tx, Ty, Tz, nv, Nprocs=1)."""
    return list(a.shape[::-1]) + [1]


def save(path: str | Path, Q: np.ndarray, rhoi: np.ndarray, step: int = 0, dt: float = 0.0,
         grid: dict | None = None) -> Path:
    """Writes Q (7, Tz, Ty, Tx) and rho_i (ns, Tz, Ty, Tx) as float64."""
    d = Path(path)
    d.mkdir(parents=True, exist_ok=True)
    q = np.ascontiguousarray(Q, dtype="<f8")
    r = np.ascontiguousarray(rhoi, dtype="<f8")
    if q.ndim != 4 or r.ndim != 4 or q.shape[0] != 7 or q.shape[1:] != r.shape[1:]:
        raise ValueError(f"bad shapes Q {q.shape}, rhoi {r.shape}")
    q.tofile(d / "Q_h.bin")
    r.tofile(d / "rhoi_h.bin")
    meta = {"format": FORMAT, "step": int(step), "dt": float(dt), "dtype": "<f8",
            "order": "column-major (Julia): i fastest, then j, k, variable, rank",
            "datasets": {"Q_h": {"file": "Q_h.bin", "shape": _julia_shape(q)},
                         "ρi_h": {"file": "rhoi_h.bin", "shape": _julia_shape(r)}},
            "grid": grid or {}}
    (d / "meta.json").write_text(json.dumps(meta, indent=1, ensure_ascii=False))
    return d


def load(path: str | Path) -> tuple[np.ndarray, np.ndarray, dict]:
    """Reads a checkpoint back as (Q, rho_i, meta) in this package's (nv, Tz, Ty, Tx) order."""
    d = Path(path)
    meta = json.loads((d / "meta.json").read_text())
    if meta.get("format") != FORMAT:
        raise ValueError(f"{d}: not a {FORMAT!r} checkpoint")
    out = []
    for name in ("Q_h", "ρi_h"):
        ds = meta["datasets"][name]
        tx, ty, tz, nv, nprocs = ds["shape"]
        if nprocs != 1:
            raise ValueError(f"{d}: {name} holds {nprocs} rank slabs; one GPU reads one")
        a = np.fromfile(d / ds["file"], dtype="<f8")
        if a.size != tx * ty * tz * nv:
            raise ValueError(f"{d}: {ds['file']} has {a.size} values, expected "
                             f"{tx * ty * tz * nv}")
        out.append(a.reshape(nv, tz, ty, tx))
    return out[0], out[1], meta


def save_case(path: str | Path, dc, step: int = 0) -> Path:
    """Checkpoints a DeviceCase's current primitive state (FP64 on disk whatever its
    precision, as the reference stores Float64)."""
    Q, r = dc.primitives()
    c = dc.case
    return save(path, Q, r, step, dc.dt, {"nx": c.nx, "ny": c.ny, "nz": c.nz, "ns": c.ns,
                                          "ng": int(dc.grid.ng)})


def restore_case(path: str | Path, dc) -> dict:
    """Loads a checkpoint into a DeviceCase of the same grid: the primitive state, then U
    (prim2c, utils.jl:71-92) and the transport of the state, as a restart does."""
    import torch
    Q, r, meta = load(path)
    cur = dc.cur
    if tuple(Q.shape) != tuple(dc.Q[cur].shape) or tuple(r.shape) != tuple(dc.rhoi[cur].shape):
        raise ValueError(f"checkpoint grid {Q.shape[1:]} x ns {r.shape[0]} does not match the "
                         f"case {tuple(dc.Q[cur].shape[1:])} x ns {dc.rhoi[cur].shape[0]}")
    q64 = torch.from_numpy(Q).to(dc.device)
    dc.Q[cur].copy_(q64)
    dc.rhoi[cur].copy_(torch.from_numpy(r).to(dc.device))
    dc.restore_conserved(q64)
    return meta
