"""Resumable state snapshots of a handle.

The reference writes phi, psi, mu, nu, p, u, R1..R3 and Q of the present
level to MAT files every save_interval steps (src/simulation.jl:113-143,
scripts/Main.jl:130-153) and cannot restart from them: the old level, A0 and
dt are not kept.  A snapshot here holds everything a run needs to continue
bit for bit: both time levels (physical fields and spectra), the SAV scalars
of both levels, A0, dt and the index of the next step.

Format (numpy .npz, format tag "vsav-snapshot-1"), per level L in
{present, old}:
    L_phi, L_psi, L_mu, L_nu      float64 [V][(Nz)][Ny][Nx]
    L_u                           float64 [R][nd][(Nz)][Ny][Nx]
    L_p                           float64 [R][(Nz)][Ny][Nx]
    L_<field>_hat                 complex128, the same leading axes, last axis Nx/2+1
    L_scalars                     float64 [R][4]  (Q, R1, R2, R3)
and A0 [V], dt [R], n_next (the step index to pass to the next run), and
meta (JSON: grid, V, R, run sizes, precision).  Arrays are in C order, x
fastest, i.e. the reference's column-major Julia arrays.
"""
from __future__ import annotations

import json

import numpy as np

FORMAT = "vsav-snapshot-1"
FIELDS = ("phi", "psi", "mu", "nu", "u", "p")
LEVELS = ((0, "present"), (1, "old"))


def save(h, path: str, n_next: int, extra: dict | None = None) -> None:
    """Write the state of handle h; n_next is the step index the run continues with."""
    arrays = {}
    for lvl, tag in LEVELS:
        for f in FIELDS:
            arrays[f"{tag}_{f}"] = h.get_field(f, lvl)
            arrays[f"{tag}_{f}_hat"] = h.get_field(f + "_hat", lvl)
        arrays[f"{tag}_scalars"] = h.get_scalars(lvl)
    arrays["A0"] = h.get_A0()
    arrays["dt"] = h.get_dt()
    arrays["n_next"] = np.int64(n_next)
    meta = {"format": FORMAT, "nd": h.nd, "Nx": h.Nx, "Ny": h.Ny, "Nz": h.Nz, "V": h.V, "R": h.R,
            "run_sizes": list(h.run_sizes), "precision": getattr(h, "precision", None)}
    if extra:
        meta.update(extra)
    arrays["meta"] = np.array(json.dumps(meta))
    np.savez(path, **arrays)


def load(h, path: str) -> int:
    """Restore a snapshot into handle h (same grid, vesicles and runs); returns n_next."""
    z = np.load(path)
    meta = json.loads(str(z["meta"]))
    if meta.get("format") != FORMAT:
        raise ValueError(f"not a {FORMAT} file: {path}")
    for k in ("nd", "Nx", "Ny", "Nz", "V", "R"):
        if meta[k] != getattr(h, k):
            raise ValueError(f"snapshot {k} = {meta[k]} does not match the handle ({getattr(h, k)})")
    if list(meta["run_sizes"]) != list(h.run_sizes):
        raise ValueError("snapshot run sizes do not match the handle")
    for lvl, tag in LEVELS:
        for f in FIELDS:
            h.set_field(f, z[f"{tag}_{f}"], lvl)
            h.set_field(f + "_hat", z[f"{tag}_{f}_hat"], lvl)
        h.set_scalars(z[f"{tag}_scalars"], lvl)
    h.set_A0(z["A0"])
    h.set_dt(z["dt"])
    return int(z["n_next"])
