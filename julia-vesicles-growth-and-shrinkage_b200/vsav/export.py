"""Headless field export: the arrays the reference draws with CairoMakie
(scripts/visualize.jl) written as raw float32 volumes with NRRD detached headers
(readable by ParaView, 3D Slicer, or numpy), and its time series as CSV.

* ``plot_field`` of ``phi_plot`` (simulation.jl:124-128, Main.jl:119-131): the
  per-run sum of the vesicle fields + N - 1, 2D;
* ``plot_iso`` (visualize.jl:166-218): its input, the 3D phase field of each
  vesicle (the isosurface phi = 0 is extracted by whatever reads the volume);
* ``plot_velocity`` (visualize.jl:64-84): the speed |u| and the components;
* ``plot_vector`` of the energy and area-ratio histories (Main.jl:160-173).

The fields are reduced and narrowed to float32 on the device
(``vsav_export_f32``); only the float32 frames cross to the host.
"""
from __future__ import annotations

import os

import numpy as np

NRRD_MAGIC = "NRRD0004"


def write_nrrd(base: str, arr, spacing, origin=None, kinds=None) -> tuple:
    """Writes ``base.raw`` (little-endian float32, x fastest) and the detached
    header ``base.nhdr``.  arr: C-order [..., Nz][Ny][Nx]; spacing/origin per
    spatial axis in x, y(, z) order.  Returns the two paths."""
    a = np.ascontiguousarray(arr, dtype="<f4")
    nd = len(spacing)
    if a.ndim < nd:
        raise ValueError("array has fewer axes than spacings")
    sizes = list(a.shape[::-1])                      # NRRD lists the fastest axis first
    raw = base + ".raw"
    hdr = base + ".nhdr"
    a.tofile(raw)
    extra = a.ndim - nd
    kinds = kinds or (["domain"] * nd + ["list"] * extra)
    sp = [repr(float(s)) for s in spacing] + ["nan"] * extra
    org = origin if origin is not None else [0.0] * nd
    with open(hdr, "w") as f:
        f.write(f"{NRRD_MAGIC}\n")
        f.write("type: float\n")
        f.write(f"dimension: {a.ndim}\n")
        f.write("sizes: " + " ".join(str(s) for s in sizes) + "\n")
        f.write("spacings: " + " ".join(sp) + "\n")
        f.write("kinds: " + " ".join(kinds) + "\n")
        if extra == 0:
            f.write("space origin: (" + ",".join(repr(float(o)) for o in org) + ")\n")
        f.write("endian: little\n")
        f.write("encoding: raw\n")
        f.write(f"data file: {os.path.basename(raw)}\n")
    return raw, hdr


def read_nrrd(hdr: str) -> np.ndarray:
    """Reads a header written by write_nrrd back into a C-order float32 array."""
    meta = {}
    with open(hdr) as f:
        if f.readline().strip() != NRRD_MAGIC:
            raise ValueError("not an NRRD0004 header")
        for line in f:
            if ":" in line:
                k, v = line.split(":", 1)
                meta[k.strip()] = v.strip()
    sizes = [int(s) for s in meta["sizes"].split()]
    raw = os.path.join(os.path.dirname(hdr), meta["data file"])
    return np.fromfile(raw, dtype="<f4").reshape(sizes[::-1])


def spacing_of(cfg) -> list:
    s = [cfg.Lx / cfg.Nx, cfg.Ly / cfg.Ny]
    if getattr(cfg, "Nz", 0):
        s.append(cfg.Lz / cfg.Nz)
    return s


def export_frame(h, cfg, outdir: str, tag: str, level: int = 0) -> list:
    """One frame of the reference's plots as raw arrays: 2D phi_plot (per run),
    3D the phase field of every vesicle (isosurface input), and the speed |u|.
    Returns the header paths written."""
    os.makedirs(outdir, exist_ok=True)
    sp = spacing_of(cfg)
    out = []
    if h.nd == 2:
        phi_sum = h.export_f32("phi_sum", level)
        for r in range(h.R):
            out.append(write_nrrd(os.path.join(outdir, f"phi_{tag}" + (f"_run{r}" if h.R > 1 else "")), phi_sum[r], sp)[1])
    else:
        phi = h.export_f32("phi", level)
        for v in range(h.V):
            out.append(write_nrrd(os.path.join(outdir, f"phi_{tag}" + (f"_v{v}" if h.V > 1 else "")), phi[v], sp)[1])
    speed = h.export_f32("speed", level)
    for r in range(h.R):
        out.append(write_nrrd(os.path.join(outdir, f"speed_{tag}" + (f"_run{r}" if h.R > 1 else "")), speed[r], sp)[1])
    return out


def write_history(path: str, t, values, name: str) -> str:
    """plot_vector's data (Main.jl:160-173): a CSV of t and one column per run."""
    v = np.asarray(values, dtype=np.float64)
    if v.ndim == 1:
        v = v[:, None]
    t = np.asarray(t, dtype=np.float64)
    cols = [name] if v.shape[1] == 1 else [f"{name}_run{r}" for r in range(v.shape[1])]
    with open(path, "w") as f:
        f.write("t," + ",".join(cols) + "\n")
        for i in range(v.shape[0]):
            f.write(repr(float(t[i])) + "," + ",".join(repr(float(x)) for x in v[i]) + "\n")
    return path
