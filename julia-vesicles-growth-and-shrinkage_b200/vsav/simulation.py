"""run_simulation (src/simulation.jl:2-155) on the device, with the reference's
defaults (set_para_base, Init.jl:8-69 / Init_3d.jl:8-62), its two-phase time
grid, its save schedule and its outputs:

* every save point: the state as a MAT file (``state_2d_t{t}.mat`` /
  ``state_3d_t{t}.mat`` with phi, psi, mu, nu, p, u, R1, R2, R3, Q in the
  reference's array shapes, simulation.jl:113-143) and, in place of the PNG of
  ``phi_plot``, its raw float32 frame with an NRRD header (``export.py``);
* the end (Main.jl:109-174): ``state_*_final.mat``, the final frame, and the
  energy and area-ratio histories as CSV instead of line plots.

The time steps between save points run as one ``vsav_run`` call each (CUDA-graph
replayed steps, per-step dt from the schedule, per-step monitor)."""
from __future__ import annotations

import math
import os
from types import SimpleNamespace

import numpy as np

from . import export
from .core import Handle

SQ2 = math.sqrt(2.0)


def set_para_base(dt: float, T: float, ndim: int = 2) -> SimpleNamespace:
    """The reference's Config defaults: Init.jl:8-69 (2D: N = 1, 256^2 on [0, 1)^2,
    goal :s) and Init_3d.jl:8-62 (3D: 128^3 on [0, 1)^3, goal :g)."""
    eps, gb = 0.01, 0.1
    gin = gout = 1e5
    if ndim == 2:
        N, n, L, goal = 1, 256, 1.0, "s"
        psi_in = [0.65] if goal == "g" else [0.1]
    else:
        N, n, L, goal = 1, 128, 1.0, "g"
        psi_in = [0.1] if goal == "s" else [0.65]
    return SimpleNamespace(
        N=N, epsilon=eps, M_phi=1.0, M0_psi=0.5, eta=1.0, gamma_surf=1.0, gamma_area=5e4,
        gamma_bend=gb, gamma_in=gin, beta_in=0.0, psi_in_v=psi_in, gamma_out=gout, beta_out=0.0,
        psi_out_v=[0.8], lamda=1.0, S1=(3 * SQ2 / 8) * eps * gb, S2=0.0, S3=gb / eps ** 3,
        S4=min(gin, gout), C1=1.0, C2=5.0e5, C3=1.0e6, dt=dt, T=T, Nx=n, Ny=n, Lx=L * N, Ly=L,
        tol=1e-12, goal=goal, Nz=(n if ndim == 3 else 0), Lz=(L if ndim == 3 else 0.0))


def _float_range(a: float, b: float, step: float) -> np.ndarray:
    """Julia's range(a, b, step=step) for floats: a + i*step for i = 0 .. floor((b - a)/step),
    the count taken with the tolerance of an exact multiple."""
    q = (b - a) / step
    n = int(math.floor(q + 1e-10 * max(1.0, abs(q))))
    return a + step * np.arange(n + 1, dtype=np.float64)


def time_grid(dt: float, T: float) -> np.ndarray:
    """simulation.jl:15-19: 100 steps of 1e-7 up to 1e-5, then steps of dt up to T."""
    t1 = _float_range(0.0, 1e-5, 1e-7)
    t2 = _float_range(1e-5, T, dt)
    return np.concatenate([t1, t2[1:]])


def save_steps(Dt: np.ndarray, save_interval: float) -> list:
    """The steps n (1-based) after which the reference saves (simulation.jl:113-115):
    floor((Dt[n] + 1e-12) / save_interval) grew since the last save; the label
    is the time Dt[n] (the step's start)."""
    out, last = [], -1
    for n in range(1, len(Dt)):
        idx = math.floor((Dt[n - 1] + 1e-12) / save_interval)
        if idx > last:
            out.append(n)
            last = idx
    return out


def _mat_state(h: Handle) -> dict:
    """The saved dictionary of simulation.jl:118-129 in the reference's (column-
    major) shapes: phi/psi/mu/nu (Nx, Ny[, Nz], N), p (Nx, Ny[, Nz]), u (..., nd)."""
    def jl(a):                                   # C-order [N][(Nz)][Ny][Nx] -> (Nx, Ny, (Nz,) N)
        return np.ascontiguousarray(np.transpose(a))
    d = {k: jl(h.get_field(k)) for k in ("phi", "psi", "mu", "nu")}
    d["p"] = jl(h.get_field("p")[0])
    d["u"] = jl(h.get_field("u")[0])
    q = h.get_scalars()[0]
    d.update(Q=float(q[0]), R1=float(q[1]), R2=float(q[2]), R3=float(q[3]))
    return d


def run_simulation(dt_val: float, T_val: float, state_type: int, save_path: str = "./results",
                   save_interval: float = 0.001, mat_folder: str | None = None, ndim: int = 2,
                   precision: str = "fp64", blob_u=None, conf=None, **handle_opts):
    """run_simulation(dt_val, T_val, state_type; save_path, save_interval)
    (simulation.jl:2-155, with Main.jl's final outputs).  Returns (handle, energy
    history, area-ratio history, Dt); the handle holds the final state.
    blob_u: the 20 uniform draws of state_type 4 (default: numpy's generator)."""
    from scipy.io import savemat
    conf = conf or set_para_base(dt_val, T_val, ndim)
    mat_folder = mat_folder or os.path.join(save_path, "MAT")
    os.makedirs(save_path, exist_ok=True)
    os.makedirs(mat_folder, exist_ok=True)
    h = Handle(conf, precision=precision, **handle_opts)
    if state_type == 4 and blob_u is None:
        blob_u = np.random.default_rng().uniform(size=20)
    h.generate_initial_condition(state_type, conf.goal, blob_u if state_type == 4 else None)
    Dt = time_grid(dt_val, T_val)
    Nt = len(Dt)
    tag_dim = "3d" if h.nd == 3 else "2d"
    saves = set(save_steps(Dt, save_interval))
    energy, area = [], []
    n = 1
    while n <= Nt - 1:
        # run up to and including the next save step (or the end)
        m = min([s for s in saves if s >= n] + [Nt - 1])
        dts = np.diff(Dt)[n - 1:m]
        E, A = h.run(n, m - n + 1, dt=dts, monitor=True)
        energy.extend(E[:, 0])
        area.extend(A[:, 0])
        if m in saves:
            t_str = f"{Dt[m - 1]:.2e}"
            savemat(os.path.join(mat_folder, f"state_{tag_dim}_t{t_str}.mat"), _mat_state(h))
            export.export_frame(h, conf, save_path, f"t{t_str}")
        n = m + 1
    # Main.jl:109-174
    savemat(os.path.join(mat_folder, f"state_{tag_dim}_final.mat"), _mat_state(h))
    export.export_frame(h, conf, save_path, "final")
    if len(energy) > 1:
        t = Dt[1:len(energy) + 1]
        export.write_history(os.path.join(save_path, "energy_history.csv"), t, energy, "modified_energy")
        export.write_history(os.path.join(save_path, "area_history.csv"), t, area, "area_ratio")
    return h, np.array(energy), np.array(area), Dt
