"""Thin object wrapper over the libvsav C ABI: one ``Handle`` = one device
state (two time levels + the Step-1 cache and work buffers) for R independent
runs holding V vesicle fields in total."""
from __future__ import annotations

import ctypes as ct
import warnings
from typing import Optional, Sequence

import numpy as np

from . import _lib as L


class VsavError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"libvsav error {code}: {msg}")
        self.code = code


class WCNegativeError(VsavError):
    """W_i + C_i < 0 (the reference raises error("FATAL: W + C < 0"), Utils.jl:162,180,188)."""


class NotConvergedWarning(UserWarning):
    """psi BiCGSTAB hit itmax (the reference's @warn, Solvers.jl:76)."""


PRECISION = {"fp64": 0, "fp32": 1, "mixed": 2}
PSI_FORM = {"full": 0, "half": 1}
PSI_PRECOND = {"diag": 0, "flex_diag": 1, "learned": 2}


class Handle:
    def __init__(self, cfg, precision: str = "fp64", psi_form: Optional[str] = None,
                 run_sizes: Optional[Sequence[int]] = None, psi_itmax: int = 20,
                 psi_rtol: Optional[float] = None, psi_atol: float = 1e-14, device: int = 0,
                 psi_precond: str = "diag", psi_net=None, graph: bool = True, psi3d_variable: bool = False,
                 psi_stop: str = "krylov", psi_check: bool = False):
        """cfg: any object with the reference Config fields (Types.jl:27-74);
        psi_in_v / psi_out_v hold one value per vesicle field of all runs.
        psi_precond: "diag" (the reference's left-preconditioned BiCGSTAB),
        "flex_diag" / "learned" (flexible right-preconditioned BiCGSTAB with the
        diagonal, or the diagonal plus the learned correction whose parameters
        psi_net gives: an array of 7409 values or a path to an .npz with
        "theta").  psi3d_variable: 3D Step 1 with the 2D scheme's variable psi
        mobility and BiCGSTAB instead of the reference's constant-mobility
        spectral division.  psi_stop: "krylov" (Krylov.jl's stop on the
        preconditioned residual, the reference) or "true" (stop on ||b - A x||).
        psi_check: measure ||b - A x|| / ||b|| of every psi system after each
        solve (true_residuals())."""
        self.lib = L.load()
        self.nd = 3 if getattr(cfg, "Nz", 0) else 2
        self.Nx, self.Ny = int(cfg.Nx), int(cfg.Ny)
        self.Nz = int(cfg.Nz) if self.nd == 3 else 1
        self.nkx = self.Nx // 2 + 1
        self.run_sizes = [int(cfg.N)] if run_sizes is None else [int(x) for x in run_sizes]
        self.R = len(self.run_sizes)
        self.V = int(sum(self.run_sizes))
        self.precision = precision
        self.psi_form = psi_form or "full"
        self._psi_in = np.ascontiguousarray(np.broadcast_to(np.asarray(cfg.psi_in_v, float), (self.V,)), dtype=np.float64)
        self._psi_out = np.ascontiguousarray(np.broadcast_to(np.asarray(cfg.psi_out_v, float), (self.V,)), dtype=np.float64)
        c = L.VsavConfig()
        c.ndim = self.nd
        c.Nx, c.Ny, c.Nz = self.Nx, self.Ny, self.Nz
        c.N = self.run_sizes[0]
        for k in ("epsilon", "M_phi", "M0_psi", "eta", "gamma_surf", "gamma_area", "gamma_bend", "gamma_in",
                  "beta_in", "gamma_out", "beta_out", "lamda", "S1", "S2", "S3", "S4", "C1", "C2", "C3",
                  "dt", "T", "Lx", "Ly", "tol"):
            setattr(c, k, float(getattr(cfg, k)))
        c.Lz = float(getattr(cfg, "Lz", 0.0) or 0.0)
        c.psi_in_v = L.dptr(self._psi_in)
        c.psi_out_v = L.dptr(self._psi_out)
        o = L.VsavOptions()
        self.lib.vsav_default_options(ct.byref(o), ct.byref(c))
        o.precision = PRECISION[precision]
        o.psi_form = PSI_FORM[self.psi_form]
        o.psi_precond = PSI_PRECOND[psi_precond]
        o.graph = 1 if graph else 0
        o.psi3d_variable = 1 if psi3d_variable else 0
        self.psi3d_variable = bool(psi3d_variable)
        o.psi_stop = {"krylov": 0, "true": 1}[psi_stop]
        o.psi_check = 1 if psi_check else 0
        self.psi_precond = psi_precond
        o.psi_itmax = psi_itmax
        o.psi_rtol = cfg.tol if psi_rtol is None else psi_rtol
        o.psi_atol = psi_atol
        o.n_runs = self.R
        self._rs = (ct.c_int32 * self.R)(*self.run_sizes)
        o.run_sizes = self._rs
        o.device = device
        h = ct.c_void_p()
        rc = self.lib.vsav_create(ct.byref(c), ct.byref(o), ct.byref(h))
        if rc != 0:
            raise VsavError(rc, self.lib.vsav_create_error().decode())
        self.h = h
        self.last_status = L.VsavStatus()
        if psi_net is not None:
            self.set_psi_net(psi_net)

    # -- lifetime -----------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            self.lib.vsav_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, rc):
        if rc < 0:
            msg = self.lib.vsav_last_error(self.h).decode()
            if rc == L.VSAV_E_WC_NEGATIVE:
                raise WCNegativeError(rc, msg)
            raise VsavError(rc, msg)
        if rc == L.VSAV_W_NOT_CONVERGED:
            warnings.warn(f"BiCGSTAB did not converge: max iters {self.last_status.psi_max_iters}, "
                          f"{self.last_status.psi_not_converged} of {self.last_status.psi_systems} systems",
                          NotConvergedWarning, stacklevel=3)
        return rc

    # -- shapes -------------------------------------------------------------
    @property
    def sp(self):
        return (self.Nz, self.Ny, self.Nx) if self.nd == 3 else (self.Ny, self.Nx)

    @property
    def hsp(self):
        return (self.Nz, self.Ny, self.nkx) if self.nd == 3 else (self.Ny, self.nkx)

    def field_shape(self, name):
        hat = name.endswith("_hat")
        s = self.hsp if hat else self.sp
        base = name[:-4] if hat else name
        if base == "u":
            return (self.R, self.nd) + s
        if base == "p":
            return (self.R,) + s
        return (self.V,) + s

    # -- state --------------------------------------------------------------
    def set_field(self, name, arr, level=0):
        dt = np.complex128 if name.endswith("_hat") else np.float64
        a = np.ascontiguousarray(np.asarray(arr, dtype=dt).reshape(self.field_shape(name)))
        self._chk(self.lib.vsav_set_field(self.h, level, L.FIELD_ID[name], L.dptr(a)))

    def get_field(self, name, level=0):
        dt = np.complex128 if name.endswith("_hat") else np.float64
        a = np.empty(self.field_shape(name), dtype=dt)
        self._chk(self.lib.vsav_get_field(self.h, level, L.FIELD_ID[name], L.dptr(a)))
        return a

    EXPORT = {"phi_sum": 0, "speed": 1}

    def export_f32(self, what: str, level: int = 0) -> np.ndarray:
        """Float32 frame computed on the device (vsav_export_f32): "phi_sum"
        (per run, the sum of its vesicle fields + N - 1, simulation.jl:124),
        "speed" (per run, |u|), or a physical field name ("phi", "psi", "mu",
        "nu", "u", "p") narrowed to float32."""
        if what in self.EXPORT:
            code, shape = self.EXPORT[what], (self.R,) + self.sp
        else:
            code, shape = 100 + L.FIELD_ID[what], self.field_shape(what)
        a = np.empty(shape, dtype=np.float32)
        self._chk(self.lib.vsav_export_f32(self.h, level, code, a.ctypes.data_as(ct.POINTER(ct.c_float))))
        return a

    def set_scalars(self, q4, level=0):
        a = np.ascontiguousarray(np.asarray(q4, dtype=np.float64).reshape(self.R, 4))
        self._chk(self.lib.vsav_set_scalars(self.h, level, L.dptr(a)))

    def get_scalars(self, level=0):
        a = np.empty((self.R, 4))
        self._chk(self.lib.vsav_get_scalars(self.h, level, L.dptr(a)))
        return a

    def set_dt(self, dt):
        a = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, float), (self.R,)), dtype=np.float64)
        self._chk(self.lib.vsav_set_dt(self.h, L.dptr(a)))

    def get_dt(self):
        a = np.empty(self.R)
        self._chk(self.lib.vsav_get_dt(self.h, L.dptr(a)))
        return a

    def set_A0(self, a0):
        a = np.ascontiguousarray(np.asarray(a0, dtype=np.float64).reshape(self.V))
        self._chk(self.lib.vsav_set_A0(self.h, L.dptr(a)))

    def get_A0(self):
        a = np.empty(self.V)
        self._chk(self.lib.vsav_get_A0(self.h, L.dptr(a)))
        return a

    def init_shapes(self, shapes):
        """Initial state from seeded shape parameters, evaluated on the device
        (2D): one dict per vesicle field with cx, cy, a, b, rot, psi_in, psi_out
        and modes [(m, amp, phase), ...] (at most 8); u = p = 0; then init_state."""
        if len(shapes) != self.V:
            raise ValueError(f"need {self.V} shapes, got {len(shapes)}")
        arr = (L.VsavShape2D * self.V)()
        for k, sh in enumerate(shapes):
            s = arr[k]
            for f in ("cx", "cy", "a", "b", "rot", "psi_in", "psi_out"):
                setattr(s, f, float(sh[f]))
            modes = list(sh.get("modes", []))
            if len(modes) > 8:
                raise ValueError("at most 8 modes per shape")
            s.nmodes = len(modes)
            for j, (m, amp, ph) in enumerate(modes):
                s.m[j], s.amp[j], s.phase[j] = int(m), float(amp), float(ph)
        self._chk(self.lib.vsav_init_shapes2d(self.h, arr))

    def generate_initial_condition(self, state_type: int, goal: str = "s", blob_u=None):
        """generate_initial_condition(conf, ops, state_type) (Init.jl:74-216,
        Init_3d.jl:67-152) on the device for every run, then init_state's
        initialisation.  goal: "g" or "s"; blob_u: for state_type 4, 20 uniform
        draws per run ([R][20], the reference's rand() calls in order)."""
        if goal not in ("g", "s"):
            raise ValueError(f"what's the goal? now it is {goal}")
        u = None
        if blob_u is not None:
            u = np.ascontiguousarray(blob_u, dtype=np.float64).reshape(-1)
            if u.size != 20 * self.R:
                raise ValueError(f"blob_u needs 20 draws per run ({20 * self.R}), got {u.size}")
        self._chk(self.lib.vsav_generate_initial_condition(self.h, int(state_type), ord(goal),
                                                           None if u is None else L.dptr(u)))

    def init_state(self, phi, psi, u=None, p=None):
        """generate_initial_condition's FFTs (Init.jl:199-216) + simulation.jl:22-53."""
        self.set_field("phi", phi)
        self.set_field("psi", psi)
        self.set_field("u", np.zeros(self.field_shape("u")) if u is None else u)
        self.set_field("p", np.zeros(self.field_shape("p")) if p is None else p)
        self._chk(self.lib.vsav_init_state(self.h, 0))

    # -- steps --------------------------------------------------------------
    def step1(self, n):
        rc = self.lib.vsav_step1(self.h, n, ct.byref(self.last_status))
        return self._chk(rc)

    def step2(self, n):
        self._chk(self.lib.vsav_step2(self.h, n))

    def step3(self):
        self._chk(self.lib.vsav_step3(self.h))

    def step4(self, n):
        self._chk(self.lib.vsav_step4(self.h, n))

    def step5(self, n):
        self._chk(self.lib.vsav_step5(self.h, n))

    def step6(self):
        self._chk(self.lib.vsav_step6(self.h))

    def step7(self, n):
        self._chk(self.lib.vsav_step7(self.h, n))

    def update_state(self):
        self._chk(self.lib.vsav_update_state(self.h))

    def run(self, n0, nsteps, dt=None, monitor=False):
        """nsteps full steps from step index n0; returns (energy, area_ratio) [nsteps][R] if monitor."""
        dtp = None
        if dt is not None:
            dta = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, float).reshape(-1, 1) if np.ndim(dt) == 1 else np.asarray(dt, float), (nsteps, self.R)), dtype=np.float64)
            dtp = L.dptr(dta)
        E = np.empty((nsteps, self.R)) if monitor else None
        A = np.empty((nsteps, self.R)) if monitor else None
        rc = self.lib.vsav_run(self.h, n0, nsteps, dtp, L.dptr(E) if monitor else None,
                               L.dptr(A) if monitor else None, ct.byref(self.last_status))
        self._chk(rc)
        return (E, A) if monitor else None

    def time_run(self, n0, nsteps, monitor=True):
        """nsteps full steps timed on the device with CUDA events (ms)."""
        ms = np.zeros(1)
        rc = self.lib.vsav_time_run(self.h, n0, nsteps, None, int(monitor), L.dptr(ms))
        if rc == L.VSAV_W_NOT_CONVERGED:
            warnings.warn(f"BiCGSTAB did not converge in at least one of the {nsteps} timed steps",
                          NotConvergedWarning, stacklevel=2)
        else:
            self._chk(rc)
        return float(ms[0])

    KCLASS = ("fft_cols", "fft_rows_r2c", "fft_rows_c2r", "fft_rows_c2c", "psi_rows_fused", "psi_combine",
              "pointwise", "psi_net", "fft_cols_f32")

    def profile(self, enable):
        self._chk(self.lib.vsav_profile(self.h, {True: 1, False: 0, "reset": 2}[enable]))

    def profile_read(self):
        out = {}
        for i, k in enumerate(self.KCLASS):
            a = np.zeros(3)
            self._chk(self.lib.vsav_profile_read(self.h, i, L.dptr(a)))
            out[k] = dict(launches=int(a[0]), ms=float(a[1]), bytes=float(a[2]))
        return out

    def monitor(self):
        E = np.empty(self.R)
        A = np.empty(self.R)
        self._chk(self.lib.vsav_monitor(self.h, L.dptr(E), L.dptr(A)))
        return E, A

    # -- intermediates ------------------------------------------------------
    CACHE = ("phi_11", "phi_12", "phi_13", "phi_14", "phi_21", "psi_11", "psi_12", "psi_21",
             "mu_11", "mu_12", "mu_13", "mu_14", "mu_21", "nu_11", "nu_12", "nu_21")
    STEP3 = ("phi_1_hat", "psi_1_hat", "phi_2_hat", "psi_2_hat", "mu_1_hat", "nu_1_hat", "mu_2_hat", "nu_2_hat")

    def get_cache(self, name):
        a = np.empty((self.V,) + self.hsp, dtype=np.complex128)
        self._chk(self.lib.vsav_get_work(self.h, 0, self.CACHE.index(name), L.dptr(a)))
        return a

    def get_step3(self, name):
        a = np.empty((self.V,) + self.hsp, dtype=np.complex128)
        self._chk(self.lib.vsav_get_work(self.h, 1, self.STEP3.index(name), L.dptr(a)))
        return a

    def get_u_tilde(self, idx, hat=False):
        shp = (self.R, self.nd) + (self.hsp if hat else self.sp)
        a = np.empty(shp, dtype=np.complex128 if hat else np.float64)
        self._chk(self.lib.vsav_get_work(self.h, 2 if hat else 3, idx, L.dptr(a)))
        return a

    def get_H(self, idx):
        a = np.empty((self.V,) + self.sp)
        self._chk(self.lib.vsav_get_work(self.h, 4, idx, L.dptr(a)))
        return a

    def scalar_work(self, what):
        n = {0: 6 * self.R, 1: self.R, 2: 2 * self.R, 3: self.V, 4: self.R, 5: 12 * self.R, 6: 3 * self.R}[what]
        a = np.empty(n)
        self._chk(self.lib.vsav_get_scalar_work(self.h, what, L.dptr(a)))
        return a

    def psi_stats(self):
        return self.scalar_work(5).reshape(3 * self.R, 4)

    def has_psi_solve(self):
        """True where Step 1 solves psi by BiCGSTAB (2D, or 3D with psi3d_variable)."""
        return self.nd == 2 or self.psi3d_variable

    def true_residuals(self):
        """||b - A x|| / ||b|| of each psi system of the last Step 1 (needs psi_check)."""
        return self.scalar_work(6)

    def tuning(self):
        """The FFT kernel variants this handle uses and where they came from
        (vsav_get_tuning), as a dict."""
        import json
        need = ct.c_int64()
        self._chk(self.lib.vsav_get_tuning(self.h, None, 0, ct.byref(need)))
        buf = ct.create_string_buffer(need.value)
        self._chk(self.lib.vsav_get_tuning(self.h, buf, need.value, ct.byref(need)))
        return json.loads(buf.value.decode())

    # -- transforms ---------------------------------------------------------
    def rfft(self, f):
        f = np.ascontiguousarray(np.asarray(f, dtype=np.float64))
        nf = f.size // int(np.prod(self.sp))
        out = np.empty((nf,) + self.hsp, dtype=np.complex128)
        self._chk(self.lib.vsav_transform(self.h, 0, nf, L.dptr(f), L.dptr(out)))
        return out.reshape(f.shape[:-self.nd] + self.hsp)

    def irfft(self, F, mult=None):
        F = np.ascontiguousarray(np.asarray(F, dtype=np.complex128))
        nf = F.size // int(np.prod(self.hsp))
        kind = 1 if mult is None else 10 + {"dx": 1, "dy": 2, "dz": 3, "lap": 4, "bih": 5}[mult]
        out = np.empty((nf,) + self.sp)
        self._chk(self.lib.vsav_transform(self.h, kind, nf, L.dptr(F), L.dptr(out)))
        return out.reshape(F.shape[:-self.nd] + self.sp)

    # -- learned psi preconditioner ----------------------------------------
    def set_psi_net(self, theta):
        """Network parameters of the learned psi preconditioner (array of 7409
        values or path of an .npz holding "theta")."""
        if isinstance(theta, str):
            theta = np.load(theta)["theta"]
        th = np.ascontiguousarray(theta, dtype=np.float64)
        if th.size != self.lib.vsav_net_nparams():
            raise ValueError("theta must hold %d values" % self.lib.vsav_net_nparams())
        self._chk(self.lib.vsav_set_psi_net(self.h, L.dptr(th)))

    def harvest(self, max_snapshots: int):
        """Keep the BiCGSTAB iterates of every later psi solve (0: off)."""
        self._chk(self.lib.vsav_psi_harvest(self.h, int(max_snapshots)))

    def harvest_read(self, out=None):
        """Iterates of the last psi solve: (x [K][3V][Ny][Nx], r [K][3V][Ny][Nx],
        x_star [3V][Ny][Nx], M [V][Ny][Nx]) as float32 arrays; physical real
        parts, r = M^-1 (b - A x_k).  With `out` (a device buffer address and
        its capacity in floats) the data is copied there instead and
        (nsnap, nfloats) is returned."""
        ns = ct.c_int32()
        nf = ct.c_int64()
        if out is not None:
            ptr, cap = out
            self._chk(self.lib.vsav_psi_harvest_read(self.h, ct.c_void_p(ptr), int(cap), ct.byref(ns), ct.byref(nf)))
            return ns.value, nf.value
        self._chk(self.lib.vsav_psi_harvest_read(self.h, None, 0, ct.byref(ns), ct.byref(nf)))
        buf = np.empty(nf.value, np.float32)
        self._chk(self.lib.vsav_psi_harvest_read(self.h, buf.ctypes.data_as(ct.c_void_p), buf.size, ct.byref(ns),
                                                 ct.byref(nf)))
        K, F, P = ns.value, 3 * self.V, self.Nx * self.Ny
        xr = buf[:2 * K * F * P].reshape(K, 2, F, self.Ny, self.Nx)
        xs = buf[2 * K * F * P:(2 * K + 1) * F * P].reshape(F, self.Ny, self.Nx)
        M = buf[(2 * K + 1) * F * P:].reshape(self.V, self.Ny, self.Nx)
        return xr[:, 0], xr[:, 1], xs, M
