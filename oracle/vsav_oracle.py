"""CPU FP64 restatement of the reference pseudo-spectral SAV time step.

TEST INFRASTRUCTURE ONLY.  This module is the oracle that the CUDA library is
checked against.  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU
baseline legs of ``bench.py`` may import it; the product path never does.

It restates, in NumPy float64 on pocketfft (``numpy.fft``), the algorithm of
Forstylime/Julia-Vesicles-growth-and-shrinkage:

* ``src/Types.jl`` / ``src/Types_3d.jl``        -- Config, FieldState, BDF coeffs
* ``src/SpectralUtils.jl`` / ``..._3d.jl``      -- wavenumbers, D1, Laplacian ...
* ``src/Utils.jl`` / ``src/Utils_3d.jl``        -- energy densities, W1..W3, H1..H3, MG
* ``src/Solvers.jl`` / ``src/Solvers_3d.jl``    -- solve_step1 .. solve_step7
* ``src/simulation.jl``                         -- initialisation + loop body
* ``src/Init.jl`` / ``src/Init_3d.jl``          -- set_para_base defaults

Array layout is C order with x fastest: a Julia ``(Nx, Ny, N)`` array is a NumPy
``[N][Ny][Nx]`` array (3D: ``[N][Nz][Ny][Nx]``), half spectra are
``[N][Ny][Nx//2+1]``.  The c2r convention is the one FFTW and pocketfft share:
complex inverse along y (and z) first, then a 1-D c2r along x that uses only the
real part of the kx=0 and kx=Nx/2 bins.

Third-party arithmetic that is not vendored in the reference:

* FFTW.jl 1.10.0 / FFTW_jll 3.3.11 (Manifest.toml:372-382): replaced by pocketfft.
* Krylov.jl 0.10.6 ``bicgstab`` (Manifest.toml:852-856, call site
  src/Solvers.jl:73-75): restated below from its published algorithm
  (left preconditioner M applied by multiplication, shadow vector c = b,
  x0 = 0, stop when ||M^-1 r|| <= atol + rtol*||M^-1 b|| or after itmax).
  No reference test exercises it, so this part of the oracle is pinned only
  by the operator-level known-answer tests of test/test_Types_Ops.jl.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, replace
from typing import Optional

import numpy as np

SQ2 = math.sqrt(2.0)


# ---------------------------------------------------------------------------
# instrumentation: counts the reference's logical operations so algorithmic
# bytes per step can be derived (transform count, pointwise passes, psi iters)
# ---------------------------------------------------------------------------
class OpCounter:
    def __init__(self):
        self.reset()

    def reset(self):
        self.rfft = 0          # number of real fields (per N-batch element) forward
        self.irfft = 0
        self.cfft = 0          # full complex transforms (per vesicle field)
        self.psi_iters = []    # BiCGSTAB iteration counts per solve
        self.psi_solved = []

    def as_dict(self):
        return dict(rfft=self.rfft, irfft=self.irfft, cfft=self.cfft,
                    psi_iters=list(self.psi_iters), psi_solved=list(self.psi_solved))


# ---------------------------------------------------------------------------
# Config  (src/Types.jl:27-134, src/Types_3d.jl:27-140)
# ---------------------------------------------------------------------------
@dataclass
class Config:
    N: int
    epsilon: float
    M_phi: float
    M0_psi: float
    eta: float
    gamma_surf: float
    gamma_area: float
    gamma_bend: float
    gamma_in: float
    beta_in: float
    psi_in_v: np.ndarray
    gamma_out: float
    beta_out: float
    psi_out_v: np.ndarray
    lamda: float
    S1: float
    S2: float
    S3: float
    S4: float
    C1: float
    C2: float
    C3: float
    dt: float
    T: float
    Nx: int
    Ny: int
    Lx: float
    Ly: float
    tol: float
    goal: str = "s"
    Nz: int = 0          # 0 => 2D
    Lz: float = 0.0
    # derived (Types.jl:113-117)
    Nt: int = field(init=False)
    dx: float = field(init=False)
    dy: float = field(init=False)
    dz: float = field(init=False)
    spe_len: int = field(init=False)

    def __post_init__(self):
        self.psi_in_v = np.asarray(self.psi_in_v, dtype=np.float64)
        self.psi_out_v = np.asarray(self.psi_out_v, dtype=np.float64)
        self.Nt = int(round(self.T / self.dt))
        self.dx = self.Lx / self.Nx
        self.dy = self.Ly / self.Ny
        self.dz = self.Lz / self.Nz if self.Nz else 1.0
        nz = self.Nz if self.Nz else 1
        self.spe_len = (self.Nx // 2 + 1) * self.Ny * nz * self.N

    @property
    def ndim(self):
        return 3 if self.Nz else 2

    @property
    def shape(self):          # spatial shape, C order
        return (self.Nz, self.Ny, self.Nx) if self.Nz else (self.Ny, self.Nx)

    @property
    def hshape(self):
        return (self.Nz, self.Ny, self.Nx // 2 + 1) if self.Nz else (self.Ny, self.Nx // 2 + 1)

    @property
    def cell(self):           # dx*dy(*dz): integrate() weight (Utils.jl:26)
        return self.dx * self.dy * (self.dz if self.Nz else 1.0)


def set_para_base(dt: float, T: float, ndim: int = 2) -> Config:
    """Reference defaults: src/Init.jl:8-69 (2D), src/Init_3d.jl:8-62 (3D)."""
    eps, gb = 0.01, 0.1
    gin = gout = 1e5
    if ndim == 2:
        goal, N, nx, L = "s", 1, 256, 1.0
        psi_in = [0.65] if goal == "g" else [0.1]
    else:
        goal, N, nx, L = "g", 1, 128, 1.0
        psi_in = [0.1] if goal == "s" else [0.65]
    return Config(
        N=N, epsilon=eps, M_phi=1.0, M0_psi=0.5, eta=1.0, gamma_surf=1.0,
        gamma_area=5e4, gamma_bend=gb, gamma_in=gin, beta_in=0.0, psi_in_v=psi_in,
        gamma_out=gout, beta_out=0.0, psi_out_v=[0.8], lamda=1.0,
        S1=(3 * SQ2 / 8) * eps * gb, S2=0.0, S3=gb / eps ** 3, S4=min(gin, gout),
        C1=1.0, C2=5.0e5, C3=1.0e6, dt=dt, T=T, Nx=nx, Ny=nx, Lx=L, Ly=L,
        tol=1e-12, goal=goal, Nz=(nx if ndim == 3 else 0), Lz=(L if ndim == 3 else 0.0))


# ---------------------------------------------------------------------------
# BDF coefficients (src/Types.jl:407-426)
# ---------------------------------------------------------------------------
@dataclass(frozen=True)
class BDFCoeff:
    a: float
    b: float
    c: float


def bdf_coeff(n: int) -> BDFCoeff:
    return BDFCoeff(1.0, -1.0, 0.0) if n == 1 else BDFCoeff(1.5, -2.0, 0.5)


# ---------------------------------------------------------------------------
# FieldState (src/Types.jl:167-265)
# ---------------------------------------------------------------------------
@dataclass
class FieldState:
    phi: np.ndarray
    phi_hat: np.ndarray
    psi: np.ndarray
    psi_hat: np.ndarray
    u: np.ndarray
    u_hat: np.ndarray
    p: np.ndarray
    p_hat: np.ndarray
    mu: np.ndarray
    mu_hat: np.ndarray
    nu: np.ndarray
    nu_hat: np.ndarray
    Q: float = 0.0
    R1: float = 0.0
    R2: float = 0.0
    R3: float = 0.0
    A0: np.ndarray = field(default_factory=lambda: np.zeros(1))
    dt: float = 0.0

    def copy(self):
        return FieldState(**{k: (v.copy() if isinstance(v, np.ndarray) else v)
                             for k, v in self.__dict__.items()})


def update_state(dest: FieldState, src: FieldState) -> FieldState:
    """src/Types.jl:243-265: arrays + Q,R1..R3 copied; A0 and dt are NOT copied."""
    for k in ("phi", "phi_hat", "psi", "psi_hat", "u", "u_hat", "p", "p_hat",
              "mu", "mu_hat", "nu", "nu_hat"):
        getattr(dest, k)[...] = getattr(src, k)
    dest.Q, dest.R1, dest.R2, dest.R3 = src.Q, src.R1, src.R2, src.R3
    return dest


# ---------------------------------------------------------------------------
# Operators (src/SpectralUtils.jl:36-118, src/SpectralUtils_3d.jl:36-124)
# ---------------------------------------------------------------------------
class Operators:
    def __init__(self, cfg: Config, counter: Optional[OpCounter] = None, workers: Optional[int] = None):
        self.cfg = cfg
        self.workers = workers
        self.counter = counter or OpCounter()
        nd = cfg.ndim
        # 2*pi*rfftfreq(Nx, Nx/Lx): Nyquist POSITIVE (SpectralUtils.jl:42)
        kx = 2 * np.pi * np.fft.rfftfreq(cfg.Nx, d=cfg.Lx / cfg.Nx)
        # 2*pi*fftfreq(Nx, Nx/Lx): Nyquist NEGATIVE (SpectralUtils.jl:43)
        kx0 = 2 * np.pi * np.fft.fftfreq(cfg.Nx, d=cfg.Lx / cfg.Nx)
        ky = 2 * np.pi * np.fft.fftfreq(cfg.Ny, d=cfg.Ly / cfg.Ny)
        if nd == 2:
            self.kx = kx.reshape(1, -1)
            self.kx0 = kx0.reshape(1, -1)
            self.ky = ky.reshape(-1, 1)
            self.kz = None
            K2 = self.kx ** 2 + self.ky ** 2
            self.D1 = (1j * self.kx, 1j * self.ky)
            self.D1_full = (1j * self.kx0, 1j * self.ky)
            self.Laplacian = -K2
            self.Laplacian_full = -(self.kx0 ** 2 + self.ky ** 2)
            self.Biharmonic = K2 ** 2
        else:
            kz = 2 * np.pi * np.fft.fftfreq(cfg.Nz, d=cfg.Lz / cfg.Nz)
            self.kx = kx.reshape(1, 1, -1)
            self.kx0 = kx0.reshape(1, 1, -1)
            self.ky = ky.reshape(1, -1, 1)
            self.kz = kz.reshape(-1, 1, 1)
            self.D1 = (1j * self.kx, 1j * self.ky, 1j * self.kz)
            self.D1_full = (1j * self.kx0, 1j * self.ky, 1j * self.kz)
            self.Laplacian = -(self.kx ** 2 + self.ky ** 2 + self.kz ** 2)
            self.Laplacian_full = -(self.kx0 ** 2 + self.ky ** 2 + self.kz ** 2)
            self.Biharmonic = self.Laplacian ** 2
        self.K = (self.kx, self.ky) if nd == 2 else (self.kx, self.ky, self.kz)
        self.axes = tuple(range(-nd, 0))
        self.inv_s = 1.0 / float(np.prod(cfg.shape))

    # --- transforms (to_spectral!/to_physical!, SpectralUtils.jl:132-148) ---
    def _nb(self, a, nd):
        return int(np.prod(a.shape[:-nd])) if a.ndim > nd else 1

    # numpy.fft and scipy.fft are both pocketfft; scipy's takes a thread count
    def _mod(self):
        if self.workers:
            import scipy.fft as sf
            return sf, dict(workers=self.workers)
        return np.fft, {}

    def rfft(self, f):
        self.counter.rfft += self._nb(f, self.cfg.ndim)
        m, kw = self._mod()
        return m.rfftn(f, axes=self.axes, **kw)

    def irfft(self, F):
        self.counter.irfft += self._nb(F, self.cfg.ndim)
        m, kw = self._mod()
        return m.irfftn(F, s=self.cfg.shape, axes=self.axes, **kw)

    def fft(self, f):
        self.counter.cfft += self._nb(f, self.cfg.ndim)
        m, kw = self._mod()
        return m.fftn(f, axes=self.axes, **kw)

    def ifft(self, F):
        self.counter.cfft += self._nb(F, self.cfg.ndim)
        m, kw = self._mod()
        return m.ifftn(F, axes=self.axes, **kw)


def build_operators(cfg: Config, counter: Optional[OpCounter] = None, workers: Optional[int] = None) -> Operators:
    return Operators(cfg, counter, workers)


def mult(u_hat, v_hat, ops: Operators):
    """SpectralUtils.jl:158-167: product of two fields given by their spectra."""
    return ops.rfft(ops.irfft(u_hat) * ops.irfft(v_hat))


# ---------------------------------------------------------------------------
# Utils (src/Utils.jl, src/Utils_3d.jl)
# ---------------------------------------------------------------------------
def g(phi):                 # Utils.jl:8
    return 0.25 * (phi ** 2 - 1.0) ** 2


def g_prime(phi):           # Utils.jl:11
    return phi * (phi ** 2 - 1.0)


def p_phi(phi):             # Utils.jl:14
    return -0.5 * phi ** 3 + 1.5 * phi


def p_phi_prime(phi):       # Utils.jl:17
    return -1.5 * phi ** 2 + 1.5


def get_M_psi(phi, cfg):    # Utils.jl:20
    return 0.1 * (1.0 - cfg.M0_psi * (phi ** 2 - 1.0) ** 2)


def integrate(f, cfg):      # Utils.jl:26
    return float(np.sum(f)) * cfg.cell


def integrate_sq(f, cfg):   # Utils.jl:29
    return float(np.sum(np.abs(f) ** 2)) * cfg.cell


def _vshape(cfg, v):        # reshape(conf.psi_in_v, 1, 1, :) -> broadcast over [N][...]
    return np.asarray(v).reshape((-1,) + (1,) * cfg.ndim)


def f_surf(phi, ops, cfg):
    """Utils.jl:36-42.  The 3D file (Utils_3d.jl:36-42) also uses only d/dx, d/dy."""
    ph = ops.rfft(phi)
    gx = ops.irfft(ops.D1[0] * ph)
    gy = ops.irfft(ops.D1[1] * ph)
    e = cfg.epsilon
    return (3 * SQ2 / 4) * (g(phi) / e) + e * (gx ** 2 + gy ** 2) / 2


def f_bend(phi, ops, cfg):
    """Utils.jl:45-50."""
    ph = ops.rfft(phi)
    e = cfg.epsilon
    lap = ops.irfft(ops.Laplacian * ph)
    return (3 * SQ2 / (16 * e)) * (g_prime(phi) / e - e * lap) ** 2


def f_osmotic(phi, psi, cfg):
    """Utils.jl:53-60."""
    P = p_phi(phi)
    pin, pout = _vshape(cfg, cfg.psi_in_v), _vshape(cfg, cfg.psi_out_v)
    f_in = 0.5 * cfg.gamma_in * (psi - pin) ** 2 + cfg.beta_in
    f_out = 0.5 * cfg.gamma_out * (psi - pout) ** 2 + cfg.beta_out
    return ((1 + P) / 2) * f_in + ((1 - P) / 2) * f_out


def calculate_area(phi, ops, cfg):
    """Utils.jl:66-73: per-vesicle integral of f_surf."""
    surf = f_surf(phi, ops, cfg)
    return np.array([integrate(surf[n], cfg) for n in range(cfg.N)])


def compute_modified_energy(present: FieldState, old: FieldState, ops, cfg):
    """Utils.jl:96-141 (Utils_3d.jl:96-141 is identical: no z terms in the
    pressure and S2 parts)."""
    kinetic = 0.25 * integrate_sq(present.u, cfg) + 0.25 * integrate_sq(2 * present.u - old.u, cfg)
    gpx = ops.irfft(ops.D1[0] * present.p_hat)
    gpy = ops.irfft(ops.D1[1] * present.p_hat)
    pressure = (present.dt ** 2 / 3.0) * (integrate_sq(gpx, cfg) + integrate_sq(gpy, cfg))

    def se(rn, ro):
        return 0.5 * rn ** 2 + 0.5 * (2 * rn - ro) ** 2
    R_energy = se(present.R1, old.R1) + se(present.R2, old.R2) + se(present.R3, old.R3)
    Q_energy = 0.5 * se(present.Q, old.Q)
    phi_star = 2 * present.phi - old.phi
    psi_star = 2 * present.psi - old.psi
    phi_star_hat = 2 * present.phi_hat - old.phi_hat
    lap_new = ops.irfft(ops.Laplacian * present.phi_hat)
    lap_star = ops.irfft(ops.Laplacian * phi_star_hat)
    gx_new = ops.irfft(ops.D1[0] * present.phi_hat)
    gy_new = ops.irfft(ops.D1[1] * present.phi_hat)
    gx_star = ops.irfft(ops.D1[0] * phi_star_hat)
    gy_star = ops.irfft(ops.D1[1] * phi_star_hat)
    S1t = 0.25 * cfg.S1 * (integrate_sq(lap_new, cfg) + integrate_sq(lap_star, cfg))
    S2t = 0.25 * cfg.S2 * (integrate_sq(gx_new, cfg) + integrate_sq(gy_new, cfg)
                           + integrate_sq(gx_star, cfg) + integrate_sq(gy_star, cfg))
    S3t = 0.25 * cfg.S3 * (integrate_sq(present.phi, cfg) + integrate_sq(phi_star, cfg))
    S4t = 0.25 * cfg.S4 * (integrate_sq(present.psi, cfg) + integrate_sq(psi_star, cfg))
    return (kinetic + pressure + cfg.lamda * R_energy + Q_energy
            + cfg.lamda * (S1t + S2t + S3t + S4t)
            - cfg.lamda * (cfg.C1 + cfg.C2 + cfg.C3) - 0.5)


def get_omega(phi, ops, cfg):
    """Utils.jl:148-153."""
    ph = ops.rfft(phi)
    e = cfg.epsilon
    lap = ops.irfft(ops.Laplacian * ph)
    return (phi ** 3 - phi) / e - e * lap


class WCNegative(RuntimeError):
    """Utils.jl:162,180,188: error("FATAL: W + C < 0")."""


def get_W1(phi, ops, cfg, A0):
    """Utils.jl:159-164."""
    A = calculate_area(phi, ops, cfg)
    W1 = float(np.sum(0.5 * cfg.gamma_area * (A - A0) ** 2))
    if W1 + cfg.C1 < 0:
        raise WCNegative(f"FATAL: W1 + C1 < 0, W1 = {W1}")
    return W1


def get_W2(phi, ops, cfg):
    """Utils.jl:166-182.  E2 uses only the x and y gradients in 3D as well."""
    ph = ops.rfft(phi)
    Fs = cfg.gamma_surf * integrate(f_surf(phi, ops, cfg), cfg)
    Fb = cfg.gamma_bend * integrate(f_bend(phi, ops, cfg), cfg)
    lap = ops.irfft(ops.Laplacian * ph)
    gx = ops.irfft(ops.D1[0] * ph)
    gy = ops.irfft(ops.D1[1] * ph)
    E2 = integrate(0.5 * cfg.S1 * lap ** 2 + 0.5 * cfg.S2 * (gx ** 2 + gy ** 2)
                   + 0.5 * cfg.S3 * phi ** 2, cfg)
    W2 = Fs + Fb - E2
    if W2 + cfg.C2 < 0:
        raise WCNegative(f"FATAL: W2 + C2 < 0, W2 = {W2}")
    return W2


def get_W3(phi, psi, cfg):
    """Utils.jl:184-190."""
    W_osm = integrate(f_osmotic(phi, psi, cfg), cfg)
    E3 = 0.5 * cfg.S4 * integrate_sq(psi, cfg)
    W3 = W_osm - E3
    if W3 + cfg.C3 < 0:
        raise WCNegative(f"FATAL: W3 + C3 < 0, W3 = {W3}")
    return W3


def get_H1(phi, ops, cfg, A0):
    """Utils.jl:198-206."""
    W1 = get_W1(phi, ops, cfg, A0)
    R1 = math.sqrt(W1 + cfg.C1)
    A = calculate_area(phi, ops, cfg)
    omega = get_omega(phi, ops, cfg)
    factor = cfg.gamma_area * (A - A0) * (3 * SQ2 / 4)
    return (_vshape(cfg, factor) * omega) / R1


def get_H2(phi, ops, cfg):
    """Utils.jl:208-226."""
    ph = ops.rfft(phi)
    W2 = get_W2(phi, ops, cfg)
    R2 = math.sqrt(W2 + cfg.C2)
    e = cfg.epsilon
    omega = get_omega(phi, ops, cfg)
    oh = ops.rfft(omega)
    lap_omega = ops.irfft(ops.Laplacian * oh)
    H2_sb = (cfg.gamma_surf * (3 * SQ2 / 4) * omega
             + cfg.gamma_bend * (3 * SQ2 / (8 * e)) * (omega * (3 * phi ** 2 - 1) / e - e * lap_omega))
    bih = ops.irfft(ops.Biharmonic * ph)
    lap = ops.irfft(ops.Laplacian * ph)
    H2_lin = cfg.S1 * bih - cfg.S2 * lap + cfg.S3 * phi
    return (H2_sb - H2_lin) / R2


def get_H3(phi, psi, cfg):
    """Utils.jl:228-236."""
    W3 = get_W3(phi, psi, cfg)
    R3 = math.sqrt(W3 + cfg.C3)
    pin, pout = _vshape(cfg, cfg.psi_in_v), _vshape(cfg, cfg.psi_out_v)
    f_in = 0.5 * cfg.gamma_in * (psi - pin) ** 2 + cfg.beta_in
    f_out = 0.5 * cfg.gamma_out * (psi - pout) ** 2 + cfg.beta_out
    return (0.5 * p_phi_prime(phi) * (f_in - f_out)) / R3


def get_MG(phi, psi, cfg):
    """Utils.jl:238-248."""
    W3 = get_W3(phi, psi, cfg)
    R3 = math.sqrt(W3 + cfg.C3)
    P = p_phi(phi)
    pin, pout = _vshape(cfg, cfg.psi_in_v), _vshape(cfg, cfg.psi_out_v)
    dF_in = cfg.gamma_in * (psi - pin)
    dF_out = cfg.gamma_out * (psi - pout)
    G1 = 0.5 * (1 + P) * dF_in + 0.5 * (1 - P) * dF_out
    G2 = cfg.S4 * psi
    return (G1 - G2) / R3


# ---------------------------------------------------------------------------
# Krylov.jl 0.10.6 bicgstab, restated (call site src/Solvers.jl:73-75)
# ---------------------------------------------------------------------------
@dataclass
class KrylovStats:
    niter: int
    solved: bool
    status: str
    rNorms: list


def bicgstab(A, b, M=None, atol=1e-14, rtol=1e-12, itmax=20):
    """Preconditioned BiCGSTAB with x0 = 0, shadow vector c = b and the
    preconditioner M applied on the left by multiplication (ldiv = false),
    so the residual that is tracked and tested is M^-1 (b - A x).
    Inner products are conjugate-linear in the first argument."""
    n = b.size
    c = b
    x = np.zeros_like(b)
    r = M(b) if M is not None else b.copy()
    p = r.copy()
    rNorm = float(np.linalg.norm(r))
    rNorms = [rNorm]
    if rNorm == 0:
        return x, KrylovStats(0, True, "x = 0 is a zero-residual solution", rNorms)
    if itmax == 0:
        itmax = 2 * n
    eps = atol + rtol * rNorm
    next_rho = np.vdot(c, r)
    if next_rho == 0:
        return x, KrylovStats(0, False, "Breakdown bᴴc = 0", rNorms)
    solved = rNorm <= eps
    iters = 0
    tired = iters >= itmax
    breakdown = False
    while not (solved or tired or breakdown):
        iters += 1
        rho = next_rho
        y = p
        q = A(y)
        v = M(q) if M is not None else q
        alpha = rho / np.vdot(c, v)
        s = r - alpha * v
        x = x + alpha * y
        z = s
        d = A(z)
        t = M(d) if M is not None else d
        omega = np.vdot(t, s) / np.vdot(t, t)
        x = x + omega * z
        r = s - omega * t
        next_rho = np.vdot(c, r)
        beta = (next_rho / rho) * (alpha / omega)
        p = r + beta * (p - omega * v)
        rNorm = float(np.linalg.norm(r))
        rNorms.append(rNorm)
        resid_decrease_mach = (rNorm + 1.0 <= 1.0)
        solved = (rNorm <= eps) or resid_decrease_mach
        tired = iters >= itmax
        breakdown = (alpha == 0) or np.isnan(alpha)
    if solved:
        status = "solution good enough given atol and rtol"
    elif breakdown:
        status = "breakdown αₖ == 0"
    else:
        status = "maximum number of iterations exceeded"
    return x, KrylovStats(iters, bool(solved), status, rNorms)


# ---------------------------------------------------------------------------
# Step 1 cache (src/Types.jl:358-385)
# ---------------------------------------------------------------------------
STEP1_FIELDS = ("phi_11", "mu_11", "psi_11", "nu_11", "phi_12", "mu_12", "psi_12", "nu_12",
                "phi_13", "mu_13", "phi_14", "mu_14", "phi_21", "mu_21", "psi_21", "nu_21")


class Step1Cache(dict):
    def __getattr__(self, k):
        return self[k]


# ---------------------------------------------------------------------------
# Solvers (src/Solvers.jl, src/Solvers_3d.jl)
# ---------------------------------------------------------------------------
class Oracle:
    """Holds cfg/ops and exposes solve_step1..7 with the reference's argument
    meaning.  ``psi_solver_opts`` overrides the BiCGSTAB tolerances (the
    reference uses atol=1e-14, rtol=cfg.tol, itmax=20)."""

    def __init__(self, cfg: Config, psi_atol=1e-14, psi_rtol=None, psi_itmax=20,
                 counter: Optional[OpCounter] = None, workers: Optional[int] = None,
                 psi3d_variable: bool = False):
        self.cfg = cfg
        self.ops = build_operators(cfg, counter, workers)
        self.psi_atol = psi_atol
        self.psi_rtol = cfg.tol if psi_rtol is None else psi_rtol
        self.psi_itmax = psi_itmax
        self.last_psi_stats = []
        # 3D with the 2D scheme's variable mobility M_psi(phi*) and its BiCGSTAB
        # (an extension: Solvers_3d.jl:28-30 use the constant M0_psi)
        self.psi3d_variable = psi3d_variable

    @property
    def counter(self):
        return self.ops.counter

    # -- step 1 ------------------------------------------------------------
    def solve_step1(self, present: FieldState, old: FieldState, bdf: BDFCoeff) -> Step1Cache:
        cfg, ops = self.cfg, self.ops
        if cfg.ndim == 3:
            return self._solve_step1_3d(present, old, bdf)
        dt = present.dt
        a, b, c = bdf.a, bdf.b, bdf.c
        A0 = present.A0
        phi_star = 2.0 * present.phi - old.phi                     # Solvers.jl:21-24
        psi_star = 2.0 * present.psi - old.psi
        phi_star_hat = 2.0 * present.phi_hat - old.phi_hat
        psi_star_hat = 2.0 * present.psi_hat - old.psi_hat
        M_psi = get_M_psi(phi_star, cfg)                           # :26-27
        M_max = float(np.max(M_psi))
        L_phi = cfg.S1 * ops.Biharmonic - cfg.S2 * ops.Laplacian + cfg.S3   # :28
        L_psi = cfg.S4
        lhs_phi = (a / dt) + cfg.M_phi * L_phi                     # :30
        D1f = ops.D1_full
        a_dt = a / dt

        def A_psi(xv):                                              # :39-53
            x = xv.reshape((cfg.N,) + cfg.shape)
            b1 = L_psi * x
            b2 = D1f[0] * b1
            b3 = D1f[1] * b1
            b4 = ops.ifft(b2)
            b5 = ops.ifft(b3)
            b4 = M_psi * b4
            b5 = M_psi * b5
            b2 = ops.fft(b4)
            b3 = ops.fft(b5)
            y = a_dt * x - (D1f[0] * b2 + D1f[1] * b3)
            return y.reshape(-1)

        P_inv_diag = 1.0 / (a_dt - M_max * ops.Laplacian_full * L_psi)   # :57

        def prec(rv):                                               # :59-64
            return (rv.reshape((cfg.N,) + cfg.shape) * P_inv_diag).reshape(-1)

        nkx = cfg.Nx // 2 + 1

        def solve_psi(rhs_rhat):                                    # :68-81
            rhs_phys = ops.irfft(rhs_rhat)
            rhs_full = ops.fft(rhs_phys)
            sol, st = bicgstab(A_psi, rhs_full.reshape(-1), M=prec, atol=self.psi_atol,
                               rtol=self.psi_rtol, itmax=self.psi_itmax)
            self.last_psi_stats.append(st)
            ops.counter.psi_iters.append(st.niter)
            ops.counter.psi_solved.append(st.solved)
            return sol.reshape((cfg.N,) + cfg.shape)[..., :nkx].copy()

        self.last_psi_stats = []
        cache = Step1Cache()
        # 11  (:86-92)
        rh = -(b * present.phi_hat + c * old.phi_hat) / dt
        cache["phi_11"] = rh / lhs_phi
        cache["mu_11"] = L_phi * cache.phi_11
        rh = -(b * present.psi_hat + c * old.psi_hat) / dt
        cache["psi_11"] = solve_psi(rh)
        cache["nu_11"] = L_psi * cache.psi_11
        # 12  (:95-107)
        H1h = ops.rfft(get_H1(phi_star, ops, cfg, A0))
        cache["phi_12"] = (-cfg.M_phi * H1h) / lhs_phi
        cache["mu_12"] = L_phi * cache.phi_12 + H1h
        Gh = ops.rfft(get_MG(phi_star, psi_star, cfg))
        gGx = ops.irfft(ops.D1[0] * Gh)
        gGy = ops.irfft(ops.D1[1] * Gh)
        t2 = ops.rfft(M_psi * gGx)
        t3 = ops.rfft(M_psi * gGy)
        rh = ops.D1[0] * t2 + ops.D1[1] * t3
        cache["psi_12"] = solve_psi(rh)
        cache["nu_12"] = L_psi * cache.psi_12 + Gh
        # 13 & 14  (:110-115)
        H2h = ops.rfft(get_H2(phi_star, ops, cfg))
        H3h = ops.rfft(get_H3(phi_star, psi_star, cfg))
        cache["phi_13"] = (-cfg.M_phi * H2h) / lhs_phi
        cache["phi_14"] = (-cfg.M_phi * H3h) / lhs_phi
        cache["mu_13"] = L_phi * cache.phi_13 + H2h
        cache["mu_14"] = L_phi * cache.phi_14 + H3h
        # 21  (:118-134)
        u_star = 2.0 * present.u - old.u
        gx = ops.irfft(ops.D1[0] * phi_star_hat)
        gy = ops.irfft(ops.D1[1] * phi_star_hat)
        t = u_star[0] * gx + u_star[1] * gy
        th = ops.rfft(t)
        cache["phi_21"] = -th / lhs_phi
        cache["mu_21"] = L_phi * cache.phi_21
        gx = ops.irfft(ops.D1[0] * psi_star_hat)
        gy = ops.irfft(ops.D1[1] * psi_star_hat)
        t = u_star[0] * gx + u_star[1] * gy
        th = ops.rfft(t)
        cache["psi_21"] = solve_psi(-th)
        cache["nu_21"] = L_psi * cache.psi_21
        return cache

    def _psi_solver_3d(self, M_psi, a_dt):
        """The 2D psi solve (Solvers.jl:39-81) restated on 3D full spectra:
        A x = a_dt x - sum_d D1_full[d] F(M_psi F^-1(D1_full[d] S4 x)), d = x, y, z,
        diagonal preconditioner 1/(a_dt - M_max S4 Laplacian_full), Krylov.jl
        BiCGSTAB, solution truncated to the half spectrum."""
        cfg, ops = self.cfg, self.ops
        D1f = ops.D1_full
        L_psi = cfg.S4
        M_max = float(np.max(M_psi))
        P_inv_diag = 1.0 / (a_dt - M_max * ops.Laplacian_full * L_psi)
        shp = (cfg.N,) + cfg.shape
        nkx = cfg.Nx // 2 + 1

        def A_psi(xv):
            x = xv.reshape(shp)
            b1 = L_psi * x
            acc = 0
            for d in range(3):
                acc = acc + D1f[d] * ops.fft(M_psi * ops.ifft(D1f[d] * b1))
            return (a_dt * x - acc).reshape(-1)

        def prec(rv):
            return (rv.reshape(shp) * P_inv_diag).reshape(-1)

        def solve(rhs_rhat):
            rhs_full = ops.fft(ops.irfft(rhs_rhat))
            sol, st = bicgstab(A_psi, rhs_full.reshape(-1), M=prec, atol=self.psi_atol,
                               rtol=self.psi_rtol, itmax=self.psi_itmax)
            self.last_psi_stats.append(st)
            ops.counter.psi_iters.append(st.niter)
            ops.counter.psi_solved.append(st.solved)
            return sol.reshape(shp)[..., :nkx].copy()
        return solve

    def _solve_step1_3d(self, present, old, bdf):
        """Solvers_3d.jl:14-92: psi by spectral division with constant M0_psi;
        with psi3d_variable, the 2D scheme's M_psi(phi*) (Utils_3d.jl:20) and
        its BiCGSTAB (Solvers.jl:26-81) instead."""
        cfg, ops = self.cfg, self.ops
        dt = present.dt
        a, b, c = bdf.a, bdf.b, bdf.c
        A0 = present.A0
        phi_star = 2.0 * present.phi - old.phi
        psi_star = 2.0 * present.psi - old.psi
        phi_star_hat = 2.0 * present.phi_hat - old.phi_hat
        psi_star_hat = 2.0 * present.psi_hat - old.psi_hat
        L_phi = cfg.S1 * ops.Biharmonic - cfg.S2 * ops.Laplacian + cfg.S3
        L_psi = cfg.S4
        lhs_phi = (a / dt) + cfg.M_phi * L_phi
        if self.psi3d_variable:
            M_psi = get_M_psi(phi_star, cfg)
            self.last_psi_stats = []
            psi_div = self._psi_solver_3d(M_psi, a / dt)
        else:
            M_psi = cfg.M0_psi
            lhs_psi = (a / dt) - cfg.M0_psi * L_psi * ops.Laplacian

            def psi_div(rh):
                return rh / lhs_psi
        cache = Step1Cache()
        rh = -(b * present.phi_hat + c * old.phi_hat) / dt
        cache["phi_11"] = rh / lhs_phi
        cache["mu_11"] = L_phi * cache.phi_11
        rh = -(b * present.psi_hat + c * old.psi_hat) / dt
        cache["psi_11"] = psi_div(rh)
        cache["nu_11"] = L_psi * cache.psi_11
        H1h = ops.rfft(get_H1(phi_star, ops, cfg, A0))
        cache["phi_12"] = (-cfg.M_phi * H1h) / lhs_phi
        cache["mu_12"] = L_phi * cache.phi_12 + H1h
        Gh = ops.rfft(get_MG(phi_star, psi_star, cfg))
        gG = [ops.irfft(ops.D1[d] * Gh) for d in range(3)]
        tc = [ops.rfft(M_psi * gG[d]) for d in range(3)]
        rh = ops.D1[0] * tc[0] + ops.D1[1] * tc[1] + ops.D1[2] * tc[2]
        cache["psi_12"] = psi_div(rh)
        cache["nu_12"] = L_psi * cache.psi_12 + Gh
        H2h = ops.rfft(get_H2(phi_star, ops, cfg))
        H3h = ops.rfft(get_H3(phi_star, psi_star, cfg))
        cache["phi_13"] = (-cfg.M_phi * H2h) / lhs_phi
        cache["phi_14"] = (-cfg.M_phi * H3h) / lhs_phi
        cache["mu_13"] = L_phi * cache.phi_13 + H2h
        cache["mu_14"] = L_phi * cache.phi_14 + H3h
        u_star = 2.0 * present.u - old.u
        gr = [ops.irfft(ops.D1[d] * phi_star_hat) for d in range(3)]
        t = u_star[0] * gr[0] + u_star[1] * gr[1] + u_star[2] * gr[2]
        th = ops.rfft(t)
        cache["phi_21"] = -th / lhs_phi
        cache["mu_21"] = L_phi * cache.phi_21
        gr = [ops.irfft(ops.D1[d] * psi_star_hat) for d in range(3)]
        t = u_star[0] * gr[0] + u_star[1] * gr[1] + u_star[2] * gr[2]
        th = ops.rfft(t)
        cache["psi_21"] = psi_div(-th)
        cache["nu_21"] = L_psi * cache.psi_21
        return cache

    # -- step 2 (Solvers.jl:144-234, Solvers_3d.jl:99-188) -------------------
    def solve_step2(self, present, old, cache, bdf):
        cfg, ops = self.cfg, self.ops
        a, b, c = bdf.a, bdf.b, bdf.c
        phi_n, phi_nm1 = present.phi, old.phi
        phi_star = 2.0 * phi_n - phi_nm1
        psi_n, psi_nm1 = present.psi, old.psi
        psi_star = 2.0 * psi_n - psi_nm1
        H1 = get_H1(phi_star, ops, cfg, present.A0)
        H2 = get_H2(phi_star, ops, cfg)
        H3 = get_H3(phi_star, psi_star, cfg)
        G = get_MG(phi_star, psi_star, cfg)

        def int_dot(A, B):
            return float(np.sum(A * B)) * cfg.cell

        tph = b * phi_n + c * phi_nm1
        tps = b * psi_n + c * psi_nm1
        U1 = -(b * present.R1 + c * old.R1) / a + int_dot(H1, tph) / (2.0 * a)
        U2 = -(b * present.R2 + c * old.R2) / a + int_dot(H2, tph) / (2.0 * a)
        U3 = -(b * present.R3 + c * old.R3) / a + (int_dot(H3, tph) + int_dot(G, tps)) / (2.0 * a)
        phi_12 = ops.irfft(cache.phi_12)
        phi_13 = ops.irfft(cache.phi_13)
        phi_14 = ops.irfft(cache.phi_14)
        psi_12 = ops.irfft(cache.psi_12)
        phi_11 = ops.irfft(cache.phi_11)
        psi_11 = ops.irfft(cache.psi_11)
        phi_21 = ops.irfft(cache.phi_21)
        psi_21 = ops.irfft(cache.psi_21)
        L = np.zeros((3, 3))
        R1v = np.zeros(3)
        L[0, 0] = 1.0 - 0.5 * int_dot(H1, phi_12)
        L[0, 1] = -0.5 * int_dot(H1, phi_13)
        L[0, 2] = -0.5 * int_dot(H1, phi_14)
        L[1, 0] = -0.5 * int_dot(H2, phi_12)
        L[1, 1] = 1.0 - 0.5 * int_dot(H2, phi_13)
        L[1, 2] = -0.5 * int_dot(H2, phi_14)
        L[2, 0] = -0.5 * int_dot(H3, phi_12)
        L[2, 1] = -0.5 * int_dot(H3, phi_13)
        L[2, 2] = 1.0 - 0.5 * (int_dot(H3, phi_14) + int_dot(G, psi_12))
        R1v[0] = 0.5 * int_dot(H1, phi_11) + U1
        R1v[1] = 0.5 * int_dot(H2, phi_11) + U2
        R1v[2] = 0.5 * (int_dot(H3, phi_11) + int_dot(G, psi_11)) + U3
        R2v = np.zeros(3)
        R2v[0] = 0.5 * int_dot(H1, phi_21)
        R2v[1] = 0.5 * int_dot(H2, phi_21)
        R2v[2] = 0.5 * (int_dot(H3, phi_21) + int_dot(G, psi_21))
        s1 = np.linalg.solve(L, R1v)
        s2 = np.linalg.solve(L.copy(), R2v)
        return dict(R_11_np1=s1[0], R_21_np1=s1[1], R_31_np1=s1[2],
                    R_12_np1=s2[0], R_22_np1=s2[1], R_32_np1=s2[2])

    # -- step 3 (Solvers.jl:242-259) ---------------------------------------
    @staticmethod
    def solve_step3(cache, s2):
        R11, R21, R31 = s2["R_11_np1"], s2["R_21_np1"], s2["R_31_np1"]
        R12, R22, R32 = s2["R_12_np1"], s2["R_22_np1"], s2["R_32_np1"]
        C = cache
        return dict(
            phi_1_hat=C.phi_11 + R11 * C.phi_12 + R21 * C.phi_13 + R31 * C.phi_14,
            mu_1_hat=C.mu_11 + R11 * C.mu_12 + R21 * C.mu_13 + R31 * C.mu_14,
            psi_1_hat=C.psi_11 + R31 * C.psi_12,
            nu_1_hat=C.nu_11 + R31 * C.nu_12,
            phi_2_hat=C.phi_21 + R12 * C.phi_12 + R22 * C.phi_13 + R32 * C.phi_14,
            mu_2_hat=C.mu_21 + R12 * C.mu_12 + R22 * C.mu_13 + R32 * C.mu_14,
            psi_2_hat=C.psi_21 + R32 * C.psi_12,
            nu_2_hat=C.nu_21 + R32 * C.nu_12)

    # -- step 4 (Solvers.jl:267-337, Solvers_3d.jl:221-292) ------------------
    def solve_step4(self, present, old, bdf):
        cfg, ops = self.cfg, self.ops
        nd = cfg.ndim
        dt, eta, lamda = present.dt, cfg.eta, cfg.lamda
        a, b, c = bdf.a, bdf.b, bdf.c
        phi_star = 2.0 * present.phi - old.phi
        psi_star = 2.0 * present.psi - old.psi
        u_star = 2.0 * present.u - old.u
        u_star_hat = 2.0 * present.u_hat - old.u_hat
        mu_star_hat = 2.0 * present.mu_hat - old.mu_hat
        nu_star_hat = 2.0 * present.nu_hat - old.nu_hat
        lhs = (a / dt) - eta * ops.Laplacian
        uh1 = np.empty_like(present.u_hat)
        for d in range(nd):
            uh1[d] = -(b * present.u_hat[d] + c * old.u_hat[d]) / dt - ops.D1[d] * present.p_hat
        conv = np.zeros_like(present.u)
        if nd == 2:
            dux_dx = ops.irfft(ops.D1[0] * u_star_hat[0])
            dux_dy = ops.irfft(ops.D1[1] * u_star_hat[0])
            duy_dx = ops.irfft(ops.D1[0] * u_star_hat[1])
            duy_dy = ops.irfft(ops.D1[1] * u_star_hat[1])
            conv[0] = u_star[0] * dux_dx + u_star[1] * dux_dy
            conv[1] = u_star[0] * duy_dx + u_star[1] * duy_dy
            dmu = [ops.irfft(ops.D1[d] * mu_star_hat) for d in range(2)]
            dnu = [ops.irfft(ops.D1[d] * nu_star_hat) for d in range(2)]
            coupl = [phi_star * dmu[d] + psi_star * dnu[d] for d in range(2)]
            uh2 = np.empty_like(present.u_hat)
            for d in range(2):
                uh2[d] = ops.rfft(-conv[d] - lamda * np.sum(coupl[d], axis=0))
        else:
            for d in range(3):
                for comp in range(3):
                    der = ops.irfft(ops.D1[d] * u_star_hat[comp])
                    conv[comp] += u_star[d] * der
            if cfg.N != 1:
                raise ValueError("the 3D coupling term (Solvers_3d.jl:260-267) is defined for N == 1 only")
            coupl = []
            for d in range(3):
                dmu = ops.irfft(ops.D1[d] * mu_star_hat)
                dnu = ops.irfft(ops.D1[d] * nu_star_hat)
                coupl.append((phi_star * dmu + psi_star * dnu)[0])
            uh2 = np.empty_like(present.u_hat)
            for d in range(3):
                uh2[d] = ops.rfft(-conv[d] - lamda * coupl[d])
        uh1 = uh1 / lhs
        uh2 = uh2 / lhs
        return dict(u_tilde_1_hat=uh1, u_tilde_2_hat=uh2,
                    u_tilde_1=ops.irfft(uh1), u_tilde_2=ops.irfft(uh2))

    # -- step 5 (Solvers.jl:344-423, Solvers_3d.jl:299-392) ------------------
    def solve_step5(self, present, old, s3, s4, bdf):
        cfg, ops = self.cfg, self.ops
        nd = cfg.ndim
        a, b, c = bdf.a, bdf.b, bdf.c
        lamda = cfg.lamda
        # 3D uses conf.dt here (Solvers_3d.jl:386-387); 2D uses present.dt
        dt = present.dt if nd == 2 else cfg.dt
        phi_star_hat = 2.0 * present.phi_hat - old.phi_hat
        psi_star_hat = 2.0 * present.psi_hat - old.psi_hat
        mu_star_hat = 2.0 * present.mu_hat - old.mu_hat
        nu_star_hat = 2.0 * present.nu_hat - old.nu_hat
        u_star_hat = 2.0 * present.u_hat - old.u_hat
        u_star = 2.0 * present.u - old.u
        gphi = [ops.irfft(ops.D1[d] * phi_star_hat) for d in range(nd)]
        gpsi = [ops.irfft(ops.D1[d] * psi_star_hat) for d in range(nd)]
        gmu = [ops.irfft(ops.D1[d] * mu_star_hat) for d in range(nd)]
        gnu = [ops.irfft(ops.D1[d] * nu_star_hat) for d in range(nd)]
        conv = []
        du = [[ops.irfft(ops.D1[d] * u_star_hat[comp]) for d in range(nd)] for comp in range(nd)]
        for comp in range(nd):
            conv.append(sum(u_star[d] * du[comp][d] for d in range(nd)))
        mu_1 = ops.irfft(s3["mu_1_hat"])
        nu_1 = ops.irfft(s3["nu_1_hat"])
        mu_2 = ops.irfft(s3["mu_2_hat"])
        nu_2 = ops.irfft(s3["nu_2_hat"])
        ut1, ut2 = s4["u_tilde_1"], s4["u_tilde_2"]
        adv_phi = sum(u_star[d] * gphi[d] for d in range(nd))
        adv_psi = sum(u_star[d] * gpsi[d] for d in range(nd))
        phi_star = 2.0 * present.phi - old.phi
        psi_star = 2.0 * present.psi - old.psi
        t3 = [np.sum(phi_star * gmu[d] + psi_star * gnu[d], axis=0) for d in range(nd)]

        def dot(A, B):
            return float(np.sum(A * B))
        t11 = dot(adv_phi, mu_1)
        t12 = dot(adv_psi, nu_1)
        t13 = sum(dot(t3[d], ut1[d]) for d in range(nd))
        t14 = sum(dot(conv[d], ut1[d]) for d in range(nd))
        theta_1 = cfg.cell * (lamda * (t11 + t12 + t13) + t14)
        t21 = dot(adv_phi, mu_2)
        t22 = dot(adv_psi, nu_2)
        t23 = sum(dot(t3[d], ut2[d]) for d in range(nd))
        t24 = sum(dot(conv[d], ut2[d]) for d in range(nd))
        theta_2 = cfg.cell * (lamda * (t21 + t22 + t23) + t24)
        rhs_Q = -(b * present.Q + c * old.Q) / dt + theta_1
        lhs_Q = (a / dt) - theta_2
        self.last_theta = (theta_1, theta_2)
        return rhs_Q / lhs_Q

    # -- step 6 (Solvers.jl:431-453) ---------------------------------------
    @staticmethod
    def solve_step6(s2, s3, s4, Q):
        return dict(
            phi_hat=s3["phi_1_hat"] + Q * s3["phi_2_hat"],
            psi_hat=s3["psi_1_hat"] + Q * s3["psi_2_hat"],
            mu_hat=s3["mu_1_hat"] + Q * s3["mu_2_hat"],
            nu_hat=s3["nu_1_hat"] + Q * s3["nu_2_hat"],
            R1=s2["R_11_np1"] + Q * s2["R_12_np1"],
            R2=s2["R_21_np1"] + Q * s2["R_22_np1"],
            R3=s2["R_31_np1"] + Q * s2["R_32_np1"],
            u_tilde_hat=s4["u_tilde_1_hat"] + Q * s4["u_tilde_2_hat"])

    # -- step 7 (Solvers.jl:459-498, Solvers_3d.jl:428-467) ------------------
    def solve_step7(self, present, s6, bdf):
        cfg, ops = self.cfg, self.ops
        nd = cfg.ndim
        a, dt, eta = bdf.a, present.dt, cfg.eta
        ut = s6["u_tilde_hat"]
        div = sum(ops.D1[d] * ut[d] for d in range(nd))
        factor = a / dt
        with np.errstate(divide="ignore", invalid="ignore"):
            dp = factor * div / ops.Laplacian
        dp[(0,) * nd] = 0.0
        u_np1 = np.empty_like(ut)
        for d in range(nd):
            u_np1[d] = ut[d] - (dt / a) * ops.D1[d] * dp
        p_np1 = present.p_hat + dp - eta * div
        return dict(u_hat=u_np1, p_hat=p_np1)

    # -- one full time step: simulation.jl:73-110 ---------------------------
    def step(self, present: FieldState, old: FieldState, n: int, dt: float):
        cfg, ops = self.cfg, self.ops
        present.dt = dt
        bdf = bdf_coeff(n)
        c1 = self.solve_step1(present, old, bdf)
        s2 = self.solve_step2(present, old, c1, bdf)
        s3 = self.solve_step3(c1, s2)
        s4 = self.solve_step4(present, old, bdf)
        Q = self.solve_step5(present, old, s3, s4, bdf)
        s6 = self.solve_step6(s2, s3, s4, Q)
        s7 = self.solve_step7(present, s6, bdf)
        update_state(old, present)
        present.phi_hat = s6["phi_hat"]
        present.psi_hat = s6["psi_hat"]
        present.mu_hat = s6["mu_hat"]
        present.nu_hat = s6["nu_hat"]
        present.u_hat = s7["u_hat"]
        present.p_hat = s7["p_hat"]
        present.phi = ops.irfft(present.phi_hat)
        present.psi = ops.irfft(present.psi_hat)
        present.mu = ops.irfft(present.mu_hat)
        present.nu = ops.irfft(present.nu_hat)
        present.p = ops.irfft(present.p_hat)
        present.u = ops.irfft(present.u_hat)
        present.R1, present.R2, present.R3 = s6["R1"], s6["R2"], s6["R3"]
        present.Q = Q
        return dict(step1=c1, step2=s2, step3=s3, step4=s4, Q=Q, step6=s6, step7=s7)

    def monitor(self, present, old):
        """simulation.jl:146-148."""
        cfg, ops = self.cfg, self.ops
        E = compute_modified_energy(present, old, ops, cfg)
        A = calculate_area(present.phi, ops, cfg)
        return E, float(np.sum(np.abs(A - present.A0)) / np.sum(present.A0))


# ---------------------------------------------------------------------------
# generate_initial_condition's shapes (Init.jl:74-197, Init_3d.jl:67-137)
# ---------------------------------------------------------------------------
class InitError(ValueError):
    """The cases generate_initial_condition rejects (its error() calls, and the
    UndefVarErrors of centres / 2D names it never defines)."""


def reference_shapes(cfg: Config, state_type: int, blob_u=None):
    """phi, psi [N][(Nz)][Ny][Nx] of generate_initial_condition(conf, ops,
    state_type) (2D: Init.jl:74-197; 3D: Init_3d.jl:67-137).  blob_u: the 20
    rand() values state_type 4 draws (Init.jl:155-159, in draw order: an, pn for
    k = 1..10), which the reference takes from Julia's global RNG."""
    N, eps, goal = cfg.N, cfg.epsilon, cfg.goal
    Lx, Ly, dx, dy = cfg.Lx, cfg.Ly, cfg.dx, cfg.dy
    den = SQ2 * eps
    X = (np.arange(cfg.Nx) * dx)                      # range(0, Lx - dx, length=Nx), Init.jl:81-82
    Y = (np.arange(cfg.Ny) * dy)
    if cfg.ndim == 3:
        Z = np.arange(cfg.Nz) * cfg.dz
        X3, Y3, Z3 = X[None, None, :], Y[None, :, None], Z[:, None, None]
        phi = np.zeros((N,) + cfg.shape)
        if N == 1:                                    # Init_3d.jl:86-90
            cx, cy, cz = [Lx / 2], [Ly / 2], [cfg.Lz / 2]
        elif N == 2:
            cx, cy, cz = [0.73, 1.27], [Ly / 2] * 2, [cfg.Lz / 2] * 2
        elif N == 3:
            cx, cy, cz = [Lx / 4, Lx / 2, 3 * Lx / 4], [Ly / 2] * 3, [cfg.Lz / 2] * 3
        else:
            raise InitError(f"N = {N}: no vesicle centres (Init_3d.jl:86-99 define N <= 3)")
        if N == 1:                                    # Init_3d.jl:101-108
            if state_type > 6:
                raise InitError(f"state_type {state_type} is invalid for N = 1")
            if state_type == 1:
                R = 0.2 * Lx
                dist = np.sqrt((X3 - cx[0]) ** 2 / 2 + (Y3 - cy[0]) ** 2 / 2 + (Z3 - cz[0]) ** 2)
                phi[0] = np.tanh((R - dist) / den)
        elif N == 2:                                  # Init_3d.jl:109-126
            if state_type <= 6:
                raise InitError(f"state_type {state_type} is invalid for N = 2")
            if state_type == 7:
                if goal == "s":
                    raise InitError("state_type 7 needs goal g")
                raise InitError("state_type 7 is not defined in 3D (Init_3d.jl:118-125 use the 2D names X, Y)")
    else:
        X2, Y2 = X[None, :], Y[:, None]
        phi = np.zeros((N,) + cfg.shape)
        if N == 1:                                    # Init.jl:86-100
            cx, cy = [Lx / 2], [Ly / 2]
        elif N == 2:
            if goal == "g":
                cx = [0.75, 1.25]
            elif goal == "s":
                cx = [0.65, 1.35]
            else:
                raise InitError(f"what's the goal? now it is {goal}")
            cy = [Ly / 2, Ly / 2]
        elif N == 3:
            cx, cy = [Lx / 4, Lx / 2, 3 * Lx / 4], [Ly / 2] * 3
        else:
            raise InitError(f"N = {N}: no vesicle centres (Init.jl:86-100 define N <= 3)")

        def star(n, R0, amp, k=10):
            ddx, ddy = X2 - cx[n], Y2 - cy[n]
            r = np.sqrt(ddx ** 2 + ddy ** 2)
            theta = np.arctan2(ddx, ddy)              # Julia atan(X - cx, Y - cy)
            return np.tanh((R0 + amp * np.cos(k * theta) - r) / den)

        if N == 1:                                    # Init.jl:102-160
            if state_type > 6:
                raise InitError(f"state_type {state_type} is invalid for N = 1")
            ddx, ddy = X2 - cx[0], Y2 - cy[0]
            if state_type == 1:                       # ellipse
                R = 0.2 * Lx
                dist = np.sqrt(ddx ** 2 / 2 + ddy ** 2)
                phi[0] = np.tanh((R - dist) / den)
            elif state_type == 2:                     # smoothed triangle
                radius, sm = 0.65 * Lx, 40.0
                ks, kc = math.sqrt(3) / 2, 0.5
                d1 = -ddy + 0 * ddx
                d2 = ks * ddx + kc * ddy
                d3 = -ks * ddx + kc * ddy
                mx = np.maximum(d1, np.maximum(d2, d3))
                ds = mx + (1 / sm) * np.log(np.exp(sm * (d1 - mx)) + np.exp(sm * (d2 - mx)) + np.exp(sm * (d3 - mx)))
                phi[0] = -np.tanh((ds - radius / 3) / den)
            elif state_type == 3:                     # star
                R0, amp = (0.3, 0.01) if goal == "s" else (0.18, 0.02)
                phi[0] = star(0, R0, amp)
            elif state_type == 4:                     # random blob
                R0, amp = (0.3, 0.15) if goal == "s" else (0.2, 0.25)
                if blob_u is None or len(blob_u) < 20:
                    raise InitError("state_type 4 needs its 20 uniform draws")
                r = np.sqrt(ddx ** 2 + ddy ** 2)
                theta = np.arctan2(ddx, ddy)
                R = np.full(theta.shape, R0)
                for k in range(1, 11):
                    an = (blob_u[2 * k - 2] * 2 - 1) * amp / k
                    pn = blob_u[2 * k - 1] * 2 * math.pi
                    R = R + an * R0 * np.cos(k * theta + pn)
                phi[0] = np.tanh((R - r) / den)
        else:                                         # Init.jl:161-189
            if state_type <= 6:
                raise InitError(f"state_type {state_type} is invalid for N = {N}")
            for n in range(N):
                if state_type == 7:
                    if goal == "s":
                        raise InitError("state_type 7 needs goal g")
                    phi[n] = star(n, 0.2, 0.02)
                elif state_type == 8:
                    if goal == "g":
                        raise InitError("state_type 8 needs goal s")
                    phi[n] = star(n, 0.3, 0.01)
    psi = -0.1 * phi + 0.7 if goal == "s" else -0.35 * phi + 0.45   # Init.jl:191-197
    return phi, psi


# ---------------------------------------------------------------------------
# initialisation: simulation.jl:22-53 (with a given initial phi/psi)
# ---------------------------------------------------------------------------
def make_state(cfg: Config, phi: np.ndarray, psi: np.ndarray, ops: Operators) -> FieldState:
    """generate_initial_condition (Init.jl:199-216) for caller-supplied phi, psi."""
    nd = cfg.ndim
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    psi = np.ascontiguousarray(psi, dtype=np.float64)
    u = np.zeros((nd,) + cfg.shape)
    p = np.zeros(cfg.shape)
    mu = np.zeros_like(phi)
    nu = np.zeros_like(phi)
    return FieldState(phi=phi, phi_hat=ops.rfft(phi), psi=psi, psi_hat=ops.rfft(psi),
                      u=u, u_hat=ops.rfft(u), p=p, p_hat=ops.rfft(p), mu=mu,
                      mu_hat=ops.rfft(mu), nu=nu, nu_hat=ops.rfft(nu),
                      Q=1.0, R1=1.0, R2=1.0, R3=1.0, A0=np.zeros(1), dt=0.0)


def init_state(cfg: Config, present: FieldState, ops: Operators) -> FieldState:
    """simulation.jl:25-50: A0, R1..R3, Q, initial mu/nu."""
    A0 = calculate_area(present.phi, ops, cfg)
    present.A0 = A0
    present.R1 = math.sqrt(get_W1(present.phi, ops, cfg, A0) + cfg.C1)
    present.R2 = math.sqrt(get_W2(present.phi, ops, cfg) + cfg.C2)
    present.R3 = math.sqrt(get_W3(present.phi, present.psi, cfg) + cfg.C3)
    present.Q = 1.0
    L_phi = cfg.S1 * ops.Biharmonic - cfg.S2 * ops.Laplacian + cfg.S3
    H1 = get_H1(present.phi, ops, cfg, A0)
    H2 = get_H2(present.phi, ops, cfg)
    H3 = get_H3(present.phi, present.psi, cfg)
    G = get_MG(present.phi, present.psi, cfg)
    present.mu_hat = (L_phi * present.phi_hat + present.R1 * ops.rfft(H1)
                      + present.R2 * ops.rfft(H2) + present.R3 * ops.rfft(H3))
    present.nu_hat = cfg.S4 * present.psi_hat + present.R3 * ops.rfft(G)
    present.mu = ops.irfft(present.mu_hat)
    present.nu = ops.irfft(present.nu_hat)
    return present


def run(cfg: Config, phi0, psi0, nsteps: int, dt_schedule=None, monitor=True,
        oracle: Optional[Oracle] = None, callback=None):
    """run_simulation (simulation.jl:2-155) with a caller-supplied initial
    condition and a uniform dt schedule by default (no snapshot I/O)."""
    orc = oracle or Oracle(cfg)
    present = make_state(cfg, phi0, psi0, orc.ops)
    init_state(cfg, present, orc.ops)
    old = present.copy()
    energy, area = [], []
    for n in range(1, nsteps + 1):
        dt = cfg.dt if dt_schedule is None else dt_schedule[n - 1]
        orc.step(present, old, n, dt)
        if monitor:
            E, ar = orc.monitor(present, old)
            energy.append(E)
            area.append(ar)
        if callback is not None:
            callback(n, present, old)
    return present, old, energy, area, orc
