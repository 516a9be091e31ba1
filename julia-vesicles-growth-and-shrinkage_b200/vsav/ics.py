"""Seeded synthetic initial conditions and parameter sets for the benchmark
workloads of the SAV vesicle step.

The reference builds its initial conditions in ``generate_initial_condition``
(src/Init.jl:74-216, src/Init_3d.jl:67-152) with hard-coded shapes on a
[0, L)^d grid.  The workloads here use the same tanh phase-field profile
``phi = tanh((R(theta) - r) / (sqrt(2) eps))`` (Init.jl:113) on the periodic
box [-pi, pi)^d, with seeded shapes:

* ``single2d``  : 128^2, one ellipse 1.2/0.8 + Fourier modes 2..6 (amp 0.02)
* ``multi2d``   : N non-overlapping ellipses, radii U[0.4,0.7], axis ratio
                  U[0.6,1], centres with min gap 4 eps, inside psi U[lo,hi]
* ``single3d``  : ellipsoid 1.2/0.9/0.7 + real spherical harmonics l<=6 (amp 0.02)

psi is 'inside' / 'outside' blended by the same profile: psi = pin (1+phi)/2 + pout (1-phi)/2.
Coefficients follow set_para_base (Init.jl:8-69) with S1, S3 recomputed at the
workload's eps (Init.jl:40-43).
"""
from __future__ import annotations

import math

import numpy as np

SQ2 = math.sqrt(2.0)

# The time steps of the workloads.  The configurations name dt = 1e-4 (128^2, and
# 128^3) and 5e-5 (512^2 x 4); at those steps the reference scheme itself stops with
# its fatal W3 + C3 < 0 within 4-21 steps (the oracle, tests/test_oracle_dt.py), so
# every workload runs at the largest probed step (1e-4, 5e-5, 2e-5, 1e-5, 5e-6,
# 2e-6) that stays stable over its step count: 1e-5, except 512^2 x 4, whose
# 500 steps need 5e-6 (at 1e-5 it stops at step 121; tests/test_gpu_configs.py).
DT_2D = 1e-5
DT_3D = 1e-5
DT_512x4 = 5e-6


def params(eps: float, N: int, psi_in, psi_out, dt: float, T: float, Nx: int, Ny: int,
           L: float = 2 * math.pi, Nz: int = 0, tol: float = 1e-12, goal: str = "s") -> dict:
    """Keyword arguments of the reference Config (Types.jl:101-111) with the
    set_para_base coefficients (Init.jl:40-68) at the given eps."""
    gb = 0.1
    gin = gout = 1e5
    S3 = gb / eps ** 3
    # The SAV constant C2 must keep W2 + C2 > 0 (Utils.jl:180).  W2 contains
    # -E2 ~ -S3/2 * int(phi^2) ~ -S3/2 * N |Omega|; the reference's C2 = 5e5
    # (Init.jl:63) is sized for its unit box with one vesicle.  Keep it where it
    # suffices and scale it (5x margin) otherwise.
    area = L ** (3 if Nz else 2)
    C2 = max(5.0e5, 5.0 * 0.5 * S3 * N * area)
    return dict(
        N=N, epsilon=eps, M_phi=1.0, M0_psi=0.5, eta=1.0, gamma_surf=1.0, gamma_area=5e4,
        gamma_bend=gb, gamma_in=gin, beta_in=0.0, psi_in_v=list(map(float, psi_in)),
        gamma_out=gout, beta_out=0.0, psi_out_v=list(map(float, psi_out)), lamda=1.0,
        S1=(3 * SQ2 / 8) * eps * gb, S2=0.0, S3=S3, S4=min(gin, gout),
        C1=1.0, C2=C2, C3=1.0e6, dt=dt, T=T, Nx=Nx, Ny=Ny, Lx=L, Ly=L, tol=tol, goal=goal,
        Nz=Nz, Lz=(L if Nz else 0.0))


def grid(n: int, L: float = 2 * math.pi):
    return -L / 2 + L * np.arange(n) / n


def _blend(phi, pin, pout):
    return pin * (1 + phi) / 2 + pout * (1 - phi) / 2


def single2d_shape(seed: int = 0, a: float = 1.2, b: float = 0.8, amp: float = 0.02, psi_inside: float = 0.6,
                   psi_outside: float = 0.2):
    """The single2d shape as parameters (for the device generator, vsav_init_shapes2d)."""
    rng = np.random.default_rng(seed)
    modes = [(m, amp, rng.uniform(0, 2 * np.pi)) for m in range(2, 7)]
    return dict(cx=0.0, cy=0.0, a=a, b=b, rot=0.0, psi_in=psi_inside, psi_out=psi_outside, modes=modes)


def single2d(n: int = 128, eps: float = 0.08, seed: int = 0, a: float = 1.2, b: float = 0.8,
             amp: float = 0.02, psi_inside: float = 0.6, psi_outside: float = 0.2):
    """phi, psi arrays [1][n][n]."""
    rng = np.random.default_rng(seed)
    x = grid(n)
    X, Y = np.meshgrid(x, x, indexing="xy")        # X[j, i] = x_i, rows are y
    th = np.arctan2(Y, X)
    r = np.hypot(X, Y)
    R = a * b / np.sqrt((b * np.cos(th)) ** 2 + (a * np.sin(th)) ** 2)
    for m in range(2, 7):
        R = R + amp * np.cos(m * th + rng.uniform(0, 2 * np.pi))
    phi = np.tanh((R - r) / (SQ2 * eps))[None]
    psi = _blend(phi, psi_inside, psi_outside)
    return phi, psi


def multi2d_shapes(N: int, eps: float, seed: int, psi_lo: float = 0.4, psi_hi: float = 0.8,
                   psi_outside: float = 0.2, L: float = 2 * math.pi, max_tries: int = 20000):
    """The multi2d shapes as parameters (same seeded draws as multi2d)."""
    rng = np.random.default_rng(seed)
    shapes = _place(rng, N, eps, L, max_tries)
    pin = rng.uniform(psi_lo, psi_hi, size=N)
    return [dict(cx=cx, cy=cy, a=rad, b=rad * ratio, rot=rot, psi_in=float(pin[k]), psi_out=psi_outside, modes=[])
            for k, (cx, cy, rad, ratio, rot) in enumerate(shapes)]


def _place(rng, N, eps, L, max_tries):
    """Rejection-sampled non-overlapping ellipse parameters (cx, cy, rad, ratio, rot)."""
    shapes = []
    tries = 0
    while len(shapes) < N:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("could not place vesicles")
        rad = rng.uniform(0.4, 0.7)
        ratio = rng.uniform(0.6, 1.0)
        rot = rng.uniform(0, np.pi)
        lim = L / 2 - rad - 4 * eps
        cx, cy = rng.uniform(-lim, lim, size=2)
        ok = all(math.hypot(cx - s[0], cy - s[1]) >= rad + s[2] + 4 * eps for s in shapes)
        if ok:
            shapes.append((cx, cy, rad, ratio, rot))
    return shapes


def multi2d(n: int, N: int, eps: float, seed: int, psi_lo: float = 0.4, psi_hi: float = 0.8,
            psi_outside: float = 0.2, L: float = 2 * math.pi, max_tries: int = 20000):
    """N non-overlapping seeded ellipses.  Returns phi, psi [N][n][n] and the
    per-vesicle inside psi values."""
    rng = np.random.default_rng(seed)
    x = grid(n, L)
    X, Y = np.meshgrid(x, x, indexing="xy")
    shapes = _place(rng, N, eps, L, max_tries)
    phi = np.empty((N, n, n))
    psi = np.empty((N, n, n))
    pin = rng.uniform(psi_lo, psi_hi, size=N)
    for k, (cx, cy, rad, ratio, rot) in enumerate(shapes):
        dx = X - cx
        dy = Y - cy
        xr = np.cos(rot) * dx + np.sin(rot) * dy
        yr = -np.sin(rot) * dx + np.cos(rot) * dy
        th = np.arctan2(yr, xr)
        r = np.hypot(xr, yr)
        a, b = rad, rad * ratio
        R = a * b / np.sqrt((b * np.cos(th)) ** 2 + (a * np.sin(th)) ** 2)
        phi[k] = np.tanh((R - r) / (SQ2 * eps))
        psi[k] = _blend(phi[k], pin[k], psi_outside)
    return phi, psi, pin


def _real_sph_harm(l, m, theta, ph):
    """Real spherical harmonic (unnormalised associated Legendre form)."""
    from scipy.special import lpmv
    P = lpmv(abs(m), l, np.cos(theta))
    if m > 0:
        return P * np.cos(m * ph)
    if m < 0:
        return P * np.sin(-m * ph)
    return P


def single3d(n: int = 128, eps: float = 0.1, seed: int = 0, axes=(1.2, 0.9, 0.7),
             amp: float = 0.02, lmax: int = 6, psi_inside: float = 0.6, psi_outside: float = 0.2):
    """phi, psi [1][n][n][n] (z, y, x)."""
    rng = np.random.default_rng(seed)
    x = grid(n)
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    r = np.sqrt(X ** 2 + Y ** 2 + Z ** 2)
    theta = np.arccos(np.clip(Z / np.maximum(r, 1e-300), -1, 1))
    ph = np.arctan2(Y, X)
    a, b, c = axes
    st, ct = np.sin(theta), np.cos(theta)
    R = 1.0 / np.sqrt((st * np.cos(ph) / a) ** 2 + (st * np.sin(ph) / b) ** 2 + (ct / c) ** 2)
    pert = np.zeros_like(r)
    for l in range(1, lmax + 1):
        for m in range(-l, l + 1):
            Ylm = _real_sph_harm(l, m, theta, ph)
            s = np.max(np.abs(Ylm))
            if s > 0:
                pert += rng.uniform(-1, 1) * Ylm / s
    pert *= amp / max(np.max(np.abs(pert)), 1e-300)
    phi = np.tanh((R + pert - r) / (SQ2 * eps))[None]
    psi = _blend(phi, psi_inside, psi_outside)
    return phi, psi


def ensemble(n_runs: int = 64, n: int = 256, eps: float = 0.08, seed: int = 0, nmin: int = 1, nmax: int = 4,
             dt: float = 1e-5):
    """Batched ensemble: n_runs independent 2D runs at n^2, each with N ~ U{nmin..nmax}
    seeded vesicles (multi2d shapes), inside psi U[0.3, 0.9].  Returns (config kwargs
    with per-field psi_in_v/psi_out_v, run_sizes, phi [V][n][n], psi [V][n][n]);
    C2 is sized for the largest run (the constant is shared by the handle)."""
    rng = np.random.default_rng(seed)
    sizes = [int(k) for k in rng.integers(nmin, nmax + 1, size=n_runs)]
    phis, psis, tin = [], [], []
    for r, N in enumerate(sizes):
        phi, psi, _ = multi2d(n, N, eps, seed * 1000 + r, 0.3, 0.9)
        phis.append(phi)
        psis.append(psi)
        tin += [0.65 if k % 2 == 0 else 0.1 for k in range(N)]
    kw = params(eps, max(sizes), tin, [0.8] * len(tin), dt, 100 * dt, n, n)
    return kw, sizes, np.concatenate(phis), np.concatenate(psis)


def ensemble_shapes(n_runs: int = 64, eps: float = 0.08, seed: int = 0, nmin: int = 1, nmax: int = 4):
    """The shapes of ensemble() as parameters, run after run (device generator)."""
    rng = np.random.default_rng(seed)
    sizes = [int(k) for k in rng.integers(nmin, nmax + 1, size=n_runs)]
    out = []
    for r, N in enumerate(sizes):
        out += multi2d_shapes(N, eps, seed * 1000 + r, 0.3, 0.9)
    return sizes, out


# ---------------------------------------------------------------------------
# the five benchmark workloads
# ---------------------------------------------------------------------------
def workload(name: str, seed: int = 0, n_override: int | None = None,
             N_override: int | None = None, eps_override: float | None = None):
    """Returns (config kwargs, phi0, psi0, nsteps).  The overrides shrink a
    workload for tests (same construction, smaller grid / fewer vesicles)."""
    if name == "single2d_128":            # plain method, CPU-runnable
        n = n_override or 128
        eps = eps_override or 0.08
        phi, psi = single2d(n, eps, seed)
        kw = params(eps, 1, [0.1], [0.8], DT_2D, 200 * DT_2D, n, n)
        return kw, phi, psi, 200
    if name in ("multi2d_512x4", "multi2d_1024x8", "ensemble_256"):
        n, N, eps, dt, steps = {
            "multi2d_512x4": (512, 4, 0.04, DT_512x4, 500),
            "multi2d_1024x8": (1024, 8, 0.02, DT_2D, 100),
            "ensemble_256": (256, 2, 0.08, DT_2D, 100),
        }[name]
        n = n_override or n
        N = N_override or N
        eps = eps_override or eps
        lo, hi = (0.3, 0.9) if name == "ensemble_256" else (0.4, 0.8)
        phi, psi, pin = multi2d(n, N, eps, seed, lo, hi)
        # osmotic targets: alternate growth (0.65) and shrinkage (0.1) goals (Init.jl:17-38)
        targets = [0.65 if k % 2 == 0 else 0.1 for k in range(N)]
        kw = params(eps, N, targets, [0.8] * N, dt, steps * dt, n, n)
        return kw, phi, psi, steps
    if name == "single3d_128":
        n = n_override or 128
        eps = eps_override or 0.1
        phi, psi = single3d(n, eps, seed)
        kw = params(eps, 1, [0.65], [0.8], DT_3D, 100 * DT_3D, n, n, Nz=n, goal="g")
        return kw, phi, psi, 100
    raise KeyError(name)
