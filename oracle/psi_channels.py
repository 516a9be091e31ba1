"""How large the anti-Hermitian channel of the full-complex psi solve is.

    python oracle/psi_channels.py [workload] [dt]    # default multi2d_1024x8 1e-5
                                                    # writes profiles/psi_channels_<workload>.json

Study infrastructure (not product code; NumPy FP64 on the oracle's operators).
The reference solves the psi system on full complex spectra (src/Solvers.jl:39-75)
and keeps the first Nx/2+1 columns of the solution (Solvers.jl:79).  With the
reflection-conjugation (J x)(k) = conj(x(-k)) -- J x = x for the spectrum of a
real field -- write D1_full = D_s + D_n, D_n the Nyquist column/row of the
derivative multipliers (fftfreq puts -N/2 there, SpectralUtils.jl:43).  D_s
commutes with J, D_n anti-commutes (conj(i(-N/2)) = -i(-N/2)), and
G = F M_psi F^-1 commutes with J (M_psi is real), so

    A = A_0 + A_1,  A_0 = a_dt - S4 sum_d (D_s G D_s + D_n G D_n)   (J A_0 = A_0 J)
                    A_1 =      - S4 sum_d (D_s G D_n + D_n G D_s)   (J A_1 = -A_1 J).

For a real right-hand side (J b = b) the solution x = x_h + x_a (J x_h = x_h,
J x_a = -x_a) satisfies

    A_0 x_h + A_1 x_a = b,     A_0 x_a + A_1 x_h = 0,

a coupled system over both channels.  A_0 alone is the real-field ("HALF")
operator; x_a is driven by the Nyquist lines through A_1 and is spread over all
wavenumbers by G.  This script solves the FULL system on the two right-hand
sides of Step 1 (the psi_11 history term and the psi_12 mobility term, as
oracle/precond_bound.py builds them) to a true relative residual of 1e-12 and
reports:

  anti_hermitian_rel     ||x_a|| / ||x||
  a1_coupling_rel        ||A_1 x_h|| / ||b||   (what drives x_a)
  kept_half_effect_rel   ||irfft(half(x)) - irfft(half(x_h))|| / ||irfft(half(x))||:
                         how much the kept anti-Hermitian channel changes the
                         physical psi field the reference goes on with
  real_only_rel          the same for the solution of the real-field system
                         A_0 y = b alone (the "real-part solve")
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)

from oracle import precond_bound as PB  # noqa: E402
from oracle import vsav_oracle as O  # noqa: E402


def J(x):
    """(J x)(k) = conj(x(-k)) on full [.., Ny, Nx] spectra."""
    y = np.flip(x, axis=(-2, -1))
    return np.conj(np.roll(y, 1, axis=(-2, -1)))


def main(workload="multi2d_1024x8", dt=1e-5):
    S = PB.setup(workload, dt)
    A, M, fft, ifft, Dg = S["A"], S["M"], S["fft"], S["ifft"], S["Dg"]
    cfg = S["cfg"]
    Nx, Ny = cfg["Nx"], cfg["Ny"]
    a_dt = 1.5 / dt                                        # BDF2 a / dt, as precond_bound.setup
    ops = O.build_operators(O.Config(**cfg))
    kx0 = ops.kx0.reshape(-1)
    ky = ops.ky.reshape(-1)
    s4 = O.Config(**cfg).S4
    Dx = 1j * np.broadcast_to(kx0.reshape(1, -1), (Ny, Nx))
    Dy = 1j * np.broadcast_to(ky.reshape(-1, 1), (Ny, Nx))
    nx_mask = np.zeros((Ny, Nx)); nx_mask[:, Nx // 2] = 1.0
    ny_mask = np.zeros((Ny, Nx)); ny_mask[Ny // 2, :] = 1.0
    Ds = (Dx * (1 - nx_mask), Dy * (1 - ny_mask))
    Dn = (Dx * nx_mask, Dy * ny_mask)

    def G(z):
        return fft(M * ifft(z))

    def A0(x):
        acc = 0
        for d in range(2):
            acc = acc + Ds[d] * G(Ds[d] * x) + Dn[d] * G(Dn[d] * x)
        return a_dt * x - s4 * acc

    def A1(x):
        acc = 0
        for d in range(2):
            acc = acc + Ds[d] * G(Dn[d] * x) + Dn[d] * G(Ds[d] * x)
        return -s4 * acc

    def half_phys(x):
        return np.fft.irfft2(x[..., : Nx // 2 + 1], s=(Ny, Nx))

    P = lambda r: Dg * r  # noqa: E731
    out = {"workload": workload, "dt": dt, "grid": [Ny, Nx], "rhs": {}}
    for name, b in S["rhs"].items():
        its, hist, x = solve(A, b, P)
        xh, xa = 0.5 * (x + J(x)), 0.5 * (x - J(x))
        check = float(np.linalg.norm(A0(x) + A1(x) - A(x)) / np.linalg.norm(A(x)))
        its0, hist0, y = solve(A0, b, P)
        ph = half_phys(x)
        out["rhs"][name] = {
            "iterations_full": its, "true_residual_full": hist[-1],
            "split_check_rel": check,
            "anti_hermitian_rel": float(np.linalg.norm(xa) / np.linalg.norm(x)),
            "a1_coupling_rel": float(np.linalg.norm(A1(xh)) / np.linalg.norm(b)),
            "kept_half_effect_rel": float(np.linalg.norm(ph - half_phys(xh)) / np.linalg.norm(ph)),
            "iterations_real_only": its0,
            "real_only_rel": float(np.linalg.norm(ph - half_phys(y)) / np.linalg.norm(ph)),
        }
        print(name, json.dumps(out["rhs"][name]), flush=True)
    path = os.path.join(ROOT, "profiles", f"psi_channels_{workload}.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path)


def solve(A, b, P, tol=1e-12, itmax=60):
    """flexible BiCGSTAB (x0 = 0, shadow b) to a true relative residual tol; returns x"""
    x = np.zeros_like(b)
    r = b.copy()
    c = b.copy()
    p = r.copy()
    nb = np.linalg.norm(b)
    rho = np.vdot(c, r)
    hist = [1.0]
    its = 0
    while its < itmax:
        its += 1
        ph = P(p)
        v = A(ph)
        al = rho / np.vdot(c, v)
        s = r - al * v
        sh = P(s)
        t = A(sh)
        om = np.vdot(t, s) / np.vdot(t, t)
        x = x + al * ph + om * sh
        r = s - om * t
        hist.append(float(np.linalg.norm(b - A(x)) / nb))
        if hist[-1] <= tol:
            break
        rho2 = np.vdot(c, r)
        beta = (rho2 / rho) * (al / om)
        rho = rho2
        p = r + beta * (p - om * v)
    return its, hist, x


if __name__ == "__main__":
    a = sys.argv[1:]
    main(a[0] if a else "multi2d_1024x8", float(a[1]) if len(a) > 1 else 1e-5)
