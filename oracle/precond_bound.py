"""How many BiCGSTAB iterations a better psi preconditioner could save.

    python oracle/precond_bound.py [workload] [dt]    # default multi2d_512x4 1e-5
                                                     # writes profiles/precond_bound_<workload>.json

Study infrastructure (not product code; NumPy FP64 on the oracle's operators).
It takes the psi operator of Step 1 (src/Solvers.jl:39-53)

    A x = a_dt x - sum_d D1_full[d] F( M_psi F^-1( D1_full[d] S4 x ) ),

with M_psi = get_M_psi(phi*) (src/Utils.jl:20), and solves two right-hand
sides of the shapes Step 1 builds -- the psi_11 history term
-(b psi^n + c psi^n-1)/dt (Solvers.jl:90-91) and the psi_12 term
D1 . F(M_psi F^-1(D1 G)) (Solvers.jl:99-106) -- by flexible right-preconditioned
BiCGSTAB to a true relative residual of 1e-8 with:

  diag         the reference's diagonal 1 / (a_dt - M_max S4 Laplacian) (Solvers.jl:57)
  scale_sqrtM  diag, then the physical scaling sqrt(M_max / M_psi)
  sym_sqrtM    diag^1/2, the scaling M_max / M_psi, diag^1/2
  local_symbol the local symbol 1 / (a_dt + S4 M_psi(x) |k|^2) interpolated
               between the two constant-mobility diagonals at M_min and M_max
  neumann1     2 D - D A D (one extra operator application per use)
  lsq_stencil  diag + a linear, M_psi-conditioned 3x3 stencil on Re F^-1(D r):
               z = sum over taps and powers of Mt = (M_psi - 0.075)/0.025 of
               theta * Mt^q * y(x + tap); theta fitted by least squares on the
               solver's own residuals (the form a learned network that is linear
               in the residual would take)

M_psi dips from 0.1 to 0.05 only across the interfaces (width ~epsilon), and
S4 |k|^2 M_psi dominates a_dt for all but the lowest modes, so the diagonal
already bounds the preconditioned spectrum to about [0.5, 1]; the remaining
error sits in the interface bands (the grad M_psi terms), which local
corrections do not capture.
"""
import json
import os
import sys
import time

import numpy as np
import scipy.fft as sf

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "julia-vesicles-growth-and-shrinkage_b200"))

from oracle import vsav_oracle as O  # noqa: E402
from vsav import ics  # noqa: E402

W = os.cpu_count() or 1


def setup(workload, dt):
    kw, phi, psi, _ = ics.workload(workload, seed=0)
    kw["dt"] = dt
    cfg = O.Config(**kw)
    ops = O.build_operators(cfg, workers=W)
    M = O.get_M_psi(phi, cfg)
    a_dt = 1.5 / dt                                        # BDF2 a / dt
    S4 = cfg.S4
    D1f = ops.D1_full
    fft = lambda x: sf.fft2(x, workers=W)                  # noqa: E731
    ifft = lambda x: sf.ifft2(x, workers=W)                # noqa: E731

    def A(x):                                              # Solvers.jl:39-53
        b1 = S4 * x
        return a_dt * x - (D1f[0] * fft(M * ifft(D1f[0] * b1)) + D1f[1] * fft(M * ifft(D1f[1] * b1)))

    Mmax, Mmin = float(M.max()), float(M.min())
    Dg = 1.0 / (a_dt - Mmax * ops.Laplacian_full * S4)     # Solvers.jl:57
    Dmin = 1.0 / (a_dt - Mmin * ops.Laplacian_full * S4)
    psi_hat = fft(psi.astype(complex))
    rhs = {"psi_11": (2.0 * psi_hat - 0.5 * psi_hat) / dt}   # -(b psi^n + c psi^n-1)/dt with psi^n-1 = psi^n
    Gh = fft(O.get_MG(phi, psi, cfg).astype(complex))
    rhs["psi_12"] = D1f[0] * fft(M * ifft(D1f[0] * Gh)) + D1f[1] * fft(M * ifft(D1f[1] * Gh))
    return dict(A=A, M=M, Mmax=Mmax, Mmin=Mmin, Dg=Dg, Dmin=Dmin, fft=fft, ifft=ifft, rhs=rhs, cfg=kw)


def flexible_bicgstab(A, b, P, tol=1e-8, itmax=40, collect=None):
    """x0 = 0, shadow c = b; stop on the true residual ||b - A x|| <= tol ||b||."""
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
        if collect is not None:
            collect.append(s.copy())
        sh = P(s)
        t = A(sh)
        om = np.vdot(t, s) / np.vdot(t, t)
        x = x + al * ph + om * sh
        r = s - om * t
        if collect is not None:
            collect.append(r.copy())
        hist.append(float(np.linalg.norm(b - A(x)) / nb))
        if hist[-1] <= tol:
            break
        rho2 = np.vdot(c, r)
        beta = (rho2 / rho) * (al / om)
        rho = rho2
        p = r + beta * (p - om * v)
    return its, hist


def preconditioners(S):
    A, M, Mmax, Mmin, Dg, Dmin, fft, ifft = (S[k] for k in ("A", "M", "Mmax", "Mmin", "Dg", "Dmin", "fft", "ifft"))
    chi = (Mmax - M) / (Mmax - Mmin)
    return {
        "diag": lambda r: Dg * r,
        "scale_sqrtM": lambda r: fft(np.sqrt(Mmax / M) * ifft(Dg * r)),
        "sym_sqrtM": lambda r: np.sqrt(Dg) * fft((Mmax / M) * ifft(np.sqrt(Dg) * r)),
        "local_symbol": lambda r: fft(chi * ifft(Dmin * r) + (1 - chi) * ifft(Dg * r)),
        "neumann1": lambda r: 2 * Dg * r - Dg * A(Dg * r),
    }


def lsq_stencil(S, npowers=4):
    """Fit the linear M-conditioned 3x3 stencil correction on the residuals of
    two diagonal-preconditioned iterations of both right-hand sides."""
    A, M, Dg, fft, ifft = (S[k] for k in ("A", "M", "Dg", "fft", "ifft"))
    Mt = (M - 0.075) / 0.025
    basis = [Mt ** q for q in range(npowers)]
    taps = [(dy, dx) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]

    def feats(r):
        y = ifft(Dg * r).real
        return [B * np.roll(y, (-dy, -dx), axis=(-2, -1)) for (dy, dx) in taps for B in basis]

    rows, rhs = [], []
    for b in S["rhs"].values():
        res = [b]
        flexible_bicgstab(A, b, lambda r: Dg * r, itmax=2, collect=res)
        for r in res:
            r = r / np.linalg.norm(r)
            rows.append(np.stack([A(fft(f)).ravel() for f in feats(r)], 1))
            rhs.append((r - A(Dg * r)).ravel())
    Am = np.concatenate(rows, 0)
    bv = np.concatenate(rhs, 0)
    Ar = np.concatenate([Am.real, Am.imag], 0)
    br = np.concatenate([bv.real, bv.imag], 0)
    theta, *_ = np.linalg.lstsq(Ar, br, rcond=None)
    fit = float(np.linalg.norm(Ar @ theta - br) / np.linalg.norm(br))
    return (lambda r: Dg * r + fft(sum(t * f for t, f in zip(theta, feats(r))))), fit


def main():
    workload = sys.argv[1] if len(sys.argv) > 1 else "multi2d_512x4"
    dt = float(sys.argv[2]) if len(sys.argv) > 2 else 1e-5
    S = setup(workload, dt)
    precs = preconditioners(S)
    P_lsq, fit = lsq_stencil(S)
    precs["lsq_stencil"] = P_lsq
    out = {"workload": workload, "dt": dt, "tolerance": "true relative residual 1e-8",
           "M_psi_range": [S["Mmin"], S["Mmax"]], "lsq_one_step_residual": fit,
           "operator_applications_per_iteration": {k: (4 if k == "neumann1" else 2) for k in precs}, "runs": {}}
    for bn, b in S["rhs"].items():
        for name, P in precs.items():
            t0 = time.time()
            its, hist = flexible_bicgstab(S["A"], b, P)
            out["runs"][f"{bn}/{name}"] = {"iterations": its, "true_residuals": hist}
            print(f"{workload} {bn:7s} {name:13s} iterations {its:2d}  ({time.time() - t0:.1f} s)", flush=True)
    path = os.path.join(ROOT, "profiles", f"precond_bound_{workload}.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path)


if __name__ == "__main__":
    main()
