"""Algorithmic transform traffic of one SAV time step, counted by the oracle.

    python oracle/count_bytes.py            # writes profiles/algorithmic_bytes.json

Test / measurement infrastructure (not product code): the oracle's OpCounter
counts the reference's transforms per step -- real transforms (rfft, irfft)
and full complex transforms (fft, ifft of the psi BiCGSTAB) per vesicle
field -- on a reduced grid (the counts do not depend on the grid size).  The
step's algorithmic bytes follow from the counts at full size:

  * a real transform of one field reads its input and writes its output
    once: s P + 2 s H bytes (P = points per field, H = (Nx/2+1) Ny [Nz]
    half-spectrum points, s = bytes per real);
  * a full complex transform of one field: 2 * 2 s P in the full-complex
    form the reference solves in; s P + 2 s H in the half-spectrum
    real-equivalent form (one real transform);
  * a BiCGSTAB iteration adds its vector passes (Krylov.jl's updates and dot
    products, KRYLOV_VECTOR_PASSES vectors read or written per iteration and
    field) of 2 s P (full) or 2 s H (half) bytes each;
  * pointwise work outside the solver (SAV functionals, k-space divisions) is
    not counted, so the total is a lower bound of the step's traffic.

The psi part is given per BiCGSTAB iteration, so a measurement multiplies it
by the iteration counts it observed.
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "julia-vesicles-growth-and-shrinkage_b200"))

from oracle import vsav_oracle as O  # noqa: E402
from vsav import ics  # noqa: E402

# vectors read or written per BiCGSTAB iteration and field: s = r - alpha v (3), x += alpha p
# + omega s and r = s - omega t (7), p = r + beta (p - omega v) (4), the dot products <c, v>,
# <t, s>, <t, t>, <c, r>, ||r|| (6), the two preconditioner applications (4)
KRYLOV_VECTOR_PASSES = 24

# workload, reduced grid (n, Nz), full-size grid for the byte totals
CASES = {
    "single2d_128": (64, None),
    "multi2d_512x4": (64, None),
    "multi2d_1024x8": (64, None),
    "single3d_128": (32, 32),
    "ensemble_256": (64, None),
}


def counts(workload, n):
    kw, phi, psi, _ = ics.workload(workload, seed=0, n_override=n)
    kw["dt"] = 1e-5 if kw.get("Nz", 0) == 0 else 1e-4
    cfg = O.Config(**kw)
    orc = O.Oracle(cfg)
    pres = O.make_state(cfg, phi, psi, orc.ops)
    O.init_state(cfg, pres, orc.ops)
    old = pres.copy()
    c = orc.counter
    orc.step(pres, old, 1, cfg.dt)                   # BDF1
    orc.monitor(pres, old)
    c.reset()
    orc.step(pres, old, 2, cfg.dt)                   # a BDF2 step, the steady state
    orc.monitor(pres, old)
    iters = list(c.psi_iters)
    nsolve = len(iters)
    # complex transforms: per BiCGSTAB iteration and field two operator applications of
    # four transforms each; the rest is the forward transform of each right-hand side
    per_iter_cfft = 8                                # per field: two operator applications
    cfft_fixed = c.cfft - per_iter_cfft * cfg.N * sum(iters)
    if cfg.ndim == 2:
        assert cfft_fixed == nsolve * cfg.N, (c.cfft, iters)   # the forward transform of each right-hand side
    return dict(real_transforms=c.rfft + c.irfft, cfft_fixed=cfft_fixed, cfft_per_iteration=per_iter_cfft,
                psi_solves=nsolve, psi_iters_reduced_grid=iters, N=cfg.N, ndim=cfg.ndim)


def main():
    out = {"convention": __doc__.split("The psi part")[0].strip(), "krylov_vector_passes": KRYLOV_VECTOR_PASSES}
    for wl, (n, nz) in CASES.items():
        c = counts(wl, n)
        kw, _, _, _ = ics.workload(wl, seed=0)
        Nx, Ny, Nz = kw["Nx"], kw["Ny"], kw.get("Nz", 0) or 1
        N = kw["N"]
        P = Nx * Ny * Nz
        H = (Nx // 2 + 1) * Ny * Nz
        rec = dict(c, grid=[Nx, Ny] + ([Nz] if Nz > 1 else []), vesicles=N, P=P, H=H)
        for s, name in ((8, "fp64"), (4, "fp32")):
            real = s * P + 2 * s * H
            rec[name] = {
                "nonpsi_transform_bytes": c["real_transforms"] * real,
                "psi_fixed_bytes_full": c["cfft_fixed"] * 4 * s * P,
                "psi_fixed_bytes_half": c["cfft_fixed"] * real,
                # per iteration of one system (its N fields)
                "psi_bytes_per_iteration_full": N * (c["cfft_per_iteration"] * 4 * s * P
                                                     + KRYLOV_VECTOR_PASSES * 2 * s * P),
                "psi_bytes_per_iteration_half": N * (c["cfft_per_iteration"] * real
                                                     + KRYLOV_VECTOR_PASSES * 2 * s * H),
            }
        out[wl] = rec
        print(wl, json.dumps(rec["fp64"]), flush=True)
    path = os.path.join(ROOT, "profiles", "algorithmic_bytes.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path)


if __name__ == "__main__":
    main()
