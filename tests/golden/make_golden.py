"""Generates the golden fixtures of the SAV step from the CPU oracle.

    python tests/golden/make_golden.py

Each fixture holds the seeded initial condition, the config keyword
arguments, and the oracle's state after K steps (fields, SAV scalars, modified
energy, area ratio, BiCGSTAB iteration counts).  The GPU parity tests load them,
so they need neither the reference nor a rerun of the oracle.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "julia-vesicles-growth-and-shrinkage_b200"))

from oracle import vsav_oracle as O  # noqa: E402
from vsav import ics  # noqa: E402

CASES = {
    # name: (workload, n, N, eps, dt, steps)
    "single2d_n64": ("single2d_128", 64, None, None, 1e-6, 4),
    "multi2d_n64_N2": ("multi2d_512x4", 64, 2, 0.2, 1e-6, 3),
    "single3d_n32": ("single3d_128", 32, None, 0.3, 1e-5, 3),
}


def make(name):
    wl, n, N, eps, dt, steps = CASES[name]
    kw, phi, psi, _ = ics.workload(wl, seed=0, n_override=n, N_override=N, eps_override=eps)
    kw["dt"] = dt
    kw["T"] = steps * dt
    cfg = O.Config(**kw)
    pres, old, E, A, orc = O.run(cfg, phi, psi, steps)
    out = dict(phi0=phi, psi0=psi,
               phi=pres.phi, psi=pres.psi, mu=pres.mu, nu=pres.nu, u=pres.u, p=pres.p,
               scalars=np.array([pres.Q, pres.R1, pres.R2, pres.R3]), A0=pres.A0,
               energy=np.array(E), area=np.array(A),
               psi_iters=np.array(orc.counter.psi_iters, dtype=np.int32))
    kwj = {k: (list(v) if isinstance(v, (list, np.ndarray)) else v) for k, v in kw.items()}
    np.savez_compressed(os.path.join(HERE, name + ".npz"), config=json.dumps(kwj), steps=steps, **out)
    print(name, "energy", E, "iters", orc.counter.psi_iters)


if __name__ == "__main__":
    for nm in (sys.argv[1:] or CASES):
        make(nm)
