"""Generates the golden fixtures of the SAV step from the CPU oracle.

    python tests/golden/make_golden.py [name ...]

Two kinds of fixture:

* small cases (CASES): the seeded initial condition, the config keyword
  arguments and the oracle's full state after K steps (fields, SAV scalars,
  modified energy, area ratio, BiCGSTAB iteration counts);
* the benchmark configurations at their full sizes (CONFIG_CASES: 128^2 x 1,
  512^2 x 4, 128^3 x 1, 1024^2 x 8), whose fields are too large to commit:
  the workload is rebuilt from its seed (vsav.ics), and each field of the
  final state is kept as a strided sample, its L2 norm and its projections on
  two seeded standard-normal vectors.  Scalars, the whole energy / area
  history and every BiCGSTAB iteration count are kept in full, and so is
  each field's round-off floor: its relative change when the oracle reruns
  from the initial phi perturbed by a relative 1e-15.

The GPU parity tests load these, so they need neither the reference nor a
rerun of the oracle.  The oracle runs with all host threads.
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "julia-vesicles-growth-and-shrinkage_b200"))

from oracle import vsav_oracle as O  # noqa: E402
from vsav import ics  # noqa: E402

FIELDS = ("phi", "psi", "mu", "nu", "u", "p")

CASES = {
    # name: (workload, n, N, eps, dt, steps)
    "single2d_n64": ("single2d_128", 64, None, None, 1e-6, 4),
    "multi2d_n64_N2": ("multi2d_512x4", 64, 2, 0.2, 1e-6, 3),
    "single3d_n32": ("single3d_128", 32, None, 0.3, 1e-5, 3),
}

# the benchmark configurations at full size: (workload, dt, steps, sample stride, seed)
# dt: the largest of the probed steps at which the reference scheme stays stable
# over the configuration's step count (vsav/ics.py, tests/test_oracle_dt.py,
# tests/test_gpu_configs.py)
CONFIG_CASES = {
    "cfg_single2d_128": ("single2d_128", 1e-5, 200, 2, 0),
    "cfg_multi2d_512x4": ("multi2d_512x4", 5e-6, 12, 8, 0),
    "cfg_single3d_128": ("single3d_128", 1e-5, 12, 8, 0),
    "cfg_multi2d_1024x8": ("multi2d_1024x8", 1e-5, 2, 16, 0),
}
PROJ_SEEDS = (101, 202)
PERTURB_SEED = 7


def sample(a, stride):
    """a[..., ::stride, ::stride] over the spatial axes (2 or 3) of a field array."""
    nd = 3 if a.ndim == 4 else 2
    idx = (Ellipsis,) + (slice(None, None, stride),) * nd
    return np.ascontiguousarray(a[idx])


def projection(a, seed):
    """<w, a> with w standard normal of a's size (numpy PCG64, `seed`), and ||w||."""
    w = np.random.default_rng(seed).standard_normal(a.size)
    return float(w @ a.ravel()), float(np.linalg.norm(w))


def config_state(name, oracle_workers=None):
    """(config kwargs, phi0, psi0, steps, stride) of a configuration case."""
    wl, dt, steps, stride, seed = CONFIG_CASES[name]
    kw, phi, psi, _ = ics.workload(wl, seed=seed)
    kw["dt"] = dt
    kw["T"] = steps * dt
    return kw, phi, psi, steps, stride


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


def make_config(name):
    t0 = time.time()
    wl, dt, steps, stride, seed = CONFIG_CASES[name]
    kw, phi, psi, steps, stride = config_state(name)
    cfg = O.Config(**kw)
    orc = O.Oracle(cfg, workers=os.cpu_count())
    pres, old, E, A, orc = O.run(cfg, phi, psi, steps, oracle=orc)
    out = dict(scalars=np.array([pres.Q, pres.R1, pres.R2, pres.R3]), A0=pres.A0,
               energy=np.array(E), area=np.array(A),
               psi_iters=np.array(orc.counter.psi_iters, dtype=np.int32))
    # the trajectory's own round-off floor: the oracle's change in each field when the
    # initial phi is perturbed by a relative 1e-15 (seeded); a comparison of two FP64
    # implementations cannot be expected to agree more closely than this
    rng = np.random.default_rng(PERTURB_SEED)
    phi_p = phi * (1.0 + 1e-15 * rng.standard_normal(phi.shape))
    pres_p, _, _, _, _ = O.run(cfg, phi_p, psi, steps, oracle=O.Oracle(cfg, workers=os.cpu_count()), monitor=False)
    for k in FIELDS:
        a, b = getattr(pres, k), getattr(pres_p, k)
        out[k + "_floor"] = np.linalg.norm(a - b) / max(np.linalg.norm(a), 1e-300)
    for k in FIELDS:
        a = getattr(pres, k)
        out[k + "_sample"] = sample(a, stride)
        out[k + "_norm"] = np.linalg.norm(a)
        out[k + "_proj"] = np.array([projection(a, s) for s in PROJ_SEEDS])
    kwj = {k: (list(v) if isinstance(v, (list, np.ndarray)) else v) for k, v in kw.items()}
    meta = dict(workload=wl, seed=seed, steps=steps, stride=stride, dt=dt, proj_seeds=list(PROJ_SEEDS),
                oracle_seconds=time.time() - t0)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), config=json.dumps(kwj), meta=json.dumps(meta), **out)
    print(name, f"{time.time() - t0:.1f}s", "energy", E[:3], "...", E[-1], "iters", orc.counter.psi_iters[-6:],
          flush=True)


if __name__ == "__main__":
    for nm in (sys.argv[1:] or list(CASES) + list(CONFIG_CASES)):
        (make_config if nm in CONFIG_CASES else make)(nm)
