"""Which transforms set the FP32 floor of the time step: rounding study on the oracle.

    python oracle/fp32_floor.py [workload] [steps] [variant,...]   # default multi2d_1024x8 3, all variants
                                    # writes (adds to) profiles/fp32_floor_<workload>_<steps>steps.json

Study infrastructure (not product code; NumPy FP64 on the oracle).  The oracle's
time step (src/simulation.jl:73-110, Steps 1-7 of src/Solvers.jl) runs with the
outputs of selected transforms rounded to FP32 (complex64 / float32 and back),
which is the first-order effect of running those transforms -- and the fields
they produce -- in FP32.  Sites, by the step that calls the transform:

  psi     the full complex fft / ifft of the psi BiCGSTAB (operator and right-hand
          side, Solvers.jl:39-53,68-69): an FP32 psi solve without refinement
  step1   the real transforms of Step 1 outside the psi solve: H1..H3 and MG
          (Solvers.jl:96-116), grad G, grad phi*, grad psi* and the advection terms
  step4   Step 4's transforms (Solvers.jl:267-338): the velocity derivatives,
          grad mu*, grad nu* and the coupling phi* grad mu* + psi* grad nu*
  step5   Step 5's transforms (Solvers.jl:344-423): grad phi*, grad psi*, grad mu*,
          grad nu*, the velocity derivatives and mu_1, nu_1, mu_2, nu_2
  update  the six irffts of the state update (simulation.jl:88-110)
  state   (not a transform) the spectral state phi^, psi^, mu^, nu^, u^, p^ stored in
          FP32 after every step, as the FP32-bulk path keeps it

Variants and what they answer:

  all          every site: the FP32-bulk path's arithmetic, to first order
  not_step45   every site except Steps 4 and 5, which stay FP64.  This keeps MORE in
               FP64 than keeping only the mu^/nu^ chain and the coupling wide (grad mu*,
               grad nu*, the coupling sum), so if it misses 1e-5 the narrower split misses
               too
  psi_only     only the psi solve in FP32 (no refinement)
  step1_only, step45_only, update_only, state_only   one site each
  update_state the state update's transforms and the stored spectral state
  transforms_fp64_state   every transform of Steps 1, 4, 5 and the psi solve in FP32, the
               state and its update in FP64
  psi_tol1e-6  no rounding; the psi BiCGSTAB stopped at rtol 1e-6 (the tolerance an
               FP32 psi solve reaches) instead of conf.tol

Each variant reports the relative L2 error of every field and of Q, R1..R3 against
the unrounded FP64 run after the same steps, and the maximum over the fields.
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "julia-vesicles-growth-and-shrinkage_b200"))

from oracle import vsav_oracle as O  # noqa: E402
from vsav import ics  # noqa: E402

STEP_SITES = {"solve_step1": "step1", "_solve_step1_3d": "step1", "solve_step4": "step4",
              "solve_step5": "step5", "step": "update", "monitor": "monitor"}

VARIANTS = {
    "fp64": set(),
    "all": {"psi", "step1", "step4", "step5", "update", "state"},
    "not_step45": {"psi", "step1", "update", "state"},
    "psi_only": {"psi"},
    "step1_only": {"step1"},
    "step45_only": {"step4", "step5"},
    "update_only": {"update"},
    "state_only": {"state"},
    "update_state": {"update", "state"},
    "psi_tol1e-6": {"tol:1e-6"},
    "transforms_fp64_state": {"psi", "step1", "step4", "step5"},
}

FIELDS = ("phi", "psi", "mu", "nu", "u", "p")
SCALARS = ("Q", "R1", "R2", "R3")


def _r32(a):
    if np.iscomplexobj(a):
        return a.astype(np.complex64).astype(np.complex128)
    return a.astype(np.float32).astype(np.float64)


class RoundingOps(O.Operators):
    """The oracle's transforms, with the outputs of the chosen sites rounded to FP32."""

    def __init__(self, cfg, sites, workers=None):
        super().__init__(cfg, workers=workers)
        self.sites = set(sites)

    def _site(self):
        f = sys._getframe(2)
        while f is not None:
            s = STEP_SITES.get(f.f_code.co_name)
            if s:
                return s
            f = f.f_back
        return "other"

    def _out(self, y, site):
        return _r32(y) if site in self.sites else y

    def rfft(self, f):
        return self._out(super().rfft(f), self._site())

    def irfft(self, F):
        return self._out(super().irfft(F), self._site())

    def fft(self, f):
        return self._out(super().fft(f), "psi")

    def ifft(self, F):
        return self._out(super().ifft(F), "psi")


def run_variant(cfg, phi, psi, steps, sites, workers):
    tol = [float(x[4:]) for x in sites if x.startswith("tol:")]
    orc = O.Oracle(cfg, psi_rtol=tol[0] if tol else None)
    orc.ops = RoundingOps(cfg, sites, workers)
    pres = O.make_state(cfg, phi, psi, orc.ops)
    O.init_state(cfg, pres, orc.ops)
    old = pres.copy()
    energy = []
    for n in range(1, steps + 1):
        orc.step(pres, old, n, cfg.dt)
        if "state" in sites:
            for name in ("phi_hat", "psi_hat", "mu_hat", "nu_hat", "u_hat", "p_hat"):
                setattr(pres, name, _r32(getattr(pres, name)))
        energy.append(orc.monitor(pres, old)[0])
    return pres, energy


def rel(a, b):
    nb = float(np.linalg.norm(np.ravel(b)))
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b))) / max(nb, 1e-300)


def main(workload="multi2d_1024x8", steps=3, names=None):
    kw, phi, psi, _ = ics.workload(workload, seed=0)
    kw["dt"] = 1e-5
    cfg = O.Config(**kw)
    workers = os.cpu_count()
    out = {"workload": workload, "grid": list(cfg.shape), "vesicles": cfg.N, "dt": cfg.dt, "steps": steps,
           "threads": workers, "method": "oracle step with the outputs of the named transform sites rounded "
           "to FP32; errors are relative L2 against the unrounded FP64 oracle after the same steps",
           "variants": {}}
    t0 = time.time()
    ref, e_ref = run_variant(cfg, phi, psi, steps, VARIANTS["fp64"], workers)
    out["fp64_seconds"] = time.time() - t0
    for name, sites in VARIANTS.items():
        if name == "fp64" or (names and name not in names):
            continue
        t0 = time.time()
        st, e = run_variant(cfg, phi, psi, steps, sites, workers)
        errs = {k: rel(getattr(st, k), getattr(ref, k)) for k in FIELDS}
        errs.update({k: abs(getattr(st, k) - getattr(ref, k)) / max(abs(getattr(ref, k)), 1e-300) for k in SCALARS})
        out["variants"][name] = {
            "sites": sorted(sites), "rel_err": errs,
            "max_field_err": max(errs[k] for k in FIELDS),
            "energy_non_increasing": bool(all(e[i + 1] <= e[i] * (1 + 1e-12) for i in range(len(e) - 1))),
            "seconds": time.time() - t0}
        print(name, json.dumps(out["variants"][name]), flush=True)
    path = os.path.join(ROOT, "profiles", f"fp32_floor_{workload}_{steps}steps.json")
    if os.path.exists(path):                 # add to the variants of an earlier run of this case
        with open(path) as f:
            old = json.load(f)
        old["variants"].update(out["variants"])
        out["variants"] = old["variants"]
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path)


if __name__ == "__main__":
    a = sys.argv[1:]
    main(a[0] if a else "multi2d_1024x8", int(a[1]) if len(a) > 1 else 3,
         a[2].split(",") if len(a) > 2 else None)
