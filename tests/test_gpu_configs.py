"""GPU parity at the benchmark configurations' full sizes.

The goldens (tests/golden/make_golden.py, CONFIG_CASES) hold the CPU oracle's
state after K steps of each configuration -- 128^2 x 1 for its 200 steps,
512^2 x 4 and 128^3 x 1 for 12 steps (past the BDF1 -> BDF2 switch), 1024^2 x
8 for 2 steps -- as strided samples, L2 norms and seeded projections of
every field, plus the scalars, the whole energy / area histories and every
BiCGSTAB iteration count, and each field's round-off floor (the oracle's
own change under a 1e-15 relative perturbation of the initial phi).  The
FP64 GPU path must match them to 1e-10 relative, or to ten times a field's
floor where that is larger (the mixed path, psi to a true relative residual
of 1e-8, to 1e-5).
Beyond the oracle's reach, the FP64 GPU path runs the configurations' full
step counts at the chosen dt with a non-increasing modified energy.
"""
import json
import os

import numpy as np
import pytest

from helpers import Cfg, rel

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIELDS = ("phi", "psi", "mu", "nu", "u", "p")
NAMES = ["cfg_single2d_128", "cfg_multi2d_512x4", "cfg_single3d_128", "cfg_multi2d_1024x8"]


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    kw = json.loads(str(z["config"]))
    meta = json.loads(str(z["meta"]))
    return kw, meta, {k: z[k] for k in z.files if k not in ("config", "meta")}


def initial(meta, kw):
    from vsav import ics
    _, phi, psi, _ = ics.workload(meta["workload"], seed=meta["seed"])
    return phi, psi


def field_errors(h, g, meta):
    """Per field: relative L2 error of the strided sample, of the norm, and the
    largest projection error relative to ||w|| ||a|| (each <= the field's
    relative L2 error)."""
    import sys
    sys.path.insert(0, GOLDEN)
    from make_golden import projection, sample
    out = {}
    for k in FIELDS:
        a = h.get_field(k)
        if k in ("u", "p"):
            a = a[0]                        # the handle's run axis (one run); the oracle has none
        es = rel(sample(a, meta["stride"]), g[k + "_sample"])
        en = abs(np.linalg.norm(a) - g[k + "_norm"]) / max(g[k + "_norm"], 1e-300)
        ep = 0.0
        for (pv, wn), s in zip(g[k + "_proj"], meta["proj_seeds"]):
            p, _ = projection(a, s)
            ep = max(ep, abs(p - pv) / max(wn * g[k + "_norm"], 1e-300))
        out[k] = max(es, en, ep)
    return out


def fp64_bar(g, k):
    """The FP64 parity bar of field k: 1e-10, or 10x the golden's recorded round-off floor."""
    return max(1e-10, 10.0 * float(g[k + "_floor"]))


def run_steps(h, steps):
    """Steps 1..steps one vsav_run call each (graph replays after the first),
    with the BiCGSTAB iteration counts of every step."""
    E, A, iters = [], [], []
    for n in range(1, steps + 1):
        e, a = h.run(n, 1, monitor=True)
        E.append(e[0, 0])
        A.append(a[0, 0])
        if h.has_psi_solve():
            iters += [int(x) for x in h.psi_stats()[:, 0]]
    return np.array(E), np.array(A), iters


@pytest.mark.parametrize("name", NAMES)
def test_fp64_matches_oracle_at_full_size(name):
    from vsav import Handle
    kw, meta, g = load(name)
    phi, psi = initial(meta, kw)
    h = Handle(Cfg(**kw), precision="fp64")
    h.init_state(phi, psi)
    np.testing.assert_allclose(h.get_A0(), g["A0"], rtol=1e-12)
    E, A, iters = run_steps(h, meta["steps"])
    err = field_errors(h, g, meta)
    # 1e-10, or ten times the field's own round-off floor where the trajectory amplifies
    # a 1e-15 change of the initial state beyond 1e-11 (the velocity at 1024^2 x 8)
    bad = {k: (v, fp64_bar(g, k)) for k, v in err.items() if not v < fp64_bar(g, k)}
    assert not bad, (bad, err)
    # Q is O(1e-6) in the 3D run: an absolute floor of 1e-12 on Q, R1..R3
    np.testing.assert_allclose(h.get_scalars()[0], g["scalars"], rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(E, g["energy"], rtol=1e-10)
    np.testing.assert_allclose(A, g["area"], rtol=1e-8, atol=1e-13)
    if iters:
        assert iters == [int(x) for x in g["psi_iters"]]
    assert np.all(np.diff(E) <= 0)
    h.close()


@pytest.mark.parametrize("name", ["cfg_single2d_128", "cfg_multi2d_512x4", "cfg_multi2d_1024x8"])
def test_mixed_matches_oracle_at_full_size(name):
    """FP64 fields and transforms, the psi BiCGSTAB in FP32 inside FP64
    refinement, stopped on the true residual at 1e-8: every field within 1e-5."""
    from vsav import Handle
    kw, meta, g = load(name)
    phi, psi = initial(meta, kw)
    h = Handle(Cfg(**kw), precision="mixed", psi_rtol=1e-8, psi_stop="true", psi_check=True)
    h.init_state(phi, psi)
    E, A = h.run(1, meta["steps"], monitor=True)
    err = field_errors(h, g, meta)
    assert max(err.values()) < 1e-5, err
    np.testing.assert_allclose(h.get_scalars()[0], g["scalars"], rtol=1e-5)
    np.testing.assert_allclose(E[:, 0], g["energy"], rtol=1e-5)
    assert np.all(np.diff(E[:, 0]) <= 0)
    # the measured FP64 residual of the last step's solves reaches the requested 1e-8
    assert np.max(h.true_residuals()) < 1e-8 * 1.05, h.true_residuals()
    h.close()


@pytest.mark.parametrize("workload,dt,steps", [("multi2d_512x4", 5e-6, 500), ("multi2d_1024x8", 1e-5, 100),
                                               ("single3d_128", 1e-5, 100), ("single2d_128", 1e-5, 200)])
def test_full_step_count_is_stable(workload, dt, steps):
    """The configuration's whole step count at the chosen dt: no fatal W + C < 0,
    finite scalars, modified energy non-increasing, psi solves within itmax."""
    from vsav import Handle, ics
    kw, phi, psi, _ = ics.workload(workload, seed=0)
    kw["dt"] = dt
    h = Handle(Cfg(**kw), precision="fp64")
    h.init_state(phi, psi)
    E, A = h.run(1, steps, monitor=True)
    assert np.all(np.isfinite(E)) and np.all(np.diff(E[:, 0]) <= 0)
    assert np.all(np.isfinite(h.get_scalars()))
    h.close()


def test_512x4_at_1e5_stops_before_its_500_steps():
    """The evidence for 512^2 x 4's smaller step: at dt = 1e-5 the reference
    scheme (FP64 path, = the oracle to 1e-10) ends in the fatal W3 + C3 < 0
    before step 130 (step 121 with seed 0)."""
    from vsav import Handle, WCNegativeError, ics
    kw, phi, psi, _ = ics.workload("multi2d_512x4", seed=0)
    kw["dt"] = 1e-5
    h = Handle(Cfg(**kw), precision="fp64")
    h.init_state(phi, psi)
    with pytest.raises(WCNegativeError):
        h.run(1, 130, monitor=True)
    h.close()


@pytest.mark.parametrize("stop", ["krylov", "true"])
def test_true_residual_check_and_stop(stop):
    """psi_check measures ||b - A x|| / ||b||: with the true-residual stop the
    measured residual is at the requested tolerance; with Krylov.jl's
    preconditioned stop (the reference) it is larger, since the diagonal
    preconditioner damps the high wavenumbers the residual lives at."""
    from vsav import Handle
    kw, meta, g = load("cfg_multi2d_512x4")
    phi, psi = initial(meta, kw)
    h = Handle(Cfg(**kw), precision="fp64", psi_rtol=1e-8, psi_stop=stop, psi_check=True)
    h.init_state(phi, psi)
    h.run(1, 3, monitor=True)
    tr = h.true_residuals()
    st = h.psi_stats()
    assert np.all(st[:, 1] == 1), st              # solved
    if stop == "true":
        assert np.all(tr <= 1e-8 * 1.05), tr
        assert np.all(tr > 1e-12), tr
    else:
        assert np.all(tr > 0.0)
    h.close()


@pytest.mark.parametrize("tma", ["0", "1"])
def test_mixed_both_column_pass_forms(tma, monkeypatch):
    """The psi column passes in their classic form and in the TMA-fed
    persistent form (VSAV_PSI_TMA forces either; the autotuner otherwise
    picks the faster): both reproduce the oracle at 512^2 x 4 within the
    mixed bar, and the handle reports the form it ran."""
    from vsav import Handle
    monkeypatch.setenv("VSAV_PSI_TMA", tma)
    kw, meta, g = load("cfg_multi2d_512x4")
    phi, psi = initial(meta, kw)
    h = Handle(Cfg(**kw), precision="mixed", psi_rtol=1e-8, psi_stop="true", psi_check=True)
    assert h.tuning()["psi_fp32"]["psi_column_passes"] == ("tma" if tma == "1" else "classic")
    h.init_state(phi, psi)
    E, A = h.run(1, meta["steps"], monitor=True)
    err = field_errors(h, g, meta)
    assert max(err.values()) < 1e-5, err
    assert np.max(h.true_residuals()) < 1e-8 * 1.05, h.true_residuals()
    h.close()


@pytest.mark.parametrize("var", [0, 1])
def test_tma_tile_shapes(var, tmp_path, monkeypatch):
    """Each block shape of the TMA-fed column passes (0: E 16 / 512 threads,
    1: E 8 / 512 with half-width tiles), pinned through a tuning file: the mixed
    path reproduces the oracle at 512^2 x 4 within its bar."""
    import json as js
    from vsav import Handle
    key = "4:512x512x1:V4:R1:f0"               # the FP32 psi helper of this configuration
    code = 1 | var << 1 | var << 3             # TMA on, both passes in shape `var`
    path = tmp_path / "tune.json"
    path.write_text(js.dumps({key: [0] * 9 + [0, code]}))
    monkeypatch.setenv("VSAV_TUNE_FILE", str(path))
    kw, meta, g = load("cfg_multi2d_512x4")
    phi, psi = initial(meta, kw)
    h = Handle(Cfg(**kw), precision="mixed", psi_rtol=1e-8, psi_stop="true", psi_check=True)
    t = h.tuning()["psi_fp32"]
    assert t["source"] == "file" and t["psi_column_passes"] == "tma", t
    shape = {0: "E16/NT512", 1: "E8/NT512"}[var]
    assert t["variants"]["psi_inv2_tma"] == shape and t["variants"]["psi_comb_tma"] == shape, t
    h.init_state(phi, psi)
    E, A = h.run(1, meta["steps"], monitor=True)
    err = field_errors(h, g, meta)
    assert max(err.values()) < 1e-5, err
    assert np.max(h.true_residuals()) < 1e-8 * 1.05, h.true_residuals()
    h.close()
