"""The 3D variable-mobility psi solve on the GPU (vsav_options.psi3d_variable)
against the oracle's restatement: the 2D scheme's M_psi(phi*) and
diagonal-preconditioned BiCGSTAB (Solvers.jl:26-81) on 3D full spectra, in
place of the reference's constant-mobility division (Solvers_3d.jl:28-30)."""
import numpy as np
import pytest

from helpers import Cfg, rel

pytestmark = pytest.mark.gpu

FIELDS = ("phi", "psi", "mu", "nu", "u", "p")


def kw3(n=32, M0=0.5, dt=1e-5):
    from vsav import ics
    kw = ics.params(0.2, 1, [0.65], [0.8], dt, 100 * dt, n, n, Nz=n, goal="g")
    kw["M0_psi"] = M0
    return kw


def oracle_run(kw, phi, psi, steps, variable=True):
    from oracle import vsav_oracle as O
    c = O.Config(**kw)
    orc = O.Oracle(c, psi3d_variable=variable)
    pres, _, E, A, _ = O.run(c, phi, psi, steps, oracle=orc)
    return pres, np.array(E), orc


def handle(kw, **opt):
    from vsav import Handle
    return Handle(Cfg(**kw), **opt)


@pytest.mark.parametrize("graph", [True, False])
def test_variable_mobility_3d_vs_oracle(graph):
    from vsav import ics
    kw = kw3()
    phi, psi = ics.single3d(32, 0.2, 1)
    steps = 3
    pres, E, orc = oracle_run(kw, phi, psi, steps)
    h = handle(kw, psi3d_variable=True, graph=graph)
    h.init_state(phi, psi)
    Eg, _ = h.run(1, steps, monitor=True)
    for k in FIELDS:
        assert rel(h.get_field(k), getattr(pres, k)) < 1e-10, (k, rel(h.get_field(k), getattr(pres, k)))
    np.testing.assert_allclose(Eg[:, 0], E, rtol=1e-10)
    st = h.psi_stats()
    assert np.all(st[:, 1] == 1)
    assert list(st[:, 0].astype(int)) == [s.niter for s in orc.last_psi_stats]
    h.close()


def test_constant_mobility_limit_matches_the_reference_3d_path():
    """M0_psi = 0 makes M_psi the constant 0.1: the Krylov path must give the
    reference's own 3D spectral division run with M0_psi = 0.1."""
    from vsav import ics
    phi, psi = ics.single3d(32, 0.2, 2)
    hv = handle(kw3(M0=0.0), psi3d_variable=True)
    hc = handle(kw3(M0=0.1))
    for h in (hv, hc):
        h.init_state(phi, psi)
        h.run(1, 3)
    for k in FIELDS:
        assert rel(hv.get_field(k), hc.get_field(k)) < 1e-10, k
    assert hv.psi_stats()[:, 0].max() <= 2
    hv.close()
    hc.close()


def test_variable_mobility_3d_fp32():
    from vsav import ics
    kw = kw3()
    phi, psi = ics.single3d(32, 0.2, 1)
    pres, E, _ = oracle_run(kw, phi, psi, 3)
    h = handle(kw, psi3d_variable=True, precision="fp32", psi_rtol=1e-8, psi_itmax=60)
    h.init_state(phi, psi)
    Eg, _ = h.run(1, 3, monitor=True)
    for k, bar in (("phi", 1e-5), ("psi", 1e-5), ("nu", 1e-5)):
        assert rel(h.get_field(k), getattr(pres, k)) < bar, k
    assert np.max(np.abs(Eg[:, 0] - E) / np.abs(E)) < 1e-5
    h.close()


def test_variable_mobility_3d_mixed():
    """FP64 fields with the 3D psi BiCGSTAB in FP32 inside FP64 refinement: at conf.tol 1e-12
    (two FP32 sweeps of 1e-6) the fields stay at FP64 accuracy."""
    from vsav import ics
    kw = kw3()
    phi, psi = ics.single3d(32, 0.2, 1)
    pres, E, _ = oracle_run(kw, phi, psi, 3)
    h = handle(kw, psi3d_variable=True, precision="mixed")
    h.init_state(phi, psi)
    Eg, _ = h.run(1, 3, monitor=True)
    for k in FIELDS:
        assert rel(h.get_field(k), getattr(pres, k)) < 1e-8, (k, rel(h.get_field(k), getattr(pres, k)))
    np.testing.assert_allclose(Eg[:, 0], E, rtol=1e-9)
    assert np.all(h.psi_stats()[:, 1] == 1)
    h.close()


def test_variable_mobility_3d_ensemble():
    """Two 3D runs in one handle solve their psi systems independently."""
    from vsav import ics
    kw = kw3()
    runs = [ics.single3d(32, 0.2, s) for s in (1, 2)]
    kwe = dict(kw, psi_in_v=kw["psi_in_v"] * 2, psi_out_v=kw["psi_out_v"] * 2)
    he = handle(kwe, run_sizes=[1, 1], psi3d_variable=True)
    he.init_state(np.concatenate([r[0] for r in runs]), np.concatenate([r[1] for r in runs]))
    he.run(1, 2)
    for r, (phi, psi) in enumerate(runs):
        h = handle(kw, psi3d_variable=True)
        h.init_state(phi, psi)
        h.run(1, 2)
        assert rel(he.get_field("psi")[r:r + 1], h.get_field("psi")) < 1e-12
        h.close()
    he.close()


def test_variable_mobility_3d_rejects_other_forms():
    from vsav import VsavError
    with pytest.raises(VsavError):
        handle(kw3(n=16), psi3d_variable=True, psi_form="half")
    with pytest.raises(VsavError):
        handle(kw3(n=16), psi3d_variable=True, psi_precond="flex_diag")
