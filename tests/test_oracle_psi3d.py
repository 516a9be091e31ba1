"""The 3D variable-mobility psi solve (an extension of the reference, whose 3D
Step 1 divides by a constant-mobility symbol, Solvers_3d.jl:28-30): the 2D
scheme's M_psi(phi*) and BiCGSTAB (Solvers.jl:26-81) on 3D full spectra.

Pin: with M0_psi = 0 the mobility is the constant 0.1 (Utils_3d.jl:20), the
operator is diagonal, and the solve must reproduce the reference's own 3D path
run with M0_psi = 0.1."""
import numpy as np

from helpers import rel
from oracle import vsav_oracle as O


def cfg3(n=16, M0=0.5):
    from vsav import ics
    kw = ics.params(0.2, 1, [0.65], [0.8], 1e-5, 1e-3, n, n, Nz=n, goal="g")
    kw["M0_psi"] = M0
    return O.Config(**kw)


def state(c, seed=1):
    from vsav import ics
    phi, psi = ics.single3d(c.Nx, c.epsilon, seed)
    return phi, psi


def test_constant_mobility_reduces_to_the_reference_3d_path():
    cv, cc = cfg3(M0=0.0), cfg3(M0=0.1)
    phi, psi = state(cv)
    pv, _, Ev, _, ov = O.run(cv, phi, psi, 3, oracle=O.Oracle(cv, psi3d_variable=True))
    pc, _, Ec, _, _ = O.run(cc, phi, psi, 3)
    for k in ("phi", "psi", "u", "mu", "nu"):
        assert rel(getattr(pv, k), getattr(pc, k)) < 1e-10, k
    np.testing.assert_allclose(Ev, Ec, rtol=1e-11)
    assert max(ov.counter.psi_iters) <= 2


def test_variable_mobility_converges_and_changes_psi():
    c = cfg3(M0=0.5)
    phi, psi = state(c)
    orc = O.Oracle(c, psi3d_variable=True)
    pv, _, Ev, _, _ = O.run(c, phi, psi, 3, oracle=orc)
    assert all(s.solved for s in orc.last_psi_stats)
    assert max(orc.counter.psi_iters) < 20
    pc, _, _, _, _ = O.run(c, phi, psi, 3)
    assert rel(pv.psi, pc.psi) > 1e-8                    # the mobility field matters
    assert np.all(np.diff(Ev) <= 0)
