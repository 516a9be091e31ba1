"""generate_initial_condition on the device (vsav_generate_initial_condition)
against the oracle's restatement of Init.jl / Init_3d.jl."""
import math

import numpy as np
import pytest

from helpers import Cfg, rel

pytestmark = pytest.mark.gpu


def conf(N=1, goal="s", n=256, ndim=2, run_sizes=None):
    from vsav import ics
    V = sum(run_sizes) if run_sizes else N
    Nmax = max(run_sizes) if run_sizes else N
    kw = ics.params(0.01, Nmax, [0.1] * V, [0.8] * V, 1e-6, 1e-3, n, n, L=1.0,
                    Nz=(n if ndim == 3 else 0), goal=goal)
    kw["Lx"] = 1.0 * Nmax                                 # Init.jl:10-11: Nx = Ny = 256, Lx = 1.0 * N
    return kw


def oracle_conf(kw, N):
    from oracle.vsav_oracle import Config
    k = dict(kw)
    k["N"] = N
    k["psi_in_v"] = kw["psi_in_v"][:N]
    k["psi_out_v"] = kw["psi_out_v"][:N]
    return Config(**k)


def handle(kw, run_sizes=None, precision="fp64"):
    from vsav import Handle
    return Handle(Cfg(**kw), run_sizes=run_sizes, precision=precision)


CASES = [(1, "s", 1), (1, "s", 2), (1, "s", 3), (1, "s", 4), (1, "g", 1), (1, "g", 3), (1, "g", 4),
         (2, "g", 7), (2, "s", 8), (3, "g", 7), (1, "s", 5)]


@pytest.mark.parametrize("N,goal,st", CASES)
def test_reference_shapes_2d(N, goal, st):
    from oracle.vsav_oracle import reference_shapes
    kw = conf(N, goal)
    u = np.random.default_rng(st).uniform(size=20)
    h = handle(kw)
    h.generate_initial_condition(st, goal, u if st == 4 else None)
    phi, psi = reference_shapes(oracle_conf(kw, N), st, u)
    if phi.any():
        assert rel(h.get_field("phi"), phi) < 1e-13
    else:
        assert not h.get_field("phi").any()
    assert rel(h.get_field("psi"), psi) < 1e-13
    assert not h.get_field("u").any()
    # the rest of the initialisation is init_state's, from the same fields; mu = L_phi phi_hat
    # + ... amplifies last-bit differences of phi_hat by up to L_phi(k_max) / S3 (~1e5 here)
    h2 = handle(kw)
    h2.init_state(h.get_field("phi"), h.get_field("psi"))
    for k, tol in (("phi_hat", 1e-14), ("psi_hat", 1e-14), ("mu", 1e-10), ("nu", 1e-12)):
        assert rel(h.get_field(k), h2.get_field(k)) < tol, k
    np.testing.assert_allclose(h.get_scalars(), h2.get_scalars(), rtol=1e-12)
    h.close()
    h2.close()


def test_reference_ellipsoid_3d_fp32():
    from oracle.vsav_oracle import reference_shapes
    kw = conf(1, "g", n=64, ndim=3)
    h = handle(kw, precision="fp32")
    h.generate_initial_condition(1, "g")
    phi, psi = reference_shapes(oracle_conf(kw, 1), 1)
    assert rel(h.get_field("phi"), phi) < 1e-7
    assert rel(h.get_field("psi"), psi) < 1e-7
    h.close()


def test_reference_shapes_per_run():
    """An ensemble: each run gets the shapes of its own N and its own blob draws."""
    from oracle.vsav_oracle import reference_shapes
    rs = [1, 1, 1]
    kw = conf(run_sizes=rs)
    u = np.random.default_rng(7).uniform(size=(3, 20))
    h = handle(kw, run_sizes=rs)
    h.generate_initial_condition(4, "s", u)
    got = h.get_field("phi")
    for r in range(3):
        phi, _ = reference_shapes(oracle_conf(kw, 1), 4, u[r])
        assert rel(got[r], phi[0]) < 1e-13
    assert rel(got[0], got[1]) > 1e-3
    h.close()
    rs = [2, 3]
    kw = conf(run_sizes=rs, goal="g")
    h = handle(kw, run_sizes=rs)
    h.generate_initial_condition(7, "g")
    got = h.get_field("phi")
    p2, _ = reference_shapes(oracle_conf(kw, 2), 7)
    p3, _ = reference_shapes(oracle_conf(kw, 3), 7)
    assert rel(got[:2], p2) < 1e-13 and rel(got[2:], p3) < 1e-13
    h.close()


@pytest.mark.parametrize("N,goal,st", [(1, "s", 7), (2, "g", 1), (2, "s", 7), (2, "g", 8), (1, "s", 4)])
def test_reference_errors(N, goal, st):
    """The reference's error() cases (and state_type 4 without its draws) are
    argument errors; the handle stays usable."""
    from vsav import VsavError
    h = handle(conf(N, goal, n=32))
    with pytest.raises(VsavError):
        h.generate_initial_condition(st, goal)
    h.generate_initial_condition(1 if N == 1 else (7 if goal == "g" else 8), goal)
    h.close()
