"""Pins the oracle: rerunning it reproduces the committed golden fixtures
(tests/golden/make_golden.py) bit-for-bit up to FP64 summation order."""
import numpy as np
import pytest

from helpers import load_golden, rel
from oracle import vsav_oracle as O


@pytest.mark.parametrize("name", ["single2d_n64", "multi2d_n64_N2"])
def test_oracle_reproduces_golden(name):
    kw, g = load_golden(name)
    cfg = O.Config(**kw)
    steps = int(g["steps"])
    pres, old, E, A, orc = O.run(cfg, g["phi0"], g["psi0"], steps)
    for k in ("phi", "psi", "mu", "nu", "u", "p"):
        assert rel(getattr(pres, k), g[k]) < 1e-12, k
    np.testing.assert_allclose([pres.Q, pres.R1, pres.R2, pres.R3], g["scalars"], rtol=1e-12)
    np.testing.assert_allclose(E, g["energy"], rtol=1e-12)
    assert list(orc.counter.psi_iters) == list(g["psi_iters"])


def test_oracle_energy_non_increasing():
    """The modified energy (Utils.jl:96-141) is non-increasing along the
    golden trajectories (the unconditional stability of the SAV scheme)."""
    for name in ("single2d_n64", "multi2d_n64_N2", "single3d_n32"):
        _, g = load_golden(name)
        assert np.all(np.diff(g["energy"]) <= 0), name


def test_bicgstab_restatement_solves():
    """The restated Krylov bicgstab solves a small SPD-like complex system."""
    rng = np.random.default_rng(3)
    n = 40
    B = rng.standard_normal((n, n))
    A = np.eye(n) * 4 + 0.3 * (B + B.T) / np.sqrt(n)
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    d = 1.0 / np.diag(A)
    x, st = O.bicgstab(lambda v: A @ v, b, M=lambda r: d * r, atol=1e-14, rtol=1e-12, itmax=60)
    assert st.solved
    assert np.linalg.norm(A @ x - b) / np.linalg.norm(b) < 1e-10
    # itmax reached -> not solved, iterate returned
    x2, st2 = O.bicgstab(lambda v: A @ v, b, M=lambda r: d * r, atol=0.0, rtol=1e-30, itmax=3)
    assert not st2.solved and st2.niter == 3 and "maximum" in st2.status


def test_wc_negative_raises():
    """W3 + C3 < 0 is fatal in the reference (Utils.jl:188)."""
    kw, g = load_golden("single2d_n64")
    kw = dict(kw, C3=-1e9)
    cfg = O.Config(**kw)
    with pytest.raises(O.WCNegative):
        O.run(cfg, g["phi0"], g["psi0"], 1)
