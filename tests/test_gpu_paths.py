"""The alternative code paths selected by environment switches give the
default path's results: the unfused psi operator (VSAV_PSI_FUSED=0), the psi
operator in L2-sized chunks of fields (VSAV_PSI_CHUNK_MB), eager launches
instead of CUDA-graph replay (VSAV_GRAPH=0), and either form of the operator's
forward pass (VSAV_PSI_SPLIT=1: k_psi_cols_fwd2 + k_psi_combz; 0: the fused
k_psi_cols_comb), whichever the autotuner picked, and the operator's x pass as
the classic kernel (VSAV_PSI_BULK=0) or as each block shape of the bulk-copy-fed
persistent kernel (VSAV_PSI_BULK=2, 3, 4; FP32 psi solves only), and the y pass of
the field transforms as the classic kernel (VSAV_COLS_TMA=0) or as each block
shape of the TMA-fed persistent kernel (VSAV_COLS_TMA=2, 3), and their c2r x pass
as the classic kernel or the bulk-copy-fed persistent one (VSAV_C2R_BULK=0, 1)."""
import numpy as np
import pytest

from helpers import Cfg, rel

pytestmark = pytest.mark.gpu

FIELDS = ("phi", "psi", "mu", "nu", "u", "p")


def run(kw, phi, psi, prec, steps=3):
    from vsav import Handle
    h = Handle(Cfg(**kw), precision=prec, psi_rtol=1e-8 if prec == "fp32" else None, psi_itmax=60)
    h.init_state(phi, psi)
    E, _ = h.run(1, steps, monitor=True)
    out = {k: h.get_field(k) for k in FIELDS}
    out["E"] = E[:, 0]
    out["iters"] = h.psi_stats()[:, 0].copy()
    h.close()
    return out


@pytest.mark.parametrize("prec", ["fp64", "mixed", "fp32"])
@pytest.mark.parametrize("env", [("VSAV_PSI_FUSED", "0"), ("VSAV_PSI_CHUNK_MB", "1"), ("VSAV_GRAPH", "0"),
                                 ("VSAV_PSI_SPLIT", "1"), ("VSAV_PSI_SPLIT", "0"), ("VSAV_PSI_BULK", "0"),
                                 ("VSAV_PSI_BULK", "2"), ("VSAV_PSI_BULK", "3"), ("VSAV_PSI_BULK", "4"),
                                 ("VSAV_COLS_TMA", "0"), ("VSAV_COLS_TMA", "2"), ("VSAV_COLS_TMA", "3")])
def test_switches_keep_the_results(prec, env, monkeypatch):
    from vsav import ics
    kw, phi, psi, _ = ics.workload("multi2d_512x4", seed=2, n_override=256, N_override=2, eps_override=0.08)
    kw["dt"] = 1e-6
    base = run(kw, phi, psi, prec)
    monkeypatch.setenv(*env)
    alt = run(kw, phi, psi, prec)
    # FP64 (and the FP64-refined mixed path): the same solve up to rounding order; FP32: the
    # alternative kernels round differently, and mu/u/p amplify the FP32 floor (FP32-bulk bars)
    if prec == "fp32" and env[0] != "VSAV_GRAPH":
        tol = {"phi": 1e-5, "psi": 1e-5, "nu": 1e-5, "mu": 1e-3, "u": 1e-3, "p": 1e-3}
    else:
        tol = {k: 1e-10 for k in FIELDS}
    for k in FIELDS:
        assert rel(alt[k], base[k]) < tol[k], (k, rel(alt[k], base[k]))
    np.testing.assert_allclose(alt["E"], base["E"], rtol=1e-6 if prec == "fp32" else 1e-10)
    if prec != "fp32":
        assert np.array_equal(alt["iters"], base["iters"])


@pytest.mark.parametrize("n", [512, 1024, 2048])
@pytest.mark.parametrize("shape", ["2", "3", "4"])
def test_bulk_x_pass_block_shapes(n, shape, monkeypatch):
    """Every block shape of the bulk-copy-fed x pass at the row lengths 512, 1024
    and 2048 (E 32 is usable from 1024 on) gives the classic kernel's results in
    the mixed path, whose FP32 psi solves run through it."""
    from vsav import ics
    kw, phi, psi, _ = ics.workload("multi2d_512x4", seed=3, n_override=n, N_override=1, eps_override=0.08)
    kw["dt"] = 1e-6
    monkeypatch.setenv("VSAV_PSI_BULK", "0")
    base = run(kw, phi, psi, "mixed", steps=2)
    monkeypatch.setenv("VSAV_PSI_BULK", shape)
    alt = run(kw, phi, psi, "mixed", steps=2)
    for k in FIELDS:
        assert rel(alt[k], base[k]) < 1e-10, (k, rel(alt[k], base[k]))
    np.testing.assert_allclose(alt["E"], base["E"], rtol=1e-10)


@pytest.mark.parametrize("n", [256, 512, 1024])
@pytest.mark.parametrize("shape", ["2", "3"])
def test_field_column_tma_block_shapes(n, shape, monkeypatch):
    """Both block shapes of the TMA-fed y pass of the field transforms at the column
    lengths 256, 512 and 1024 give the classic kernel's results on the FP64 parity
    path (every field transform of Steps 1-7 and the state update runs through it).
    The classic variant the autotuner picks may split the radix differently, so the
    fields agree up to rounding order, which the velocity amplifies (1e-10 bar)."""
    from vsav import ics
    kw, phi, psi, _ = ics.workload("multi2d_512x4", seed=4, n_override=n, N_override=2, eps_override=0.08)
    kw["dt"] = 1e-6
    monkeypatch.setenv("VSAV_COLS_TMA", "0")
    base = run(kw, phi, psi, "fp64", steps=2)
    monkeypatch.setenv("VSAV_COLS_TMA", shape)
    alt = run(kw, phi, psi, "fp64", steps=2)
    for k in FIELDS:
        assert rel(alt[k], base[k]) < 1e-10, (k, rel(alt[k], base[k]))
    np.testing.assert_allclose(alt["E"], base["E"], rtol=1e-10)
    assert np.array_equal(alt["iters"], base["iters"])


@pytest.mark.parametrize("n", [512, 1024, 2048])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_c2r_bulk_pass(n, prec, monkeypatch):
    """The bulk-copy-fed c2r x pass at the row lengths 512, 1024 and 2048 (half-length
    transforms of 256, 512 and 1024 points) gives the classic kernel's results: every
    half-spectrum to real field transform of Steps 1-7 and the state update runs
    through it.  The classic variant the autotuner picks may split the radix
    differently, so the bar is rounding order amplified by the velocity (1e-10)."""
    from vsav import ics
    kw, phi, psi, _ = ics.workload("multi2d_512x4", seed=5, n_override=n, N_override=1, eps_override=0.08)
    kw["dt"] = 1e-6
    monkeypatch.setenv("VSAV_C2R_BULK", "0")
    base = run(kw, phi, psi, prec, steps=2)
    monkeypatch.setenv("VSAV_C2R_BULK", "1")
    alt = run(kw, phi, psi, prec, steps=2)
    for k in FIELDS:
        assert rel(alt[k], base[k]) < 1e-10, (k, rel(alt[k], base[k]))
    np.testing.assert_allclose(alt["E"], base["E"], rtol=1e-10)
    assert np.array_equal(alt["iters"], base["iters"])
