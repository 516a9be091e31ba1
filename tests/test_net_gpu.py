"""GPU checks of the learned psi preconditioner, through the C ABI:
forward and gradient kernels against the FP64 NumPy reference
(oracle/precond_net.py, same BF16-rounded weights), the fused tensor-core
inference kernel, Adam training, the flexible BiCGSTAB with the diagonal and
with the learned correction, and the harvest of training pairs.
Bars: FP32 kernels within 1e-5 (forward) / 1e-4 (gradient) relative L2 of
the FP64 reference; the fused kernel (BF16 activations) within 2e-2."""
import warnings

import numpy as np
import pytest

from helpers import Cfg, load_golden, rel

pytestmark = pytest.mark.gpu


def _theta(seed=0):
    from oracle import precond_net as P
    rng = np.random.default_rng(seed)
    th = P.init_params(seed)
    th += 0.02 * rng.standard_normal(th.size)          # non-zero biases, non-trivial last layer
    return th


@pytest.mark.parametrize("periodic,shape", [(True, (2, 2, 32, 48)), (False, (3, 2, 30, 27))])
def test_forward_and_gradient_vs_oracle(periodic, shape):
    from oracle import precond_net as P
    from vsav.net import Net
    rng = np.random.default_rng(2)
    th = _theta(1)
    x = rng.standard_normal(shape).astype(np.float32)
    B, _, H, W = shape
    Ho, Wo = (H, W) if periodic else (H - 10, W - 10)
    t = rng.standard_normal((B, 1, Ho, Wo)).astype(np.float32)
    n = Net(B * H * W)
    n.set_params(th)
    assert np.array_equal(n.get_params(rounded=True), P.round_weights(th.astype(np.float32).astype(np.float64)))
    ref_out = P.forward(th.astype(np.float32).astype(np.float64), x.astype(np.float64), periodic)
    out = n.forward(x, periodic=periodic)
    assert rel(out, ref_out) < 1e-5
    L_ref, g_ref, _ = P.loss_and_grad(th.astype(np.float32).astype(np.float64), x.astype(np.float64),
                                      t.astype(np.float64), periodic)
    L, g = n.grad(x, t, periodic)
    assert abs(L - L_ref) <= 1e-5 * L_ref
    assert rel(g, g_ref) < 1e-4
    # per layer too (each layer's weight block and bias block)
    k = 0
    for i, o in P.LAYERS:
        w = slice(k, k + o * i * 9)
        b = slice(k + o * i * 9, k + o * i * 9 + o)
        assert rel(g[w], g_ref[w]) < 1e-4 and rel(g[b], g_ref[b]) < 1e-4
        k += o * i * 9 + o
    n.close()


def test_residual_loss_gradient_vs_oracle():
    from oracle import precond_net as P
    from vsav.net import Net
    rng = np.random.default_rng(6)
    th = _theta(4)
    x = rng.standard_normal((3, 2, 30, 30)).astype(np.float32)
    t = (0.1 * rng.standard_normal((3, 1, 20, 20))).astype(np.float32)
    n = Net(3 * 30 * 30)
    n.set_params(th)
    th32 = th.astype(np.float32).astype(np.float64)
    L_ref, g_ref = P.residual_loss_and_grad(th32, x.astype(np.float64), t.astype(np.float64), 0.02)
    L, g = n.grad(x, t, periodic=False, residual_c0=0.02)
    assert abs(L - L_ref) <= 1e-4 * L_ref
    assert rel(g, g_ref) < 1e-4
    n.close()


def test_fused_tensor_core_inference():
    from oracle import precond_net as P
    from vsav.net import Net
    rng = np.random.default_rng(3)
    th = _theta(2)
    x = rng.standard_normal((3, 2, 64, 96)).astype(np.float32)
    x = x[:, :, :, :64].copy()
    n = Net(3 * 64 * 64)
    n.set_params(th)
    ref = P.forward(th.astype(np.float32).astype(np.float64), x.astype(np.float64), True)
    out32 = n.forward(x, periodic=True, fused=False)
    out_tc = n.forward(x, periodic=True, fused=True)
    assert rel(out32, ref) < 1e-5
    assert rel(out_tc, ref) < 2e-2
    # a second call reuses the packed fragments and gives the same result
    assert np.array_equal(n.forward(x, periodic=True, fused=True), out_tc)
    n.close()


@pytest.mark.parametrize("B,H,W", [(3, 64, 64), (1, 32, 32), (2, 32, 128), (5, 128, 64)])
def test_tcgen05_inference(B, H, W):
    """The fused tcgen05 kernel (implicit GEMM on the fifth-generation tensor
    cores, accumulators in tensor memory) computes the network of the FP64
    oracle with BF16 activations, like the mma.sync kernel: the same error
    bound against the oracle, and close to the mma.sync kernel (the two differ
    only in the FP32 summation order, through BF16 roundings of activations)."""
    from oracle import precond_net as P
    from vsav.net import Net
    rng = np.random.default_rng(11 + B + H)
    th = _theta(5)
    x = rng.standard_normal((B, 2, H, W)).astype(np.float32)
    n = Net(B * H * W)
    n.set_params(th)
    ref = P.forward(th.astype(np.float32).astype(np.float64), x.astype(np.float64), True)
    out_mma = n.forward(x, periodic=True, impl=1)
    out_tc = n.forward(x, periodic=True, impl=2)
    assert rel(out_tc, ref) < 2e-2, rel(out_tc, ref)
    assert rel(out_tc, out_mma) < 2e-2, rel(out_tc, out_mma)
    # every output pixel is written: no tile or M-tile is skipped
    assert np.isfinite(out_tc).all()
    assert np.array_equal(n.forward(x, periodic=True, impl=2), out_tc)
    n.close()


def test_training_reduces_loss():
    """Adam on the GPU kernels fits a teacher network of the same shape."""
    import torch
    from oracle import precond_net as P
    from vsav.net import Net
    rng = np.random.default_rng(4)
    S, nc = 21, 256
    x = rng.standard_normal((nc, 2, S, S))
    t = P.forward(_theta(7), x, False)
    xd = torch.tensor(x, dtype=torch.float32, device="cuda").contiguous()
    td = torch.tensor(t, dtype=torch.float32, device="cuda").contiguous()
    n = Net(64 * S * S)
    n.set_params(P.init_params(0))
    l0 = n.eval(xd.data_ptr(), td.data_ptr(), nc, S, 64)
    losses = n.train(xd.data_ptr(), td.data_ptr(), nc, S, batch=32, nsteps=300, lr=3e-3, seed=1)
    l1 = n.eval(xd.data_ptr(), td.data_ptr(), nc, S, 64)
    # per-crop weights: uniform weights give the unweighted loss
    wd = torch.full((nc,), 2.0, dtype=torch.float32, device="cuda")
    assert abs(n.eval(xd.data_ptr(), td.data_ptr(), nc, S, 64, w_dev=wd.data_ptr()) - l1) <= 1e-6 * l1
    assert np.all(np.isfinite(losses))
    assert l1 < 0.5 * l0, (l0, l1)
    # the reported per-step loss is the batch's normalised loss
    assert losses[-20:].mean() < losses[:20].mean()
    n.close()


def _handle(kw, **opt):
    from vsav import Handle
    return Handle(Cfg(**kw), **opt)


def test_flexible_diag_matches_reference_solve():
    """Flexible right-preconditioned BiCGSTAB (diagonal) gives the reference
    solve's result to the solver tolerance."""
    kw, g = load_golden("single2d_n64")
    out = {}
    for pc in ("diag", "flex_diag"):
        h = _handle(kw, precision="fp64", psi_precond=pc, psi_itmax=60)
        h.init_state(g["phi0"], g["psi0"])
        h.run(1, 2)
        out[pc] = {k: h.get_field(k) for k in ("phi", "psi", "mu", "nu", "u", "p")}
        out[pc + "_it"] = h.psi_stats()[:, 0]
        h.close()
    for k in ("phi", "psi", "mu", "nu", "u", "p"):
        assert rel(out["flex_diag"][k], out["diag"][k]) < 1e-8, k
    assert np.all(out["flex_diag_it"] > 0)


@pytest.mark.parametrize("net_tc", ["1", "0"])
@pytest.mark.parametrize("prec", ["fp32", "mixed"])
def test_learned_preconditioner_solves_to_tolerance(prec, net_tc, monkeypatch):
    """Any network (here an untrained one) only changes the Krylov path: the
    flexible solve still reaches the same solution, with the network on the
    mma.sync kernel (the default) or the tcgen05 kernel (VSAV_NET_TC=1)."""
    monkeypatch.setenv("VSAV_NET_TC", net_tc)
    kw, g = load_golden("multi2d_n64_N2")
    ref = _handle(kw, precision="fp64")
    ref.init_state(g["phi0"], g["psi0"])
    ref.run(1, 2)
    psi_ref = ref.get_field("psi")
    ref.close()
    h = _handle(kw, precision=prec, psi_precond="learned", psi_net=_theta(3), psi_itmax=60,
                psi_rtol=1e-7 if prec == "fp32" else None)
    h.init_state(g["phi0"], g["psi0"])
    h.run(1, 2)
    st = h.psi_stats()
    assert np.all(st[:, 1] == 1), st
    assert rel(h.get_field("psi"), psi_ref) < (1e-5 if prec == "fp32" else 1e-9)
    h.close()


def test_learned_needs_weights_and_fp32():
    from vsav.core import VsavError
    kw, g = load_golden("single2d_n64")
    with pytest.raises(VsavError):
        _handle(kw, precision="fp64", psi_precond="learned")
    h = _handle(kw, precision="fp32", psi_precond="learned")
    h.init_state(g["phi0"], g["psi0"])
    with pytest.raises(VsavError):
        h.run(1, 1)
    h.close()


def test_harvest_pairs():
    kw, g = load_golden("multi2d_n64_N2")
    h = _handle(kw, precision="fp64", psi_itmax=40, psi_rtol=1e-13)
    h.init_state(g["phi0"], g["psi0"])
    h.harvest(8)
    h.run(1, 1)
    xk, rk, xs, M = h.harvest_read()
    K = xk.shape[0]
    assert 2 <= K <= 8 and xk.shape[1:] == (6, 64, 64) and xs.shape == (6, 64, 64) and M.shape == (2, 64, 64)
    assert np.all(xk[0] == 0) and np.linalg.norm(rk[0]) > 0
    e0 = np.linalg.norm(xs - xk[0])
    eK = np.linalg.norm(xs - xk[-1])
    assert eK < 1e-2 * e0
    # M_psi = 0.1 (1 - M0 (phi^2 - 1)^2) lies in [0.1 (1 - M0), 0.1]
    assert M.max() <= 0.1 + 1e-6 and M.min() >= 0.1 * (1 - kw["M0_psi"]) - 1e-6
    # the solution of the solve is the Step-1 psi cache field psi_11 (split 11); that one is the
    # half-spectrum truncation (c2r convention) of the full-spectrum solution, whose real part
    # x* is, so the two agree up to the anti-Hermitian part of the solve
    psi11 = np.fft.irfft2(h.get_cache("psi_11"), s=(64, 64))
    assert rel(xs[:2], psi11) < 5e-2
    h.harvest(0)
    h.close()


def _gain_case(prec, pc, rtol, itmax, nsteps=1):
    """multi2d at 256^2, eps 0.08 (the interface spans as many grid points as
    in the 512^2, eps 0.04 training runs), 4 vesicles, a seed the training
    harvest did not use.  Returns per-step psi stats and fields."""
    import os
    from vsav import ics
    kw, phi, psi, _ = ics.workload("multi2d_512x4", seed=7, n_override=256, eps_override=0.08)
    kw["dt"] = 1e-6
    wpath = os.path.join(os.path.dirname(__import__("vsav").__file__), "precond_weights.npz")
    h = _handle(kw, precision=prec, psi_precond=pc, psi_itmax=itmax, psi_rtol=rtol,
                psi_net=wpath if pc == "learned" else None)
    h.init_state(phi, psi)
    stats = []
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")          # itmax-limited solves warn by design
        for n in range(1, nsteps + 1):
            h.run(n, 1)
            stats.append(h.psi_stats().copy())
    out = {k: h.get_field(k) for k in ("phi", "psi", "u")}
    h.close()
    return np.array(stats), out


def test_learned_preconditioner_gain():
    """What the trained network gains over the same flexible BiCGSTAB with the
    diagonal alone: after one and after two iterations (same right-hand sides,
    same stopping scale) the residual it leaves is smaller, on a configuration
    the training did not see.  Both solves then reach the same solution."""
    for k in (1, 2):
        st_d, _ = _gain_case("fp32", "flex_diag", 1e-12, k)
        st_l, _ = _gain_case("fp32", "learned", 1e-12, k)
        # systems 0 and 1 (splits 11 and 12); split 21 has a zero right-hand side at step 1 (u = 0)
        rd, rl = st_d[0, :2, 3], st_l[0, :2, 3]
        assert np.all(rl < 0.9 * rd), (k, rl, rd)
    st_d, out_d = _gain_case("fp32", "flex_diag", 1e-6, 60, nsteps=2)
    st_l, out_l = _gain_case("fp32", "learned", 1e-6, 60, nsteps=2)
    assert np.all(st_d[:, :, 1] == 1) and np.all(st_l[:, :, 1] == 1)
    _, ref = _gain_case("fp64", "diag", 1e-12, 20, nsteps=2)
    for key in ("phi", "psi"):
        assert rel(out_l[key], ref[key]) < 1e-5, key
        assert rel(out_d[key], ref[key]) < 1e-5, key
