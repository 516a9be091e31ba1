"""CPU checks of the NumPy reference of the learned psi-preconditioner network
(oracle/precond_net.py): finite-difference gradients, BF16 rounding, shapes.
The GPU kernels are checked against this reference in test_net_gpu.py."""
import numpy as np
import pytest

from oracle import precond_net as P


def _loss_exact(theta, x, t, periodic):
    """1/2 sum (out - t)^2 with theta used as is (no rounding)."""
    a = x
    for li, (W, b) in enumerate(P.unpack(theta)):
        z = P.conv(a, W, b, periodic)
        a = np.maximum(z, 0.0) if li < len(P.LAYERS) - 1 else z
    return 0.5 * float(np.sum((a - t) ** 2))


def test_param_count_matches_library_layout():
    assert P.n_params() == 7409
    from vsav import net
    assert net.n_params() == P.n_params()


def test_bf16_rounding_nearest_even():
    # 1 + 2^-8 is halfway between 1 and 1 + 2^-7: ties to even -> 1
    assert P.to_bf16(np.array([1.0 + 2 ** -8]))[0] == 1.0
    assert P.to_bf16(np.array([1.0 + 3 * 2 ** -8]))[0] == 1.0 + 2 ** -6
    assert P.to_bf16(np.array([-3.0]))[0] == -3.0
    x = np.random.default_rng(0).standard_normal(1000)
    r = P.to_bf16(x)
    assert np.all(np.abs(r - x) <= np.abs(x) * 2 ** -8 * 1.0001)
    assert np.array_equal(P.to_bf16(r), r)


@pytest.mark.parametrize("periodic,shape,oshape", [(True, (2, 2, 9, 10), (2, 1, 9, 10)),
                                                   (False, (2, 2, 14, 15), (2, 1, 4, 5))])
def test_gradient_finite_differences(periodic, shape, oshape):
    rng = np.random.default_rng(1)
    th = P.round_weights(P.init_params(0) + 0.01 * rng.standard_normal(P.n_params()))
    x = rng.standard_normal(shape)
    t = rng.standard_normal(oshape)
    L, g, gx = P.loss_and_grad(th, x, t, periodic)
    assert abs(L - _loss_exact(th, x, t, periodic)) <= 1e-12 * abs(L)
    h = 1e-6
    for k in rng.choice(P.n_params(), 40, replace=False):
        tp, tm = th.copy(), th.copy()
        tp[k] += h
        tm[k] -= h
        fd = (_loss_exact(tp, x, t, periodic) - _loss_exact(tm, x, t, periodic)) / (2 * h)
        assert abs(fd - g[k]) <= 1e-5 * max(1.0, abs(g[k])), (k, fd, g[k])
    k = (1, 0, 3, 4)
    xp, xm = x.copy(), x.copy()
    xp[k] += h
    xm[k] -= h
    fd = (_loss_exact(th, xp, t, periodic) - _loss_exact(th, xm, t, periodic)) / (2 * h)
    assert abs(fd - gx[k]) <= 1e-5 * max(1.0, abs(gx[k]))


def test_adam_step():
    th = np.array([1.0, -2.0])
    m = np.zeros(2)
    v = np.zeros(2)
    g = np.array([0.5, -0.25])
    th2, m2, v2 = P.adam(th, m, v, g, 1, 0.1)
    # first step of Adam moves every parameter by lr against the gradient sign
    assert np.allclose(th2, th - 0.1 * np.sign(g), atol=1e-6)


def test_residual_loss_gradient():
    """residual_op_adjoint is the transpose of residual_op, and the residual
    loss gradient matches finite differences."""
    rng = np.random.default_rng(5)
    u = rng.standard_normal((2, 7, 9))
    R = rng.standard_normal((2, 7, 9))
    R[:, 0, :] = R[:, -1, :] = R[:, :, 0] = R[:, :, -1] = 0
    m = 0.05 + 0.05 * rng.random((2, 7, 9))
    assert abs(np.sum(R * P.residual_op(u, m, 0.3)) - np.sum(P.residual_op_adjoint(R, m, 0.3) * u)) < 1e-12
    th = P.round_weights(P.init_params(1) + 0.01 * rng.standard_normal(P.n_params()))
    x = rng.standard_normal((2, 2, 16, 17))
    t = rng.standard_normal((2, 1, 6, 7))
    w = np.array([1.0, 3.0])
    L, g = P.residual_loss_and_grad(th, x, t, 0.01, w)

    def Lf(tt):
        a = x
        for li, (W, b) in enumerate(P.unpack(tt)):
            z = P.conv(a, W, b, False)
            a = np.maximum(z, 0.0) if li < 4 else z
        m2 = 0.075 + 0.025 * x[:, 1, 5:-5, 5:-5]
        Rr = P.residual_op(a[:, 0] - t[:, 0], m2, 0.01)
        Lt = P.residual_op(t[:, 0], m2, 0.01)
        return np.sum(w[:, None, None] * Rr ** 2) / np.sum(w[:, None, None] * Lt ** 2)
    assert abs(Lf(th) - L) < 1e-12 * L
    for k in rng.choice(P.n_params(), 20, replace=False):
        tp, tm = th.copy(), th.copy()
        tp[k] += 1e-6
        tm[k] -= 1e-6
        fd = (Lf(tp) - Lf(tm)) / 2e-6
        assert abs(fd - g[k]) <= 1e-5 * max(1.0, abs(g[k])), (k, fd, g[k])
