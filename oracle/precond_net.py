"""FP64 NumPy reference of the learned psi preconditioner network.

TEST INFRASTRUCTURE ONLY: the GPU training and inference kernels of the
library are checked against these functions; nothing in the library calls
them.

The reference solves the Step-1 psi systems with a diagonal spectral
preconditioner only (src/Solvers.jl:53-75); the learned correction added on
top of it has no counterpart there.  Network: five 3x3 convolutions,
2 -> 16 -> 16 -> 16 -> 16 -> 1 channels, ReLU after the first four, no
activation after the last.  Input channels: the diagonally preconditioned
residual in physical space (normalised by its RMS) and the psi mobility
M_psi = 0.1 (1 - M0 (phi^2 - 1)^2) (Utils.jl:20) mapped to [-1, 1].
Convolution weights are used BF16-rounded (round to nearest even), biases in
full precision; gradients are taken with respect to the rounded weights.

Parameter vector layout, layer by layer: W[o][i][ky][kx] then bias[o].
Convolutions are cross-correlations, out[o][y][x] = b[o] +
sum_i,ky,kx W[o][i][ky][kx] in[i][y + ky - 1][x + kx - 1], either periodic
(indices wrap, output size = input size) or valid (no padding, output is 2
smaller in each dimension; in[i][y + ky][x + kx]).
"""
from __future__ import annotations

import numpy as np

LAYERS = ((2, 16), (16, 16), (16, 16), (16, 16), (16, 1))


def n_params() -> int:
    return sum(o * i * 9 + o for i, o in LAYERS)


def unpack(theta):
    """List of (W [O][I][3][3], b [O]) views into theta."""
    out = []
    k = 0
    for i, o in LAYERS:
        W = theta[k:k + o * i * 9].reshape(o, i, 3, 3)
        k += o * i * 9
        b = theta[k:k + o]
        k += o
        out.append((W, b))
    return out


def to_bf16(x):
    """Round to BF16 (nearest even) through FP32; returned as float64."""
    x32 = np.ascontiguousarray(x, dtype=np.float32)
    u = x32.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def round_weights(theta):
    """theta with the convolution weights BF16-rounded (biases kept)."""
    t = np.array(theta, dtype=np.float64)
    k = 0
    for i, o in LAYERS:
        t[k:k + o * i * 9] = to_bf16(t[k:k + o * i * 9])
        k += o * i * 9 + o
    return t


def init_params(seed=0):
    """He-style initialisation, last layer scaled down."""
    rng = np.random.default_rng(seed)
    th = np.zeros(n_params())
    k = 0
    for li, (i, o) in enumerate(LAYERS):
        std = np.sqrt(2.0 / (9 * i)) * (0.1 if li == len(LAYERS) - 1 else 1.0)
        th[k:k + o * i * 9] = rng.normal(0, std, o * i * 9)
        k += o * i * 9 + o
    return th


def conv(x, W, b, periodic):
    """x [B][I][H][W] -> [B][O][H'][W']."""
    B, I, H, Wd = x.shape
    O = W.shape[0]
    if periodic:
        out = np.broadcast_to(b[None, :, None, None], (B, O, H, Wd)).copy()
        for ky in range(3):
            for kx in range(3):
                xs = np.roll(x, shift=(1 - ky, 1 - kx), axis=(2, 3))   # xs[y] = x[y + ky - 1]
                out += np.einsum("oi,bihw->bohw", W[:, :, ky, kx], xs, optimize=True)
        return out
    Ho, Wo = H - 2, Wd - 2
    out = np.broadcast_to(b[None, :, None, None], (B, O, Ho, Wo)).copy()
    for ky in range(3):
        for kx in range(3):
            out += np.einsum("oi,bihw->bohw", W[:, :, ky, kx], x[:, :, ky:ky + Ho, kx:kx + Wo], optimize=True)
    return out


def conv_backward(x, W, g, periodic):
    """Gradients of sum(g * conv(x, W, b)) w.r.t. W, b and x."""
    B, I, H, Wd = x.shape
    dW = np.zeros_like(W)
    db = g.sum(axis=(0, 2, 3))
    dx = np.zeros_like(x)
    if periodic:
        for ky in range(3):
            for kx in range(3):
                xs = np.roll(x, shift=(1 - ky, 1 - kx), axis=(2, 3))
                dW[:, :, ky, kx] = np.einsum("bohw,bihw->oi", g, xs, optimize=True)
                gi = np.einsum("oi,bohw->bihw", W[:, :, ky, kx], g, optimize=True)
                dx += np.roll(gi, shift=(ky - 1, kx - 1), axis=(2, 3))
        return dW, db, dx
    Ho, Wo = H - 2, Wd - 2
    for ky in range(3):
        for kx in range(3):
            dW[:, :, ky, kx] = np.einsum("bohw,bihw->oi", g, x[:, :, ky:ky + Ho, kx:kx + Wo], optimize=True)
            dx[:, :, ky:ky + Ho, kx:kx + Wo] += np.einsum("oi,bohw->bihw", W[:, :, ky, kx], g, optimize=True)
    return dW, db, dx


def forward(theta, x, periodic, keep=False):
    """Network output [B][1][H'][W'] (and the pre-activations when keep)."""
    layers = unpack(round_weights(theta))
    acts = [x]
    a = x
    for li, (W, b) in enumerate(layers):
        z = conv(a, W, b, periodic)
        a = np.maximum(z, 0.0) if li < len(layers) - 1 else z
        acts.append(a)
    return (a, acts) if keep else a


def backward(theta, acts, g, periodic):
    """Gradients (dtheta, dx) of sum(g * out) given the activations of forward."""
    layers = unpack(round_weights(theta))
    grad = np.zeros(n_params())
    gviews = unpack(grad)
    for li in range(len(layers) - 1, -1, -1):
        W, _ = layers[li]
        dW, db, dx = conv_backward(acts[li], W, g, periodic)
        gviews[li][0][...] = dW
        gviews[li][1][...] = db
        g = dx * (acts[li] > 0) if li > 0 else dx
    return grad, g


def residual_op(u, m, c0):
    """L u = c0 u - div_h(M grad_h u) in grid units at the interior points of
    u [B][H][W] (5-point conservative stencil, face M = mean of the two
    cells; zero on the border)."""
    R = np.zeros_like(u)
    c = (slice(None), slice(1, -1), slice(1, -1))
    uc, mc = u[c], m[c]
    me = 0.5 * (mc + m[:, 1:-1, 2:]); mw = 0.5 * (mc + m[:, 1:-1, :-2])
    mn = 0.5 * (mc + m[:, 2:, 1:-1]); ms = 0.5 * (mc + m[:, :-2, 1:-1])
    R[c] = c0 * uc - (me * (u[:, 1:-1, 2:] - uc) - mw * (uc - u[:, 1:-1, :-2])
                      + mn * (u[:, 2:, 1:-1] - uc) - ms * (uc - u[:, :-2, 1:-1]))
    return R


def residual_op_adjoint(R, m, c0):
    """L^T R for residual_op (R zero on the border)."""
    B, H, W = R.shape
    g = c0 * R.copy()
    for dy, dx in ((0, 1), (0, -1), (1, 0), (-1, 0)):
        # face between x and x + (dy, dx): contributes m_f (R_x - R_{x+d}) to g_x for x, x+d in range
        ys = slice(max(0, -dy), H - max(0, dy)); xs = slice(max(0, -dx), W - max(0, dx))
        yn = slice(max(0, dy), H - max(0, -dy)); xn = slice(max(0, dx), W - max(0, -dx))
        mf = 0.5 * (m[:, ys, xs] + m[:, yn, xn])
        g[:, ys, xs] += mf * (R[:, ys, xs] - R[:, yn, xn])
    return g


def residual_loss_and_grad(theta, x, t, c0, w=None):
    """Residual-norm loss of valid crops: sum w |L(out - t)|^2 / sum w |L t|^2,
    M = 0.075 + 0.025 * input channel 1 at the output points; (L, dL/dtheta)."""
    out, acts = forward(theta, x, False, keep=True)
    m = 0.075 + 0.025 * x[:, 1, 5:-5, 5:-5]
    w = np.ones(x.shape[0]) if w is None else np.asarray(w, float)
    R = residual_op(out[:, 0] - t[:, 0], m, c0)
    Lt = residual_op(t[:, 0], m, c0)
    den = float(np.sum(w[:, None, None] * Lt * Lt))
    L = float(np.sum(w[:, None, None] * R * R)) / den
    gout = (2.0 / den) * w[:, None, None] * residual_op_adjoint(R, m, c0)
    grad, _ = backward(theta, acts, gout[:, None], False)
    return L, grad


def loss_and_grad(theta, x, t, periodic):
    """L = 1/2 sum (out - t)^2; returns (L, dL/dtheta, dL/dx)."""
    layers = unpack(round_weights(theta))
    out, acts = forward(theta, x, periodic, keep=True)
    g = out - t
    L = 0.5 * float(np.sum(g * g))
    grad = np.zeros(n_params())
    gviews = unpack(grad)
    for li in range(len(layers) - 1, -1, -1):
        W, _ = layers[li]
        dW, db, dx = conv_backward(acts[li], W, g, periodic)
        gviews[li][0][...] = dW
        gviews[li][1][...] = db
        g = dx * (acts[li] > 0) if li > 0 else dx
    return L, grad, g


def normalised_loss(theta, x, t, periodic):
    """sum (out - t)^2 / sum t^2 (the training loss) and its theta gradient."""
    L, grad, _ = loss_and_grad(theta, x, t, periodic)
    s = float(np.sum(t * t))
    return 2.0 * L / s, 2.0 * grad / s


def adam(theta, m, v, grad, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update (in place on copies); step counts from 1."""
    m = b1 * m + (1 - b1) * grad
    v = b2 * v + (1 - b2) * grad * grad
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return theta - lr * mh / (np.sqrt(vh) + eps), m, v
