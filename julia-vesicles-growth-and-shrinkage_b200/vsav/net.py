"""The learned psi-preconditioner network on the GPU (vsav_net_* of the C ABI):
parameters, forward, gradient and Adam training on crop sets.

Five 3x3 convolutions, 2 -> 16 -> 16 -> 16 -> 16 -> 1 channels, ReLU after
the first four; BF16-rounded convolution weights, FP32 biases, FP32
accumulation.  Inputs [B][2][H][W] float32: channel 0 the diagonally
preconditioned psi residual in physical space divided by its RMS, channel 1
(M_psi - 0.075) / 0.025.  Output [B][1][H'][W']: the correction, in units of
that RMS, that takes the diagonal preconditioner's result towards the error.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np

from . import _lib as L

LAYERS = ((2, 16), (16, 16), (16, 16), (16, 16), (16, 1))


def n_params() -> int:
    return sum(o * i * 9 + o for i, o in LAYERS)


def init_params(seed: int = 0) -> np.ndarray:
    """He-style initialisation with the last layer scaled by 0.1, zero biases."""
    rng = np.random.default_rng(seed)
    th = np.zeros(n_params())
    k = 0
    for li, (i, o) in enumerate(LAYERS):
        std = np.sqrt(2.0 / (9 * i)) * (0.1 if li == len(LAYERS) - 1 else 1.0)
        th[k:k + o * i * 9] = rng.normal(0, std, o * i * 9)
        k += o * i * 9 + o
    return th


def _fptr(a):
    if isinstance(a, int):
        return ct.c_void_p(a)
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ct.c_void_p)


class Net:
    def __init__(self, cap_pixels: int, device: int = 0):
        self.lib = L.load()
        h = ct.c_void_p()
        rc = self.lib.vsav_net_create(int(cap_pixels), int(device), ct.byref(h))
        if rc != 0:
            raise RuntimeError(f"vsav_net_create failed ({rc}): {self.lib.vsav_net_last_error(None).decode()}")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.vsav_net_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, rc):
        if rc != 0:
            raise RuntimeError(f"libvsav net error {rc}: {self.lib.vsav_net_last_error(self.h).decode()}")

    def set_params(self, theta):
        th = np.ascontiguousarray(theta, dtype=np.float64)
        assert th.size == n_params()
        self._chk(self.lib.vsav_net_set_params(self.h, L.dptr(th)))

    def get_params(self, rounded: bool = False) -> np.ndarray:
        th = np.empty(n_params())
        self._chk(self.lib.vsav_net_get_params(self.h, L.dptr(th), int(rounded)))
        return th

    def forward(self, x: np.ndarray, periodic: bool = True, fused: bool = False, impl: int = None) -> np.ndarray:
        """Network output; impl 0: FP32 per-layer kernels, 1 (fused=True): the
        fused mma.sync kernel, 2: the fused tcgen05 kernel."""
        impl = (1 if fused else 0) if impl is None else int(impl)
        x = np.ascontiguousarray(x, dtype=np.float32)
        B, C, H, W = x.shape
        assert C == 2
        Ho, Wo = (H, W) if periodic else (H - 10, W - 10)
        out = np.empty((B, 1, Ho, Wo), np.float32)
        self._chk(self.lib.vsav_net_forward(self.h, _fptr(x), B, H, W, int(periodic), impl, _fptr(out)))
        return out

    def grad(self, x: np.ndarray, t: np.ndarray, periodic: bool, residual_c0=None):
        """(1/2 sum (out - t)^2, its gradient w.r.t. theta); with residual_c0
        the normalised residual-norm loss of train() instead."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        B, _, H, W = x.shape
        loss = ct.c_double()
        g = np.empty(n_params())
        kind, c0 = (0, 0.0) if residual_c0 is None else (1, float(residual_c0))
        self._chk(self.lib.vsav_net_grad(self.h, _fptr(x), _fptr(t), B, H, W, int(periodic), kind, c0, ct.byref(loss),
                                         L.dptr(g)))
        return loss.value, g

    def train(self, x_dev: int, t_dev: int, ncrops: int, S: int, batch: int, nsteps: int, lr: float,
              seed: int = 0, w_dev: int = 0, flip: bool = False, residual_c0=None) -> np.ndarray:
        """nsteps Adam steps on device crop sets (addresses of float32
        [ncrops][2][S][S] and [ncrops][1][S-10][S-10], optional per-crop loss
        weights [ncrops]); per-step weighted normalised loss.  residual_c0:
        use the residual-norm loss with operator constant c0 (grid units)."""
        losses = np.empty(max(nsteps, 1))
        kind, c0 = (0, 0.0) if residual_c0 is None else (1, float(residual_c0))
        self._chk(self.lib.vsav_net_train(self.h, ct.c_void_p(x_dev), ct.c_void_p(t_dev), ct.c_void_p(w_dev or None),
                                          int(ncrops), int(S), int(batch), int(nsteps), float(lr), int(seed), int(flip),
                                          kind, c0, L.dptr(losses)))
        return losses[:nsteps]

    def eval(self, x_dev: int, t_dev: int, ncrops: int, S: int, batch: int, w_dev: int = 0, residual_c0=None) -> float:
        loss = ct.c_double()
        kind, c0 = (0, 0.0) if residual_c0 is None else (1, float(residual_c0))
        self._chk(self.lib.vsav_net_eval(self.h, ct.c_void_p(x_dev), ct.c_void_p(t_dev), ct.c_void_p(w_dev or None),
                                         int(ncrops), int(S), int(batch), kind, c0, ct.byref(loss)))
        return loss.value
