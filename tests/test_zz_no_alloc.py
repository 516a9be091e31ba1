"""The allocation-free inverse FFT entry point (vsav_irfft2d_f32_noalloc).

It serves callers that cannot allocate GPU memory themselves, e.g. code
running inside an application whose device memory belongs to an arena or
pool, or code that must not call the allocator.  Its output must match the
handle path's irfft (vsav_transform) to FP32 round-off, on repeated calls
(the shared scratch array keeps the previous call's contents).  This file is
collected last on purpose."""
import ctypes as ct
import math

import numpy as np
import pytest

from helpers import Cfg

pytestmark = pytest.mark.gpu

TOL = 6e-7      # the FP32 transform tolerance of the parity tests


def _handle_irfft(Nx, Ny, H, mult):
    from test_gpu_parity import kat_cfg
    from vsav import Handle
    h = Handle(Cfg(**kat_cfg(Nx, Ny)), precision="fp32")
    out = h.irfft(H, mult)
    h.close()
    return out


def test_noalloc_irfft_matches_handle_path():
    import torch
    from vsav import _lib
    lib = _lib.load()
    Nx, Ny, nf = 256, 128, 3
    rng = np.random.default_rng(11)
    H = rng.standard_normal((nf, Ny, Nx // 2 + 1)) + 1j * rng.standard_normal((nf, Ny, Nx // 2 + 1))
    spec = torch.from_numpy(np.ascontiguousarray(H.astype(np.complex64)).view(np.float32)).cuda()
    out = torch.empty((nf, Ny, Nx), dtype=torch.float32, device="cuda")
    L = 2 * math.pi
    for mult, name in ((1, "dx"), (4, "lap")):           # two calls in a row, then compare both
        ref = _handle_irfft(Nx, Ny, H, name)
        for _ in range(2):
            out.fill_(float("nan"))
            rc = lib.vsav_irfft2d_f32_noalloc(spec.data_ptr(), out.data_ptr(), nf, Nx, Ny, L, L, mult, None)
            assert rc == 0, lib.vsav_noalloc_error().decode()
            torch.cuda.synchronize()
            got = out.cpu().numpy().astype(np.float64)
            err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
            assert err < TOL, (name, err)


def test_noalloc_rejects_oversized_batch():
    import torch
    from vsav import _lib
    lib = _lib.load()
    Nx = Ny = 1024
    nf = 2                       # 2 * 1024 * 513 complex > 1 Mi: beyond the fixed scratch
    spec = torch.zeros((1, 2), dtype=torch.float32, device="cuda")
    out = torch.zeros((1,), dtype=torch.float32, device="cuda")
    rc = lib.vsav_irfft2d_f32_noalloc(spec.data_ptr(), out.data_ptr(), nf, Nx, Ny, 1.0, 1.0, 0, None)
    assert rc == -1
    assert "exceeds the fixed scratch" in lib.vsav_noalloc_error().decode()
