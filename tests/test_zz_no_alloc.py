"""The allocation-free inverse FFT entry point (vsav_irfft2d_f32_noalloc).

It serves callers that cannot allocate GPU memory themselves, e.g. code
running inside an application whose device memory belongs to an arena or
pool, or code that must not call the allocator.  Its output must match
NumPy's irfft2 of the multiplied half spectrum (FP64) to FP32 round-off and
the handle path's irfft, on two calls in a row (the shared scratch array
keeps the previous call's contents).  Shapes cover the smallest accepted
transform (Nx=32, Ny=8; the handle path's FP32 transforms start at Ny=16, so
Ny=8 is compared with NumPy alone), the longest columns (Ny=2048) and the
longest rows (Nx=2048), and every multiplier the entry point accepts.  This file is
collected last on purpose."""
import math

import numpy as np
import pytest

from helpers import Cfg

pytestmark = pytest.mark.gpu

TOL = 6e-7      # the FP32 transform tolerance of the parity tests
MULTS = {0: None, 1: "dx", 2: "dy", 4: "lap", 5: "bih"}


def _numpy_irfft(H, mult, Lx, Ly):
    """irfft2 of mult * H in FP64 with the reference's wavenumbers: rfftfreq
    along x (Nyquist +pi Nx/Lx) and fftfreq along y (Nyquist negative),
    src/SpectralUtils.jl:42-47."""
    nf, Ny, nkx = H.shape
    Nx = 2 * (nkx - 1)
    kx = np.fft.rfftfreq(Nx, d=1.0 / Nx) * (2 * math.pi / Lx)
    ky = np.fft.fftfreq(Ny, d=1.0 / Ny) * (2 * math.pi / Ly)
    KX, KY = np.meshgrid(kx, ky)
    k2 = KX ** 2 + KY ** 2
    m = {0: np.ones_like(KX), 1: 1j * KX, 2: 1j * KY, 4: -k2, 5: k2 ** 2}[mult]
    return np.fft.irfft2(H * m[None], s=(Ny, Nx), axes=(1, 2))


def _handle_irfft(Nx, Ny, H, mult):
    """The handle path's FP32 irfft (its FP32 handles need Ny >= 16)."""
    from test_gpu_parity import kat_cfg
    from vsav import Handle
    h = Handle(Cfg(**kat_cfg(Nx, Ny)), precision="fp32")
    try:
        return h.irfft(H, MULTS[mult])
    finally:
        h.close()


@pytest.mark.parametrize("Nx,Ny,nf", [(32, 8, 2), (32, 16, 2), (256, 128, 3), (32, 2048, 2), (2048, 8, 3),
                                      (2048, 16, 3)])
@pytest.mark.parametrize("mult", [0, 1, 2, 4, 5])
def test_noalloc_irfft_matches_numpy(Nx, Ny, nf, mult):
    import torch
    from vsav import _lib
    lib = _lib.load()
    rng = np.random.default_rng(11 + Nx + Ny + mult)
    H = rng.standard_normal((nf, Ny, Nx // 2 + 1)) + 1j * rng.standard_normal((nf, Ny, Nx // 2 + 1))
    H = H.astype(np.complex64)
    spec = torch.from_numpy(np.ascontiguousarray(H).view(np.float32)).cuda()
    out = torch.empty((nf, Ny, Nx), dtype=torch.float32, device="cuda")
    L = 2 * math.pi
    ref = _numpy_irfft(H.astype(np.complex128), mult, L, L)
    handle = _handle_irfft(Nx, Ny, H.astype(np.complex128), mult) if Ny >= 16 else None
    if handle is not None:
        assert np.linalg.norm(handle - ref) / np.linalg.norm(ref) < TOL
    for call in range(2):                    # two calls in a row through the shared scratch
        out.fill_(float("nan"))
        rc = lib.vsav_irfft2d_f32_noalloc(spec.data_ptr(), out.data_ptr(), nf, Nx, Ny, L, L, mult, None)
        assert rc == 0, lib.vsav_noalloc_error().decode()
        assert lib.vsav_noalloc_error().decode() == ""
        torch.cuda.synchronize()
        got = out.cpu().numpy().astype(np.float64)
        err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
        assert err < TOL, (call, err)
        if handle is not None:
            err_h = np.linalg.norm(got - handle) / np.linalg.norm(handle)
            assert err_h < TOL, (call, err_h)


def test_noalloc_rejects_oversized_batch_and_clears_its_error():
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
    # a following good call clears the message
    spec = torch.zeros((1, 8, 17, 2), dtype=torch.float32, device="cuda")
    out = torch.zeros((1, 8, 32), dtype=torch.float32, device="cuda")
    rc = lib.vsav_irfft2d_f32_noalloc(spec.data_ptr(), out.data_ptr(), 1, 32, 8, 1.0, 1.0, 0, None)
    assert rc == 0 and lib.vsav_noalloc_error().decode() == ""
    torch.cuda.synchronize()
