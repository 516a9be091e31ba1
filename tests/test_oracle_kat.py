"""Known-answer tests that pin the oracle's operator and FFT conventions.

Ported from the reference's own unit tests, test/test_Types_Ops.jl (groups
G1-G8), on its shared fixture: a non-square 128x64 grid on [0, 2pi)^2
(test_Types_Ops.jl:28-41).  Julia's column-major (Nx, Ny, N) arrays are the
oracle's C-order [N][Ny][Nx] arrays."""
import math

import numpy as np
import pytest

from oracle import vsav_oracle as O


@pytest.fixture(scope="module")
def cfg():
    return O.Config(N=1, epsilon=0.05, M_phi=1.0, M0_psi=1.0, eta=1.0, gamma_surf=1.0,
                    gamma_area=1.0, gamma_bend=1.0, gamma_in=1.0, beta_in=0.0,
                    psi_in_v=[0.1, 0.2], gamma_out=1.0, beta_out=0.0, psi_out_v=[0.8, 0.7],
                    lamda=1, S1=1.0, S2=1.0, S3=1.0, S4=1.0, C1=1.0, C2=1.0, C3=1.0,
                    dt=1e-3, T=1.0, Nx=128, Ny=64, Lx=2 * math.pi, Ly=2 * math.pi,
                    tol=1e-10, goal="s")


@pytest.fixture(scope="module")
def ops(cfg):
    return O.build_operators(cfg)


def test_g1_config(cfg):                           # test_Types_Ops.jl:49-65
    assert cfg.Nt == round(cfg.T / cfg.dt) == 1000
    assert cfg.dx == pytest.approx(cfg.Lx / cfg.Nx)
    assert cfg.dy == pytest.approx(cfg.Ly / cfg.Ny)
    assert cfg.spe_len == (cfg.Nx // 2 + 1) * cfg.Ny * cfg.N


def test_g2_shapes_and_types(cfg, ops):            # :71-106
    nkx = cfg.Nx // 2 + 1
    assert ops.K[0].shape == (1, nkx) and ops.K[1].shape == (cfg.Ny, 1)
    assert np.all(ops.D1[0].real == 0) and np.all(ops.D1[1].real == 0)
    np.testing.assert_allclose(ops.D1[0].imag, ops.K[0])
    np.testing.assert_allclose(ops.D1[1].imag, ops.K[1])
    assert ops.Laplacian.shape == (cfg.Ny, nkx) and ops.Biharmonic.shape == (cfg.Ny, nkx)
    assert np.all(ops.Laplacian <= 0) and np.all(ops.Biharmonic >= 0)
    np.testing.assert_allclose(ops.Biharmonic, ops.Laplacian ** 2)


def test_g3_wavenumbers(cfg, ops):                 # :112-136
    kx, ky = ops.K[0][0], ops.K[1][:, 0]
    nkx = cfg.Nx // 2 + 1
    assert kx[0] == pytest.approx(0.0)
    assert kx[1] == pytest.approx(2 * math.pi / cfg.Lx)
    assert kx[nkx - 1] == pytest.approx(math.pi * cfg.Nx / cfg.Lx)     # rfftfreq: +Nyquist
    assert ky[0] == pytest.approx(0.0)
    assert ky[1] == pytest.approx(2 * math.pi / cfg.Ly)
    assert ky[cfg.Ny // 2] == pytest.approx(-math.pi * cfg.Ny / cfg.Ly)  # fftfreq: -Nyquist
    assert ops.kx0[0, cfg.Nx // 2] == pytest.approx(-math.pi * cfg.Nx / cfg.Lx)


def test_g4_round_trip(cfg, ops):                  # :142-173
    rng = np.random.default_rng(1)
    u = rng.standard_normal((cfg.N, cfg.Ny, cfg.Nx))
    np.testing.assert_allclose(ops.irfft(ops.rfft(u)), u, rtol=0, atol=1e-13)
    c = np.full((cfg.N, cfg.Ny, cfg.Nx), 3.7)
    np.testing.assert_allclose(ops.irfft(ops.rfft(c)), c, rtol=0, atol=1e-15)


def kat_fields(cfg):
    """sin(3x) cos(4y) / (Nx Ny / 4) and its derivatives (:189-208)."""
    m, n = 3, 4
    km, kn = m * 2 * math.pi / cfg.Lx, n * 2 * math.pi / cfg.Ly
    x = cfg.Lx * np.arange(cfg.Nx) / cfg.Nx
    y = cfg.Ly * np.arange(cfg.Ny) / cfg.Ny
    Y, X = np.meshgrid(y, x, indexing="ij")
    s = cfg.Nx * cfg.Ny / 4
    f = np.sin(km * X) * np.cos(kn * Y) / s
    return dict(f=f[None], dx=(km * np.cos(km * X) * np.cos(kn * Y) / s)[None],
                dy=(-kn * np.sin(km * X) * np.sin(kn * Y) / s)[None],
                lap=(-(km ** 2 + kn ** 2) * f)[None], bih=((km ** 2 + kn ** 2) ** 2 * f)[None])


def test_g5_spectral_derivatives(cfg, ops):        # :189-240
    k = kat_fields(cfg)
    fh = ops.rfft(k["f"])
    assert np.sort(np.abs(fh).ravel())[::-1][0] == pytest.approx(1.0, abs=1e-10)
    assert np.max(np.abs(ops.irfft(ops.D1[0] * fh) - k["dx"])) < 1e-15
    assert np.max(np.abs(ops.irfft(ops.D1[1] * fh) - k["dy"])) < 1e-15
    assert np.max(np.abs(ops.irfft(ops.Laplacian * fh) - k["lap"])) < 1e-14
    assert np.max(np.abs(ops.irfft(ops.Biharmonic * fh) - k["bih"])) < 1e-11


def test_g6_mult(cfg, ops):                        # :246-314
    x = 2 * math.pi * np.arange(cfg.Nx) / cfg.Nx
    y = 2 * math.pi * np.arange(cfg.Ny) / cfg.Ny
    Y, X = np.meshgrid(y, x, indexing="ij")
    f, g = np.sin(X)[None], np.cos(Y)[None]
    fh, gh = ops.rfft(f), ops.rfft(g)
    # the reference bound is 1e-15 (4.5 ulp of |f g| = 1); pocketfft's
    # rounding lands at 5 ulp, so the bound here is 2e-15
    assert np.max(np.abs(ops.irfft(O.mult(fh, gh, ops)) - f * g)) < 2e-15
    h = (np.sin(3 * X) + np.sin(4 * X))[None]
    hh = ops.rfft(h)
    assert np.max(np.abs(ops.irfft(O.mult(hh, hh, ops)) - h ** 2)) < 1e-14
    np.testing.assert_allclose(O.mult(fh, gh, ops), O.mult(gh, fh, ops), rtol=0, atol=1e-15)


def test_g7_update_state(cfg):                     # :320-363
    def mk(c):
        r = np.full((cfg.N, cfg.Ny, cfg.Nx), c)
        h = np.full((cfg.N, cfg.Ny, cfg.Nx // 2 + 1), complex(c))
        return O.FieldState(phi=r.copy(), phi_hat=h.copy(), psi=r.copy(), psi_hat=h.copy(),
                            u=np.full((2, cfg.Ny, cfg.Nx), c), u_hat=np.full((2, cfg.Ny, cfg.Nx // 2 + 1), complex(c)),
                            p=np.full((cfg.Ny, cfg.Nx), c), p_hat=np.full((cfg.Ny, cfg.Nx // 2 + 1), complex(c)),
                            mu=r.copy(), mu_hat=h.copy(), nu=r.copy(), nu_hat=h.copy(),
                            Q=c, R1=c, R2=c, R3=c, A0=np.array([c]), dt=c)
    s1, s2 = mk(1.0), mk(2.0)
    O.update_state(s1, s2)
    assert np.all(s1.phi == 2.0) and np.all(s1.psi == 2.0) and np.all(s1.phi_hat.real == 2.0)
    assert s1.Q == 2.0 and s1.R1 == 2.0
    assert s1.A0[0] == 1.0 and s1.dt == 1.0         # A0 and dt are not copied (Types.jl:257-262)
    s2.phi[0, 0, 0] = 99.0
    assert s1.phi[0, 0, 0] == 2.0


def test_g8_bdf():                                 # :369-395
    b1, b2 = O.bdf_coeff(1), O.bdf_coeff(2)
    assert (b1.a, b1.b, b1.c) == (1.0, -1.0, 0.0)
    assert (b2.a, b2.b, b2.c) == (1.5, -2.0, 0.5)
    dt = 0.01
    approx = (b2.a * 1.0 + b2.b * (1 - dt) ** 2 + b2.c * (1 - 2 * dt) ** 2) / dt
    assert abs(approx - 2.0) < 1e-2


def test_c2r_convention_non_hermitian(cfg, ops):
    """The c2r used by the reference on non-Hermitian half spectra: complex
    inverse along y, then a 1-D c2r along x that keeps only Re of the kx=0
    and kx=Nx/2 bins (FFTW rdft2 / pocketfft)."""
    rng = np.random.default_rng(7)
    H = rng.standard_normal((cfg.N, cfg.Ny, cfg.Nx // 2 + 1)) + 1j * rng.standard_normal((cfg.N, cfg.Ny, cfg.Nx // 2 + 1))
    col = np.fft.ifft(H, axis=-2)
    ref = np.empty((cfg.N, cfg.Ny, cfg.Nx))
    L = cfg.Nx
    k = np.arange(1, L // 2)
    n = np.arange(L)
    for j in range(cfg.Ny):
        c = col[0, j]
        ref[0, j] = (c[0].real + c[L // 2].real * (-1.0) ** n
                     + 2 * np.real(np.exp(2j * np.pi * np.outer(n, k) / L) @ c[1:L // 2])) / L
    np.testing.assert_allclose(ops.irfft(H), ref, rtol=0, atol=1e-14)
