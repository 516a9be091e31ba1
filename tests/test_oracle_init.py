"""The oracle's restatement of generate_initial_condition (Init.jl:74-216,
Init_3d.jl:67-152).  The reference has no test of it (test/test.jl only calls it
with state_type 1 before timing the steps), so it is pinned by analytic facts of
each shape: areas, the angle convention of Julia's atan(X - cx, Y - cy), mirror
symmetry, the psi map, and the error() cases."""
import math

import numpy as np
import pytest

from oracle import vsav_oracle as O


def cfg(N=1, goal="s", n=256, ndim=2):
    c = O.set_para_base(1e-6, 1e-3, ndim=ndim)
    if ndim == 3:
        c = O.replace(c, Nx=n, Ny=n, Nz=n)
    else:
        c = O.replace(c, Nx=n * N, Ny=n, Lx=1.0 * N)
    return O.replace(c, N=N, goal=goal, psi_in_v=[0.1] * N, psi_out_v=[0.8] * N)


def test_ellipse_area_and_centre():
    c = cfg()
    phi, psi = O.reference_shapes(c, 1)
    R = 0.2 * c.Lx
    # semi-axes sqrt(2) R along x and R along y (Init.jl:108)
    assert abs(np.mean(phi[0] > 0) * c.Lx * c.Ly - math.pi * math.sqrt(2) * R * R) < 2e-3
    assert phi[0, c.Ny // 2, c.Nx // 2] == pytest.approx(math.tanh(R / (math.sqrt(2) * c.epsilon)), abs=1e-15)
    np.testing.assert_allclose(psi, -0.1 * phi + 0.7, rtol=0, atol=1e-15)


def test_star_angle_is_measured_from_the_y_axis():
    """R(theta) = R0 + amp cos(10 theta), theta = atan(X - cx, Y - cy): along +y
    theta = 0 (R0 + amp), along +x theta = pi/2 (cos 5 pi = -1, R0 - amp)."""
    for goal, R0, amp in (("s", 0.3, 0.01), ("g", 0.18, 0.02)):
        c = cfg(goal=goal)
        phi, _ = O.reference_shapes(c, 3)
        i0, j0, den = c.Nx // 2, c.Ny // 2, math.sqrt(2) * c.epsilon
        for d in (40, 70, 90):
            r = d * c.dx
            assert phi[0, j0 + d, i0] == pytest.approx(math.tanh((R0 + amp - r) / den), abs=1e-14)
            assert phi[0, j0, i0 + d] == pytest.approx(math.tanh((R0 - amp - r) / den), abs=1e-14)


def test_blob_draws_enter_in_the_reference_order():
    c = cfg()
    # u = 0.5 everywhere: every an = 0, a circle of R0 = 0.3
    phi, _ = O.reference_shapes(c, 4, np.full(20, 0.5))
    star, _ = O.reference_shapes(c, 3)                 # goal s: R0 = 0.3 with amp 0.01
    X = np.arange(c.Nx) * c.dx - 0.5
    r = np.sqrt(X[None, :] ** 2 + X[:, None] ** 2)
    np.testing.assert_allclose(phi[0], np.tanh((0.3 - r) / (math.sqrt(2) * c.epsilon)), atol=1e-15)
    assert np.abs(phi - star).max() > 1e-3
    # only k = 1: an_1 = (u0*2-1)*0.15, pn_1 = u1*2pi; theta = 0 along +y
    u = np.full(20, 0.5)
    u[0], u[1] = 1.0, 0.25
    phi, _ = O.reference_shapes(c, 4, u)
    i0, d = c.Nx // 2, 60
    Rk = 0.3 + 0.15 * 0.3 * math.cos(0 + 0.5 * math.pi)          # theta = 0
    Rx = 0.3 + 0.15 * 0.3 * math.cos(0.5 * math.pi + 0.5 * math.pi)  # theta = pi/2
    den = math.sqrt(2) * c.epsilon
    assert phi[0, i0 + d, i0] == pytest.approx(math.tanh((Rk - d * c.dx) / den), abs=1e-14)
    assert phi[0, i0, i0 + d] == pytest.approx(math.tanh((Rx - d * c.dx) / den), abs=1e-14)
    with pytest.raises(O.InitError):
        O.reference_shapes(c, 4)


def test_triangle_mirror_symmetry_and_inradius():
    c = cfg()
    phi, _ = O.reference_shapes(c, 2)
    # x -> 2 cx - x swaps the two slanted half-planes
    np.testing.assert_allclose(phi[0, :, 1:], phi[0, :, :0:-1], atol=1e-14)
    # area of the equilateral triangle with inradius 0.65 Lx / 3, slightly rounded by the smooth max
    rin = 0.65 * c.Lx / 3
    area = np.mean(phi[0] > 0) * c.Lx * c.Ly
    assert 0.95 * 3 * math.sqrt(3) * rin ** 2 < area < 3 * math.sqrt(3) * rin ** 2


def test_two_and_three_vesicle_stars():
    c = cfg(N=2, goal="g")
    phi, psi = O.reference_shapes(c, 7)
    assert phi.shape == (2, c.Ny, c.Nx)
    # centres 0.75 / 1.25 (goal g), R0 = 0.2: each field is the other shifted by 0.5 / dx cells
    s = int(round(0.5 / c.dx))
    np.testing.assert_allclose(phi[1], np.roll(phi[0], s, axis=1), atol=1e-13)
    np.testing.assert_allclose(psi, -0.35 * phi + 0.45, atol=1e-15)
    c = cfg(N=2, goal="s")
    phi, _ = O.reference_shapes(c, 8)
    assert abs(np.mean(phi[0] > 0) * c.Lx * c.Ly - math.pi * 0.09) < 2e-3
    c = cfg(N=3, goal="g")
    phi, _ = O.reference_shapes(c, 7)
    assert phi.shape == (3, c.Ny, c.Nx)


def test_ellipsoid_volume_3d():
    c = cfg(ndim=3, n=64, goal="g")
    phi, psi = O.reference_shapes(c, 1)
    R = 0.2 * c.Lx
    vol = np.mean(phi[0] > 0) * c.Lx * c.Ly * c.Lz
    assert abs(vol - 4 / 3 * math.pi * 2 * R ** 3) < 0.02 * vol
    np.testing.assert_allclose(psi, -0.35 * phi + 0.45, atol=1e-15)


@pytest.mark.parametrize("N,goal,st,ndim", [(1, "s", 7, 2), (2, "g", 1, 2), (2, "x", 7, 2), (2, "s", 7, 2),
                                             (2, "g", 8, 2), (4, "g", 7, 2), (1, "g", 7, 3), (2, "g", 7, 3)])
def test_rejected_cases(N, goal, st, ndim):
    c = cfg(N=N, goal=goal, n=32, ndim=ndim)
    with pytest.raises(O.InitError):
        O.reference_shapes(c, st)


@pytest.mark.parametrize("N,st,ndim", [(1, 5, 2), (1, 6, 2), (1, 0, 2), (2, 9, 2), (1, 2, 3), (3, 1, 3)])
def test_unhandled_types_leave_phi_zero(N, st, ndim):
    c = cfg(N=N, goal="g", n=32, ndim=ndim)
    phi, psi = O.reference_shapes(c, st)
    assert not phi.any()
    np.testing.assert_allclose(psi, 0.45)
