"""Float32 frames made on the device (vsav_export_f32) and the run_simulation
mirror (simulation.jl:2-155 with Main.jl's outputs) writing MAT files, NRRD
frames and CSV histories."""
import os

import numpy as np
import pytest

from helpers import Cfg, rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_export_frames_match_the_fields(prec):
    from vsav import Handle, ics
    rs = [2, 3]
    kw, phi, psi, _ = ics.workload("multi2d_512x4", seed=4, n_override=64, N_override=5, eps_override=0.2)
    kw["dt"] = 1e-6
    h = Handle(Cfg(**kw), run_sizes=rs, precision=prec)
    h.init_state(phi, psi)
    h.run(1, 2)
    ph = h.get_field("phi")
    s = h.export_f32("phi_sum")
    np.testing.assert_allclose(s[0], ph[0] + ph[1] + 1, rtol=0, atol=2e-6)
    np.testing.assert_allclose(s[1], ph[2] + ph[3] + ph[4] + 2, rtol=0, atol=3e-6)
    u = h.get_field("u")
    np.testing.assert_allclose(h.export_f32("speed"), np.sqrt((u ** 2).sum(axis=1)), rtol=1e-6, atol=1e-30)
    for k in ("phi", "psi", "mu", "nu", "u", "p"):
        a = h.export_f32(k)
        assert a.dtype == np.float32 and a.shape == h.field_shape(k)
        np.testing.assert_array_equal(a, h.get_field(k).astype(np.float32))
    h.close()


# conf.tol = 1e-12 in 20 iterations is not always reached on this grid; the reference warns the same way
@pytest.mark.filterwarnings("ignore:BiCGSTAB did not converge")
def test_run_simulation_driver(tmp_path):
    """The driver advances exactly like one vsav_run over the reference's time
    grid, and writes what the reference writes (MAT states, frames, histories)."""
    from scipy.io import loadmat
    from vsav import Handle
    from vsav.export import read_nrrd
    from vsav.simulation import run_simulation, save_steps, set_para_base, time_grid
    dt, T, si = 1e-6, 1.4e-5, 4e-6
    conf = set_para_base(dt, T)
    conf.Nx = conf.Ny = 128                      # a smaller grid of the reference's case
    conf.epsilon = 0.02
    out = str(tmp_path / "res")
    h, E, A, Dt = run_simulation(dt, T, 3, save_path=out, save_interval=si, conf=conf)
    Dt2 = time_grid(dt, T)
    assert np.array_equal(Dt, Dt2) and len(E) == len(Dt) - 1
    # the same steps in one call from the same initial condition
    h2 = Handle(conf)
    h2.generate_initial_condition(3, conf.goal)
    E2, A2 = h2.run(1, len(Dt) - 1, dt=np.diff(Dt), monitor=True)
    for k in ("phi", "psi", "mu", "nu", "u", "p"):
        assert rel(h.get_field(k), h2.get_field(k)) < 1e-12, k
    np.testing.assert_allclose(E, E2[:, 0], rtol=1e-12)
    # the energy decreases at fixed dt; the reference's fixed BDF2 coefficients across the jump
    # from 1e-7 to 1e-6 (simulation.jl:15-19, 76-77) carry no such guarantee at the switch
    assert np.all(np.diff(E[:100]) <= 0)
    # outputs
    files = set(os.listdir(out))
    mats = set(os.listdir(os.path.join(out, "MAT")))
    for n in save_steps(Dt, si):
        t = f"{Dt[n - 1]:.2e}"
        assert f"state_2d_t{t}.mat" in mats and f"phi_t{t}.nhdr" in files and f"speed_t{t}.nhdr" in files
    assert "state_2d_final.mat" in mats and "energy_history.csv" in files and "area_history.csv" in files
    m = loadmat(os.path.join(out, "MAT", "state_2d_final.mat"))
    assert m["phi"].shape == (128, 128, 1) and m["u"].shape == (128, 128, 2)
    np.testing.assert_array_equal(m["phi"][:, :, 0], h.get_field("phi")[0].T)
    np.testing.assert_array_equal(m["u"][:, :, 1], h.get_field("u")[0, 1].T)
    assert m["Q"].item() == h.get_scalars()[0, 0]
    fr = read_nrrd(os.path.join(out, "phi_final.nhdr"))
    np.testing.assert_array_equal(fr, h.get_field("phi")[0].astype(np.float32))   # N = 1: phi + 0
    hist = np.loadtxt(os.path.join(out, "energy_history.csv"), delimiter=",", skiprows=1)
    np.testing.assert_allclose(hist[:, 1], E, rtol=1e-15)
    np.testing.assert_allclose(hist[:, 0], Dt[1:], rtol=1e-15)
    h.close()
    h2.close()
