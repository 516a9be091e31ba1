"""Host logic of the run_simulation mirror and the headless export (no GPU):
the reference's time grid and save schedule (simulation.jl:15-19, 113-115),
set_para_base (Init.jl:8-69, Init_3d.jl:8-62), NRRD frames and CSV histories."""
import math

import numpy as np
import pytest

from oracle import vsav_oracle as O


def test_time_grid_two_phases():
    from vsav.simulation import time_grid
    Dt = time_grid(1e-6, 1e-4)
    # range(0, 1e-5, step=1e-7): 101 points; range(1e-5, 1e-4, step=1e-6)[2:end]: 90 points
    assert len(Dt) == 191
    d = np.diff(Dt)
    np.testing.assert_allclose(d[:100], 1e-7, rtol=1e-9)
    np.testing.assert_allclose(d[100:], 1e-6, rtol=1e-9)
    assert Dt[100] == pytest.approx(1e-5, rel=1e-12) and Dt[-1] == pytest.approx(1e-4, rel=1e-12)
    # T not a multiple of dt: the last point stays below T
    Dt = time_grid(3e-6, 2e-5)
    assert Dt[-1] <= 2e-5 and Dt[-1] + 3e-6 > 2e-5


def test_save_schedule_labels_the_step_start():
    from vsav.simulation import save_steps, time_grid
    Dt = time_grid(1e-6, 1e-4)
    s = save_steps(Dt, 2e-5)
    # the first step always saves (index 0 > -1); then whenever Dt[n] crosses a multiple
    assert s[0] == 1
    labels = [Dt[n - 1] for n in s]
    assert [math.floor((t + 1e-12) / 2e-5) for t in labels] == list(range(len(s)))
    assert len(s) == 5          # t = 0, 2e-5, 4e-5, 6e-5, 8e-5 (1e-4 is the end time, never a step start)


@pytest.mark.parametrize("ndim", [2, 3])
def test_set_para_base_matches_the_oracle(ndim):
    from vsav.simulation import set_para_base
    a = set_para_base(1e-6, 1e-3, ndim)
    b = O.set_para_base(1e-6, 1e-3, ndim)
    for k in ("N", "epsilon", "M_phi", "M0_psi", "eta", "gamma_surf", "gamma_area", "gamma_bend", "gamma_in",
              "beta_in", "gamma_out", "beta_out", "lamda", "S1", "S2", "S3", "S4", "C1", "C2", "C3", "dt", "T",
              "Nx", "Ny", "Lx", "Ly", "tol", "goal", "Nz", "Lz"):
        assert getattr(a, k) == getattr(b, k), k
    np.testing.assert_array_equal(a.psi_in_v, b.psi_in_v)
    np.testing.assert_array_equal(a.psi_out_v, b.psi_out_v)


def test_nrrd_round_trip(tmp_path):
    from vsav.export import read_nrrd, write_nrrd
    a = np.random.default_rng(0).standard_normal((4, 6, 8)).astype(np.float32)
    raw, hdr = write_nrrd(str(tmp_path / "vol"), a, [0.5, 0.25, 0.125])
    txt = open(hdr).read()
    assert txt.startswith("NRRD0004\n") and "sizes: 8 6 4" in txt and "encoding: raw" in txt
    assert "spacings: 0.5 0.25 0.125" in txt and "data file: vol.raw" in txt
    np.testing.assert_array_equal(read_nrrd(hdr), a)
    assert (tmp_path / "vol.raw").stat().st_size == a.nbytes


def test_history_csv(tmp_path):
    from vsav.export import write_history
    p = write_history(str(tmp_path / "e.csv"), [0.1, 0.2], [3.0, 2.5], "modified_energy")
    rows = open(p).read().splitlines()
    assert rows[0] == "t,modified_energy" and rows[1] == "0.1,3.0" and rows[2] == "0.2,2.5"
