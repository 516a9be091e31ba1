"""GPU parity of libvsav against the CPU oracle and its golden fixtures,
through the C ABI.  Bars: FP64 path within 1e-10 relative L2 of the oracle on
every field and SAV scalar (the reference-faithful path); FP32 bulk path
within 1e-5; transforms at round-off (2.5e-16 FP64, 1.2e-7 FP32 measured)."""
import math
import warnings

import numpy as np
import pytest

from helpers import Cfg, load_golden, rel

pytestmark = pytest.mark.gpu

FIELDS = ("phi", "psi", "mu", "nu", "u", "p")


def make(kw, **opt):
    from vsav import Handle
    return Handle(Cfg(**kw), **opt)


def kat_cfg(Nx=128, Ny=64):
    # the shared fixture of test/test_Types_Ops.jl:28-41 (non-square, L = 2 pi)
    return dict(N=1, epsilon=0.05, M_phi=1.0, M0_psi=1.0, eta=1.0, gamma_surf=1.0, gamma_area=1.0,
                gamma_bend=1.0, gamma_in=1.0, beta_in=0.0, psi_in_v=[0.1], gamma_out=1.0, beta_out=0.0,
                psi_out_v=[0.8], lamda=1.0, S1=1.0, S2=1.0, S3=1.0, S4=1.0, C1=1.0, C2=1.0, C3=1.0,
                dt=1e-3, T=1.0, Nx=Nx, Ny=Ny, Lx=2 * math.pi, Ly=2 * math.pi, tol=1e-10, goal="s")


@pytest.mark.parametrize("prec,tol", [("fp64", 2e-15), ("fp32", 6e-7)])
def test_transform_parity_2d(prec, tol):
    from oracle import vsav_oracle as O
    kw = kat_cfg()
    h = make(kw, precision=prec)
    ops = O.build_operators(O.Config(**kw))
    rng = np.random.default_rng(0)
    f = rng.standard_normal((3, 64, 128))
    assert rel(h.rfft(f), np.fft.rfft2(f)) < tol
    H = rng.standard_normal((3, 64, 65)) + 1j * rng.standard_normal((3, 64, 65))   # non-Hermitian
    assert rel(h.irfft(H), np.fft.irfft2(H, s=(64, 128))) < tol
    for m, mul in (("dx", ops.D1[0]), ("dy", ops.D1[1]), ("lap", ops.Laplacian), ("bih", ops.Biharmonic)):
        assert rel(h.irfft(H, m), np.fft.irfft2(mul * H, s=(64, 128))) < tol, m
    h.close()


@pytest.mark.parametrize("prec,tol", [("fp64", 2e-15), ("fp32", 6e-7)])
def test_transform_parity_3d(prec, tol):
    kw, g = load_golden("single3d_n32")
    h = make(kw, precision=prec)
    rng = np.random.default_rng(1)
    f = rng.standard_normal((1, 32, 32, 32))
    assert rel(h.rfft(f), np.fft.rfftn(f, axes=(1, 2, 3))) < tol
    H = rng.standard_normal((1, 32, 32, 17)) + 1j * rng.standard_normal((1, 32, 32, 17))
    assert rel(h.irfft(H), np.fft.irfftn(H, s=(32, 32, 32), axes=(1, 2, 3))) < tol
    h.close()


def test_spectral_derivative_kats_gpu():
    """test_Types_Ops.jl G4/G5 on the device FP64 transforms, same bounds."""
    from test_oracle_kat import kat_fields
    from oracle import vsav_oracle as O
    kw = kat_cfg()
    cfg = O.Config(**kw)
    h = make(kw)
    rng = np.random.default_rng(1)
    u = rng.standard_normal((1, 64, 128))
    assert np.max(np.abs(h.irfft(h.rfft(u)) - u)) < 1e-13
    c = np.full((1, 64, 128), 3.7)
    assert np.max(np.abs(h.irfft(h.rfft(c)) - c)) < 1e-15
    k = kat_fields(cfg)
    fh = h.rfft(k["f"])
    assert abs(np.sort(np.abs(fh).ravel())[::-1][0] - 1.0) < 1e-10
    assert np.max(np.abs(h.irfft(fh, "dx") - k["dx"])) < 1e-15
    assert np.max(np.abs(h.irfft(fh, "dy") - k["dy"])) < 1e-15
    assert np.max(np.abs(h.irfft(fh, "lap") - k["lap"])) < 1e-14
    assert np.max(np.abs(h.irfft(fh, "bih") - k["bih"])) < 1e-11
    h.close()


@pytest.mark.parametrize("name", ["single2d_n64", "multi2d_n64_N2", "single3d_n32"])
def test_fp64_step_parity_vs_golden(name):
    kw, g = load_golden(name)
    steps = int(g["steps"])
    h = make(kw, precision="fp64")
    h.init_state(g["phi0"], g["psi0"])
    np.testing.assert_allclose(h.get_A0(), g["A0"], rtol=1e-12)
    E, A = h.run(1, steps, monitor=True)
    for k in FIELDS:
        assert rel(h.get_field(k), g[k]) < 1e-10, (k, rel(h.get_field(k), g[k]))
    np.testing.assert_allclose(h.get_scalars()[0], g["scalars"], rtol=1e-10)
    np.testing.assert_allclose(E[:, 0], g["energy"], rtol=1e-10)
    np.testing.assert_allclose(A[:, 0], g["area"], rtol=1e-8, atol=1e-13)
    if "3d" not in name:
        # same BiCGSTAB iteration counts as the oracle in the last step
        assert list(h.psi_stats()[:, 0].astype(int)) == list(g["psi_iters"][-3:])
    h.close()


def test_fp64_step_intermediates():
    """Every solve_stepK output of the first two steps (BDF1 then BDF2)."""
    from oracle import vsav_oracle as O
    from vsav import Handle
    kw, g = load_golden("single2d_n64")
    cfg = O.Config(**kw)
    h = make(kw)
    h.init_state(g["phi0"], g["psi0"])
    orc = O.Oracle(cfg)
    pres = O.make_state(cfg, g["phi0"], g["psi0"], orc.ops)
    O.init_state(cfg, pres, orc.ops)
    old = pres.copy()
    for n in (1, 2):
        pres.dt = cfg.dt
        bdf = O.bdf_coeff(n)
        c1 = orc.solve_step1(pres, old, bdf)
        h.step1(n)
        for k in Handle.CACHE:
            # scale: the largest member of the same family (phi_12 is exactly 0 at step 1)
            fam = [c1[j] for j in Handle.CACHE if j[:3] == k[:3]]
            scale = max(np.linalg.norm(x) for x in fam)
            assert np.linalg.norm(h.get_cache(k) - c1[k]) <= 1e-10 * scale, k
        s2 = orc.solve_step2(pres, old, c1, bdf)
        h.step2(n)
        np.testing.assert_allclose(h.scalar_work(0), [s2[k] for k in ("R_11_np1", "R_21_np1", "R_31_np1",
                                                                   "R_12_np1", "R_22_np1", "R_32_np1")], rtol=1e-10)
        s3 = orc.solve_step3(c1, s2)
        h.step3()
        for k in Handle.STEP3:
            assert rel(h.get_step3(k), s3[k]) < 1e-10, k
        s4 = orc.solve_step4(pres, old, bdf)
        h.step4(n)
        assert rel(h.get_u_tilde(0, hat=True)[0], s4["u_tilde_1_hat"]) < 1e-10
        assert rel(h.get_u_tilde(1, hat=True)[0], s4["u_tilde_2_hat"]) < 1e-10
        Q = orc.solve_step5(pres, old, s3, s4, bdf)
        h.step5(n)
        assert abs(h.scalar_work(1)[0] - Q) <= 1e-10 * abs(Q)
        s6 = orc.solve_step6(s2, s3, s4, Q)
        h.step6()
        s7 = orc.solve_step7(pres, s6, bdf)
        h.step7(n)
        O.update_state(old, pres)
        for k in ("phi_hat", "psi_hat", "mu_hat", "nu_hat"):
            setattr(pres, k, s6[k])
        pres.u_hat, pres.p_hat = s7["u_hat"], s7["p_hat"]
        for k in FIELDS:
            setattr(pres, k, orc.ops.irfft(getattr(pres, k + "_hat")))
        pres.R1, pres.R2, pres.R3, pres.Q = s6["R1"], s6["R2"], s6["R3"], Q
        h.update_state()
        for k in FIELDS + ("phi_hat", "u_hat", "p_hat"):
            assert rel(h.get_field(k), getattr(pres, k)) < 1e-10, k
    h.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_ensemble_runs_are_independent(prec):
    """R runs of different vesicle counts in one handle advance exactly like
    separate handles (per-run SAV scalars, velocity and psi systems), also
    with the mixed-precision solve and graph-replayed steps."""
    from vsav import ics
    kwa, phia, psia, _ = ics.workload("multi2d_512x4", seed=1, n_override=64, N_override=1, eps_override=0.2)
    kwb, phib, psib, _ = ics.workload("multi2d_512x4", seed=2, n_override=64, N_override=2, eps_override=0.2)
    for kw in (kwa, kwb):
        kw["dt"] = 1e-6
    kwe = dict(kwa, N=1, psi_in_v=kwa["psi_in_v"] + kwb["psi_in_v"], psi_out_v=kwa["psi_out_v"] + kwb["psi_out_v"])
    he = make(kwe, run_sizes=[1, 2], precision=prec)
    he.init_state(np.concatenate([phia, phib]), np.concatenate([psia, psib]))
    Ee, _ = he.run(1, 3, monitor=True)
    # mixed: the two handles' FP32 inner sweeps differ in rounding (autotuned FFT variants of
    # different batch sizes); the FP64 refinement brings psi to conf.tol = 1e-12, and u, driven
    # by the amplified mu, agrees to a few 1e-12
    tol_u = 1e-12 if prec == "fp64" else 1e-11
    for r, (kw, phi, psi, sl) in enumerate(((kwa, phia, psia, slice(0, 1)), (kwb, phib, psib, slice(1, 3)))):
        h = make(kw, precision=prec)
        h.init_state(phi, psi)
        E, _ = h.run(1, 3, monitor=True)
        assert rel(he.get_field("phi")[sl], h.get_field("phi")) < 1e-12
        assert rel(he.get_field("u")[r], h.get_field("u")[0]) < tol_u
        np.testing.assert_allclose(he.get_scalars()[r], h.get_scalars()[0], rtol=1e-12)
        np.testing.assert_allclose(Ee[:, r], E[:, 0], rtol=1e-12)
        h.close()
    he.close()


def test_ensemble_3d_runs_are_independent():
    """Two 3D runs (one vesicle each, the reference's 3D coupling) in one handle
    advance like two separate handles."""
    from vsav import ics
    runs = [ics.workload("single3d_128", seed=s, n_override=32) for s in (1, 2)]
    for kw, *_ in runs:
        kw["dt"] = 1e-5
    kwa = runs[0][0]
    kwe = dict(kwa, N=1, psi_in_v=kwa["psi_in_v"] + runs[1][0]["psi_in_v"],
               psi_out_v=kwa["psi_out_v"] + runs[1][0]["psi_out_v"])
    he = make(kwe, run_sizes=[1, 1])
    he.init_state(np.concatenate([runs[0][1], runs[1][1]]), np.concatenate([runs[0][2], runs[1][2]]))
    Ee, _ = he.run(1, 3, monitor=True)
    for r, (kw, phi, psi, _) in enumerate(runs):
        h = make(kw)
        h.init_state(phi, psi)
        E, _ = h.run(1, 3, monitor=True)
        assert rel(he.get_field("phi")[r:r + 1], h.get_field("phi")) < 1e-12
        assert rel(he.get_field("u")[r], h.get_field("u")[0]) < 1e-12
        np.testing.assert_allclose(he.get_scalars()[r], h.get_scalars()[0], rtol=1e-12)
        np.testing.assert_allclose(Ee[:, r], E[:, 0], rtol=1e-12)
        h.close()
    he.close()


# FP32-bulk bars (relative L2 after the fixture's steps).  The fields of the
# 1e-5 accuracy bar (phi, psi, u, the energies, R1-R3, Q) are held to 1e-5
# except where the precision split itself sets the floor:
#  * mu = L_phi phi_hat + ... amplifies the FP32 FFT round-off floor of phi_hat
#    by L_phi(k_max)/L_phi(0) = (S1 k^4 + S3)/S3 (22x at 64^2, ~100x on the
#    32^3 fixture), so mu carries ~1e-7 x that factor;
#  * R1 enters through A - A0, a difference of two O(1) areas computed from
#    FP32 gradients, so its error is ~1e-7 / |A - A0| relative to R1's change;
#  * u and p are driven by the coupling phi* grad mu* + psi* grad nu*
#    (Solvers.jl:304-318), so they inherit mu's amplified floor (1.3e-5 at
#    64^2 with one vesicle, 1.4e-4 with two, 1.6e-4 on the 32^3 fixture).
FP32_BARS = {"phi": 1e-5, "psi": 1e-5, "u": 3e-4, "nu": 1e-5, "p": 3e-4, "mu": 1e-3,
             "Q": 1e-5, "R1": 1e-4, "R2": 1e-5, "R3": 1e-5, "energy": 1e-5}


@pytest.mark.parametrize("name", ["single2d_n64", "multi2d_n64_N2", "single3d_n32"])
def test_fp32_bulk_vs_fp64_oracle(name):
    """FP32 fields and FFTs, FP64 SAV inner products / 3x3 / Q, against the
    FP64 oracle's golden trajectory."""
    kw, g = load_golden(name)
    steps = int(g["steps"])
    h = make(kw, precision="fp32", psi_rtol=1e-8, psi_itmax=60)
    h.init_state(g["phi0"], g["psi0"])
    E, A = h.run(1, steps, monitor=True)
    err = {k: rel(h.get_field(k), g[k]) for k in ("phi", "psi", "mu", "nu", "u", "p")}
    sc = h.get_scalars()[0]
    for i, k in enumerate(("Q", "R1", "R2", "R3")):
        err[k] = abs(sc[i] - g["scalars"][i]) / abs(g["scalars"][i])
    err["energy"] = float(np.max(np.abs(E[:, 0] - g["energy"]) / np.abs(g["energy"])))
    bad = {k: v for k, v in err.items() if not v < FP32_BARS[k]}
    assert not bad, (bad, err)
    assert np.all(np.diff(E[:, 0]) <= 0)
    h.close()


def test_energy_non_increasing_fp64_128():
    from vsav import ics
    kw, phi, psi, _ = ics.workload("single2d_128")
    kw["dt"] = 1e-6
    h = make(kw)
    h.init_state(phi, psi)
    E, A = h.run(1, 20, monitor=True)
    assert np.all(np.diff(E[:, 0]) <= 0)
    h.close()


def test_wc_negative_is_an_error():
    from vsav import WCNegativeError
    kw, g = load_golden("single2d_n64")
    h = make(dict(kw, C3=-1e9))
    with pytest.raises(WCNegativeError):
        h.init_state(g["phi0"], g["psi0"])
    h.close()


def test_not_converged_is_a_warning():
    """itmax reached: the reference warns and keeps the iterate (Solvers.jl:76)."""
    from vsav import NotConvergedWarning
    kw, g = load_golden("single2d_n64")
    h = make(kw, psi_itmax=2)
    h.init_state(g["phi0"], g["psi0"])
    with pytest.warns(NotConvergedWarning):
        h.step1(1)
    st = h.psi_stats()
    assert st[0, 0] == 2 and st[0, 1] == 0
    h.close()


def test_half_form_converges():
    """The half-spectrum psi form converges in as many iterations as the
    reference form on a resolved interface."""
    from vsav import ics
    kw, phi, psi, _ = ics.workload("multi2d_512x4", seed=0, n_override=128, N_override=2, eps_override=0.2)
    kw["dt"] = 1e-6
    h = make(kw, psi_form="half")
    h.init_state(phi, psi)
    h.step1(1)
    st = h.psi_stats()
    assert np.all(st[:, 1] == 1) and np.max(st[:, 0]) <= 12
    h.close()


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_transforms_are_deterministic(prec):
    """Every transform is bitwise reproducible (no races, fixed reduction order)."""
    kw = kat_cfg(256, 128)
    h = make(kw, precision=prec)
    rng = np.random.default_rng(5)
    f = rng.standard_normal((3, 128, 256))
    H = rng.standard_normal((3, 128, 129)) + 1j * rng.standard_normal((3, 128, 129))
    F0, B0, D0 = h.rfft(f), h.irfft(H), h.irfft(H, "bih")
    for _ in range(10):
        assert np.array_equal(h.rfft(f), F0)
        assert np.array_equal(h.irfft(H), B0)
        assert np.array_equal(h.irfft(H, "bih"), D0)
    h.close()


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_steps_are_deterministic(prec):
    kw, g = load_golden("multi2d_n64_N2")
    out = []
    for _ in range(2):
        h = make(kw, precision=prec)
        h.init_state(g["phi0"], g["psi0"])
        h.run(1, 2)
        out.append((h.get_field("phi"), h.get_field("u"), h.get_scalars()))
        h.close()
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("name", ["single2d_n64", "multi2d_n64_N2"])
def test_mixed_precision_vs_golden(name):
    """FP64 fields with the psi BiCGSTAB in FP32 + FP64 iterative refinement:
    FP64-level agreement with the oracle."""
    kw, g = load_golden(name)
    h = make(kw, precision="mixed")
    h.init_state(g["phi0"], g["psi0"])
    E, A = h.run(1, int(g["steps"]), monitor=True)
    for k in FIELDS:
        assert rel(h.get_field(k), g[k]) < 1e-9, (k, rel(h.get_field(k), g[k]))
    np.testing.assert_allclose(h.get_scalars()[0], g["scalars"], rtol=1e-9)
    np.testing.assert_allclose(E[:, 0], g["energy"], rtol=1e-9)
    h.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_step_graph_matches_eager(prec):
    """vsav_run replays steps 2.. as CUDA graphs (Krylov loops as conditional
    WHILE nodes): same results as the eager launches, bit for bit, the same
    BiCGSTAB iteration counts, and the same number of kernels executed."""
    from vsav import _lib
    kw, g = load_golden("multi2d_n64_N2")
    out = {}
    for graph in (False, True):
        h = make(kw, precision=prec, graph=graph)
        h.init_state(g["phi0"], g["psi0"])
        h.run(1, 1, monitor=True)                   # BDF1 step: always eager
        c0 = _lib.load().vsav_launch_count()
        E, A = h.run(2, 4, monitor=True)
        launches = _lib.load().vsav_launch_count() - c0
        out[graph] = ({k: h.get_field(k) for k in FIELDS}, h.get_scalars(), E, A, h.psi_stats(), launches)
        h.close()
    fe, se, Ee, Ae, pe, le = out[False]
    fg, sg, Eg, Ag, pg, lg = out[True]
    for k in FIELDS:
        assert np.array_equal(fe[k], fg[k]), k
    assert np.array_equal(se, sg) and np.array_equal(Ee, Eg) and np.array_equal(Ae, Ag)
    assert np.array_equal(pe, pg)
    # the graph runs the same kernels plus, per Krylov loop, its condition kernel
    # (once before the loop and once per iteration) and the activity refresh of
    # the last iteration, which the eager loop skips: iterations + 2 per loop
    loops = 4 * (1 if prec == "fp64" else 2)
    assert le < lg <= le + loops * (20 + 2), (le, lg)


def test_full_size_1024x8_properties():
    """At the headline size (1024^2, 8 vesicles), where the CPU oracle is too slow to
    compare step by step, size-independent properties: the FP64 transforms round-trip
    to machine precision, the mixed path stays within 1e-5 of the FP64 path on every
    field after 2 steps (psi to relative residual 1e-8), and the modified energy does
    not increase."""
    from vsav import ics
    kw, phi, psi, _ = ics.workload("multi2d_1024x8", seed=3)
    kw["dt"] = 1e-6
    h64 = make(kw, precision="fp64")
    f = np.random.default_rng(0).standard_normal((2, 1024, 1024))
    assert rel(h64.irfft(h64.rfft(f)), f) < 1e-15
    h64.init_state(phi, psi)
    E64, _ = h64.run(1, 2, monitor=True)
    ref = {k: h64.get_field(k) for k in FIELDS}
    h64.close()
    hm = make(kw, precision="mixed", psi_rtol=1e-8)
    hm.init_state(phi, psi)
    Em, _ = hm.run(1, 2, monitor=True)
    for k in FIELDS:
        assert rel(hm.get_field(k), ref[k]) < 1e-5, k
    assert np.all(np.diff(Em[:, 0]) <= 0) and np.all(np.diff(E64[:, 0]) <= 0)
    assert np.max(np.abs(Em - E64) / np.abs(E64)) < 1e-5
    hm.close()


@pytest.mark.parametrize("which", ["single2d", "multi2d", "ensemble"])
def test_device_shapes_match_host_generator(which):
    """vsav_init_shapes2d evaluates the seeded shapes on the device: the same
    phi/psi (and so the same state after two steps) as the host generator."""
    from vsav import ics
    run_sizes = None
    if which == "single2d":
        kw, phi, psi, _ = ics.workload("single2d_128", n_override=64)
        shapes = [ics.single2d_shape(seed=0)]
    elif which == "multi2d":
        kw, phi, psi, _ = ics.workload("multi2d_512x4", seed=3, n_override=128, N_override=3, eps_override=0.1)
        shapes = ics.multi2d_shapes(3, 0.1, 3)
    else:
        kw, run_sizes, phi, psi = ics.ensemble(n_runs=4, n=64, eps=0.2)
        sizes, shapes = ics.ensemble_shapes(n_runs=4, eps=0.2)
        assert sizes == run_sizes
    kw["dt"] = 1e-6
    hd = make(kw, run_sizes=run_sizes)
    hd.init_shapes(shapes)
    hh = make(kw, run_sizes=run_sizes)
    hh.init_state(phi, psi)
    for k in ("phi", "psi", "mu", "nu"):
        assert rel(hd.get_field(k), hh.get_field(k)) < 1e-12, k
    hd.run(1, 2)
    hh.run(1, 2)
    for k in FIELDS:
        assert rel(hd.get_field(k), hh.get_field(k)) < 1e-10, k
    hd.close()
    hh.close()
