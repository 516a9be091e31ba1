"""Resumable snapshots (vsav/snapshot.py): the file format round trip on the
CPU with a stand-in handle, and a bit-exact resume on the GPU."""
import numpy as np
import pytest

from helpers import Cfg, load_golden


class FakeHandle:
    """Host-side stand-in with the Handle accessors the snapshot module uses."""

    def __init__(self, nd=2, Nx=16, Ny=8, Nz=1, sizes=(2, 1), seed=0):
        self.nd, self.Nx, self.Ny, self.Nz = nd, Nx, Ny, Nz
        self.run_sizes = list(sizes)
        self.R, self.V = len(sizes), sum(sizes)
        self.precision = "fp64"
        rng = np.random.default_rng(seed)
        self.f = {}
        for lvl in (0, 1):
            for name in ("phi", "psi", "mu", "nu", "u", "p"):
                for hat in (False, True):
                    key = name + ("_hat" if hat else "")
                    shp = self.shape(key)
                    a = rng.standard_normal(shp)
                    self.f[(lvl, key)] = a + 1j * rng.standard_normal(shp) if hat else a
            self.f[(lvl, "scalars")] = rng.standard_normal((self.R, 4))
        self.f["A0"] = rng.random(self.V)
        self.f["dt"] = rng.random(self.R)

    def shape(self, key):
        last = self.Nx // 2 + 1 if key.endswith("_hat") else self.Nx
        base = key.replace("_hat", "")
        sp = (self.Ny, last)
        return (self.R, self.nd) + sp if base == "u" else ((self.R,) + sp if base == "p" else (self.V,) + sp)

    def get_field(self, k, lvl=0): return self.f[(lvl, k)].copy()
    def set_field(self, k, a, lvl=0): self.f[(lvl, k)] = np.array(a)
    def get_scalars(self, lvl=0): return self.f[(lvl, "scalars")].copy()
    def set_scalars(self, a, lvl=0): self.f[(lvl, "scalars")] = np.array(a)
    def get_A0(self): return self.f["A0"].copy()
    def set_A0(self, a): self.f["A0"] = np.array(a)
    def get_dt(self): return self.f["dt"].copy()
    def set_dt(self, a): self.f["dt"] = np.array(a)


def test_snapshot_round_trip(tmp_path):
    from vsav import snapshot
    a, b = FakeHandle(seed=1), FakeHandle(seed=2)
    p = str(tmp_path / "s.npz")
    snapshot.save(a, p, n_next=17)
    assert snapshot.load(b, p) == 17
    assert set(a.f) == set(b.f)
    for k in a.f:
        assert np.array_equal(a.f[k], b.f[k]), k


def test_snapshot_rejects_other_shapes(tmp_path):
    from vsav import snapshot
    p = str(tmp_path / "s.npz")
    snapshot.save(FakeHandle(), p, n_next=3)
    with pytest.raises(ValueError):
        snapshot.load(FakeHandle(Nx=32), p)
    with pytest.raises(ValueError):
        snapshot.load(FakeHandle(sizes=(1, 2)), p)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_resume_is_bit_exact(tmp_path, prec):
    """3 steps, snapshot, 2 more steps == a new handle loading the snapshot and
    running the same 2 steps (the reference cannot resume at all)."""
    from vsav import Handle, snapshot
    kw, g = load_golden("multi2d_n64_N2")
    h = Handle(Cfg(**kw), precision=prec)
    h.init_state(g["phi0"], g["psi0"])
    h.run(1, 3)
    p = str(tmp_path / "snap.npz")
    snapshot.save(h, p, n_next=4)
    E1, _ = h.run(4, 2, monitor=True)
    ref = {k: h.get_field(k) for k in ("phi", "psi", "mu", "nu", "u", "p")}
    q1 = h.get_scalars()
    h.close()
    h2 = Handle(Cfg(**kw), precision=prec)
    n = snapshot.load(h2, p)
    assert n == 4
    E2, _ = h2.run(n, 2, monitor=True)
    for k, v in ref.items():
        assert np.array_equal(h2.get_field(k), v), k
    assert np.array_equal(h2.get_scalars(), q1)
    assert np.array_equal(E1, E2)
    h2.close()
