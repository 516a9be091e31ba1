"""CPU-side checks of the drop-in boundary: the C-ABI library exists, loads,
exports every function that include/vsav.h declares, and fails loudly (an
error code, no silent fallback) when no CUDA device is present."""
import os
import re

import numpy as np
import pytest

from conftest import ROOT, cuda_available

HEADER = os.path.join(ROOT, "include", "vsav.h")


def declared_functions():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|int64_t|void|const char\*)\s+(vsav_\w+)\s*\(", txt, re.M)))


def test_header_declares_the_reference_entry_points():
    names = declared_functions()
    for n in ("vsav_create", "vsav_destroy", "vsav_set_field", "vsav_get_field", "vsav_init_state",
              "vsav_step1", "vsav_step2", "vsav_step3", "vsav_step4", "vsav_step5", "vsav_step6",
              "vsav_step7", "vsav_update_state", "vsav_run", "vsav_monitor", "vsav_transform"):
        assert n in names


def test_library_exports_every_declared_symbol():
    from vsav import _lib
    lib = _lib.load()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(_lib.EXPORTS) == declared_functions()


def test_struct_layouts_match_header():
    """The ctypes mirrors have the field order of the C structs."""
    from vsav import _lib
    txt = open(HEADER).read()
    for cname, py in (("vsav_config", _lib.VsavConfig), ("vsav_options", _lib.VsavOptions),
                      ("vsav_status", _lib.VsavStatus), ("vsav_shape2d", _lib.VsavShape2D)):
        body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (cname, cname), txt, re.S).group(1)
        body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
        names = []
        for decl in body.split(";"):
            decl = decl.strip()
            if not decl:
                continue
            decl = re.sub(r"^(const\s+)?\w+\s*\**\s*", "", decl)
            names += [re.sub(r"\[\d+\]$", "", x.strip().lstrip("*")) for x in decl.split(",")]
        assert names == [f[0] for f in py._fields_], cname


@pytest.mark.skipif(cuda_available(), reason="needs a machine without a CUDA device")
def test_create_fails_loudly_without_gpu():
    from helpers import Cfg
    from vsav import Handle, VsavError, ics
    kw, phi, psi, _ = ics.workload("single2d_128", n_override=64)
    with pytest.raises(VsavError) as e:
        Handle(Cfg(**kw))
    assert e.value.code == -2          # VSAV_E_CUDA


def test_invalid_sizes_rejected_before_device_use():
    """Non-power-of-two grids are rejected with VSAV_E_INVALID."""
    from helpers import Cfg
    from vsav import Handle, VsavError, ics
    kw, phi, psi, _ = ics.workload("single2d_128", n_override=64)
    kw["Nx"] = 96
    with pytest.raises(VsavError) as e:
        Handle(Cfg(**kw))
    assert e.value.code == -1 and "power of two" in str(e.value)


def test_workloads_are_seeded():
    from vsav import ics
    a = ics.workload("multi2d_512x4", seed=5, n_override=64, N_override=3, eps_override=0.2)
    b = ics.workload("multi2d_512x4", seed=5, n_override=64, N_override=3, eps_override=0.2)
    assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])
    phi = a[1]
    assert phi.shape == (3, 64, 64) and np.all(np.abs(phi) <= 1)
    # vesicles do not overlap: at most one field is inside (phi > 0) at each point
    assert np.max(np.sum(phi > 0, axis=0)) <= 1


def test_net_and_psi_entry_points_reject_bad_arguments():
    """The learned-preconditioner and harvest entry points validate their
    arguments and report errors (no device needed for these paths)."""
    import ctypes as ct
    from vsav import _lib
    lib = _lib.load()
    assert lib.vsav_net_nparams() == 7409
    out = ct.c_void_p()
    assert lib.vsav_net_create(0, 0, ct.byref(out)) == -1          # empty capacity
    assert lib.vsav_net_destroy(None) == -1
    th = np.zeros(7409)
    assert lib.vsav_net_set_params(None, _lib.dptr(th)) == -1
    assert lib.vsav_set_psi_net(None, _lib.dptr(th)) == -1
    assert lib.vsav_psi_harvest(None, 4) == -1
    assert lib.vsav_get_dt(None, _lib.dptr(th)) == -1


def test_initial_condition_and_export_entry_points_reject_a_null_handle():
    import ctypes as ct
    from vsav import _lib
    lib = _lib.load()
    u = np.zeros(20)
    assert lib.vsav_generate_initial_condition(None, 1, ord("s"), None) == -1
    assert lib.vsav_generate_initial_condition(None, 4, ord("s"), _lib.dptr(u)) == -1
    shapes = (_lib.VsavShape2D * 1)()
    assert lib.vsav_init_shapes2d(None, shapes) == -1
    f = np.zeros(16, dtype=np.float32)
    assert lib.vsav_export_f32(None, 0, 0, f.ctypes.data_as(ct.POINTER(ct.c_float))) == -1


@pytest.mark.skipif(cuda_available(), reason="needs a machine without a CUDA device")
def test_net_create_fails_loudly_without_gpu():
    import ctypes as ct
    from vsav import _lib
    lib = _lib.load()
    out = ct.c_void_p()
    assert lib.vsav_net_create(1024, 0, ct.byref(out)) == -2       # VSAV_E_CUDA
    assert b"CUDA" in lib.vsav_net_last_error(None)
