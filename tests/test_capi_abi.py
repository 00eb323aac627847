"""The C ABI library loads and exports every symbol include/usv.h declares (CPU only)."""
import ctypes

import pytest

from ultrasound_solver_b200 import _native, build


@pytest.fixture(scope="module")
def lib():
    build.build()
    return _native.load()


def test_header_declares_entry_points():
    names = _native.header_functions()
    assert "usv_gmres_solve" in names and "usv_operator_apply" in names
    assert len(names) >= 15


def test_every_declared_symbol_is_exported(lib):
    for name in _native.header_functions():
        assert hasattr(lib, name), name
        assert name in _native._SIGNATURES, f"{name} has no ctypes signature"


def test_struct_sizes_match_header(lib):
    # natural C alignment of the structs in include/usv.h (4 bytes of padding before dx)
    assert ctypes.sizeof(_native.Scene) == 176
    assert _native.Scene.dx.offset == 40
    assert ctypes.sizeof(_native.GmresParams) == 72
    assert ctypes.sizeof(_native.GmresProfile) == 160
    assert ctypes.sizeof(_native.GmresStats) == 40


def test_host_only_entry_points(lib):
    assert lib.usv_abi_version() == 2
    assert lib.usv_status_string(0) == b"ok"
    s = _native.Scene()
    s.nx = s.ny = s.nz = 9
    s.dx, s.omega, s.pml_order = 1e-3, 2.5e5, 3
    nbytes = ctypes.c_size_t()
    assert lib.usv_operator_bytes(ctypes.byref(s), ctypes.byref(nbytes)) == 0
    assert nbytes.value > 9 ** 3 * 100
    s.pml_cells, s.pml_order, s.pml_strength, s.pml_faces = 5, 2, 2.0, 1
    # PML on a reflecting face is rejected before any device work
    assert lib.usv_operator_bytes(ctypes.byref(s), ctypes.byref(nbytes)) == _native.USV_ERR_ARG
    p = _native.GmresParams()
    p.restart, p.maxiter, p.rtol, p.backward_error_tol = 30, 300, 1e-6, 1e-4
    s.pml_cells = 0
    assert lib.usv_gmres_workspace_bytes(ctypes.byref(s), ctypes.byref(p), 4,
                                         ctypes.byref(nbytes)) == 0
    assert nbytes.value >= 9 ** 3 * 31 * 4 * 8
    p.restart = 0
    assert lib.usv_gmres_workspace_bytes(ctypes.byref(s), ctypes.byref(p), 4,
                                         ctypes.byref(nbytes)) == _native.USV_ERR_ARG


def test_scene_validation_messages():
    from ultrasound_solver_b200.scene import make_scene
    with pytest.raises(ValueError, match="PML may only be placed on open faces"):
        make_scene((20, 20, 20), 1e-3, 2.5e5, {"-x": "reflecting"},
                   {"cells": 3, "faces": ["-x"]})
    with pytest.raises(ValueError, match="PML leaves no physical interior"):
        make_scene((7, 20, 20), 1e-3, 2.5e5, {"-x": "open", "+x": "open"}, {"cells": 3})
    with pytest.raises(ValueError, match="impedance requires"):
        make_scene((9, 9, 9), 1e-3, 2.5e5, {"+x": "impedance"})
    with pytest.raises(ValueError, match="Unsupported boundary"):
        make_scene((9, 9, 9), 1e-3, 2.5e5, {"+x": "absorbing"})
    s = make_scene((9, 9, 9), 1e-3, 2.5e5, {"+x": {"type": "impedance", "impedance": [400, 1]},
                                             "-y": "soft", "+z": "open"}, {"cells": 2})
    assert list(s.face_kind) == [0, 3, 2, 0, 0, 1] and s.pml_faces == 32
