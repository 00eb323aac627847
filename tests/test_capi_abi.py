"""The C ABI library loads and exports every symbol include/usv.h declares (CPU only)."""
import ctypes

import numpy as np
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
    assert ctypes.sizeof(_native.GmresParams) == 80
    assert ctypes.sizeof(_native.GmresProfile) == 160
    assert ctypes.sizeof(_native.GmresStats) == 40


def test_host_only_entry_points(lib):
    assert lib.usv_abi_version() == _native.ABI_VERSION == 3
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


def _arnoldi(A, v, m):
    n = A.shape[0]
    V = np.zeros((n, m + 1), complex)
    H = np.zeros((m + 1, m), complex)
    V[:, 0] = v / np.linalg.norm(v)
    for j in range(m):
        w = A @ V[:, j]
        for _ in range(2):
            h = V[:, :j + 1].conj().T @ w
            w -= V[:, :j + 1] @ h
            H[:j + 1, j] += h
        H[j + 1, j] = np.linalg.norm(w)
        V[:, j + 1] = w / H[j + 1, j]
    return H


@pytest.mark.parametrize("m,k,aug", [(30, 10, 0), (40, 10, 4), (60, 16, 8)])
def test_harmonic_ritz_matches_scipy(lib, m, k, aug):
    """Host harmonic Ritz step of the recycled cycles against scipy's generalized eig."""
    import scipy.linalg as sl
    rng = np.random.default_rng(m)
    n = 400
    A = (np.diag(np.linspace(-1, 3, n) + 0.05j)
         + 0.3 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / np.sqrt(n))
    G = _arnoldi(A, rng.standard_normal(n) + 0j, m)
    W = np.vstack([np.eye(m), np.zeros((1, m))]).astype(complex)
    if aug:  # leading columns of a recycled cycle: Vhat^H Ut is a general block
        W[:, :aug] = rng.standard_normal((m + 1, aug)) + 1j * rng.standard_normal((m + 1, aug))
    Gf, Wf = np.asfortranarray(G), np.asfortranarray(W)
    P = np.zeros((m, k), complex, order="F")
    th = np.zeros(k, complex)
    rc = lib.usv_harmonic_ritz(m, k, Gf.ctypes.data, Wf.ctypes.data, P.ctypes.data, th.ctypes.data)
    assert rc == 0
    M1, M2 = G.conj().T @ G, G.conj().T @ W
    want = np.sort(np.abs(sl.eig(M1, M2, right=False)))[:k]
    np.testing.assert_allclose(np.sort(np.abs(th)), want, rtol=1e-9)
    for i in range(k):
        assert abs(np.linalg.norm(P[:, i]) - 1) < 1e-12
        assert np.linalg.norm(M1 @ P[:, i] - th[i] * (M2 @ P[:, i])) <= 1e-10 * np.linalg.norm(M1)
    assert lib.usv_harmonic_ritz(m, m + 1, Gf.ctypes.data, Wf.ctypes.data, P.ctypes.data,
                                 th.ctypes.data) == 1


def test_scene_batch_workspace_and_argument_checks(lib):
    """usv_gmres_scenes_workspace_bytes (host only): the workspace covers the
    largest scene; a scene index out of range, or a scene with fewer nodes
    than the restart length (which would cut every scene's cycle), is refused."""
    def scene(n):
        s = _native.Scene()
        s.nx = s.ny = s.nz = n
        s.dx, s.omega, s.pml_order = 1e-3, 2.5e5, 3
        return s
    scenes = (_native.Scene * 2)(scene(9), scene(12))
    p = _native.GmresParams()
    p.restart, p.maxiter, p.rtol, p.backward_error_tol = 30, 100, 1e-6, 1e-4
    p.precision, p.history_capacity = _native.PREC_MIXED, 4
    owner = (ctypes.c_int * 3)(0, 1, 1)
    nbytes = ctypes.c_size_t()
    assert lib.usv_gmres_scenes_workspace_bytes(2, scenes, owner, ctypes.byref(p), 3,
                                                ctypes.byref(nbytes)) == _native.USV_OK
    one = (_native.Scene * 1)(scene(12))
    same = (ctypes.c_int * 3)(0, 0, 0)
    big = ctypes.c_size_t()
    assert lib.usv_gmres_scenes_workspace_bytes(1, one, same, ctypes.byref(p), 3,
                                                ctypes.byref(big)) == _native.USV_OK
    assert nbytes.value == big.value  # laid out for the largest scene
    bad = (ctypes.c_int * 3)(0, 2, 1)
    assert lib.usv_gmres_scenes_workspace_bytes(2, scenes, bad, ctypes.byref(p), 3,
                                                ctypes.byref(nbytes)) == _native.USV_ERR_ARG
    tiny = (_native.Scene * 2)(scene(3), scene(12))  # 27 nodes < restart 30
    assert lib.usv_gmres_scenes_workspace_bytes(2, tiny, owner, ctypes.byref(p), 3,
                                                ctypes.byref(nbytes)) == _native.USV_ERR_ARG


def test_header_constants_match_the_python_layer():
    """Every integer #define of include/usv.h has the same value in _native
    (USV_ERR_* / USV_OK / USV_ABI_VERSION by their full name, the others by
    the name after USV_)."""
    import re
    header = (build.INCLUDE / "usv.h").read_text()
    seen = 0
    for name, value in re.findall(r"^#define (USV_[A-Z0-9_]+) (\d+)", header, re.M):
        if name == "USV_ABI_VERSION":
            py = "ABI_VERSION"
        elif name.startswith(("USV_ERR_", "USV_OK")):
            py = name
        else:
            py = name[len("USV_"):]
        assert hasattr(_native, py), f"{name} has no _native.{py}"
        assert getattr(_native, py) == int(value), (name, getattr(_native, py), value)
        seen += 1
    assert seen >= 30
