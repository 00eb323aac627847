"""ctypes binding of the C ABI declared in include/usv.h.

The library is the in-tree ``_lib/libusv_b200.so`` built for sm_100a by
``python -m ultrasound_solver_b200.build``. There is no fallback: if it is
missing, or no CUDA device is present, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

from . import build as _build

ABI_VERSION = 3
USV_OK = 0
USV_ERR_ARG = 1
USV_ERR_CUDA = 2
USV_ERR_WORKSPACE = 3
USV_ERR_NOT_CONVERGED = 4
USV_ERR_NONFINITE = 5
USV_ERR_SOURCE_PML = 6
USV_ERR_SOURCE_SOFT = 7
USV_ERR_SOURCE_CLEARANCE = 8
USV_ERR_TOO_LARGE = 9
USV_ERR_DEVICE_TIMEOUT = 10

FACE_REFLECTING, FACE_OPEN, FACE_SOFT, FACE_IMPEDANCE = 0, 1, 2, 3
APPLY_A, APPLY_AH, APPLY_ABS_A, APPLY_ABS_AH, APPLY_K, APPLY_KH = range(6)
PREC_FP64, PREC_MIXED, PREC_MIXED_BF16 = 0, 1, 2
GMRES_ORTH_CPASYNC = 1
GMRES_COMBINE_MMA_SYNC = 2
GMRES_DOTS_C64_ROWS = 4
STENCIL_AUTO, STENCIL_COEF_ROWS, STENCIL_RECORD_TILES = 0, 1, 2
LOSS_FOCAL_PRESSURE, LOSS_FOCAL_CONTRAST, LOSS_CONTRAST_RATIO = 0, 1, 2


class Scene(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("face_kind", C.c_int32 * 6),
                ("dx", C.c_double), ("omega", C.c_double),
                ("impedance_re", C.c_double * 6), ("impedance_im", C.c_double * 6),
                ("pml_cells", C.c_int32), ("pml_order", C.c_int32),
                ("pml_strength", C.c_double), ("pml_faces", C.c_int32),
                ("reserved", C.c_int32)]


KFAMILIES = 8
KFAMILY_NAMES = ("arnoldi_dots", "arnoldi_orth", "lsq", "update", "residual", "gates",
                 "recycle_pair", "recycle_dots")


class GmresProfile(C.Structure):
    _fields_ = [("launches", C.c_int32 * KFAMILIES),
                ("milliseconds", C.c_double * KFAMILIES), ("bytes", C.c_double * KFAMILIES)]


class GmresParams(C.Structure):
    _fields_ = [("restart", C.c_int32), ("maxiter", C.c_int32), ("rtol", C.c_double),
                ("backward_error_tol", C.c_double), ("precision", C.c_int32),
                ("adjoint", C.c_int32), ("full_cycles", C.c_int32), ("use_graph", C.c_int32),
                ("block_nodes", C.c_int32), ("history_capacity", C.c_int32),
                ("history", C.POINTER(C.c_double)),
                ("profile", C.POINTER(GmresProfile)),
                ("recycle", C.c_int32), ("recycle_every", C.c_int32),
                ("max_ctas", C.c_int32), ("kernel_variant", C.c_int32)]


class GmresStats(C.Structure):
    _fields_ = [("status", C.c_int32), ("info", C.c_int32), ("iterations", C.c_int32),
                ("cycles", C.c_int32), ("scaled_residual", C.c_double),
                ("backward_error", C.c_double), ("initial_residual", C.c_double)]


_P = C.c_void_p
_D = C.c_double
_I = C.c_int
_I64 = C.c_int64
_SZ = C.c_size_t
_SP = C.POINTER(Scene)

_SIGNATURES = {
    "usv_abi_version": ([], _I),
    "usv_harmonic_ritz": ([_I, _I, _P, _P, _P, _P], _I),
    "usv_z_transfer": ([_P, _P, _P, _P, _P, _I, _I, _P], _I),
    "usv_status_string": ([_I], C.c_char_p),
    "usv_device_info": ([C.POINTER(_I), C.POINTER(_I), C.POINTER(_I)], _I),
    "usv_operator_bytes": ([_SP, C.POINTER(_SZ)], _I),
    "usv_operator_build": ([_SP, _P, _P, _P, _SZ, _P], _I),
    "usv_operator_apply": ([_SP, _P, _I, _I, _P, _P, _I, _I64, _P], _I),
    "usv_operator_apply_kernel": ([_SP, _P, _I, _I, _I, _P, _P, _I, _I64, _P], _I),
    "usv_operator_export": ([_SP, _P, _P, _P, _P, _P, _P, _P], _I),
    "usv_gmres_workspace_bytes": ([_SP, C.POINTER(GmresParams), _I, C.POINTER(_SZ)], _I),
    "usv_gmres_solve": ([_SP, _P, C.POINTER(GmresParams), _P, _P, _I, _I64, _P, _SZ,
                         C.POINTER(GmresStats), _P], _I),
    "usv_gmres_scenes_workspace_bytes": ([_I, _SP, _P, C.POINTER(GmresParams), _I,
                                          C.POINTER(_SZ)], _I),
    "usv_gmres_solve_scenes": ([_I, _SP, _P, _P, C.POINTER(GmresParams), _P, _P, _I, _I64, _P,
                                _SZ, C.POINTER(GmresStats), _P], _I),
    "usv_materials_blend": ([_SP, _P, _P, _D, _D, _D, _D, _P, _P, _D, _D, _P, _P, _P], _I),
    "usv_source_masses": ([_SP, _P, _P, _P, _I, _D, _P, _P, _P, _I, _P, _P], _I),
    "usv_source_rhs": ([_SP, _P, _I, _P, _D, _P, _I, _I64, _P], _I),
    "usv_source_phase_grad": ([_SP, _P, _I, _P, _P, _P, _D, _P, _P], _I),
    "usv_material_vjp": ([_SP, _P, _P, _P, _P, _P, _P, _P, _P], _I),
    "usv_basis_field": ([_P, _I64, _I, _I, _P, _P, _P], _I),
    "usv_basis_adjoint_workspace_bytes": ([_I64, _I, C.POINTER(_SZ)], _I),
    "usv_basis_adjoint": ([_P, _I64, _I, _I, _P, _P, _P, _P, _P, _SZ, _P], _I),
    "usv_loss_workspace_bytes": ([_I64, C.POINTER(_SZ)], _I),
    "usv_loss": ([_I, _P, _I64, _P, _P, _I, _D, _D, _D, _D, _P, _P, _P, _SZ, _P], _I),
    "usv_basis_adjoint_noalloc": ([_P, _I64, _I, _I, _P, _P, _P, _P, _P], _I),
    "usv_basis_target_response": ([_P, _I64, _I64, _I64, _I, _I, _P, _I, _D, _P, _P], _I),
}

_lib = None


def header_functions() -> list[str]:
    """Function names declared in include/usv.h."""
    text = (_build.INCLUDE / "usv.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(usv_\w+)\s*\(", text, re.M)))


def load(path: Path | None = None, build_if_missing: bool = False):
    """Load the shared library (no compute call is made)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    target = Path(path) if path else _build.library_path()
    if not target.exists():
        if build_if_missing:
            _build.build()
        else:
            raise RuntimeError(f"CUDA library {target} is missing; build it with "
                               "`python -m ultrasound_solver_b200.build`")
    lib = C.CDLL(str(target))
    for name, (args, res) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    if lib.usv_abi_version() != ABI_VERSION:
        raise RuntimeError("libusv_b200 ABI version mismatch")
    if path is None:
        _lib = lib
    return lib


def status_string(status: int) -> str:
    return load().usv_status_string(status).decode()


def check(status: int, what: str = "usv") -> None:
    """Map a status code to the reference's exception types."""
    if status == USV_OK:
        return
    msg = f"{what}: {status_string(status)}"
    if status in (USV_ERR_ARG, USV_ERR_SOURCE_PML, USV_ERR_SOURCE_SOFT,
                  USV_ERR_SOURCE_CLEARANCE, USV_ERR_WORKSPACE, USV_ERR_TOO_LARGE):
        raise ValueError(msg)
    raise RuntimeError(msg)


def ptr(tensor) -> C.c_void_p:
    return C.c_void_p(tensor.data_ptr())


def stream_handle(torch_module, device=None) -> C.c_void_p:
    return C.c_void_p(torch_module.cuda.current_stream(device).cuda_stream)
