"""The no-allocation phase-gradient entry point against the workspace one.

``usv_basis_adjoint_noalloc`` serves callers that cannot allocate device
memory at the moment they need the phase gradient: a process whose device
memory is handed to its own pool at start-up, a real-time control loop that
must not pay cudaMalloc latency or risk running out of memory mid-run, or code
that runs while a CUDA graph is being captured. It keeps its partial sums in a
1 MiB static device array instead of a caller-provided workspace (and accepts
at most 4096 emitters). These tests call it through the C ABI twice in a row
and compare both results with ``usv_basis_adjoint``. This file is collected
last on purpose, so a run that stops at the first failure has already run
everything else.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from ultrasound_solver_b200 import _native as N

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12  # both accumulate in FP64; only the summation order differs


def _case(n, m, precision, seed):
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    gen = torch.Generator(device=dev).manual_seed(seed)
    dtype = torch.complex64 if precision == N.PREC_MIXED else torch.complex128
    basis = torch.randn(m, n, dtype=dtype, device=dev, generator=gen)
    cot = torch.randn(n, dtype=torch.complex128, device=dev, generator=gen)
    phases = torch.rand(m, dtype=torch.float64, device=dev, generator=gen) * (2 * np.pi)
    return dev, basis, cot, phases


def _workspace_result(lib, dev, basis, cot, phases, n, m, precision):
    nbytes = C.c_size_t()
    assert lib.usv_basis_adjoint_workspace_bytes(n, m, C.byref(nbytes)) == N.USV_OK
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device=dev)
    resp = torch.empty(m, dtype=torch.complex128, device=dev)
    grad = torch.empty(m, dtype=torch.float64, device=dev)
    st = lib.usv_basis_adjoint(N.ptr(basis), n, m, precision, N.ptr(cot), N.ptr(phases),
                               N.ptr(resp), N.ptr(grad), N.ptr(ws), nbytes.value,
                               N.stream_handle(torch, dev))
    assert st == N.USV_OK
    torch.cuda.synchronize()
    return resp, grad


def _rel(a, b):
    return float((torch.linalg.norm(a - b) / torch.linalg.norm(b)).item())


@pytest.mark.parametrize("n,m,precision", [
    (300_001, 256, N.PREC_MIXED),      # one pass over the chunks
    (300_001, 256, N.PREC_FP64),
    (600_001, 1024, N.PREC_MIXED),     # more chunks than the static array holds per emitter
])
def test_noalloc_matches_workspace_entry_point(n, m, precision):
    lib = N.load()
    dev, basis, cot, phases = _case(n, m, precision, seed=n + m)
    resp_ref, grad_ref = _workspace_result(lib, dev, basis, cot, phases, n, m, precision)
    for _ in range(2):  # the second call sees the first call's leftovers in the array
        resp = torch.full((m,), complex(np.nan, np.nan), dtype=torch.complex128, device=dev)
        grad = torch.full((m,), np.nan, dtype=torch.float64, device=dev)
        st = lib.usv_basis_adjoint_noalloc(N.ptr(basis), n, m, precision, N.ptr(cot),
                                           N.ptr(phases), N.ptr(resp), N.ptr(grad),
                                           N.stream_handle(torch, dev))
        assert st == N.USV_OK
        torch.cuda.synchronize()
        assert _rel(resp, resp_ref) <= REL_TOL
        assert _rel(grad, grad_ref) <= REL_TOL


def test_noalloc_rejects_too_many_emitters():
    lib = N.load()
    dev, basis, cot, phases = _case(4096, 8, N.PREC_MIXED, seed=3)
    grad = torch.empty(4097, dtype=torch.float64, device=dev)
    # rejected on the host before any launch: nothing reads past the 8 columns
    st = lib.usv_basis_adjoint_noalloc(N.ptr(basis), 4096, 4097, N.PREC_MIXED, N.ptr(cot),
                                       N.ptr(phases), None, N.ptr(grad),
                                       N.stream_handle(torch, dev))
    assert st == N.USV_ERR_TOO_LARGE
    assert "no-allocation" in N.status_string(st)


def test_noalloc_against_fp64_host_gradient():
    """Pinned independently of the workspace entry point: the gradient
    Re(conj((G^H g)_m) i e^{i phi_m}) and the response G^H g computed on the
    host in FP64 (numpy) for one complex128 case."""
    lib = N.load()
    n, m = 20_011, 16
    dev, basis, cot, phases = _case(n, m, N.PREC_FP64, seed=7)
    resp = torch.empty(m, dtype=torch.complex128, device=dev)
    grad = torch.empty(m, dtype=torch.float64, device=dev)
    st = lib.usv_basis_adjoint_noalloc(N.ptr(basis), n, m, N.PREC_FP64, N.ptr(cot),
                                       N.ptr(phases), N.ptr(resp), N.ptr(grad),
                                       N.stream_handle(torch, dev))
    assert st == N.USV_OK
    torch.cuda.synchronize()
    G = basis.cpu().numpy().T            # (n, m): column m is emitter m
    g = cot.cpu().numpy()
    phi = phases.cpu().numpy()
    resp_host = G.conj().T @ g
    grad_host = np.real(np.conj(resp_host) * 1j * np.exp(1j * phi))
    np.testing.assert_allclose(resp.cpu().numpy(), resp_host, rtol=1e-12,
                               atol=1e-12 * np.abs(resp_host).max())
    np.testing.assert_allclose(grad.cpu().numpy(), grad_host, rtol=1e-10,
                               atol=1e-12 * np.abs(grad_host).max())
