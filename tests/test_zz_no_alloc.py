"""The allocation-free periodic field solve, through the C ABI.

Callers that cannot call cudaMalloc (their own memory pool owns the device, or
their stepping loop must not trigger an allocation's implicit synchronisation)
hand in their own device buffers; the library's FFT work arrays then come from
a static device array.  This file sorts last so that a stop-at-first-failure run
has already run every other test; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import apic

pytestmark = pytest.mark.gpu
TOL = 1e-12  # the tolerance of the FP64 field-solve parity tests


def _noalloc_solve(torch, dims, n, length, eps, rho):
    lib = apic.lib()
    fn = lib.apic_field_solve_periodic_nd_noalloc
    fn.argtypes = [C.c_int, C.POINTER(C.c_size_t), C.POINTER(C.c_double), C.c_double, C.c_void_p, C.c_void_p,
                   C.c_void_p, C.c_void_p]
    N = int(np.prod(n))
    d_rho = torch.from_numpy(np.ascontiguousarray(rho)).cuda()
    d_phi = torch.full((N,), float("nan"), dtype=torch.float64, device="cuda")
    d_E = torch.full((dims * N,), float("nan"), dtype=torch.float64, device="cuda")
    ns = (C.c_size_t * 3)(*(list(n) + [1] * (3 - len(n))))
    Ls = (C.c_double * 3)(*(list(length) + [1.0] * (3 - len(length))))
    stream = torch.cuda.current_stream().cuda_stream
    rc = fn(dims, ns, Ls, eps, d_rho.data_ptr(), d_phi.data_ptr(), d_E.data_ptr(), stream)
    assert rc == 0, lib.apic_simnd_last_error(None)
    torch.cuda.synchronize()
    return d_phi.cpu().numpy(), d_E.cpu().numpy().reshape(dims, N)


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("dims,n", [(2, (128, 64)), (3, (32, 16, 16))])
def test_noalloc_solve_matches_allocating_solve_twice(dims, n):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(31 + dims)
    length = [0.9 * (a + 1) for a in range(dims)]
    for call in range(2):  # two calls in a row: the shared array must not carry state
        rho = rng.standard_normal(int(np.prod(n))) + 2.0 * call
        phi_ref, E_ref = apic.field_solve_periodic_nd(dims, n, length, 1.7, rho)
        phi, E = _noalloc_solve(torch, dims, n, length, 1.7, rho)
        assert np.all(np.isfinite(phi)) and np.all(np.isfinite(E))
        assert _rel(phi, phi_ref) < TOL, (call, _rel(phi, phi_ref))
        assert _rel(E, E_ref) < TOL, (call, _rel(E, E_ref))


def test_noalloc_rejects_meshes_beyond_the_array():
    torch = pytest.importorskip("torch")
    lib = apic.lib()
    fn = lib.apic_field_solve_periodic_nd_noalloc
    fn.argtypes = [C.c_int, C.POINTER(C.c_size_t), C.POINTER(C.c_double), C.c_double, C.c_void_p, C.c_void_p,
                   C.c_void_p, C.c_void_p]
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    ns = (C.c_size_t * 3)(512, 512, 1)
    Ls = (C.c_double * 3)(1.0, 1.0, 1.0)
    rc = fn(2, ns, Ls, 1.0, buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), None)
    assert rc == 3  # APIC_ERR_CAPACITY
    assert b"scratch array holds 65536" in lib.apic_simnd_last_error(None)


def test_noalloc_rejects_host_buffers():
    """A host buffer (the older allocating API took host arrays) is refused
    before any kernel could touch it."""
    torch = pytest.importorskip("torch")
    lib = apic.lib()
    fn = lib.apic_field_solve_periodic_nd_noalloc
    fn.argtypes = [C.c_int, C.POINTER(C.c_size_t), C.POINTER(C.c_double), C.c_double, C.c_void_p, C.c_void_p,
                   C.c_void_p, C.c_void_p]
    host = np.zeros(2 * 64 * 64)
    dev = torch.zeros(2 * 64 * 64, dtype=torch.float64, device="cuda")
    ns = (C.c_size_t * 3)(64, 64, 1)
    Ls = (C.c_double * 3)(1.0, 1.0, 1.0)
    for args in ((host.ctypes.data, dev.data_ptr(), dev.data_ptr()),
                 (dev.data_ptr(), host.ctypes.data, dev.data_ptr()),
                 (dev.data_ptr(), dev.data_ptr(), host.ctypes.data)):
        rc = fn(2, ns, Ls, 1.0, *args, None)
        assert rc == 1, rc  # APIC_ERR_INVALID
        assert b"device or managed memory" in lib.apic_simnd_last_error(None) or \
            b"not a device pointer" in lib.apic_simnd_last_error(None)
