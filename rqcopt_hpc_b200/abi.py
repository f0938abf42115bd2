"""ctypes declarations of the C ABI (include/rqcopt_gpu.h) shared by the Python host mirror.

The structures are layout-identical to the reference's C types:
``struct statevector {numeric* data; int nqubits;}`` and the row-major
``struct mat4x4 {double complex data[16];}``, which from numpy is a
C-contiguous complex128 array of shape (..., 4, 4).
"""
from __future__ import annotations

import ctypes as C

import numpy as np


class Statevector(C.Structure):
    _fields_ = [("data", C.c_void_p), ("nqubits", C.c_int)]


class StatevectorArray(C.Structure):
    """struct statevector_array: 2^nqubits x nstates amplitudes, states interleaved."""
    _fields_ = [("data", C.c_void_p), ("nqubits", C.c_int), ("nstates", C.c_int)]


class Pcg32(C.Structure):
    """struct pcg32_random: one PCG32 generator (state, stream)."""
    _fields_ = [("state", C.c_uint64), ("inc", C.c_uint64)]


class RngState(C.Structure):
    """struct rng_state: the two PCG32 generators of the reference's rng_state."""
    _fields_ = [("gen", Pcg32 * 2)]

    def tuple(self):
        return tuple((g.state, g.inc) for g in self.gen)


class QuantumCircuitCache(C.Structure):
    _fields_ = [("psi_list", C.POINTER(Statevector)), ("nqubits", C.c_int), ("ngates", C.c_int)]


class TruncatedCGParams(C.Structure):
    _fields_ = [("maxiter", C.c_int), ("abstol", C.c_double), ("reltol", C.c_double)]


TARGET_FUNC = C.CFUNCTYPE(C.c_double, C.POINTER(C.c_double), C.c_void_p)
TARGET_GRAD_FUNC = C.CFUNCTYPE(C.c_double, C.POINTER(C.c_double), C.c_void_p, C.POINTER(C.c_double))
TARGET_GRAD_HESS_FUNC = C.CFUNCTYPE(C.c_double, C.POINTER(C.c_double), C.c_void_p, C.POINTER(C.c_double),
                                   C.POINTER(C.c_double))
HVP_FUNC = C.CFUNCTYPE(None, C.POINTER(C.c_double), C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double))
RETRACT_FUNC = C.CFUNCTYPE(None, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_void_p, C.POINTER(C.c_double))
LINEAR_FUNC = C.CFUNCTYPE(C.c_int, C.POINTER(Statevector), C.c_void_p, C.POINTER(Statevector))


class RTRParams(C.Structure):
    _fields_ = [("tcg_params", TruncatedCGParams), ("rho_trust", C.c_double), ("radius_init", C.c_double),
                ("maxradius", C.c_double), ("g_func", C.c_void_p), ("g_data", C.c_void_p),
                ("g_iter", C.POINTER(C.c_double))]


def default_rtr_params(n: int) -> RTRParams:
    """Defaults of set_rtr_default_params (src/trust_region.h:68-77)."""
    p = RTRParams()
    p.tcg_params.maxiter = 2 * n
    p.tcg_params.abstol = 1e-8
    p.tcg_params.reltol = 1e-6
    p.rho_trust = 0.125
    p.radius_init = 0.01
    p.maxradius = 0.1
    return p


def default_tcg_params(n: int) -> TruncatedCGParams:
    """Defaults of set_truncated_cg_default_params (src/trust_region.h:23-28)."""
    p = TruncatedCGParams()
    p.maxiter = 2 * n
    p.abstol = 1e-8
    p.reltol = 1e-6
    return p


class BrickwallTarget(C.Structure):
    """struct rqcopt_brickwall_target: matrix-free brickwall target evaluated on the device."""
    _fields_ = [("vlist", C.c_void_p), ("nlayers", C.c_int), ("perms", C.POINTER(C.POINTER(C.c_int)))]


class DenseTarget(C.Structure):
    """struct rqcopt_dense_target: a dense row-major 2^n x 2^n target matrix."""
    _fields_ = [("u", C.c_void_p), ("nqubits", C.c_int)]


class CircuitTarget(C.Structure):
    """struct rqcopt_circuit_target: matrix-free general-circuit target evaluated on the device."""
    _fields_ = [("gates", C.c_void_p), ("ngates", C.c_int), ("wires", C.POINTER(C.c_int))]


def ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def cplx(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.complex128)


def ints(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def perm_pointers(perms: np.ndarray):
    """`const int* perms[]` from a (nlayers, L) int32 array; keep the returned tuple alive."""
    perms = ints(perms)
    arr = (C.POINTER(C.c_int) * perms.shape[0])()
    for k in range(perms.shape[0]):
        arr[k] = C.cast(perms[k].ctypes.data, C.POINTER(C.c_int))
    return arr, perms


def sv(a: np.ndarray, nqubits: int) -> Statevector:
    return Statevector(a.ctypes.data, nqubits)


def wrap_ufunc(fn):
    """Wrap a Python map numpy(2^L complex) -> numpy(2^L complex) as a `linear_func`."""

    def cb(psi_p, udata, out_p):
        try:
            psi = psi_p.contents
            out = out_p.contents
            n = 1 << psi.nqubits
            x = np.ctypeslib.as_array(C.cast(psi.data, C.POINTER(C.c_double)), shape=(2 * n,)).view(np.complex128)
            y = np.ctypeslib.as_array(C.cast(out.data, C.POINTER(C.c_double)), shape=(2 * n,)).view(np.complex128)
            y[:] = fn(x.copy())
            return 0
        except Exception:  # a failing target is reported as the reference's -2
            return -1

    return LINEAR_FUNC(cb)


def fixture_ufunc(x: np.ndarray) -> np.ndarray:
    """The synthetic sparse target map of the reference tests (test/test_target.c:16-34)."""
    n = x.shape[0]
    i = np.arange(n)
    return ((-1.1 + 0.8j) * x[((i + 3) * 113) % n] + (0.4 - 0.7j) * x[((i + 9) * 173) % n]
            + (0.5 + 0.1j) * x[i] + (-0.3 + 0.2j) * x[((i + 4) * 199) % n])
