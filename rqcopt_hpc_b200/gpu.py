"""Python host mirror of the rqcopt_hpc interface, calling librqcopt_gpu.so through its C ABI.

Function names, argument meaning and error behaviour follow the reference's C
functions (src/gate.h, src/quantum_circuit.h, src/brickwall_circuit.h,
src/target.h, src/trust_region.h, src/brickwall_opt.h, src/circuit_opt.h):
statevectors and gates are numpy complex128 arrays, perms an (nlayers, L)
integer array, and integer error codes are raised as ``RqcError``.  Arrays
passed in live in host memory, so every call exercises the staging path of the
C ABI; torch CUDA tensors may be passed where a statevector is expected to
keep data on the device.

Loading fails loudly (``OSError``) when the compiled library is missing: there
is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .abi import (HVP_FUNC, LINEAR_FUNC, RETRACT_FUNC, TARGET_FUNC, TARGET_GRAD_FUNC, TARGET_GRAD_HESS_FUNC,
                  BrickwallTarget, CircuitTarget, DenseTarget, QuantumCircuitCache, RngState, RTRParams, Statevector,
                  StatevectorArray,
                  TruncatedCGParams, cplx, default_rtr_params, default_tcg_params, ints, perm_pointers, ptr,
                  wrap_ufunc)

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "librqcopt_gpu.so")

_lib = None

VP = C.c_void_p
I = C.c_int
D = C.c_double
PSV = C.POINTER(Statevector)
PD = C.POINTER(C.c_double)


class RqcError(RuntimeError):
    def __init__(self, fn, code):
        super().__init__(f"{fn} failed with code {code}")
        self.code = code


_SIGS = {
    "allocate_statevector": (I, [I, PSV]),
    "free_statevector": (None, [PSV]),
    "add_statevectors": (None, [PSV, PSV, PSV]),
    "transpose_statevector": (None, [PSV, VP, PSV]),
    "apply_gate": (None, [VP, I, I, PSV, PSV]),
    "apply_gate_backward": (None, [VP, I, I, PSV, PSV, PSV, VP]),
    "apply_quantum_circuit": (I, [VP, I, VP, PSV, PSV]),
    "allocate_quantum_circuit_cache": (I, [I, I, C.POINTER(QuantumCircuitCache)]),
    "free_quantum_circuit_cache": (None, [C.POINTER(QuantumCircuitCache)]),
    "quantum_circuit_forward": (I, [VP, I, VP, PSV, C.POINTER(QuantumCircuitCache), PSV]),
    "quantum_circuit_backward": (I, [VP, I, VP, C.POINTER(QuantumCircuitCache), PSV, PSV, VP]),
    "quantum_circuit_gates_hessian_vector_product": (I, [VP, VP, I, VP, PSV, PSV, PSV, VP, VP]),
    "apply_brickwall_unitary": (I, [VP, I, VP, PSV, PSV]),
    "brickwall_unitary_forward": (I, [VP, I, VP, PSV, C.POINTER(QuantumCircuitCache), PSV]),
    "brickwall_unitary_backward": (I, [VP, I, VP, C.POINTER(QuantumCircuitCache), PSV, PSV, VP]),
    "circuit_unitary_target": (I, [VP, VP, VP, I, VP, I, VP]),
    "circuit_unitary_target_and_gradient": (I, [VP, VP, VP, I, VP, I, VP, VP]),
    "circuit_unitary_target_and_projected_gradient": (I, [VP, VP, VP, I, VP, I, VP, VP]),
    "circuit_unitary_target_hessian_vector_product": (I, [VP, VP, VP, VP, I, VP, I, VP, VP, VP]),
    "circuit_unitary_target_projected_hessian_vector_product": (I, [VP, VP, VP, VP, I, VP, I, VP, VP, VP]),
    "brickwall_unitary_target": (I, [VP, VP, VP, I, I, VP, VP]),
    "brickwall_unitary_target_and_gradient": (I, [VP, VP, VP, I, I, VP, VP, VP]),
    "brickwall_unitary_target_and_projected_gradient": (I, [VP, VP, VP, I, I, VP, VP, VP]),
    "brickwall_unitary_target_hessian_vector_product": (I, [VP, VP, VP, VP, I, VP, I, VP, VP, VP]),
    "brickwall_unitary_target_projected_hessian_vector_product": (I, [VP, VP, VP, VP, I, VP, I, VP, VP, VP]),
    "truncated_cg_hvp": (C.c_bool, [VP, VP, VP, VP, I, D, C.POINTER(TruncatedCGParams), VP]),
    "riemannian_trust_region_optimize_hvp": (None, [VP, VP, VP, VP, VP, VP, I, VP, I, C.POINTER(RTRParams), I, VP, VP]),
    "optimize_brickwall_circuit_hvp": (None, [VP, VP, VP, I, I, VP, C.POINTER(RTRParams), I, VP, VP]),
    "optimize_quantum_circuit": (None, [VP, VP, VP, I, I, VP, C.POINTER(RTRParams), I, VP, VP]),
    "real_to_tangent": (None, [VP, VP, VP]),
    "tangent_to_real": (None, [VP, VP, VP]),
    "project_tangent": (None, [VP, VP, VP]),
    "polar_factor": (None, [VP, VP]),
    "retract": (None, [VP, VP, VP]),
    "multiply_matrices": (None, [VP, VP, VP]),
    "inverse_matrix": (I, [VP, VP]),
    "symmetric_triple_matrix_product": (None, [VP, VP, VP, VP]),
    "allocate_statevector_array": (I, [I, I, C.POINTER(StatevectorArray)]),
    "free_statevector_array": (None, [C.POINTER(StatevectorArray)]),
    "apply_gate_to_array": (None, [VP, I, I, C.POINTER(StatevectorArray), C.POINTER(StatevectorArray)]),
    "apply_gate_backward_array": (None, [VP, I, I, C.POINTER(StatevectorArray), PSV, VP]),
    "apply_gate_placeholder": (None, [I, I, PSV, C.POINTER(StatevectorArray)]),
    "brickwall_unitary_backward_hessian": (I, [VP, I, VP, C.POINTER(QuantumCircuitCache), PSV, PSV, VP, VP]),
    "apply_brickwall_unitary_gate_placeholder": (I, [VP, I, VP, I, C.POINTER(QuantumCircuitCache),
                                                     C.POINTER(StatevectorArray)]),
    "brickwall_unitary_target_gradient_hessian": (I, [VP, VP, VP, I, I, VP, VP, VP, VP]),
    "brickwall_unitary_target_gradient_vector_hessian_matrix": (I, [VP, VP, VP, I, I, VP, VP, VP, VP]),
    "truncated_cg_hmat": (C.c_bool, [VP, VP, I, D, C.POINTER(TruncatedCGParams), VP]),
    "riemannian_trust_region_optimize_hmat": (None, [VP, VP, VP, VP, VP, I, VP, I, C.POINTER(RTRParams), I, VP, VP]),
    "optimize_brickwall_circuit_hmat": (None, [VP, VP, VP, I, I, VP, C.POINTER(RTRParams), I, VP, VP]),
    "brickwall_blockenc_target": (I, [VP, VP, VP, I, I, VP, VP]),
    "brickwall_blockenc_target_and_gradient": (I, [VP, VP, VP, I, I, VP, VP, VP]),
    "brickwall_blockenc_target_and_gradient_vector": (I, [VP, VP, VP, I, I, VP, VP, VP]),
    "brickwall_blockenc_target_gradient_hessian": (I, [VP, VP, VP, I, I, VP, VP, VP, VP, VP]),
    "brickwall_blockenc_target_gradient_vector_hessian_matrix": (I, [VP, VP, VP, I, I, VP, VP, VP, VP]),
    "seed_rng_state": (None, [C.c_uint64, C.POINTER(RngState)]),
    "haar_random_statevector": (None, [PSV, C.POINTER(RngState)]),
    "circuit_unitary_target_sampling": (I, [VP, VP, VP, I, VP, I, C.c_long, C.POINTER(RngState), VP]),
    "brickwall_unitary_target_sampling": (I, [VP, VP, VP, I, I, VP, C.c_long, C.POINTER(RngState), VP]),
    "brickwall_unitary_target_gradient_hessian_sampling": (I, [VP, VP, VP, I, I, VP, C.c_long, C.POINTER(RngState),
                                                              VP, VP, VP]),
    "brickwall_unitary_target_gradient_vector_hessian_matrix_sampling": (I, [VP, VP, VP, I, I, VP, C.c_long,
                                                                            C.POINTER(RngState), VP, VP, VP]),
    "optimize_brickwall_circuit_hmat_sampling": (None, [VP, VP, VP, I, I, VP, C.c_long, C.POINTER(RngState),
                                                        C.POINTER(RTRParams), I, VP, VP]),
    "rqcopt_brickwall_ufunc": (I, [PSV, VP, PSV]),
    "rqcopt_circuit_ufunc": (I, [PSV, VP, PSV]),
    "rqcopt_dense_ufunc": (I, [PSV, VP, PSV]),
    "rqcopt_gpu_set_precision": (I, [I]),
    "rqcopt_gpu_get_precision": (I, []),
    "rqcopt_gpu_set_refine_threshold": (None, [D]),
    "rqcopt_gpu_set_workspace_limit": (None, [C.c_size_t]),
    "rqcopt_gpu_set_column_chunk": (None, [C.c_long]),
    "rqcopt_gpu_set_column_range": (I, [C.c_long, C.c_long]),
    "rqcopt_gpu_set_reconstruct": (None, [I]),
    "rqcopt_gpu_set_autotune": (I, [I]),
    "rqcopt_gpu_last_config": (I, [VP, VP, VP, VP, VP]),
    "rqcopt_gpu_set_c64_fp32_pipe": (None, [I]),
    "rqcopt_gpu_last_error": (I, []),
    "rqcopt_gpu_optimizer_trace": (I, [VP, VP, VP, VP, I]),
    "rqcopt_gpu_set_gates_per_pass": (I, [I]),
    "rqcopt_gpu_set_real_pairs": (None, [I]),
    "rqcopt_gpu_set_real_samples": (None, [I]),
    "rqcopt_gpu_launch_count": (C.c_ulonglong, []),
    "rqcopt_gpu_reset_launch_count": (None, []),
    "rqcopt_gpu_enable_kernel_timing": (None, [I]),
    "rqcopt_gpu_kernel_time": (I, [I, PD, C.POINTER(C.c_long)]),
    "rqcopt_gpu_stream": (VP, []),
    "rqcopt_apply_quantum_circuit_c64": (I, [VP, I, VP, VP, VP, I]),
    "rqcopt_brickwall_batch_evaluate": (I, [VP, I, VP, I, I, VP, VP, VP]),
    "rqcopt_optimize_brickwall_batch": (I, [VP, I, VP, I, I, VP, VP]),
    "rqcopt_batch_create": (VP, [I, I]),
    "rqcopt_batch_destroy": (None, [VP]),
    "rqcopt_batch_add": (I, [VP, VP, VP, I, I, D]),
    "rqcopt_batch_run": (I, [VP, I]),
    "rqcopt_batch_finished": (I, [VP, VP, I]),
    "rqcopt_batch_result": (I, [VP, I, VP, VP, VP]),
    "rqcopt_batch_release": (I, [VP, I]),
    "rqcopt_batch_rounds": (C.c_long, [VP]),
    "rqcopt_batch_set_sharing": (I, [VP, I]),
    "rqcopt_batch_evaluations": (C.c_long, [VP, C.POINTER(C.c_long)]),
    "rqcopt_batch_footprint": (C.c_size_t, [I, I]),
}

PRECISION_C128, PRECISION_MIXED, PRECISION_C64 = 0, 1, 2
KC_APPLY, KC_FORWARD, KC_REVERSE, KC_FUSED, KC_HESS = 0, 1, 2, 3, 4


def lib():
    """The loaded C library (raises OSError if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} not found: build it with `python -m rqcopt_hpc_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(fn, ret):
    if ret != 0:
        raise RqcError(fn, ret)


def _check_void(fn):
    err = lib().rqcopt_gpu_last_error()
    if err != 0:
        raise RqcError(fn, err)


def _sv(a, L):
    """Statevector over a numpy complex128 array or a CUDA tensor (device pointer)."""
    if hasattr(a, "data_ptr"):
        return Statevector(a.data_ptr(), L)
    return Statevector(a.ctypes.data, L)


def _nq(psi):
    n = psi.shape[0] if hasattr(psi, "shape") else len(psi)
    L = int(n).bit_length() - 1
    assert 1 << L == n, "statevector length must be a power of two"
    return L


# ------------------------------------------------------------------------ gates and circuits

def transpose_statevector(psi, perm):
    """Qubit i of psi moved to qubit perm[i] (src/statevector.c:72-98)."""
    psi, perm = cplx(psi), ints(perm)
    L = _nq(psi)
    out = np.empty_like(psi)
    lib().transpose_statevector(C.byref(_sv(psi, L)), ptr(perm), C.byref(_sv(out, L)))
    _check_void("transpose_statevector")
    return out


def add_statevectors(psi1, psi2):
    """psi1 + psi2 (src/statevector.c:132-142); numpy arrays or CUDA tensors."""
    if hasattr(psi1, "data_ptr"):
        import torch
        out = torch.empty_like(psi1)
    else:
        psi1, psi2 = cplx(psi1), cplx(psi2)
        out = np.empty_like(psi1)
    L = _nq(psi1)
    lib().add_statevectors(C.byref(_sv(psi1, L)), C.byref(_sv(psi2, L)), C.byref(_sv(out, L)))
    _check_void("add_statevectors")
    return out


def apply_gate(V, i, j, psi):
    psi = cplx(psi)
    L = _nq(psi)
    out = np.empty_like(psi)
    V = cplx(V)
    lib().apply_gate(ptr(V), i, j, C.byref(_sv(psi, L)), C.byref(_sv(out, L)))
    _check_void("apply_gate")
    return out


def apply_gate_backward(V, i, j, psi, dpsi_out):
    psi, dpsi_out, V = cplx(psi), cplx(dpsi_out), cplx(V)
    L = _nq(psi)
    dpsi = np.empty_like(psi)
    dV = np.empty((4, 4), np.complex128)
    lib().apply_gate_backward(ptr(V), i, j, C.byref(_sv(psi, L)), C.byref(_sv(dpsi_out, L)), C.byref(_sv(dpsi, L)), ptr(dV))
    _check_void("apply_gate_backward")
    return dpsi, dV


def apply_quantum_circuit(gates, wires, psi):
    gates, wires, psi = cplx(gates), ints(wires), cplx(psi)
    L = _nq(psi)
    out = np.empty_like(psi)
    _check("apply_quantum_circuit", lib().apply_quantum_circuit(ptr(gates), gates.shape[0], ptr(wires),
                                                               C.byref(_sv(psi, L)), C.byref(_sv(out, L))))
    return out


class Cache:
    """quantum_circuit_cache allocated through the library (managed memory states)."""

    def __init__(self, nqubits, ngates):
        self.c = QuantumCircuitCache()
        _check("allocate_quantum_circuit_cache", lib().allocate_quantum_circuit_cache(nqubits, ngates, C.byref(self.c)))

    def state(self, k):
        s = self.c.psi_list[k]
        n = 1 << s.nqubits
        return np.ctypeslib.as_array(C.cast(s.data, C.POINTER(C.c_double)), shape=(2 * n,)).view(np.complex128).copy()

    def __del__(self):
        if _lib is not None and self.c.psi_list:
            _lib.free_quantum_circuit_cache(C.byref(self.c))


def quantum_circuit_forward(gates, wires, psi, cache=None):
    gates, wires, psi = cplx(gates), ints(wires), cplx(psi)
    L = _nq(psi)
    cache = cache or Cache(L, gates.shape[0])
    out = np.empty_like(psi)
    _check("quantum_circuit_forward", lib().quantum_circuit_forward(ptr(gates), gates.shape[0], ptr(wires),
                                                                   C.byref(_sv(psi, L)), C.byref(cache.c),
                                                                   C.byref(_sv(out, L))))
    return out, cache


def quantum_circuit_backward(gates, wires, cache, dpsi_out):
    gates, wires, dpsi_out = cplx(gates), ints(wires), cplx(dpsi_out)
    L = _nq(dpsi_out)
    dpsi = np.empty_like(dpsi_out)
    dgates = np.empty((gates.shape[0], 4, 4), np.complex128)
    _check("quantum_circuit_backward", lib().quantum_circuit_backward(ptr(gates), gates.shape[0], ptr(wires),
                                                                     C.byref(cache.c), C.byref(_sv(dpsi_out, L)),
                                                                     C.byref(_sv(dpsi, L)), ptr(dgates)))
    return dpsi, dgates


def quantum_circuit_gates_hessian_vector_product(gates, gatedirs, wires, psi, phi):
    gates, gatedirs, wires, psi, phi = cplx(gates), cplx(gatedirs), ints(wires), cplx(psi), cplx(phi)
    L = _nq(psi)
    out = np.empty_like(psi)
    dg = np.empty((gates.shape[0], 4, 4), np.complex128)
    hg = np.empty_like(dg)
    _check("quantum_circuit_gates_hessian_vector_product",
           lib().quantum_circuit_gates_hessian_vector_product(ptr(gates), ptr(gatedirs), gates.shape[0], ptr(wires),
                                                              C.byref(_sv(psi, L)), C.byref(_sv(phi, L)),
                                                              C.byref(_sv(out, L)), ptr(dg), ptr(hg)))
    return out, dg, hg


def apply_brickwall_unitary(vlist, perms, psi):
    vlist, psi = cplx(vlist), cplx(psi)
    L = _nq(psi)
    pp, keep = perm_pointers(perms)
    out = np.empty_like(psi)
    _check("apply_brickwall_unitary", lib().apply_brickwall_unitary(ptr(vlist), vlist.shape[0], C.cast(pp, VP),
                                                                   C.byref(_sv(psi, L)), C.byref(_sv(out, L))))
    return out


def brickwall_unitary_forward(vlist, perms, psi, cache=None):
    vlist, psi = cplx(vlist), cplx(psi)
    L = _nq(psi)
    pp, keep = perm_pointers(perms)
    cache = cache or Cache(L, vlist.shape[0] * (L // 2))
    out = np.empty_like(psi)
    _check("brickwall_unitary_forward", lib().brickwall_unitary_forward(ptr(vlist), vlist.shape[0], C.cast(pp, VP),
                                                                       C.byref(_sv(psi, L)), C.byref(cache.c),
                                                                       C.byref(_sv(out, L))))
    return out, cache


def brickwall_unitary_backward(vlist, perms, cache, dpsi_out):
    vlist, dpsi_out = cplx(vlist), cplx(dpsi_out)
    L = _nq(dpsi_out)
    pp, keep = perm_pointers(perms)
    dpsi = np.empty_like(dpsi_out)
    dv = np.empty((vlist.shape[0], 4, 4), np.complex128)
    _check("brickwall_unitary_backward", lib().brickwall_unitary_backward(ptr(vlist), vlist.shape[0], C.cast(pp, VP),
                                                                         C.byref(cache.c), C.byref(_sv(dpsi_out, L)),
                                                                         C.byref(_sv(dpsi, L)), ptr(dv)))
    return dpsi, dv


# ------------------------------------------------------------------------ full-Hessian primitives
# Statevector arrays are numpy complex128 arrays of shape (2^L, nstates), amplitude-major
# (the reference's interleaved layout).

def _sva(a, L):
    return StatevectorArray(a.ctypes.data, L, a.shape[1])


def apply_gate_to_array(V, i, j, psi):
    V, psi = cplx(V), cplx(psi)
    L = _nq(psi)
    out = np.empty_like(psi)
    lib().apply_gate_to_array(ptr(V), i, j, C.byref(_sva(psi, L)), C.byref(_sva(out, L)))
    _check_void("apply_gate_to_array")
    return out


def apply_gate_backward_array(V, i, j, psi, dpsi_out):
    V, psi, dpsi_out = cplx(V), cplx(psi), cplx(dpsi_out)
    L = _nq(psi)
    dg = np.empty((psi.shape[1], 4, 4), np.complex128)
    lib().apply_gate_backward_array(ptr(V), i, j, C.byref(_sva(psi, L)), C.byref(_sv(dpsi_out, L)), ptr(dg))
    _check_void("apply_gate_backward_array")
    return dg


def apply_gate_placeholder(i, j, psi):
    psi = cplx(psi)
    L = _nq(psi)
    out = np.empty((psi.shape[0], 16), np.complex128)
    lib().apply_gate_placeholder(i, j, C.byref(_sv(psi, L)), C.byref(_sva(out, L)))
    _check_void("apply_gate_placeholder")
    return out


def _host_cache(states):
    """quantum_circuit_cache over host arrays (kept alive by the returned tuple)."""
    states = [cplx(s) for s in states]
    L = _nq(states[0])
    arr = (Statevector * len(states))(*[Statevector(s.ctypes.data, L) for s in states])
    c = QuantumCircuitCache(C.cast(arr, C.POINTER(Statevector)), L, len(states))
    return c, (arr, states)


def brickwall_unitary_backward_hessian(vlist, perms, cache, dpsi_out):
    """cache: a Cache from brickwall_unitary_forward or a list of the gate input states."""
    vlist, dpsi_out = cplx(vlist), cplx(dpsi_out)
    L, nl = _nq(dpsi_out), vlist.shape[0]
    pp, keep = perm_pointers(perms)
    c, hold = (cache.c, None) if isinstance(cache, Cache) else _host_cache(cache)
    dpsi = np.empty_like(dpsi_out)
    dv = np.empty((nl, 4, 4), np.complex128)
    hess = np.empty((16 * nl, 16 * nl), np.complex128)
    _check("brickwall_unitary_backward_hessian",
           lib().brickwall_unitary_backward_hessian(ptr(vlist), nl, C.cast(pp, VP), C.byref(c), C.byref(_sv(dpsi_out, L)),
                                                    C.byref(_sv(dpsi, L)), ptr(dv), ptr(hess)))
    return dpsi, dv, hess


def apply_brickwall_unitary_gate_placeholder(vlist, perms, l, cache):
    vlist = cplx(vlist)
    pp, keep = perm_pointers(perms)
    c, hold = (cache.c, None) if isinstance(cache, Cache) else _host_cache(cache)
    out = np.empty((1 << c.nqubits, 16), np.complex128)
    _check("apply_brickwall_unitary_gate_placeholder",
           lib().apply_brickwall_unitary_gate_placeholder(ptr(vlist), vlist.shape[0], C.cast(pp, VP), l, C.byref(c),
                                                          C.byref(_sva(out, c.nqubits))))
    return out


# ------------------------------------------------------------------------ targets

class Target:
    """A target U for the basis-column sums: a Python callable (host callback, one
    call per column), a device-native brickwall / circuit target, or a dense matrix
    (library host target: a basis column is a column copy)."""

    def __init__(self, fn=None, brickwall=None, circuit=None, dense=None):
        self._keep = []
        if dense is not None:
            u = cplx(dense)
            n = int(u.shape[0]).bit_length() - 1
            if u.ndim != 2 or u.shape[0] != u.shape[1] or 1 << n != u.shape[0]:
                raise ValueError("dense target must be a 2^n x 2^n matrix")
            self.desc = DenseTarget(u.ctypes.data, n)
            self._keep.append(u)
            self.ufunc = C.cast(lib().rqcopt_dense_ufunc, VP)
            self.udata = C.cast(C.pointer(self.desc), VP)
        elif fn is not None:
            self.cb = wrap_ufunc(fn)
            self.ufunc = C.cast(self.cb, VP)
            self.udata = None
        elif brickwall is not None:
            vlist, perms = brickwall
            vlist = cplx(vlist)
            pp, pk = perm_pointers(perms)
            self.desc = BrickwallTarget(vlist.ctypes.data, vlist.shape[0], pp)
            self._keep += [vlist, pp, pk]
            self.ufunc = C.cast(lib().rqcopt_brickwall_ufunc, VP)
            self.udata = C.cast(C.pointer(self.desc), VP)
        elif circuit is not None:
            gates, wires = cplx(circuit[0]), ints(circuit[1])
            self.desc = CircuitTarget(gates.ctypes.data, gates.shape[0], C.cast(wires.ctypes.data, C.POINTER(C.c_int)))
            self._keep += [gates, wires]
            self.ufunc = C.cast(lib().rqcopt_circuit_ufunc, VP)
            self.udata = C.cast(C.pointer(self.desc), VP)
        else:
            raise ValueError("target needs fn, brickwall or circuit")


def circuit_unitary_target(target, gates, wires, nqubits):
    gates, wires = cplx(gates), ints(wires)
    f = np.zeros(1, np.complex128)
    _check("circuit_unitary_target", lib().circuit_unitary_target(target.ufunc, target.udata, ptr(gates), gates.shape[0],
                                                                 ptr(wires), nqubits, ptr(f)))
    return f[0]


def circuit_unitary_target_and_gradient(target, gates, wires, nqubits):
    gates, wires = cplx(gates), ints(wires)
    f = np.zeros(1, np.complex128)
    dg = np.empty((gates.shape[0], 4, 4), np.complex128)
    _check("circuit_unitary_target_and_gradient",
           lib().circuit_unitary_target_and_gradient(target.ufunc, target.udata, ptr(gates), gates.shape[0], ptr(wires),
                                                     nqubits, ptr(f), ptr(dg)))
    return f[0], dg


def circuit_unitary_target_and_projected_gradient(target, gates, wires, nqubits):
    gates, wires = cplx(gates), ints(wires)
    f = np.zeros(1, np.complex128)
    g = np.empty(16 * gates.shape[0])
    _check("circuit_unitary_target_and_projected_gradient",
           lib().circuit_unitary_target_and_projected_gradient(target.ufunc, target.udata, ptr(gates), gates.shape[0],
                                                               ptr(wires), nqubits, ptr(f), ptr(g)))
    return f[0], g


def circuit_unitary_target_hessian_vector_product(target, gates, gatedirs, wires, nqubits):
    gates, gatedirs, wires = cplx(gates), cplx(gatedirs), ints(wires)
    f = np.zeros(1, np.complex128)
    dg = np.empty((gates.shape[0], 4, 4), np.complex128)
    hg = np.empty_like(dg)
    _check("circuit_unitary_target_hessian_vector_product",
           lib().circuit_unitary_target_hessian_vector_product(target.ufunc, target.udata, ptr(gates), ptr(gatedirs),
                                                               gates.shape[0], ptr(wires), nqubits, ptr(f), ptr(dg),
                                                               ptr(hg)))
    return f[0], dg, hg


def circuit_unitary_target_projected_hessian_vector_product(target, gates, gatedirs, wires, nqubits):
    gates, gatedirs, wires = cplx(gates), cplx(gatedirs), ints(wires)
    f = np.zeros(1, np.complex128)
    g = np.empty(16 * gates.shape[0])
    h = np.empty_like(g)
    _check("circuit_unitary_target_projected_hessian_vector_product",
           lib().circuit_unitary_target_projected_hessian_vector_product(target.ufunc, target.udata, ptr(gates),
                                                                         ptr(gatedirs), gates.shape[0], ptr(wires),
                                                                         nqubits, ptr(f), ptr(g), ptr(h)))
    return f[0], g, h


def brickwall_unitary_target(target, vlist, perms, nqubits):
    vlist = cplx(vlist)
    pp, keep = perm_pointers(perms)
    f = np.zeros(1, np.complex128)
    _check("brickwall_unitary_target", lib().brickwall_unitary_target(target.ufunc, target.udata, ptr(vlist),
                                                                     vlist.shape[0], nqubits, C.cast(pp, VP), ptr(f)))
    return f[0]


def brickwall_unitary_target_and_gradient(target, vlist, perms, nqubits):
    vlist = cplx(vlist)
    pp, keep = perm_pointers(perms)
    f = np.zeros(1, np.complex128)
    dv = np.empty((vlist.shape[0], 4, 4), np.complex128)
    _check("brickwall_unitary_target_and_gradient",
           lib().brickwall_unitary_target_and_gradient(target.ufunc, target.udata, ptr(vlist), vlist.shape[0], nqubits,
                                                       C.cast(pp, VP), ptr(f), ptr(dv)))
    return f[0], dv


def brickwall_unitary_target_and_projected_gradient(target, vlist, perms, nqubits):
    vlist = cplx(vlist)
    pp, keep = perm_pointers(perms)
    f = np.zeros(1, np.complex128)
    g = np.empty(16 * vlist.shape[0])
    _check("brickwall_unitary_target_and_projected_gradient",
           lib().brickwall_unitary_target_and_projected_gradient(target.ufunc, target.udata, ptr(vlist), vlist.shape[0],
                                                                 nqubits, C.cast(pp, VP), ptr(f), ptr(g)))
    return f[0], g


def brickwall_unitary_target_hessian_vector_product(target, vlist, vdirs, perms, nqubits):
    vlist, vdirs = cplx(vlist), cplx(vdirs)
    pp, keep = perm_pointers(perms)
    f = np.zeros(1, np.complex128)
    dv = np.empty((vlist.shape[0], 4, 4), np.complex128)
    hv = np.empty_like(dv)
    _check("brickwall_unitary_target_hessian_vector_product",
           lib().brickwall_unitary_target_hessian_vector_product(target.ufunc, target.udata, ptr(vlist), ptr(vdirs),
                                                                 vlist.shape[0], C.cast(pp, VP), nqubits, ptr(f), ptr(dv),
                                                                 ptr(hv)))
    return f[0], dv, hv


def brickwall_unitary_target_projected_hessian_vector_product(target, vlist, vdirs, perms, nqubits):
    vlist, vdirs = cplx(vlist), cplx(vdirs)
    pp, keep = perm_pointers(perms)
    f = np.zeros(1, np.complex128)
    g = np.empty(16 * vlist.shape[0])
    h = np.empty_like(g)
    _check("brickwall_unitary_target_projected_hessian_vector_product",
           lib().brickwall_unitary_target_projected_hessian_vector_product(target.ufunc, target.udata, ptr(vlist),
                                                                           ptr(vdirs), vlist.shape[0], C.cast(pp, VP),
                                                                           nqubits, ptr(f), ptr(g), ptr(h)))
    return f[0], g, h


def brickwall_unitary_target_gradient_hessian(target, vlist, perms, nqubits):
    """f, per-layer gradients and the complex (16 nlayers)^2 Hessian."""
    vlist = cplx(vlist)
    nl = vlist.shape[0]
    pp, keep = perm_pointers(perms)
    f = np.zeros(1, np.complex128)
    dv = np.empty((nl, 4, 4), np.complex128)
    hess = np.empty((16 * nl, 16 * nl), np.complex128)
    _check("brickwall_unitary_target_gradient_hessian",
           lib().brickwall_unitary_target_gradient_hessian(target.ufunc, target.udata, ptr(vlist), nl, nqubits,
                                                           C.cast(pp, VP), ptr(f), ptr(dv), ptr(hess)))
    return f[0], dv, hess


def brickwall_unitary_target_gradient_vector_hessian_matrix(target, vlist, perms, nqubits):
    """f, the Riemannian gradient vector and the real symmetric Hessian matrix."""
    vlist = cplx(vlist)
    nl = vlist.shape[0]
    pp, keep = perm_pointers(perms)
    f = np.zeros(1, np.complex128)
    g = np.empty(16 * nl)
    H = np.empty((16 * nl, 16 * nl))
    _check("brickwall_unitary_target_gradient_vector_hessian_matrix",
           lib().brickwall_unitary_target_gradient_vector_hessian_matrix(target.ufunc, target.udata, ptr(vlist), nl,
                                                                         nqubits, C.cast(pp, VP), ptr(f), ptr(g), ptr(H)))
    return f[0], g, H


# ------------------------------------------------------------------------ block-encoding target
# || P^dag W P - H ||_F^2 / 2 with H (`target`) acting on nqubits / 2 qubits.

def _blockenc(name, target, vlist, perms, nqubits, outs):
    vlist = cplx(vlist)
    pp, keep = perm_pointers(perms)
    f = np.zeros(1)
    _check(name, getattr(lib(), name)(target.ufunc, target.udata, ptr(vlist), vlist.shape[0], nqubits, C.cast(pp, VP),
                                      ptr(f), *[ptr(o) for o in outs]))
    return (f[0],) + tuple(outs)


def brickwall_blockenc_target(target, vlist, perms, nqubits):
    return _blockenc("brickwall_blockenc_target", target, vlist, perms, nqubits, [])[0]


def brickwall_blockenc_target_and_gradient(target, vlist, perms, nqubits):
    nl = np.shape(vlist)[0]
    return _blockenc("brickwall_blockenc_target_and_gradient", target, vlist, perms, nqubits,
                     [np.empty((nl, 4, 4), np.complex128)])


def brickwall_blockenc_target_and_gradient_vector(target, vlist, perms, nqubits):
    nl = np.shape(vlist)[0]
    return _blockenc("brickwall_blockenc_target_and_gradient_vector", target, vlist, perms, nqubits, [np.empty(16 * nl)])


def brickwall_blockenc_target_gradient_hessian(target, vlist, perms, nqubits):
    nl = np.shape(vlist)[0]
    m = 16 * nl
    return _blockenc("brickwall_blockenc_target_gradient_hessian", target, vlist, perms, nqubits,
                     [np.empty((nl, 4, 4), np.complex128), np.empty((m, m), np.complex128),
                      np.empty((m, m), np.complex128)])


def brickwall_blockenc_target_gradient_vector_hessian_matrix(target, vlist, perms, nqubits):
    nl = np.shape(vlist)[0]
    m = 16 * nl
    return _blockenc("brickwall_blockenc_target_gradient_vector_hessian_matrix", target, vlist, perms, nqubits,
                     [np.empty(m), np.empty((m, m))])


# ------------------------------------------------------------------------ sampling estimator
# Haar-random states drawn on the GPU from the reference's PCG32x2 stream; every call
# advances `rng` exactly as the reference's call does.

def seed_rng_state(seed: int) -> RngState:
    rng = RngState()
    lib().seed_rng_state(seed, C.byref(rng))
    return rng


def haar_random_statevector(nqubits, rng):
    out = np.empty(1 << nqubits, np.complex128)
    lib().haar_random_statevector(C.byref(_sv(out, nqubits)), C.byref(rng))
    _check_void("haar_random_statevector")
    return out


def circuit_unitary_target_sampling(target, gates, wires, nqubits, nsamples, rng):
    gates, wires = cplx(gates), ints(wires)
    f = np.zeros(1, np.complex128)
    _check("circuit_unitary_target_sampling",
           lib().circuit_unitary_target_sampling(target.ufunc, target.udata, ptr(gates), gates.shape[0], ptr(wires),
                                                 nqubits, nsamples, C.byref(rng), ptr(f)))
    return f[0]


def brickwall_unitary_target_sampling(target, vlist, perms, nqubits, nsamples, rng):
    vlist = cplx(vlist)
    pp, keep = perm_pointers(perms)
    f = np.zeros(1, np.complex128)
    _check("brickwall_unitary_target_sampling",
           lib().brickwall_unitary_target_sampling(target.ufunc, target.udata, ptr(vlist), vlist.shape[0], nqubits,
                                                   C.cast(pp, VP), nsamples, C.byref(rng), ptr(f)))
    return f[0]


def brickwall_unitary_target_gradient_hessian_sampling(target, vlist, perms, nqubits, nsamples, rng):
    vlist = cplx(vlist)
    nl = vlist.shape[0]
    pp, keep = perm_pointers(perms)
    f = np.zeros(1, np.complex128)
    dv = np.empty((nl, 4, 4), np.complex128)
    hess = np.empty((16 * nl, 16 * nl), np.complex128)
    _check("brickwall_unitary_target_gradient_hessian_sampling",
           lib().brickwall_unitary_target_gradient_hessian_sampling(target.ufunc, target.udata, ptr(vlist), nl, nqubits,
                                                                    C.cast(pp, VP), nsamples, C.byref(rng), ptr(f),
                                                                    ptr(dv), ptr(hess)))
    return f[0], dv, hess


def brickwall_unitary_target_gradient_vector_hessian_matrix_sampling(target, vlist, perms, nqubits, nsamples, rng):
    vlist = cplx(vlist)
    nl = vlist.shape[0]
    pp, keep = perm_pointers(perms)
    f = np.zeros(1, np.complex128)
    g = np.empty(16 * nl)
    H = np.empty((16 * nl, 16 * nl))
    _check("brickwall_unitary_target_gradient_vector_hessian_matrix_sampling",
           lib().brickwall_unitary_target_gradient_vector_hessian_matrix_sampling(
               target.ufunc, target.udata, ptr(vlist), nl, nqubits, C.cast(pp, VP), nsamples, C.byref(rng), ptr(f),
               ptr(g), ptr(H)))
    return f[0], g, H


def optimize_brickwall_circuit_hmat_sampling(target, vlist_start, perms, nqubits, nsamples, rng, niter, params=None):
    vlist_start = cplx(vlist_start)
    nl = vlist_start.shape[0]
    pp, keep = perm_pointers(perms)
    params = params or default_rtr_params(16 * nl)
    f_iter = np.empty(niter + 1)
    vopt = np.empty_like(vlist_start)
    lib().optimize_brickwall_circuit_hmat_sampling(target.ufunc, target.udata, ptr(vlist_start), nl, nqubits,
                                                   C.cast(pp, VP), nsamples, C.byref(rng), C.byref(params), niter,
                                                   ptr(f_iter), ptr(vopt))
    _check_void("optimize_brickwall_circuit_hmat_sampling")
    return f_iter, vopt


# ------------------------------------------------------------------------ trust region and optimisers

def truncated_cg_hmat(grad, hess, radius, params=None):
    grad = np.ascontiguousarray(grad, dtype=np.float64)
    hess = np.ascontiguousarray(hess, dtype=np.float64)
    n = grad.shape[0]
    params = params or default_tcg_params(n)
    z = np.empty(n)
    b = lib().truncated_cg_hmat(ptr(grad), ptr(hess), n, radius, C.byref(params), ptr(z))
    _check_void("truncated_cg_hmat")
    return z, bool(b)


def riemannian_trust_region_optimize_hmat(f, f_deriv_hess, retract_fn, n, x_init, niter, params=None):
    """RTR with Python callbacks f(x) -> float, f_deriv_hess(x) -> (f, grad, hess) and
    retract_fn(x, eta) -> x_new over real vectors x of length m."""
    x_init = np.ascontiguousarray(x_init, dtype=np.float64)
    m = x_init.shape[0]
    params = params or default_rtr_params(n)

    def cf(xp, fd):
        return float(f(np.ctypeslib.as_array(xp, shape=(m,)).copy()))

    def cfdh(xp, fd, g, h):
        fx, gv, hv = f_deriv_hess(np.ctypeslib.as_array(xp, shape=(m,)).copy())
        np.ctypeslib.as_array(g, shape=(n,))[:] = gv
        np.ctypeslib.as_array(h, shape=(n * n,))[:] = np.asarray(hv).ravel()
        return float(fx)

    def cr(xp, eta, rd, xs):
        np.ctypeslib.as_array(xs, shape=(m,))[:] = retract_fn(np.ctypeslib.as_array(xp, shape=(m,)).copy(),
                                                             np.ctypeslib.as_array(eta, shape=(n,)).copy())

    fcb, dcb, rcb = TARGET_FUNC(cf), TARGET_GRAD_HESS_FUNC(cfdh), RETRACT_FUNC(cr)
    f_iter = np.empty(niter + 1)
    x_final = np.empty(m)
    lib().riemannian_trust_region_optimize_hmat(C.cast(fcb, VP), C.cast(dcb, VP), None, C.cast(rcb, VP), None, n,
                                                ptr(x_init), m, C.byref(params), niter, ptr(f_iter), ptr(x_final))
    _check_void("riemannian_trust_region_optimize_hmat")
    return f_iter, x_final


def optimize_brickwall_circuit_hmat(target, vlist_start, perms, nqubits, niter, params=None):
    vlist_start = cplx(vlist_start)
    nl = vlist_start.shape[0]
    pp, keep = perm_pointers(perms)
    params = params or default_rtr_params(16 * nl)
    f_iter = np.empty(niter + 1)
    vopt = np.empty_like(vlist_start)
    lib().optimize_brickwall_circuit_hmat(target.ufunc, target.udata, ptr(vlist_start), nl, nqubits, C.cast(pp, VP),
                                          C.byref(params), niter, ptr(f_iter), ptr(vopt))
    _check_void("optimize_brickwall_circuit_hmat")
    return f_iter, vopt


def truncated_cg_hvp(grad, hvp_fn, radius, params=None, x=None):
    """Steihaug tCG with a Python Hessian-vector product `hvp_fn(vec) -> H vec`."""
    grad = np.ascontiguousarray(grad, dtype=np.float64)
    n = grad.shape[0]
    params = params or default_tcg_params(n)

    def cb(xp, fdata, vec, hvp):
        v = np.ctypeslib.as_array(vec, shape=(n,))
        h = np.ctypeslib.as_array(hvp, shape=(n,))
        h[:] = hvp_fn(v.copy())

    f_hvp = HVP_FUNC(cb)
    z = np.empty(n)
    xv = ptr(np.ascontiguousarray(x, dtype=np.float64)) if x is not None else None
    b = lib().truncated_cg_hvp(xv, ptr(grad), C.cast(f_hvp, VP), None, n, radius, C.byref(params), ptr(z))
    _check_void("truncated_cg_hvp")
    return z, bool(b)


def optimize_brickwall_circuit_hvp(target, vlist_start, perms, nqubits, niter, params=None):
    vlist_start = cplx(vlist_start)
    nl = vlist_start.shape[0]
    pp, keep = perm_pointers(perms)
    params = params or default_rtr_params(16 * nl)
    f_iter = np.empty(niter + 1)
    vopt = np.empty_like(vlist_start)
    lib().optimize_brickwall_circuit_hvp(target.ufunc, target.udata, ptr(vlist_start), nl, nqubits, C.cast(pp, VP),
                                         C.byref(params), niter, ptr(f_iter), ptr(vopt))
    _check_void("optimize_brickwall_circuit_hvp")
    return f_iter, vopt


def optimize_quantum_circuit(target, gates_start, wires, nqubits, niter, params=None):
    gates_start, wires = cplx(gates_start), ints(wires)
    ng = gates_start.shape[0]
    params = params or default_rtr_params(16 * ng)
    f_iter = np.empty(niter + 1)
    gopt = np.empty_like(gates_start)
    lib().optimize_quantum_circuit(target.ufunc, target.udata, ptr(gates_start), ng, nqubits, ptr(wires),
                                   C.byref(params), niter, ptr(f_iter), ptr(gopt))
    _check_void("optimize_quantum_circuit")
    return f_iter, gopt


# ------------------------------------------------------------------------ matrix helpers

def real_to_tangent(r, v):
    r, v = np.ascontiguousarray(r, dtype=np.float64), cplx(v)
    z = np.empty((4, 4), np.complex128)
    lib().real_to_tangent(ptr(r), ptr(v), ptr(z))
    return z


def tangent_to_real(v, z):
    v, z = cplx(v), cplx(z)
    r = np.empty(16)
    lib().tangent_to_real(ptr(v), ptr(z), ptr(r))
    return r


def project_tangent(u, z):
    u, z = cplx(u), cplx(z)
    p = np.empty((4, 4), np.complex128)
    lib().project_tangent(ptr(u), ptr(z), ptr(p))
    return p


def polar_factor(a):
    a = cplx(a)
    u = np.empty((4, 4), np.complex128)
    lib().polar_factor(ptr(a), ptr(u))
    return u


def multiply_matrices(a, b):
    a, b = cplx(a), cplx(b)
    c = np.empty((4, 4), np.complex128)
    lib().multiply_matrices(ptr(a), ptr(b), ptr(c))
    return c


def retract(u, eta):
    """Polar retraction of the unitary u along the tangent vector given by 16 reals (src/matrix.c:517-531)."""
    u, eta = cplx(u), np.ascontiguousarray(eta, dtype=np.float64)
    v = np.empty((4, 4), np.complex128)
    lib().retract(ptr(u), ptr(eta), ptr(v))
    return v


def inverse_matrix(a):
    a = cplx(a)
    ai = np.empty((4, 4), np.complex128)
    ret = lib().inverse_matrix(ptr(a), ptr(ai))
    return ret, ai


# ------------------------------------------------------------------------ configuration

def set_precision(mode: int):
    _check("rqcopt_gpu_set_precision", lib().rqcopt_gpu_set_precision(mode))


def set_gates_per_pass(k: int):
    _check("rqcopt_gpu_set_gates_per_pass", lib().rqcopt_gpu_set_gates_per_pass(k))


def set_autotune(on: bool):
    """Autotuning of the basis-column sums (on by default); turning it on also releases the
    settings fixed by set_gates_per_pass / set_column_chunk / set_reconstruct."""
    _check("rqcopt_gpu_set_autotune", lib().rqcopt_gpu_set_autotune(1 if on else 0))


def last_config():
    """Configuration of the last target evaluation: gates per pass, column chunk (0: from
    the workspace), reconstruction, sample ms per column and whether the autotuner chose it."""
    g, r, f = C.c_int(), C.c_int(), C.c_int()
    ch, ms = C.c_long(), C.c_double()
    tuned = lib().rqcopt_gpu_last_config(C.byref(g), C.byref(ch), C.byref(r), C.byref(f), C.byref(ms))
    if tuned < 0:
        raise RqcError("rqcopt_gpu_last_config", tuned)
    return {"gates_per_pass": g.value, "column_chunk": ch.value, "reconstruct": bool(r.value),
            "c64_fp32_pipe": bool(f.value), "ms_per_column": ms.value, "tuned": bool(tuned)}


def set_c64_fp32_pipe(on: bool):
    """complex64 fused passes in FP32 FMAs (True) or on the TF32 MMA (False)."""
    lib().rqcopt_gpu_set_c64_fp32_pipe(1 if on else 0)


def set_reconstruct(on: bool):
    """complex128 reverse passes rebuild states with adjoint gates (True) or recompute them (False)."""
    lib().rqcopt_gpu_set_reconstruct(1 if on else 0)


def set_column_chunk(cols: int):
    lib().rqcopt_gpu_set_column_chunk(cols)


def optimizer_trace():
    """Per-iteration (accepted, on_boundary, tcg_inner_iterations, refined) arrays of the
    last Hessian-vector-product optimisation on this device."""
    n = lib().rqcopt_gpu_optimizer_trace(None, None, None, None, 0)
    if n < 0:
        raise RqcError("rqcopt_gpu_optimizer_trace", n)
    a, b, c, d = (np.zeros(n, np.int32) for _ in range(4))
    lib().rqcopt_gpu_optimizer_trace(a.ctypes.data, b.ctypes.data, c.ctypes.data, d.ctypes.data, n)
    return {"accepted": a, "on_boundary": b, "inner": c, "refined": d}


def set_column_range(begin: int = 0, end: int = 0):
    """Restrict the target functions' basis-column sums to [begin, end) (end 0: to the last column)."""
    _check("rqcopt_gpu_set_column_range", lib().rqcopt_gpu_set_column_range(begin, end))


def set_workspace_limit(nbytes: int):
    lib().rqcopt_gpu_set_workspace_limit(nbytes)


def launch_count() -> int:
    return int(lib().rqcopt_gpu_launch_count())


def reset_launch_count():
    lib().rqcopt_gpu_reset_launch_count()


def enable_kernel_timing(on: bool):
    lib().rqcopt_gpu_enable_kernel_timing(1 if on else 0)


def kernel_time(kernel_class: int):
    ms = C.c_double()
    n = C.c_long()
    _check("rqcopt_gpu_kernel_time", lib().rqcopt_gpu_kernel_time(kernel_class, C.byref(ms), C.byref(n)))
    return ms.value, n.value
