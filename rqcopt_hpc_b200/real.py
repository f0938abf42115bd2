"""Python host mirror of the reference's real-orthogonal build (compiled without
COMPLEX_CIRCUIT), calling librqcopt_gpu_real.so through its C ABI
(include/rqcopt_gpu_real.h).

Function names, arguments and return values are those of ``rqcopt_hpc_b200.gpu``
with real arrays: statevectors and gates are numpy float64, a tangent direction of
a gate has 6 real parameters (src/matrix.c:245-271, 288-300), and the functions the
real build does not have (the full-Hessian matrix forms, their optimisers, the
block-encoding gradient vector) are absent.  Loading fails loudly when the library
is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .abi import (HVP_FUNC, LINEAR_FUNC, BrickwallTarget, CircuitTarget, DenseTarget, QuantumCircuitCache, RngState,
                  Statevector, StatevectorArray, default_rtr_params, default_tcg_params, ints, perm_pointers, ptr)

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "librqcopt_gpu_real.so")
NTAN = 6

_lib = None
VP = C.c_void_p


class RqcError(RuntimeError):
    def __init__(self, fn, code):
        super().__init__(f"{fn} failed with code {code}")
        self.code = code


_VOID = {"free_statevector", "add_statevectors", "transpose_statevector", "apply_gate", "apply_gate_backward", "apply_gate_to_array",
         "apply_gate_backward_array", "apply_gate_placeholder", "free_quantum_circuit_cache", "seed_rng_state",
         "haar_random_statevector", "free_statevector_array", "optimize_brickwall_circuit_hvp",
         "optimize_quantum_circuit", "riemannian_trust_region_optimize_hvp", "riemannian_trust_region_optimize_hmat",
         "real_to_tangent", "tangent_to_real", "project_tangent", "polar_factor", "multiply_matrices", "retract",
         "real_to_antisymm", "antisymm_to_real", "rqcopt_gpu_reset_launch_count"}


def lib():
    """The loaded real-build library (raises OSError if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} not found: build it with `python -m rqcopt_hpc_b200.build`")
        L = C.CDLL(LIB_PATH)
        L.truncated_cg_hvp.restype = C.c_bool
        L.truncated_cg_hmat.restype = C.c_bool
        L.rqcopt_gpu_launch_count.restype = C.c_ulonglong
        L.seed_rng_state.argtypes = [C.c_uint64, C.POINTER(RngState)]
        for name in _VOID:
            getattr(L, name).restype = None
        _lib = L
    return _lib


def _call(name, *args):
    ret = getattr(lib(), name)(*args)
    if ret != 0:
        raise RqcError(name, ret)


def _void(name, *args):
    getattr(lib(), name)(*args)
    err = lib().rqcopt_gpu_last_error()
    if err != 0:
        raise RqcError(name, err)


def real(a) -> np.ndarray:
    a = np.asarray(a)
    if np.iscomplexobj(a):
        if np.any(a.imag != 0):
            raise TypeError("the real build takes real arrays")
        a = a.real
    return np.ascontiguousarray(a, dtype=np.float64)


def _nq(psi):
    L = int(psi.shape[0]).bit_length() - 1
    assert 1 << L == psi.shape[0], "statevector length must be a power of two"
    return L


def _sv(a, L):
    return C.byref(Statevector(a.ctypes.data, L))


def _sva(a, L):
    return C.byref(StatevectorArray(a.ctypes.data, L, a.shape[1]))


# ------------------------------------------------------------------------ gates and circuits

def transpose_statevector(psi, perm):
    psi, perm = real(psi), ints(perm)
    L = _nq(psi)
    out = np.empty_like(psi)
    _void("transpose_statevector", _sv(psi, L), ptr(perm), _sv(out, L))
    return out


def apply_gate(V, i, j, psi):
    V, psi = real(V), real(psi)
    L = _nq(psi)
    out = np.empty_like(psi)
    _void("apply_gate", ptr(V), i, j, _sv(psi, L), _sv(out, L))
    return out


def apply_gate_backward(V, i, j, psi, dpsi_out):
    V, psi, dpsi_out = real(V), real(psi), real(dpsi_out)
    L = _nq(psi)
    dpsi, dV = np.empty_like(psi), np.empty((4, 4))
    _void("apply_gate_backward", ptr(V), i, j, _sv(psi, L), _sv(dpsi_out, L), _sv(dpsi, L), ptr(dV))
    return dpsi, dV


def apply_quantum_circuit(gates, wires, psi):
    gates, wires, psi = real(gates), ints(wires), real(psi)
    L = _nq(psi)
    out = np.empty_like(psi)
    _call("apply_quantum_circuit", ptr(gates), gates.shape[0], ptr(wires), _sv(psi, L), _sv(out, L))
    return out


class Cache:
    """quantum_circuit_cache of the real library (host memory states)."""

    def __init__(self, nqubits, ngates):
        self.c = QuantumCircuitCache()
        _call("allocate_quantum_circuit_cache", nqubits, ngates, C.byref(self.c))

    def state(self, k):
        s = self.c.psi_list[k]
        return np.ctypeslib.as_array(C.cast(s.data, C.POINTER(C.c_double)), shape=(1 << s.nqubits,)).copy()

    def __del__(self):
        if _lib is not None and self.c.psi_list:
            _lib.free_quantum_circuit_cache(C.byref(self.c))


def quantum_circuit_forward(gates, wires, psi):
    gates, wires, psi = real(gates), ints(wires), real(psi)
    L = _nq(psi)
    cache, out = Cache(L, gates.shape[0]), np.empty_like(psi)
    _call("quantum_circuit_forward", ptr(gates), gates.shape[0], ptr(wires), _sv(psi, L), C.byref(cache.c), _sv(out, L))
    return out, cache


def quantum_circuit_backward(gates, wires, cache, dpsi_out):
    gates, wires, dpsi_out = real(gates), ints(wires), real(dpsi_out)
    L = _nq(dpsi_out)
    dpsi, dg = np.empty_like(dpsi_out), np.empty((gates.shape[0], 4, 4))
    _call("quantum_circuit_backward", ptr(gates), gates.shape[0], ptr(wires), C.byref(cache.c), _sv(dpsi_out, L),
          _sv(dpsi, L), ptr(dg))
    return dpsi, dg


def quantum_circuit_gates_hessian_vector_product(gates, gatedirs, wires, psi, phi):
    gates, gatedirs, wires, psi, phi = real(gates), real(gatedirs), ints(wires), real(psi), real(phi)
    L = _nq(psi)
    out, dg = np.empty_like(psi), np.empty((gates.shape[0], 4, 4))
    hg = np.empty_like(dg)
    _call("quantum_circuit_gates_hessian_vector_product", ptr(gates), ptr(gatedirs), gates.shape[0], ptr(wires),
          _sv(psi, L), _sv(phi, L), _sv(out, L), ptr(dg), ptr(hg))
    return out, dg, hg


def apply_brickwall_unitary(vlist, perms, psi):
    vlist, psi = real(vlist), real(psi)
    L = _nq(psi)
    pp, keep = perm_pointers(perms)
    out = np.empty_like(psi)
    _call("apply_brickwall_unitary", ptr(vlist), vlist.shape[0], C.cast(pp, VP), _sv(psi, L), _sv(out, L))
    return out


def brickwall_unitary_forward(vlist, perms, psi):
    vlist, psi = real(vlist), real(psi)
    L = _nq(psi)
    pp, keep = perm_pointers(perms)
    cache, out = Cache(L, vlist.shape[0] * (L // 2)), np.empty_like(psi)
    _call("brickwall_unitary_forward", ptr(vlist), vlist.shape[0], C.cast(pp, VP), _sv(psi, L), C.byref(cache.c),
          _sv(out, L))
    return out, cache


def brickwall_unitary_backward(vlist, perms, cache, dpsi_out):
    vlist, dpsi_out = real(vlist), real(dpsi_out)
    L = _nq(dpsi_out)
    pp, keep = perm_pointers(perms)
    dpsi, dv = np.empty_like(dpsi_out), np.empty((vlist.shape[0], 4, 4))
    _call("brickwall_unitary_backward", ptr(vlist), vlist.shape[0], C.cast(pp, VP), C.byref(cache.c), _sv(dpsi_out, L),
          _sv(dpsi, L), ptr(dv))
    return dpsi, dv


def brickwall_unitary_backward_hessian(vlist, perms, cache, dpsi_out):
    vlist, dpsi_out = real(vlist), real(dpsi_out)
    L, nl = _nq(dpsi_out), vlist.shape[0]
    pp, keep = perm_pointers(perms)
    dpsi, dv, hess = np.empty_like(dpsi_out), np.empty((nl, 4, 4)), np.empty((16 * nl, 16 * nl))
    _call("brickwall_unitary_backward_hessian", ptr(vlist), nl, C.cast(pp, VP), C.byref(cache.c), _sv(dpsi_out, L),
          _sv(dpsi, L), ptr(dv), ptr(hess))
    return dpsi, dv, hess


def apply_gate_to_array(V, i, j, psi):
    V, psi = real(V), real(psi)
    L = _nq(psi)
    out = np.empty_like(psi)
    _void("apply_gate_to_array", ptr(V), i, j, _sva(psi, L), _sva(out, L))
    return out


def apply_gate_backward_array(V, i, j, psi, dpsi_out):
    V, psi, dpsi_out = real(V), real(psi), real(dpsi_out)
    L = _nq(psi)
    dg = np.empty((psi.shape[1], 4, 4))
    _void("apply_gate_backward_array", ptr(V), i, j, _sva(psi, L), _sv(dpsi_out, L), ptr(dg))
    return dg


def apply_gate_placeholder(i, j, psi):
    psi = real(psi)
    L = _nq(psi)
    out = np.empty((1 << L, 16))
    _void("apply_gate_placeholder", i, j, _sv(psi, L), _sva(out, L))
    return out


def apply_brickwall_unitary_gate_placeholder(vlist, perms, l, cache):
    vlist = real(vlist)
    pp, keep = perm_pointers(perms)
    L = cache.c.nqubits
    out = np.empty((1 << L, 16))
    _call("apply_brickwall_unitary_gate_placeholder", ptr(vlist), vlist.shape[0], C.cast(pp, VP), l, C.byref(cache.c),
          _sva(out, L))
    return out


# ------------------------------------------------------------------------ targets

def _wrap_real_ufunc(fn):
    def cb(psi_p, udata, out_p):
        try:
            psi, out = psi_p.contents, out_p.contents
            n = 1 << psi.nqubits
            x = np.ctypeslib.as_array(C.cast(psi.data, C.POINTER(C.c_double)), shape=(n,))
            y = np.ctypeslib.as_array(C.cast(out.data, C.POINTER(C.c_double)), shape=(n,))
            y[:] = fn(x.copy())
            return 0
        except Exception:
            return -1

    return LINEAR_FUNC(cb)


class Target:
    """A real target: a Python callable (one call per column), a device-native brickwall
    or circuit of real gates, or a dense real matrix."""

    def __init__(self, fn=None, brickwall=None, circuit=None, dense=None):
        self._keep = []
        if dense is not None:
            u = real(dense)
            n = int(u.shape[0]).bit_length() - 1
            if u.ndim != 2 or u.shape[0] != u.shape[1] or 1 << n != u.shape[0]:
                raise ValueError("dense target must be a 2^n x 2^n matrix")
            self.desc = DenseTarget(u.ctypes.data, n)
            self._keep.append(u)
            self.ufunc = C.cast(lib().rqcopt_dense_ufunc, VP)
            self.udata = C.cast(C.pointer(self.desc), VP)
        elif fn is not None:
            self.cb = _wrap_real_ufunc(fn)
            self.ufunc, self.udata = C.cast(self.cb, VP), None
        elif brickwall is not None:
            vlist = real(brickwall[0])
            pp, pk = perm_pointers(brickwall[1])
            self.desc = BrickwallTarget(vlist.ctypes.data, vlist.shape[0], pp)
            self._keep += [vlist, pp, pk]
            self.ufunc = C.cast(lib().rqcopt_brickwall_ufunc, VP)
            self.udata = C.cast(C.pointer(self.desc), VP)
        elif circuit is not None:
            gates, wires = real(circuit[0]), ints(circuit[1])
            self.desc = CircuitTarget(gates.ctypes.data, gates.shape[0], C.cast(wires.ctypes.data, C.POINTER(C.c_int)))
            self._keep += [gates, wires]
            self.ufunc = C.cast(lib().rqcopt_circuit_ufunc, VP)
            self.udata = C.cast(C.pointer(self.desc), VP)
        else:
            raise ValueError("target needs fn, brickwall, circuit or dense")


def _f():
    return np.zeros(1)


def circuit_unitary_target(target, gates, wires, nqubits):
    gates, wires, f = real(gates), ints(wires), _f()
    _call("circuit_unitary_target", target.ufunc, target.udata, ptr(gates), gates.shape[0], ptr(wires), nqubits, ptr(f))
    return f[0]


def circuit_unitary_target_and_gradient(target, gates, wires, nqubits):
    gates, wires, f = real(gates), ints(wires), _f()
    dg = np.empty((gates.shape[0], 4, 4))
    _call("circuit_unitary_target_and_gradient", target.ufunc, target.udata, ptr(gates), gates.shape[0], ptr(wires),
          nqubits, ptr(f), ptr(dg))
    return f[0], dg


def circuit_unitary_target_and_projected_gradient(target, gates, wires, nqubits):
    gates, wires, f = real(gates), ints(wires), _f()
    g = np.empty(NTAN * gates.shape[0])
    _call("circuit_unitary_target_and_projected_gradient", target.ufunc, target.udata, ptr(gates), gates.shape[0],
          ptr(wires), nqubits, ptr(f), ptr(g))
    return f[0], g


def circuit_unitary_target_hessian_vector_product(target, gates, gatedirs, wires, nqubits):
    gates, gatedirs, wires, f = real(gates), real(gatedirs), ints(wires), _f()
    dg = np.empty((gates.shape[0], 4, 4))
    hg = np.empty_like(dg)
    _call("circuit_unitary_target_hessian_vector_product", target.ufunc, target.udata, ptr(gates), ptr(gatedirs),
          gates.shape[0], ptr(wires), nqubits, ptr(f), ptr(dg), ptr(hg))
    return f[0], dg, hg


def circuit_unitary_target_projected_hessian_vector_product(target, gates, gatedirs, wires, nqubits):
    gates, gatedirs, wires, f = real(gates), real(gatedirs), ints(wires), _f()
    g, h = np.empty(NTAN * gates.shape[0]), np.empty(NTAN * gates.shape[0])
    _call("circuit_unitary_target_projected_hessian_vector_product", target.ufunc, target.udata, ptr(gates),
          ptr(gatedirs), gates.shape[0], ptr(wires), nqubits, ptr(f), ptr(g), ptr(h))
    return f[0], g, h


def brickwall_unitary_target(target, vlist, perms, nqubits):
    vlist, f = real(vlist), _f()
    pp, keep = perm_pointers(perms)
    _call("brickwall_unitary_target", target.ufunc, target.udata, ptr(vlist), vlist.shape[0], nqubits, C.cast(pp, VP),
          ptr(f))
    return f[0]


def brickwall_unitary_target_and_gradient(target, vlist, perms, nqubits):
    vlist, f = real(vlist), _f()
    pp, keep = perm_pointers(perms)
    dv = np.empty((vlist.shape[0], 4, 4))
    _call("brickwall_unitary_target_and_gradient", target.ufunc, target.udata, ptr(vlist), vlist.shape[0], nqubits,
          C.cast(pp, VP), ptr(f), ptr(dv))
    return f[0], dv


def brickwall_unitary_target_and_projected_gradient(target, vlist, perms, nqubits):
    vlist, f = real(vlist), _f()
    pp, keep = perm_pointers(perms)
    g = np.empty(NTAN * vlist.shape[0])
    _call("brickwall_unitary_target_and_projected_gradient", target.ufunc, target.udata, ptr(vlist), vlist.shape[0],
          nqubits, C.cast(pp, VP), ptr(f), ptr(g))
    return f[0], g


def brickwall_unitary_target_hessian_vector_product(target, vlist, vdirs, perms, nqubits):
    vlist, vdirs, f = real(vlist), real(vdirs), _f()
    pp, keep = perm_pointers(perms)
    dv = np.empty((vlist.shape[0], 4, 4))
    hv = np.empty_like(dv)
    _call("brickwall_unitary_target_hessian_vector_product", target.ufunc, target.udata, ptr(vlist), ptr(vdirs),
          vlist.shape[0], C.cast(pp, VP), nqubits, ptr(f), ptr(dv), ptr(hv))
    return f[0], dv, hv


def brickwall_unitary_target_projected_hessian_vector_product(target, vlist, vdirs, perms, nqubits):
    vlist, vdirs, f = real(vlist), real(vdirs), _f()
    pp, keep = perm_pointers(perms)
    g, h = np.empty(NTAN * vlist.shape[0]), np.empty(NTAN * vlist.shape[0])
    _call("brickwall_unitary_target_projected_hessian_vector_product", target.ufunc, target.udata, ptr(vlist),
          ptr(vdirs), vlist.shape[0], C.cast(pp, VP), nqubits, ptr(f), ptr(g), ptr(h))
    return f[0], g, h


def brickwall_unitary_target_gradient_hessian(target, vlist, perms, nqubits):
    vlist, f = real(vlist), _f()
    nl = vlist.shape[0]
    pp, keep = perm_pointers(perms)
    dv, hess = np.empty((nl, 4, 4)), np.empty((16 * nl, 16 * nl))
    _call("brickwall_unitary_target_gradient_hessian", target.ufunc, target.udata, ptr(vlist), nl, nqubits,
          C.cast(pp, VP), ptr(f), ptr(dv), ptr(hess))
    return f[0], dv, hess


def brickwall_blockenc_target(target, vlist, perms, nqubits):
    vlist, f = real(vlist), _f()
    pp, keep = perm_pointers(perms)
    _call("brickwall_blockenc_target", target.ufunc, target.udata, ptr(vlist), vlist.shape[0], nqubits, C.cast(pp, VP),
          ptr(f))
    return f[0]


def brickwall_blockenc_target_and_gradient(target, vlist, perms, nqubits):
    vlist, f = real(vlist), _f()
    pp, keep = perm_pointers(perms)
    dv = np.empty((vlist.shape[0], 4, 4))
    _call("brickwall_blockenc_target_and_gradient", target.ufunc, target.udata, ptr(vlist), vlist.shape[0], nqubits,
          C.cast(pp, VP), ptr(f), ptr(dv))
    return f[0], dv


def brickwall_blockenc_target_gradient_hessian(target, vlist, perms, nqubits):
    vlist, f = real(vlist), _f()
    nl = vlist.shape[0]
    pp, keep = perm_pointers(perms)
    dv, hess = np.empty((nl, 4, 4)), np.empty((16 * nl, 16 * nl))
    _call("brickwall_blockenc_target_gradient_hessian", target.ufunc, target.udata, ptr(vlist), nl, nqubits,
          C.cast(pp, VP), ptr(f), ptr(dv), ptr(hess))
    return f[0], dv, hess


# ------------------------------------------------------------------------ sampling

def seed_rng_state(seed: int) -> RngState:
    rng = RngState()
    lib().seed_rng_state(seed, C.byref(rng))
    return rng


def haar_random_statevector(nqubits, rng):
    out = np.empty(1 << nqubits)
    _void("haar_random_statevector", _sv(out, nqubits), C.byref(rng))
    return out


def circuit_unitary_target_sampling(target, gates, wires, nqubits, nsamples, rng):
    gates, wires, f = real(gates), ints(wires), _f()
    _call("circuit_unitary_target_sampling", target.ufunc, target.udata, ptr(gates), gates.shape[0], ptr(wires), nqubits,
          C.c_long(nsamples), C.byref(rng), ptr(f))
    return f[0]


def brickwall_unitary_target_sampling(target, vlist, perms, nqubits, nsamples, rng):
    vlist, f = real(vlist), _f()
    pp, keep = perm_pointers(perms)
    _call("brickwall_unitary_target_sampling", target.ufunc, target.udata, ptr(vlist), vlist.shape[0], nqubits,
          C.cast(pp, VP), C.c_long(nsamples), C.byref(rng), ptr(f))
    return f[0]


def brickwall_unitary_target_gradient_hessian_sampling(target, vlist, perms, nqubits, nsamples, rng):
    vlist, f = real(vlist), _f()
    nl = vlist.shape[0]
    pp, keep = perm_pointers(perms)
    dv, hess = np.empty((nl, 4, 4)), np.empty((16 * nl, 16 * nl))
    _call("brickwall_unitary_target_gradient_hessian_sampling", target.ufunc, target.udata, ptr(vlist), nl, nqubits,
          C.cast(pp, VP), C.c_long(nsamples), C.byref(rng), ptr(f), ptr(dv), ptr(hess))
    return f[0], dv, hess


# ------------------------------------------------------------------------ trust region and optimisers

def truncated_cg_hvp(grad, hvp_fn, radius, params=None, x=None):
    grad = np.ascontiguousarray(grad, dtype=np.float64)
    n = grad.shape[0]
    params = params or default_tcg_params(n)

    def cb(xp, fdata, vec, hvp):
        np.ctypeslib.as_array(hvp, shape=(n,))[:] = hvp_fn(np.ctypeslib.as_array(vec, shape=(n,)).copy())

    f_hvp = HVP_FUNC(cb)
    z = np.empty(n)
    xv = ptr(np.ascontiguousarray(x, dtype=np.float64)) if x is not None else None
    b = lib().truncated_cg_hvp(xv, ptr(grad), C.cast(f_hvp, VP), None, n, C.c_double(radius), C.byref(params), ptr(z))
    return z, bool(b)


def truncated_cg_hmat(grad, hess, radius, params=None):
    grad, hess = np.ascontiguousarray(grad, dtype=np.float64), np.ascontiguousarray(hess, dtype=np.float64)
    n = grad.shape[0]
    params = params or default_tcg_params(n)
    z = np.empty(n)
    b = lib().truncated_cg_hmat(ptr(grad), ptr(hess), n, C.c_double(radius), C.byref(params), ptr(z))
    return z, bool(b)


def optimize_brickwall_circuit_hvp(target, vlist_start, perms, nqubits, niter, params=None):
    vlist_start = real(vlist_start)
    nl = vlist_start.shape[0]
    pp, keep = perm_pointers(perms)
    params = params or default_rtr_params(NTAN * nl)
    f_iter, vopt = np.empty(niter + 1), np.empty_like(vlist_start)
    _void("optimize_brickwall_circuit_hvp", target.ufunc, target.udata, ptr(vlist_start), nl, nqubits, C.cast(pp, VP),
          C.byref(params), niter, ptr(f_iter), ptr(vopt))
    return f_iter, vopt


def optimize_quantum_circuit(target, gates_start, wires, nqubits, niter, params=None):
    gates_start, wires = real(gates_start), ints(wires)
    ng = gates_start.shape[0]
    params = params or default_rtr_params(NTAN * ng)
    f_iter, gopt = np.empty(niter + 1), np.empty_like(gates_start)
    _void("optimize_quantum_circuit", target.ufunc, target.udata, ptr(gates_start), ng, nqubits, ptr(wires),
          C.byref(params), niter, ptr(f_iter), ptr(gopt))
    return f_iter, gopt


# ------------------------------------------------------------------------ matrix helpers (real build)

def real_to_antisymm(r):
    r, w = np.ascontiguousarray(r, dtype=np.float64), np.empty((4, 4))
    lib().real_to_antisymm(ptr(r), ptr(w))
    return w


def antisymm_to_real(w):
    w, r = real(w), np.empty(NTAN)
    lib().antisymm_to_real(ptr(w), ptr(r))
    return r


def real_to_tangent(r, v):
    r, v, z = np.ascontiguousarray(r, dtype=np.float64), real(v), np.empty((4, 4))
    lib().real_to_tangent(ptr(r), ptr(v), ptr(z))
    return z


def tangent_to_real(v, z):
    v, z, r = real(v), real(z), np.empty(NTAN)
    lib().tangent_to_real(ptr(v), ptr(z), ptr(r))
    return r


def project_tangent(u, z):
    u, z, p = real(u), real(z), np.empty((4, 4))
    lib().project_tangent(ptr(u), ptr(z), ptr(p))
    return p


def polar_factor(a):
    a, u = real(a), np.empty((4, 4))
    _void("polar_factor", ptr(a), ptr(u))
    return u


def multiply_matrices(a, b):
    a, b, c = real(a), real(b), np.empty((4, 4))
    lib().multiply_matrices(ptr(a), ptr(b), ptr(c))
    return c


def retract(u, eta):
    u, eta, v = real(u), np.ascontiguousarray(eta, dtype=np.float64), np.empty((4, 4))
    _void("retract", ptr(u), ptr(eta), ptr(v))
    return v


def launch_count() -> int:
    return int(lib().rqcopt_gpu_launch_count())


def reset_launch_count():
    lib().rqcopt_gpu_reset_launch_count()
