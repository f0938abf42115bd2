"""ctypes wrappers of the CPU checkers.  TEST INFRASTRUCTURE ONLY.

``Oracle`` wraps ``_build/librqc_oracle.so`` (the plain-C restatement in
rqc_oracle.c) and ``Reference`` wraps ``_ref/librqcopt_ref.so`` (the reference
sources compiled by the Makefile in this folder).  Only the tests, the smoke
check and the CPU-baseline leg of the benchmark use them, as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "librqc_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "librqcopt_ref.so")

VP, I, D, L_ = C.c_void_p, C.c_int, C.c_double, C.c_long


class SV(C.Structure):
    _fields_ = [("data", C.c_void_p), ("nqubits", C.c_int)]


class TcgParams(C.Structure):
    _fields_ = [("maxiter", C.c_int), ("abstol", C.c_double), ("reltol", C.c_double)]


class RtrParams(C.Structure):
    _fields_ = [("tcg", TcgParams), ("rho_trust", C.c_double), ("radius_init", C.c_double), ("maxradius", C.c_double)]


class Pcg32(C.Structure):
    _fields_ = [("state", C.c_uint64), ("inc", C.c_uint64)]


class RngState(C.Structure):
    """struct rng_state (src/rng.h:15-18): two PCG32 generators."""
    _fields_ = [("gen", Pcg32 * 2)]

    def tuple(self):
        return tuple((g.state, g.inc) for g in self.gen)


class BrickwallUdata(C.Structure):
    _fields_ = [("vlist", C.c_void_p), ("nlayers", C.c_int), ("perms", C.c_void_p)]


HVP_FUNC = C.CFUNCTYPE(None, C.POINTER(C.c_double), C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double))
LINEAR_FUNC = C.CFUNCTYPE(C.c_int, C.POINTER(SV), C.c_void_p, C.POINTER(SV))


def _c(a):
    return np.ascontiguousarray(a, dtype=np.complex128)


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _p(a):
    return C.c_void_p(a.ctypes.data)


def _nq(psi):
    return int(psi.shape[0]).bit_length() - 1


def ensure_built():
    """Build the oracle (and, when the reference sources are present, the reference)."""
    if not os.path.exists(ORACLE_LIB) or not os.path.exists(REF_LIB):
        subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


def reference_module():
    """The reference's Python module (pymodule/rqcopt_module.c) built in _ref, or None."""
    import glob
    import importlib.util
    found = glob.glob(os.path.join(HERE, "_ref", "rqcopt_hpc.*.so"))
    if not found:
        return None
    spec = importlib.util.spec_from_file_location("rqcopt_hpc", found[0])
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def default_rtr(n):
    return RtrParams(TcgParams(2 * n, 1e-8, 1e-6), 0.125, 0.01, 0.1)


class _Target:
    """Target for the oracle: 'fixture' (the reference tests' sparse map), a brickwall
    (vlist, perms) applied matrix-free, or a dense matrix."""

    def __init__(self, lib, kind, data=None):
        self.keep = []
        if kind == "fixture":
            self.ufunc = C.cast(lib.orc_fixture_ufunc, VP)
            self.udata = None
        elif kind == "brickwall":
            vlist, perms = _c(data[0]), _i(data[1])
            self.ud = BrickwallUdata(vlist.ctypes.data, vlist.shape[0], perms.ctypes.data)
            self.keep += [vlist, perms]
            self.ufunc = C.cast(lib.orc_brickwall_ufunc, VP)
            self.udata = C.cast(C.pointer(self.ud), VP)
        elif kind == "dense":
            u = _c(data)
            self.keep.append(u)
            self.ufunc = C.cast(lib.orc_dense_ufunc, VP)
            self.udata = _p(u)
        else:
            raise ValueError(kind)


class Oracle:
    def __init__(self):
        ensure_built()
        self.lib = C.CDLL(ORACLE_LIB)

    def target(self, kind, data=None):
        return _Target(self.lib, kind, data)

    def add_statevectors(self, psi1, psi2):
        psi1, psi2 = _c(psi1), _c(psi2)
        L = _nq(psi1)
        out = np.empty_like(psi1)
        self.lib.orc_add_statevectors(C.byref(SV(psi1.ctypes.data, L)), C.byref(SV(psi2.ctypes.data, L)),
                                      C.byref(SV(out.ctypes.data, L)))
        return out

    # gates and circuits
    def apply_gate(self, V, i, j, psi):
        psi, V = _c(psi), _c(V)
        out = np.empty_like(psi)
        L = _nq(psi)
        self.lib.orc_apply_gate(_p(V), i, j, C.byref(SV(psi.ctypes.data, L)), C.byref(SV(out.ctypes.data, L)))
        return out

    def apply_gate_backward(self, V, i, j, psi, dpsi_out):
        psi, dpsi_out, V = _c(psi), _c(dpsi_out), _c(V)
        L = _nq(psi)
        dpsi = np.empty_like(psi)
        dV = np.empty((4, 4), np.complex128)
        self.lib.orc_apply_gate_backward(_p(V), i, j, C.byref(SV(psi.ctypes.data, L)),
                                         C.byref(SV(dpsi_out.ctypes.data, L)), C.byref(SV(dpsi.ctypes.data, L)), _p(dV))
        return dpsi, dV

    def apply_quantum_circuit(self, gates, wires, psi):
        gates, wires, psi = _c(gates), _i(wires), _c(psi)
        L = _nq(psi)
        out = np.empty_like(psi)
        self.lib.orc_apply_circuit(_p(gates), gates.shape[0], _p(wires), C.byref(SV(psi.ctypes.data, L)),
                                   C.byref(SV(out.ctypes.data, L)))
        return out

    def _cache(self, L, n):
        states = [np.zeros(1 << L, np.complex128) for _ in range(n)]
        arr = (SV * n)(*[SV(s.ctypes.data, L) for s in states])
        return arr, states

    def quantum_circuit_forward(self, gates, wires, psi):
        gates, wires, psi = _c(gates), _i(wires), _c(psi)
        L = _nq(psi)
        arr, states = self._cache(L, gates.shape[0])
        out = np.empty_like(psi)
        self.lib.orc_circuit_forward(_p(gates), gates.shape[0], _p(wires), C.byref(SV(psi.ctypes.data, L)), arr,
                                     C.byref(SV(out.ctypes.data, L)))
        return out, states

    def quantum_circuit_backward(self, gates, wires, states, dpsi_out):
        gates, wires, dpsi_out = _c(gates), _i(wires), _c(dpsi_out)
        L = _nq(dpsi_out)
        arr = (SV * len(states))(*[SV(s.ctypes.data, L) for s in states])
        dpsi = np.empty_like(dpsi_out)
        dg = np.empty((gates.shape[0], 4, 4), np.complex128)
        self.lib.orc_circuit_backward(_p(gates), gates.shape[0], _p(wires), arr, C.byref(SV(dpsi_out.ctypes.data, L)),
                                      C.byref(SV(dpsi.ctypes.data, L)), _p(dg))
        return dpsi, dg

    def quantum_circuit_gates_hessian_vector_product(self, gates, dirs, wires, psi, phi):
        gates, dirs, wires, psi, phi = _c(gates), _c(dirs), _i(wires), _c(psi), _c(phi)
        L = _nq(psi)
        out = np.empty_like(psi)
        dg = np.empty((gates.shape[0], 4, 4), np.complex128)
        hg = np.empty_like(dg)
        self.lib.orc_circuit_gates_hvp(_p(gates), _p(dirs), gates.shape[0], _p(wires), C.byref(SV(psi.ctypes.data, L)),
                                       C.byref(SV(phi.ctypes.data, L)), C.byref(SV(out.ctypes.data, L)), _p(dg), _p(hg))
        return out, dg, hg

    def apply_brickwall_unitary(self, vlist, perms, psi):
        vlist, perms, psi = _c(vlist), _i(perms), _c(psi)
        L = _nq(psi)
        out = np.empty_like(psi)
        self.lib.orc_apply_brickwall(_p(vlist), vlist.shape[0], _p(perms), C.byref(SV(psi.ctypes.data, L)),
                                     C.byref(SV(out.ctypes.data, L)))
        return out

    # targets
    def circuit_unitary_target(self, tgt, gates, wires, L, b0=0, b1=None):
        gates, wires = _c(gates), _i(wires)
        f = np.zeros(1, np.complex128)
        self.lib.orc_circuit_target(tgt.ufunc, tgt.udata, _p(gates), gates.shape[0], _p(wires), L, L_(b0),
                                    L_(b1 if b1 is not None else 1 << L), _p(f))
        return f[0]

    def circuit_unitary_target_and_gradient(self, tgt, gates, wires, L):
        gates, wires = _c(gates), _i(wires)
        f = np.zeros(1, np.complex128)
        dg = np.empty((gates.shape[0], 4, 4), np.complex128)
        self.lib.orc_circuit_target_and_gradient(tgt.ufunc, tgt.udata, _p(gates), gates.shape[0], _p(wires), L,
                                                 L_(0), L_(1 << L), _p(f), _p(dg))
        return f[0], dg

    def circuit_unitary_target_hessian_vector_product(self, tgt, gates, dirs, wires, L, b0=0, b1=None):
        gates, dirs, wires = _c(gates), _c(dirs), _i(wires)
        f = np.zeros(1, np.complex128)
        dg = np.empty((gates.shape[0], 4, 4), np.complex128)
        hg = np.empty_like(dg)
        self.lib.orc_circuit_target_hvp(tgt.ufunc, tgt.udata, _p(gates), _p(dirs), gates.shape[0], _p(wires), L, L_(b0),
                                        L_(b1 if b1 is not None else 1 << L), _p(f), _p(dg), _p(hg))
        return f[0], dg, hg

    def circuit_unitary_target_and_projected_gradient(self, tgt, gates, wires, L):
        gates, wires = _c(gates), _i(wires)
        f = np.zeros(1, np.complex128)
        g = np.empty(16 * gates.shape[0])
        self.lib.orc_circuit_target_projected_gradient(tgt.ufunc, tgt.udata, _p(gates), gates.shape[0], _p(wires), L,
                                                       _p(f), _p(g))
        return f[0], g

    def circuit_unitary_target_projected_hessian_vector_product(self, tgt, gates, dirs, wires, L):
        gates, dirs, wires = _c(gates), _c(dirs), _i(wires)
        f = np.zeros(1, np.complex128)
        g = np.empty(16 * gates.shape[0])
        h = np.empty_like(g)
        self.lib.orc_circuit_target_projected_hvp(tgt.ufunc, tgt.udata, _p(gates), _p(dirs), gates.shape[0], _p(wires),
                                                  L, _p(f), _p(g), _p(h))
        return f[0], g, h

    def brickwall_unitary_target(self, tgt, vlist, perms, L):
        vlist, perms = _c(vlist), _i(perms)
        f = np.zeros(1, np.complex128)
        self.lib.orc_brickwall_target(tgt.ufunc, tgt.udata, _p(vlist), vlist.shape[0], L, _p(perms), _p(f))
        return f[0]

    def brickwall_unitary_target_and_gradient(self, tgt, vlist, perms, L):
        vlist, perms = _c(vlist), _i(perms)
        f = np.zeros(1, np.complex128)
        dv = np.empty((vlist.shape[0], 4, 4), np.complex128)
        self.lib.orc_brickwall_target_and_gradient(tgt.ufunc, tgt.udata, _p(vlist), vlist.shape[0], L, _p(perms),
                                                   _p(f), _p(dv))
        return f[0], dv

    def brickwall_unitary_target_and_projected_gradient(self, tgt, vlist, perms, L):
        vlist, perms = _c(vlist), _i(perms)
        f = np.zeros(1, np.complex128)
        g = np.empty(16 * vlist.shape[0])
        self.lib.orc_brickwall_target_projected_gradient(tgt.ufunc, tgt.udata, _p(vlist), vlist.shape[0], L,
                                                         _p(perms), _p(f), _p(g))
        return f[0], g

    def brickwall_unitary_target_hessian_vector_product(self, tgt, vlist, vdirs, perms, L, b0=0, b1=None):
        vlist, vdirs, perms = _c(vlist), _c(vdirs), _i(perms)
        f = np.zeros(1, np.complex128)
        dv = np.empty((vlist.shape[0], 4, 4), np.complex128)
        hv = np.empty_like(dv)
        self.lib.orc_brickwall_target_hvp(tgt.ufunc, tgt.udata, _p(vlist), _p(vdirs), vlist.shape[0], _p(perms), L,
                                          L_(b0), L_(b1 if b1 is not None else 1 << L), _p(f), _p(dv), _p(hv))
        return f[0], dv, hv

    def brickwall_unitary_target_projected_hessian_vector_product(self, tgt, vlist, vdirs, perms, L):
        vlist, vdirs, perms = _c(vlist), _c(vdirs), _i(perms)
        f = np.zeros(1, np.complex128)
        g = np.empty(16 * vlist.shape[0])
        h = np.empty_like(g)
        self.lib.orc_brickwall_target_projected_hvp(tgt.ufunc, tgt.udata, _p(vlist), _p(vdirs), vlist.shape[0],
                                                    _p(perms), L, _p(f), _p(g), _p(h))
        return f[0], g, h

    # matrix algebra
    def real_to_tangent(self, r, v):
        r, v = np.ascontiguousarray(r, np.float64), _c(v)
        z = np.empty((4, 4), np.complex128)
        self.lib.orc_real_to_tangent(_p(r), _p(v), _p(z))
        return z

    def tangent_to_real(self, v, z):
        v, z = _c(v), _c(z)
        r = np.empty(16)
        self.lib.orc_tangent_to_real(_p(v), _p(z), _p(r))
        return r

    def project_tangent(self, u, z):
        u, z = _c(u), _c(z)
        p = np.empty((4, 4), np.complex128)
        self.lib.orc_project_tangent(_p(u), _p(z), _p(p))
        return p

    def polar_factor(self, a):
        a = _c(a)
        u = np.empty((4, 4), np.complex128)
        self.lib.orc_polar_factor(_p(a), _p(u))
        return u

    def multiply(self, a, b):
        a, b = _c(a), _c(b)
        c = np.empty((4, 4), np.complex128)
        self.lib.orc_multiply(_p(a), _p(b), _p(c))
        return c

    def retract(self, u, eta):
        u, eta = _c(u), np.ascontiguousarray(eta, np.float64)
        v = np.empty((4, 4), np.complex128)
        self.lib.orc_retract(_p(u), _p(eta), _p(v))
        return v

    # trust region
    def truncated_cg_hvp(self, grad, hvp_fn, radius):
        grad = np.ascontiguousarray(grad, np.float64)
        n = grad.shape[0]

        def cb(x, fd, vec, hvp):
            np.ctypeslib.as_array(hvp, shape=(n,))[:] = hvp_fn(np.ctypeslib.as_array(vec, shape=(n,)).copy())

        f = HVP_FUNC(cb)
        z = np.empty(n)
        params = TcgParams(2 * n, 1e-8, 1e-6)
        self.lib.orc_truncated_cg_hvp.restype = C.c_bool
        b = self.lib.orc_truncated_cg_hvp(None, _p(grad), C.cast(f, VP), None, n, D(radius), C.byref(params), _p(z))
        return z, bool(b)

    def optimize_brickwall_circuit_hvp(self, tgt, vstart, perms, L, niter):
        vstart, perms = _c(vstart), _i(perms)
        nl = vstart.shape[0]
        f_iter = np.empty(niter + 1)
        vopt = np.empty_like(vstart)
        acc = np.zeros(niter, np.int32)
        bnd = np.zeros(niter, np.int32)
        params = default_rtr(16 * nl)
        self.lib.orc_optimize_brickwall_hvp(tgt.ufunc, tgt.udata, _p(vstart), nl, L, _p(perms), C.byref(params), niter,
                                            _p(f_iter), _p(vopt), _p(acc), _p(bnd))
        return f_iter, vopt, acc, bnd

    def optimize_quantum_circuit(self, tgt, gstart, wires, L, niter):
        gstart, wires = _c(gstart), _i(wires)
        ng = gstart.shape[0]
        f_iter = np.empty(niter + 1)
        gopt = np.empty_like(gstart)
        acc = np.zeros(niter, np.int32)
        bnd = np.zeros(niter, np.int32)
        params = default_rtr(16 * ng)
        self.lib.orc_optimize_circuit_hvp(tgt.ufunc, tgt.udata, _p(gstart), ng, L, _p(wires), C.byref(params), niter,
                                          _p(f_iter), _p(gopt), _p(acc), _p(bnd))
        return f_iter, gopt, acc, bnd


    # full-Hessian path (arrays: amplitude-major, [2^L, nstates])
    def apply_gate_to_array(self, V, i, j, psi):
        V, psi = _c(V), _c(psi)
        L = _nq(psi)
        out = np.empty_like(psi)
        self.lib.orc_apply_gate_to_array(_p(V), i, j, L, psi.shape[1], _p(psi), _p(out))
        return out

    def apply_gate_backward_array(self, V, i, j, psi, dpsi_out):
        psi, dpsi_out = _c(psi), _c(dpsi_out)
        L = _nq(psi)
        dg = np.empty((psi.shape[1], 4, 4), np.complex128)
        self.lib.orc_apply_gate_backward_array(i, j, L, psi.shape[1], _p(psi), _p(dpsi_out), _p(dg))
        return dg

    def apply_gate_placeholder(self, i, j, psi):
        psi = _c(psi)
        L = _nq(psi)
        out = np.empty((psi.shape[0], 16), np.complex128)
        self.lib.orc_apply_gate_placeholder(i, j, L, _p(psi), _p(out))
        return out

    def brickwall_unitary_forward(self, vlist, perms, psi):
        vlist, perms, psi = _c(vlist), _i(perms), _c(psi)
        L = _nq(psi)
        arr, states = self._cache(L, vlist.shape[0] * (L // 2))
        out = np.empty_like(psi)
        self.lib.orc_brickwall_forward(_p(vlist), vlist.shape[0], _p(perms), C.byref(SV(psi.ctypes.data, L)), arr,
                                       C.byref(SV(out.ctypes.data, L)))
        return out, states

    def brickwall_unitary_backward(self, vlist, perms, states, dpsi_out):
        """src/brickwall_circuit.c:85-124: the backward pass of the brickwall as a sequential
        circuit (layer l's gate on pairs (perms[l][2p], perms[l][2p + 1])), the gate
        gradients of each layer's L/2 pairs summed into the layer gradient."""
        vlist, perms, dpsi_out = _c(vlist), _i(perms), _c(dpsi_out)
        L, nl = _nq(dpsi_out), vlist.shape[0]
        per = L // 2
        gates = np.repeat(vlist, per, axis=0)
        wires = np.stack([perms[l, 2 * p:2 * p + 2] for l in range(nl) for p in range(per)])
        dpsi, dg = self.quantum_circuit_backward(gates, wires, [_c(s) for s in states], dpsi_out)
        return dpsi, dg.reshape(nl, per, 4, 4).sum(axis=1)

    def brickwall_unitary_backward_hessian(self, vlist, perms, states, dpsi_out):
        vlist, perms, dpsi_out = _c(vlist), _i(perms), _c(dpsi_out)
        L, nl = _nq(dpsi_out), vlist.shape[0]
        states = [_c(s) for s in states]
        arr = (SV * len(states))(*[SV(s.ctypes.data, L) for s in states])
        dpsi = np.empty_like(dpsi_out)
        dv = np.empty((nl, 4, 4), np.complex128)
        hess = np.empty((16 * nl, 16 * nl), np.complex128)
        self.lib.orc_brickwall_backward_hessian(_p(vlist), nl, _p(perms), arr, C.byref(SV(dpsi_out.ctypes.data, L)),
                                                C.byref(SV(dpsi.ctypes.data, L)), _p(dv), _p(hess))
        return dpsi, dv, hess

    def apply_brickwall_unitary_gate_placeholder(self, vlist, perms, l, states):
        vlist, perms = _c(vlist), _i(perms)
        states = [_c(s) for s in states]
        L = _nq(states[0])
        arr = (SV * len(states))(*[SV(s.ctypes.data, L) for s in states])
        out = np.empty((1 << L, 16), np.complex128)
        ret = self.lib.orc_apply_brickwall_placeholder(_p(vlist), vlist.shape[0], _p(perms), l, arr, _p(out))
        assert ret == 0
        return out

    def brickwall_unitary_target_gradient_hessian(self, tgt, vlist, perms, L):
        vlist, perms = _c(vlist), _i(perms)
        nl = vlist.shape[0]
        f = np.zeros(1, np.complex128)
        dv = np.empty((nl, 4, 4), np.complex128)
        hess = np.empty((16 * nl, 16 * nl), np.complex128)
        ret = self.lib.orc_brickwall_target_gradient_hessian(tgt.ufunc, tgt.udata, _p(vlist), nl, L, _p(perms), _p(f),
                                                             _p(dv), _p(hess))
        assert ret == 0
        return f[0], dv, hess

    def brickwall_unitary_target_gradient_vector_hessian_matrix(self, tgt, vlist, perms, L):
        vlist, perms = _c(vlist), _i(perms)
        nl = vlist.shape[0]
        f = np.zeros(1, np.complex128)
        g = np.empty(16 * nl)
        H = np.empty((16 * nl, 16 * nl))
        ret = self.lib.orc_brickwall_target_gradient_vector_hessian_matrix(tgt.ufunc, tgt.udata, _p(vlist), nl, L,
                                                                           _p(perms), _p(f), _p(g), _p(H))
        assert ret == 0
        return f[0], g, H

    def truncated_cg_hmat(self, grad, hess, radius):
        grad, hess = np.ascontiguousarray(grad, np.float64), np.ascontiguousarray(hess, np.float64)
        n = grad.shape[0]
        z = np.empty(n)
        params = TcgParams(2 * n, 1e-8, 1e-6)
        self.lib.orc_truncated_cg_hmat.restype = C.c_bool
        b = self.lib.orc_truncated_cg_hmat(_p(grad), _p(hess), n, D(radius), C.byref(params), _p(z))
        return z, bool(b)

    def optimize_brickwall_circuit_hmat(self, tgt, vstart, perms, L, niter):
        vstart, perms = _c(vstart), _i(perms)
        nl = vstart.shape[0]
        f_iter = np.empty(niter + 1)
        vopt = np.empty_like(vstart)
        acc = np.zeros(niter, np.int32)
        bnd = np.zeros(niter, np.int32)
        params = default_rtr(16 * nl)
        self.lib.orc_optimize_brickwall_hmat(tgt.ufunc, tgt.udata, _p(vstart), nl, L, _p(perms), C.byref(params),
                                             niter, _p(f_iter), _p(vopt), _p(acc), _p(bnd))
        return f_iter, vopt, acc, bnd


    # sampling estimator
    def seed_rng_state(self, seed):
        r = RngState()
        self.lib.orc_seed_rng(C.c_uint64(seed), C.byref(r))
        return r

    def haar_random_statevector(self, L, rng):
        out = np.empty(1 << L, np.complex128)
        self.lib.orc_haar_statevector(C.byref(SV(out.ctypes.data, L)), C.byref(rng))
        return out

    def brickwall_unitary_target_sampling(self, tgt, vlist, perms, L, nsamples, rng):
        vlist, perms = _c(vlist), _i(perms)
        f = np.zeros(1, np.complex128)
        ret = self.lib.orc_brickwall_target_sampling(tgt.ufunc, tgt.udata, _p(vlist), vlist.shape[0], L, _p(perms),
                                                     L_(nsamples), C.byref(rng), _p(f))
        assert ret == 0
        return f[0]

    def circuit_unitary_target_sampling(self, tgt, gates, wires, L, nsamples, rng):
        gates, wires = _c(gates), _i(wires)
        f = np.zeros(1, np.complex128)
        ret = self.lib.orc_circuit_target_sampling(tgt.ufunc, tgt.udata, _p(gates), gates.shape[0], _p(wires), L,
                                                   L_(nsamples), C.byref(rng), _p(f))
        assert ret == 0
        return f[0]

    def brickwall_unitary_target_gradient_hessian_sampling(self, tgt, vlist, perms, L, nsamples, rng):
        vlist, perms = _c(vlist), _i(perms)
        nl = vlist.shape[0]
        f = np.zeros(1, np.complex128)
        dv = np.empty((nl, 4, 4), np.complex128)
        hess = np.empty((16 * nl, 16 * nl), np.complex128)
        ret = self.lib.orc_brickwall_target_gradient_hessian_sampling(tgt.ufunc, tgt.udata, _p(vlist), nl, L,
                                                                      _p(perms), L_(nsamples), C.byref(rng), _p(f),
                                                                      _p(dv), _p(hess))
        assert ret == 0
        return f[0], dv, hess

    def brickwall_unitary_target_gradient_vector_hessian_matrix_sampling(self, tgt, vlist, perms, L, nsamples, rng):
        vlist, perms = _c(vlist), _i(perms)
        nl = vlist.shape[0]
        f = np.zeros(1, np.complex128)
        g = np.empty(16 * nl)
        H = np.empty((16 * nl, 16 * nl))
        ret = self.lib.orc_brickwall_target_gradient_vector_hessian_matrix_sampling(
            tgt.ufunc, tgt.udata, _p(vlist), nl, L, _p(perms), L_(nsamples), C.byref(rng), _p(f), _p(g), _p(H))
        assert ret == 0
        return f[0], g, H

    def optimize_brickwall_circuit_hmat_sampling(self, tgt, vstart, perms, L, nsamples, rng, niter):
        vstart, perms = _c(vstart), _i(perms)
        nl = vstart.shape[0]
        f_iter = np.empty(niter + 1)
        vopt = np.empty_like(vstart)
        params = default_rtr(16 * nl)
        self.lib.orc_optimize_brickwall_hmat_sampling(tgt.ufunc, tgt.udata, _p(vstart), nl, L, _p(perms),
                                                      L_(nsamples), C.byref(rng), C.byref(params), niter,
                                                      _p(f_iter), _p(vopt), None, None)
        return f_iter, vopt


    # block-encoding target (hfunc acts on nqubits / 2 qubits)
    def brickwall_blockenc_target(self, tgt, vlist, perms, L):
        vlist, perms = _c(vlist), _i(perms)
        f = np.zeros(1)
        assert self.lib.orc_blockenc_target(tgt.ufunc, tgt.udata, _p(vlist), vlist.shape[0], L, _p(perms), _p(f)) == 0
        return f[0]

    def brickwall_blockenc_target_and_gradient(self, tgt, vlist, perms, L):
        vlist, perms = _c(vlist), _i(perms)
        f = np.zeros(1)
        dv = np.empty((vlist.shape[0], 4, 4), np.complex128)
        assert self.lib.orc_blockenc_target_and_gradient(tgt.ufunc, tgt.udata, _p(vlist), vlist.shape[0], L, _p(perms),
                                                         _p(f), _p(dv)) == 0
        return f[0], dv

    def brickwall_blockenc_target_and_gradient_vector(self, tgt, vlist, perms, L):
        vlist, perms = _c(vlist), _i(perms)
        f = np.zeros(1)
        g = np.empty(16 * vlist.shape[0])
        assert self.lib.orc_blockenc_target_and_gradient_vector(tgt.ufunc, tgt.udata, _p(vlist), vlist.shape[0], L,
                                                                _p(perms), _p(f), _p(g)) == 0
        return f[0], g

    def brickwall_blockenc_target_gradient_hessian(self, tgt, vlist, perms, L):
        vlist, perms = _c(vlist), _i(perms)
        nl = vlist.shape[0]
        f = np.zeros(1)
        dv = np.empty((nl, 4, 4), np.complex128)
        h1 = np.empty((16 * nl, 16 * nl), np.complex128)
        h2 = np.empty_like(h1)
        assert self.lib.orc_blockenc_target_gradient_hessian(tgt.ufunc, tgt.udata, _p(vlist), nl, L, _p(perms), _p(f),
                                                             _p(dv), _p(h1), _p(h2)) == 0
        return f[0], dv, h1, h2

    def brickwall_blockenc_target_gradient_vector_hessian_matrix(self, tgt, vlist, perms, L):
        vlist, perms = _c(vlist), _i(perms)
        nl = vlist.shape[0]
        f = np.zeros(1)
        g = np.empty(16 * nl)
        H = np.empty((16 * nl, 16 * nl))
        assert self.lib.orc_blockenc_target_gradient_vector_hessian_matrix(tgt.ufunc, tgt.udata, _p(vlist), nl, L,
                                                                           _p(perms), _p(f), _p(g), _p(H)) == 0
        return f[0], g, H


class Reference:
    """The reference's own C sources compiled in _ref/ (built only where the sources exist)."""

    def __init__(self):
        if not os.path.exists(REF_LIB):
            raise FileNotFoundError(REF_LIB)
        self.lib = C.CDLL(REF_LIB)

    @staticmethod
    def available():
        return os.path.exists(REF_LIB)

    def brickwall_hvp_columns(self, vlist, vdirs, perms, L, tvlist, tperms, b0, b1):
        vlist, vdirs, perms, tvlist, tperms = _c(vlist), _c(vdirs), _i(perms), _c(tvlist), _i(tperms)
        G = vlist.shape[0] * (L // 2)
        f = np.zeros(2)
        dg = np.empty((G, 4, 4), np.complex128)
        hg = np.empty_like(dg)
        ret = self.lib.refdrv_brickwall_hvp_columns(_p(vlist), _p(vdirs), vlist.shape[0], _p(perms), L, _p(tvlist),
                                                    tvlist.shape[0], _p(tperms), L_(b0), L_(b1), _p(f), _p(dg), _p(hg))
        assert ret == 0
        return f[0] + 1j * f[1], dg, hg

    def brickwall_projected_hvp(self, vlist, vdirs, perms, L, tvlist, tperms):
        vlist, vdirs, perms, tvlist, tperms = _c(vlist), _c(vdirs), _i(perms), _c(tvlist), _i(tperms)
        f = np.zeros(2)
        g = np.empty(16 * vlist.shape[0])
        h = np.empty_like(g)
        ret = self.lib.refdrv_brickwall_projected_hvp(_p(vlist), _p(vdirs), vlist.shape[0], _p(perms), L, _p(tvlist),
                                                      tvlist.shape[0], _p(tperms), _p(f), _p(g), _p(h))
        assert ret == 0
        return f[0] + 1j * f[1], g, h

    def optimize_brickwall(self, vstart, perms, L, tvlist, tperms, niter):
        vstart, perms, tvlist, tperms = _c(vstart), _i(perms), _c(tvlist), _i(tperms)
        f_iter = np.empty(niter + 1)
        vopt = np.empty_like(vstart)
        self.lib.refdrv_optimize_brickwall(_p(vstart), vstart.shape[0], L, _p(perms), _p(tvlist), tvlist.shape[0],
                                           _p(tperms), niter, _p(f_iter), _p(vopt))
        return f_iter, vopt

    def truncated_cg_hvp(self, grad, hvp_fn, radius):
        grad = np.ascontiguousarray(grad, np.float64)
        n = grad.shape[0]

        def cb(x, fd, vec, hvp):
            np.ctypeslib.as_array(hvp, shape=(n,))[:] = hvp_fn(np.ctypeslib.as_array(vec, shape=(n,)).copy())

        f = HVP_FUNC(cb)
        z = np.empty(n)
        params = TcgParams(2 * n, 1e-8, 1e-6)
        self.lib.truncated_cg_hvp.restype = C.c_bool
        b = self.lib.truncated_cg_hvp(None, _p(grad), C.cast(f, VP), None, n, D(radius), C.byref(params), _p(z))
        return z, bool(b)

    # full-Hessian path of the reference
    def gradient_vector_hessian_matrix(self, vlist, perms, L, tvlist, tperms):
        vlist, perms, tvlist, tperms = _c(vlist), _i(perms), _c(tvlist), _i(tperms)
        nl = vlist.shape[0]
        f = np.zeros(2)
        g = np.empty(16 * nl)
        H = np.empty((16 * nl, 16 * nl))
        ret = self.lib.refdrv_gradient_vector_hessian_matrix(_p(vlist), nl, _p(perms), L, _p(tvlist), tvlist.shape[0],
                                                             _p(tperms), _p(f), _p(g), _p(H))
        assert ret == 0
        return f[0] + 1j * f[1], g, H

    def gradient_hessian(self, vlist, perms, L, tvlist, tperms):
        vlist, perms, tvlist, tperms = _c(vlist), _i(perms), _c(tvlist), _i(tperms)
        nl = vlist.shape[0]
        f = np.zeros(2)
        dv = np.empty((nl, 4, 4), np.complex128)
        hess = np.empty((16 * nl, 16 * nl), np.complex128)
        ret = self.lib.refdrv_gradient_hessian(_p(vlist), nl, _p(perms), L, _p(tvlist), tvlist.shape[0], _p(tperms),
                                               _p(f), _p(dv), _p(hess))
        assert ret == 0
        return f[0] + 1j * f[1], dv, hess

    def optimize_brickwall_hmat(self, vstart, perms, L, tvlist, tperms, niter):
        vstart, perms, tvlist, tperms = _c(vstart), _i(perms), _c(tvlist), _i(tperms)
        f_iter = np.empty(niter + 1)
        vopt = np.empty_like(vstart)
        self.lib.refdrv_optimize_brickwall_hmat(_p(vstart), vstart.shape[0], L, _p(perms), _p(tvlist),
                                                tvlist.shape[0], _p(tperms), niter, _p(f_iter), _p(vopt))
        return f_iter, vopt

    def forward_backward_hessian(self, vlist, perms, psi, dpsi_out):
        """One brickwall_unitary_forward + brickwall_unitary_backward_hessian of a single
        state (the 16-qubit benchmark of the reference's examples)."""
        vlist, perms, psi, dpsi_out = _c(vlist), _i(perms), _c(psi), _c(dpsi_out)
        L, nl = _nq(psi), vlist.shape[0]
        psi_out = np.empty_like(psi)
        dpsi = np.empty_like(psi)
        dv = np.empty((nl, 4, 4), np.complex128)
        hess = np.empty((16 * nl, 16 * nl), np.complex128)
        ret = self.lib.refdrv_forward_backward_hessian(_p(vlist), nl, _p(perms), L, _p(psi), _p(dpsi_out),
                                                       _p(psi_out), _p(dpsi), _p(dv), _p(hess))
        assert ret == 0
        return psi_out, dpsi, dv, hess

    def hessian_columns(self, vlist, perms, L, tvlist, tperms, b0, b1):
        """Sums of f, gradients and complex Hessian over basis columns [b0, b1)."""
        vlist, perms, tvlist, tperms = _c(vlist), _i(perms), _c(tvlist), _i(tperms)
        nl = vlist.shape[0]
        f = np.zeros(2)
        dv = np.empty((nl, 4, 4), np.complex128)
        hess = np.empty((16 * nl, 16 * nl), np.complex128)
        ret = self.lib.refdrv_hessian_columns(_p(vlist), nl, _p(perms), L, _p(tvlist), tvlist.shape[0], _p(tperms),
                                              L_(b0), L_(b1), _p(f), _p(dv), _p(hess))
        assert ret == 0
        return f[0] + 1j * f[1], dv, hess


    # sampling estimator of the reference
    def seed_rng_state(self, seed):
        r = RngState()
        self.lib.seed_rng_state(C.c_uint64(seed), C.byref(r))
        return r

    def haar_random_statevector(self, L, rng):
        out = np.empty(1 << L, np.complex128)
        self.lib.haar_random_statevector(C.byref(SV(out.ctypes.data, L)), C.byref(rng))
        return out

    def sampling(self, mode, vlist, perms, L, target, nsamples, rng):
        """mode 0: f; 1: f, dvlist, complex hess; 2: f, grad_vec, H.  target: (tvlist, tperms)
        for a brickwall target or a dense matrix."""
        vlist, perms = _c(vlist), _i(perms)
        nl = vlist.shape[0]
        if isinstance(target, tuple):
            tv, tp, td = _c(target[0]), _i(target[1]), None
        else:
            tv, tp, td = None, None, _c(target)
        f = np.zeros(2)
        o1 = o2 = None
        if mode == 1:
            o1, o2 = np.empty((nl, 4, 4), np.complex128), np.empty((16 * nl, 16 * nl), np.complex128)
        elif mode == 2:
            o1, o2 = np.empty(16 * nl), np.empty((16 * nl, 16 * nl))
        ret = self.lib.refdrv_sampling(mode, _p(vlist), nl, _p(perms), L, _p(tv) if tv is not None else None,
                                       tv.shape[0] if tv is not None else 0, _p(tp) if tp is not None else None,
                                       _p(td) if td is not None else None, L_(nsamples), C.byref(rng), _p(f),
                                       _p(o1) if o1 is not None else None, _p(o2) if o2 is not None else None)
        assert ret == 0
        fc = f[0] + 1j * f[1]
        return fc if mode == 0 else (fc, o1, o2)

    def optimize_brickwall_hmat_sampling(self, vstart, perms, L, tvlist, tperms, nsamples, rng, niter):
        vstart, perms, tvlist, tperms = _c(vstart), _i(perms), _c(tvlist), _i(tperms)
        f_iter = np.empty(niter + 1)
        vopt = np.empty_like(vstart)
        self.lib.refdrv_optimize_brickwall_hmat_sampling(_p(vstart), vstart.shape[0], L, _p(perms), _p(tvlist),
                                                         tvlist.shape[0], _p(tperms), L_(nsamples), C.byref(rng),
                                                         niter, _p(f_iter), _p(vopt))
        return f_iter, vopt

    def blockenc(self, mode, vlist, perms, L, hvlist, hperms):
        """Block-encoding target of the reference with a brickwall H on L / 2 qubits: mode 0 f,
        1 f and gradient, 2 f, gradient vector, 3 f, gradient and hess1, hess2, 4 f, gradient
        vector and H."""
        vlist, perms, hvlist, hperms = _c(vlist), _i(perms), _c(hvlist), _i(hperms)
        nl = vlist.shape[0]
        m = 16 * nl
        f = np.zeros(1)
        o = [None, None, None]
        if mode == 1:
            o[0] = np.empty((nl, 4, 4), np.complex128)
        elif mode == 2:
            o[0] = np.empty(m)
        elif mode == 3:
            o = [np.empty((nl, 4, 4), np.complex128), np.empty((m, m), np.complex128), np.empty((m, m), np.complex128)]
        elif mode == 4:
            o = [np.empty(m), np.empty((m, m)), None]
        ret = self.lib.refdrv_blockenc(mode, _p(vlist), nl, _p(perms), L, _p(hvlist), hvlist.shape[0], _p(hperms),
                                       _p(f), *[(_p(x) if x is not None else None) for x in o])
        assert ret == 0
        return (f[0],) + tuple(x for x in o if x is not None)

    def blockenc_hessian_columns(self, vlist, perms, L, hvlist, hperms, b0, b1):
        """f of the block-encoding Hessian column loop over half-register columns [b0, b1)."""
        vlist, perms, hvlist, hperms = _c(vlist), _i(perms), _c(hvlist), _i(hperms)
        f = np.zeros(1)
        ret = self.lib.refdrv_blockenc_hessian_columns(_p(vlist), vlist.shape[0], _p(perms), L, _p(hvlist),
                                                       hvlist.shape[0], _p(hperms), L_(b0), L_(b1), _p(f))
        assert ret == 0
        return f[0]


# ---------------------------------------------------------------------------- real build
# The reference compiled without COMPLEX_CIRCUIT (src/config.h:14-22): real states and
# gates, 6 tangent parameters per gate (src/matrix.c:245-271, 288-300), one real normal
# per amplitude of a sample state (src/statevector.c:115-121).

REAL_REF_LIB = os.path.join(HERE, "_ref", "librqcopt_ref_real.so")
_UPPER = (1, 2, 3, 6, 7, 11)
TARGET_FUNC = C.CFUNCTYPE(C.c_double, C.POINTER(C.c_double), C.c_void_p)
TARGET_GRAD_FUNC = C.CFUNCTYPE(C.c_double, C.POINTER(C.c_double), C.c_void_p, C.POINTER(C.c_double))
RETRACT_FUNC = C.CFUNCTYPE(None, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_void_p, C.POINTER(C.c_double))


def real_fixture_map(x):
    """The reference tests' synthetic target map in the real build (test/test_target.c:26-27)."""
    n = x.shape[0]
    i = np.arange(n)
    return -1.1 * x[((i + 3) * 113) % n] - 0.7 * x[((i + 9) * 173) % n] + 0.5 * x[i] + 0.3 * x[((i + 4) * 199) % n]


def real_antisymm(r6):
    """6 reals -> real antisymmetric 4x4 matrix, isometrically (src/matrix.c:245-271)."""
    w = np.zeros((4, 4))
    for k, e in enumerate(_UPPER):
        w[e // 4, e % 4] = r6[k] / np.sqrt(2.0)
        w[e % 4, e // 4] = -w[e // 4, e % 4]
    return w


def _to6(r16):
    """The complex build's 16 parameters of real antisymmetric matrices (their entries) -> the
    real build's 6 (src/matrix.c:288-300)."""
    r16 = np.asarray(r16).reshape(-1, 16)
    return (np.sqrt(2.0) * r16[:, list(_UPPER)]).ravel()


def _re(x):
    if isinstance(x, tuple):
        return tuple(_re(y) for y in x)
    if isinstance(x, np.ndarray) and np.iscomplexobj(x):
        return np.ascontiguousarray(x.real)
    if isinstance(x, complex):
        return x.real
    return x


class _FnTarget:
    def __init__(self, fn):
        def cb(psi_p, udata, out_p):
            psi, out = psi_p.contents, out_p.contents
            n = 1 << psi.nqubits
            x = np.ctypeslib.as_array(C.cast(psi.data, C.POINTER(C.c_double)), shape=(2 * n,)).view(np.complex128)
            y = np.ctypeslib.as_array(C.cast(out.data, C.POINTER(C.c_double)), shape=(2 * n,)).view(np.complex128)
            y[:] = fn(x.copy())
            return 0

        self.cb = LINEAR_FUNC(cb)
        self.ufunc = C.cast(self.cb, VP)
        self.udata = None


class RealOracle:
    """The reference's real build restated as the complex restatement (Oracle) on real
    inputs: for real gates, states and targets every product and sum the complex build
    forms has a zero imaginary part and the real build's value as real part, and its
    conjugations are the identity; the real parts of the results are returned.  What the
    builds do differently is restated here: the 6-parameter tangents (a real
    antisymmetric w has the 16 complex-build parameters w.ravel(), and the 6 real-build
    ones sqrt(2) w[upper]), real sample states, the single block-encoding Hessian
    hess1 + hess2 (src/target.c:1595-1597), and the optimisers over 6 parameters per
    gate (src/brickwall_opt.c:22-149, src/circuit_opt.c)."""

    name = "real-oracle"

    def __init__(self):
        self.o = Oracle()

    def target(self, kind, data=None):
        if kind == "fixture":
            return _FnTarget(real_fixture_map)
        if kind in ("brickwall", "host_brickwall"):
            return self.o.target("brickwall", (_c(data[0]), data[1]))
        if kind == "dense":
            return self.o.target("dense", _c(data))
        raise ValueError(kind)

    def __getattr__(self, name):
        fn = getattr(self.o, name)

        def call(*args, **kw):
            return _re(fn(*[_c(a) if isinstance(a, np.ndarray) and a.dtype == np.float64 and a.ndim >= 2 else a
                            for a in args], **kw))

        return call

    # states: complex copies of real 1-d inputs (gate-level functions)
    def _cs(self, fn, *args):
        return _re(fn(*[_c(a) if isinstance(a, np.ndarray) and a.dtype == np.float64 else a for a in args]))

    def apply_gate(self, V, i, j, psi):
        return self._cs(self.o.apply_gate, V, i, j, psi)

    def apply_gate_backward(self, V, i, j, psi, dout):
        return self._cs(self.o.apply_gate_backward, V, i, j, psi, dout)

    def apply_quantum_circuit(self, gates, wires, psi):
        return _re(self.o.apply_quantum_circuit(_c(gates), wires, _c(psi)))

    def quantum_circuit_forward(self, gates, wires, psi):
        out, cache = self.o.quantum_circuit_forward(_c(gates), wires, _c(psi))
        return _re(out), cache

    def quantum_circuit_backward(self, gates, wires, cache, dout):
        return _re(self.o.quantum_circuit_backward(_c(gates), wires, cache, _c(dout)))

    def quantum_circuit_gates_hessian_vector_product(self, gates, dirs, wires, psi, phi):
        return _re(self.o.quantum_circuit_gates_hessian_vector_product(_c(gates), _c(dirs), wires, _c(psi), _c(phi)))

    def apply_brickwall_unitary(self, vlist, perms, psi):
        return _re(self.o.apply_brickwall_unitary(_c(vlist), perms, _c(psi)))

    def brickwall_unitary_forward(self, vlist, perms, psi):
        out, states = self.o.brickwall_unitary_forward(_c(vlist), perms, _c(psi))
        return _re(out), states

    def brickwall_unitary_backward_hessian(self, vlist, perms, states, dout):
        return _re(self.o.brickwall_unitary_backward_hessian(_c(vlist), perms, states, _c(dout)))

    def apply_gate_to_array(self, V, i, j, psi):
        return _re(self.o.apply_gate_to_array(_c(V), i, j, _c(psi)))

    def apply_gate_backward_array(self, V, i, j, psi, dout):
        return _re(self.o.apply_gate_backward_array(_c(V), i, j, _c(psi), _c(dout)))

    def apply_gate_placeholder(self, i, j, psi):
        return _re(self.o.apply_gate_placeholder(i, j, _c(psi)))

    # projected forms: 6 parameters per gate
    def circuit_unitary_target_and_projected_gradient(self, t, gates, wires, L):
        f, g = self.o.circuit_unitary_target_and_projected_gradient(t, _c(gates), wires, L)
        return f.real, _to6(g)

    def circuit_unitary_target_projected_hessian_vector_product(self, t, gates, dirs, wires, L):
        f, g, h = self.o.circuit_unitary_target_projected_hessian_vector_product(t, _c(gates), _c(dirs), wires, L)
        return f.real, _to6(g), _to6(h)

    def brickwall_unitary_target_and_projected_gradient(self, t, vlist, perms, L):
        f, g = self.o.brickwall_unitary_target_and_projected_gradient(t, _c(vlist), perms, L)
        return f.real, _to6(g)

    def brickwall_unitary_target_projected_hessian_vector_product(self, t, vlist, vdirs, perms, L):
        f, g, h = self.o.brickwall_unitary_target_projected_hessian_vector_product(t, _c(vlist), _c(vdirs), perms, L)
        return f.real, _to6(g), _to6(h)

    def brickwall_blockenc_target_gradient_hessian(self, t, vlist, perms, L):
        f, dv, h1, h2 = self.o.brickwall_blockenc_target_gradient_hessian(t, _c(vlist), perms, L)
        return f, dv.real.copy(), (h1 + h2).real.copy()

    # sampling: real normal states
    def _sampled(self, fn, *args):
        self.o.lib.orc_set_real_samples(1)
        try:
            return fn(*args)
        finally:
            self.o.lib.orc_set_real_samples(0)

    def haar_random_statevector(self, L, rng):
        return self._sampled(self.o.haar_random_statevector, L, rng).real.copy()

    def brickwall_unitary_target_sampling(self, t, vlist, perms, L, ns, rng):
        return self._sampled(self.o.brickwall_unitary_target_sampling, t, _c(vlist), perms, L, ns, rng).real

    def circuit_unitary_target_sampling(self, t, gates, wires, L, ns, rng):
        return self._sampled(self.o.circuit_unitary_target_sampling, t, _c(gates), wires, L, ns, rng).real

    def brickwall_unitary_target_gradient_hessian_sampling(self, t, vlist, perms, L, ns, rng):
        return _re(self._sampled(self.o.brickwall_unitary_target_gradient_hessian_sampling, t, _c(vlist), perms, L, ns,
                                 rng))

    # 4x4 algebra of the real build
    def real_to_antisymm(self, r6):
        return real_antisymm(r6)

    def real_to_tangent(self, r6, v):
        return np.asarray(v).real @ real_antisymm(r6)

    def tangent_to_real(self, v, z):
        t = np.asarray(v).real.T @ np.asarray(z).real
        return _to6((0.5 * (t - t.T)).ravel())

    def retract(self, v, r6):
        return self.o.polar_factor(_c(np.asarray(v).real @ (np.eye(4) + real_antisymm(r6)))).real.copy()

    # optimisers over 6 parameters per gate, on the oracle's trust region
    def _rtr(self, f, fd, hvp, k, x0, niter):
        n, m = 6 * k, 16 * k
        cf = TARGET_FUNC(lambda x, d: f(np.ctypeslib.as_array(x, shape=(m,)).reshape(k, 4, 4).copy()))

        def _fd(x, d, g):
            fx, gv = fd(np.ctypeslib.as_array(x, shape=(m,)).reshape(k, 4, 4).copy())
            np.ctypeslib.as_array(g, shape=(n,))[:] = gv
            return fx

        def _hvp(x, d, vec, out):
            v = np.ctypeslib.as_array(x, shape=(m,)).reshape(k, 4, 4).copy()
            r = np.ctypeslib.as_array(vec, shape=(n,)).copy()
            np.ctypeslib.as_array(out, shape=(n,))[:] = hvp(v, r)

        def _retract(x, eta, rd, xs):
            v = np.ctypeslib.as_array(x, shape=(m,)).reshape(k, 4, 4)
            e = np.ctypeslib.as_array(eta, shape=(n,)).reshape(k, 6)
            np.ctypeslib.as_array(xs, shape=(m,))[:] = np.stack([self.retract(v[i], e[i]) for i in range(k)]).ravel()

        cfd, chvp, cret = TARGET_GRAD_FUNC(_fd), HVP_FUNC(_hvp), RETRACT_FUNC(_retract)
        x0 = np.ascontiguousarray(x0, np.float64)
        f_iter, xf = np.empty(niter + 1), np.empty(m)
        params = default_rtr(n)
        self.o.lib.orc_rtr_optimize_hvp(C.cast(cf, VP), C.cast(cfd, VP), C.cast(chvp, VP), None, C.cast(cret, VP), None,
                                        n, _p(x0), m, C.byref(params), niter, _p(f_iter), _p(xf), None, None)
        return f_iter, xf.reshape(k, 4, 4)

    def optimize_brickwall_circuit_hvp(self, t, vstart, perms, L, niter):
        k = vstart.shape[0]
        return self._rtr(
            lambda v: self.brickwall_unitary_target(t, v, perms, L).real,
            lambda v: self.brickwall_unitary_target_and_projected_gradient(t, v, perms, L),
            lambda v, r: self.brickwall_unitary_target_projected_hessian_vector_product(
                t, v, np.stack([self.real_to_tangent(r[6 * i:6 * i + 6], v[i]) for i in range(k)]), perms, L)[2],
            k, vstart, niter)

    def optimize_quantum_circuit(self, t, gstart, wires, L, niter):
        k = gstart.shape[0]
        return self._rtr(
            lambda g: self.circuit_unitary_target(t, g, wires, L).real,
            lambda g: self.circuit_unitary_target_and_projected_gradient(t, g, wires, L),
            lambda g, r: self.circuit_unitary_target_projected_hessian_vector_product(
                t, g, np.stack([self.real_to_tangent(r[6 * i:6 * i + 6], g[i]) for i in range(k)]), wires, L)[2],
            k, gstart, niter)


class _RefRtrParams(C.Structure):
    _fields_ = [("tcg", TcgParams), ("rho_trust", C.c_double), ("radius_init", C.c_double), ("maxradius", C.c_double),
                ("g_func", C.c_void_p), ("g_data", C.c_void_p), ("g_iter", C.c_void_p)]


class _RefBrickwall(C.Structure):
    _fields_ = [("vlist", C.c_void_p), ("nlayers", C.c_int), ("perms", C.c_void_p)]


class RealReference:
    """The reference's own sources compiled without COMPLEX_CIRCUIT in _ref/, called
    through their public functions (real arrays; perms as `const int*[]`)."""

    name = "real-reference"

    def __init__(self):
        if not os.path.exists(REAL_REF_LIB):
            raise FileNotFoundError(REAL_REF_LIB)
        self.lib = C.CDLL(REAL_REF_LIB)
        self.lib.truncated_cg_hvp.restype = C.c_bool

    @staticmethod
    def available():
        return os.path.exists(REAL_REF_LIB)

    @staticmethod
    def _r(a):
        return np.ascontiguousarray(np.asarray(a).real if np.iscomplexobj(a) else a, dtype=np.float64)

    @staticmethod
    def _perms(perms):
        perms = _i(perms)
        arr = (C.c_void_p * perms.shape[0])(*[perms[k].ctypes.data for k in range(perms.shape[0])])
        return arr, perms

    def target(self, kind, data=None):
        if kind == "brickwall":
            t = _RealRefTarget()
            t.vlist = self._r(data[0])
            t.pp, t.pk = self._perms(data[1])
            t.desc = _RefBrickwall(t.vlist.ctypes.data, t.vlist.shape[0], C.cast(t.pp, VP))
            t.ufunc = C.cast(self.lib.refdrv_real_brickwall_ufunc, VP)
            t.udata = C.cast(C.pointer(t.desc), VP)
            return t
        fn = real_fixture_map if kind == "fixture" else (lambda x, u=self._r(data): u @ x)
        return _RealRefTarget(fn)

    def _bw(self, name, t, vlist, perms, L, outs, *extra):
        vlist = self._r(vlist)
        pp, keep = self._perms(perms)
        f = np.zeros(1)
        ret = getattr(self.lib, name)(t.ufunc, t.udata, _p(vlist), vlist.shape[0], L, C.cast(pp, VP), *extra, _p(f),
                                      *[_p(o) for o in outs])
        assert ret == 0, name
        return f[0]

    def brickwall_unitary_target(self, t, vlist, perms, L):
        return self._bw("brickwall_unitary_target", t, vlist, perms, L, [])

    def brickwall_unitary_target_and_gradient(self, t, vlist, perms, L):
        dv = np.empty((len(vlist), 4, 4))
        return self._bw("brickwall_unitary_target_and_gradient", t, vlist, perms, L, [dv]), dv

    def brickwall_unitary_target_and_projected_gradient(self, t, vlist, perms, L):
        g = np.empty(6 * len(vlist))
        return self._bw("brickwall_unitary_target_and_projected_gradient", t, vlist, perms, L, [g]), g

    def brickwall_unitary_target_gradient_hessian(self, t, vlist, perms, L):
        m = 16 * len(vlist)
        dv, h = np.empty((len(vlist), 4, 4)), np.empty((m, m))
        return self._bw("brickwall_unitary_target_gradient_hessian", t, vlist, perms, L, [dv, h]), dv, h

    def brickwall_blockenc_target_gradient_hessian(self, t, vlist, perms, L):
        m = 16 * len(vlist)
        dv, h = np.empty((len(vlist), 4, 4)), np.empty((m, m))
        return self._bw("brickwall_blockenc_target_gradient_hessian", t, vlist, perms, L, [dv, h]), dv, h

    def _hvp(self, name, t, vlist, vdirs, perms, L, outs):
        vlist, vdirs = self._r(vlist), self._r(vdirs)
        pp, keep = self._perms(perms)
        f = np.zeros(1)
        ret = getattr(self.lib, name)(t.ufunc, t.udata, _p(vlist), _p(vdirs), vlist.shape[0], C.cast(pp, VP), L, _p(f),
                                      *[_p(o) for o in outs])
        assert ret == 0, name
        return f[0]

    def brickwall_unitary_target_hessian_vector_product(self, t, vlist, vdirs, perms, L):
        dv, hv = np.empty((len(vlist), 4, 4)), np.empty((len(vlist), 4, 4))
        return self._hvp("brickwall_unitary_target_hessian_vector_product", t, vlist, vdirs, perms, L, [dv, hv]), dv, hv

    def brickwall_unitary_target_projected_hessian_vector_product(self, t, vlist, vdirs, perms, L):
        g, h = np.empty(6 * len(vlist)), np.empty(6 * len(vlist))
        return (self._hvp("brickwall_unitary_target_projected_hessian_vector_product", t, vlist, vdirs, perms, L, [g, h]),
                g, h)

    def seed_rng_state(self, seed):
        rng = RngState()
        self.lib.seed_rng_state.argtypes = [C.c_uint64, C.POINTER(RngState)]
        self.lib.seed_rng_state(seed, C.byref(rng))
        return rng

    def brickwall_unitary_target_gradient_hessian_sampling(self, t, vlist, perms, L, ns, rng):
        m = 16 * len(vlist)
        dv, h = np.empty((len(vlist), 4, 4)), np.empty((m, m))
        f = self._bw("brickwall_unitary_target_gradient_hessian_sampling", t, vlist, perms, L, [dv, h], C.c_long(ns),
                     C.byref(rng))
        return f, dv, h

    def brickwall_hvp_columns(self, vlist, vdirs, perms, L, tvlist, tperms, b0, b1):
        """Grad+HVP column sum over basis columns [b0, b1) (per-gate sums; brickwall target)."""
        vlist, vdirs, tvlist = self._r(vlist), self._r(vdirs), self._r(tvlist)
        perms, tperms = _i(perms), _i(tperms)
        G = vlist.shape[0] * (L // 2)
        f, dg, hg = np.zeros(1), np.empty((G, 4, 4)), np.empty((G, 4, 4))
        ret = self.lib.refdrv_real_brickwall_hvp_columns(_p(vlist), _p(vdirs), vlist.shape[0], _p(perms), L, _p(tvlist),
                                                         tvlist.shape[0], _p(tperms), L_(b0), L_(b1), _p(f), _p(dg),
                                                         _p(hg))
        assert ret == 0
        return f[0], dg, hg

    def circuit_unitary_target_projected_hessian_vector_product(self, t, gates, dirs, wires, L):
        gates, dirs, wires = self._r(gates), self._r(dirs), _i(wires)
        f, g, h = np.zeros(1), np.empty(6 * gates.shape[0]), np.empty(6 * gates.shape[0])
        ret = self.lib.circuit_unitary_target_projected_hessian_vector_product(
            t.ufunc, t.udata, _p(gates), _p(dirs), gates.shape[0], _p(wires), L, _p(f), _p(g), _p(h))
        assert ret == 0
        return f[0], g, h

    def optimize_quantum_circuit(self, t, gstart, wires, L, niter):
        gstart, wires = self._r(gstart), _i(wires)
        ng = gstart.shape[0]
        params = _RefRtrParams(TcgParams(12 * ng, 1e-8, 1e-6), 0.125, 0.01, 0.1, None, None, None)
        f_iter, gopt = np.empty(niter + 1), np.empty_like(gstart)
        self.lib.optimize_quantum_circuit(t.ufunc, t.udata, _p(gstart), ng, L, _p(wires), C.byref(params), niter,
                                          _p(f_iter), _p(gopt))
        return f_iter, gopt

    def optimize_brickwall_circuit_hvp(self, t, vstart, perms, L, niter):
        vstart = self._r(vstart)
        nl = vstart.shape[0]
        pp, keep = self._perms(perms)
        params = _RefRtrParams(TcgParams(12 * nl, 1e-8, 1e-6), 0.125, 0.01, 0.1, None, None, None)
        f_iter, vopt = np.empty(niter + 1), np.empty_like(vstart)
        self.lib.optimize_brickwall_circuit_hvp(t.ufunc, t.udata, _p(vstart), nl, L, C.cast(pp, VP), C.byref(params),
                                                niter, _p(f_iter), _p(vopt))
        return f_iter, vopt


class _RealRefTarget:
    def __init__(self, fn=None):
        if fn is not None:
            def cb(psi_p, udata, out_p):
                psi, out = psi_p.contents, out_p.contents
                n = 1 << psi.nqubits
                x = np.ctypeslib.as_array(C.cast(psi.data, C.POINTER(C.c_double)), shape=(n,))
                np.ctypeslib.as_array(C.cast(out.data, C.POINTER(C.c_double)), shape=(n,))[:] = fn(x.copy())
                return 0

            self.cb = LINEAR_FUNC(cb)
            self.ufunc, self.udata = C.cast(self.cb, VP), None
