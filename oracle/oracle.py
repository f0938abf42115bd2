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

    def circuit_unitary_target_hessian_vector_product(self, tgt, gates, dirs, wires, L):
        gates, dirs, wires = _c(gates), _c(dirs), _i(wires)
        f = np.zeros(1, np.complex128)
        dg = np.empty((gates.shape[0], 4, 4), np.complex128)
        hg = np.empty_like(dg)
        self.lib.orc_circuit_target_hvp(tgt.ufunc, tgt.udata, _p(gates), _p(dirs), gates.shape[0], _p(wires), L, L_(0),
                                        L_(1 << L), _p(f), _p(dg), _p(hg))
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
