"""The allocation-free gate backward pass, rqcopt_apply_gate_backward_noalloc.

It exists for callers that cannot allocate device memory when they need the
pass (their device memory belongs to their own pool, or they run on a thread
that must not take the synchronisation an allocation implies).  It must give
what the ordinary apply_gate_backward gives, call after call, from its static
scratch.  This file is collected last so that a failure here stops a `-x` run
only after every other test has run; it also passes on its own in a fresh
process.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import crandn, rel_err

pytestmark = pytest.mark.gpu

MAX_QUBITS = 25


def _entry(gpu):
    from rqcopt_hpc_b200.abi import Statevector
    f = gpu.lib().rqcopt_apply_gate_backward_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(Statevector), C.POINTER(Statevector),
                  C.POINTER(Statevector), C.c_void_p, C.c_void_p]
    return f, Statevector


def _on_device(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


def _call(f, SV, V, i, j, psi_d, dout_d, dpsi_d, L, dgate_ptr, stream=None):
    return f(V.ctypes.data, i, j, C.byref(SV(psi_d.data_ptr(), L)), C.byref(SV(dout_d.data_ptr(), L)),
             C.byref(SV(dpsi_d.data_ptr(), L)), dgate_ptr, stream)


def test_noalloc_matches_apply_gate_backward_on_two_calls(gpu, oracle):
    import torch
    f, SV = _entry(gpu)
    rng = np.random.default_rng(7)
    # two calls in a row: a multi-tile state, then a single-tile state with the wires swapped
    for L, i, j in [(18, 3, 11), (9, 7, 2)]:
        V = np.ascontiguousarray(crandn((4, 4), rng))
        psi, dout = crandn(1 << L, rng), crandn(1 << L, rng)
        dpsi_ref, dV_ref = gpu.apply_gate_backward(V, i, j, psi, dout)
        dpsi_orc, dV_orc = oracle.apply_gate_backward(V, i, j, psi, dout)

        psi_d, dout_d = _on_device(psi), _on_device(dout)
        dpsi_d = torch.empty_like(psi_d)
        dV = np.zeros((4, 4), np.complex128)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        rc = _call(f, SV, V, i, j, psi_d, dout_d, dpsi_d, L, dV.ctypes.data)
        free_after = torch.cuda.mem_get_info()[0]
        assert rc == 0
        assert rel_err(dpsi_d.cpu().numpy(), dpsi_ref) <= 1e-12
        assert rel_err(dV, dV_ref) <= 1e-12
        # and directly against the CPU oracle of the reference's apply_gate_backward
        assert rel_err(dpsi_d.cpu().numpy(), dpsi_orc) <= 1e-12
        assert rel_err(dV, dV_orc) <= 1e-12
        if L == 9:   # the scratch was set up by the first call; no device memory is taken now
            assert free_after == free_before


def test_noalloc_at_the_size_limit_and_the_smallest_state(gpu, oracle):
    """25 qubits fill every tile slot of the static scratch; 2 qubits use one group."""
    import torch
    f, SV = _entry(gpu)
    rng = np.random.default_rng(11)
    for L, i, j in [(MAX_QUBITS, 24, 0), (2, 1, 0)]:
        V = np.ascontiguousarray(crandn((4, 4), rng))
        psi, dout = crandn(1 << L, rng), crandn(1 << L, rng)
        dpsi_orc, dV_orc = oracle.apply_gate_backward(V, i, j, psi, dout)
        psi_d, dout_d = _on_device(psi), _on_device(dout)
        del psi, dout
        dpsi_d = torch.empty_like(psi_d)
        dV = np.zeros((4, 4), np.complex128)
        assert _call(f, SV, V, i, j, psi_d, dout_d, dpsi_d, L, dV.ctypes.data) == 0
        assert rel_err(dpsi_d.cpu().numpy(), dpsi_orc) <= 1e-12
        assert rel_err(dV, dV_orc) <= 1e-12
        del psi_d, dout_d, dpsi_d
        torch.cuda.empty_cache()


def test_noalloc_on_a_caller_stream_with_device_dgate(gpu, oracle):
    """Work issued on the caller's own stream; dgate in device memory."""
    import torch
    f, SV = _entry(gpu)
    rng = np.random.default_rng(13)
    L, i, j = 14, 5, 9
    V = np.ascontiguousarray(crandn((4, 4), rng))
    psi, dout = crandn(1 << L, rng), crandn(1 << L, rng)
    dpsi_orc, dV_orc = oracle.apply_gate_backward(V, i, j, psi, dout)
    psi_d, dout_d = _on_device(psi), _on_device(dout)
    dpsi_d = torch.empty_like(psi_d)
    dV_d = torch.zeros((4, 4), dtype=torch.complex128, device="cuda")
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    for _ in range(2):
        assert _call(f, SV, V, i, j, psi_d, dout_d, dpsi_d, L, dV_d.data_ptr(), C.c_void_p(s.cuda_stream)) == 0
        assert rel_err(dpsi_d.cpu().numpy(), dpsi_orc) <= 1e-12
        assert rel_err(dV_d.cpu().numpy(), dV_orc) <= 1e-12


def test_noalloc_rejects_states_beyond_the_scratch(gpu):
    import torch
    f, SV = _entry(gpu)
    V = np.eye(4, dtype=np.complex128)
    small = torch.zeros(4, dtype=torch.complex128, device="cuda")
    dV = np.zeros((4, 4), np.complex128)
    # the qubit count is checked before any amplitude is touched
    L = MAX_QUBITS + 1
    rc = f(V.ctypes.data, 0, 1, C.byref(SV(small.data_ptr(), L)), C.byref(SV(small.data_ptr(), L)),
           C.byref(SV(small.data_ptr(), L)), dV.ctypes.data, None)
    assert rc == -6


def test_noalloc_rejects_host_statevectors(gpu):
    f, SV = _entry(gpu)
    V = np.eye(4, dtype=np.complex128)
    psi = np.zeros(16, np.complex128)
    out = np.zeros(16, np.complex128)
    dV = np.zeros((4, 4), np.complex128)
    rc = f(V.ctypes.data, 0, 1, C.byref(SV(psi.ctypes.data, 4)), C.byref(SV(psi.ctypes.data, 4)),
           C.byref(SV(out.ctypes.data, 4)), dV.ctypes.data, None)
    assert rc == -6
