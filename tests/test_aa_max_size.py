"""The largest states the single-state passes take: complex128 at L=30 and complex64
at L=31, 16 GiB per state (offsets beyond 2^31 amplitudes and 2^32 bytes); one
qubit less each where the device has less than 72 GiB free (the file runs first
among the GPU tests, before the evaluation engines have sized their workspaces).

At this size no CPU checker finishes, so the checks are size-independent
properties of apply_quantum_circuit (src/quantum_circuit.c:13-35):
- the circuit followed by its adjoint gates in reverse order returns the input
  (complex128 1e-12, complex64 1e-5, absolute per amplitude of a unit-norm state);
- the fused passes (4 gates per HBM round trip, TMA tiles) equal one kernel per
  gate (the same 4x4 products per amplitude in the same order) to 1e-14 / 1e-6;
- the norm stays 1.
The gates act on random distinct qubit pairs, including the highest qubits, so the
group members of a gate lie up to 2^30 amplitudes apart.  Three states and the
library's per-gate scratch hold four states (64 GiB at full size); comparisons run
in slices of 2^26 amplitudes.
"""
import ctypes

import numpy as np
import pytest

from helpers import haar_unitary

pytestmark = pytest.mark.gpu

G = 24
SLICE = 1 << 26


def _max_abs_diff(torch, a, b):
    m = 0.0
    for s in range(0, a.numel(), SLICE):
        m = max(m, float(torch.max(torch.abs(a[s:s + SLICE] - b[s:s + SLICE]))))
    return m


def _norm(torch, a):
    acc = 0.0
    for s in range(0, a.numel(), SLICE):
        acc += float(torch.sum(torch.abs(a[s:s + SLICE]) ** 2, dtype=torch.float64))
    return acc ** 0.5


@pytest.fixture
def _big(gpu):
    import torch
    torch.cuda.empty_cache()
    free, total = torch.cuda.mem_get_info()
    if free < (40 << 30):
        pytest.skip(f"needs 40 GiB of free device memory, {free >> 30} GiB free")
    yield torch, 0 if free >= (72 << 30) else 1
    gpu.set_gates_per_pass(4)
    gpu.set_autotune(True)
    torch.cuda.empty_cache()


@pytest.mark.parametrize("L0,prec", [(30, "c128"), (31, "c64")])
def test_largest_states_round_trip_and_fused_equals_per_gate(gpu, _big, L0, prec):
    torch, less = _big
    L = L0 - less
    from rqcopt_hpc_b200.abi import Statevector
    lib = gpu.lib()
    rng = np.random.default_rng(300 + L)
    gates = np.stack([haar_unitary(rng) for _ in range(G)])
    wires = np.array([rng.choice(L, 2, replace=False) for _ in range(G)], np.int32)
    wires[0] = (0, L - 1)          # the most and least significant qubits
    wires[1] = (L - 1, 1)
    adj = np.ascontiguousarray(np.conj(np.transpose(gates[::-1], (0, 2, 1))))
    wrev = np.ascontiguousarray(wires[::-1])
    dtype, tol, same = (torch.complex128, 1e-12, 1e-14) if prec == "c128" else (torch.complex64, 1e-5, 1e-6)
    gen = torch.Generator(device="cuda").manual_seed(L)
    psi = torch.randn(1 << L, dtype=dtype, device="cuda", generator=gen)
    psi /= _norm(torch, psi)
    out = torch.empty_like(psi)
    if prec == "c128":
        def run(g, w, a, b):
            sa, sb = Statevector(a.data_ptr(), L), Statevector(b.data_ptr(), L)
            return lib.apply_quantum_circuit(g.ctypes.data, G, w.ctypes.data, ctypes.byref(sa), ctypes.byref(sb))
    else:
        def run(g, w, a, b):
            return lib.rqcopt_apply_quantum_circuit_c64(g.ctypes.data, G, w.ctypes.data, a.data_ptr(), b.data_ptr(), L)
    gpu.set_gates_per_pass(4)
    assert run(gates, wires, psi, out) == 0
    torch.cuda.synchronize()
    assert abs(_norm(torch, out) - 1) <= tol
    back = torch.empty_like(psi)
    assert run(adj, wrev, out, back) == 0
    torch.cuda.synchronize()
    assert _max_abs_diff(torch, back, psi) <= tol
    del back
    gpu.set_gates_per_pass(1)
    ref = torch.empty_like(psi)
    assert run(gates, wires, psi, ref) == 0
    torch.cuda.synchronize()
    assert _max_abs_diff(torch, out, ref) <= same
