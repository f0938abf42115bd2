"""The reference's Python module (pymodule/rqcopt_module.c, module `rqcopt_hpc`) on the
GPU library: the same two functions, arguments, return values, argument checks and
exception types.

    import rqcopt_hpc_b200.rqcopt_hpc as rqcopt_hpc
    gates_opt, f_iter = rqcopt_hpc.optimize_quantum_circuit(nqubits, U, gates_start, wires, niter)
    Vlist_opt, f_iter = rqcopt_hpc.optimize_brickwall_circuit(L, U, Vlist_start, perms, niter, nsamples=0, seed=42)

U is the dense 2^L x 2^L target (complex double, C-contiguous), applied through the
library's dense target (`rqcopt_dense_ufunc`, a column copy per basis column).  The
general-circuit optimiser is the trust region with Hessian-vector products
(src/circuit_opt.c:104-124), the brickwall optimiser the full-Hessian one
(src/brickwall_opt.c:159-186) or, with nsamples > 0, its sampling form seeded with
`seed` (src/brickwall_opt.c:244-265), all with the default trust-region parameters
(pymodule/rqcopt_module.c:220-226, 485-503).
"""
from __future__ import annotations

from collections.abc import Sequence

import numpy as np

from . import gpu


def _check_u(U, n, what):
    if not isinstance(U, np.ndarray):
        U = np.asarray(U)
    if U.ndim != 2:
        raise ValueError(f"'U' must have degree 2, received {U.ndim}")
    if U.shape[0] != 1 << n or U.shape[1] != 1 << n:
        raise ValueError(f"'U' must have dimensions 2^{what} x 2^{what}, received a {U.shape[0]} x {U.shape[1]} "
                         f"matrix and {what} = {n}")
    if U.dtype != np.complex128:
        raise TypeError("'U' must have 'complex double' entries")
    if not U.flags["C_CONTIGUOUS"]:
        raise SyntaxError("'U' does not have contiguous C storage format")
    return U


def _gates(seq, name):
    out = []
    for i, g in enumerate(seq):
        try:
            a = np.asarray(g, dtype=np.complex128)
        except (TypeError, ValueError):
            raise SyntaxError(f"cannot interpret {name}[{i}] as complex matrix") from None
        if a.ndim != 2 or a.shape != (4, 4):
            dims = a.shape if a.ndim == 2 else (a.size, 1)
            raise ValueError(f"{name}[{i}] must be a 4 x 4 matrix, received a {dims[0]} x {dims[1]} matrix")
        out.append(a)
    return np.ascontiguousarray(np.stack(out))


def _is_seq(x):
    return isinstance(x, (Sequence, np.ndarray)) and not isinstance(x, (str, bytes))


def optimize_quantum_circuit(nqubits, U, gates_start, wires, niter):
    """Optimize the two-qubit gates in a quantum circuit to approximate a unitary matrix
    using a trust-region method; returns (gates_opt, f_iter)."""
    if nqubits <= 0:
        raise ValueError(f"'nqubits' must be positive, received nqubits = {nqubits}")
    U = _check_u(U, nqubits, "nqubits")
    if not _is_seq(gates_start):
        raise SyntaxError("'gates_start' must be a sequence")
    if len(gates_start) == 0:
        raise ValueError("sequence of initial quantum gates cannot be empty")
    if not _is_seq(wires):
        raise SyntaxError("'wires' must be a sequence")
    if len(wires) != len(gates_start):
        raise ValueError("'gates_start' and 'wires' sequences must have the same length")
    if niter <= 0:
        raise ValueError(f"'niter' must be a positive integer, received {niter}")
    gates = _gates(gates_start, "gates_start")
    w = np.empty((len(wires), 2), np.int32)
    for i, pair in enumerate(wires):
        if not _is_seq(pair):
            raise SyntaxError(f"'wires[{i}]' must be a sequence")
        if len(pair) != 2:
            raise ValueError(f"'wires[{i}]' must be a sequence of length 2")
        for j in range(2):
            try:
                w[i, j] = int(pair[j])
            except (TypeError, ValueError):
                raise ValueError(f"cannot interpret 'wires[{i}][{j}]' as integer") from None
            if not 0 <= w[i, j] < nqubits:
                raise ValueError(f"index 'wires[{i}][{j}] = {w[i, j]}' outside of [0, nqubits) index range")
        if w[i, 0] == w[i, 1]:
            raise ValueError(f"wire indices for gate {i} are not distinct, received index {w[i, 0]} twice")
    f_iter, gates_opt = gpu.optimize_quantum_circuit(gpu.Target(dense=U), gates, w, nqubits, niter)
    return gates_opt, f_iter


def optimize_brickwall_circuit(L, U, Vlist_start, perms, niter, nsamples=0, seed=42):
    """Optimize the quantum gates in a brickwall layout to approximate a unitary matrix
    using a trust-region method; returns (Vlist_opt, f_iter)."""
    if L <= 0 or L % 2 != 0:
        raise ValueError(f"'L' must be positive and even, received L = {L}")
    U = _check_u(U, L, "L")
    if not _is_seq(Vlist_start):
        raise SyntaxError("'Vlist_start' must be a sequence")
    nlayers = len(Vlist_start)
    if nlayers == 0:
        raise ValueError("sequence of initial quantum gates cannot be empty")
    if not _is_seq(perms):
        raise SyntaxError("'perms' must be a sequence")
    if len(perms) != nlayers:
        raise ValueError("'Vlist_start' and 'perms' sequences must have the same length (equal to the number of layers)")
    if niter <= 0:
        raise ValueError(f"'niter' must be a positive integer, received {niter}")
    if nsamples < 0:
        raise ValueError("'nsamples' cannot be negative")
    vlist = _gates(Vlist_start, "Vlist_start")
    p = np.empty((nlayers, L), np.int32)
    for i, perm in enumerate(perms):
        if not _is_seq(perm):
            raise SyntaxError(f"'perms[{i}]' must be a sequence")
        if len(perm) != L:
            raise ValueError(f"'perms[{i}]' must be a sequence of length L = {L}")
        for j in range(L):
            try:
                p[i, j] = int(perm[j])
            except (TypeError, ValueError):
                raise ValueError(f"cannot interpret 'perms[{i}][{j}]' as integer") from None
        if sorted(p[i].tolist()) != list(range(L)):
            raise ValueError(f"'perms[{i}]' is not a valid permutation")
    target = gpu.Target(dense=U)
    if nsamples == 0:
        f_iter, vopt = gpu.optimize_brickwall_circuit_hmat(target, vlist, p, L, niter)
    else:
        rng = gpu.seed_rng_state(seed)
        f_iter, vopt = gpu.optimize_brickwall_circuit_hmat_sampling(target, vlist, p, L, nsamples, rng, niter)
    return vopt, f_iter
