"""The reference's example drivers on the GPU library.

ising1d (examples/ising1d/ising1d_dynamics_opt.c, ising1d_dynamics_opt_sampling.c):
a brickwall of 3 layers on 6 qubits approximating expiH (the time evolution of an
Ising chain) with the full-Hessian trust region, or its sampling form (16 Haar
states, seed 42); input expiH, Vlist_start, perm0 .. perm2.

molecular (examples/molecular/molecular_dynamics_opt.c): a general circuit of 18
two-qubit gates on 5 qubits approximating expiH (a molecular Hamiltonian's time
evolution) with the HVP trust region; input expiH, gates_start, wires.

Both run 10 iterations with the default trust-region parameters and a dense target,
as the reference drivers do.

    python -m rqcopt_hpc_b200.examples ising1d ising1d_dynamics_opt_n3_init.hdf5 [--sampling] [--out r.npz]
    python -m rqcopt_hpc_b200.examples molecular molecular_dynamics_opt_init.hdf5 [--out r.npz]

The programs print the wall time and the f iterates like the reference drivers and
save the optimised gates (complex as [..., 2] doubles, the reference's layout) and
f_iter.
"""
from __future__ import annotations

import argparse
import time

import numpy as np

from . import h5read, rqcopt_hpc


def _cplx(a):
    return a[..., 0] + 1j * a[..., 1]


def load_ising1d(arrays: dict):
    """(expiH, Vlist_start, perms) from the arrays of an ising1d init file."""
    v = _cplx(arrays["Vlist_start"])
    perms = [arrays[f"perm{i}"].astype(int).tolist() for i in range(v.shape[0])]
    return np.ascontiguousarray(_cplx(arrays["expiH"])), v, perms


def load_molecular(arrays: dict):
    """(expiH, gates_start, wires) from the arrays of the molecular init file."""
    return (np.ascontiguousarray(_cplx(arrays["expiH"])), _cplx(arrays["gates_start"]),
            arrays["wires"].astype(int).tolist())


def _nq(u):
    return int(u.shape[0]).bit_length() - 1


def run_ising1d(u, vlist_start, perms, niter=10, sampling=False, nsamples=16, seed=42):
    """The ising1d drivers; returns (vlist_opt, f_iter, seconds)."""
    t0 = time.perf_counter()
    kw = {"nsamples": nsamples, "seed": seed} if sampling else {}
    vopt, f_iter = rqcopt_hpc.optimize_brickwall_circuit(_nq(u), u, list(vlist_start), perms, niter, **kw)
    return vopt, f_iter, time.perf_counter() - t0


def run_molecular(u, gates_start, wires, niter=10):
    """The molecular driver; returns (gates_opt, f_iter, seconds)."""
    t0 = time.perf_counter()
    gopt, f_iter = rqcopt_hpc.optimize_quantum_circuit(_nq(u), u, list(gates_start), wires, niter)
    return gopt, f_iter, time.perf_counter() - t0


def main(argv=None):
    ap = argparse.ArgumentParser(description="the reference's example drivers on the GPU library")
    ap.add_argument("example", choices=["ising1d", "molecular"])
    ap.add_argument("init", help="the example's *_init.hdf5 input file")
    ap.add_argument("--sampling", action="store_true", help="ising1d: sampling trace estimator (16 samples, seed 42)")
    ap.add_argument("--niter", type=int, default=10)
    ap.add_argument("--out", default=None, help="write the optimised gates and f_iter to this .npz file")
    a = ap.parse_args(argv)
    arrays = h5read.read_all(a.init)
    if a.example == "ising1d":
        gates, f_iter, wall = run_ising1d(*load_ising1d(arrays), a.niter, a.sampling)
        key = "Vlist"
    else:
        gates, f_iter, wall = run_molecular(*load_molecular(arrays), a.niter)
        key = "gates"
    print(f"wall time: {wall:g}")
    for i, f in enumerate(f_iter):
        print(f"f_iter[{i}] = {f:.12f}")
    if a.out:
        np.savez(a.out, **{key: np.stack([gates.real, gates.imag], axis=-1), "f_iter": f_iter})


if __name__ == "__main__":
    main()
