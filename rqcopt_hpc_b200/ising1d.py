"""The reference's ising1d example (examples/ising1d/ising1d_dynamics_opt.c and
ising1d_dynamics_opt_sampling.c) on the GPU library: optimise a brickwall circuit of
3 layers on 6 qubits to approximate expiH (the time evolution of an Ising chain),
with the full-Hessian trust region, or with its sampling form (16 Haar states, seed
42), 10 iterations, default trust-region parameters.

    python -m rqcopt_hpc_b200.ising1d ising1d_dynamics_opt_n3_init.hdf5 [--sampling] [--out result.npz]

The input file holds expiH (2^6 x 2^6 complex as [..., 2] doubles), Vlist_start
(3 x 4 x 4 complex) and perm0 .. perm2.  The program prints the wall time and the f
iterates like the reference drivers and saves Vlist (same [..., 2] layout) and f_iter.
"""
from __future__ import annotations

import argparse
import time

import numpy as np

from . import h5read, rqcopt_hpc


def load_init(arrays: dict):
    """(expiH, Vlist_start, perms) from the arrays of an ising1d init file."""
    u = np.ascontiguousarray(arrays["expiH"][..., 0] + 1j * arrays["expiH"][..., 1])
    v = arrays["Vlist_start"][..., 0] + 1j * arrays["Vlist_start"][..., 1]
    perms = [arrays[f"perm{i}"].astype(int).tolist() for i in range(v.shape[0])]
    return u, v, perms


def run(u, vlist_start, perms, niter=10, sampling=False, nsamples=16, seed=42):
    """Optimise as the reference driver does; returns (vlist_opt, f_iter, seconds)."""
    nqubits = int(u.shape[0]).bit_length() - 1
    t0 = time.perf_counter()
    if sampling:
        vopt, f_iter = rqcopt_hpc.optimize_brickwall_circuit(nqubits, u, list(vlist_start), perms, niter,
                                                            nsamples=nsamples, seed=seed)
    else:
        vopt, f_iter = rqcopt_hpc.optimize_brickwall_circuit(nqubits, u, list(vlist_start), perms, niter)
    return vopt, f_iter, time.perf_counter() - t0


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("init", help="ising1d_dynamics_opt_n3_init.hdf5")
    ap.add_argument("--sampling", action="store_true", help="sampling trace estimator (16 samples, seed 42)")
    ap.add_argument("--niter", type=int, default=10)
    ap.add_argument("--out", default=None, help="write Vlist and f_iter to this .npz file")
    a = ap.parse_args(argv)
    u, v, perms = load_init(h5read.read_all(a.init))
    vopt, f_iter, wall = run(u, v, perms, a.niter, a.sampling)
    print(f"wall time: {wall:g}")
    for i, f in enumerate(f_iter):
        print(f"f_iter[{i}] = {f:.12f}")
    if a.out:
        np.savez(a.out, Vlist=np.stack([vopt.real, vopt.imag], axis=-1), f_iter=f_iter)


if __name__ == "__main__":
    main()
