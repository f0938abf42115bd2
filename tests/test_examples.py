"""The reference's ising1d example (examples/ising1d): its input and the outputs the
reference stored for it (full-Hessian trust region, and its sampling form with 16
samples and seed 42; 10 iterations each) as golden vectors.

CPU: the HDF5 reader reads the example files (where the reference is present); the
compiled reference module reproduces the stored full-Hessian run exactly, and the
oracle restatement to 1e-12 (f iterates) and 1e-9 (gates).  GPU: the library through
the Python module to 1e-10 and 1e-9.

The sampling run is pinned through its first 8 iterates (f_iter[0..7]).  Its Haar
states come from libm's log and sin, whose last bits differ between machines.  The
compiled reference here matches the stored run exactly up to f_iter[7], then departs
from it at the 5e-7 relative level as the trust region nears convergence."""
import os

import numpy as np
import pytest

from helpers import GOLDEN

from oracle.oracle import reference_module

EX = os.path.join(GOLDEN, "examples")
REF_EXAMPLES = "/root/reference/examples/ising1d"


def _load(name):
    with np.load(os.path.join(EX, f"{name}.npz")) as z:
        return {k: z[k] for k in z.files}


def _init():
    from rqcopt_hpc_b200.ising1d import load_init
    return load_init(_load("ising1d_n3_init"))


def _expected(name):
    d = _load(name)
    return d["Vlist"][..., 0] + 1j * d["Vlist"][..., 1], d["f_iter"]


@pytest.mark.skipif(not os.path.isdir(REF_EXAMPLES), reason="reference examples not present")
def test_reader_reads_the_example_files():
    from rqcopt_hpc_b200 import h5read
    for f, name in [("ising1d_dynamics_opt_n3_init.hdf5", "ising1d_n3_init"),
                    ("ising1d_dynamics_opt_n3.hdf5", "ising1d_n3")]:
        a, b = h5read.read_all(os.path.join(REF_EXAMPLES, f)), _load(name)
        assert sorted(a) == sorted(b) and all(np.array_equal(a[k], b[k]) for k in a)


@pytest.mark.skipif(reference_module() is None, reason="reference module build not present")
@pytest.mark.parametrize("sampling", [False, True])
def test_reference_module_reproduces_stored_outputs(sampling):
    u, v, perms = _init()
    ref = reference_module()
    if sampling:
        vo, fi = ref.optimize_brickwall_circuit(6, u, list(v), perms, 10, nsamples=16, seed=42)
    else:
        vo, fi = ref.optimize_brickwall_circuit(6, u, list(v), perms, 10)
    ve, fe = _expected("ising1d_sampling_n3" if sampling else "ising1d_n3")
    if sampling:
        assert np.max(np.abs(fi[:8] - fe[:8])) <= 1e-14 * np.max(np.abs(fe))
    else:
        assert np.array_equal(fi, fe) and np.array_equal(vo, ve)


@pytest.mark.parametrize("sampling", [False, True])
def test_oracle_reproduces_stored_outputs(oracle, sampling):
    u, v, perms = _init()
    t = oracle.target("dense", u)
    p = np.asarray(perms, np.int32)
    if sampling:
        fi, vo = oracle.optimize_brickwall_circuit_hmat_sampling(t, v, p, 6, 16, oracle.seed_rng_state(42), 10)[:2]
    else:
        fi, vo = oracle.optimize_brickwall_circuit_hmat(t, v, p, 6, 10)[:2]
    ve, fe = _expected("ising1d_sampling_n3" if sampling else "ising1d_n3")
    n = 8 if sampling else len(fe)
    assert np.max(np.abs(fi[:n] - fe[:n])) <= 1e-12 * np.max(np.abs(fe))
    if not sampling:
        assert np.max(np.abs(vo - ve)) <= 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("sampling", [False, True])
def test_gpu_reproduces_stored_outputs(gpu, sampling):
    from rqcopt_hpc_b200.ising1d import run
    u, v, perms = _init()
    vo, fi, _ = run(u, v, perms, 10, sampling)
    ve, fe = _expected("ising1d_sampling_n3" if sampling else "ising1d_n3")
    n = 8 if sampling else len(fe)
    assert np.max(np.abs(fi[:n] - fe[:n])) <= 1e-10 * np.max(np.abs(fe))
    if not sampling:
        assert np.max(np.abs(vo - ve)) <= 1e-9
