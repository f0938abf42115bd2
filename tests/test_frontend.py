"""The Python front end (rqcopt_hpc_b200.rqcopt_hpc) against the reference's own Python
module (pymodule/rqcopt_module.c, built in oracle/_ref): the same exceptions for invalid
arguments (CPU), and the same optimisation results on the GPU (f iterates to 1e-10,
gates to 1e-9), exact and sampled."""
import numpy as np
import pytest

from helpers import haar_unitary, periodic_perms

from oracle.oracle import reference_module

REF = reference_module()
needs_ref = pytest.mark.skipif(REF is None, reason="reference module build not present")


def _unitary(n, seed):
    rng = np.random.default_rng(seed)
    z = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / np.sqrt(2)
    q, r = np.linalg.qr(z)
    return np.ascontiguousarray(q * (np.diagonal(r) / np.abs(np.diagonal(r))))


def _brickwall_args(L=6, nl=3, seed=1):
    rng = np.random.default_rng(seed)
    return L, _unitary(1 << L, seed + 1), [haar_unitary(rng) for _ in range(nl)], periodic_perms(L, nl).tolist()


INVALID_BRICKWALL = [
    lambda a: (5,) + a[1:],                                   # odd L
    lambda a: (a[0], a[1][:8]) + a[2:],                        # wrong U dimensions
    lambda a: (a[0], a[1].real.copy()) + a[2:],                # real U
    lambda a: (a[0], np.asfortranarray(a[1])) + a[2:],         # not C-contiguous
    lambda a: (a[0], a[1], [], a[3]),                          # no gates
    lambda a: (a[0], a[1], a[2], a[3][:2]),                    # perms length
    lambda a: (a[0], a[1], [np.eye(3)] + a[2][1:], a[3]),      # 3 x 3 gate
    lambda a: (a[0], a[1], a[2], [[0, 0, 1, 2, 3, 4]] + a[3][1:]),   # not a permutation
    lambda a: (a[0], a[1], a[2], [[0, 1, 2]] + a[3][1:]),      # perm length
]


@needs_ref
@pytest.mark.parametrize("k", range(len(INVALID_BRICKWALL)))
def test_brickwall_argument_errors_match_reference(k):
    from rqcopt_hpc_b200 import rqcopt_hpc
    args = INVALID_BRICKWALL[k](_brickwall_args())
    with pytest.raises(Exception) as ours:
        rqcopt_hpc.optimize_brickwall_circuit(*args, 2)
    with pytest.raises(Exception) as theirs:
        REF.optimize_brickwall_circuit(*args, 2)
    assert type(ours.value) is type(theirs.value)
    assert str(ours.value) == str(theirs.value)


@needs_ref
def test_circuit_argument_errors_match_reference():
    from rqcopt_hpc_b200 import rqcopt_hpc
    U = _unitary(16, 3)
    gates = [haar_unitary(np.random.default_rng(k)) for k in range(3)]
    for args in [(4, U, gates, [[0, 1], [1, 2]], 2), (4, U, gates, [[0, 1], [1, 1], [2, 3]], 2),
                 (4, U, gates, [[0, 1], [1, 7], [2, 3]], 2), (0, U, gates, [[0, 1]] * 3, 2),
                 (4, U, gates, [[0, 1], [1, 2], [2, 3]], 0)]:
        with pytest.raises(Exception) as ours:
            rqcopt_hpc.optimize_quantum_circuit(*args)
        with pytest.raises(Exception) as theirs:
            REF.optimize_quantum_circuit(*args)
        assert type(ours.value) is type(theirs.value) and str(ours.value) == str(theirs.value)


@needs_ref
@pytest.mark.gpu
@pytest.mark.parametrize("nsamples", [0, 24])
def test_optimize_brickwall_circuit_matches_reference_module(gpu, nsamples):
    from rqcopt_hpc_b200 import rqcopt_hpc
    L, U, vlist, perms = _brickwall_args()
    v, f = rqcopt_hpc.optimize_brickwall_circuit(L, U, vlist, perms, 4, nsamples=nsamples, seed=7)
    vr, fr = REF.optimize_brickwall_circuit(L, U, vlist, perms, 4, nsamples=nsamples, seed=7)
    assert np.max(np.abs(f - fr)) <= 1e-10 * np.max(np.abs(fr))
    assert np.max(np.abs(v - vr)) <= 1e-9


@needs_ref
@pytest.mark.gpu
def test_optimize_quantum_circuit_matches_reference_module(gpu):
    from rqcopt_hpc_b200 import rqcopt_hpc
    U = _unitary(16, 5)
    rng = np.random.default_rng(6)
    gates = [haar_unitary(rng) for _ in range(5)]
    wires = [[0, 1], [2, 3], [1, 2], [3, 0], [0, 2]]
    g, f = rqcopt_hpc.optimize_quantum_circuit(4, U, gates, wires, 4)
    gr, fr = REF.optimize_quantum_circuit(4, U, gates, wires, 4)
    assert np.max(np.abs(f - fr)) <= 1e-10 * np.max(np.abs(fr))
    assert np.max(np.abs(g - gr)) <= 1e-9
