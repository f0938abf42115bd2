"""transpose_statevector (src/statevector.c:72-98) of both libraries against the
reference's golden vectors (test/test_statevector.c:23-64, 1e-12); it runs on the
host, so these tests need no GPU."""
import os

import numpy as np
import pytest

from helpers import GOLDEN, golden, udist


def test_transpose_statevector_complex():
    from rqcopt_hpc_b200 import gpu
    d = golden("transpose_statevector")
    assert udist(gpu.transpose_statevector(d["psi"], d["perm"]), d["chi"]) <= 1e-12
    with pytest.raises(gpu.RqcError) as e:
        gpu.transpose_statevector(d["psi"], np.zeros_like(d["perm"]))
    assert e.value.code == -6


def test_transpose_statevector_real():
    from rqcopt_hpc_b200 import real
    with np.load(os.path.join(GOLDEN, "real", "transpose_statevector.npz")) as z:
        d = {k: z[k] for k in z.files}
    assert udist(real.transpose_statevector(d["psi"], d["perm"]), d["chi"]) <= 1e-12
    with pytest.raises(real.RqcError) as e:
        real.transpose_statevector(d["psi"], np.arange(d["perm"].size + 1)[1:])
    assert e.value.code == -6


def test_transpose_is_a_permutation_of_qubits():
    """Transposing with perm and then with its inverse is the identity, and the result is
    numpy's axis transposition of the state as an L-axis tensor (qubit 0 the first
    axis): output axis a is input axis perm[a]."""
    from rqcopt_hpc_b200 import gpu
    rng = np.random.default_rng(3)
    L = 7
    psi = rng.standard_normal(1 << L) + 1j * rng.standard_normal(1 << L)
    perm = rng.permutation(L)
    inv = np.argsort(perm)
    assert np.array_equal(gpu.transpose_statevector(gpu.transpose_statevector(psi, perm), inv), psi)
    expected = np.transpose(psi.reshape((2,) * L), axes=perm).ravel()
    assert np.array_equal(gpu.transpose_statevector(psi, perm), expected)
