"""Convert the reference's HDF5 golden vectors for the hot path into .npz fixtures.

Run in a checkout that has the reference project next to it:

    python tests/golden/make_golden.py /root/reference/test/data

Each ``test_<name>_cplx.hdf5`` (complex-circuit fixtures of the reference's
``test/data`` directory, generated there by ``test/test_*.py``) becomes
``tests/golden/<name>.npz`` with the same dataset names and the interleaved
(real, imag) layout unchanged; the real-build fixtures (``test_<name>_real.hdf5``)
go to ``tests/golden/real/``, and the ising1d example's input and the outputs the
reference stored for it (``examples/ising1d/*.hdf5``), and the same for the
molecular example, to ``tests/golden/examples/``.
The reader is ``rqcopt_hpc_b200.h5read``.
"""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
from rqcopt_hpc_b200 import h5read  # noqa: E402

FIXTURES = [
    "apply_gate", "apply_gate_backward", "apply_quantum_circuit", "quantum_circuit_backward",
    "quantum_circuit_gates_hessian_vector_product", "apply_brickwall_unitary", "brickwall_unitary_backward",
    "circuit_unitary_target", "circuit_unitary_target_and_gradient",
    "circuit_unitary_target_hessian_vector_product", "circuit_unitary_target_projected_hessian_vector_product",
    "brickwall_unitary_target", "brickwall_unitary_target_and_gradient",
    "brickwall_unitary_target_and_projected_gradient", "brickwall_unitary_target_hessian_vector_product",
    "brickwall_unitary_target_projected_hessian_vector_product",
    "real_to_tangent", "project_tangent", "polar_factor", "multiply", "transpose_statevector",
    # full-Hessian path
    "apply_gate_to_array", "apply_gate_placeholder", "brickwall_unitary_backward_hessian",
    "brickwall_unitary_target_gradient_hessian", "brickwall_unitary_target_gradient_vector_hessian_matrix",
    # sampling estimator
    "brickwall_unitary_target_sampling", "brickwall_unitary_target_gradient_hessian_sampling",
    "brickwall_unitary_target_gradient_vector_hessian_matrix_sampling",
    # block-encoding target
    "brickwall_blockenc_target", "brickwall_blockenc_target_and_gradient",
    "brickwall_blockenc_target_and_gradient_vector", "brickwall_blockenc_target_gradient_hessian",
    "brickwall_blockenc_target_gradient_vector_hessian_matrix",
]


# the reference's real-orthogonal build (``test_<name>_real.hdf5``) -> ``tests/golden/real/<name>.npz``
REAL_FIXTURES = [
    "apply_gate", "apply_gate_backward", "apply_gate_to_array", "apply_gate_placeholder", "apply_quantum_circuit",
    "quantum_circuit_backward", "quantum_circuit_gates_hessian_vector_product", "apply_brickwall_unitary",
    "brickwall_unitary_backward", "brickwall_unitary_backward_hessian", "circuit_unitary_target",
    "circuit_unitary_target_and_gradient", "circuit_unitary_target_hessian_vector_product",
    "circuit_unitary_target_projected_hessian_vector_product", "brickwall_unitary_target",
    "brickwall_unitary_target_and_gradient", "brickwall_unitary_target_hessian_vector_product",
    "brickwall_unitary_target_projected_hessian_vector_product", "brickwall_unitary_target_gradient_hessian",
    "brickwall_unitary_target_sampling", "brickwall_unitary_target_gradient_hessian_sampling",
    "brickwall_blockenc_target", "brickwall_blockenc_target_and_gradient", "brickwall_blockenc_target_gradient_hessian",
    "real_to_tangent", "project_tangent", "polar_factor", "multiply", "transpose_statevector",
]


# the example inputs and the outputs the reference stored for them: ising1d (examples/ising1d),
# ising1d_dynamics_opt.c (full-Hessian trust region, 10 iterations) and
# ising1d_dynamics_opt_sampling.c (16 samples, seed 42)
EXAMPLES = {
    "ising1d_n3_init": "ising1d/ising1d_dynamics_opt_n3_init.hdf5",
    "ising1d_n3": "ising1d/ising1d_dynamics_opt_n3.hdf5",
    "ising1d_sampling_n3": "ising1d/ising1d_dynamics_opt_sampling_n3.hdf5",
    # examples/molecular/molecular_dynamics_opt.c: general circuit, HVP trust region
    "molecular_init": "molecular/molecular_dynamics_opt_init.hdf5",
    "molecular": "molecular/molecular_dynamics_opt.hdf5",
}


def main(data_dir):
    out_dir = os.path.dirname(os.path.abspath(__file__))
    for name in FIXTURES:
        arrays = h5read.read_all(os.path.join(data_dir, f"test_{name}_cplx.hdf5"))
        np.savez(os.path.join(out_dir, f"{name}.npz"), **arrays)
    os.makedirs(os.path.join(out_dir, "real"), exist_ok=True)
    for name in REAL_FIXTURES:
        arrays = h5read.read_all(os.path.join(data_dir, f"test_{name}_real.hdf5"))
        np.savez(os.path.join(out_dir, "real", f"{name}.npz"), **arrays)
    arrays = h5read.read_all(os.path.join(data_dir, "test_truncated_cg.hdf5"))
    np.savez(os.path.join(out_dir, "truncated_cg.npz"), **arrays)
    examples_dir = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(data_dir))), "examples")
    os.makedirs(os.path.join(out_dir, "examples"), exist_ok=True)
    for name, rel in EXAMPLES.items():
        arrays = h5read.read_all(os.path.join(examples_dir, rel))
        np.savez(os.path.join(out_dir, "examples", f"{name}.npz"), **arrays)
    print(f"wrote {len(FIXTURES) + 1} + {len(REAL_FIXTURES)} (real build) + {len(EXAMPLES)} (example) fixtures to {out_dir}")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference/test/data")
