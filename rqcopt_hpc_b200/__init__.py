"""B200 implementation of the rqcopt_hpc matrix-free circuit-optimisation path.

The product is the C-ABI shared library ``librqcopt_gpu.so`` (CUDA C++ for
sm_100a, sources in ``csrc/``, interface in ``include/rqcopt_gpu.h``) that
exports the reference's C functions, and ``librqcopt_gpu_real.so``
(``include/rqcopt_gpu_real.h``), the reference's real-orthogonal build on top of it.
Python modules:

- ``gpu``: host mirror of the C interface; ``real``: the same for the real build;
- ``batch``, ``serving``: many small problems per launch and the request loop;
- ``rqcopt_hpc``: the reference's Python module (``optimize_quantum_circuit``,
  ``optimize_brickwall_circuit``) on the GPU library;
- ``examples``: the reference's example drivers; ``h5read``: a reader for the
  project's HDF5 files;
- ``build``: compiles both libraries in-tree.
"""

__all__ = ["gpu", "real", "abi", "batch", "serving", "rqcopt_hpc", "examples", "h5read", "build"]
