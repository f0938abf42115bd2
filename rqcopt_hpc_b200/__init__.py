"""B200 implementation of the rqcopt_hpc matrix-free circuit-optimisation path.

The product is the C-ABI shared library ``librqcopt_gpu.so`` (CUDA C++ for
sm_100a, sources in ``csrc/``, interface in ``include/rqcopt_gpu.h``) that
exports the reference's C functions.  ``rqcopt_hpc_b200.gpu`` is the Python
host mirror of that interface; ``rqcopt_hpc_b200.build`` compiles the library
in-tree.
"""

__all__ = ["gpu", "abi", "build"]
