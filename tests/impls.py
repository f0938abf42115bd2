"""Two implementations behind one interface for the parity suite: the CPU oracle and
the GPU library (through its C ABI).  Targets are named by kind: 'fixture' (the
reference tests' sparse map), ('brickwall', (vlist, perms)) applied matrix-free,
('dense', U) or ('host_brickwall', (vlist, perms)) -- the brickwall as an
ordinary host callback, which exercises the generic callback path of the GPU
library."""
from __future__ import annotations

import numpy as np

from helpers import fixture_ufunc_np


class GpuImpl:
    name = "gpu"

    def __init__(self):
        from rqcopt_hpc_b200 import gpu as g
        self.g = g
        g.lib()

    def target(self, kind, data=None):
        g = self.g
        if kind == "fixture":
            return g.Target(fn=fixture_ufunc_np)
        if kind == "brickwall":
            return g.Target(brickwall=data)
        if kind == "dense":
            u = np.asarray(data)
            return g.Target(fn=lambda x: u @ x)
        if kind == "host_brickwall":
            vlist, perms = data
            return g.Target(fn=lambda x: g.apply_brickwall_unitary(vlist, perms, x))
        if kind == "circuit":
            return g.Target(circuit=data)
        raise ValueError(kind)

    def __getattr__(self, name):
        return getattr(self.g, name)


class OracleImpl:
    name = "oracle"

    def __init__(self):
        from oracle.oracle import Oracle
        self.o = Oracle()

    def target(self, kind, data=None):
        if kind in ("brickwall", "host_brickwall"):
            return self.o.target("brickwall", data)
        if kind == "circuit":
            raise NotImplementedError("the oracle takes general-circuit targets as dense matrices")
        return self.o.target(kind, data)

    def __getattr__(self, name):
        return getattr(self.o, name)
