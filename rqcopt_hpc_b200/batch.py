"""Batched brickwall evaluation and optimisation (include/rqcopt_batch.h).

A problem is ``(L, vlist, perms, target_vlist, target_perms)``: a brickwall
circuit of ``len(vlist)`` layer gates on the pairs of ``perms[l]`` fitted to a
brickwall target applied matrix-free, the objective of the reference's
``brickwall_unitary_target*`` functions (src/target.c:467-678) and of
``optimize_brickwall_circuit_hvp`` (src/brickwall_opt.c:107-149).  Many such
problems run together on one GPU; see :class:`Batch` for the slot interface a
request loop uses.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import gpu
from .abi import RTRParams, cplx, default_rtr_params, perm_pointers

EVAL_F, EVAL_GRAD, EVAL_HVP = 0, 1, 2


class BatchProblem(C.Structure):
    _fields_ = [("nqubits", C.c_int), ("nlayers", C.c_int), ("vlist", C.c_void_p), ("perms", C.c_void_p),
                ("target_nlayers", C.c_int), ("target_vlist", C.c_void_p), ("target_perms", C.c_void_p)]


def _pack(problems):
    """ctypes problem array plus the numpy arrays it points into (kept alive by the caller)."""
    keep = []
    arr = (BatchProblem * len(problems))()
    for k, (L, vlist, perms, tvlist, tperms) in enumerate(problems):
        v, tv = cplx(vlist), cplx(tvlist)
        pp, k1 = perm_pointers(perms)
        tp, k2 = perm_pointers(tperms)
        keep += [v, tv, pp, k1, tp, k2]
        arr[k] = BatchProblem(int(L), v.shape[0], v.ctypes.data, C.cast(pp, C.c_void_p).value, tv.shape[0],
                              tv.ctypes.data, C.cast(tp, C.c_void_p).value)
    return arr, keep


def _check(fn, ret):
    if ret < 0:
        raise gpu.RqcError(fn, ret)
    return ret


def evaluate(problems, vdirs=None, mode=EVAL_HVP, precision=gpu.PRECISION_C64):
    """f (complex), projected gradients and projected HVPs of every problem in one batched pass."""
    arr, keep = _pack(problems)
    n = [16 * len(p[1]) for p in problems]
    f = np.zeros(2 * len(problems))
    grad = np.zeros(sum(n))
    hvp = np.zeros(sum(n))
    dptr = None
    if mode == EVAL_HVP:
        dl = [cplx(d) for d in vdirs]
        keep += dl
        dptr = (C.c_void_p * len(dl))(*[d.ctypes.data for d in dl])
    _check("rqcopt_brickwall_batch_evaluate",
           gpu.lib().rqcopt_brickwall_batch_evaluate(C.byref(arr), len(problems), dptr, mode, precision,
                                                     f.ctypes.data, grad.ctypes.data, hvp.ctypes.data))
    off = np.cumsum([0] + n)
    fc = f[0::2] + 1j * f[1::2]
    return fc, [grad[off[k]:off[k + 1]] for k in range(len(n))], [hvp[off[k]:off[k + 1]] for k in range(len(n))]


def optimize(problems, niter, precision=gpu.PRECISION_C64, params=None):
    """optimize_brickwall_circuit_hvp for every problem at once: (f_iter [count][niter+1], [vlist_opt])."""
    arr, keep = _pack(problems)
    nl = [len(p[1]) for p in problems]
    f_iter = np.zeros((len(problems), niter + 1))
    vopt = np.zeros((sum(nl), 4, 4), np.complex128)
    pa = None
    if params is not None:
        pa = (RTRParams * len(problems))(*params)
    _check("rqcopt_optimize_brickwall_batch",
           gpu.lib().rqcopt_optimize_brickwall_batch(C.byref(arr), len(problems), pa, niter, precision,
                                                     f_iter.ctypes.data, vopt.ctypes.data))
    off = np.cumsum([0] + nl)
    return f_iter, [vopt[off[k]:off[k + 1]] for k in range(len(nl))]


def footprint(L, nlayers):
    """Device bytes one problem holds in a batch."""
    return int(gpu.lib().rqcopt_batch_footprint(L, nlayers))


class Batch:
    """Slots of a running batch: problems join (add) and leave (result + release)
    between rounds; run(k) advances every active problem by up to k evaluations."""

    def __init__(self, capacity, max_iterations, sharing=False):
        self.h = gpu.lib().rqcopt_batch_create(capacity, max_iterations)
        if not self.h:
            raise gpu.RqcError("rqcopt_batch_create", gpu.lib().rqcopt_gpu_last_error())
        if sharing:
            gpu.lib().rqcopt_batch_set_sharing(self.h, 1)
        self.capacity = capacity
        self._nl = {}
        self._niter = {}

    def add(self, problem, niter, precision=gpu.PRECISION_C64, params=None, grad_tol=0.0):
        arr, keep = _pack([problem])
        p = C.byref(params) if params is not None else None
        slot = _check("rqcopt_batch_add",
                      gpu.lib().rqcopt_batch_add(self.h, C.byref(arr), p, niter, precision, float(grad_tol)))
        self._nl[slot] = len(problem[1])
        self._niter[slot] = niter
        return slot

    def run(self, rounds):
        return _check("rqcopt_batch_run", gpu.lib().rqcopt_batch_run(self.h, rounds))

    def finished(self, max_slots=None):
        m = max_slots or self.capacity
        buf = np.zeros(m, np.int32)
        k = _check("rqcopt_batch_finished", gpu.lib().rqcopt_batch_finished(self.h, buf.ctypes.data, m))
        return [int(x) for x in buf[:k]]

    def result(self, slot):
        """(f_iter, vlist_opt) of a finished slot (f_iter ends at the last iteration run), else None."""
        f = np.zeros(self._niter[slot] + 1)
        v = np.zeros((self._nl[slot], 4, 4), np.complex128)
        it = C.c_int(0)
        r = _check("rqcopt_batch_result",
                   gpu.lib().rqcopt_batch_result(self.h, slot, f.ctypes.data, v.ctypes.data, C.byref(it)))
        if r != 1:
            return None
        return f[:it.value + 1], v

    def release(self, slot):
        _check("rqcopt_batch_release", gpu.lib().rqcopt_batch_release(self.h, slot))
        self._nl.pop(slot, None)
        self._niter.pop(slot, None)

    @property
    def rounds(self):
        return int(gpu.lib().rqcopt_batch_rounds(self.h))

    def evaluations(self):
        """(evaluations, of them Hessian-vector products) run so far."""
        h = C.c_long(0)
        n = _check("rqcopt_batch_evaluations", gpu.lib().rqcopt_batch_evaluations(self.h, C.byref(h)))
        return int(n), int(h.value)

    def close(self):
        if self.h:
            gpu.lib().rqcopt_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _main():
    """python -m rqcopt_hpc_b200.batch: optimise `count` seeded brickwall instances together."""
    import argparse
    import time
    from .workloads import batched_instances, brickwall_problem
    ap = argparse.ArgumentParser(description=_main.__doc__)
    ap.add_argument("--count", type=int, default=512)
    ap.add_argument("--L", type=int, default=0, help="fixed qubit count (default: even L uniform over 6..12)")
    ap.add_argument("--niter", type=int, default=2)
    ap.add_argument("--precision", default="c64", choices=["c64", "mixed", "c128"])
    ap.add_argument("--plain", action="store_true",
                    help="also run the per-instance complex128 optimiser on every instance and compare")
    a = ap.parse_args()
    prec = {"c64": gpu.PRECISION_C64, "mixed": gpu.PRECISION_MIXED, "c128": gpu.PRECISION_C128}[a.precision]
    if a.L:
        probs = [brickwall_problem(a.L, (3, 5, 7, 9)[i % 4], 3, 30 + i, 10000 + i) for i in range(a.count)]
    else:
        probs = batched_instances(a.count)
    b = Batch(a.count, a.niter)
    for p in probs:
        b.add(p, a.niter, prec)
    t0 = time.perf_counter()
    while b.run(8) > 0:
        pass
    el = time.perf_counter() - t0
    ev, hv = b.evaluations()
    print(f"{a.count} instances x {a.niter} iterations ({a.precision}): {el:.3f} s, {b.rounds} rounds, "
          f"{ev} evaluations ({hv} HVP), {ev / el:.1f} evaluations/s")
    fb = np.array([b.result(s)[0][-1] for s in range(a.count)])
    b.close()
    if a.plain:
        gpu.set_precision(gpu.PRECISION_C128)
        seen = set()
        for (L, vl, pm, tv, tp) in probs:   # set-up of every size class outside the timed loop
            if (L, len(vl)) not in seen:
                seen.add((L, len(vl)))
                gpu.optimize_brickwall_circuit_hvp(gpu.Target(brickwall=(tv, tp)), vl, pm, L, a.niter)
        t0 = time.perf_counter()
        fp = np.array([gpu.optimize_brickwall_circuit_hvp(gpu.Target(brickwall=(tv, tp)), vl, pm, L, a.niter)[0][-1]
                       for (L, vl, pm, tv, tp) in probs])
        ep = time.perf_counter() - t0
        print(f"per-instance complex128 loop: {ep:.3f} s; batched speed-up {ep / el:.2f}x; "
              f"max relative difference of the final f {np.max(np.abs(fb - fp) / np.abs(fp)):.2e}")


if __name__ == "__main__":
    _main()
