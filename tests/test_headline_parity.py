"""Parity at the headline size: L=16, a depth-9 periodic brickwall (Haar gates,
seed 10) against a depth-5 brickwall target (seed 11), tangent direction seed 12.

A full evaluation over all 65,536 basis columns takes hours on the CPU, so the
GPU library's column range (rqcopt_gpu_set_column_range) restricts its sums to
contiguous column samples, and the reference's own per-column function
(quantum_circuit_gates_hessian_vector_product, the loop body of
src/target.c:335-369), compiled from the reference sources in oracle/_ref, sums
the same columns; where that build is absent the oracle's C restatement does.
Bars: complex128 1e-12 relative in f and in every per-gate gradient and
Hessian-vector entry (infinity norm relative to the reference's largest entry),
for the fused passes and for the one-gate-per-pass engine; complex64 passes 1e-5.
"""
import numpy as np
import pytest

from helpers import brickwall_instance, random_tangent_dirs, real_to_antisymm, rel_err

pytestmark = pytest.mark.gpu

L, DEPTH, TDEPTH = 16, 9, 5
# a range at the start of the column space, and a ragged one in the middle (its
# length is not a multiple of the 4- or 8-column groups of the fused passes)
RANGES = [(0, 8), (30001, 30014)]


def _c2():
    vlist, perms, tvlist, tperms = brickwall_instance(L, DEPTH, 10, TDEPTH, 11)
    r = random_tangent_dirs(vlist, 12)
    vdirs = np.stack([vlist[k] @ real_to_antisymm(r[k]) for k in range(DEPTH)])
    per = L // 2
    gates = np.repeat(vlist, per, axis=0)
    dirs = np.repeat(vdirs, per, axis=0)
    wires = np.concatenate([perms[l].reshape(per, 2) for l in range(DEPTH)]).astype(np.int32)
    return vlist, vdirs, perms, tvlist, tperms, gates, dirs, wires


def _reference_sums(vlist, vdirs, perms, tvlist, tperms, b0, b1):
    from oracle.oracle import Oracle, Reference
    if Reference.available():
        return Reference().brickwall_hvp_columns(vlist, vdirs, perms, L, tvlist, tperms, b0, b1)
    o = Oracle()
    per = L // 2
    gates = np.repeat(vlist, per, axis=0)
    dirs = np.repeat(vdirs, per, axis=0)
    wires = np.concatenate([perms[l].reshape(per, 2) for l in range(DEPTH)]).astype(np.int32)
    tgt = o.target("brickwall", (tvlist, tperms))
    return o.circuit_unitary_target_hessian_vector_product(tgt, gates, dirs, wires, L, b0, b1)


@pytest.fixture(scope="module")
def c2_reference():
    vlist, vdirs, perms, tvlist, tperms, gates, dirs, wires = _c2()
    return {rg: _reference_sums(vlist, vdirs, perms, tvlist, tperms, *rg) for rg in RANGES}


@pytest.fixture
def _restore(gpu):
    yield
    gpu.set_column_range(0, 0)
    gpu.set_precision(gpu.PRECISION_C128)
    gpu.set_autotune(True)


def _check(f, dg, hg, ref, tol):
    fr, dgr, hgr = ref
    assert abs(f - fr) <= tol * abs(fr), (f, fr)
    assert rel_err(dg, dgr) <= tol
    assert rel_err(hg, hgr) <= tol


@pytest.mark.parametrize("gates_per_pass", [4, 1])
def test_c2_column_samples_complex128_match_reference(gpu, c2_reference, _restore, gates_per_pass):
    vlist, vdirs, perms, tvlist, tperms, gates, dirs, wires = _c2()
    tgt = gpu.Target(brickwall=(tvlist, tperms))
    gpu.set_precision(gpu.PRECISION_C128)
    gpu.set_gates_per_pass(gates_per_pass)
    for rg in RANGES:
        gpu.set_column_range(*rg)
        f, dg, hg = gpu.circuit_unitary_target_hessian_vector_product(tgt, gates, dirs, wires, L)
        _check(f, dg, hg, c2_reference[rg], 1e-12)
        # the brickwall form sums the per-gate results of each layer
        fb, dv, hv = gpu.brickwall_unitary_target_hessian_vector_product(tgt, vlist, vdirs, perms, L)
        fr, dgr, hgr = c2_reference[rg]
        per = L // 2
        _check(fb, dv, hv, (fr, dgr.reshape(DEPTH, per, 4, 4).sum(1), hgr.reshape(DEPTH, per, 4, 4).sum(1)), 1e-12)


def test_c2_column_samples_complex64_passes(gpu, c2_reference, _restore):
    vlist, vdirs, perms, tvlist, tperms, gates, dirs, wires = _c2()
    tgt = gpu.Target(brickwall=(tvlist, tperms))
    gpu.set_precision(gpu.PRECISION_C64)
    for rg in RANGES:
        gpu.set_column_range(*rg)
        f, dg, hg = gpu.circuit_unitary_target_hessian_vector_product(tgt, gates, dirs, wires, L)
        _check(f, dg, hg, c2_reference[rg], 1e-5)


def test_column_ranges_partition_the_full_sum(gpu, _restore):
    """Size-independent check: the sums over a partition of the columns into ragged
    ranges add up to the full evaluation (L=10, both precisions' engines)."""
    vlist, perms, tvlist, tperms = brickwall_instance(10, 5, 3, 3, 4)
    r = random_tangent_dirs(vlist, 5)
    vdirs = np.stack([vlist[k] @ real_to_antisymm(r[k]) for k in range(5)])
    tgt = gpu.Target(brickwall=(tvlist, tperms))
    for prec, tol in ((gpu.PRECISION_C128, 1e-12), (gpu.PRECISION_C64, 1e-5)):
        gpu.set_precision(prec)
        gpu.set_column_range(0, 0)
        full = gpu.brickwall_unitary_target_hessian_vector_product(tgt, vlist, vdirs, perms, 10)
        cuts = [0, 3, 100, 101, 517, 1024]
        parts = []
        for a, b in zip(cuts[:-1], cuts[1:]):
            gpu.set_column_range(a, b)
            parts.append(gpu.brickwall_unitary_target_hessian_vector_product(tgt, vlist, vdirs, perms, 10))
        f = sum(p[0] for p in parts)
        dv = sum(p[1] for p in parts)
        hv = sum(p[2] for p in parts)
        assert abs(f - full[0]) <= tol * abs(full[0])
        assert rel_err(dv, full[1]) <= tol
        assert rel_err(hv, full[2]) <= tol


def test_column_range_rejects_bad_ranges(gpu, _restore):
    from rqcopt_hpc_b200.gpu import RqcError
    for a, b in [(-1, 0), (5, 5), (7, 3), (0, -2)]:
        with pytest.raises(RqcError):
            gpu.set_column_range(a, b)
