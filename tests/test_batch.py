"""Batched brickwall engine (include/rqcopt_batch.h) against the CPU oracle and the
single-problem GPU path.  Bars: complex128 1e-12 relative in f, projected
gradient and projected HVP (infinity norm relative to the reference value's);
complex64 passes 1e-5; batched trust-region runs reproduce the single-problem
optimiser's f_iter to 1e-10 in complex128."""
import numpy as np
import pytest

from helpers import brickwall_instance, random_tangent_dirs, real_to_antisymm, rel_err

pytestmark = pytest.mark.gpu


def _dirs(vlist, seed):
    r = random_tangent_dirs(vlist, seed)
    return np.stack([vlist[k] @ real_to_antisymm(r[k]) for k in range(vlist.shape[0])])


def _problem(L, depth, tdepth, seed):
    vlist, perms, tvlist, tperms = brickwall_instance(L, depth, seed, tdepth, seed + 1000)
    return (L, vlist, perms, tvlist, tperms)


@pytest.fixture(autouse=True)
def _defaults(gpu):
    gpu.set_precision(gpu.PRECISION_C128)
    yield
    gpu.set_precision(gpu.PRECISION_C128)


def _single(gpu, p, vdirs):
    L, vlist, perms, tvlist, tperms = p
    return gpu.brickwall_unitary_target_projected_hessian_vector_product(gpu.Target(brickwall=(tvlist, tperms)), vlist,
                                                                        vdirs, perms, L)


def test_batch_c128_matches_oracle(gpu, oracle):
    from rqcopt_hpc_b200 import batch
    probs = [_problem(4, 3, 3, 11), _problem(6, 5, 3, 12), _problem(8, 4, 2, 13)]
    dirs = [_dirs(p[1], 50 + k) for k, p in enumerate(probs)]
    f, g, h = batch.evaluate(probs, dirs, batch.EVAL_HVP, gpu.PRECISION_C128)
    for k, p in enumerate(probs):
        L, vlist, perms, tvlist, tperms = p
        fo, go, ho = oracle.brickwall_unitary_target_projected_hessian_vector_product(
            oracle.target("brickwall", (tvlist, tperms)), vlist, dirs[k], perms, L)
        assert abs(f[k] - fo) <= 1e-12 * abs(fo)
        assert rel_err(g[k], go) <= 1e-12
        assert rel_err(h[k], ho) <= 1e-12


def test_batch_mixed_sizes_match_single_path(gpu):
    """Instances of every size class in one batch: shared-memory tiles of many
    columns (small L), one column per tile (L = 12) and global-memory tiles (L = 14
    complex64, L >= 12 complex128)."""
    from rqcopt_hpc_b200 import batch
    probs = [_problem(L, d, 3, 20 + L) for L, d in [(6, 3), (8, 5), (10, 3), (12, 3), (2, 2), (14, 2)]]
    dirs = [_dirs(p[1], 70 + k) for k, p in enumerate(probs)]
    ref = [_single(gpu, p, dirs[k]) for k, p in enumerate(probs)]
    f, g, h = batch.evaluate(probs, dirs, batch.EVAL_HVP, gpu.PRECISION_C128)
    for k in range(len(probs)):
        assert abs(f[k] - ref[k][0]) <= 1e-12 * abs(ref[k][0]), probs[k][0]
        assert rel_err(g[k], ref[k][1]) <= 1e-12, probs[k][0]
        assert rel_err(h[k], ref[k][2]) <= 1e-12, probs[k][0]
    f32, g32, h32 = batch.evaluate(probs, dirs, batch.EVAL_HVP, gpu.PRECISION_C64)
    for k in range(len(probs)):
        assert abs(f32[k] - ref[k][0]) <= 1e-5 * max(abs(ref[k][0]), 1), probs[k][0]
        assert rel_err(g32[k], ref[k][1]) <= 1e-5, probs[k][0]
        assert rel_err(h32[k], ref[k][2]) <= 1e-5, probs[k][0]


def test_batch_modes(gpu):
    from rqcopt_hpc_b200 import batch
    probs = [_problem(8, 5, 3, 31), _problem(10, 3, 3, 32)]
    dirs = [_dirs(p[1], 90 + k) for k, p in enumerate(probs)]
    fh, gh, _ = batch.evaluate(probs, dirs, batch.EVAL_HVP, gpu.PRECISION_C128)
    fg, gg, _ = batch.evaluate(probs, None, batch.EVAL_GRAD, gpu.PRECISION_C128)
    ff, _, _ = batch.evaluate(probs, None, batch.EVAL_F, gpu.PRECISION_C128)
    for k in range(len(probs)):
        assert abs(fg[k] - fh[k]) <= 1e-13 * abs(fh[k])
        assert abs(ff[k] - fh[k]) <= 1e-13 * abs(fh[k])
        assert rel_err(gg[k], gh[k]) <= 1e-13


def test_batch_optimize_retraces_single_optimizer(gpu):
    from rqcopt_hpc_b200 import batch
    probs = [_problem(6, 3, 3, 41), _problem(8, 5, 3, 42), _problem(4, 3, 2, 43)]
    niter = 6
    f_iter, vopt = batch.optimize(probs, niter, gpu.PRECISION_C128)
    for k, p in enumerate(probs):
        L, vlist, perms, tvlist, tperms = p
        fs, vs = gpu.optimize_brickwall_circuit_hvp(gpu.Target(brickwall=(tvlist, tperms)), vlist, perms, L, niter)
        assert np.max(np.abs(f_iter[k] - fs)) <= 1e-10 * np.max(np.abs(fs)), (k, f_iter[k], fs)
        assert np.max(np.abs(vopt[k] - vs)) <= 1e-9


def test_batch_mixed_precision_optimize(gpu):
    """Batched mixed precision (complex64 HVPs, complex128 once the gradient norm falls
    below 1e-5) on problems the trust region drives to convergence within 80 iterations
    (the tCG takes many inner steps once the steps leave the trust-region boundary): the
    final f of every problem equals the single-problem complex128 optimiser's to 1e-10
    relative, and the batched complex128 run retraces it."""
    from rqcopt_hpc_b200 import batch
    from rqcopt_hpc_b200.workloads import brickwall_problem
    probs = [brickwall_problem(6, 3, 3, 0, 1), brickwall_problem(8, 3, 3, 0, 1), brickwall_problem(6, 5, 3, 5, 6)]
    niter = 80
    f128, _ = batch.optimize(probs, niter, gpu.PRECISION_C128)
    fmix, _ = batch.optimize(probs, niter, gpu.PRECISION_MIXED)
    f64, _ = batch.optimize(probs, 4, gpu.PRECISION_C64)
    for k, (L, vlist, perms, tvlist, tperms) in enumerate(probs):
        fs, _ = gpu.optimize_brickwall_circuit_hvp(gpu.Target(brickwall=(tvlist, tperms)), vlist, perms, L, niter)
        # the same first value (complex128 f in mixed mode) and a monotone trust-region decrease
        assert fmix[k][0] == f128[k][0]
        assert np.all(np.diff(fmix[k]) <= 1e-9 * abs(fmix[k][0]))
        assert abs(f128[k][-1] - fs[-1]) <= 1e-10 * abs(fs[-1])
        assert abs(fmix[k][-1] - fs[-1]) <= 1e-10 * abs(fs[-1]), (k, fmix[k][-1], fs[-1])
        assert abs(f64[k][0] - f128[k][0]) <= 1e-5 * abs(f128[k][0])


def test_batch_slots_admit_and_retire(gpu):
    """Problems join a running batch and leave it when done; each result equals the
    one of the same problem run alone."""
    from rqcopt_hpc_b200 import batch
    probs = [_problem(6, 3, 3, 61), _problem(8, 3, 3, 62), _problem(4, 3, 3, 63), _problem(6, 5, 3, 64)]
    niters = [4, 3, 5, 2]
    alone = [batch.optimize([p], niters[k], gpu.PRECISION_C64)[0][0] for k, p in enumerate(probs)]
    b = batch.Batch(capacity=3, max_iterations=8)
    slots = {}
    slots[b.add(probs[0], niters[0])] = 0
    slots[b.add(probs[1], niters[1])] = 1
    b.run(5)
    slots[b.add(probs[2], niters[2])] = 2
    results = {}
    pending = [3]
    for _ in range(200):
        active = b.run(4)
        for s in b.finished():
            f, v = b.result(s)
            results[slots.pop(s)] = f
            b.release(s)
            if pending:
                k = pending.pop()
                slots[b.add(probs[k], niters[k])] = k
        if active == 0 and not pending and not slots:
            break
    b.close()
    assert sorted(results) == [0, 1, 2, 3]
    for k in range(4):
        assert np.max(np.abs(results[k] - alone[k])) <= 1e-12 * np.max(np.abs(alone[k])), k


def test_serving_mix_equals_alone(gpu):
    """Requests admitted into a running batch as they arrive: every result is
    bit-identical to the same request run alone."""
    from rqcopt_hpc_b200 import batch, serving
    from rqcopt_hpc_b200.workloads import brickwall_problem
    reqs = [serving.Request(k, brickwall_problem(L, d, 3, 500 + k, 600 + k), 6, 1e-8, 0.002 * k,
                            gpu.PRECISION_MIXED)
            for k, (L, d) in enumerate([(6, 3), (8, 5), (4, 3), (10, 3), (6, 7), (8, 3), (12, 3), (4, 5)])]
    b = batch.Batch(capacity=4, max_iterations=6, sharing=True)
    srv = serving.Server(b, capacity=4, hbm_budget_bytes=150e9, footprint=batch.footprint, rounds_per_step=3)
    done, left = serving.run_arrivals(srv, reqs, wall_limit=300.0)
    b.close()
    assert not left and len(done) == len(reqs)
    for r in done:
        alone = batch.Batch(capacity=1, max_iterations=6)
        s = alone.add(r.problem, r.niter, r.precision, grad_tol=r.grad_tol)
        while alone.run(8) > 0:
            pass
        f_alone, _ = alone.result(s)
        alone.close()
        assert np.array_equal(r.f_iter, f_alone), (r.rid, r.f_iter, f_alone)
