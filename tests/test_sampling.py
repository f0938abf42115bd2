"""Sampling estimator of the GPU library (Haar-random states drawn on the device from
the reference's PCG32x2 stream) against the CPU oracle on the same seeds.  The
device log and sin may differ from the host's in the last bit, so the states agree to
~1e-16 and the estimates to 1e-12 relative; the generator state after each call is
identical.  L = 14 exercises the per-gate sweep, smaller L the layer kernel."""
import numpy as np
import pytest

from helpers import brickwall_instance, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _defaults(gpu):
    gpu.set_precision(gpu.PRECISION_C128)
    yield
    gpu.set_column_chunk(0)


def _same_rng(a, b):
    return a.tuple() == b.tuple()


def test_seed_and_haar_states(gpu, oracle):
    rg, ro = gpu.seed_rng_state(677), oracle.seed_rng_state(677)
    assert _same_rng(rg, ro)
    for L in (1, 6, 13):
        a = gpu.haar_random_statevector(L, rg)
        b = oracle.haar_random_statevector(L, ro)
        assert rel_err(a, b) <= 1e-14
        assert abs(np.linalg.norm(a) - 1) <= 1e-14
        assert _same_rng(rg, ro)


@pytest.mark.parametrize("L,depth,ns,chunk", [(6, 3, 200, 0), (8, 4, 64, 10), (12, 2, 3, 0)])
def test_sampled_target_matches_oracle(gpu, oracle, L, depth, ns, chunk):
    vlist, perms, tvlist, tperms = brickwall_instance(L, depth, 3, 3, 4)
    tg, to = gpu.Target(brickwall=(tvlist, tperms)), oracle.target("brickwall", (tvlist, tperms))
    gpu.set_column_chunk(chunk)
    rg, ro = gpu.seed_rng_state(11), oracle.seed_rng_state(11)
    f = gpu.brickwall_unitary_target_sampling(tg, vlist, perms, L, ns, rg)
    fo = oracle.brickwall_unitary_target_sampling(to, vlist, perms, L, ns, ro)
    assert abs(f - fo) <= 1e-12 * abs(fo) and _same_rng(rg, ro)
    f, g, H = gpu.brickwall_unitary_target_gradient_vector_hessian_matrix_sampling(tg, vlist, perms, L, ns, rg)
    fo, go, Ho = oracle.brickwall_unitary_target_gradient_vector_hessian_matrix_sampling(to, vlist, perms, L, ns, ro)
    assert abs(f - fo) <= 1e-12 * abs(fo)
    assert rel_err(g, go) <= 1e-12 and rel_err(H, Ho) <= 1e-12 and _same_rng(rg, ro)
    assert np.array_equal(H, H.T)


def test_sampled_hessian_per_gate_sweep(gpu, oracle):
    """L = 14 runs the per-gate sweep kernel; two samples keep the oracle fast."""
    vlist, perms, tvlist, tperms = brickwall_instance(14, 2, 5, 2, 6)
    tg, to = gpu.Target(brickwall=(tvlist, tperms)), oracle.target("brickwall", (tvlist, tperms))
    rg, ro = gpu.seed_rng_state(3), oracle.seed_rng_state(3)
    f, dv, hess = gpu.brickwall_unitary_target_gradient_hessian_sampling(tg, vlist, perms, 14, 2, rg)
    fo, dvo, hesso = oracle.brickwall_unitary_target_gradient_hessian_sampling(to, vlist, perms, 14, 2, ro)
    assert abs(f - fo) <= 1e-12 * abs(fo)
    assert rel_err(dv, dvo) <= 1e-12 and rel_err(hess, hesso) <= 1e-12 and _same_rng(rg, ro)


def test_sampled_circuit_target_host_callback(gpu, oracle):
    rng = np.random.default_rng(8)
    L, G = 7, 9
    gates = np.stack([np.linalg.qr(rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4)))[0] for _ in range(G)])
    wires = np.array([rng.choice(L, 2, replace=False) for _ in range(G)], np.int32)
    u = np.linalg.qr(rng.standard_normal((1 << L, 1 << L)) + 1j * rng.standard_normal((1 << L, 1 << L)))[0]
    rg, ro = gpu.seed_rng_state(21), oracle.seed_rng_state(21)
    f = gpu.circuit_unitary_target_sampling(gpu.Target(fn=lambda x: u @ x), gates, wires, L, 50, rg)
    fo = oracle.circuit_unitary_target_sampling(oracle.target("dense", u), gates, wires, L, 50, ro)
    assert abs(f - fo) <= 1e-12 * abs(fo) and _same_rng(rg, ro)


def test_sampled_optimizer_retraces_oracle(gpu, oracle):
    vlist, perms, tvlist, tperms = brickwall_instance(6, 3, 0, 3, 1)
    rg, ro = gpu.seed_rng_state(7), oracle.seed_rng_state(7)
    f, v = gpu.optimize_brickwall_circuit_hmat_sampling(gpu.Target(brickwall=(tvlist, tperms)), vlist, perms, 6, 30,
                                                        rg, 4)
    fo, vo = oracle.optimize_brickwall_circuit_hmat_sampling(oracle.target("brickwall", (tvlist, tperms)), vlist,
                                                             perms, 6, 30, ro, 4)
    assert rel_err(f, fo) <= 1e-10 and rel_err(v, vo) <= 1e-9 and _same_rng(rg, ro)
