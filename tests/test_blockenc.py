"""Block-encoding target || P^dag W P - H ||_F^2 / 2 on the GPU against the CPU oracle:
f, gradients, the two complex Hessians (the residual's second derivative and the
Gauss-Newton term) and the projected matrix, to 1e-12 relative; H as a device-native
brickwall on L/2 qubits and as a host callback; ragged column chunks; L = 14 runs the
per-gate sweep, smaller L the layer kernel."""
import numpy as np
import pytest

from helpers import brickwall_instance, fixture_ufunc_np, periodic_perms, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _defaults(gpu):
    gpu.set_precision(gpu.PRECISION_C128)
    yield
    gpu.set_column_chunk(0)


def _case(L, depth, hdepth, seed):
    vlist, perms, _, _ = brickwall_instance(L, depth, seed, 1, seed + 1)
    hv, _, _, _ = brickwall_instance(L // 2, hdepth, seed + 2, 1, seed + 3)
    return vlist, perms, hv, periodic_perms(L // 2, hdepth)


def _compare(gpu, oracle, tg, to, vlist, perms, L, hessian=True):
    f, dv = gpu.brickwall_blockenc_target_and_gradient(tg, vlist, perms, L)
    fo, dvo = oracle.brickwall_blockenc_target_and_gradient(to, vlist, perms, L)
    assert abs(f - fo) <= 1e-12 * abs(fo) and rel_err(dv, dvo) <= 1e-12
    assert abs(gpu.brickwall_blockenc_target(tg, vlist, perms, L) - fo) <= 1e-12 * abs(fo)
    f, g = gpu.brickwall_blockenc_target_and_gradient_vector(tg, vlist, perms, L)
    fo, go = oracle.brickwall_blockenc_target_and_gradient_vector(to, vlist, perms, L)
    assert rel_err(g, go) <= 1e-12
    if not hessian:
        return
    f, dv, h1, h2 = gpu.brickwall_blockenc_target_gradient_hessian(tg, vlist, perms, L)
    fo, dvo, h1o, h2o = oracle.brickwall_blockenc_target_gradient_hessian(to, vlist, perms, L)
    assert rel_err(h1, h1o) <= 1e-12 and rel_err(h2, h2o) <= 1e-12
    # hess1 symmetric by construction; hess2's diagonal blocks are summed directly, so
    # Hermitian to rounding, as in the reference (test_target.c:1899-1920)
    assert np.array_equal(h1, h1.T) and np.max(np.abs(h2 - h2.conj().T)) <= 1e-12
    f, g, H = gpu.brickwall_blockenc_target_gradient_vector_hessian_matrix(tg, vlist, perms, L)
    fo, go, Ho = oracle.brickwall_blockenc_target_gradient_vector_hessian_matrix(to, vlist, perms, L)
    assert rel_err(g, go) <= 1e-12 and rel_err(H, Ho) <= 1e-12 and np.array_equal(H, H.T)


def test_blockenc_device_brickwall_h(gpu, oracle):
    vlist, perms, hv, hp = _case(8, 4, 2, 3)
    _compare(gpu, oracle, gpu.Target(brickwall=(hv, hp)), oracle.target("brickwall", (hv, hp)), vlist, perms, 8)


def test_blockenc_host_callback_h(gpu, oracle):
    vlist, perms, _, _ = _case(10, 3, 2, 5)
    _compare(gpu, oracle, gpu.Target(fn=fixture_ufunc_np), oracle.target("fixture"), vlist, perms, 10)


def test_blockenc_ragged_chunks(gpu):
    vlist, perms, hv, hp = _case(8, 3, 2, 7)
    tg = gpu.Target(brickwall=(hv, hp))
    ref = gpu.brickwall_blockenc_target_gradient_hessian(tg, vlist, perms, 8)
    gpu.set_column_chunk(5)            # 16 columns in chunks of 5, 5, 5, 1
    out = gpu.brickwall_blockenc_target_gradient_hessian(tg, vlist, perms, 8)
    assert abs(out[0] - ref[0]) <= 1e-13 * abs(ref[0])
    for a, b in zip(out[1:], ref[1:]):
        assert rel_err(a, b) <= 1e-13


def test_blockenc_per_gate_sweep(gpu, oracle):
    """L = 14 (H on 7 qubits as a host callback; one layer keeps the oracle's placeholder
    loops short)."""
    vlist, perms, _, _ = _case(14, 1, 2, 9)
    _compare(gpu, oracle, gpu.Target(fn=fixture_ufunc_np), oracle.target("fixture"), vlist, perms, 14)
