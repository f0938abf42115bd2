"""Full-Hessian ("hmat") path of the GPU library against the CPU oracle, the
compiled reference where present, and the library's own matrix-free HVP path.
Bars: complex128 1e-12 relative (infinity norm relative to the reference value's)
for f, gradients and Hessians; the dense-Hessian tCG reproduces the oracle's
sequential arithmetic to 1e-14; trust-region runs retrace the oracle's f_iter to
1e-10."""
import numpy as np
import pytest

from helpers import brickwall_instance, crandn, rel_err, random_tangent_dirs, real_to_antisymm

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _defaults(gpu):
    gpu.set_precision(gpu.PRECISION_C128)
    yield
    gpu.set_precision(gpu.PRECISION_C128)
    gpu.set_column_chunk(0)


def _c1(L=8, depth=5, tdepth=3, seed=0):
    return brickwall_instance(L, depth, seed, tdepth, seed + 1)


def test_target_hessian_matches_oracle(gpu, oracle):
    vlist, perms, tvlist, tperms = _c1()
    tg = gpu.Target(brickwall=(tvlist, tperms))
    to = oracle.target("brickwall", (tvlist, tperms))
    f, dv, hess = gpu.brickwall_unitary_target_gradient_hessian(tg, vlist, perms, 8)
    fo, dvo, hesso = oracle.brickwall_unitary_target_gradient_hessian(to, vlist, perms, 8)
    assert abs(f - fo) <= 1e-12 * abs(fo)
    assert rel_err(dv, dvo) <= 1e-12
    assert rel_err(hess, hesso) <= 1e-12
    assert np.array_equal(hess, hess.T)
    f, g, H = gpu.brickwall_unitary_target_gradient_vector_hessian_matrix(tg, vlist, perms, 8)
    fo, go, Ho = oracle.brickwall_unitary_target_gradient_vector_hessian_matrix(to, vlist, perms, 8)
    assert abs(f - fo) <= 1e-12 * abs(fo)
    assert rel_err(g, go) <= 1e-12
    assert rel_err(H, Ho) <= 1e-12
    assert np.array_equal(H, H.T)


def test_target_hessian_matches_compiled_reference(gpu):
    ref_mod = pytest.importorskip("oracle.oracle")
    if not ref_mod.Reference.available():
        pytest.skip("reference build not present")
    ref = ref_mod.Reference()
    vlist, perms, tvlist, tperms = _c1(L=6, depth=4, seed=7)
    tg = gpu.Target(brickwall=(tvlist, tperms))
    f, g, H = gpu.brickwall_unitary_target_gradient_vector_hessian_matrix(tg, vlist, perms, 6)
    fr, gr, Hr = ref.gradient_vector_hessian_matrix(vlist, perms, 6, tvlist, tperms)
    assert abs(f - fr) <= 1e-12 * abs(fr)
    assert rel_err(g, gr) <= 1e-12
    assert rel_err(H, Hr) <= 1e-12


def test_column_chunks_and_host_target(gpu):
    """Several column chunks, and the same target as a host callback, give the same sums."""
    vlist, perms, tvlist, tperms = _c1(L=8, depth=4, seed=3)
    tg = gpu.Target(brickwall=(tvlist, tperms))
    f0, dv0, h0 = gpu.brickwall_unitary_target_gradient_hessian(tg, vlist, perms, 8)
    gpu.set_column_chunk(24)      # ragged: 256 = 10 * 24 + 16
    f1, dv1, h1 = gpu.brickwall_unitary_target_gradient_hessian(tg, vlist, perms, 8)
    gpu.set_column_chunk(0)
    th = gpu.Target(fn=lambda x: gpu.apply_brickwall_unitary(tvlist, tperms, x))
    f2, dv2, h2 = gpu.brickwall_unitary_target_gradient_hessian(th, vlist, perms, 8)
    for f, dv, h in [(f1, dv1, h1), (f2, dv2, h2)]:
        assert abs(f - f0) <= 1e-13 * abs(f0)
        assert rel_err(dv, dv0) <= 1e-13
        assert rel_err(h, h0) <= 1e-13


@pytest.mark.parametrize("L,depth", [(10, 6), (12, 5)])
def test_hessian_agrees_with_matrix_free_hvp(gpu, L, depth):
    """Size-independent check at sizes the CPU oracle cannot finish quickly: the dense
    Hessians applied to a direction equal the matrix-free HVP path's result."""
    vlist, perms, tvlist, tperms = _c1(L=L, depth=depth, seed=20 + L)
    tg = gpu.Target(brickwall=(tvlist, tperms))
    f, dv, hess = gpu.brickwall_unitary_target_gradient_hessian(tg, vlist, perms, L)
    z = crandn(vlist.shape, np.random.default_rng(L))
    fh, dvh, hz = gpu.brickwall_unitary_target_hessian_vector_product(tg, vlist, z, perms, L)
    assert abs(f - fh) <= 1e-12 * abs(fh)
    assert rel_err(dv, dvh) <= 1e-12
    assert rel_err((hess @ z.ravel()).reshape(hz.shape), hz) <= 1e-12
    assert np.array_equal(hess, hess.T)
    r = random_tangent_dirs(vlist, L + 1)
    vdirs = np.stack([vlist[k] @ real_to_antisymm(r[k]) for k in range(depth)])
    fg, g, H = gpu.brickwall_unitary_target_gradient_vector_hessian_matrix(tg, vlist, perms, L)
    _, gp, hvp = gpu.brickwall_unitary_target_projected_hessian_vector_product(tg, vlist, vdirs, perms, L)
    assert rel_err(g, gp) <= 1e-12
    assert rel_err(H @ r.ravel(), hvp) <= 1e-11


def test_backward_hessian_single_state_matches_oracle(gpu, oracle):
    vlist, perms, _, _ = _c1(L=10, depth=3, seed=5)
    rng = np.random.default_rng(9)
    psi, dout = crandn(1 << 10, rng), crandn(1 << 10, rng)
    out, cache = gpu.brickwall_unitary_forward(vlist, perms, psi)
    dpsi, dv, hess = gpu.brickwall_unitary_backward_hessian(vlist, perms, cache, dout)
    outo, states = oracle.brickwall_unitary_forward(vlist, perms, psi)
    dpsio, dvo, hesso = oracle.brickwall_unitary_backward_hessian(vlist, perms, states, dout)
    assert rel_err(out, outo) <= 1e-12
    assert rel_err(dpsi, dpsio) <= 1e-12
    assert rel_err(dv, dvo) <= 1e-12
    assert rel_err(hess, hesso) <= 1e-12
    # the same cache as host arrays
    host_states = [cache.state(k) for k in range(len(states))]
    dpsi2, dv2, hess2 = gpu.brickwall_unitary_backward_hessian(vlist, perms, host_states, dout)
    assert np.array_equal(hess2, hess) and np.array_equal(dv2, dv) and np.array_equal(dpsi2, dpsi)


def test_gate_placeholder_circuit_matches_oracle(gpu, oracle):
    vlist, perms, _, _ = _c1(L=8, depth=4, seed=6)
    psi = crandn(256, np.random.default_rng(4))
    _, states = oracle.brickwall_unitary_forward(vlist, perms, psi)
    for l in range(4):
        a = gpu.apply_brickwall_unitary_gate_placeholder(vlist, perms, l, states)
        b = oracle.apply_brickwall_unitary_gate_placeholder(vlist, perms, l, states)
        assert rel_err(a, b) <= 1e-12


def test_array_kernels_match_oracle(gpu, oracle):
    rng = np.random.default_rng(11)
    V = crandn((4, 4), rng)
    for L, ns, (i, j) in [(7, 3, (6, 0)), (9, 16, (2, 3)), (5, 1, (4, 1))]:
        arr = crandn((1 << L, ns), rng)
        dout = crandn(1 << L, rng)
        assert rel_err(gpu.apply_gate_to_array(V, i, j, arr), oracle.apply_gate_to_array(V, i, j, arr)) <= 1e-14
        assert rel_err(gpu.apply_gate_backward_array(V, i, j, arr, dout),
                       oracle.apply_gate_backward_array(V, i, j, arr, dout)) <= 1e-12
        assert np.array_equal(gpu.apply_gate_placeholder(i, j, arr[:, 0]), oracle.apply_gate_placeholder(i, j, arr[:, 0]))


def test_truncated_cg_hmat_matches_oracle(gpu, oracle):
    rng = np.random.default_rng(12)
    for n, shift in [(48, 3.0), (80, -0.5), (144, 0.2)]:
        a = rng.standard_normal((n, n))
        hess = 0.5 * (a + a.T) + shift * np.eye(n)
        grad = rng.standard_normal(n)
        for radius in (0.05, 10.0):
            z, b = gpu.truncated_cg_hmat(grad, hess, radius)
            zo, bo = oracle.truncated_cg_hmat(grad, hess, radius)
            assert b == bo
            assert np.max(np.abs(z - zo)) <= 1e-14 * max(1.0, np.max(np.abs(zo)))


def test_optimize_hmat_retraces_oracle(gpu, oracle):
    vlist, perms, tvlist, tperms = _c1(L=8, depth=3, seed=0)
    niter = 5
    f, v = gpu.optimize_brickwall_circuit_hmat(gpu.Target(brickwall=(tvlist, tperms)), vlist, perms, 8, niter)
    fo, vo, acc, bnd = oracle.optimize_brickwall_circuit_hmat(oracle.target("brickwall", (tvlist, tperms)), vlist,
                                                              perms, 8, niter)
    assert rel_err(f, fo) <= 1e-10
    assert rel_err(v, vo) <= 1e-9
    assert f[-1] < f[0]


def test_rtr_hmat_with_host_callbacks(gpu, oracle):
    """The generic dense-Hessian trust region driven by Python callbacks retraces the
    device-resident brickwall driver."""
    vlist, perms, tvlist, tperms = _c1(L=6, depth=3, seed=2)
    tg = gpu.Target(brickwall=(tvlist, tperms))
    nl = vlist.shape[0]

    def unpack(x):
        return x.view(np.complex128).reshape(nl, 4, 4)

    def f(x):
        return gpu.brickwall_unitary_target(tg, unpack(x), perms, 6).real

    def fdh(x):
        fx, g, H = gpu.brickwall_unitary_target_gradient_vector_hessian_matrix(tg, unpack(x), perms, 6)
        return fx.real, g, H

    def retract(x, eta):
        v = unpack(x)
        return np.stack([gpu.retract(v[k], eta[16 * k:16 * k + 16]) for k in range(nl)]).view(np.float64).ravel()

    x0 = np.ascontiguousarray(vlist).view(np.float64).ravel()
    f_iter, xf = gpu.riemannian_trust_region_optimize_hmat(f, fdh, retract, 16 * nl, x0, 4)
    f_dev, v_dev = gpu.optimize_brickwall_circuit_hmat(tg, vlist, perms, 6, 4)
    assert rel_err(f_iter, f_dev) <= 1e-12
    assert rel_err(unpack(xf), v_dev) <= 1e-12
