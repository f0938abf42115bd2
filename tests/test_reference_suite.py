"""The reference's hot-path tests (test/test_gate.c, test_quantum_circuit.c,
test_brickwall_circuit.c, test_target.c, test_matrix.c, test_trust_region.c),
restated once and run against two implementations: the CPU oracle (which pins
the oracle to the reference's golden vectors) and the GPU library through its
C ABI (marked gpu).  Tolerances are the reference tests' own: 1e-12 for states
and f against the golden vectors, 1e-8 (1e-7 for brickwall HVPs) for
derivatives against central differences with h = 1e-5, 1e-14 for the projected
gradient and the tCG solution."""
import numpy as np
import pytest

from helpers import golden, stack, udist, num_grad_backward, num_grad_wirtinger, num_grad_forward
from impls import GpuImpl, OracleImpl

IMPLS = [pytest.param("oracle", id="oracle"), pytest.param("gpu", id="gpu", marks=pytest.mark.gpu)]
_cache = {}


@pytest.fixture(params=IMPLS)
def impl(request):
    name = request.param
    if name == "gpu":
        request.getfixturevalue("gpu")
    if name not in _cache:
        _cache[name] = GpuImpl() if name == "gpu" else OracleImpl()
    return _cache[name]


# ------------------------------------------------------------------ test_gate.c

def test_apply_gate(impl):
    d = golden("apply_gate")
    for k, (i, j) in enumerate([(2, 5), (4, 1), (3, 4)]):
        chi = impl.apply_gate(d["V"], i, j, d["psi"])
        assert udist(chi, d[f"chi{k + 1}"]) <= 1e-12


def test_apply_gate_backward(impl):
    d = golden("apply_gate_backward")
    V, psi, dout = d["V"], d["psi"], d["dpsi_out"]
    for i, j in [(2, 5), (4, 1), (3, 4)]:
        dpsi, dV = impl.apply_gate_backward(V, i, j, psi, dout)
        num_psi = num_grad_backward(lambda x: impl.apply_gate(V, i, j, x), psi, dout)
        assert udist(dpsi, num_psi) <= 1e-8
        num_V = num_grad_backward(lambda g: impl.apply_gate(g, i, j, psi), V, dout)
        assert udist(dV, num_V) <= 1e-8


# ------------------------------------------------------------------ test_quantum_circuit.c

def test_apply_quantum_circuit(impl):
    d = golden("apply_quantum_circuit")
    gates = stack(d, "G", 4)
    out = impl.apply_quantum_circuit(gates, d["wires"], d["psi"])
    assert udist(out, d["psi_out"]) <= 1e-12


def test_quantum_circuit_backward(impl):
    d = golden("quantum_circuit_backward")
    gates, wires, psi, dout = stack(d, "G", 5), d["wires"], d["psi"], d["dpsi_out"]
    out, cache = impl.quantum_circuit_forward(gates, wires, psi)
    assert udist(out, d["psi_out"]) <= 1e-12
    dpsi, dgates = impl.quantum_circuit_backward(gates, wires, cache, dout)
    num_psi = num_grad_backward(lambda x: impl.apply_quantum_circuit(gates, wires, x), psi, dout)
    assert udist(dpsi, num_psi) <= 1e-8
    num_g = num_grad_backward(lambda g: impl.apply_quantum_circuit(g, wires, psi), gates, dout)
    assert udist(dgates, num_g) <= 1e-8


def test_quantum_circuit_gates_hessian_vector_product(impl):
    d = golden("quantum_circuit_gates_hessian_vector_product")
    gates, dirs, wires, psi, phi = stack(d, "G", 6), stack(d, "Z", 6), d["wires"], d["psi"], d["phi"]
    out, dg, hg = impl.quantum_circuit_gates_hessian_vector_product(gates, dirs, wires, psi, phi)
    assert udist(out, d["psi_out"]) <= 1e-12
    num_g = num_grad_backward(lambda g: impl.apply_quantum_circuit(g, wires, psi), gates, phi)
    assert udist(dg, num_g) <= 1e-8

    def directed(g):
        _, cache = impl.quantum_circuit_forward(g, wires, psi)
        _, dgs = impl.quantum_circuit_backward(g, wires, cache, phi)
        return np.sum(dgs * dirs)

    num_h = num_grad_backward(lambda g: np.atleast_1d(directed(g)), gates, np.ones(1))
    assert udist(hg, num_h) <= 1e-8


# ------------------------------------------------------------------ test_brickwall_circuit.c

def test_apply_brickwall_unitary(impl):
    d = golden("apply_brickwall_unitary")
    vlist, perms = stack(d, "V", 4), stack(d, "perm", 4)
    for k, nl in enumerate([3, 4]):
        chi = impl.apply_brickwall_unitary(vlist[:nl], perms[:nl], d["psi"])
        assert udist(chi, d[f"chi{k}"]) <= 1e-12


def test_brickwall_unitary_backward(impl):
    d = golden("brickwall_unitary_backward")
    vlist, perms, psi, dout = stack(d, "V", 4), stack(d, "perm", 4), d["psi"], d["dpsi_out"]
    for nl in [3, 4]:
        out, cache = impl.brickwall_unitary_forward(vlist[:nl], perms[:nl], psi)
        assert udist(out, d[f"psi_out{nl - 3}"]) <= 1e-12
        dpsi, dv = impl.brickwall_unitary_backward(vlist[:nl], perms[:nl], cache, dout)
        num_psi = num_grad_backward(lambda x: impl.apply_brickwall_unitary(vlist[:nl], perms[:nl], x), psi, dout)
        assert udist(dpsi, num_psi) <= 1e-8
        num_v = num_grad_backward(lambda v: impl.apply_brickwall_unitary(v, perms[:nl], psi), vlist[:nl], dout)
        assert udist(dv, num_v) <= 1e-8


# ------------------------------------------------------------------ test_target.c

def test_circuit_unitary_target(impl):
    d = golden("circuit_unitary_target")
    f = impl.circuit_unitary_target(impl.target("fixture"), stack(d, "G", 5), d["wires"], 7)
    assert abs(f - d["f"]) <= 1e-12


def test_circuit_unitary_target_and_gradient(impl):
    d = golden("circuit_unitary_target_and_gradient")
    t = impl.target("fixture")
    gates, wires = stack(d, "G", 5), d["wires"]
    f, dg = impl.circuit_unitary_target_and_gradient(t, gates, wires, 8)
    assert abs(f - d["f"]) <= 1e-12
    num = num_grad_wirtinger(lambda g: impl.circuit_unitary_target(t, g, wires, 8), gates)
    assert udist(dg, num) <= 1e-8


def test_circuit_unitary_target_hessian_vector_product(impl):
    d = golden("circuit_unitary_target_hessian_vector_product")
    t = impl.target("fixture")
    gates, dirs, wires = stack(d, "G", 6), stack(d, "Z", 6), d["wires"]
    f, dg, hg = impl.circuit_unitary_target_hessian_vector_product(t, gates, dirs, wires, 7)
    assert abs(f - d["f"]) <= 1e-12
    num = num_grad_wirtinger(lambda g: impl.circuit_unitary_target(t, g, wires, 7), gates)
    assert udist(dg, num) <= 1e-8
    directed = lambda g: np.sum(impl.circuit_unitary_target_and_gradient(t, g, wires, 7)[1] * dirs)
    num_h = num_grad_backward(lambda g: np.atleast_1d(directed(g)), gates, np.ones(1))
    assert udist(hg, num_h) <= 1e-8
    num_f = num_grad_forward(lambda g: impl.circuit_unitary_target_and_gradient(t, g, wires, 7)[1], gates, dirs)
    assert udist(hg, num_f) <= 1e-8


def _tangent_project(impl, gates, mats):
    return np.concatenate([impl.tangent_to_real(gates[k], mats[k]) for k in range(gates.shape[0])])


def test_circuit_unitary_target_projected_hessian_vector_product(impl):
    d = golden("circuit_unitary_target_projected_hessian_vector_product")
    t = impl.target("fixture")
    gates, dirs, wires = stack(d, "G", 6), stack(d, "Z", 6), d["wires"]
    f, g, h = impl.circuit_unitary_target_projected_hessian_vector_product(t, gates, dirs, wires, 7)
    assert abs(f - d["f"]) <= 1e-12

    def proj_grad(gs):
        _, gv = impl.circuit_unitary_target_and_projected_gradient(t, gs, wires, 7)
        return np.stack([impl.real_to_tangent(gv[16 * k:16 * k + 16], gs[k]) for k in range(gs.shape[0])])

    num = num_grad_forward(proj_grad, gates, dirs)
    assert udist(h, _tangent_project(impl, gates, num)) <= 1e-8


def test_brickwall_unitary_target(impl):
    d = golden("brickwall_unitary_target")
    t = impl.target("fixture")
    vlist, perms = stack(d, "V", 5), stack(d, "perm", 5)
    for k, nl in enumerate([4, 5]):
        f = impl.brickwall_unitary_target(t, vlist[:nl], perms[:nl], 8)
        assert abs(f - d[f"f{k}"]) <= 1e-12


def test_brickwall_unitary_target_and_gradient(impl):
    d = golden("brickwall_unitary_target_and_gradient")
    t = impl.target("fixture")
    vlist, perms = stack(d, "V", 5), stack(d, "perm", 5)
    for k, nl in enumerate([4, 5]):
        f, dv = impl.brickwall_unitary_target_and_gradient(t, vlist[:nl], perms[:nl], 8)
        assert abs(f - d[f"f{k}"]) <= 1e-12
        num = num_grad_wirtinger(lambda v: impl.brickwall_unitary_target(t, v, perms[:nl], 8), vlist[:nl])
        assert udist(dv, num) <= 1e-8
        assert udist(dv, d[f"dVlist{k}"]) <= 1e-12


def test_brickwall_unitary_target_and_projected_gradient(impl):
    d = golden("brickwall_unitary_target_and_projected_gradient")
    t = impl.target("fixture")
    f, g = impl.brickwall_unitary_target_and_projected_gradient(t, stack(d, "V", 3), stack(d, "perm", 3), 6)
    assert abs(f - d["f"]) <= 1e-12
    assert udist(g, d["grad"]) <= 1e-14


def test_brickwall_unitary_target_hessian_vector_product(impl):
    d = golden("brickwall_unitary_target_hessian_vector_product")
    t = impl.target("fixture")
    vlist, vdirs, perms = stack(d, "V", 5), stack(d, "Z", 5), stack(d, "perm", 5)
    f, dv, hv = impl.brickwall_unitary_target_hessian_vector_product(t, vlist, vdirs, perms, 6)
    assert abs(f - d["f"]) <= 1e-12
    num = num_grad_wirtinger(lambda v: impl.brickwall_unitary_target(t, v, perms, 6), vlist)
    assert udist(dv, num) <= 1e-8
    directed = lambda v: np.sum(impl.brickwall_unitary_target_and_gradient(t, v, perms, 6)[1] * vdirs)
    num_h = num_grad_backward(lambda v: np.atleast_1d(directed(v)), vlist, np.ones(1))
    assert udist(hv, num_h) <= 1e-7
    num_f = num_grad_forward(lambda v: impl.brickwall_unitary_target_and_gradient(t, v, perms, 6)[1], vlist, vdirs)
    assert udist(hv, num_f) <= 1e-7


def test_brickwall_unitary_target_projected_hessian_vector_product(impl):
    d = golden("brickwall_unitary_target_projected_hessian_vector_product")
    t = impl.target("fixture")
    vlist, vdirs, perms = stack(d, "V", 4), stack(d, "Z", 4), stack(d, "perm", 4)
    f, g, h = impl.brickwall_unitary_target_projected_hessian_vector_product(t, vlist, vdirs, perms, 6)
    assert abs(f - d["f"]) <= 1e-12

    def proj_grad(vs):
        _, gv = impl.brickwall_unitary_target_and_projected_gradient(t, vs, perms, 6)
        return np.stack([impl.real_to_tangent(gv[16 * k:16 * k + 16], vs[k]) for k in range(vs.shape[0])])

    num = num_grad_forward(proj_grad, vlist, vdirs)
    assert udist(h, _tangent_project(impl, vlist, num)) <= 1e-8


# ------------------------------------------------------------------ test_matrix.c

def test_real_to_tangent(impl):
    d = golden("real_to_tangent")
    r = d["r"].ravel()
    z = impl.real_to_tangent(r, d["v"])
    assert np.max(np.abs(impl.tangent_to_real(d["v"], z) - r)) <= 1e-14


def test_project_tangent(impl):
    d = golden("project_tangent")
    assert udist(impl.project_tangent(d["u"], d["z"]), d["p"]) <= 1e-12


def test_polar_factor(impl):
    d = golden("polar_factor")
    assert udist(impl.polar_factor(d["a"]), d["u"]) <= 1e-12


def test_multiply(impl):
    d = golden("multiply")
    mul = impl.multiply_matrices if impl.name == "gpu" else impl.multiply
    assert udist(mul(d["a"], d["b"]), d["c"]) <= 1e-12


# ------------------------------------------------------------------ test_trust_region.c

def test_truncated_cg_hvp(impl):
    d = golden("truncated_cg")
    grad, hess = d["grad"], d["hess"]
    z, on_boundary = impl.truncated_cg_hvp(grad, lambda v: hess @ v, 1.5)
    assert np.max(np.abs(z - d["z"])) <= 1e-14
    assert on_boundary == bool(d["on_boundary"])


# ------------------------------------------------------------------ full-Hessian path
# test_gate.c:203-330, test_brickwall_circuit.c:297-460, test_target.c:1139-1285, 1391-1484,
# test_trust_region.c:88-145

def test_apply_gate_to_array(impl):
    d = golden("apply_gate_to_array")
    for k, (i, j) in enumerate([(2, 5), (4, 1), (3, 4)]):
        chi = impl.apply_gate_to_array(d["V"], i, j, d["psi"])
        assert udist(chi, d[f"chi{k + 1}"]) <= 1e-12


def test_apply_gate_placeholder(impl):
    d = golden("apply_gate_placeholder")
    assert udist(impl.apply_gate_placeholder(2, 5, d["psi"]).ravel(), d["psi_out1"]) <= 1e-12
    assert udist(impl.apply_gate_placeholder(5, 1, d["psi"]).ravel(), d["psi_out2"]) <= 1e-12


def test_brickwall_unitary_backward_hessian(impl):
    d = golden("brickwall_unitary_backward_hessian")
    V, Z, P = stack(d, "V", 4), stack(d, "Z", 4), stack(d, "perm", 4)
    psi, dout = d["psi"], d["dpsi_out"]
    for nl in (3, 4):
        v, z, p = V[:nl], Z[:nl], P[:nl]
        out, cache = impl.brickwall_unitary_forward(v, p, psi)
        assert udist(out, d[f"psi_out{nl - 3}"]) <= 1e-12
        dpsi, dv, hess = impl.brickwall_unitary_backward_hessian(v, p, cache, dout)
        assert udist(hess, hess.T) <= 1e-12
        num_psi = num_grad_backward(lambda x: impl.apply_brickwall_unitary(v, p, x), psi, dout)
        assert udist(dpsi, num_psi) <= 1e-8
        num_v = num_grad_backward(lambda w: impl.apply_brickwall_unitary(w, p, psi), v, dout)
        assert udist(dv, num_v) <= 1e-8

        def grad_of(w):
            _, c = impl.brickwall_unitary_forward(w, p, psi)
            return impl.brickwall_unitary_backward_hessian(w, p, c, dout)[1]

        num_h = num_grad_backward(grad_of, v, z)
        assert udist((hess @ z.ravel()).reshape(nl, 4, 4), num_h) <= 1e-8


def test_brickwall_unitary_target_gradient_hessian(impl):
    d = golden("brickwall_unitary_target_gradient_hessian")
    t = impl.target("fixture")
    V, Z, P = stack(d, "V", 5), stack(d, "Z", 5), stack(d, "perm", 5)
    for k, nl in enumerate([4, 5]):
        v, z, p = V[:nl], Z[:nl], P[:nl]
        f, dv, hess = impl.brickwall_unitary_target_gradient_hessian(t, v, p, 6)
        assert udist(hess, hess.T) <= 1e-12
        assert abs(f - d[f"f{k}"]) <= 1e-12
        assert udist(dv, d[f"dVlist{k}"]) <= 1e-12
        assert udist(hess, d[f"hess{k}"]) <= 1e-12
        num_h = num_grad_wirtinger(lambda w: impl.brickwall_unitary_target_and_gradient(t, w, p, 6)[1], v, z)
        assert udist((hess @ z.ravel()).reshape(nl, 4, 4), num_h) <= 1e-7


def test_brickwall_unitary_target_gradient_vector_hessian_matrix(impl):
    d = golden("brickwall_unitary_target_gradient_vector_hessian_matrix")
    t = impl.target("fixture")
    f, g, H = impl.brickwall_unitary_target_gradient_vector_hessian_matrix(t, stack(d, "V", 5), stack(d, "perm", 5), 6)
    assert abs(f - d["f"]) <= 1e-12
    assert np.max(np.abs(g - d["grad"])) <= 1e-14
    assert np.max(np.abs(H - H.T)) <= 1e-14
    assert np.max(np.abs(H - d["H"])) <= 1e-13


def test_truncated_cg_hmat(impl):
    d = golden("truncated_cg")
    z, on_boundary = impl.truncated_cg_hmat(d["grad"], d["hess"], 1.5)
    assert np.max(np.abs(z - d["z"])) <= 1e-14
    assert on_boundary == bool(d["on_boundary"])


# ------------------------------------------------------------------ sampling estimator
# test_target.c:563-624, 1291-1388, 1487-1563: estimates from 10,000 Haar-random states
# within the reference's statistical bars of the exact values; the Hessian estimate is
# symmetric.

def test_brickwall_unitary_target_sampling(impl):
    d = golden("brickwall_unitary_target_sampling")
    t = impl.target("dense", d["U"])
    vlist, perms = stack(d, "V", 3), stack(d, "perm", 3)
    rng = impl.seed_rng_state(677)
    f = impl.brickwall_unitary_target_sampling(t, vlist, perms, 8, 10000, rng)
    f_ref = impl.brickwall_unitary_target(t, vlist, perms, 8)
    assert abs(f - f_ref) / abs(f_ref) <= 0.2


def test_brickwall_unitary_target_gradient_hessian_sampling(impl):
    d = golden("brickwall_unitary_target_gradient_hessian_sampling")
    t = impl.target("dense", d["U"])
    vlist, perms = stack(d, "V", 3), stack(d, "perm", 3)
    rng = impl.seed_rng_state(823)
    f, dv, hess = impl.brickwall_unitary_target_gradient_hessian_sampling(t, vlist, perms, 6, 10000, rng)
    assert udist(hess, hess.T) <= 1e-12
    f_ref, dv_ref, hess_ref = impl.brickwall_unitary_target_gradient_hessian(t, vlist, perms, 6)
    assert abs(f - f_ref) / abs(f_ref) <= 0.2
    for j in range(3):
        assert udist(dv[j], dv_ref[j]) <= 0.2
    assert udist(hess, hess_ref) <= 0.4


def test_brickwall_unitary_target_gradient_vector_hessian_matrix_sampling(impl):
    d = golden("brickwall_unitary_target_gradient_vector_hessian_matrix_sampling")
    t = impl.target("fixture")
    vlist, perms = stack(d, "V", 5), stack(d, "perm", 5)
    rng = impl.seed_rng_state(401)
    f, g, H = impl.brickwall_unitary_target_gradient_vector_hessian_matrix_sampling(t, vlist, perms, 6, 10000, rng)
    assert np.max(np.abs(H - H.T)) <= 1e-14
    f_ref, g_ref, H_ref = impl.brickwall_unitary_target_gradient_vector_hessian_matrix(t, vlist, perms, 6)
    assert abs(f - f_ref) / abs(f_ref) <= 0.2
    assert np.max(np.abs(g - g_ref)) <= 0.3
    assert np.max(np.abs(H - H_ref)) <= 0.4


# ------------------------------------------------------------------ block-encoding target
# test_target.c:1578-2160: H is the synthetic map on nqubits / 2 qubits

def test_brickwall_blockenc_target(impl):
    d = golden("brickwall_blockenc_target")
    t = impl.target("fixture")
    vlist, perms = stack(d, "V", 5), stack(d, "perm", 5)
    for k, nl in enumerate([4, 5]):
        assert abs(impl.brickwall_blockenc_target(t, vlist[:nl], perms[:nl], 8) - d[f"f{k}"]) <= 1e-12


def test_brickwall_blockenc_target_and_gradient(impl):
    d = golden("brickwall_blockenc_target_and_gradient")
    t = impl.target("fixture")
    vlist, perms = stack(d, "V", 5), stack(d, "perm", 5)
    for k, nl in enumerate([4, 5]):
        f, dv = impl.brickwall_blockenc_target_and_gradient(t, vlist[:nl], perms[:nl], 8)
        assert abs(f - d[f"f{k}"]) <= 1e-12
        assert udist(dv, d[f"dVlist{k}"]) <= 1e-12
        # f is real: the gradient convention is twice the Wirtinger derivative (test_target.c:1724-1729)
        num = 2 * num_grad_wirtinger(lambda v: impl.brickwall_blockenc_target(t, v, perms[:nl], 8), vlist[:nl])
        assert udist(dv, num) <= 1e-8


def test_brickwall_blockenc_target_and_gradient_vector(impl):
    d = golden("brickwall_blockenc_target_and_gradient_vector")
    t = impl.target("fixture")
    f, g = impl.brickwall_blockenc_target_and_gradient_vector(t, stack(d, "V", 3), stack(d, "perm", 3), 6)
    assert abs(f - d["f"]) <= 1e-12
    assert np.max(np.abs(g - d["grad"])) <= 1e-14


def test_brickwall_blockenc_target_gradient_hessian(impl):
    d = golden("brickwall_blockenc_target_gradient_hessian")
    t = impl.target("fixture")
    vlist, perms = stack(d, "V", 5), stack(d, "perm", 5)
    for k, nl in enumerate([4, 5]):
        f, dv, h1, h2 = impl.brickwall_blockenc_target_gradient_hessian(t, vlist[:nl], perms[:nl], 6)
        assert udist(h1, h1.T) <= 1e-12
        assert udist(h2, h2.conj().T) <= 1e-12
        assert abs(f - d[f"f{k}"]) <= 1e-12
        assert udist(dv, d[f"dVlist{k}"]) <= 1e-12
        assert udist(h1, d[f"hess1_{k}"]) <= 1e-12
        assert udist(h2, d[f"hess2_{k}"]) <= 1e-12


def test_brickwall_blockenc_target_gradient_vector_hessian_matrix(impl):
    d = golden("brickwall_blockenc_target_gradient_vector_hessian_matrix")
    t = impl.target("fixture")
    f, g, H = impl.brickwall_blockenc_target_gradient_vector_hessian_matrix(t, stack(d, "V", 5), stack(d, "perm", 5), 6)
    assert abs(f - d["f"]) <= 1e-12
    assert np.max(np.abs(g - d["grad"])) <= 1e-14
    assert np.max(np.abs(H - H.T)) <= 1e-14
    assert np.max(np.abs(H - d["H"])) <= 1e-13
