"""The reference's real-orthogonal build (compiled without COMPLEX_CIRCUIT): its
hot-path tests restated on its golden vectors (test/data/test_*_real.hdf5), run against
the CPU restatement (oracle.RealOracle) and the GPU library librqcopt_gpu_real.so
(marked gpu), with the reference tests' tolerances: 1e-12 for states and f against the
golden vectors, 1e-8 (1e-7 for the Hessian products, 1e-6 for the block-encoding
Hessian) against central differences with h = 1e-5, 1e-14 for the tangent round trip.
The restatement is also compared with the reference's real build compiled in
oracle/_ref on seeded inputs (f, gradients, HVPs, Hessians to 1e-13, a trust-region
run to 1e-10), and the GPU library with both."""
import os

import numpy as np
import pytest

from helpers import GOLDEN, brickwall_instance, num_grad_backward, num_grad_forward, periodic_perms, rel_err, stack, \
    udist

from oracle.oracle import RealOracle, RealReference, real_antisymm, real_fixture_map

IMPLS = [pytest.param("oracle", id="oracle"), pytest.param("gpu", id="gpu", marks=pytest.mark.gpu)]
_cache = {}


def golden_real(name):
    with np.load(os.path.join(GOLDEN, "real", f"{name}.npz")) as z:
        return {k: z[k] for k in z.files}


class _GpuReal:
    name = "gpu"

    def __init__(self):
        from rqcopt_hpc_b200 import real
        self.r = real
        real.lib()

    def target(self, kind, data=None):
        if kind == "fixture":
            return self.r.Target(fn=real_fixture_map)
        if kind == "brickwall":
            return self.r.Target(brickwall=data)
        if kind == "dense":
            return self.r.Target(dense=data)
        raise ValueError(kind)

    def __getattr__(self, name):
        return getattr(self.r, name)


@pytest.fixture(params=IMPLS)
def impl(request):
    name = request.param
    if name == "gpu":
        request.getfixturevalue("gpu")
    if name not in _cache:
        _cache[name] = _GpuReal() if name == "gpu" else RealOracle()
    return _cache[name]


def _real_orthogonal(rng, n=4):
    q, r = np.linalg.qr(rng.standard_normal((n, n)))
    return q * np.sign(np.diagonal(r))


def _real_instance(L, depth, seed, tdepth, tseed):
    rng, trng = np.random.default_rng(seed), np.random.default_rng(tseed)
    return (np.stack([_real_orthogonal(rng) for _ in range(depth)]), periodic_perms(L, depth),
            np.stack([_real_orthogonal(trng) for _ in range(tdepth)]), periodic_perms(L, tdepth))


def _ngrad(f, x, dy=None, h=1e-5):
    """Real backward numerical gradient (test/numerical_gradient.c:9-47)."""
    dy = np.ones(1) if dy is None else dy
    return num_grad_backward(lambda y: np.atleast_1d(f(y.real)), x, dy, h).real


# ------------------------------------------------------------------ test_gate.c, test_quantum_circuit.c

def test_apply_gate(impl):
    d = golden_real("apply_gate")
    for k, (i, j) in enumerate([(2, 5), (4, 1), (3, 4)]):
        assert udist(impl.apply_gate(d["V"], i, j, d["psi"]), d[f"chi{k + 1}"]) <= 1e-12


def test_apply_gate_backward(impl):
    d = golden_real("apply_gate_backward")
    V, psi, dout = d["V"], d["psi"], d["dpsi_out"]
    for i, j in [(2, 5), (4, 1), (3, 4)]:
        dpsi, dV = impl.apply_gate_backward(V, i, j, psi, dout)
        assert udist(dpsi, _ngrad(lambda x: impl.apply_gate(V, i, j, x), psi, dout)) <= 1e-8
        assert udist(dV, _ngrad(lambda g: impl.apply_gate(g, i, j, psi), V, dout)) <= 1e-8


def test_apply_gate_to_array_and_placeholder(impl):
    d = golden_real("apply_gate_to_array")
    for k, (i, j) in enumerate([(2, 5), (4, 1), (3, 4)]):
        assert udist(impl.apply_gate_to_array(d["V"], i, j, d["psi"]), d[f"chi{k + 1}"]) <= 1e-12
    d = golden_real("apply_gate_placeholder")
    assert udist(np.asarray(impl.apply_gate_placeholder(2, 5, d["psi"])).ravel(), d["psi_out1"]) <= 1e-12
    assert udist(np.asarray(impl.apply_gate_placeholder(5, 1, d["psi"])).ravel(), d["psi_out2"]) <= 1e-12


def test_apply_quantum_circuit(impl):
    d = golden_real("apply_quantum_circuit")
    assert udist(impl.apply_quantum_circuit(stack(d, "G", 4), d["wires"], d["psi"]), d["psi_out"]) <= 1e-12


def test_quantum_circuit_backward(impl):
    d = golden_real("quantum_circuit_backward")
    gates, wires, psi, dout = stack(d, "G", 5), d["wires"], d["psi"], d["dpsi_out"]
    out, cache = impl.quantum_circuit_forward(gates, wires, psi)
    assert udist(out, d["psi_out"]) <= 1e-12
    dpsi, dg = impl.quantum_circuit_backward(gates, wires, cache, dout)
    assert udist(dpsi, _ngrad(lambda x: impl.apply_quantum_circuit(gates, wires, x), psi, dout)) <= 1e-8
    assert udist(dg, _ngrad(lambda g: impl.apply_quantum_circuit(g, wires, psi), gates, dout)) <= 1e-8


def test_quantum_circuit_gates_hessian_vector_product(impl):
    d = golden_real("quantum_circuit_gates_hessian_vector_product")
    gates, dirs, wires, psi, phi = stack(d, "G", 6), stack(d, "Z", 6), d["wires"], d["psi"], d["phi"]
    out, dg, hg = impl.quantum_circuit_gates_hessian_vector_product(gates, dirs, wires, psi, phi)
    assert udist(out, d["psi_out"]) <= 1e-12
    assert udist(dg, _ngrad(lambda g: impl.apply_quantum_circuit(g, wires, psi), gates, phi)) <= 1e-8

    def directed(g):
        _, cache = impl.quantum_circuit_forward(g, wires, psi)
        return np.sum(impl.quantum_circuit_backward(g, wires, cache, phi)[1] * dirs)

    assert udist(hg, _ngrad(directed, gates)) <= 1e-8


# ------------------------------------------------------------------ test_brickwall_circuit.c

def test_apply_brickwall_unitary(impl):
    d = golden_real("apply_brickwall_unitary")
    vlist, perms = stack(d, "V", 4), stack(d, "perm", 4)
    for k, nl in enumerate([3, 4]):
        assert udist(impl.apply_brickwall_unitary(vlist[:nl], perms[:nl], d["psi"]), d[f"chi{k}"]) <= 1e-12


def test_brickwall_unitary_backward(impl):
    d = golden_real("brickwall_unitary_backward")
    vlist, perms, psi, dout = stack(d, "V", 4), stack(d, "perm", 4), d["psi"], d["dpsi_out"]
    for nl in (3, 4):
        out, cache = impl.brickwall_unitary_forward(vlist[:nl], perms[:nl], psi)
        assert udist(out, d[f"psi_out{nl - 3}"]) <= 1e-12
        dpsi, dv = impl.brickwall_unitary_backward(vlist[:nl], perms[:nl], cache, dout)
        assert udist(dpsi, _ngrad(lambda x: impl.apply_brickwall_unitary(vlist[:nl], perms[:nl], x), psi, dout)) <= 1e-8
        assert udist(dv, _ngrad(lambda v: impl.apply_brickwall_unitary(v, perms[:nl], psi), vlist[:nl], dout)) <= 1e-8


def test_brickwall_unitary_backward_hessian(impl):
    d = golden_real("brickwall_unitary_backward_hessian")
    V, Z, P, psi, dout = stack(d, "V", 4), stack(d, "Z", 4), stack(d, "perm", 4), d["psi"], d["dpsi_out"]
    for nl in (3, 4):
        v, z, p = V[:nl], Z[:nl], P[:nl]
        out, cache = impl.brickwall_unitary_forward(v, p, psi)
        assert udist(out, d[f"psi_out{nl - 3}"]) <= 1e-12
        dpsi, dv, hess = impl.brickwall_unitary_backward_hessian(v, p, cache, dout)
        assert udist(hess, hess.T) <= 1e-12
        assert udist(dpsi, _ngrad(lambda x: impl.apply_brickwall_unitary(v, p, x), psi, dout)) <= 1e-8
        assert udist(dv, _ngrad(lambda w: impl.apply_brickwall_unitary(w, p, psi), v, dout)) <= 1e-8

        def grad_of(w):
            _, c = impl.brickwall_unitary_forward(w, p, psi)
            return impl.brickwall_unitary_backward_hessian(w, p, c, dout)[1]

        num_h = num_grad_backward(lambda w: grad_of(w.real), v, z).real
        assert udist((hess @ z.ravel()).reshape(nl, 4, 4), num_h) <= 1e-8


# ------------------------------------------------------------------ test_target.c (real build)

def test_circuit_unitary_target(impl):
    d = golden_real("circuit_unitary_target")
    assert abs(impl.circuit_unitary_target(impl.target("fixture"), stack(d, "G", 5), d["wires"], 7) - d["f"]) <= 1e-12


def test_circuit_unitary_target_and_gradient(impl):
    d = golden_real("circuit_unitary_target_and_gradient")
    t, gates, wires = impl.target("fixture"), stack(d, "G", 5), d["wires"]
    f, dg = impl.circuit_unitary_target_and_gradient(t, gates, wires, 8)
    assert abs(f - d["f"]) <= 1e-12
    assert udist(dg, _ngrad(lambda g: impl.circuit_unitary_target(t, g, wires, 8), gates)) <= 1e-8


def test_circuit_unitary_target_hessian_vector_product(impl):
    d = golden_real("circuit_unitary_target_hessian_vector_product")
    t, gates, dirs, wires = impl.target("fixture"), stack(d, "G", 6), stack(d, "Z", 6), d["wires"]
    f, dg, hg = impl.circuit_unitary_target_hessian_vector_product(t, gates, dirs, wires, 7)
    assert abs(f - d["f"]) <= 1e-12
    assert udist(dg, _ngrad(lambda g: impl.circuit_unitary_target(t, g, wires, 7), gates)) <= 1e-8
    directed = lambda g: np.sum(impl.circuit_unitary_target_and_gradient(t, g, wires, 7)[1] * dirs)
    assert udist(hg, _ngrad(directed, gates)) <= 1e-8


def _tangent_project(impl, gates, mats):
    return np.concatenate([impl.tangent_to_real(gates[k], mats[k]) for k in range(gates.shape[0])])


def test_circuit_unitary_target_projected_hessian_vector_product(impl):
    d = golden_real("circuit_unitary_target_projected_hessian_vector_product")
    t, gates, dirs, wires = impl.target("fixture"), stack(d, "G", 6), stack(d, "Z", 6), d["wires"]
    f, g, h = impl.circuit_unitary_target_projected_hessian_vector_product(t, gates, dirs, wires, 7)
    assert abs(f - d["f"]) <= 1e-12
    assert g.shape == h.shape == (36,)

    def proj_grad(gs):
        gs = gs.real
        _, gv = impl.circuit_unitary_target_and_projected_gradient(t, gs, wires, 7)
        return np.stack([impl.real_to_tangent(gv[6 * k:6 * k + 6], gs[k]) for k in range(gs.shape[0])])

    num = num_grad_forward(proj_grad, gates, dirs).real
    assert udist(h, _tangent_project(impl, gates, num)) <= 1e-8


def test_brickwall_unitary_target(impl):
    d = golden_real("brickwall_unitary_target")
    vlist, perms = stack(d, "V", 5), stack(d, "perm", 5)
    for k, nl in enumerate([4, 5]):
        assert abs(impl.brickwall_unitary_target(impl.target("fixture"), vlist[:nl], perms[:nl], 8) - d[f"f{k}"]) <= 1e-12


def test_brickwall_unitary_target_and_gradient(impl):
    d = golden_real("brickwall_unitary_target_and_gradient")
    t, vlist, perms = impl.target("fixture"), stack(d, "V", 5), stack(d, "perm", 5)
    for k, nl in enumerate([4, 5]):
        f, dv = impl.brickwall_unitary_target_and_gradient(t, vlist[:nl], perms[:nl], 8)
        assert abs(f - d[f"f{k}"]) <= 1e-12
        assert udist(dv, d[f"dVlist{k}"]) <= 1e-12
        assert udist(dv, _ngrad(lambda v: impl.brickwall_unitary_target(t, v, perms[:nl], 8), vlist[:nl])) <= 1e-8


def test_brickwall_unitary_target_hessian_vector_product(impl):
    d = golden_real("brickwall_unitary_target_hessian_vector_product")
    t, vlist, vdirs, perms = impl.target("fixture"), stack(d, "V", 5), stack(d, "Z", 5), stack(d, "perm", 5)
    f, dv, hv = impl.brickwall_unitary_target_hessian_vector_product(t, vlist, vdirs, perms, 6)
    assert abs(f - d["f"]) <= 1e-12
    assert udist(dv, _ngrad(lambda v: impl.brickwall_unitary_target(t, v, perms, 6), vlist)) <= 1e-8
    directed = lambda v: np.sum(impl.brickwall_unitary_target_and_gradient(t, v, perms, 6)[1] * vdirs)
    assert udist(hv, _ngrad(directed, vlist)) <= 1e-7


def test_brickwall_unitary_target_projected_hessian_vector_product(impl):
    d = golden_real("brickwall_unitary_target_projected_hessian_vector_product")
    t, vlist, vdirs, perms = impl.target("fixture"), stack(d, "V", 4), stack(d, "Z", 4), stack(d, "perm", 4)
    f, g, h = impl.brickwall_unitary_target_projected_hessian_vector_product(t, vlist, vdirs, perms, 6)
    assert abs(f - d["f"]) <= 1e-12

    def proj_grad(vs):
        vs = vs.real
        _, gv = impl.brickwall_unitary_target_and_projected_gradient(t, vs, perms, 6)
        return np.stack([impl.real_to_tangent(gv[6 * k:6 * k + 6], vs[k]) for k in range(vs.shape[0])])

    num = num_grad_forward(proj_grad, vlist, vdirs).real
    assert udist(h, _tangent_project(impl, vlist, num)) <= 1e-8


def test_brickwall_unitary_target_gradient_hessian(impl):
    d = golden_real("brickwall_unitary_target_gradient_hessian")
    t, V, Z, P = impl.target("fixture"), stack(d, "V", 5), stack(d, "Z", 5), stack(d, "perm", 5)
    for k, nl in enumerate([4, 5]):
        v, z, p = V[:nl], Z[:nl], P[:nl]
        f, dv, hess = impl.brickwall_unitary_target_gradient_hessian(t, v, p, 6)
        assert udist(hess, hess.T) <= 1e-12
        assert abs(f - d[f"f{k}"]) <= 1e-12
        assert udist(dv, d[f"dVlist{k}"]) <= 1e-12
        assert udist(hess, d[f"hess{k}"]) <= 1e-12
        num = num_grad_backward(lambda w: impl.brickwall_unitary_target_and_gradient(t, w.real, p, 6)[1], v, z).real
        assert udist((hess @ z.ravel()).reshape(nl, 4, 4), num) <= 1e-7


def test_brickwall_unitary_target_sampling(impl):
    d = golden_real("brickwall_unitary_target_sampling")
    t, vlist, perms = impl.target("dense", d["U"]), stack(d, "V", 3), stack(d, "perm", 3)
    f = impl.brickwall_unitary_target_sampling(t, vlist, perms, 8, 10000, impl.seed_rng_state(677))
    f_ref = impl.brickwall_unitary_target(t, vlist, perms, 8)
    assert abs(f - f_ref) / abs(f_ref) <= 0.2


def test_brickwall_unitary_target_gradient_hessian_sampling(impl):
    d = golden_real("brickwall_unitary_target_gradient_hessian_sampling")
    t, vlist, perms = impl.target("dense", d["U"]), stack(d, "V", 3), stack(d, "perm", 3)
    f, dv, hess = impl.brickwall_unitary_target_gradient_hessian_sampling(t, vlist, perms, 6, 10000,
                                                                          impl.seed_rng_state(823))
    assert udist(hess, hess.T) <= 1e-12
    f_ref, dv_ref, hess_ref = impl.brickwall_unitary_target_gradient_hessian(t, vlist, perms, 6)
    assert abs(f - f_ref) / abs(f_ref) <= 0.2
    for j in range(3):
        assert udist(dv[j], dv_ref[j]) <= 0.2
    assert udist(hess, hess_ref) <= 0.4


def test_brickwall_blockenc_target(impl):
    d = golden_real("brickwall_blockenc_target")
    vlist, perms = stack(d, "V", 5), stack(d, "perm", 5)
    for k, nl in enumerate([4, 5]):
        assert abs(impl.brickwall_blockenc_target(impl.target("fixture"), vlist[:nl], perms[:nl], 8) - d[f"f{k}"]) <= 1e-12


def test_brickwall_blockenc_target_and_gradient(impl):
    d = golden_real("brickwall_blockenc_target_and_gradient")
    t, vlist, perms = impl.target("fixture"), stack(d, "V", 5), stack(d, "perm", 5)
    for k, nl in enumerate([4, 5]):
        f, dv = impl.brickwall_blockenc_target_and_gradient(t, vlist[:nl], perms[:nl], 8)
        assert abs(f - d[f"f{k}"]) <= 1e-12
        assert udist(dv, d[f"dVlist{k}"]) <= 1e-12
        assert udist(dv, _ngrad(lambda v: impl.brickwall_blockenc_target(t, v, perms[:nl], 8), vlist[:nl])) <= 1e-8


def test_brickwall_blockenc_target_gradient_hessian(impl):
    d = golden_real("brickwall_blockenc_target_gradient_hessian")
    t, V, Z, P = impl.target("fixture"), stack(d, "V", 5), stack(d, "Z", 5), stack(d, "perm", 5)
    for k, nl in enumerate([4, 5]):
        v, z, p = V[:nl], Z[:nl], P[:nl]
        f, dv, hess = impl.brickwall_blockenc_target_gradient_hessian(t, v, p, 6)
        assert abs(f - d[f"f{k}"]) <= 1e-12
        assert udist(dv, d[f"dVlist{k}"]) <= 1e-12
        assert udist(hess, d[f"hess{k}"]) <= 1e-12
        num = num_grad_backward(lambda w: impl.brickwall_blockenc_target_and_gradient(t, w.real, p, 6)[1], v, z).real
        assert udist((hess @ z.ravel()).reshape(nl, 4, 4), num) <= 1e-6


# ------------------------------------------------------------------ test_matrix.c (real build)

def test_real_to_tangent(impl):
    d = golden_real("real_to_tangent")
    z = impl.real_to_tangent(d["r"], d["v"])
    assert np.max(np.abs(impl.tangent_to_real(d["v"], z) - d["r"])) <= 1e-14


def test_project_tangent(impl):
    d = golden_real("project_tangent")
    assert udist(impl.project_tangent(d["u"], d["z"]), d["p"]) <= 1e-12


def test_polar_factor(impl):
    d = golden_real("polar_factor")
    assert udist(impl.polar_factor(d["a"]), d["u"]) <= 1e-12


def test_multiply(impl):
    d = golden_real("multiply")
    mul = impl.multiply_matrices if impl.name == "gpu" else (lambda a, b: a @ b)
    assert udist(mul(d["a"], d["b"]), d["c"]) <= 1e-12


# ------------------------------------------------------------------ against the compiled real build

ref_needed = pytest.mark.skipif(not RealReference.available(), reason="reference real build not present")


def _seeded(L=8, depth=4, tdepth=3, seed=3):
    vlist, perms, tv, tp = _real_instance(L, depth, seed, tdepth, seed + 1)
    rng = np.random.default_rng(seed + 2)
    vdirs = np.stack([vlist[k] @ real_antisymm(rng.standard_normal(6)) for k in range(depth)])
    return vlist, perms, tv, tp, vdirs


def _compare_with_reference(impl, ref, tol):
    L = 8
    vlist, perms, tv, tp, vdirs = _seeded(L)
    ti, tr = impl.target("brickwall", (tv, tp)), ref.target("brickwall", (tv, tp))
    f, g, h = impl.brickwall_unitary_target_projected_hessian_vector_product(ti, vlist, vdirs, perms, L)
    fr, gr, hr = ref.brickwall_unitary_target_projected_hessian_vector_product(tr, vlist, vdirs, perms, L)
    assert abs(f - fr) <= tol * abs(fr) and rel_err(g, gr) <= tol and rel_err(h, hr) <= tol
    f, dv, hv = impl.brickwall_unitary_target_hessian_vector_product(ti, vlist, vdirs, perms, L)
    fr, dvr, hvr = ref.brickwall_unitary_target_hessian_vector_product(tr, vlist, vdirs, perms, L)
    assert rel_err(dv, dvr) <= tol and rel_err(hv, hvr) <= tol
    f, dv, hess = impl.brickwall_unitary_target_gradient_hessian(ti, vlist, perms, L)
    fr, dvr, hessr = ref.brickwall_unitary_target_gradient_hessian(tr, vlist, perms, L)
    assert abs(f - fr) <= tol * abs(fr) and rel_err(dv, dvr) <= tol and rel_err(hess, hessr) <= tol
    hv, hp = vlist[:2], periodic_perms(L // 2, 2)
    th, thr = impl.target("brickwall", (hv, hp)), ref.target("brickwall", (hv, hp))
    f, dv, hess = impl.brickwall_blockenc_target_gradient_hessian(th, vlist, perms, L)
    fr, dvr, hessr = ref.brickwall_blockenc_target_gradient_hessian(thr, vlist, perms, L)
    assert abs(f - fr) <= tol * abs(fr) and rel_err(dv, dvr) <= tol and rel_err(hess, hessr) <= tol
    # sampled: the same real sample states from the same generator state
    f, dv, hess = impl.brickwall_unitary_target_gradient_hessian_sampling(ti, vlist, perms, L, 40, impl.seed_rng_state(5))
    fr, dvr, hessr = ref.brickwall_unitary_target_gradient_hessian_sampling(tr, vlist, perms, L, 40, ref.seed_rng_state(5))
    assert abs(f - fr) <= 1e3 * tol * abs(fr) and rel_err(dv, dvr) <= 1e3 * tol and rel_err(hess, hessr) <= 1e3 * tol
    # trust region over 6 parameters per gate
    fi, vo = impl.optimize_brickwall_circuit_hvp(ti, vlist, perms, L, 4)
    fir, vor = ref.optimize_brickwall_circuit_hvp(tr, vlist, perms, L, 4)
    assert rel_err(fi, fir) <= 1e-10 and rel_err(vo, vor) <= 1e-9
    assert np.max(np.abs(np.einsum("kij,kil->kjl", vo, vo) - np.eye(4))) <= 1e-13


@ref_needed
def test_real_oracle_matches_compiled_real_build():
    _compare_with_reference(RealOracle(), RealReference(), 1e-13)


def _circuit_case(L=7, ng=9, seed=21):
    rng = np.random.default_rng(seed)
    gates = np.stack([_real_orthogonal(rng) for _ in range(ng)])
    wires = np.stack([rng.choice(L, 2, replace=False) for _ in range(ng)]).astype(np.int32)
    dirs = np.stack([gates[k] @ real_antisymm(rng.standard_normal(6)) for k in range(ng)])
    return gates, wires, dirs


@ref_needed
def test_real_oracle_circuit_paths_match_compiled_real_build():
    """General circuits against the dense real target of the reference tests' map:
    projected HVP to 1e-13 and a 4-iteration optimize_quantum_circuit to 1e-10."""
    o, r = RealOracle(), RealReference()
    gates, wires, dirs = _circuit_case()
    to, tr = o.target("fixture"), r.target("fixture")
    f, g, h = o.circuit_unitary_target_projected_hessian_vector_product(to, gates, dirs, wires, 7)
    fr, gr, hr = r.circuit_unitary_target_projected_hessian_vector_product(tr, gates, dirs, wires, 7)
    assert abs(f - fr) <= 1e-13 * abs(fr) and rel_err(g, gr) <= 1e-13 and rel_err(h, hr) <= 1e-13
    fi, go = o.optimize_quantum_circuit(to, gates, wires, 7, 4)
    fir, gor = r.optimize_quantum_circuit(tr, gates, wires, 7, 4)
    assert rel_err(fi, fir) <= 1e-10 and rel_err(go, gor) <= 1e-9


@ref_needed
@pytest.mark.gpu
def test_gpu_real_build_matches_compiled_real_build(gpu):
    _compare_with_reference(_GpuReal(), RealReference(), 1e-12)


@pytest.mark.gpu
def test_gpu_real_build_matches_real_oracle_at_l12(gpu):
    """A size the compiled reference takes long for: f, projected gradient and HVP at
    L=12 against the restatement (device-native brickwall target; dense target for f)."""
    L = 12
    vlist, perms, tv, tp = _real_instance(L, 5, 9, 3, 10)
    rng = np.random.default_rng(11)
    vdirs = np.stack([vlist[k] @ real_antisymm(rng.standard_normal(6)) for k in range(5)])
    g, o = _GpuReal(), RealOracle()
    f, gv, hv = g.brickwall_unitary_target_projected_hessian_vector_product(g.target("brickwall", (tv, tp)), vlist, vdirs,
                                                                            perms, L)
    fo, gvo, hvo = o.brickwall_unitary_target_projected_hessian_vector_product(o.target("brickwall", (tv, tp)), vlist,
                                                                               vdirs, perms, L)
    assert abs(f - fo) <= 1e-12 * abs(fo) and rel_err(gv, gvo) <= 1e-12 and rel_err(hv, hvo) <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("L,precision,gpp,chunk", [(14, "c128", 4, 0), (12, "mixed", 4, 0), (12, "c64", 4, 40),
                                                   (10, "c128", 1, 24), (10, "c64", 1, 0)])
def test_paired_columns_equal_plain_columns(gpu, L, precision, gpp, chunk):
    """Size-independent check of the paired basis columns: the complex library on real
    gates and a real target, with and without rqcopt_gpu_set_real_pairs, gives the same
    f, gradient and HVP (real parts; complex128 1e-12, complex64 passes 1e-5 as the
    mixed engine's own bar), on the fused engine (4 gates per pass) and the per-gate
    engine (1), with ragged column chunks."""
    vlist, perms, tv, tp = _real_instance(L, 6, 40 + L, 3, 41 + L)
    rng = np.random.default_rng(L)
    vdirs = np.stack([vlist[k] @ real_antisymm(rng.standard_normal(6)) for k in range(6)])
    t = gpu.Target(brickwall=(tv.astype(complex), tp))
    prec = {"c128": gpu.PRECISION_C128, "mixed": gpu.PRECISION_MIXED, "c64": gpu.PRECISION_C64}[precision]
    tol = 1e-12 if precision == "c128" else 1e-5
    gpu.set_precision(prec)
    gpu.set_gates_per_pass(gpp)
    gpu.set_column_chunk(chunk)
    try:
        plain = gpu.brickwall_unitary_target_hessian_vector_product(t, vlist.astype(complex), vdirs.astype(complex),
                                                                     perms, L)
        gpu.lib().rqcopt_gpu_set_real_pairs(1)
        try:
            paired = gpu.brickwall_unitary_target_hessian_vector_product(t, vlist.astype(complex),
                                                                          vdirs.astype(complex), perms, L)
        finally:
            gpu.lib().rqcopt_gpu_set_real_pairs(0)
    finally:
        gpu.set_precision(gpu.PRECISION_C128)
        gpu.set_gates_per_pass(4)
        gpu.set_column_chunk(0)
    f0, dv0, hv0 = plain
    f1, dv1, hv1 = paired
    assert abs(f1.imag) == 0 and np.all(dv1.imag == 0) and np.all(hv1.imag == 0)
    assert abs(f1.real - f0.real) <= tol * abs(f0.real)
    assert rel_err(dv1.real, dv0.real) <= tol and rel_err(hv1.real, hv0.real) <= tol
    # the plain evaluation of a real problem has zero imaginary parts up to rounding
    assert np.max(np.abs(dv0.imag)) <= 10 * tol * np.max(np.abs(dv0.real))


def test_real_library_rejects_invalid_arguments():
    """Invalid sizes, permutations and wires are refused with the library's argument error
    (-6) before any device work, as in the complex library (no GPU needed)."""
    from rqcopt_hpc_b200 import real
    vlist, perms, tv, tp = _real_instance(6, 3, 1, 2, 2)
    t = real.Target(brickwall=(tv, tp))
    calls = [lambda: real.brickwall_unitary_target(t, vlist, perms, 5),
             lambda: real.brickwall_unitary_target_and_projected_gradient(t, vlist, np.zeros((3, 6), np.int32), 6),
             lambda: real.circuit_unitary_target(t, vlist, [[0, 0], [1, 2], [2, 3]], 6),
             lambda: real.brickwall_blockenc_target(t, vlist, perms, 5)]
    for call in calls:
        with pytest.raises(real.RqcError) as e:
            call()
        assert e.value.code == -6
