"""GPU library against the CPU oracle on the seeded brickwall workloads, through
the C ABI.  Bar: 1e-12 relative (infinity norm relative to the oracle's infinity
norm) in f, gradient and HVP for the complex128 path; 1e-5 for complex64
passes.  Also checks the host-callback target path, general circuits,
column chunking and the forward/adjoint round trip at a larger size."""
import numpy as np
import pytest

from helpers import (brickwall_instance, crandn, haar_unitary, periodic_perms, random_tangent_dirs,
                     real_to_antisymm, rel_err)

pytestmark = pytest.mark.gpu


def _dirs(vlist, seed):
    r = random_tangent_dirs(vlist, seed)
    return np.stack([vlist[k] @ real_to_antisymm(r[k]) for k in range(vlist.shape[0])])


@pytest.fixture(autouse=True)
def _defaults(gpu):
    gpu.set_precision(gpu.PRECISION_C128)
    gpu.set_column_chunk(0)
    yield
    gpu.set_precision(gpu.PRECISION_C128)
    gpu.set_column_chunk(0)


@pytest.mark.parametrize("L,depth,tdepth", [(4, 3, 3), (6, 5, 3), (8, 5, 3), (10, 7, 3)])
def test_brickwall_projected_hvp_matches_oracle(gpu, oracle, L, depth, tdepth):
    vlist, perms, tvlist, tperms = brickwall_instance(L, depth, 100 + L, tdepth, 200 + L)
    vdirs = _dirs(vlist, 300 + L)
    f, g, h = gpu.brickwall_unitary_target_projected_hessian_vector_product(
        gpu.Target(brickwall=(tvlist, tperms)), vlist, vdirs, perms, L)
    fo, go, ho = oracle.brickwall_unitary_target_projected_hessian_vector_product(
        oracle.target("brickwall", (tvlist, tperms)), vlist, vdirs, perms, L)
    assert abs(f - fo) <= 1e-12 * abs(fo)
    assert rel_err(g, go) <= 1e-12
    assert rel_err(h, ho) <= 1e-12


def test_chunked_columns_match_single_chunk(gpu):
    L = 8
    vlist, perms, tvlist, tperms = brickwall_instance(L, 5, 7, 3, 8)
    vdirs = _dirs(vlist, 9)
    t = gpu.Target(brickwall=(tvlist, tperms))
    ref = gpu.brickwall_unitary_target_projected_hessian_vector_product(t, vlist, vdirs, perms, L)
    for chunk in (1, 3, 64, 100):
        gpu.set_column_chunk(chunk)
        got = gpu.brickwall_unitary_target_projected_hessian_vector_product(t, vlist, vdirs, perms, L)
        assert abs(got[0] - ref[0]) <= 1e-12 * abs(ref[0])
        assert rel_err(got[1], ref[1]) <= 1e-12 and rel_err(got[2], ref[2]) <= 1e-12


def test_host_callback_target_matches_device_target(gpu):
    L = 6
    vlist, perms, tvlist, tperms = brickwall_instance(L, 3, 11, 3, 12)
    vdirs = _dirs(vlist, 13)
    dev = gpu.brickwall_unitary_target_projected_hessian_vector_product(
        gpu.Target(brickwall=(tvlist, tperms)), vlist, vdirs, perms, L)
    host = gpu.brickwall_unitary_target_projected_hessian_vector_product(
        gpu.Target(fn=lambda x: gpu.apply_brickwall_unitary(tvlist, tperms, x)), vlist, vdirs, perms, L)
    for a, b in zip(dev, host):
        assert rel_err(a, b) <= 1e-12


def test_general_circuit_hvp_matches_oracle(gpu, oracle):
    L, G = 7, 9
    rng = np.random.default_rng(21)
    gates = np.stack([haar_unitary(rng) for _ in range(G)])
    wires = np.array([rng.choice(L, 2, replace=False) for _ in range(G)], np.int32)
    dirs = 0.5 * crandn((G, 4, 4), rng)
    u = crandn((1 << L, 1 << L), rng)
    fg = gpu.circuit_unitary_target_hessian_vector_product(gpu.Target(fn=lambda x: u @ x), gates, dirs, wires, L)
    fo = oracle.circuit_unitary_target_hessian_vector_product(oracle.target("dense", u), gates, dirs, wires, L)
    assert abs(fg[0] - fo[0]) <= 1e-12 * abs(fo[0])
    assert rel_err(fg[1], fo[1]) <= 1e-12
    assert rel_err(fg[2], fo[2]) <= 1e-12


def test_circuit_target_descriptor(gpu, oracle):
    L = 6
    vlist, perms, tvlist, tperms = brickwall_instance(L, 3, 31, 3, 32)
    per = L // 2
    tgates = np.repeat(tvlist, per, axis=0)
    twires = np.concatenate([tperms[l].reshape(per, 2) for l in range(3)]).astype(np.int32)
    a = gpu.brickwall_unitary_target(gpu.Target(circuit=(tgates, twires)), vlist, perms, L)
    b = oracle.brickwall_unitary_target(oracle.target("brickwall", (tvlist, tperms)), vlist, perms, L)
    assert abs(a - b) <= 1e-12 * abs(b)


def test_complex64_passes_within_single_precision(gpu, oracle):
    L = 8
    vlist, perms, tvlist, tperms = brickwall_instance(L, 5, 0, 3, 1)
    vdirs = _dirs(vlist, 2)
    gpu.set_precision(gpu.PRECISION_C64)
    f, g, h = gpu.brickwall_unitary_target_projected_hessian_vector_product(
        gpu.Target(brickwall=(tvlist, tperms)), vlist, vdirs, perms, L)
    fo, go, ho = oracle.brickwall_unitary_target_projected_hessian_vector_product(
        oracle.target("brickwall", (tvlist, tperms)), vlist, vdirs, perms, L)
    assert abs(f - fo) <= 1e-5 * abs(fo)
    assert rel_err(g, go) <= 1e-5
    assert rel_err(h, ho) <= 1e-5


def test_trust_region_retraces_oracle(gpu, oracle):
    """f iterates, final gates and the accept / reject and on-boundary decision of every
    iteration equal the oracle's (src/trust_region.c:330-352)."""
    L = 8
    vlist, perms, tvlist, tperms = brickwall_instance(L, 5, 0, 3, 1)
    gpu.set_precision(gpu.PRECISION_C128)
    f_g, v_g = gpu.optimize_brickwall_circuit_hvp(gpu.Target(brickwall=(tvlist, tperms)), vlist, perms, L, 10)
    tr = gpu.optimizer_trace()
    f_o, v_o, acc, bnd = oracle.optimize_brickwall_circuit_hvp(oracle.target("brickwall", (tvlist, tperms)),
                                                                vlist, perms, L, 10)
    assert rel_err(f_g, f_o) <= 1e-12
    assert rel_err(v_g, v_o) <= 1e-10
    assert np.array_equal(tr["accepted"], acc)
    assert np.array_equal(tr["on_boundary"], bnd)
    assert not tr["refined"].any() or np.all(tr["refined"] == 1)   # complex128 throughout


def test_general_circuit_trust_region_decisions_match_oracle(gpu, oracle):
    L = 6
    rng = np.random.default_rng(77)
    gates = np.stack([haar_unitary(rng) for _ in range(7)])
    wires = np.array([rng.choice(L, 2, replace=False) for _ in range(7)], np.int32)
    _, _, tvlist, tperms = brickwall_instance(L, 1, 0, 3, 78)
    gpu.set_precision(gpu.PRECISION_C128)
    f_g, g_g = gpu.optimize_quantum_circuit(gpu.Target(brickwall=(tvlist, tperms)), gates, wires, L, 12)
    tr = gpu.optimizer_trace()
    f_o, g_o, acc, bnd = oracle.optimize_quantum_circuit(oracle.target("brickwall", (tvlist, tperms)), gates, wires,
                                                         L, 12)
    assert rel_err(f_g, f_o) <= 1e-12
    assert np.array_equal(tr["accepted"], acc)
    assert np.array_equal(tr["on_boundary"], bnd)


@pytest.mark.parametrize("L,depth,seed,niter", [(8, 3, 0, 60), (6, 5, 5, 80)])
def test_mixed_precision_reaches_the_complex128_optimum(gpu, oracle, L, depth, seed, niter):
    """Mixed precision (complex64 HVPs until the gradient norm falls below 1e-5, then
    complex128) on problems the trust region drives to convergence within niter
    iterations (the oracle's gradient norm ends below 1e-8): the refinement engages,
    tCG takes several inner steps, and the final f agrees with the complex128 run and
    with the oracle's FP64 run to 1e-10 relative."""
    vlist, perms, tvlist, tperms = brickwall_instance(L, depth, seed, 3, seed + 1)
    tgt = gpu.Target(brickwall=(tvlist, tperms))
    try:
        gpu.set_precision(gpu.PRECISION_C128)
        f128, v128 = gpu.optimize_brickwall_circuit_hvp(tgt, vlist, perms, L, niter)
        gpu.set_precision(gpu.PRECISION_MIXED)
        fmix, vmix = gpu.optimize_brickwall_circuit_hvp(tgt, vlist, perms, L, niter)
        tr = gpu.optimizer_trace()
    finally:
        gpu.set_precision(gpu.PRECISION_C128)
    f_o, v_o, _, _ = oracle.optimize_brickwall_circuit_hvp(oracle.target("brickwall", (tvlist, tperms)), vlist, perms,
                                                           L, niter)
    assert tr["refined"][0] == 0 and tr["refined"][-1] == 1, tr["refined"]
    assert tr["inner"].max() >= 3
    assert abs(fmix[-1] - f128[-1]) <= 1e-10 * abs(f128[-1]), (fmix[-1], f128[-1])
    assert abs(fmix[-1] - f_o[-1]) <= 1e-10 * abs(f_o[-1])
    # the mixed run's reported f values are complex128 evaluations: each equals the oracle's f at its iterate
    _, g_final = oracle.brickwall_unitary_target_and_projected_gradient(oracle.target("brickwall", (tvlist, tperms)),
                                                                        vmix, perms, L)
    assert np.linalg.norm(g_final) <= 1e-6


def test_add_statevectors_matches_oracle(gpu, oracle):
    """src/statevector.c:132-142 on host arrays (staged), device tensors and managed
    statevectors from allocate_statevector."""
    import ctypes as C
    import torch
    from rqcopt_hpc_b200.abi import Statevector
    rng = np.random.default_rng(91)
    for L in (1, 3, 20):
        a, b = crandn(1 << L, rng), crandn(1 << L, rng)
        want = oracle.add_statevectors(a, b)
        assert np.array_equal(gpu.add_statevectors(a, b), want)
        ta, tb = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
        assert np.array_equal(gpu.add_statevectors(ta, tb).cpu().numpy(), want)
    lib = gpu.lib()
    L = 10
    sv = [Statevector() for _ in range(3)]
    for s in sv:
        assert lib.allocate_statevector(L, C.byref(s)) == 0
    try:
        a, b = crandn(1 << L, rng), crandn(1 << L, rng)
        for s, v in zip(sv[:2], (a, b)):
            C.memmove(s.data, v.ctypes.data, v.nbytes)
        lib.add_statevectors(C.byref(sv[0]), C.byref(sv[1]), C.byref(sv[2]))
        assert lib.rqcopt_gpu_last_error() == 0
        out = np.empty(1 << L, np.complex128)
        C.memmove(out.ctypes.data, sv[2].data, out.nbytes)
        assert np.array_equal(out, oracle.add_statevectors(a, b))
    finally:
        for s in sv:
            lib.free_statevector(C.byref(s))


@pytest.mark.parametrize("L,depth,chunk", [(8, 5, 0), (10, 7, 24), (12, 3, 0)])
def test_reconstructing_reverse_pass_matches_recomputing(gpu, oracle, L, depth, chunk):
    """complex128 reverse passes: rebuilding the states inside a pass with adjoint gates
    (the default for unitary gates) and recomputing them from the pass input give the
    same f, gradient and HVP, both within 1e-12 of the oracle (L <= 10); ragged chunks."""
    vlist, perms, tvlist, tperms = brickwall_instance(L, depth, 40 + L, 3, 41 + L)
    vdirs = _dirs(vlist, 42 + L)
    tgt = gpu.Target(brickwall=(tvlist, tperms))
    gpu.set_column_chunk(chunk)
    try:
        res = {}
        for on in (True, False):
            gpu.set_reconstruct(on)
            res[on] = (gpu.brickwall_unitary_target_projected_hessian_vector_product(tgt, vlist, vdirs, perms, L),
                       gpu.brickwall_unitary_target_and_projected_gradient(tgt, vlist, perms, L))
    finally:
        gpu.set_reconstruct(True)
    (f1, g1, h1), (fg1, gg1) = res[True]
    (f0, g0, h0), (fg0, gg0) = res[False]
    assert abs(f1 - f0) <= 1e-13 * abs(f0)
    assert rel_err(g1, g0) <= 1e-13 and rel_err(h1, h0) <= 1e-13
    assert abs(fg1 - fg0) <= 1e-13 * abs(fg0) and rel_err(gg1, gg0) <= 1e-13
    if L <= 10:
        fo, go, ho = oracle.brickwall_unitary_target_projected_hessian_vector_product(
            oracle.target("brickwall", (tvlist, tperms)), vlist, vdirs, perms, L)
        assert abs(f1 - fo) <= 1e-12 * abs(fo)
        assert rel_err(g1, go) <= 1e-12 and rel_err(h1, ho) <= 1e-12


@pytest.mark.parametrize("L,depth,chunk", [(8, 5, 0), (10, 7, 40), (12, 3, 0)])
def test_complex64_fp32_pipe_matches_tf32_mma(gpu, oracle, L, depth, chunk):
    """complex64 fused passes on the FP32 pipe (four threads per amplitude group) and on
    the TF32 MMA (three-term split): f, gradient and HVP (and f / gradient evaluations)
    agree with each other and with the oracle within the complex64 bar 1e-5; ragged chunks."""
    vlist, perms, tvlist, tperms = brickwall_instance(L, depth, 50 + L, 3, 51 + L)
    vdirs = _dirs(vlist, 52 + L)
    tgt = gpu.Target(brickwall=(tvlist, tperms))
    gpu.set_precision(gpu.PRECISION_C64)
    gpu.set_column_chunk(chunk)
    try:
        res = {}
        for on in (True, False):
            gpu.set_c64_fp32_pipe(on)
            res[on] = (gpu.brickwall_unitary_target_projected_hessian_vector_product(tgt, vlist, vdirs, perms, L),
                       gpu.brickwall_unitary_target_and_projected_gradient(tgt, vlist, perms, L),
                       gpu.brickwall_unitary_target(tgt, vlist, perms, L))
            assert gpu.last_config()["c64_fp32_pipe"] == on
    finally:
        gpu.set_autotune(True)
    fo, go, ho = oracle.brickwall_unitary_target_projected_hessian_vector_product(
        oracle.target("brickwall", (tvlist, tperms)), vlist, vdirs, perms, L)
    for on in (True, False):
        (f, g, h), (fg, gg), ff = res[on]
        assert abs(f - fo) <= 1e-5 * abs(fo) and abs(fg - fo) <= 1e-5 * abs(fo) and abs(ff - fo) <= 1e-5 * abs(fo)
        assert rel_err(g, go) <= 1e-5 and rel_err(h, ho) <= 1e-5 and rel_err(gg, go) <= 1e-5


@pytest.mark.parametrize("L", [12, 16, 21])
def test_single_state_tile_kernels_agree(gpu, oracle, L):
    """apply_quantum_circuit with several gates per HBM round trip (TMA bulk tiles) and
    with one kernel per gate give the same state (complex128 1e-13 relative; the oracle
    at L <= 16), with 2-4 gates per pass and wires on the lowest and highest qubits."""
    rng = np.random.default_rng(30 + L)
    G = 23
    psi = crandn(1 << L, rng)
    gates = np.stack([haar_unitary(rng) for _ in range(G)])
    wires = np.array([rng.choice(L, 2, replace=False) for _ in range(G)], np.int32)
    wires[0] = (L - 1, 0)
    wires[1] = (L - 2, L - 1)
    try:
        gpu.set_gates_per_pass(1)
        ref = gpu.apply_quantum_circuit(gates, wires, psi)
        for gpp in (2, 3, 4):
            gpu.set_gates_per_pass(gpp)
            assert rel_err(gpu.apply_quantum_circuit(gates, wires, psi), ref) <= 1e-13, gpp
    finally:
        gpu.set_autotune(True)
    if L <= 16:
        assert rel_err(ref, oracle.apply_quantum_circuit(gates, wires, psi)) <= 1e-12


def test_forward_adjoint_round_trip(gpu):
    """Forward through 64 random Haar gates on random distinct pairs, then the adjoint
    gates in reverse order, recovers the input state (L = 20, complex128)."""
    L, G = 20, 64
    rng = np.random.default_rng(20)
    psi = crandn(1 << L, rng)
    psi /= np.linalg.norm(psi)
    gates = np.stack([haar_unitary(rng) for _ in range(G)])
    wires = np.array([rng.choice(L, 2, replace=False) for _ in range(G)], np.int32)
    out = gpu.apply_quantum_circuit(gates, wires, psi)
    back = gpu.apply_quantum_circuit(np.conj(np.transpose(gates[::-1], (0, 2, 1))), wires[::-1], out)
    assert np.max(np.abs(back - psi)) <= 1e-12
    assert abs(np.linalg.norm(out) - 1) <= 1e-12


@pytest.mark.parametrize("L,depth", [(4, 3), (6, 5), (9, 4), (12, 5)])
@pytest.mark.parametrize("per_pass", [2, 3, 4])
def test_fused_passes_match_per_gate_engine(gpu, L, depth, per_pass):
    """Fused passes of 2-4 gates against one kernel per gate: f, gradient and HVP
    to 1e-12 for brickwalls of even and odd size (odd L: general circuit)."""
    rng = np.random.default_rng(1000 + L)
    if L % 2 == 0:
        vlist, perms, tvlist, tperms = brickwall_instance(L, depth, 40 + L, 3, 50 + L)
        vdirs = _dirs(vlist, 60 + L)
        t = gpu.Target(brickwall=(tvlist, tperms))
        run = lambda: gpu.brickwall_unitary_target_projected_hessian_vector_product(t, vlist, vdirs, perms, L)
    else:
        G = 3 * depth
        gates = np.stack([haar_unitary(rng) for _ in range(G)])
        wires = np.array([rng.choice(L, 2, replace=False) for _ in range(G)], np.int32)
        dirs = 0.3 * crandn((G, 4, 4), rng)
        tg = np.stack([haar_unitary(rng) for _ in range(6)])
        tw = np.array([rng.choice(L, 2, replace=False) for _ in range(6)], np.int32)
        t = gpu.Target(circuit=(tg, tw))
        run = lambda: gpu.circuit_unitary_target_hessian_vector_product(t, gates, dirs, wires, L)
    gpu.set_gates_per_pass(1)
    ref = run()
    gpu.set_gates_per_pass(per_pass)
    got = run()
    gpu.set_gates_per_pass(4)
    for a, b in zip(got, ref):
        assert rel_err(a, b) <= 1e-12


@pytest.mark.parametrize("mode", ["f", "grad"])
def test_fused_f_and_gradient_modes(gpu, oracle, mode):
    L = 8
    vlist, perms, tvlist, tperms = brickwall_instance(L, 5, 70, 3, 71)
    t = gpu.Target(brickwall=(tvlist, tperms))
    to = oracle.target("brickwall", (tvlist, tperms))
    if mode == "f":
        a, b = gpu.brickwall_unitary_target(t, vlist, perms, L), oracle.brickwall_unitary_target(to, vlist, perms, L)
        assert abs(a - b) <= 1e-12 * abs(b)
    else:
        fa, ga = gpu.brickwall_unitary_target_and_gradient(t, vlist, perms, L)
        fb, gb = oracle.brickwall_unitary_target_and_gradient(to, vlist, perms, L)
        assert abs(fa - fb) <= 1e-12 * abs(fb)
        assert rel_err(ga, gb) <= 1e-12


@pytest.mark.parametrize("per_pass", [1, 2, 4])
def test_single_state_fused_passes(gpu, oracle, per_pass):
    """apply_quantum_circuit on one L=14 state with 1-4 gates per round trip (random
    pairs, adjacent and wrapped, either order) against the oracle to 1e-12."""
    L, G = 14, 23
    rng = np.random.default_rng(77)
    psi = crandn(1 << L, rng)
    gates = np.stack([haar_unitary(rng) for _ in range(G)])
    wires = np.array([rng.choice(L, 2, replace=False) for _ in range(G)], np.int32)
    wires[0] = (L - 1, L - 2)
    wires[1] = (0, L - 1)
    gpu.set_gates_per_pass(per_pass)
    out = gpu.apply_quantum_circuit(gates, wires, psi)
    gpu.set_gates_per_pass(4)
    ref = oracle.apply_quantum_circuit(gates, wires, psi)
    assert rel_err(out, ref) <= 1e-12


@pytest.mark.parametrize("gpp", [1, 4])
def test_complex64_circuit_matches_complex128(gpu, gpp):
    """rqcopt_apply_quantum_circuit_c64 against apply_quantum_circuit (complex128) on
    random pairs, per-gate and fused passes; the adjoint circuit recovers the input."""
    import ctypes
    import torch
    from rqcopt_hpc_b200.abi import Statevector
    L, G = 12, 24
    rng = np.random.default_rng(77)
    gates = np.stack([haar_unitary(rng) for _ in range(G)])
    wires = np.array([rng.choice(L, 2, replace=False) for _ in range(G)], np.int32)
    adj = np.ascontiguousarray(np.conj(np.transpose(gates[::-1], (0, 2, 1))))
    wrev = np.ascontiguousarray(wires[::-1])
    psi = crandn(1 << L, rng)
    psi /= np.linalg.norm(psi)
    gpu.set_gates_per_pass(gpp)
    try:
        ref = np.empty_like(psi)
        assert gpu.lib().apply_quantum_circuit(gates.ctypes.data, G, wires.ctypes.data,
                                               ctypes.byref(Statevector(psi.ctypes.data, L)),
                                               ctypes.byref(Statevector(ref.ctypes.data, L))) == 0
        x = torch.from_numpy(psi.astype(np.complex64)).cuda()
        y, z = torch.empty_like(x), torch.empty_like(x)
        assert gpu.lib().rqcopt_apply_quantum_circuit_c64(gates.ctypes.data, G, wires.ctypes.data, x.data_ptr(),
                                                          y.data_ptr(), L) == 0
        assert gpu.lib().rqcopt_apply_quantum_circuit_c64(adj.ctypes.data, G, wrev.ctypes.data, y.data_ptr(),
                                                          z.data_ptr(), L) == 0
        assert np.max(np.abs(y.cpu().numpy() - ref)) <= 1e-5 * np.max(np.abs(ref))
        assert np.max(np.abs(z.cpu().numpy() - psi)) <= 1e-5 * np.max(np.abs(psi))
        # host pointers are rejected
        assert gpu.lib().rqcopt_apply_quantum_circuit_c64(gates.ctypes.data, G, wires.ctypes.data, psi.ctypes.data,
                                                          ref.ctypes.data, L) == -6
    finally:
        gpu.set_gates_per_pass(4)


@pytest.mark.parametrize("L,depth,per_pass", [(6, 3, 4), (9, 4, 3), (12, 5, 4), (12, 5, 2)])
@pytest.mark.parametrize("unitary", [True, False])
def test_complex64_reverse_paths_match_complex128(gpu, L, depth, per_pass, unitary):
    """complex64 passes against complex128 (1e-5): unitary gates take the reverse pass
    that rebuilds states with adjoint gates, perturbed (non-unitary) gates the one that
    recomputes them; gradient and HVP modes of a general circuit."""
    rng = np.random.default_rng(2000 + L + 10 * per_pass)
    G = 3 * depth
    gates = np.stack([haar_unitary(rng) for _ in range(G)])
    if not unitary:
        gates = gates + 0.05 * crandn((G, 4, 4), rng)
    wires = np.array([rng.choice(L, 2, replace=False) for _ in range(G)], np.int32)
    dirs = 0.3 * crandn((G, 4, 4), rng)
    tg = np.stack([haar_unitary(rng) for _ in range(6)])
    tw = np.array([rng.choice(L, 2, replace=False) for _ in range(6)], np.int32)
    t = gpu.Target(circuit=(tg, tw))
    gpu.set_gates_per_pass(per_pass)
    try:
        gpu.set_precision(gpu.PRECISION_C128)
        ref_h = gpu.circuit_unitary_target_hessian_vector_product(t, gates, dirs, wires, L)
        ref_g = gpu.circuit_unitary_target_and_gradient(t, gates, wires, L)
        gpu.set_precision(gpu.PRECISION_C64)
        got_h = gpu.circuit_unitary_target_hessian_vector_product(t, gates, dirs, wires, L)
        got_g = gpu.circuit_unitary_target_and_gradient(t, gates, wires, L)
    finally:
        gpu.set_precision(gpu.PRECISION_C128)
        gpu.set_gates_per_pass(4)
    for a, b in zip(got_h, ref_h):
        assert rel_err(a, b) <= 1e-5
    for a, b in zip(got_g, ref_g):
        assert rel_err(a, b) <= 1e-5


@pytest.mark.parametrize("L", [2, 3, 4, 5])
def test_smallest_registers_match_oracle(gpu, oracle, L):
    """The smallest registers, on both sides of the engine switch (one kernel per gate
    below 4 qubits, fused passes from 4): apply_quantum_circuit and the circuit target's
    f, gradient and HVP against the oracle to 1e-12 (complex128) and 1e-5 (complex64
    passes), dense target through the host callback."""
    rng = np.random.default_rng(700 + L)
    G = 7
    gates = np.stack([haar_unitary(rng) for _ in range(G)])
    wires = np.array([rng.choice(L, 2, replace=False) for _ in range(G)], np.int32)
    dirs = 0.5 * crandn((G, 4, 4), rng)
    u = crandn((1 << L, 1 << L), rng)
    psi = crandn(1 << L, rng)
    psi /= np.linalg.norm(psi)
    assert np.max(np.abs(gpu.apply_quantum_circuit(gates, wires, psi) -
                         oracle.apply_quantum_circuit(gates, wires, psi))) <= 1e-12
    fo = oracle.circuit_unitary_target_hessian_vector_product(oracle.target("dense", u), gates, dirs, wires, L)
    try:
        for prec, tol in ((gpu.PRECISION_C128, 1e-12), (gpu.PRECISION_C64, 1e-5)):
            gpu.set_precision(prec)
            fg = gpu.circuit_unitary_target_hessian_vector_product(gpu.Target(fn=lambda x: u @ x), gates, dirs, wires, L)
            assert abs(fg[0] - fo[0]) <= tol * abs(fo[0])
            assert rel_err(fg[1], fo[1]) <= tol
            assert rel_err(fg[2], fo[2]) <= tol
    finally:
        gpu.set_precision(gpu.PRECISION_C128)
