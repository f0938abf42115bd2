"""The oracle restatement against the reference's own C sources compiled in
oracle/_ref (CPU).  Inputs are the seeded L=8, depth-5 brickwall workload (gates
seed 0, depth-3 target seed 1, HVP direction seed 2)."""
import numpy as np
import pytest

from helpers import brickwall_instance, random_tangent_dirs, rel_err, real_to_antisymm

ref_mod = pytest.importorskip("oracle.oracle")
if not ref_mod.Reference.available():
    pytest.skip("reference build not present", allow_module_level=True)


@pytest.fixture(scope="module")
def ref():
    return ref_mod.Reference()


def _c1():
    vlist, perms, tvlist, tperms = brickwall_instance(8, 5, 0, 3, 1)
    r = random_tangent_dirs(vlist, 2)
    vdirs = np.stack([vlist[k] @ real_to_antisymm(r[k]) for k in range(vlist.shape[0])])
    return vlist, perms, tvlist, tperms, vdirs


def test_projected_hvp_matches_reference(oracle, ref):
    vlist, perms, tvlist, tperms, vdirs = _c1()
    t = oracle.target("brickwall", (tvlist, tperms))
    f, g, h = oracle.brickwall_unitary_target_projected_hessian_vector_product(t, vlist, vdirs, perms, 8)
    fr, gr, hr = ref.brickwall_projected_hvp(vlist, vdirs, perms, 8, tvlist, tperms)
    assert abs(f - fr) <= 1e-12 * abs(fr)
    assert rel_err(g, gr) <= 1e-12
    assert rel_err(h, hr) <= 1e-12


def test_column_range_matches_reference(oracle, ref):
    vlist, perms, tvlist, tperms = brickwall_instance(10, 5, 3, 3, 4)
    vdirs = np.stack([vlist[k] @ real_to_antisymm(np.random.default_rng(5).standard_normal(16)) for k in range(5)])
    t = oracle.target("brickwall", (tvlist, tperms))
    f, dv, hv = oracle.brickwall_unitary_target_hessian_vector_product(t, vlist, vdirs, perms, 10, 100, 116)
    fr, dg, hg = ref.brickwall_hvp_columns(vlist, vdirs, perms, 10, tvlist, tperms, 100, 116)
    dvr = dg.reshape(5, 5, 4, 4).sum(axis=1)
    hvr = hg.reshape(5, 5, 4, 4).sum(axis=1)
    assert abs(f - fr) <= 1e-12 * abs(fr)
    assert rel_err(dv, dvr) <= 1e-12
    assert rel_err(hv, hvr) <= 1e-12


def test_headline_size_column_sample_matches_reference(oracle, ref):
    """L=16, depth 9 against a depth-5 target (seeds 10 / 11 / 12): per-gate sums of two
    basis columns, the pin of the oracle at the headline size."""
    vlist, perms, tvlist, tperms = brickwall_instance(16, 9, 10, 5, 11)
    r = random_tangent_dirs(vlist, 12)
    vdirs = np.stack([vlist[k] @ real_to_antisymm(r[k]) for k in range(9)])
    gates, dirs = np.repeat(vlist, 8, axis=0), np.repeat(vdirs, 8, axis=0)
    wires = np.concatenate([perms[l].reshape(8, 2) for l in range(9)]).astype(np.int32)
    t = oracle.target("brickwall", (tvlist, tperms))
    f, dg, hg = oracle.circuit_unitary_target_hessian_vector_product(t, gates, dirs, wires, 16, 40000, 40002)
    fr, dgr, hgr = ref.brickwall_hvp_columns(vlist, vdirs, perms, 16, tvlist, tperms, 40000, 40002)
    assert abs(f - fr) <= 1e-12 * abs(fr)
    assert rel_err(dg, dgr) <= 1e-12
    assert rel_err(hg, hgr) <= 1e-12


def test_trust_region_iterates_match_reference(oracle, ref):
    vlist, perms, tvlist, tperms, _ = _c1()
    t = oracle.target("brickwall", (tvlist, tperms))
    f_o, v_o, acc, bnd = oracle.optimize_brickwall_circuit_hvp(t, vlist, perms, 8, 10)
    f_r, v_r = ref.optimize_brickwall(vlist, perms, 8, tvlist, tperms, 10)
    assert rel_err(f_o, f_r) <= 1e-12
    assert rel_err(v_o, v_r) <= 1e-10
    assert f_o[-1] < f_o[0]


def test_sampling_oracle_matches_reference(oracle, ref):
    """PCG32x2 seeding and Haar states bit for bit; sampled f, gradient and Hessian and a
    sampled full-Hessian optimisation to rounding; identical generator state after each call."""
    ro, rr = oracle.seed_rng_state(677), ref.seed_rng_state(677)
    assert ro.tuple() == rr.tuple()
    assert np.array_equal(oracle.haar_random_statevector(6, ro), ref.haar_random_statevector(6, rr))
    assert ro.tuple() == rr.tuple()
    vlist, perms, tvlist, tperms = brickwall_instance(6, 3, 0, 3, 1)
    t = oracle.target("brickwall", (tvlist, tperms))
    ro, rr = oracle.seed_rng_state(5), ref.seed_rng_state(5)
    fo = oracle.brickwall_unitary_target_sampling(t, vlist, perms, 6, 100, ro)
    fr = ref.sampling(0, vlist, perms, 6, (tvlist, tperms), 100, rr)
    assert abs(fo - fr) <= 1e-14 * abs(fr) and ro.tuple() == rr.tuple()
    ro, rr = oracle.seed_rng_state(6), ref.seed_rng_state(6)
    fo, go, Ho = oracle.brickwall_unitary_target_gradient_vector_hessian_matrix_sampling(t, vlist, perms, 6, 40, ro)
    fr, gr, Hr = ref.sampling(2, vlist, perms, 6, (tvlist, tperms), 40, rr)
    assert rel_err(go, gr) <= 1e-14 and rel_err(Ho, Hr) <= 1e-14 and ro.tuple() == rr.tuple()
    ro, rr = oracle.seed_rng_state(7), ref.seed_rng_state(7)
    fo, vo = oracle.optimize_brickwall_circuit_hmat_sampling(t, vlist, perms, 6, 30, ro, 3)
    fr, vr = ref.optimize_brickwall_hmat_sampling(vlist, perms, 6, tvlist, tperms, 30, rr, 3)
    assert rel_err(fo, fr) <= 1e-13 and rel_err(vo, vr) <= 1e-13 and ro.tuple() == rr.tuple()


def test_full_hessian_oracle_matches_reference(oracle, ref):
    vlist, perms, tvlist, tperms = brickwall_instance(8, 3, 0, 3, 1)
    t = oracle.target("brickwall", (tvlist, tperms))
    f, g, H = oracle.brickwall_unitary_target_gradient_vector_hessian_matrix(t, vlist, perms, 8)
    fr, gr, Hr = ref.gradient_vector_hessian_matrix(vlist, perms, 8, tvlist, tperms)
    assert abs(f - fr) <= 1e-14 * abs(fr) and rel_err(g, gr) <= 1e-14 and rel_err(H, Hr) <= 1e-14
    fo, vo, acc, bnd = oracle.optimize_brickwall_circuit_hmat(t, vlist, perms, 8, 3)
    fr2, vr2 = ref.optimize_brickwall_hmat(vlist, perms, 8, tvlist, tperms, 3)
    assert rel_err(fo, fr2) <= 1e-13 and rel_err(vo, vr2) <= 1e-13


def test_blockenc_oracle_matches_reference(oracle, ref):
    """Block-encoding target, H a depth-2 brickwall on 4 of the 8 qubits: f, gradients,
    both complex Hessians and the projected matrix."""
    from helpers import periodic_perms
    vlist, perms, _, _ = brickwall_instance(8, 3, 4, 1, 5)
    hv, _, _, _ = brickwall_instance(4, 2, 6, 1, 7)
    hp = periodic_perms(4, 2)
    t = oracle.target("brickwall", (hv, hp))
    f, dv, h1, h2 = oracle.brickwall_blockenc_target_gradient_hessian(t, vlist, perms, 8)
    fr, dvr, h1r, h2r = ref.blockenc(3, vlist, perms, 8, hv, hp)
    assert abs(f - fr) <= 1e-14 * abs(fr) and rel_err(dv, dvr) <= 1e-14
    assert rel_err(h1, h1r) <= 1e-14 and rel_err(h2, h2r) <= 1e-14
    f, g, H = oracle.brickwall_blockenc_target_gradient_vector_hessian_matrix(t, vlist, perms, 8)
    fr, gr, Hr = ref.blockenc(4, vlist, perms, 8, hv, hp)
    assert abs(f - fr) <= 1e-14 * abs(fr) and rel_err(g, gr) <= 1e-14 and rel_err(H, Hr) <= 1e-14
