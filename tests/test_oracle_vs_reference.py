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


def test_trust_region_iterates_match_reference(oracle, ref):
    vlist, perms, tvlist, tperms, _ = _c1()
    t = oracle.target("brickwall", (tvlist, tperms))
    f_o, v_o, acc, bnd = oracle.optimize_brickwall_circuit_hvp(t, vlist, perms, 8, 10)
    f_r, v_r = ref.optimize_brickwall(vlist, perms, 8, tvlist, tperms, 10)
    assert rel_err(f_o, f_r) <= 1e-12
    assert rel_err(v_o, v_r) <= 1e-10
    assert f_o[-1] < f_o[0]
