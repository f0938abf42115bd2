"""The autotuner of the basis-column sums (rqcopt_gpu_set_autotune): it picks gates
per pass, column chunk and the complex128 reverse variant by timing candidates on a
column sample, so every candidate must give the same f, projected gradient and
projected HVP (to 1e-12 relative in complex128; within the 1e-5 bar of complex64
passes, whose rounding depends on how gates are grouped into passes), and settings
the caller fixes must be kept."""
import itertools

import numpy as np
import pytest

from helpers import brickwall_instance, random_tangent_dirs, real_to_antisymm, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _fresh(gpu):
    gpu.set_autotune(True)
    gpu.set_precision(gpu.PRECISION_C128)
    yield
    gpu.set_autotune(True)
    gpu.set_precision(gpu.PRECISION_C128)


def _case(L=12, depth=5, tdepth=3, seed=60):
    vlist, perms, tvlist, tperms = brickwall_instance(L, depth, seed, tdepth, seed + 1)
    r = random_tangent_dirs(vlist, seed + 2)
    vdirs = np.stack([vlist[k] @ real_to_antisymm(r[k]) for k in range(depth)])
    return L, vlist, perms, tvlist, tperms, vdirs


@pytest.mark.parametrize("precision,tol", [("C128", 1e-12), ("C64", 1e-5)])
def test_every_candidate_gives_the_tuned_result(gpu, oracle, precision, tol):
    L, vlist, perms, tvlist, tperms, vdirs = _case()
    prec = getattr(gpu, f"PRECISION_{precision}")
    gpu.set_precision(prec)
    tgt = gpu.Target(brickwall=(tvlist, tperms))
    tuned = gpu.brickwall_unitary_target_projected_hessian_vector_product(tgt, vlist, vdirs, perms, L)
    cfg = gpu.last_config()
    assert cfg["tuned"] and 1 <= cfg["gates_per_pass"] <= 4 and cfg["ms_per_column"] > 0
    # the same call again reuses the choice
    again = gpu.brickwall_unitary_target_projected_hessian_vector_product(tgt, vlist, vdirs, perms, L)
    assert gpu.last_config() == cfg
    assert abs(again[0] - tuned[0]) <= 1e-14 * abs(tuned[0])
    recon = (True, False) if precision == "C128" else (True,)
    for gpp, chunk, rc in itertools.product((1, 2, 3, 4), (4096, 2048, 512), recon):
        gpu.set_gates_per_pass(gpp)
        gpu.set_column_chunk(chunk)
        gpu.set_reconstruct(rc)
        gpu.set_c64_fp32_pipe(True)
        f, g, h = gpu.brickwall_unitary_target_projected_hessian_vector_product(tgt, vlist, vdirs, perms, L)
        used = gpu.last_config()
        assert not used["tuned"] and used["gates_per_pass"] == gpp and used["column_chunk"] == chunk
        # complex128: the same sums to rounding; complex64: within the single-precision bar
        assert abs(f - tuned[0]) <= tol * abs(tuned[0]), (gpp, chunk, rc)
        assert rel_err(g, tuned[1]) <= tol, (gpp, chunk, rc)
        assert rel_err(h, tuned[2]) <= tol, (gpp, chunk, rc)
    if precision == "C128":
        fo, go, ho = oracle.brickwall_unitary_target_projected_hessian_vector_product(
            oracle.target("brickwall", (tvlist, tperms)), vlist, vdirs, perms, L)
        assert abs(tuned[0] - fo) <= tol * abs(fo)
        assert rel_err(tuned[1], go) <= tol and rel_err(tuned[2], ho) <= tol


def test_fixed_settings_are_kept(gpu):
    L, vlist, perms, tvlist, tperms, vdirs = _case(L=12, depth=3, seed=70)
    tgt = gpu.Target(brickwall=(tvlist, tperms))
    gpu.set_gates_per_pass(2)
    gpu.brickwall_unitary_target_and_projected_gradient(tgt, vlist, perms, L)
    assert gpu.last_config()["gates_per_pass"] == 2
    gpu.set_autotune(False)
    gpu.brickwall_unitary_target_and_projected_gradient(tgt, vlist, perms, L)
    cfg = gpu.last_config()
    assert not cfg["tuned"] and cfg["gates_per_pass"] == 2


def test_small_problems_run_the_defaults(gpu):
    L, vlist, perms, tvlist, tperms, vdirs = _case(L=6, depth=3, seed=80)
    tgt = gpu.Target(brickwall=(tvlist, tperms))
    gpu.brickwall_unitary_target_projected_hessian_vector_product(tgt, vlist, vdirs, perms, L)
    cfg = gpu.last_config()
    assert not cfg["tuned"] and cfg["gates_per_pass"] == 4
