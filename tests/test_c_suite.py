"""The reference's own C test programs (test/*.c and test/run_tests.c, unmodified),
compiled by `make -C oracle ref` with a shim that serves their HDF5 reads from the
.npz fixtures (oracle/shim/h5_npz.c), and linked four ways:

- run_tests_ref / run_tests_ref_real: against the reference sources themselves, the
  complex and the real-orthogonal build (checks the shim and the fixtures: every
  test must pass);
- run_tests_gpu / run_tests_gpu_real: against librqcopt_gpu.so / librqcopt_gpu_real.so
  instead, the drop-in as a reference user would link it.  On a GPU every test must
  pass.  Without one, the tests whose functions run on the host (the 4x4 manifold
  algebra) must pass, and the rest fail only for want of a device.
"""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")
HOST_SIDE = ["test_symm", "test_antisymm", "test_real_to_antisymm", "test_real_to_tangent", "test_project_tangent",
             "test_multiply", "test_inverse_matrix", "test_polar_factor"]


def _run(name):
    path = os.path.join(REF, name)
    if not os.path.exists(path):
        pytest.skip(f"{name} not built (make -C oracle ref)")
    env = dict(os.environ, RQC_GOLDEN=os.path.join(ROOT, "tests", "golden"))
    p = subprocess.run([path], cwd=ROOT, env=env, capture_output=True, text=True, timeout=1200)
    failed = re.findall(r"Test '(\w+)' failed: (.*)", p.stdout)
    m = re.search(r"Number of successful tests: (\d+) / (\d+)", p.stdout)
    assert m, p.stdout[-2000:] + p.stderr[-2000:]
    return p.returncode, int(m.group(1)), int(m.group(2)), dict(failed)


@pytest.mark.parametrize("name,total", [("run_tests_ref", 41), ("run_tests_ref_real", 36)])
def test_reference_suite_passes_on_the_reference_build(name, total):
    rc, ok, n, failed = _run(name)
    assert rc == 0 and ok == n == total, failed


@pytest.mark.parametrize("name", ["run_tests_gpu", "run_tests_gpu_real"])
def test_host_side_tests_pass_against_the_gpu_libraries(name):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: the full suite runs in test_reference_c_suite_on_the_gpu")
    rc, ok, n, failed = _run(name)
    assert n == (41 if name == "run_tests_gpu" else 36)
    bad = {t: msg for t, msg in failed.items() if t in HOST_SIDE}
    assert not bad, bad
    assert ok >= 8


@pytest.mark.gpu
@pytest.mark.parametrize("name,total", [("run_tests_gpu", 41), ("run_tests_gpu_real", 36)])
def test_reference_c_suite_on_the_gpu(gpu, name, total):
    rc, ok, n, failed = _run(name)
    assert rc == 0 and ok == n == total, failed
