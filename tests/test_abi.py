"""The C ABI: the library loads without a GPU, exports every function that
include/rqcopt_gpu.h declares, and the header compiles as C and C++.  Where the
reference sources are present, each reference declaration the header restates
is compared with it token by token (ignoring `restrict` and whitespace)."""
import os
import re
import subprocess
import ctypes

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "rqcopt_gpu.h")
LIB = os.path.join(ROOT, "rqcopt_hpc_b200", "librqcopt_gpu.so")
REAL_HEADER = os.path.join(ROOT, "include", "rqcopt_gpu_real.h")
REAL_LIB = os.path.join(ROOT, "rqcopt_hpc_b200", "librqcopt_gpu_real.so")
REF_SRC = "/root/reference/src"


def _declared_functions(text):
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"static inline[^{]*\{.*?\n\}", "", text, flags=re.S)
    names = set()
    for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b([a-z_][a-z0-9_]*)\s*\(", text, flags=re.M):
        name = m.group(1)
        if name not in ("if", "for", "while", "return", "sizeof") and not m.group(0).lstrip().startswith("typedef"):
            names.add(name)
    return names


@pytest.mark.parametrize("lib_path,header", [(LIB, HEADER), (REAL_LIB, REAL_HEADER)], ids=["complex", "real"])
def test_library_exports_every_declared_function(lib_path, header):
    assert os.path.exists(lib_path), "build the library first (python -m rqcopt_hpc_b200.build)"
    lib = ctypes.CDLL(lib_path)
    names = _declared_functions(open(header).read())
    assert len(names) > 60
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_real_library_exports_only_its_interface():
    """The real-build library hides its internals (C++ runtime instantiations included)."""
    out = subprocess.run(["nm", "-D", "--defined-only", REAL_LIB], capture_output=True, text=True, check=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    assert exported == _declared_functions(open(REAL_HEADER).read())


@pytest.mark.parametrize("lang", ["c", "c++"])
@pytest.mark.parametrize("header", ["rqcopt_gpu.h", "rqcopt_gpu_real.h"])
def test_header_compiles(tmp_path, lang, header):
    src = tmp_path / ("t.c" if lang == "c" else "t.cpp")
    src.write_text(f'#include "{header}"\n' + 'int main(void) { struct rtr_params p; set_rtr_default_params(16, &p); return p.tcg_params.maxiter == 32 ? 0 : 1; }\n')
    cc = "gcc" if lang == "c" else "g++"
    subprocess.run([cc, "-fsyntax-only", "-Wall", "-I" + os.path.dirname(HEADER), str(src)], check=True)


def _complex_branch(text, complex_build=True):
    """Keep one branch of `#ifdef COMPLEX_CIRCUIT ... [#else ...] #endif` blocks: the
    COMPLEX_CIRCUIT one (librqcopt_gpu.so) or the other (librqcopt_gpu_real.so); the
    reference does not nest them."""
    out, state = [], None
    for line in text.split("\n"):
        d = line.strip()
        if d.startswith("#ifdef COMPLEX_CIRCUIT"):
            state = "first"
        elif state and d.startswith("#else"):
            state = "second"
        elif state and d.startswith("#endif"):
            state = None
        elif state is None or (state == "first") == complex_build:
            out.append(line)
    return "\n".join(out)


def _ref_prototypes(complex_build=True):
    protos = {}
    for fn in os.listdir(REF_SRC):
        if fn.endswith(".h"):
            text = open(os.path.join(REF_SRC, fn)).read()
            text = re.sub(r"//.*", "", text)
            text = _complex_branch(text, complex_build)
            for m in re.finditer(r"^([A-Za-z_][\w\s\*]*?\b([a-z_][a-z0-9_]*)\s*\([^;{]*\))\s*;", text, flags=re.M):
                if not m.group(1).startswith("typedef"):
                    protos[m.group(2)] = m.group(1)
    return protos


def _norm(p):
    p = p.replace("restrict", " ")
    p = re.sub(r"\bconst\s+hessian_vector_product_func", "hessian_vector_product_func", p)
    p = re.sub(r"\bconst\s+(target_func|target_gradient_func)", r"\1", p)
    p = re.sub(r"\s+", " ", p).strip()
    p = re.sub(r"\s*([\(\)\*,\[\]])\s*", r"\1", p)
    return p


@pytest.mark.skipif(not os.path.isdir(REF_SRC), reason="reference sources not present")
@pytest.mark.parametrize("header,complex_build", [(HEADER, True), (REAL_HEADER, False)], ids=["complex", "real"])
def test_signatures_match_reference(header, complex_build):
    ref = _ref_prototypes(complex_build)
    text = re.sub(r"/\*.*?\*/", "", open(header).read(), flags=re.S)
    ours = {}
    for m in re.finditer(r"^([A-Za-z_][\w\s\*]*?\b([a-z_][a-z0-9_]*)\s*\([^;{]*\))\s*;", text, flags=re.M):
        if not m.group(1).startswith("typedef"):
            ours[m.group(2)] = m.group(1)
    checked = 0
    for name, proto in ours.items():
        if name in ref:
            assert _norm(proto) == _norm(ref[name]), (name, proto, ref[name])
            checked += 1
    assert checked >= 50
    if not complex_build:
        # the real build has none of the full-Hessian matrix forms
        assert not {n for n in ours if "hessian_matrix" in n or "hmat_sampling" in n or n.endswith("_hmat")} - {"truncated_cg_hmat", "riemannian_trust_region_optimize_hmat"}


def test_invalid_arguments_refused_before_device_work():
    """The full-Hessian, sampling and block-encoding entry points refuse invalid sizes
    and permutations with the argument error (-6) before touching the device (no GPU needed)."""
    import numpy as np
    from rqcopt_hpc_b200 import gpu
    from helpers import brickwall_instance
    vlist, perms, tv, tp = brickwall_instance(6, 3, 1, 2, 2)
    t = gpu.Target(brickwall=(tv, tp))
    bad_perms = np.zeros((3, 6), np.int32)
    calls = [lambda: gpu.brickwall_unitary_target_gradient_hessian(t, vlist, perms, 5),
             lambda: gpu.brickwall_unitary_target_gradient_vector_hessian_matrix(t, vlist, bad_perms, 6),
             lambda: gpu.brickwall_unitary_target_gradient_hessian_sampling(t, vlist, perms, 7, 10,
                                                                            gpu.seed_rng_state(1)),
             lambda: gpu.brickwall_blockenc_target_and_gradient(t, vlist, perms, 5),
             lambda: gpu.brickwall_blockenc_target_gradient_vector_hessian_matrix(t, vlist, bad_perms, 6)]
    for call in calls:
        with pytest.raises(gpu.RqcError) as e:
            call()
        assert e.value.code == -6


def test_core_entry_points_refuse_invalid_circuits_before_device_work():
    """Where the reference asserts (src/quantum_circuit.c:15-16, src/gate.c:12-15),
    the library refuses with the argument error (-6) before touching the device: an
    empty circuit, equal or out-of-range wires, statevectors of different sizes (no GPU
    needed)."""
    import numpy as np
    from rqcopt_hpc_b200 import gpu
    from helpers import haar_unitary
    rng = np.random.default_rng(5)
    L = 4
    gates = np.stack([haar_unitary(rng) for _ in range(3)])
    psi = np.zeros(1 << L, np.complex128)
    psi[0] = 1
    tgt = gpu.Target(fn=lambda x: x)
    bad = [np.array([[0, 1], [2, 2], [1, 3]], np.int32),     # equal wires
           np.array([[0, 1], [2, 4], [1, 3]], np.int32),     # wire beyond the register
           np.array([[0, 1], [-1, 2], [1, 3]], np.int32)]    # negative wire
    calls = [lambda: gpu.apply_quantum_circuit(gates[:0], np.zeros((0, 2), np.int32), psi)]
    for w in bad:
        calls += [lambda w=w: gpu.apply_quantum_circuit(gates, w, psi),
                  lambda w=w: gpu.circuit_unitary_target_hessian_vector_product(tgt, gates, gates, w, L)]
    calls.append(lambda: gpu.apply_gate(gates[0], 1, 1, psi))
    for call in calls:
        with pytest.raises(gpu.RqcError) as e:
            call()
        assert e.value.code == -6
    # statevectors of different sizes
    from rqcopt_hpc_b200.abi import Statevector
    import ctypes
    out = np.zeros(1 << (L + 1), np.complex128)
    w = np.array([[0, 1]], np.int32)
    ret = gpu.lib().apply_quantum_circuit(gates.ctypes.data, 1, w.ctypes.data,
                                          ctypes.byref(Statevector(psi.ctypes.data, L)),
                                          ctypes.byref(Statevector(out.ctypes.data, L + 1)))
    assert ret == -6
