"""The host random-number API (src/pcg_basic.h, src/rng.h) and normalize_statevector
(src/statevector.h:23) of both libraries against the reference's own build in
oracle/_ref: the same seeds give bit-identical streams (PCG32 words, bounded draws,
Floyd samples, uniforms, Box-Muller normals through the same host libm), and
normalisation agrees to 1e-15.  These functions run on the host: no GPU needed."""
import ctypes as C
import os

import numpy as np
import pytest

from rqcopt_hpc_b200.abi import Pcg32, RngState

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBS = {
    "complex": (os.path.join(ROOT, "rqcopt_hpc_b200", "librqcopt_gpu.so"), os.path.join(ROOT, "oracle", "_ref", "librqcopt_ref.so")),
    "real": (os.path.join(ROOT, "rqcopt_hpc_b200", "librqcopt_gpu_real.so"),
             os.path.join(ROOT, "oracle", "_ref", "librqcopt_ref_real.so")),
}


class Pcg32x2(C.Structure):
    _fields_ = [("gen", Pcg32 * 2)]


class _CF(C.Structure):
    _fields_ = [("re", C.c_float), ("im", C.c_float)]


class _CD(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


def _load(path):
    lib = C.CDLL(path)
    sigs = {
        "pcg32_srandom_r": (None, [C.c_uint64, C.c_uint64, C.POINTER(Pcg32)]),
        "pcg32_random_r": (C.c_uint32, [C.POINTER(Pcg32)]),
        "pcg32_boundedrand_r": (C.c_uint32, [C.c_uint32, C.POINTER(Pcg32)]),
        "pcg32x2_srandom_r": (None, [C.c_uint64] * 4 + [C.POINTER(Pcg32x2)]),
        "pcg32x2_random_r": (C.c_uint64, [C.POINTER(Pcg32x2)]),
        "pcg32x2_boundedrand_r": (C.c_uint64, [C.c_uint64, C.POINTER(Pcg32x2)]),
        "seed_rng_state": (None, [C.c_uint64, C.POINTER(RngState)]),
        "rand_uint32": (C.c_uint32, [C.POINTER(RngState)]),
        "rand_uint64": (C.c_uint64, [C.POINTER(RngState)]),
        "rand_interval": (C.c_uint64, [C.c_uint64, C.POINTER(RngState)]),
        "rand_choice": (None, [C.c_uint64, C.c_uint64, C.POINTER(RngState), C.c_void_p]),
        "randu": (C.c_double, [C.POINTER(RngState)]),
        "randuf": (C.c_float, [C.POINTER(RngState)]),
        "randn": (C.c_double, [C.POINTER(RngState)]),
        "randnf": (C.c_float, [C.POINTER(RngState)]),
        "normalize_statevector": (None, [C.c_void_p]),
    }
    for name, (res, args) in sigs.items():
        f = getattr(lib, name)
        f.restype, f.argtypes = res, args
    return lib


@pytest.fixture(params=["complex", "real"])
def pair(request):
    ours, ref = LIBS[request.param]
    if not os.path.exists(ref):
        pytest.skip("reference build not present")
    return request.param, _load(ours), _load(ref)


def _draws(lib, fn, n, seed, *args):
    rng = RngState()
    lib.seed_rng_state(seed, C.byref(rng))
    return [getattr(lib, fn)(*args, C.byref(rng)) for _ in range(n)], rng.tuple()


@pytest.mark.parametrize("fn,args", [("rand_uint32", ()), ("rand_uint64", ()), ("rand_interval", (1000003,)),
                                     ("rand_interval", (7,)), ("randu", ()), ("randuf", ()), ("randn", ()),
                                     ("randnf", ())])
def test_rng_state_streams_match_reference(pair, fn, args):
    _, ours, ref = pair
    for seed in (0, 42, 2 ** 63 + 5):
        a, sa = _draws(ours, fn, 500, seed, *args)
        b, sb = _draws(ref, fn, 500, seed, *args)
        assert a == b and sa == sb


def test_pcg32_generators_match_reference(pair):
    _, ours, ref = pair
    for lib_a, lib_b in [(ours, ref)]:
        ga, gb = Pcg32(), Pcg32()
        lib_a.pcg32_srandom_r(42, 54, C.byref(ga))
        lib_b.pcg32_srandom_r(42, 54, C.byref(gb))
        assert [lib_a.pcg32_random_r(C.byref(ga)) for _ in range(300)] == [lib_b.pcg32_random_r(C.byref(gb)) for _ in range(300)]
        assert [lib_a.pcg32_boundedrand_r(97, C.byref(ga)) for _ in range(300)] == \
            [lib_b.pcg32_boundedrand_r(97, C.byref(gb)) for _ in range(300)]
        pa, pb = Pcg32x2(), Pcg32x2()
        lib_a.pcg32x2_srandom_r(1, 2, 3, 3, C.byref(pa))   # equal streams are made distinct
        lib_b.pcg32x2_srandom_r(1, 2, 3, 3, C.byref(pb))
        assert [lib_a.pcg32x2_random_r(C.byref(pa)) for _ in range(300)] == \
            [lib_b.pcg32x2_random_r(C.byref(pb)) for _ in range(300)]
        assert [lib_a.pcg32x2_boundedrand_r(2 ** 40 + 3, C.byref(pa)) for _ in range(300)] == \
            [lib_b.pcg32x2_boundedrand_r(2 ** 40 + 3, C.byref(pb)) for _ in range(300)]


def test_rand_choice_matches_reference(pair):
    _, ours, ref = pair
    for bound, k in [(10, 10), (1000, 17), (5, 0)]:
        out = []
        for lib in (ours, ref):
            rng = RngState()
            lib.seed_rng_state(7, C.byref(rng))
            ret = np.zeros(max(k, 1), np.uint64)
            lib.rand_choice(bound, k, C.byref(rng), ret.ctypes.data)
            out.append(ret[:k].copy())
        assert np.array_equal(out[0], out[1])
        assert len(set(out[0].tolist())) == k and (k == 0 or out[0].max() < bound)


def test_complex_normals_match_reference():
    ours, ref = LIBS["complex"]
    if not os.path.exists(ref):
        pytest.skip("reference build not present")
    a, b = C.CDLL(ours), C.CDLL(ref)
    for lib in (a, b):
        lib.crandn.restype, lib.crandn.argtypes = _CD, [C.POINTER(RngState)]
        lib.crandnf.restype, lib.crandnf.argtypes = _CF, [C.POINTER(RngState)]
        lib.seed_rng_state.argtypes = [C.c_uint64, C.POINTER(RngState)]
    for fn in ("crandn", "crandnf"):
        vals = []
        for lib in (a, b):
            rng = RngState()
            lib.seed_rng_state(11, C.byref(rng))
            vals.append([(z.re, z.im) for z in (getattr(lib, fn)(C.byref(rng)) for _ in range(300))])
        assert vals[0] == vals[1]


def _normalize(lib, y, L):
    buf = C.create_string_buffer(16)   # struct statevector {numeric* data; int nqubits;}
    C.memmove(buf, C.byref(C.c_void_p(y.ctypes.data)), 8)
    C.memmove(C.addressof(buf) + 8, C.byref(C.c_int(L)), 4)
    lib.normalize_statevector(C.addressof(buf))


def test_normalize_statevector_matches_reference(pair):
    """Against the reference at ordinary magnitudes; the library's scaled 2-norm also
    normalises amplitudes of 1e-200 and 1e200 (where the loop BLAS the reference is
    built with here underflows or overflows), and leaves a zero state unchanged."""
    kind, ours, ref = pair
    rng = np.random.default_rng(5)

    def state(L, scale):
        x = rng.standard_normal(1 << L) + (1j * rng.standard_normal(1 << L) if kind == "complex" else 0)
        return np.ascontiguousarray(x * scale)

    for L in (0, 3, 10):
        x = state(L, 3.0)
        a, b = x.copy(), x.copy()
        _normalize(ours, a, L)
        _normalize(ref, b, L)
        assert np.max(np.abs(a - b)) <= 1e-15
        for scale in (1e-200, 1e200):
            y = state(L, scale)
            _normalize(ours, y, L)
            assert abs(np.linalg.norm(y) - 1) <= 1e-14
    zero = np.zeros(8, np.complex128 if kind == "complex" else np.float64)
    _normalize(ours, zero, 3)
    assert not np.any(zero)
