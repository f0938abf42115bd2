"""Shared test data: golden fixtures, seeded generators and finite differences."""
from __future__ import annotations

import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name: str) -> dict:
    """Fixture arrays; interleaved (..., 2) float arrays become complex."""
    out = {}
    with np.load(os.path.join(GOLDEN, f"{name}.npz")) as z:
        for k in z.files:
            a = z[k]
            if a.dtype == np.float64 and a.ndim >= 1 and a.shape[-1] == 2:
                a = a[..., 0] + 1j * a[..., 1]
            out[k] = a
    return out


def stack(d: dict, prefix: str, n: int) -> np.ndarray:
    return np.stack([d[f"{prefix}{i}"] for i in range(n)])


def haar_unitary(rng, n=4) -> np.ndarray:
    """Haar-random unitary: QR of an iid complex Gaussian matrix with the diagonal phase fix."""
    z = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / np.sqrt(2)
    q, r = np.linalg.qr(z)
    d = np.diagonal(r)
    return q * (d / np.abs(d))


def crandn(shape, rng) -> np.ndarray:
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) / np.sqrt(2)


def periodic_perms(L: int, nlayers: int) -> np.ndarray:
    """Brickwall layers alternating pairs (0,1),(2,3),... and (1,2),...,(L-1,0)."""
    even = np.arange(L)
    odd = np.roll(np.arange(L), -1)
    return np.stack([even if l % 2 == 0 else odd for l in range(nlayers)]).astype(np.int32)


def brickwall_instance(L: int, depth: int, seed: int, target_depth: int, target_seed: int):
    rng = np.random.default_rng(seed)
    vlist = np.stack([haar_unitary(rng) for _ in range(depth)])
    trng = np.random.default_rng(target_seed)
    tvlist = np.stack([haar_unitary(trng) for _ in range(target_depth)])
    return vlist, periodic_perms(L, depth), tvlist, periodic_perms(L, target_depth)


def random_tangent_dirs(vlist, seed):
    """HVP direction: 16 iid N(0,1) reals per gate mapped to the tangent space (Z = V A(r))."""
    rng = np.random.default_rng(seed)
    r = rng.standard_normal((vlist.shape[0], 16))
    return r


def real_to_antisymm(r):
    w = np.zeros((4, 4), np.complex128)
    for a in range(4):
        w[a, a] = 1j * r[5 * a]
        for c in range(a + 1, 4):
            p, q = r[4 * a + c], r[4 * c + a]
            w[a, c] = 0.5 * (p - q) + 0.5j * (p + q)
            w[c, a] = -np.conj(w[a, c])
    return w


def udist(a, b) -> float:
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b)))) if np.size(a) else 0.0


def rel_err(a, b) -> float:
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def num_grad_backward(f, x, dy, h=1e-5):
    """Backward numerical gradient of a complex map (test/numerical_gradient.c:9-47):
    grad_k = sum_j dy_j (f(x + h e_k) - f(x - h e_k))_j / (2 h); h may be complex."""
    x = np.asarray(x, np.complex128)
    g = np.zeros(x.size, np.complex128)
    dy = np.asarray(dy).ravel()
    for k in range(x.size):
        e = np.zeros(x.size, np.complex128)
        e[k] = h
        fp = np.asarray(f((x.ravel() + e).reshape(x.shape))).ravel()
        fm = np.asarray(f((x.ravel() - e).reshape(x.shape))).ravel()
        g[k] = np.sum(dy * (fp - fm)) / (2 * h)
    return g.reshape(x.shape)


def num_grad_wirtinger(f, x, dy=None, h=1e-5):
    """Wirtinger-convention backward gradient (test/numerical_gradient.c:91-103)."""
    dy = np.ones(1) if dy is None else dy
    ff = lambda y: np.atleast_1d(f(y))
    return 0.5 * (num_grad_backward(ff, x, dy, h) + num_grad_backward(ff, x, dy, 1j * h))


def num_grad_forward(f, x, direction, h=1e-5):
    """Forward numerical derivative (f(x + h d) - f(x - h d)) / (2 h) (test/numerical_gradient.c:54-82)."""
    x = np.asarray(x, np.complex128)
    return (np.asarray(f(x + h * direction)) - np.asarray(f(x - h * direction))) / (2 * h)


def fixture_ufunc_np(x: np.ndarray) -> np.ndarray:
    """The synthetic sparse target map of the reference tests (test/test_target.c:16-34)."""
    n = x.shape[0]
    i = np.arange(n)
    return ((-1.1 + 0.8j) * x[((i + 3) * 113) % n] + (0.4 - 0.7j) * x[((i + 9) * 173) % n]
            + (0.5 + 0.1j) * x[i] + (-0.3 + 0.2j) * x[((i + 4) * 199) % n])
