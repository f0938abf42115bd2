"""Seeded synthetic brickwall workloads (Haar gates by QR of complex Gaussian 4x4
matrices with the diagonal-phase fix; periodic brickwall pairs: even layers
(0,1),(2,3),..., odd layers (1,2),...,(L-1,0))."""
from __future__ import annotations

import numpy as np


def haar(rng):
    z = (rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4))) / np.sqrt(2)
    q, r = np.linalg.qr(z)
    d = np.diagonal(r)
    return q * (d / np.abs(d))


def perms_for(L, nlayers):
    even, odd = np.arange(L), np.roll(np.arange(L), -1)
    return np.stack([even if l % 2 == 0 else odd for l in range(nlayers)]).astype(np.int32)


def brickwall_problem(L, depth, tdepth, seed, tseed):
    """(L, vlist, perms, target_vlist, target_perms): Haar layer gates from seed and an
    independent Haar brickwall target of depth tdepth from tseed."""
    rng = np.random.default_rng(seed)
    vlist = np.stack([haar(rng) for _ in range(depth)])
    trng = np.random.default_rng(tseed)
    tvlist = np.stack([haar(trng) for _ in range(tdepth)])
    return (L, vlist, perms_for(L, depth), tvlist, perms_for(L, tdepth))


def batched_instances(count=512, sizes=(6, 8, 10, 12), depths=(3, 5, 7, 9), tdepth=3, seed0=30, tseed0=10000):
    """Independent instances i = 0..count-1: L uniform over the even sizes 6..12
    (brickwall targets need an even qubit count), depth uniform over depths, gates
    from seed seed0 + i, target brickwall of depth tdepth from seed tseed0 + i."""
    out = []
    for i in range(count):
        r = np.random.default_rng(seed0 + i)
        L = int(r.choice(sizes))
        depth = int(r.choice(depths))
        vlist = np.stack([haar(r) for _ in range(depth)])
        trng = np.random.default_rng(tseed0 + i)
        tvlist = np.stack([haar(trng) for _ in range(tdepth)])
        out.append((L, vlist, perms_for(L, depth), tvlist, perms_for(L, tdepth)))
    return out
