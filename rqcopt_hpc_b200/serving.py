"""Continuous-batching request loop for brickwall circuit optimisation.

Requests (one brickwall problem each, see :mod:`rqcopt_hpc_b200.batch`) arrive
over time.  The loop admits every request that has arrived as soon as a batch
slot is free and its device footprint fits the HBM budget, so new arrivals join
the next batched round while earlier requests are still iterating on the GPU;
a request leaves when it reaches its gradient tolerance or its iteration limit.
Every request keeps its gates, states and trust-region vectors resident on the
device between iterations.  Latency is time from arrival to completion.

The batch engine makes a request's arithmetic independent of what else is in
the batch (its work items and their summation order depend on the request
alone), so a result is the same whether it ran alone or in a mix.  With the
batch's cost-weighted sharing on, a request is evaluated every p-th round, p
growing with its cost per evaluation, so small requests are not held back by
large ones in the same rounds.
"""
from __future__ import annotations

import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Request:
    rid: int
    problem: tuple          # (L, vlist, perms, target_vlist, target_perms)
    niter: int
    grad_tol: float
    arrival: float          # seconds after the start of the run
    precision: int = 1      # RQCOPT_PRECISION_MIXED
    admitted: float = -1.0
    done: float = -1.0
    iterations: int = 0
    f_final: float = float("nan")
    f_iter: np.ndarray = field(default=None, repr=False)


class Server:
    """Admission by slots and device bytes; `batch` is a batch.Batch (or any object
    with add / run / finished / result / release)."""

    def __init__(self, batch, capacity, hbm_budget_bytes, footprint, rounds_per_step=4):
        self.batch = batch
        self.capacity = capacity
        self.budget = hbm_budget_bytes
        self.footprint = footprint           # (L, nlayers) -> bytes
        self.rounds_per_step = rounds_per_step
        self.queue = deque()
        self.running = {}                    # slot -> (request, bytes)
        self.used = 0
        self.completed = []
        self.rounds = 0

    def submit(self, req: Request):
        self.queue.append(req)

    def _admit(self, now):
        while self.queue and len(self.running) < self.capacity:
            req = self.queue[0]
            nbytes = self.footprint(req.problem[0], len(req.problem[1]))
            if self.used + nbytes > self.budget:
                break
            self.queue.popleft()
            slot = self.batch.add(req.problem, req.niter, req.precision, grad_tol=req.grad_tol)
            req.admitted = now
            self.running[slot] = (req, nbytes)
            self.used += nbytes

    def step(self, now):
        """Admit what has arrived, run a few rounds, retire what finished; returns the
        requests completed in this step."""
        self._admit(now)
        done = []
        if self.running:
            self.batch.run(self.rounds_per_step)
            self.rounds += self.rounds_per_step
            for slot in self.batch.finished():
                req, nbytes = self.running.pop(slot)
                f_iter, _ = self.batch.result(slot)
                self.batch.release(slot)
                self.used -= nbytes
                req.f_iter = f_iter
                req.iterations = len(f_iter) - 1
                req.f_final = float(f_iter[-1])
                done.append(req)
        self.completed += done
        return done


def latency_stats(reqs):
    lat = np.array([r.done - r.arrival for r in reqs])
    if lat.size == 0:
        return {"completed": 0}
    return {"completed": int(lat.size), "p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3), "mean_ms": float(lat.mean() * 1e3),
            "max_ms": float(lat.max() * 1e3)}


def run_arrivals(server: Server, requests, wall_limit, clock=time.perf_counter):
    """Feed requests (sorted by arrival) into the server in real time until all are done
    or wall_limit seconds have passed; returns (completed, still running or queued)."""
    t0 = clock()
    pending = deque(sorted(requests, key=lambda r: r.arrival))
    while True:
        now = clock() - t0
        while pending and pending[0].arrival <= now:
            server.submit(pending.popleft())
        if not server.running and not server.queue:
            if not pending:
                break
            # idle until the next arrival
            time.sleep(max(0.0, min(pending[0].arrival - now, 0.01)))
            continue
        done = server.step(now)
        tdone = clock() - t0
        for r in done:
            r.done = tdone
        if tdone > wall_limit:
            break
    left = list(server.queue) + [r for r, _ in server.running.values()] + list(pending)
    return server.completed, left


def c5_requests(rate=200.0, duration=60.0, seed=40, niter=100, grad_tol=1e-8, precision=1,
                sizes=(8, 10, 12, 14), depths=(3, 5, 7, 9)):
    """Poisson arrivals (seeded); L with P(L) proportional to 2^(-(L-8)/2) over the even
    sizes (brickwall targets need an even qubit count), depth uniform, gates and target
    (random brickwall of depth 3) seeded per request."""
    from .workloads import brickwall_problem
    rng = np.random.default_rng(seed)
    w = np.array([2.0 ** (-(L - 8) / 2) for L in sizes])
    w /= w.sum()
    t, reqs, rid = 0.0, [], 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            break
        L = int(rng.choice(sizes, p=w))
        depth = int(rng.choice(depths))
        reqs.append(Request(rid, brickwall_problem(L, depth, 3, 40_000 + rid, 80_000 + rid), niter, grad_tol, t,
                            precision))
        rid += 1
    return reqs
