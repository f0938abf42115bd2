"""Host logic of the serving loop (admission by slots and device bytes, retirement,
latency accounting) against a stand-in batch; runs without a GPU."""
import numpy as np

from rqcopt_hpc_b200.serving import Request, Server, c5_requests, latency_stats, run_arrivals


class FakeBatch:
    """Each problem finishes after `niter` rounds; results are f_iter = arange."""

    def __init__(self, capacity):
        self.capacity = capacity
        self.left = {}
        self.niter = {}
        self.done = []
        self.max_live = 0

    def add(self, problem, niter, precision, grad_tol=0.0):
        slot = min(set(range(self.capacity)) - set(self.left) - set(self.niter))
        self.left[slot] = niter
        self.niter[slot] = niter
        self.max_live = max(self.max_live, len(self.left))
        return slot

    def run(self, rounds):
        for s in list(self.left):
            self.left[s] -= rounds
            if self.left[s] <= 0:
                del self.left[s]
                self.done.append(s)
        return len(self.left)

    def finished(self):
        d, self.done = self.done, []
        return d

    def result(self, slot):
        return np.arange(self.niter[slot] + 1, dtype=float), None

    def release(self, slot):
        del self.niter[slot]


def _req(rid, L, niter, t):
    return Request(rid, (L, np.zeros((2, 4, 4)), None, None, None), niter, 0.0, t)


def test_admission_respects_capacity_and_budget():
    fb = FakeBatch(capacity=3)
    srv = Server(fb, capacity=3, hbm_budget_bytes=250, footprint=lambda L, nl: 100 if L < 12 else 200,
                 rounds_per_step=1)
    for k, L in enumerate([8, 8, 12, 8, 8]):
        srv.submit(_req(k, L, 2, 0.0))
    srv.step(0.0)
    # 8, 8 fit (200 <= 250); the L = 12 request (200 bytes) waits, and the queue stays in order
    assert len(srv.running) == 2 and srv.used == 200 and len(srv.queue) == 3
    srv.step(1.0)
    srv.step(2.0)
    assert [r.rid for r in srv.completed] == [0, 1]
    assert srv.used == 200 and srv.queue[0].rid == 3   # request 2 now runs alone
    for t in range(3, 12):
        srv.step(float(t))
    assert sorted(r.rid for r in srv.completed) == [0, 1, 2, 3, 4]
    assert fb.max_live <= 3 and srv.used == 0
    assert all(r.iterations == 2 and r.f_final == 2.0 for r in srv.completed)


def test_run_arrivals_latency_accounting():
    clock_t = [0.0]

    def clock():
        clock_t[0] += 0.01
        return clock_t[0]

    fb = FakeBatch(capacity=4)
    srv = Server(fb, capacity=4, hbm_budget_bytes=10 ** 9, footprint=lambda L, nl: 1, rounds_per_step=1)
    reqs = [_req(k, 8, 3, 0.05 * k) for k in range(10)]
    done, left = run_arrivals(srv, reqs, wall_limit=100.0, clock=clock)
    assert len(done) == 10 and not left
    st = latency_stats(done)
    assert st["completed"] == 10 and st["p50_ms"] > 0 and st["p99_ms"] >= st["p50_ms"]
    assert all(r.done >= r.arrival for r in done)


def test_c5_arrivals_are_seeded_and_weighted():
    a = c5_requests(rate=200.0, duration=2.0)
    b = c5_requests(rate=200.0, duration=2.0)
    assert [r.arrival for r in a] == [r.arrival for r in b]
    assert 300 < len(a) < 500
    Ls = np.array([r.problem[0] for r in a])
    assert set(Ls) <= {8, 10, 12, 14}
    # P(L) proportional to 2^(-(L-8)/2): L = 8 is the most frequent, L = 14 the least
    counts = [np.sum(Ls == L) for L in (8, 10, 12, 14)]
    assert counts[0] > counts[1] > counts[3]
