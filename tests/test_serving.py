"""Scheduler of the serving loop (protomol3_b200/serving.py) on the CPU, with a fake segment
that stands in for the GPU: FIFO admission by memory budget and slot count, chunked progress,
latency accounting."""
import numpy as np

from protomol3_b200 import serving as S
from protomol3_b200 import waterbox as W


class FakeClock:
    def __init__(self, dt=1e-3):
        self.t, self.dt = 0.0, dt

    def __call__(self):
        self.t += self.dt
        return self.t


class FakeSegment:
    """Busy for ``cost`` seconds of the fake clock per step enqueued."""
    live = []

    def __init__(self, req, clock, cost=1e-4):
        self.req, self.clock, self.cost = req, clock, cost
        self.bytes = S.estimate_bytes(req.n_atoms, req.grid)
        self.done_steps = 0
        self.busy_until = 0.0
        FakeSegment.live.append(self)

    def idle(self):
        return self.clock.t >= self.busy_until

    def enqueue(self, n):
        self.done_steps += n
        self.busy_until = self.clock.t + n * self.cost

    def finish(self):
        n = self.req.n_atoms
        return np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(16), 0.0


def _requests(sizes, steps, arrivals):
    return [S.SegmentRequest(k, W.water_box(w, seed=k + 1), st, seed=k + 7, arrival=a)
            for k, (w, st, a) in enumerate(zip(sizes, steps, arrivals))]


def _server(budget, max_active, clock):
    return S.MDServer(hbm_budget_bytes=budget, max_active=max_active, chunk=100, clock=clock,
                      segment_factory=lambda req: FakeSegment(req, clock))


def test_budget_limits_residency_and_all_finish():
    clock = FakeClock()
    reqs = _requests([200] * 6, [500] * 6, [0.0] * 6)
    one = S.estimate_bytes(reqs[0].n_atoms, reqs[0].grid)
    srv = _server(budget=int(2.5 * one), max_active=8, clock=clock)
    res = srv.run_trace(reqs)
    assert len(res) == 6
    assert srv.peak_active == 2
    assert srv.used == 0 and not srv.active and not srv.pending
    # equal work admitted in arrival order finishes in arrival order (pairwise)
    order = [r.req.rid for r in res]
    assert sorted(order[:2]) == [0, 1] and sorted(order[2:4]) == [2, 3]
    assert all(r.latency > 0 for r in res)


def test_slot_limit_and_oversized_request_runs_alone():
    clock = FakeClock()
    reqs = _requests([100, 100, 100, 3000], [300, 300, 300, 300], [0.0, 0.0, 0.0, 0.0])
    small = S.estimate_bytes(reqs[0].n_atoms, reqs[0].grid)
    srv = _server(budget=int(2.2 * small), max_active=2, clock=clock)
    res = srv.run_trace(reqs)
    assert len(res) == 4 and srv.peak_active == 2
    big = [r for r in res if r.req.rid == 3][0]
    assert big.device_bytes > srv.budget  # did not fit the budget, ran when nothing else did


def test_arrivals_wait_for_their_time_and_latency_summary():
    clock = FakeClock()
    reqs = _requests([150, 150, 150], [200, 200, 200], [0.0, 0.5, 1.0])
    srv = _server(budget=1 << 40, max_active=8, clock=clock)
    res = srv.run_trace(reqs)
    for r in res:
        assert r.t_admit >= r.req.arrival
    summ = S.latency_summary(res)
    assert summ["requests"] == 3 and summ["p99_s"] >= summ["p50_s"] > 0


def test_poisson_trace_shape():
    tr = S.poisson_trace(400, rate=2.0, seed=5)
    arr = np.array([t[0] for t in tr])
    atoms = np.array([3 * t[1] for t in tr])
    steps = np.array([t[2] for t in tr])
    assert arr[0] == 0.0 and np.all(np.diff(arr) >= 0)
    assert abs(np.diff(arr).mean() - 0.5) < 0.1
    assert atoms.min() >= 498 and atoms.max() <= 50001
    assert 1000 <= steps.min() and steps.max() <= 20000
    # log-uniform: the median size is near the geometric mean of the range
    assert 3000 < np.median(atoms) < 8000
