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


class FakeCohort:
    """Several members advancing together; busy for ``cost`` seconds per step and member."""
    made = []

    def __init__(self, members, clock, cost=1e-5):
        self.members, self.clock, self.cost = list(members), clock, cost
        self.bytes = sum(m.booked for m in self.members)
        self.busy_until = 0.0
        self.started = [m.done_steps for m in self.members]
        FakeCohort.made.append(self)

    def idle(self):
        return self.clock.t >= self.busy_until

    def left(self):
        return min(m.left() for m in self.members)

    def enqueue(self, n):
        assert 0 < n <= self.left()
        for m in self.members:
            m.done_steps += n
        self.busy_until = self.clock.t + n * self.cost * len(self.members)

    def split(self):
        done, cont = [], []
        for m in self.members:
            n = m.req.n_atoms
            if m.left() == 0:
                done.append((m, np.full((n, 3), float(m.done_steps)), np.zeros((n, 3)), np.zeros(16), 0.0))
            else:
                m.state = (np.zeros((n, 3)), np.zeros((n, 3)), np.zeros((n, 3)))
                cont.append(m)
        return done, cont


def _folding(budget, max_active, clock, **kw):
    FakeCohort.made = []
    return S.FoldingServer(hbm_budget_bytes=budget, max_active=max_active, chunk=100, clock=clock,
                           cohort_factory=lambda ms: FakeCohort(ms, clock), **kw)


def test_folding_groups_by_size_class_and_reforms_when_a_segment_completes():
    """Three small segments (steps 150, 300, 500) share one cohort, re-formed without each one
    that completes; a large one runs in its own system; every segment runs exactly its steps."""
    clock = FakeClock()
    reqs = _requests([150, 160, 170, 8000], [150, 300, 500, 250], [0.0] * 4)
    srv = _folding(1 << 40, 8, clock)
    res = srv.run_trace(reqs)
    assert sorted(r.req.rid for r in res) == [0, 1, 2, 3]
    for r in res:
        assert r.pos[0, 0] == r.req.steps  # the fake's final state records the steps run
    small = [c for c in FakeCohort.made if c.members[0].req.n_atoms < 2000]
    big = [c for c in FakeCohort.made if c.members[0].req.n_atoms >= 20000]
    assert [len(c.members) for c in small] == [3, 2, 1]
    assert [c.started for c in small] == [[0, 0, 0], [150, 150], [300]]
    assert len(big) == 1 and len(big[0].members) == 1
    assert srv.used == 0 and srv.n_members == 0 and not srv.cohorts


def test_folding_admits_fifo_by_budget_and_folds_later_arrivals_in():
    """A budget for two small segments: the third waits, then joins the survivor of the first
    cohort when that cohort is re-formed."""
    clock = FakeClock()
    reqs = _requests([150, 150, 150], [100, 400, 200], [0.0, 0.0, 0.0])
    one = S.estimate_bytes(reqs[0].n_atoms, reqs[0].grid)
    srv = _folding(int(2.5 * one), 8, clock)
    res = srv.run_trace(reqs)
    assert len(res) == 3 and srv.peak_active == 2
    first = FakeCohort.made[0]
    assert [m.req.rid for m in first.members] == [0, 1]
    second = FakeCohort.made[1]
    assert sorted(m.req.rid for m in second.members) == [1, 2]
    assert sorted(second.started) == [0, 100]


def test_folding_caps_cohort_atoms():
    clock = FakeClock()
    reqs = _requests([600] * 5, [200] * 5, [0.0] * 5)  # 1,800 atoms each
    srv = _folding(1 << 40, 8, clock, max_cohort_atoms=4000)
    srv.run_trace(reqs)
    assert [len(c.members) for c in FakeCohort.made] == [2, 2, 1]


def test_size_class():
    assert [S.size_class(n) for n in (500, 1999, 2000, 7999, 8000, 19999, 20000, 50000)] == [0, 0, 1, 1, 2, 2, 3, 3]


def test_folding_later_arrivals_join_the_running_cohort_of_their_class():
    """A segment that arrives while its class's cohort runs a chunk waits for the chunk's end
    and is folded in (the class keeps one cohort); one of another class gets its own."""
    clock = FakeClock()
    reqs = _requests([150, 160, 3000], [20000, 300, 300], [0.0, 0.05, 0.06])
    srv = _folding(1 << 40, 8, clock)
    res = srv.run_trace(reqs)
    assert sorted(r.req.rid for r in res) == [0, 1, 2]
    for r in res:
        assert r.pos[0, 0] == r.req.steps
    small = [c for c in FakeCohort.made if c.members[0].req.n_atoms < 2000]
    assert [sorted(m.req.rid for m in c.members) for c in small][:2] == [[0], [0, 1]]
    assert small[1].started[[m.req.rid for m in small[1].members].index(0)] > 0
    assert srv.peak_cohorts == 2
