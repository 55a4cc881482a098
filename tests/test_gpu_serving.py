"""Serving loop on the GPU: segments admitted together run concurrently, and each one's final
state is bit-identical to the same segment served alone (deterministic kernels, per-segment
counter-based Langevin noise).  Tolerance: exact equality of positions, velocities, energies."""
import numpy as np
import pytest

from protomol3_b200 import serving as S
from protomol3_b200 import waterbox as W

pytestmark = pytest.mark.gpu


def _reqs(arrivals=(0.0, 0.0, 0.0)):
    spec = [(200, 300, 5), (500, 400, 6), (1000, 500, 7)]  # waters, steps, seed
    return [S.SegmentRequest(k, W.water_box(w, seed=40 + k), st, seed=sd, arrival=a)
            for k, ((w, st, sd), a) in enumerate(zip(spec, arrivals))]


def _by_id(results):
    return {r.req.rid: r for r in results}


def test_each_result_alone_equals_result_in_the_mix():
    mixed = S.MDServer(max_active=8, chunk=100)
    together = _by_id(mixed.run_trace(_reqs()))
    assert mixed.peak_active == 3  # all three resident and advancing at once
    for k, req in enumerate(_reqs()):
        alone = S.MDServer(max_active=1, chunk=100).run_trace([req])[0]
        t = together[k]
        assert np.array_equal(alone.pos, t.pos)
        assert np.array_equal(alone.vel, t.vel)
        assert np.array_equal(alone.energies, t.energies) and alone.kinetic == t.kinetic
        assert np.isfinite(t.pos).all()


def test_staggered_arrivals_and_budget():
    """A budget that holds one segment serialises them; staggered arrivals are served in order
    and every segment frees its device memory when it completes.  The budget is the smallest
    request's estimate, so no request fits beside a resident one whatever the timing (a request
    above the budget still runs, alone)."""
    reqs = _reqs(arrivals=(0.0, 0.05, 0.1))
    one = min(S.estimate_bytes(r.n_atoms, r.grid) for r in reqs)
    srv = S.MDServer(hbm_budget_bytes=one, max_active=8, chunk=100)
    res = srv.run_trace(reqs)
    assert [r.req.rid for r in res] == [0, 1, 2]
    assert srv.peak_active == 1 and srv.used == 0
    free = _by_id(S.MDServer(max_active=8, chunk=100).run_trace(_reqs(arrivals=(0.0, 0.05, 0.1))))
    for r in res:
        assert np.array_equal(r.pos, free[r.req.rid].pos)


def test_folded_cohorts_give_each_segment_its_result_alone():
    """Segments of one size class folded into a batched system, re-formed as each completes
    (with the later segment folded in), and one of another class: every final state, energy and
    kinetic energy equals the segment's alone, bit for bit."""
    spec = [(200, 300, 5, 0.0), (230, 500, 6, 0.0), (180, 400, 8, 0.0), (1000, 350, 7, 0.0)]
    reqs = lambda: [S.SegmentRequest(k, W.water_box(w, seed=40 + k), st, seed=sd, arrival=a)
                    for k, (w, st, sd, a) in enumerate(spec)]
    srv = S.FoldingServer(max_active=8, chunk=100, class_bounds=(2000, 8000))
    folded = _by_id(srv.run_trace(reqs()))
    assert srv.cohorts_made >= 4  # the three small ones re-formed as each completes
    for k, req in enumerate(reqs()):
        alone = S.MDServer(max_active=1, chunk=100).run_trace([req])[0]
        t = folded[k]
        assert np.array_equal(alone.pos, t.pos), k
        assert np.array_equal(alone.vel, t.vel), k
        assert np.array_equal(alone.energies, t.energies) and alone.kinetic == t.kinetic, k
