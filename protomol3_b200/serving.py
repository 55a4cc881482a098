"""Serving loop for independent MD segments (Langevin dynamics of water boxes) on one GPU.

Requests arrive over time; each asks for ``steps`` Langevin steps of its own box.  The server
admits them first-in first-out as slots and device memory free up (an HBM budget in bytes and a
maximum number of resident segments), keeps every admitted segment's coordinates, velocities,
neighbour lists and PME grids resident on the device between chunks, and advances all resident
segments concurrently: each one is its own system on its own CUDA stream, and every scheduling
round enqueues the next chunk of steps of each segment whose previous chunk has finished, so the
work of segments admitted at different times overlaps on the device (continuous batching at
chunk granularity).  Latency is wall-clock time from a request's arrival to the moment its last
chunk is seen complete.

A segment's result does not depend on what else runs: its kernels are deterministic (fixed-point
accumulation, deterministic neighbour lists) and its Langevin noise is a counter-based function
of (seed, atom, step), so a segment run alone and in the mix gives bit-identical states.

The GPU work goes through ``GpuSegment`` (the C ABI of libpmb200 via forces.py, PyTorch streams
and events); the scheduler only needs its small interface, which the CPU tests replace by a fake.
"""
import collections
import time

import numpy as np


class SegmentRequest:
    """One MD segment: a periodic water box (dict of waterbox.water_box), the number of Langevin
    steps, the noise seed and the arrival time (seconds from the start of a trace)."""

    def __init__(self, rid, box, steps, seed, arrival=0.0, grid=None):
        self.rid = rid
        self.box = box
        self.steps = int(steps)
        self.seed = int(seed)
        self.arrival = float(arrival)
        if grid is None:
            from .waterbox import pme_grid_for
            grid = pme_grid_for(box["box"][0])
        self.grid = int(grid)
        self.n_atoms = len(box["charge"])


class SegmentResult:
    def __init__(self, req, pos, vel, energies, kinetic, t_admit, t_done, peak_bytes):
        self.req = req
        self.pos, self.vel = pos, vel
        self.energies, self.kinetic = energies, kinetic
        self.t_admit, self.t_done = t_admit, t_done
        self.latency = t_done - req.arrival
        self.device_bytes = peak_bytes


def estimate_bytes(n_atoms, grid):
    """Conservative device footprint of a segment before it exists: ~1.1 kB per atom (atom
    arrays, sorted slots, block neighbour lists at condensed-phase density, integrator state)
    plus 20 bytes per PME grid point (int64 charge grid, half-complex and real FP32 grids) plus
    2 MB of tables, with 25% headroom; the server books the measured size once a segment runs."""
    return int(1.25 * (1100.0 * n_atoms + 20.0 * float(grid) ** 3 + 2.0e6))


class GpuSegment:
    """One resident segment on the GPU (mixed precision by default)."""

    def __init__(self, req, precision="mixed", rc=9.0, switchon=7.5, temperature=300.0,
                 gamma=1.0, timestep=1.0):
        import torch
        from . import forces as F
        self.torch = torch
        self.req = req
        self.stream = torch.cuda.Stream()
        self.topo = F.Topology(req.box, precision)
        self.topo.set_stream(self.stream.cuda_stream)
        grid = req.grid
        self.fl = [F.BondedSystemForce(), F.NonbondedCutoffSystemForce(lj=("C2", switchon, rc)),
                   F.NonbondedPMEwaldSystemForce((grid,) * 3, rc)]
        self.md = F.Integrator(self.topo, self.fl, timestep=timestep, kind="langevin",
                               temperature=temperature, gamma=gamma, seed=req.seed)
        self.md.set_state(req.box["pos"], req.box["vel"])
        self.bytes = self.md.device_bytes()
        self.done_steps = 0
        self.event = None

    def idle(self):
        return self.event is None or self.event.query()

    def enqueue(self, n):
        self.md.run(n)
        self.done_steps += n
        self.event = self.torch.cuda.Event()
        self.event.record(self.stream)

    def finish(self):
        pos, vel = self.md.state()
        e, k = self.md.energies()
        self.md.close()
        self.topo.close()
        return pos, vel, e[0].copy(), float(k[0])


class MDServer:
    """First-in first-out admission by memory budget and slot count; chunked, interleaved
    execution of the resident segments."""

    def __init__(self, hbm_budget_bytes=16 << 30, max_active=32, chunk=200, segment_factory=None,
                 clock=time.perf_counter, **segment_kw):
        self.budget = int(hbm_budget_bytes)
        self.max_active = int(max_active)
        self.chunk = int(chunk)
        self.factory = segment_factory or (lambda req: GpuSegment(req, **segment_kw))
        self.clock = clock
        self.pending = collections.deque()
        self.active = []
        self.used = 0
        self.peak_used = 0
        self.peak_active = 0
        self.results = []
        self.t0 = None

    def now(self):
        return self.clock() - self.t0

    def submit(self, req):
        self.pending.append(req)

    def _admit(self):
        while self.pending and len(self.active) < self.max_active:
            req = self.pending[0]
            need = estimate_bytes(req.n_atoms, req.grid)
            # FIFO: later requests wait behind the first one that does not fit; a request larger
            # than the whole budget still runs, alone
            if self.active and self.used + need > self.budget:
                break
            self.pending.popleft()
            seg = self.factory(req)
            seg.t_admit = self.now()
            self.active.append(seg)
            self.used += seg.bytes
            self.peak_used = max(self.peak_used, self.used)
            self.peak_active = max(self.peak_active, len(self.active))

    def _advance(self):
        progressed = False
        for seg in list(self.active):
            if not seg.idle():
                continue
            left = seg.req.steps - seg.done_steps
            if left > 0:
                seg.enqueue(min(self.chunk, left))
                progressed = True
                continue
            pos, vel, e, k = seg.finish()
            self.results.append(SegmentResult(seg.req, pos, vel, e, k, seg.t_admit, self.now(), seg.bytes))
            self.active.remove(seg)
            self.used -= seg.bytes
            progressed = True
        return progressed

    def run_trace(self, requests, idle_sleep=2e-4):
        """Serves requests whose ``arrival`` times are offsets from now; returns the results in
        completion order."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        self.t0 = self.clock()
        i = 0
        while i < len(reqs) or self.pending or self.active:
            t = self.now()
            while i < len(reqs) and reqs[i].arrival <= t:
                self.submit(reqs[i])
                i += 1
            self._admit()
            if not self._advance():
                time.sleep(idle_sleep)
        return self.results


def poisson_trace(n, rate, seed=2024, atoms_lo=500, atoms_hi=50000, steps_lo=1000,
                  steps_hi=20000):
    """``n`` requests with exponential inter-arrival times (``rate`` per second), sizes
    log-uniform on [atoms_lo, atoms_hi] atoms (water boxes at 1.0 g/cm^3), step counts uniform
    on [steps_lo, steps_hi]; returns (arrival, n_waters, steps, seed) tuples."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=n) if rate > 0 else np.zeros(n)
    arrivals = np.cumsum(gaps) - gaps[0]
    atoms = np.exp(rng.uniform(np.log(atoms_lo), np.log(atoms_hi), size=n))
    waters = np.maximum(1, np.round(atoms / 3.0)).astype(int)
    steps = rng.integers(steps_lo, steps_hi + 1, size=n)
    seeds = rng.integers(1, 2 ** 31, size=n)
    return [(float(a), int(w), int(s), int(sd)) for a, w, s, sd in zip(arrivals, waters, steps, seeds)]


def latency_summary(results, t_span=None):
    lat = np.array([r.latency for r in results])
    atom_steps = float(sum(r.req.n_atoms * r.req.steps for r in results))
    span = t_span if t_span is not None else max(r.t_done for r in results) - min(r.req.arrival for r in results)
    return {"requests": len(results), "p50_s": float(np.percentile(lat, 50)),
            "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean()),
            "throughput_req_s": len(results) / span, "atom_steps_per_s": atom_steps / span,
            "span_s": span}
