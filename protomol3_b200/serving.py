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

``FoldingServer`` folds resident segments of similar size into one batched system (a cohort: one
box per segment, one launch per force stage and one CUDA graph per step for all of them).  A
batched system gives every box the bits it gets alone (list rebuilds are decided per box, pair
tiles never mix boxes, energies are summed in fixed point term by term, the Langevin noise is
keyed by the box's seed, its atom index within the box and its own step count), and a box moves
between batched systems exactly (checkpoint with the list's reference positions, restored with
its noise stream), so a cohort is re-formed whenever one of its segments completes, together with
the segments admitted since, and every result is still the one the segment gets alone.
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
        return pos, vel, e[0].copy(), float(k[0])

    def release(self):
        self.md.close()
        for f in self.fl:  # (their device tables go in the same release batch)
            f._release()
        self.topo.close()


class MDServer:
    """First-in first-out admission by memory budget and slot count; chunked, interleaved
    execution of the resident segments."""

    def __init__(self, hbm_budget_bytes=16 << 30, max_active=32, chunk=200, segment_factory=None,
                 clock=time.perf_counter, release_batch=4, **segment_kw):
        self.budget = int(hbm_budget_bytes)
        # finished systems are released in batches: freeing device memory synchronises the whole
        # device, which would stall the other segments' queued chunks once per completion
        self.release_batch = int(release_batch)
        self.graveyard = []
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

    def _retire(self, obj):
        rel = getattr(obj, "release", None)
        if rel is not None:
            self.graveyard.append(rel)
        if len(self.graveyard) >= self.release_batch:
            self._release_all()

    def _release_all(self):
        for rel in self.graveyard:
            rel()
        self.graveyard = []

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
            self._retire(seg)
            self.active.remove(seg)
            self.used -= seg.bytes
            progressed = True
        return progressed

    def _busy(self):
        return bool(self.pending or self.active)

    def run_trace(self, requests, idle_sleep=2e-4):
        """Serves requests whose ``arrival`` times are offsets from now; returns the results in
        completion order."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        self.t0 = self.clock()
        i = 0
        while i < len(reqs) or self._busy():
            t = self.now()
            while i < len(reqs) and reqs[i].arrival <= t:
                self.submit(reqs[i])
                i += 1
            self._admit()
            if not self._advance():
                time.sleep(idle_sleep)
        self._release_all()
        return self.results


class Member:
    """A segment inside a folding server: its request, the steps done, the admission time, the
    bytes booked for it and, between two cohorts, its exact state (positions, velocities and the
    neighbour list's reference positions)."""

    def __init__(self, req, booked, t_admit):
        self.req = req
        self.booked = booked
        self.t_admit = t_admit
        self.done_steps = 0
        self.state = None

    def left(self):
        return self.req.steps - self.done_steps


class GpuCohort:
    """Segments advanced together as one batched system (one box each) on one CUDA stream."""

    def __init__(self, members, precision="mixed", rc=9.0, switchon=7.5, temperature=300.0,
                 gamma=1.0, timestep=1.0):
        import torch
        from . import forces as F
        self.torch = torch
        self.members = list(members)
        boxes = [m.req.box for m in self.members]
        self.stream = torch.cuda.Stream()
        self.topo = F.Topology(boxes, precision)
        self.topo.set_stream(self.stream.cuda_stream)
        self.fl = [F.BondedSystemForce(), F.NonbondedCutoffSystemForce(lj=("C2", switchon, rc)),
                   F.NonbondedPMEwaldSystemForce((0, 0, 0), rc,
                                                 box_grids=[[m.req.grid] * 3 for m in self.members])]
        self.md = F.Integrator(self.topo, self.fl, timestep=timestep, kind="langevin",
                               temperature=temperature, gamma=gamma, seed=self.members[0].req.seed)
        pos = np.concatenate([m.state[0] if m.state else m.req.box["pos"] for m in self.members])
        vel = np.concatenate([m.state[1] if m.state else m.req.box["vel"] for m in self.members])
        if any(m.state for m in self.members):
            ref = np.concatenate([m.state[2] if m.state else m.req.box["pos"] for m in self.members])
            self.md.restore({"positions": pos, "velocities": vel, "list_reference": ref, "step": 0})
        else:
            self.md.set_state(pos, vel)
        self.md.set_box_noise(seeds=[m.req.seed for m in self.members],
                              steps=[m.done_steps for m in self.members])
        self.bytes = self.md.device_bytes()
        self.event = None

    def release(self):
        self.md.close()
        for f in self.fl:  # (their device tables go in the same release batch)
            f._release()
        self.topo.close()

    def idle(self):
        return self.event is None or self.event.query()

    def left(self):
        return min(m.left() for m in self.members)

    def enqueue(self, n):
        self.md.run(n)
        for m in self.members:
            m.done_steps += n
        self.event = self.torch.cuda.Event()
        self.event.record(self.stream)

    def split(self):
        """Ends the cohort: [(member, pos, vel, energies, kinetic)] of the completed segments and
        the others, each holding its exact state."""
        ck = self.md.checkpoint()
        e, k = self.md.energies()
        done, cont = [], []
        off = 0
        for b, m in enumerate(self.members):
            n = m.req.n_atoms
            sl = slice(off, off + n)
            off += n
            if m.left() == 0:
                done.append((m, ck["positions"][sl].copy(), ck["velocities"][sl].copy(), e[b].copy(), float(k[b])))
            else:
                m.state = (ck["positions"][sl].copy(), ck["velocities"][sl].copy(), ck["list_reference"][sl].copy())
                cont.append(m)
        return done, cont


def size_class(n_atoms, bounds=(2000, 8000, 20000)):
    """Index of the first bound above n_atoms (len(bounds) for the largest segments)."""
    for k, b in enumerate(bounds):
        if n_atoms < b:
            return k
    return len(bounds)


class FoldingServer(MDServer):
    """MDServer whose resident segments of one size class run as one batched system.

    Admission is FIFO by HBM budget (each request books its estimate) and slot count, as in
    MDServer.  Admitted segments, and the unfinished segments of a cohort whose shortest segment
    has completed, are grouped by size class (``class_bounds`` atoms; segments at or above the
    last bound run one per system) into new cohorts of at most ``max_cohort_atoms`` atoms.  Each
    idle cohort advances by min(chunk, its shortest segment's remaining steps)."""

    def __init__(self, hbm_budget_bytes=16 << 30, max_active=32, chunk=200, cohort_factory=None,
                 class_bounds=(2000, 8000, 20000), max_cohort_atoms=200000, clock=time.perf_counter,
                 release_batch=4, **segment_kw):
        super().__init__(hbm_budget_bytes, max_active, chunk, clock=clock, release_batch=release_batch,
                         **segment_kw)
        self.factory = cohort_factory or (lambda members: GpuCohort(members, **segment_kw))
        self.class_bounds = tuple(class_bounds)
        self.max_cohort_atoms = int(max_cohort_atoms)
        self.cohorts = []
        self.loose = []
        self.n_members = 0
        self.cohorts_made = 0
        self.peak_cohorts = 0
        self.device_used = 0
        self.peak_device = 0

    def _admit(self):
        while self.pending and self.n_members < self.max_active:
            req = self.pending[0]
            need = estimate_bytes(req.n_atoms, req.grid)
            if self.n_members and self.used + need > self.budget:
                break
            self.pending.popleft()
            self.loose.append(Member(req, need, self.now()))
            self.n_members += 1
            self.used += need
            self.peak_used = max(self.peak_used, self.used)
            self.peak_active = max(self.peak_active, self.n_members)

    def _form(self):
        groups = collections.defaultdict(list)
        for m in self.loose:
            groups[size_class(m.req.n_atoms, self.class_bounds)].append(m)
        self.loose = []
        for cls in sorted(groups):
            ms = groups[cls]
            if cls == len(self.class_bounds):
                parts = [[m] for m in ms]
            else:
                parts, cur, atoms = [], [], 0
                for m in ms:
                    if cur and atoms + m.req.n_atoms > self.max_cohort_atoms:
                        parts.append(cur)
                        cur, atoms = [], 0
                    cur.append(m)
                    atoms += m.req.n_atoms
                if cur:
                    parts.append(cur)
            for part in parts:
                c = self.factory(part)
                self.cohorts.append(c)
                self.cohorts_made += 1
                self.device_used += c.bytes
        self.peak_cohorts = max(self.peak_cohorts, len(self.cohorts))
        self.peak_device = max(self.peak_device, self.device_used)

    def _cls(self, c):
        return size_class(c.members[0].req.n_atoms, self.class_bounds)

    def _dissolve(self, c):
        done, cont = c.split()
        self._retire(c)
        self.cohorts.remove(c)
        self.device_used -= c.bytes
        t = self.now()
        for m, pos, vel, e, k in done:
            self.results.append(SegmentResult(m.req, pos, vel, e, k, m.t_admit, t, m.booked))
            self.used -= m.booked
            self.n_members -= 1
        self.loose.extend(cont)

    def _advance(self):
        progressed = False
        for c in list(self.cohorts):
            if c.idle() and c.left() == 0:
                self._dissolve(c)
                progressed = True
        self._admit()  # what the completed segments freed, before the survivors are re-formed
        if self.loose:
            # loose segments join their class's cohort: an idle one is dissolved and re-formed
            # with them; while every cohort of the class is busy they wait for its chunk to end
            # (one chunk at most), so that a class keeps one cohort instead of fragmenting
            big = len(self.class_bounds)
            want = {size_class(m.req.n_atoms, self.class_bounds) for m in self.loose} - {big}
            for c in list(self.cohorts):
                if c.idle() and self._cls(c) in want:
                    self._dissolve(c)
            busy = {self._cls(c) for c in self.cohorts if self._cls(c) != big}
            ready = [m for m in self.loose if size_class(m.req.n_atoms, self.class_bounds) not in busy]
            if ready:
                wait = [m for m in self.loose if size_class(m.req.n_atoms, self.class_bounds) in busy]
                self.loose = ready
                self._form()
                self.loose = wait
                progressed = True
        for c in self.cohorts:
            if c.idle():
                c.enqueue(min(self.chunk, c.left()))
                progressed = True
        return progressed

    def _busy(self):
        return bool(self.pending or self.cohorts or self.loose)


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
