#!/usr/bin/env python
"""Benchmark of the B200 nonbonded / PME force path: ns/day of one MD step on the 98,304-atom
flexible TIP3P box (32,768 waters, 99.3 A, 1.0 g/cm^3), Lennard-Jones C2 8 -> 10 A, PME
96^3 / order 4 / real-space cutoff 10 A / accuracy 1e-6, bonds + angles, leapfrog 1 fs.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Prints one JSON line (rank 0).  ``value`` is the device-resident step (inputs resident in HBM,
one CUDA graph per step, CUDA events on the launching stream, L2 flushed by a 256 MB write
before every timed step, max over ranks); ``e2e`` drives the same step through the C ABI with
pinned host buffers (positions host->device, forces and energies device->host, leapfrog update
on the host); ``roofline`` covers the dominant kernel (the fused LJ + Ewald real-space pair
kernel), ``cpu_baseline`` the reference's own force classes compiled from its sources, timed on
one host core.  For --gpus N > 1 every rank runs an independent replica (no collective).
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DT_FS = 1.0
N_WATERS = 32768
GRID = 96
RC = 10.0
SWITCHON = 8.0
FLOPS_PER_PAIR = 70  # fixed convention for the pair kernel's algorithmic work


def ns_per_day(ms_per_step, dt_fs=DT_FS):
    return 86400.0 * dt_fs * 1e-6 / (ms_per_step * 1e-3)


def workload(rank=0):
    from protomol3_b200 import waterbox as W
    return W.water_box(N_WATERS, seed=1234 + rank)


def config_dict():
    return {"workload": "TIP3P water box, 32768 waters (98304 atoms), 99.34 A periodic, LJ C2 8->10 A, "
                        "PME 96^3 order 4 rc 10 A accuracy 1e-6, bonds+angles, leapfrog 1 fs",
            "atoms": 3 * N_WATERS, "pme_grid": GRID, "cutoff": RC, "timestep_fs": DT_FS,
            "l2": "flushed (256 MB write) before every timed step"}


# ------------------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None
        self.thread = None
        self.samples = []

    # NVML read-only queries every 2 ms (a timed region of 50 steps lasts tens of milliseconds);
    # nvidia-smi at its 200 ms period is the fallback when NVML is not importable
    def _nvml_loop(self, nv, h):
        names = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
                 ("sw_power_cap", 0x4))
        smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while not self.stop_flag:
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                r = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
                self.samples.append((sm, smax, [n for n, bit in names if r & bit]))
            except Exception:
                pass
            time.sleep(0.002)

    def start(self):
        try:
            import threading
            import pynvml as nv
            nv.nvmlInit()
            vis = os.environ.get("CUDA_VISIBLE_DEVICES")
            idx = int(vis.split(",")[self.gpu]) if vis and vis.split(",")[0].isdigit() else self.gpu
            h = nv.nvmlDeviceGetHandleByIndex(idx)
            self.stop_flag = False
            self.thread = threading.Thread(target=self._nvml_loop, args=(nv, h), daemon=True)
            self.thread.start()
            return
        except Exception:
            self.thread = None
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.thread is not None:
            self.stop_flag = True
            self.thread.join(timeout=5)
            sm = [s[0] for s in self.samples]
            reasons = sorted({n for s in self.samples for n in s[2]})
            return {"sm_mhz": float(np.median(sm)) if sm else None,
                    "sm_max_mhz": float(self.samples[0][1]) if sm else None, "samples": len(sm),
                    "reasons": reasons, "source": "nvml, 2 ms period"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in open(self.path):
            t = [x.strip() for x in ln.split(",")]
            if len(t) < 9:
                continue
            try:
                sm.append(float(t[1]))
                smax.append(float(t[2]))
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if t[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "samples": len(sm),
                "reasons": sorted(reasons)}


# ------------------------------------------------------------------------------- helpers
def max_over_ranks(x, dist, device):
    """Largest value of x over the ranks: the slowest replica sets the job's time.  Every rank
    calls it at the same point (a collective); without a process group it returns x."""
    if not dist:
        return x
    import torch
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def pair_count(box, rc):
    """Exact number of unordered atom pairs within rc (minimal image) minus excluded pairs."""
    from scipy.spatial import cKDTree
    L = box["box"][0]
    pos = np.mod(box["pos"], L)
    pos[pos >= L] -= L
    tree = cKDTree(pos, boxsize=L)
    n_ordered = tree.count_neighbors(tree, rc)
    n = len(pos)
    return (n_ordered - n) // 2 - len(box["excl_pairs"])


def force_errors(f, e, f_ref, e_ref):
    """Error of forces f / energies e [Coulomb, LJ, ...] against FP64 references: RMS relative
    force error sqrt(sum |F - F_ref|^2 / sum |F_ref|^2), the largest per-atom error relative to
    that atom's force and relative to the RMS force, and the relative error of each energy term."""
    d = np.linalg.norm(f - f_ref, axis=1)
    fr = np.linalg.norm(f_ref, axis=1)
    rms = float(np.sqrt((fr ** 2).mean()))
    out = {"rms_rel_force": float(np.sqrt((d ** 2).sum() / (fr ** 2).sum())),
           "max_rel_force_per_atom": float((d / np.maximum(fr, 1e-300)).max()),
           "max_force_err_over_rms_force": float(d.max() / rms)}
    for k, name in ((0, "coulomb"), (1, "lj")):
        out["energy_rel_" + name] = float(abs(e[k] - e_ref[k]) / abs(e_ref[k]))
        out["energy_abs_" + name] = float(abs(e[k] - e_ref[k]))
    return out


def read_profile_traffic():
    """DRAM bytes per launch of the pair kernel from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "pair_kernel_water98k.md")
    if not os.path.exists(p):
        return None
    for ln in open(p):
        if ln.startswith("dram_bytes_per_launch:"):
            try:
                return float(ln.split(":")[1].split()[0])
            except ValueError:
                return None
    return None


def cpu_facts():
    """The host CPU the baseline runs on: model name, logical CPUs, CPUs this process may use."""
    model = None
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                model = ln.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    try:
        usable = len(os.sched_getaffinity(0))
    except AttributeError:
        usable = os.cpu_count()
    return {"cpu_model": model, "nproc": os.cpu_count(), "usable_cpus": usable}


class stdout_to_stderr:
    """File-descriptor level redirection of stdout to stderr while the reference's code runs: its
    report stream prints to stdout, where only the JSON line belongs."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)

    def __exit__(self, *exc):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)


def ref_force_step(box, rc, switchon, grid, steps):
    """``steps`` evaluations of LJ C2 (switchon -> rc) + PME (grid^3, order 4, accuracy 1e-6,
    real-space rc) on one core: the reference's own force classes compiled from its sources
    (oracle/_ref), else the C restatement (oracle/).  Returns (s per step, forces of the last
    evaluation, energies [Coulomb, LJ, bond, angle], kind)."""
    import ctypes as C
    from oracle import oracle as O
    s = O.System(box)
    pos = np.ascontiguousarray(box["pos"])
    f = np.zeros((s.n, 3))
    e = np.zeros(4)
    if O.ref_available():
        L = O.ref_lib()
        r = O._ref_input(s, pos, 5.0)
        c = O.RefCutoff()
        cp = O.cutoff_params(lj=("C2", switchon, rc))
        C.memmove(C.byref(c), C.byref(cp), C.sizeof(c))
        p = O.RefPME()
        p.nx = p.ny = p.nz = grid
        p.order, p.cutoff, p.accuracy, p.alpha, p.real_switch = 4, rc, 1e-6, -1.0, 0
        with stdout_to_stderr():
            t0 = time.perf_counter()
            L.ref_time_step(C.byref(r), C.byref(c), C.byref(p), int(steps), O._p(f), O._p(e))
            dt = (time.perf_counter() - t0) / steps
        return dt, f, e, "reference"
    cp = O.cutoff_params(lj=("C2", switchon, rc))
    pm = O.pme_params((grid,) * 3, rc)
    t0 = time.perf_counter()
    for _ in range(steps):
        f, e, _, _ = O.evaluate(s, pos, cutoff=cp, pme=pm)
    return (time.perf_counter() - t0) / steps, f, e, "port"


def cpu_baseline(box, steps=1):
    """The reference's own force classes (compiled from its sources into oracle/_ref) on one
    core; falls back to the C restatement (oracle/) when the compiled reference is absent.
    Also returns the forces and energies of that evaluation, the FP64 reference the accuracy of
    the timed configuration is stated against."""
    dt, f, e, kind = ref_force_step(box, RC, SWITCHON, GRID, steps)
    out = {"value": ns_per_day(dt * 1e3), "unit": "ns/day", "cores": 1, "kind": kind,
           "sample": "%d force evaluation(s) (LJ C2 + PME 96^3 with real, reciprocal and correction "
                     "terms) of the 98,304-atom box, single-threaded; %.2f s per step" % (steps, dt)}
    out.update(cpu_facts())
    return out, f, e


def _ensemble_box_step(args):
    """One box of the ensemble workload through the reference's force classes, one evaluation;
    run in a spawned worker process (no CUDA)."""
    k, n_waters, seed, grid = args
    from protomol3_b200 import waterbox as W
    box = W.water_box(n_waters, seed=seed)
    dt, _, _, kind = ref_force_step(box, BATCH_RC, BATCH_SWITCHON, grid, 1)
    return len(box["charge"]), dt, kind


def cpu_ensemble(processes=None):
    """The ensemble workload on the host the way the reference would run it: one single-threaded
    process per box, ``nproc`` of them at a time, every box evaluated once (LJ C2 7.5 -> 9 A +
    PME ~1 A spacing, order 4).  Aggregate atom-steps/s = atoms of all boxes / wall time."""
    import multiprocessing as mp
    from protomol3_b200 import waterbox as W
    # the same water counts, seeds and grids as waterbox.ensemble() gives the GPU leg
    counts = np.random.default_rng(4321).integers(100, 2001, size=256)
    work = [(k, int(n), 4321 + 1 + k, W.pme_grid_for(W.box_edge(int(n)))) for k, n in enumerate(counts)]
    nproc = processes or cpu_facts()["usable_cpus"] or 1
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(nproc) as pool:
        res = pool.map(_ensemble_box_step, work, chunksize=1)
    wall = time.perf_counter() - t0
    atoms = sum(r[0] for r in res)
    return {"value": atoms / wall, "unit": "atom-steps/s", "processes": nproc, "boxes": len(res),
            "atoms": atoms, "wall_s": wall, "kind": res[0][2],
            "single_core_atom_steps_s": atoms / sum(r[1] for r in res),
            "sample": "every box evaluated once, one single-threaded process per box, %d at a time "
                      "(process start-up included in the wall time)" % nproc}


# ------------------------------------------------------------------------------- B200 arm
def run_b200(args, rank, world, local_rank):
    import torch
    from protomol3_b200 import forces as F

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    box = workload(rank)
    # a non-default stream: the legacy default stream cannot be captured into a CUDA graph
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    # the speed knobs (skin, sort cells, pair CTAs per SM) of each precision's system, picked by
    # the autotuner from whole MD steps before anything is timed; they change no evaluated pair
    tuned = {}
    if not args.no_tune:
        from protomol3_b200 import autotune as AT
        tuner = AT.Autotuner(steps=30, warmup=10)
        for prec in ([args.precision] + (["fp64"] if args.precision == "mixed" and not args.no_fp64 else [])):
            tuned[prec] = tuner.tune_knobs([box], [GRID], RC, SWITCHON, order=4, precision=prec,
                                           stream=stream.cuda_stream)

    def make(precision):
        topo = F.Topology(box, precision)
        topo.set_stream(stream.cuda_stream)
        if precision in tuned:
            topo.set_tuning(**tuned[precision]["knobs"])
        fl = [F.BondedSystemForce(), F.NonbondedCutoffSystemForce(lj=("C2", SWITCHON, RC)),
              F.NonbondedPMEwaldSystemForce((GRID,) * 3, RC)]
        return topo, fl

    def time_md(topo, fl, steps, warmup):
        md = F.Integrator(topo, fl, timestep=DT_FS)
        md.set_state(box["pos"], box["vel"])
        for _ in range(warmup):
            flush.zero_()
            md.run(1)
        torch.cuda.synchronize()
        builds0 = topo.list_builds()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        for a, b in evs:
            flush.zero_()
            a.record(stream)
            md.run(1)
            b.record(stream)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        ms = sum(a.elapsed_time(b) for a, b in evs) / steps
        # launches: each step's graph plus the closing half kick of run(1)
        rebuilds = topo.list_builds() - builds0
        kps = (md.kernels_per_step() + 1) * steps
        pos, vel = md.state()
        if not np.isfinite(pos).all():
            raise RuntimeError("non-finite positions after the timed run")
        md.close()
        return ms, kps, rebuilds

    clocks = ClockSampler(local_rank)
    topo, fl = make(args.precision)
    clocks.start()
    ms, kps, rebuilds = time_md(topo, fl, args.steps, args.warmup)
    clk = clocks.stop()
    ms = max_over_ranks(ms, dist, "cuda")
    value = world * ns_per_day(ms)

    # stage profile of one force evaluation (cold L2) -> pair-kernel roofline
    stages = F.profile(topo, [fl[1], fl[2], fl[0]], nrep=5, flush_l2=True)
    t_pair = stages.get("pair")
    pair_slots = 256 * topo.list_tiles()  # what the timed pair launches evaluated
    peak = F.fp32_peak()
    npairs = pair_count(box, RC) if rank == 0 else None

    # end-to-end through the C ABI with pinned host buffers
    def e2e_leg(topo, fl):
        n = topo.n_atoms
        # pinned host buffers; the caller's leapfrog runs in place on the host (torch CPU ops on
        # the same memory, multi-threaded, as a C++ integrator loop of the caller would)
        tpos = torch.empty((n, 3), dtype=torch.float64, pin_memory=True)
        tfrc = torch.empty((n, 3), dtype=torch.float64, pin_memory=True)
        hpos, hfrc = tpos.numpy(), tfrc.numpy()
        hpos[:] = box["pos"]
        h = DT_FS * 0.02045482828087295
        tvel = torch.from_numpy(box["vel"].copy())
        thinv = torch.from_numpy(np.repeat(h / box["mass"], 3).reshape(n, 3))
        en = F.ScalarStructure(1)
        # 4 x the timed MD steps (200 by default): the host side of a call varies from call to call
        nsteps = max(3, 4 * args.steps)
        parts = {"enqueue": 0.0, "wait_device": 0.0, "accumulate": 0.0, "host_leapfrog": 0.0}
        for it in range(nsteps + 2):
            if it == 2:
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                parts = dict.fromkeys(parts, 0.0)
            tfrc.zero_()
            en.clear()
            F.evaluate_all(topo, fl, hpos, hfrc, en)
            t1 = time.perf_counter()
            tvel.addcmul_(tfrc, thinv)
            tpos.add_(tvel, alpha=h)
            parts["host_leapfrog"] += (time.perf_counter() - t1) * 1e3
            for k, v in topo.evaluate_times().items():
                parts[k] += v
        e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / nsteps, dist, "cuda")
        return {"value": world * ns_per_day(e2e_ms), "unit": "ns/day", "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": int(hpos.nbytes), "d2h_bytes_per_step": int(hfrc.nbytes + 16 * 8),
                "breakdown_ms": {k: v / nsteps for k, v in parts.items()}, "calls_timed": nsteps,
                "path": "pmb_evaluate (C ABI) with pinned host positions/forces + host leapfrog"}

    def forces_at_start(topo, fl):
        """Forces and energies of the nonbonded terms (LJ + PME) at the starting coordinates."""
        frc = np.zeros((topo.n_atoms, 3))
        en = F.ScalarStructure(1)
        F.evaluate_all(topo, fl, box["pos"], frc, en)
        return frc, en.table[0, :4].copy()

    e2e = e2e_leg(topo, fl) if (rank == 0 or world > 1) else None
    start = {args.precision: forces_at_start(topo, [fl[1], fl[2]])}

    # plain FP64 path on the same workload (the drop-in); the headline is the mixed path
    fp64 = None
    if args.precision == "mixed" and not args.no_fp64:
        topo64, fl64 = make("fp64")
        ms64, _, _ = time_md(topo64, fl64, max(3, args.steps // 2), 3)
        ms64 = max_over_ranks(ms64, dist, "cuda")
        fp64 = {"value": world * ns_per_day(ms64), "ms_per_step": ms64,
                "mixed_over_fp64": ns_per_day(ms) / ns_per_day(ms64),
                "e2e": e2e_leg(topo64, fl64) if (rank == 0 or world > 1) else None}
        start["fp64"] = forces_at_start(topo64, [fl64[1], fl64[2]])
        topo64.close()

    serving = None
    if rank == 0 and world == 1 and not args.no_serve:
        serving = serve_leg(n_requests=args.serve_requests)

    batched = None
    if not args.no_batch:
        batched = batch_leg(stream, flush)
        batched["ms_per_step"] = max_over_ranks(batched["ms_per_step"], dist, "cuda")
        batched["value"] = world * batched["atoms"] / (batched["ms_per_step"] * 1e-3)

    base, accuracy, cpu_ens = None, None, None
    if rank == 0 and world == 1 and not args.no_cpu:
        base, f_ref, e_ref = cpu_baseline(box, steps=args.cpu_steps)
        accuracy = {"against": "the reference's own FP64 force classes (%s) on the starting coordinates, "
                               "LJ C2 + PME" % base["kind"]}
        for prec, (f, e) in start.items():
            accuracy[prec] = force_errors(f, e, f_ref, e_ref)
        if not args.no_batch:
            cpu_ens = cpu_ensemble()
            batched["cpu_reference_nproc"] = cpu_ens
    elif rank == 0 and "fp64" in start:
        accuracy = {"against": "the plain FP64 GPU path on the starting coordinates (no CPU leg run)",
                    args.precision: force_errors(*start[args.precision], *start["fp64"])}

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    achieved = FLOPS_PER_PAIR * npairs / (t_pair * 1e-3) / 1e12 if t_pair else None
    traffic = read_profile_traffic()
    line = {
        "metric": "ns/day at 98k atoms (TIP3P, LJ C2 + PME 96^3, 1 fs leapfrog)",
        "value": value, "unit": "ns/day", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if args.precision == "mixed" else "f64", "data": "synthetic",
        "config": dict(config_dict(), precision=args.precision,
                       parallelism="replicas" if world > 1 else "single",
                       tuning={k: {"knobs": v["knobs"], "untuned_ms_per_step": v["default_ms_per_step"],
                                   "search_s": v["search_s"]} for k, v in tuned.items()}),
        "clocks": clk, "gpu_launches": kps, "list_rebuilds": rebuilds, "e2e": e2e,
        "roofline": {"bound": "fp32", "kernel": "k_pair (LJ C2 + Ewald real space)",
                     "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak if achieved and peak else None, "traffic": traffic,
                     "work": "%d FLOP x %d in-cutoff pairs per launch" % (FLOPS_PER_PAIR, npairs),
                     "pair_slots_per_launch": pair_slots,
                     "in_cutoff_fraction": npairs / pair_slots if npairs and pair_slots else None,
                     "kernel_ms": t_pair, "peak_source": "measured FP32 FMA issue rate (pmb_fp32_peak)"},
        "stages_ms": stages, "plain_fp64": fp64, "batched": batched, "serving": serving, "cpu_baseline": base,
        "accuracy": accuracy,
    }
    print(json.dumps(line), flush=True)


BATCH_RC, BATCH_SWITCHON = 9.0, 7.5


def batch_leg(stream, flush, steps=20, warmup=3, loop_steps=8, loop_boxes=None):
    """Ensemble throughput: 256 independent water boxes (100-2000 waters each, ~810k atoms,
    ~5% of them smaller than twice the cutoff), LJ C2 7.5 -> 9 A, PME at ~1 A grid spacing, order
    4, leapfrog 1 fs.  All boxes advance together in one mixed-precision system (one launch per
    force stage, one CUDA graph per step), timed with CUDA events, L2 flushed before each step;
    against it, the plain FP64 path looped box by box (one system and graph per box, every box
    timed over ``loop_steps`` steps).  Rates in atom-steps/s."""
    import torch
    from protomol3_b200 import forces as F
    from protomol3_b200 import waterbox as W
    boxes, grids = W.ensemble()
    natoms = int(sum(len(b["charge"]) for b in boxes))

    def force_set(bg):
        return [F.BondedSystemForce(), F.NonbondedCutoffSystemForce(lj=("C2", BATCH_SWITCHON, BATCH_RC)),
                F.NonbondedPMEwaldSystemForce((0, 0, 0), BATCH_RC, box_grids=bg)]

    def timed(topo, fl, pos, vel, nsteps, nwarm, precision_flush=True):
        md = F.Integrator(topo, fl, timestep=DT_FS)
        md.set_state(pos, vel)
        for _ in range(nwarm):
            md.run(1)
        torch.cuda.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(nsteps)]
        for a, b in evs:
            if precision_flush:
                flush.zero_()
            a.record(stream)
            md.run(1)
            b.record(stream)
        torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in evs)
        p, _ = md.state()
        if not np.isfinite(p).all():
            raise RuntimeError("non-finite positions in the batch leg")
        md.close()
        return ms

    pos = np.concatenate([b["pos"] for b in boxes])
    vel = np.concatenate([b["vel"] for b in boxes])
    # untuned: the fixed rules (smallest 2/3/5-smooth grid at 1 A, skin 0.8 A, 2.4 A sort cells)
    topo = F.Topology(boxes, "mixed")
    topo.set_stream(stream.cuda_stream)
    ms_default = timed(topo, force_set([(g, g, g) for g in grids]), pos, vel, steps, warmup)
    topo.close()
    # autotuned (search outside the timed region)
    from protomol3_b200 import autotune as AT
    tuner = AT.Autotuner()
    tuned = tuner.tune(boxes, BATCH_RC, BATCH_SWITCHON, order=4, precision="mixed")
    topo, fl = tuner.apply(boxes, tuned, BATCH_RC, BATCH_SWITCHON, order=4, precision="mixed")
    topo.set_stream(stream.cuda_stream)
    ms = timed(topo, fl, pos, vel, steps, warmup)
    stages = F.profile(topo, [fl[1], fl[2], fl[0]], positions=pos, nrep=3, flush_l2=True)
    topo.close()
    batched = natoms * steps / (ms * 1e-3)

    def loop(precision):
        sel = range(len(boxes)) if loop_boxes is None else range(min(loop_boxes, len(boxes)))
        loop_ms, loop_atoms = 0.0, 0
        for k in sel:
            b = boxes[k]
            t = F.Topology(b, precision)
            t.set_stream(stream.cuda_stream)
            loop_ms += timed(t, force_set([(grids[k],) * 3]), b["pos"], b["vel"], loop_steps, 2, False)
            loop_atoms += len(b["charge"])
            t.close()
        return {"value": loop_atoms * loop_steps / (loop_ms * 1e-3), "boxes_timed": len(sel),
                "steps_per_box": loop_steps, "ms_per_step_all_boxes": loop_ms / loop_steps * len(boxes) / len(sel)}
    loop64 = loop("fp64")
    loop32 = loop("mixed")
    return {"metric": "atom-steps/s, 256 water boxes of 300-6000 atoms",
            "value": batched, "unit": "atom-steps/s", "atoms": natoms, "boxes": len(boxes),
            "steps": steps, "ms_per_step": ms / steps, "precision": "mixed",
            "untuned": {"value": natoms * steps / (ms_default * 1e-3), "ms_per_step": ms_default / steps},
            "autotune": {"knobs": tuned["knobs"], "grids_changed": int(sum(g != d for g, d in zip(tuned["grids"], grids))),
                         "classes": tuned["classes"], "search_s": tuned["search_s"], "trials": tuned["trials"]},
            "stages_ms": stages,
            "plain_fp64_loop": loop64, "mixed_loop": loop32,
            "batched_over_loop": batched / loop64["value"],
            "batched_over_mixed_loop": batched / loop32["value"],
            "config": "LJ C2 7.5->9 A, PME at <= 1 A spacing (2/3/5-smooth, grid per size class and skin, "
                      "sort cells, pair CTAs per SM picked by the autotuner), order 4, rc 9 A, leapfrog 1 fs; "
                      "L2 flushed before each batched step"}


def nve_run(F, box, precision, stream, steps, chunk):
    """Leapfrog NVE from the box's state; total energy (potential of the last evaluation plus
    kinetic at the synchronised velocities) after every ``chunk`` steps."""
    topo = F.Topology(box, precision)
    topo.set_stream(stream.cuda_stream)
    fl = [F.BondedSystemForce(), F.NonbondedCutoffSystemForce(lj=("C2", SWITCHON, RC)),
          F.NonbondedPMEwaldSystemForce((GRID,) * 3, RC)]
    md = F.Integrator(topo, fl, timestep=DT_FS)
    md.set_state(box["pos"], box["vel"])
    t, etot = [], []
    for k in range(0, steps + 1, chunk):
        if k:
            md.run(chunk)
        e, kin = md.energies()
        t.append(k * DT_FS * 1e-6)  # ns
        etot.append(float(e[0, :4].sum() + kin[0]))
    pos, vel = md.state()
    md.close()
    topo.close()
    return np.array(t), np.array(etot), pos, vel


def run_nve(args):
    """NVE stability of the 98,304-atom box: energy drift (kcal/mol/ns per degree of freedom,
    least-squares slope of the total energy) in mixed precision and on the plain FP64 path, and
    whether two mixed runs give bit-identical trajectories."""
    import torch
    from protomol3_b200 import forces as F
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    box = workload(0)
    ndof = 3 * len(box["charge"]) - 3
    out = {"mode": "nve", "steps": args.steps, "timestep_fs": DT_FS, "dof": ndof,
           "config": config_dict()}
    runs = {}
    for name, prec in (("mixed", "mixed"), ("mixed_repeat", "mixed"), ("fp64", "fp64")):
        t0 = time.perf_counter()
        t, e, pos, vel = nve_run(F, box, prec, stream, args.steps, args.chunk)
        slope = float(np.polyfit(t, e, 1)[0])
        runs[name] = (pos, vel)
        out[name] = {"drift_kcal_mol_ns_dof": slope / ndof, "e_start": e[0], "e_end": e[-1],
                     "e_std": float(e.std()), "wall_s": time.perf_counter() - t0}
    out["mixed_bit_identical"] = bool(np.array_equal(runs["mixed"][0], runs["mixed_repeat"][0]) and
                                      np.array_equal(runs["mixed"][1], runs["mixed_repeat"][1]))
    d = runs["mixed"][0] - runs["fp64"][0]
    out["mixed_vs_fp64_rms_position_diff_A"] = float(np.sqrt((d ** 2).sum(1).mean()))
    print(json.dumps(out), flush=True)


def run_rigid(args):
    """Rigid water at 2 fs: the 98,304-atom box with the same force set, SHAKE after every drift
    and RATTLE after every step (the reference's defaults: epsilon 1e-5, 30 iterations), in mixed
    precision and on the plain FP64 path.  Steps are timed one by one with CUDA events and an L2
    flush before each, as in the main bench."""
    import torch
    from protomol3_b200 import constraints as CS
    from protomol3_b200 import forces as F
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    box = workload(0)
    cons = CS.rattle_shake_constraints(box)
    dt = 2.0
    out = {"mode": "rigid", "metric": "ns/day at 98k atoms, rigid TIP3P (SHAKE + RATTLE), 2 fs leapfrog",
           "unit": "ns/day", "timestep_fs": dt, "constraints": int(len(cons[0])), "steps": args.steps,
           "warmup": max(3, args.warmup),
           "config": dict(config_dict(), timestep_fs=dt, workload=config_dict()["workload"].replace(
               "leapfrog 1 fs", "rigid waters (SHAKE + RATTLE), leapfrog 2 fs"))}
    clocks = ClockSampler(0)
    for prec in ("mixed", "fp64"):
        topo = F.Topology(box, prec)
        topo.set_stream(stream.cuda_stream)
        fl = [F.BondedSystemForce(), F.NonbondedCutoffSystemForce(lj=("C2", SWITCHON, RC)),
              F.NonbondedPMEwaldSystemForce((GRID,) * 3, RC)]
        md = F.Integrator(topo, fl, timestep=dt)
        md.set_constraints(cons)
        md.set_state(box["pos"], box["vel"])
        for _ in range(max(3, args.warmup)):
            flush.zero_()
            md.run(1)
        torch.cuda.synchronize()
        b0 = topo.list_builds()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps)]
        if prec == "mixed":
            clocks.start()
        for a, b in evs:
            flush.zero_()
            a.record(stream)
            md.run(1)
            b.record(stream)
        torch.cuda.synchronize()
        if prec == "mixed":
            out["clocks"] = clocks.stop()
        ms = sum(a.elapsed_time(b) for a, b in evs) / args.steps
        sweeps = md.constraint_sweeps()
        pos, vel = md.state()
        p = pos.reshape(-1, 3)
        d2 = ((p[cons[1]] - p[cons[0]]) ** 2).sum(1)
        err = float(np.mean(np.abs(d2 - cons[2] ** 2) / (2 * cons[2] ** 2)))
        out[prec] = {"value": 86400.0 * dt * 1e-6 / (ms * 1e-3), "ms_per_step": ms,
                     "list_rebuilds": topo.list_builds() - b0, "last_sweeps_shake_rattle": list(sweeps),
                     "mean_constraint_error": err, "finite": bool(np.isfinite(pos).all())}
        md.close()
        topo.close()
    out["value"] = out["mixed"]["value"]
    out["mixed_over_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    print(json.dumps(out), flush=True)


def run_frames(args):
    """Trajectory output during the run: the 98,304-atom MD step (mixed, 1 fs) timed one by one
    as in the main bench, without output and with a DCD frame taken off the device after every
    step (device snapshot, host copy on the trajectory's own stream, writer thread), plus the
    wall time until the file holds every frame."""
    import tempfile
    import torch
    from protomol3_b200 import forces as F
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    box = workload(0)
    out = {"mode": "frames", "metric": "ms per MD step with a DCD frame every step (98k atoms, mixed)",
           "steps": args.steps, "warmup": max(3, args.warmup), "config": config_dict()}
    tmp = tempfile.mkdtemp()
    for leg in ("no_output", "dcd_every_step"):
        topo = F.Topology(box, "mixed")
        topo.set_stream(stream.cuda_stream)
        fl = [F.BondedSystemForce(), F.NonbondedCutoffSystemForce(lj=("C2", SWITCHON, RC)),
              F.NonbondedPMEwaldSystemForce((GRID,) * 3, RC)]
        md = F.Integrator(topo, fl, timestep=DT_FS)
        md.set_state(box["pos"], box["vel"])
        traj = F.Trajectory.dcd(os.path.join(tmp, "t.dcd"), topo.n_atoms) if leg != "no_output" else None
        for _ in range(max(3, args.warmup)):
            flush.zero_()
            md.run(1)
            if traj:
                md.write_frame(traj)
        if traj:
            traj.flush()
        torch.cuda.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps)]
        t0 = time.perf_counter()
        for a, b in evs:
            flush.zero_()
            a.record(stream)
            md.run(1)
            if traj:
                md.write_frame(traj)
            b.record(stream)
        torch.cuda.synchronize()
        t_dev = time.perf_counter() - t0
        if traj:
            traj.flush()
        t_all = time.perf_counter() - t0
        ms = sum(a.elapsed_time(b) for a, b in evs) / args.steps
        out[leg] = {"ms_per_step": ms, "wall_s_device_done": t_dev, "wall_s_file_done": t_all}
        if traj:
            out[leg]["frames_in_file"] = traj.frames()
            out[leg]["file_bytes"] = os.path.getsize(os.path.join(tmp, "t.dcd"))
            traj.close()
        md.close()
        topo.close()
    out["frame_cost_ms_per_step"] = out["dcd_every_step"]["ms_per_step"] - out["no_output"]["ms_per_step"]
    print(json.dumps(out), flush=True)


def serve_leg(n_requests=24, loads=(0.5, 0.8, 0.95), budget_gb=32.0, max_active=32, chunk=200,
              seed=2024):
    """Serving: Poisson streams of Langevin MD segments (water boxes log-uniform on 500-50,000
    atoms, 1,000-20,000 steps, 300 K, gamma 1/ps, 1 fs, LJ C2 7.5 -> 9 A, PME at ~1 A spacing,
    mixed precision).  Capacity is measured first with every request of the trace present at
    t = 0; then the same request mix is offered at each fraction of that capacity.  Latency is
    arrival to completion (wall clock, includes admission wait); p50/p99 per load.  The server
    folds resident segments of one size class into batched systems (FoldingServer); the capacity
    of one system per segment (MDServer) is reported beside it."""
    from protomol3_b200 import serving as S
    from protomol3_b200 import waterbox as W

    def requests(rate):
        tr = S.poisson_trace(n_requests, rate, seed=seed)
        return [S.SegmentRequest(k, W.water_box(w, seed=seed + k), st, seed=sd, arrival=a)
                for k, (a, w, st, sd) in enumerate(tr)]

    def serve(reqs, precision="mixed", fold=True):
        kind = S.FoldingServer if fold else S.MDServer
        srv = kind(hbm_budget_bytes=int(budget_gb * (1 << 30)), max_active=max_active, chunk=chunk,
                   precision=precision)
        res = srv.run_trace(reqs)
        out = S.latency_summary(res)
        out.update(peak_active=srv.peak_active, peak_booked_gb=srv.peak_used / (1 << 30))
        if fold:
            out.update(cohorts_made=srv.cohorts_made, peak_cohorts=srv.peak_cohorts,
                       peak_device_gb=srv.peak_device / (1 << 30))
        return out

    # warm-up: module load, first graph captures
    S.MDServer(max_active=2, chunk=chunk).run_trace(requests(0.0)[:2])
    S.FoldingServer(max_active=2, chunk=chunk).run_trace(requests(0.0)[:2])
    cap = serve(requests(0.0))
    capacity = cap["throughput_req_s"]
    legs = {"capacity": cap, "capacity_one_system_per_segment": serve(requests(0.0), fold=False)}
    for f in loads:
        legs["load_%02d" % round(100 * f)] = dict(serve(requests(f * capacity)), offered_req_s=f * capacity)
    # the plain FP64 path serving the same request mix, all present at t = 0
    cap64 = serve(requests(0.0), precision="fp64")
    return {"metric": "p50/p99 completion latency of Langevin MD segments (500-50,000 atoms, "
                      "1,000-20,000 steps) under Poisson load",
            "requests_per_load": n_requests, "capacity_req_s": capacity, "loads": legs,
            "plain_fp64_capacity": cap64, "capacity_over_fp64": capacity / cap64["throughput_req_s"],
            "hbm_budget_gb": budget_gb, "max_active": max_active, "chunk_steps": chunk,
            "precision": "mixed", "server": "FoldingServer (size classes < 2,000 / 8,000 / 20,000 atoms)"}


def run_profile(args):
    """A bounded case for ncu: builds the box and evaluates the force set ``--steps`` times
    through the C ABI (no MD loop, no CPU legs)."""
    import torch
    from protomol3_b200 import forces as F
    torch.cuda.set_device(0)
    box = workload(0)
    topo = F.Topology(box, args.precision)
    fl = [F.NonbondedCutoffSystemForce(lj=("C2", SWITCHON, RC)),
          F.NonbondedPMEwaldSystemForce((GRID,) * 3, RC), F.BondedSystemForce()]
    frc = np.zeros((topo.n_atoms, 3))
    for _ in range(args.steps):
        frc[:] = 0.0
        F.evaluate_all(topo, fl, box["pos"], frc, F.ScalarStructure(1))
    print(json.dumps({"mode": "profile", "precision": args.precision, "evaluations": args.steps,
                      "force_rms": float(np.sqrt((frc ** 2).mean()))}))


# ------------------------------------------------------------------------------- reference arm
def run_reference(args, rank, world):
    if rank != 0:
        return
    box = workload(0)
    steps = max(1, min(args.steps, args.ref_steps))
    for _ in range(min(args.warmup, 1)):
        cpu_baseline(box, steps=1)
    base = cpu_baseline(box, steps=steps)[0]
    line = {"metric": "ns/day at 98k atoms (TIP3P, LJ C2 + PME 96^3, 1 fs leapfrog)", "impl": "reference",
            "value": base["value"], "unit": "ns/day", "n_gpus": world, "steps": steps,
            "warmup": min(args.warmup, 1), "ms_per_step": 86400.0 * DT_FS * 1e-6 / base["value"] * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": dict(config_dict(), precision="fp64", parallelism="cpu"),
            "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": "ns/day", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--no-fp64", action="store_true", help="skip the plain FP64 comparison leg")
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--ref-steps", type=int, default=5)
    ap.add_argument("--no-batch", action="store_true", help="skip the 256-box ensemble leg")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving leg")
    ap.add_argument("--no-tune", action="store_true", help="default knobs instead of the autotuner's")
    ap.add_argument("--chunk", type=int, default=500, help="nve: steps between energy reads")
    ap.add_argument("--serve-requests", type=int, default=24, help="serve: requests per load level")
    ap.add_argument("--mode", choices=["bench", "profile", "batch", "nve", "serve", "rigid", "frames"], default="bench",
                    help="profile: only --steps force evaluations (bounded case for ncu); "
                         "batch: only the 256-box ensemble leg; nve: energy drift and "
                         "reproducibility over --steps steps; serve: latency under Poisson load; "
                         "rigid: SHAKE + RATTLE at 2 fs; frames: DCD output every step")
    args = ap.parse_args()
    if args.mode == "rigid":
        run_rigid(args)
        return
    if args.mode == "frames":
        run_frames(args)
        return
    if args.mode == "serve":
        import torch
        torch.cuda.set_device(0)
        print(json.dumps(dict(serve_leg(n_requests=args.serve_requests), mode="serve")), flush=True)
        return
    if args.mode == "nve":
        run_nve(args)
        return
    if args.mode == "profile":
        run_profile(args)
        return
    if args.mode == "batch":
        import torch
        torch.cuda.set_device(0)
        stream = torch.cuda.Stream()
        flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
        print(json.dumps(dict(batch_leg(stream, flush, steps=args.steps, warmup=max(3, args.warmup)),
                              mode="batch")), flush=True)
        return
    if args.warmup < 3:
        args.warmup = 3
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus)))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if "WORLD_SIZE" not in os.environ:
        world = 1
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_b200(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
