"""Autotuner of the batched path: picks, per workload, the speed knobs of a system of many
independent boxes and the PME grid of each box-size class, timing every candidate on the device.

The reference has no counterpart: its PME grid is set by hand (``-gridsize``,
mdl/interface/force/nonbonded/NonbondedPMEwaldSystemForce.h:1006-1008) and its cell size is
fixed by CubicCellManager (topology/CubicCellManager.cpp:53-59).  Nothing tuned here changes
which pairs are evaluated or lowers the accuracy:

* PME grid per size class (boxes whose smallest 2/3/5-smooth grid at the requested spacing is
  the same): candidates are the 2/3/5-smooth sizes from that one up to ``grid_headroom`` larger,
  never coarser than the requested spacing (a finer grid only lowers the reciprocal-space
  error).  Each candidate is timed on a batch of copies of the class's representative box, PME
  alone (spread, transforms, gather: stage times of ``pmb_profile`` with the L2 flushed), and
  the fastest is kept.  The B-spline order stays the configured one.
* System knobs (``pmb_tuning``): the Verlet skin (list size against rebuild frequency), the
  smallest sort-cell edge (how compact the 8-atom clusters are) and the pair kernel's resident
  CTAs per SM (room for the PME kernels that run beside it), by coordinate descent on the mean
  device time of whole MD steps (``pmb_md_time``) after a warm-up.
* The pair kernel's tile shape (8-atom clusters against 32-atom j-tiles) is fixed by its design;
  the knobs above are what a run can change.

Results are cached per workload signature (box sizes, cutoffs, order, precision) in memory and,
given ``cache_path``, in a JSON file, so that a second run of the same ensemble skips the search.
"""
import hashlib
import json
import os
import time

import numpy as np

from . import forces as F
from . import waterbox as W

SKINS = (0.4, 0.5, 0.8, 1.1)  # the FP64 path prefers the smaller skins, the mixed one 0.7-1.0
SORT_CELLS = (1.8, 2.4, 3.2)
# pair-kernel blocks per SM: all that fit (0; 5 of 128 threads for the mixed kernel), or fewer to
# leave room for the PME kernels that run beside it
PAIR_CTAS = (0, 4, 3)


def grid_candidates(edge, spacing=1.0, headroom=0.15, minimum=8):
    """2/3/5-smooth grid sizes n with edge / n <= spacing, from the smallest up to
    (1 + headroom) times it."""
    n0 = W.fft_friendly(max(minimum, edge / spacing))
    out, n = [], n0
    while n <= n0 * (1.0 + headroom) + 1e-9:
        out.append(n)
        n = W.fft_friendly(n + 1)
    return out


class Autotuner:
    """``tune(boxes, ...)`` returns the chosen PME grid per box and the system knobs; ``apply``
    creates the tuned system and force list."""

    def __init__(self, cache_path=None, spacing=1.0, grid_headroom=0.15, steps=30, warmup=10,
                 class_copies=8, verbose=False):
        self.cache_path = cache_path
        self.spacing = spacing
        self.grid_headroom = grid_headroom
        self.steps = steps
        self.warmup = warmup
        self.class_copies = class_copies
        self.verbose = verbose
        self._cache = {}
        if cache_path and os.path.exists(cache_path):
            with open(cache_path) as fh:
                self._cache = json.load(fh)

    # ------------------------------------------------------------------ workload and forces
    @staticmethod
    def force_list(grids, rc, switchon, order):
        """Bonded terms, LJ C2 (switchon -> rc) and PME (rc, per-box grids, order)."""
        return [F.BondedSystemForce(), F.NonbondedCutoffSystemForce(lj=("C2", switchon, rc)),
                F.NonbondedPMEwaldSystemForce((0, 0, 0), rc, order=order, box_grids=[[g] * 3 for g in grids])]

    @staticmethod
    def signature(boxes, rc, switchon, order, precision):
        h = hashlib.sha1()
        for b in boxes:
            h.update(np.asarray(b["box"], np.float64).tobytes())
            h.update(np.int64(len(b["charge"])).tobytes())
        h.update(np.array([rc, switchon, order], np.float64).tobytes())
        h.update(precision.encode())
        return h.hexdigest()

    # ------------------------------------------------------------------ measurements
    def _md_ms(self, boxes, grids, rc, switchon, order, precision, knobs, stream=None):
        topo = F.Topology(boxes, precision)
        if stream is not None:
            topo.set_stream(stream)
        topo.set_tuning(**knobs)
        md = F.Integrator(topo, self.force_list(grids, rc, switchon, order), timestep=1.0)
        pos = np.concatenate([b["pos"] for b in boxes])
        vel = np.concatenate([b["vel"] for b in boxes])
        md.set_state(pos, vel)
        md.time_steps(self.warmup)
        ms = md.time_steps(self.steps)
        md.close()
        topo.close()
        return ms

    def _descend(self, measure):
        """Coordinate descent over the system knobs from the defaults; a change is kept only
        when it is clearly (0.5%) faster."""
        knobs = {"skin": 0.8, "sort_cell": 2.4, "pair_ctas_per_sm": 0}
        trials = []

        def timed(kn):
            ms = measure(kn)
            trials.append(dict(kn, ms_per_step=ms))
            if self.verbose:
                print("autotune", kn, "%.4f ms" % ms, flush=True)
            return ms
        best = timed(knobs)
        for name, values in (("skin", SKINS), ("sort_cell", SORT_CELLS), ("pair_ctas_per_sm", PAIR_CTAS)):
            for v in values:
                if v == knobs[name]:
                    continue
                kn = dict(knobs, **{name: v})
                ms = timed(kn)
                if ms < best * 0.995:
                    best, knobs = ms, kn
        return knobs, best, trials

    def tune_knobs(self, boxes, grids, rc, switchon, order=4, precision="mixed", stream=None):
        """The system knobs alone, for fixed PME grids (e.g. one large box), by whole MD steps."""
        key = "knobs:" + self.signature(boxes, rc, switchon, order, precision) + ":" + ",".join(map(str, grids))
        if key in self._cache:
            return dict(self._cache[key], cached=True)
        t0 = time.perf_counter()
        knobs, best, trials = self._descend(
            lambda kn: self._md_ms(boxes, grids, rc, switchon, order, precision, kn, stream))
        out = {"knobs": knobs, "ms_per_step": best, "default_ms_per_step": trials[0]["ms_per_step"],
               "trials": trials, "search_s": time.perf_counter() - t0}
        self._cache[key] = out
        self._save()
        return dict(out, cached=False)

    def _save(self):
        if self.cache_path:
            with open(self.cache_path, "w") as fh:
                json.dump(self._cache, fh)

    def _pme_ms(self, box, grid, rc, order, precision):
        """PME (spread + transforms + gather) of ``class_copies`` copies of one box in one
        batched system, per copy, L2 flushed before each repetition."""
        copies = [box] * self.class_copies
        topo = F.Topology(copies, precision)
        pme = F.NonbondedPMEwaldSystemForce((0, 0, 0), rc, order=order, box_grids=[[grid] * 3] * len(copies))
        st = F.profile(topo, [pme], positions=topo.positions(), nrep=5, flush_l2=True)
        topo.close()
        return sum(st.get(k, 0.0) for k in ("pme_spread", "pme_fft", "pme_gather")) / len(copies)

    # ------------------------------------------------------------------ search
    def tune(self, boxes, rc, switchon, order=4, precision="mixed"):
        key = self.signature(boxes, rc, switchon, order, precision)
        if key in self._cache:
            out = dict(self._cache[key], cached=True)
            return out
        t0 = time.perf_counter()
        # PME grid per size class
        classes = {}
        for k, b in enumerate(boxes):
            cand = grid_candidates(b["box"][0], self.spacing, self.grid_headroom)
            classes.setdefault(cand[0], {"boxes": [], "candidates": cand})["boxes"].append(k)
        class_choice, class_times = {}, {}
        for n0, c in sorted(classes.items()):
            rep = boxes[c["boxes"][len(c["boxes"]) // 2]]
            if len(c["candidates"]) == 1:
                class_choice[n0] = n0
                continue
            times = {g: self._pme_ms(rep, g, rc, order, precision) for g in c["candidates"]}
            class_times[n0] = times
            class_choice[n0] = min(times, key=times.get)
        grids = [0] * len(boxes)
        for n0, c in classes.items():
            for k in c["boxes"]:
                grids[k] = class_choice[n0]
        # system knobs, coordinate descent from the defaults
        knobs, best, trials = self._descend(
            lambda kn: self._md_ms(boxes, grids, rc, switchon, order, precision, kn))
        out = {"grids": grids, "knobs": knobs, "ms_per_step": best,
               "default_ms_per_step": trials[0]["ms_per_step"],
               "classes": {str(n0): {"boxes": len(c["boxes"]), "candidates": c["candidates"],
                                      "chosen": class_choice[n0],
                                      "pme_ms_per_box": {str(g): t for g, t in class_times.get(n0, {}).items()}}
                           for n0, c in sorted(classes.items())},
               "trials": trials, "search_s": time.perf_counter() - t0}
        self._cache[key] = out
        self._save()
        return dict(out, cached=False)

    def apply(self, boxes, result, rc, switchon, order=4, precision="mixed"):
        """A system of ``boxes`` with the tuned knobs and the force list with the tuned grids."""
        topo = F.Topology(boxes, precision)
        topo.set_tuning(**result["knobs"])
        return topo, self.force_list(result["grids"], rc, switchon, order)
