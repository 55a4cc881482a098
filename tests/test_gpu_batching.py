"""A box gives the same bits alone and inside a batch of boxes (one system, one launch per force
stage), and when it moves from one batched run to another part-way.

What makes it so: neighbour-list rebuilds are decided box by box; every box's pair tiles start at
a multiple of the pair kernel's warp assignment, so the kernel's floating-point partial sums are
grouped as when the box is alone; energies are rounded to fixed point term by term; the Langevin
noise of an atom is keyed by its box's seed, its index within the box and its box's step count.
The oracle comparisons of batched systems are in test_gpu_parity.py; here the GPU path is
compared with itself, bit for bit.
"""
import numpy as np
import pytest

from protomol3_b200 import forces as F
from protomol3_b200 import waterbox as W

pytestmark = pytest.mark.gpu

# 100 waters: a 14.4 A edge, under twice the 9 A cutoff (lattice-image kernel instance);
# 257 and 640 waters: 19.7 and 26.8 A
SIZES = (100, 257, 640)


def boxes_and_grids(sizes=SIZES, seed=40):
    boxes = [W.water_box(n, seed=seed + n) for n in sizes]
    return boxes, [W.pme_grid_for(b["box"][0]) for b in boxes]


def force_list(grids):
    return [F.BondedSystemForce(), F.NonbondedCutoffSystemForce(lj=("C2", 7.5, 9.0)),
            F.NonbondedPMEwaldSystemForce((0, 0, 0), 9.0, box_grids=[[g] * 3 for g in grids])]


def slices(boxes):
    off = np.cumsum([0] + [len(b["charge"]) for b in boxes])
    return [slice(off[k], off[k + 1]) for k in range(len(boxes))]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_box_alone_and_in_a_batch_evaluate_bit_for_bit(precision):
    boxes, grids = boxes_and_grids()
    topo = F.Topology(boxes, precision)
    fb = np.zeros((topo.n_atoms, 3))
    eb = F.ScalarStructure(topo.n_boxes, virial=True)
    F.evaluate_all(topo, force_list(grids), np.concatenate([b["pos"] for b in boxes]), fb, eb)
    topo.close()
    for k, (b, g, sl) in enumerate(zip(boxes, grids, slices(boxes))):
        t1 = F.Topology(b, precision)
        f1 = np.zeros((t1.n_atoms, 3))
        e1 = F.ScalarStructure(1, virial=True)
        F.evaluate_all(t1, force_list([g]), b["pos"], f1, e1)
        t1.close()
        assert np.array_equal(fb[sl], f1), k
        assert np.array_equal(eb.table[k], e1.table[0]), k


def run_batch(boxes, grids, precision, steps, kind="langevin", seeds=None):
    topo = F.Topology(boxes, precision)
    md = F.Integrator(topo, force_list(grids), timestep=1.0, kind=kind, temperature=300.0, gamma=5.0)
    if seeds is not None:
        md.set_box_noise(seeds=seeds)
    md.set_state(np.concatenate([b["pos"] for b in boxes]), np.concatenate([b["vel"] for b in boxes]))
    md.run(steps)
    pos, vel = md.state()
    e, kin = md.energies()
    builds = topo.list_builds()
    md.close()
    topo.close()
    return pos, vel, e, kin, builds


@pytest.mark.parametrize("kind", ["leapfrog", "langevin"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_box_alone_and_in_a_batch_run_bit_for_bit(precision, kind):
    """300 steps (the lists of the three boxes are rebuilt at different steps): every box ends in
    the same state, with the same energies, alone and in the batch."""
    boxes, grids = boxes_and_grids()
    seeds = [101, 202, 303]
    pb, vb, eb, kb, builds = run_batch(boxes, grids, precision, 300, kind, seeds)
    assert builds > 2
    for k, (b, g, sl) in enumerate(zip(boxes, grids, slices(boxes))):
        p1, v1, e1, k1, _ = run_batch([b], [g], precision, 300, kind, [seeds[k]])
        assert np.array_equal(pb[sl], p1), k
        assert np.array_equal(vb[sl], v1), k
        assert np.array_equal(eb[k], e1[0]), k
        assert kb[k] == k1[0], k


def test_default_box_seeds_differ_and_start_at_the_runs_seed():
    """Without set_box_noise box b of a run made with seed s draws with s + b (box 0: the
    single-box stream), and every box's step count is the run's."""
    boxes, grids = boxes_and_grids()
    topo = F.Topology(boxes, "mixed")
    md = F.Integrator(topo, force_list(grids), kind="langevin", seed=77)
    seeds, steps = md.box_noise()
    assert seeds.tolist() == [77, 78, 79] and steps.tolist() == [0, 0, 0]
    md.close()
    topo.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_box_moved_between_batches_continues_bit_for_bit(precision):
    """Boxes A, B, C run 120 Langevin steps in one batch; B's state (with its neighbour list's
    reference positions and its noise stream) then moves into a batch with a new box D, where it
    has run 0 steps, and runs 180 more: it ends where B ends after 300 steps of the first batch."""
    boxes, grids = boxes_and_grids()
    seeds = [11, 22, 33]
    sl = slices(boxes)

    topo = F.Topology(boxes, precision)
    md = F.Integrator(topo, force_list(grids), kind="langevin", gamma=5.0)
    md.set_box_noise(seeds=seeds)
    md.set_state(np.concatenate([b["pos"] for b in boxes]), np.concatenate([b["vel"] for b in boxes]))
    md.run(120)
    ck = md.checkpoint()
    bseeds, bsteps = md.box_noise()
    assert bsteps.tolist() == [120, 120, 120]
    md.run(180)
    pb, vb = md.state()
    md.close()
    topo.close()

    d, gd = boxes_and_grids((180,), seed=9)
    pair = [boxes[1], d[0]]
    topo2 = F.Topology(pair, precision)
    md2 = F.Integrator(topo2, force_list([grids[1], gd[0]]), kind="langevin", gamma=5.0)
    n_b, n_d = len(boxes[1]["charge"]), len(d[0]["charge"])
    ckp = {"positions": np.concatenate([ck["positions"][sl[1]], d[0]["pos"]]),
           "velocities": np.concatenate([ck["velocities"][sl[1]], d[0]["vel"]]),
           "list_reference": np.concatenate([ck["list_reference"][sl[1]], d[0]["pos"]]),
           "step": 0}
    md2.restore(ckp)
    md2.set_box_noise(seeds=[bseeds[1], 5], steps=[bsteps[1], 0])
    md2.run(180)
    p2, v2 = md2.state()
    md2.close()
    topo2.close()
    assert np.array_equal(p2[:n_b], pb[sl[1]])
    assert np.array_equal(v2[:n_b], vb[sl[1]])
    assert p2.shape[0] == n_b + n_d


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_langevin_run_split_anywhere_gives_the_same_bits(precision):
    """run(300) and run(120) + run(97) + run(83): a Langevin run's closing and opening half
    kicks are the same operations whether they meet in one step or across two calls, so a
    segment served in chunks of any length ends in the same state."""
    boxes, grids = boxes_and_grids()
    pa, va, ea, ka, _ = run_batch(boxes, grids, precision, 300, "langevin", [7, 8, 9])
    topo = F.Topology(boxes, precision)
    md = F.Integrator(topo, force_list(grids), timestep=1.0, kind="langevin", temperature=300.0, gamma=5.0)
    md.set_box_noise(seeds=[7, 8, 9])
    md.set_state(np.concatenate([b["pos"] for b in boxes]), np.concatenate([b["vel"] for b in boxes]))
    for n in (120, 97, 83):
        md.run(n)
    pb, vb = md.state()
    eb, kb = md.energies()
    md.close()
    topo.close()
    assert np.array_equal(pa, pb) and np.array_equal(va, vb)
    assert np.array_equal(ea, eb) and np.array_equal(ka, kb)
