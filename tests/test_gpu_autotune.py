"""The batched-path autotuner on the device: the tuned ensemble keeps parity with the oracle box
by box (the tuned PME grids are never coarser than the requested spacing), the speed knobs change
results only by rounding, and a second search of the same workload comes from the cache.

Tolerances as tests/test_gpu_parity.py: mixed 1e-5 relative RMS force against the oracle at the
grid the tuner chose; knobs: FP64 1e-12, mixed 1e-6 between knob settings."""
import numpy as np
import pytest

from oracle import oracle as O
from protomol3_b200 import autotune as AT
from protomol3_b200 import forces as F
from protomol3_b200 import waterbox as W

pytestmark = pytest.mark.gpu


def rel_rms(f, ref):
    return float(np.sqrt(((f - ref) ** 2).sum() / (ref ** 2).sum()))


def ensemble():
    return [W.water_box(n, seed=90 + n) for n in (110, 180, 260, 300, 420, 700)]


def test_tuned_ensemble_keeps_parity_and_caches(tmp_path):
    boxes = ensemble()
    tuner = AT.Autotuner(cache_path=str(tmp_path / "tune.json"), steps=10, warmup=3, class_copies=4)
    res = tuner.tune(boxes, 9.0, 7.5, order=4, precision="mixed")
    assert not res["cached"]
    for b, g in zip(boxes, res["grids"]):
        assert b["box"][0] / g <= 1.0 and g in AT.grid_candidates(b["box"][0])
    assert res["knobs"]["skin"] in AT.SKINS and res["knobs"]["sort_cell"] in AT.SORT_CELLS
    assert res["ms_per_step"] <= res["default_ms_per_step"] * 1.001
    topo, fl = tuner.apply(boxes, res, 9.0, 7.5)
    f = np.zeros((topo.n_atoms, 3))
    F.evaluate_all(topo, fl, topo.positions(), f, F.ScalarStructure(topo.n_boxes))
    off = 0
    for b, g in zip(boxes, res["grids"]):
        n = len(b["charge"])
        fo, _, _, _ = O.evaluate(O.System(b), b["pos"], cutoff=O.cutoff_params(lj=("C2", 7.5, 9.0)),
                                 pme=O.pme_params((g, g, g), 9.0), bonded=True)
        assert rel_rms(f[off:off + n], fo) < 1e-5
        off += n
    topo.close()
    again = AT.Autotuner(cache_path=str(tmp_path / "tune.json")).tune(boxes, 9.0, 7.5, order=4, precision="mixed")
    assert again["cached"] and again["grids"] == res["grids"] and again["knobs"] == res["knobs"]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_knobs_change_only_the_rounding(precision):
    boxes = ensemble()
    grids = [W.pme_grid_for(b["box"][0]) for b in boxes]
    fl = AT.Autotuner.force_list(grids, 9.0, 7.5, 4)
    out = []
    for knobs in ({}, {"skin": 1.1, "sort_cell": 1.8, "pair_ctas_per_sm": 1},
                  {"skin": 0.5, "sort_cell": 3.2, "pair_ctas_per_sm": 2}):
        topo = F.Topology(boxes, precision)
        if knobs:
            topo.set_tuning(**knobs)
            assert topo.tuning() == dict({"skin": 0.8, "sort_cell": 2.4, "pair_ctas_per_sm": 0}, **knobs)
        f = np.zeros((topo.n_atoms, 3))
        F.evaluate_all(topo, fl, topo.positions(), f, F.ScalarStructure(topo.n_boxes))
        out.append(f)
        topo.close()
    tol = 1e-12 if precision == "fp64" else 1e-6
    for f in out[1:]:
        assert rel_rms(f, out[0]) < tol


def test_knob_change_between_md_runs_recaptures_the_step():
    """A tuning change re-sizes the neighbour list; the MD run captured before it captures its
    step again (its graph held the old list's buffers) and goes on as a fresh run would."""
    box = W.water_box(300, seed=5)
    g = W.pme_grid_for(box["box"][0])
    fl = AT.Autotuner.force_list([g], 9.0, 7.5, 4)
    topo = F.Topology(box, "fp64")
    md = F.Integrator(topo, fl, timestep=1.0)
    md.set_state(box["pos"], box["vel"])
    md.run(10)
    topo.set_tuning(skin=1.1, sort_cell=1.8)
    md.run(10)
    p1, v1 = md.state()
    topo2 = F.Topology(box, "fp64")
    md2 = F.Integrator(topo2, AT.Autotuner.force_list([g], 9.0, 7.5, 4), timestep=1.0)
    md2.set_state(box["pos"], box["vel"])
    md2.run(10)
    md2.run(10)
    p2, v2 = md2.state()
    assert np.abs(p1 - p2).max() < 1e-9 and np.abs(v1 - v2).max() < 1e-9
    for m, t in ((md, topo), (md2, topo2)):
        m.close()
        t.close()
