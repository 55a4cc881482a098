"""Vacuum cutoff forces on the CPU: the oracle with a box that stands in for vacuum against the
reference's own VacuumBoundaryConditions forces (golden fixture tests/golden/vacuum_ref.npz, made
by make_golden_vacuum.py: alanine from the reference's vacuum ConfigTests and a water droplet),
and the box helper of the library.  Tolerance: 1e-12 relative RMS force error and 1e-12 relative
energy (the two codes sum the same pair terms in different orders)."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from protomol3_b200 import forces as F

GOLD = os.path.join(os.path.dirname(__file__), "golden", "vacuum_ref.npz")
SETS = {"lj_c2": (("C2", 8.0, 10.0), None), "lj_c1": (("C1", 0.0, 10.0), None),
        "coul_cut": (None, ("cutoff", 0.0, 10.0)), "lj_c2_coul_c2": (("C2", 8.0, 10.0), ("C2", 8.0, 10.0)),
        "lj_c2_coul_c1": (("C2", 8.0, 10.0), ("C1", 0.0, 10.0))}
CASES = [("ala", k) for k in ("lj_c2", "lj_c1", "coul_cut", "lj_c2_coul_c2")] + [("drop", "lj_c2_coul_c1")]


def topo(g, tag, margin=10.8):
    t = {k: g[tag + "_" + k] for k in ("type", "charge", "mass", "lj", "excl_pairs", "excl_kind", "molecule", "pos")}
    t["box"] = F.vacuum_box(t["pos"], margin)
    t["origin"] = np.zeros(3)
    t["coulomb_scaling"] = 1.0
    return t


def rel_rms(a, b):
    return np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum())


@pytest.mark.parametrize("tag,name", CASES)
def test_oracle_in_a_vacuum_box_equals_reference(tag, name):
    g = np.load(GOLD)
    t = topo(g, tag)
    lj, coul = SETS[name]
    f, e, _, _ = O.evaluate(O.System(t), t["pos"], cutoff=O.cutoff_params(lj=lj, coul=coul))
    ref_f, ref_e = g["%s_%s_forces" % (tag, name)], g["%s_%s_energies" % (tag, name)]
    assert rel_rms(f, ref_f) < 1e-12
    assert np.allclose(e[:2], ref_e[:2], rtol=1e-12, atol=1e-12)


def test_vacuum_box_edges():
    p = np.array([[0.0, 0.0, 0.0], [3.0, -1.0, 2.0], [1.0, 4.0, -2.0]])
    e = F.vacuum_box(p, margin=2.0)
    assert np.allclose(e, [2 * (3 + 2) + 1, 2 * (5 + 2) + 1, 2 * (4 + 2) + 1])
    with pytest.raises(RuntimeError):
        F.vacuum_box(p, margin=-1.0)


@pytest.mark.skipif(not O.ref_md_available(), reason="reference vacuum forces not compiled here")
def test_live_reference_equals_fixture():
    g = np.load(GOLD)
    t = topo(g, "ala")
    f, e, _ = O.ref_evaluate_vacuum(O.System(t), t["pos"], O.cutoff_params(lj=("C2", 8.0, 10.0)))
    assert np.array_equal(f, g["ala_lj_c2_forces"]) and np.array_equal(e, g["ala_lj_c2_energies"])
