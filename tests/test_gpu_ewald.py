"""The exact Ewald reciprocal sum on the device (pmb_ewald_reciprocal) against the reference's
own NonbondedFullEwaldSystemForce (reciprocal term only; golden fixture, see test_ewald.py), and
the PME reciprocal term checked against it.  Tolerances: 1e-10 relative RMS force error, energy
and virial against the reference (sines and cosines formed directly rather than by the
reference's recurrences); PME at order 8 on a fine grid within 1e-5 relative of the exact sum
(the PME approximation itself)."""
import os

import numpy as np
import pytest

from protomol3_b200 import forces as F
from protomol3_b200 import waterbox as W

from test_ewald import CASES, GOLD

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tag", list(CASES))
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_ewald_equals_reference(tag, precision):
    g = np.load(GOLD)
    nw, seed, alpha, acc = CASES[tag]
    box = W.water_box(nw, seed=seed)
    topo = F.Topology(box, precision)  # the check path is FP64 in either system
    frc = np.zeros((topo.n_atoms, 3))
    en = F.ScalarStructure(1, virial=True)
    F.ewald_reciprocal(topo, box["pos"], frc, en, alpha=alpha, accuracy=acc)
    ref = g[tag + "_forces"]
    assert np.sqrt(((frc - ref) ** 2).sum() / (ref ** 2).sum()) < 1e-10
    assert abs(en[F.ScalarStructure.COULOMB] - g[tag + "_energy"]) < 1e-10 * abs(g[tag + "_energy"])
    assert np.allclose(en.virial().ravel(), g[tag + "_virial"], rtol=1e-9, atol=1e-9)
    topo.close()


def test_pme_reciprocal_against_exact_ewald():
    box = W.water_box(216, seed=4)
    topo = F.Topology(box, "fp64")
    fe = np.zeros((topo.n_atoms, 3))
    ee = F.ScalarStructure(1)
    F.ewald_reciprocal(topo, box["pos"], fe, ee, alpha=0.35, accuracy=1e-12)
    pme = F.NonbondedPMEwaldSystemForce((48, 48, 48), 9.0, order=8, alpha=0.35, real=False, reciprocal=True,
                                        correction=False)
    fp = np.zeros((topo.n_atoms, 3))
    ep = F.ScalarStructure(1)
    pme.evaluate(topo, box["pos"], fp, ep)
    assert np.sqrt(((fp - fe) ** 2).sum() / (fe ** 2).sum()) < 1e-5
    assert abs(ep[F.ScalarStructure.COULOMB] - ee[F.ScalarStructure.COULOMB]) < 1e-5 * abs(ee[F.ScalarStructure.COULOMB])
    topo.close()
