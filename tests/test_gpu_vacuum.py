"""Vacuum cutoff forces on the device (a box of pmb_vacuum_box edges, vacuum checks on) against
the reference's own VacuumBoundaryConditions forces (golden fixture, see test_vacuum.py).
Tolerance: FP64 path 1e-12 relative RMS force error, energies within 1e-9 relative plus
n_atoms x 2^-31 kcal/mol (the energies accumulate in fixed point, at most 2^-33 kcal/mol per
partial sum; the allowance of the periodic parity tests); mixed path 1e-5 relative RMS force
error and energies within 1e-5 of max(|E|, n_atoms) kcal/mol (a total such as the droplet's
Coulomb energy cancels pair terms of about 1 kcal/mol per atom, so its error scales with the
atoms, not with the total)."""
import os

import numpy as np
import pytest

from protomol3_b200 import forces as F

from test_vacuum import CASES, GOLD, SETS, rel_rms, topo

pytestmark = pytest.mark.gpu
TOL = {"fp64": (1e-12, 1e-9, 2.0 ** -31), "mixed": (1e-5, 1e-5, 0.0)}


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("tag,name", CASES)
def test_device_vacuum_equals_reference(tag, name, precision):
    g = np.load(GOLD)
    t = topo(g, tag)
    lj, coul = SETS[name]
    tp = F.Topology(t, precision)
    tp.set_vacuum()
    force = F.NonbondedCutoffSystemForce(lj=lj, coulomb=coul)
    frc = np.zeros((tp.n_atoms, 3))
    en = F.ScalarStructure(1)
    force.evaluate(tp, t["pos"], frc, en)
    ref_f, ref_e = g["%s_%s_forces" % (tag, name)], g["%s_%s_energies" % (tag, name)]
    ftol, etol, eabs = TOL[precision]
    assert rel_rms(frc, ref_f) < ftol
    for slot, k in ((F.ScalarStructure.COULOMB, 0), (F.ScalarStructure.LENNARDJONES, 1)):
        scale = max(abs(ref_e[k]), 1.0 if precision == "fp64" else float(tp.n_atoms))
        assert abs(en[slot] - ref_e[k]) <= etol * scale + eabs * tp.n_atoms
    tp.close()


def test_spread_beyond_half_an_edge_is_refused():
    g = np.load(GOLD)
    t = topo(g, "ala", margin=0.0)
    tp = F.Topology(t, "fp64")
    tp.set_vacuum()
    force = F.NonbondedCutoffSystemForce(lj=("C2", 8.0, 10.0))
    pos = t["pos"].copy()
    pos[0, 0] += 0.5 * t["box"][0]
    with pytest.raises(RuntimeError):
        force.evaluate(tp, pos, np.zeros_like(pos), F.ScalarStructure(1))
    tp.close()


def test_md_in_vacuum_refuses_atoms_spread_over_half_an_edge():
    """Device-resident MD in a vacuum box: a run whose atoms stay together goes on; once an
    atom flies off beyond half an edge from the others, the device's extent check stops the
    run's results with PMB_ERR_STATE (the minimal image would no longer be the plain
    difference)."""
    from protomol3_b200 import _lib as L
    g = np.load(GOLD)
    t = topo(g, "ala", margin=2.0)
    force = F.NonbondedCutoffSystemForce(lj=("C2", 8.0, 10.0), coulomb=("C2", 8.0, 10.0))
    for fly in (False, True):
        tp = F.Topology(t, "fp64")
        tp.set_vacuum()
        md = F.Integrator(tp, [F.BondedSystemForce(), force], timestep=1.0)
        vel = np.zeros_like(t["pos"])
        if fly:
            vel[0, 0] = 5.0  # A per internal time unit: ~0.1 A per fs, far past the margin in 100 fs
        md.set_state(t["pos"], vel)
        if fly:
            with pytest.raises(L.PMBError) as err:
                md.run(200)
                md.state()
            assert err.value.code == L.PMB_ERR_STATE and "vacuum" in str(err.value)
        else:
            md.run(50)
            pos, _ = md.state()
            assert np.isfinite(pos).all()
        md.close()
        tp.close()
