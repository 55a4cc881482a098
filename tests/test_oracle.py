"""The CPU oracle against the reference's golden vectors and the reference's own compiled code.

Golden vectors (tests/golden, made by tests/golden/make_golden.py from the reference's test data):
  * water_CHARMM_PERIODIC_L: forces at step 0 and 200, positions and velocities after 200
    leapfrog steps, energies -- compared at ProtoMol's own tolerance of 1e-5 (test/test.py:14);
  * EnergiesTest: step-0 Lennard-Jones energy of 320 united-atom pentanes (C2, 8 -> 9 A).
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from protomol3_b200 import waterbox as W

GOLD = os.path.join(os.path.dirname(__file__), "golden")
EPS = 1e-5  # test/test.py:14 DEFAULT_EPSILON


def load(name):
    return dict(np.load(os.path.join(GOLD, name)))


def test_water423_step0_forces_and_energies():
    d = load("water423_periodic.npz")
    s = O.System(d)
    cp = O.cutoff_params(lj=("C2", 0.1, 6.5), coul=("C1", 0.0, 6.5))
    f, e, _, _ = O.evaluate(s, d["pos"], cutoff=cp, bonded=True)
    assert np.abs(f - d["exp_forces0"]).max() < EPS
    # energy file columns: time PE KE TE T bond angle dihedral improper LJ Coulomb ...
    row = d["exp_energy"][0]
    np.testing.assert_allclose(e[[O.E_BOND, O.E_ANGLE, O.E_LJ, O.E_COULOMB]],
                               row[[5, 6, 9, 10]], atol=EPS * 10, rtol=1e-7)


def test_water423_leapfrog_200_steps():
    d = load("water423_periodic.npz")
    s = O.System(d)
    cp = O.cutoff_params(lj=("C2", 0.1, 6.5), coul=("C1", 0.0, 6.5))
    pos, vel, f, e = O.leapfrog(s, d["pos"], d["vel"], 0.5, 200, cutoff=cp)
    assert np.abs(pos - d["exp_pos"]).max() < EPS
    assert np.abs(vel - d["exp_vel"]).max() < EPS
    assert np.abs(f - d["exp_forces_end"]).max() < EPS
    row = d["exp_energy"][1]
    np.testing.assert_allclose(e[[O.E_BOND, O.E_ANGLE, O.E_LJ, O.E_COULOMB]],
                               row[[5, 6, 9, 10]], atol=EPS * 10, rtol=1e-7)


def test_pentane_lj_c2_energy():
    d = load("pentane320_periodic.npz")
    s = O.System(d)
    _, e, _, _ = O.evaluate(s, d["pos"], cutoff=O.cutoff_params(lj=("C2", 8.0, 9.0)))
    assert abs(e[O.E_LJ] - d["exp_lj_energy0"]) < 1e-5


def test_alpha_bisection():
    # erfc(alpha rc)/rc = 1e-6 at rc = 10 A gives alpha ~ 0.312 (the 98,304-atom workload)
    a = O.pme_alpha(10.0, 1e-6)
    assert 0.31 < a < 0.315


def test_planted_mistake_is_caught():
    """A sign error planted in the oracle's output must fail the golden comparison."""
    d = load("water423_periodic.npz")
    s = O.System(d)
    cp = O.cutoff_params(lj=("C2", 0.1, 6.5), coul=("C1", 0.0, 6.5))
    f, _, _, _ = O.evaluate(s, d["pos"], cutoff=cp, bonded=True)
    f[7, 1] = -f[7, 1]
    assert np.abs(f - d["exp_forces0"]).max() > EPS


needs_ref = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")


@needs_ref
@pytest.mark.parametrize("nw,grid,rc,order", [(216, (20,) * 3, 8.0, 4), (60, (12,) * 3, 9.0, 4),
                                              (216, (25, 18, 32), 8.0, 6), (216, (27, 16, 30), 8.0, 8)])
def test_oracle_matches_reference_pme(nw, grid, rc, order):
    b = W.water_box(nw, seed=11)
    s = O.System(b)
    pm = O.pme_params(grid, rc, order=order)
    f, e, v, _ = O.evaluate(s, b["pos"], pme=pm, virial=True)
    fr, er, vr = O.ref_evaluate(s, b["pos"], pme=pm, virial=True)
    assert np.sqrt(((f - fr) ** 2).sum() / (fr ** 2).sum()) < 1e-12
    assert abs(e[0] - er[0]) < 1e-9 * abs(er[0]) + 1e-9
    assert np.abs(v - vr).max() < 1e-8


@needs_ref
def test_oracle_matches_reference_cutoff():
    b = W.water_box(216, seed=3)
    s = O.System(b)
    cp = O.cutoff_params(lj=("C2", 7.0, 8.0), coul=("C2", 7.0, 8.0))
    f, e, v, _ = O.evaluate(s, b["pos"], cutoff=cp, bonded=True, virial=True)
    fr, er, vr = O.ref_evaluate(s, b["pos"], cutoff=cp, bonded=True, virial=True)
    assert np.abs(f - fr).max() < 1e-10
    np.testing.assert_allclose(e, er, rtol=1e-12, atol=1e-9)


@needs_ref
@pytest.mark.parametrize("nw", [100, 150, 190])
def test_oracle_matches_reference_small_box_lj(nw):
    """Boxes whose edge is under twice the cutoff (14.4-17.2 A against 2 x 9 A; about 5% of the
    ensemble workload's boxes): the reference's cutoff LJ takes one minimal image per pair
    (force/OneAtomPair.h:55-57) while its PME real term sums lattice images; the oracle follows
    both."""
    b = W.water_box(nw, seed=50 + nw)
    assert b["box"][0] < 18.0
    s = O.System(b)
    cp = O.cutoff_params(lj=("C2", 7.5, 9.0))
    grid = (W.pme_grid_for(b["box"][0]),) * 3
    pm = O.pme_params(grid, 9.0)
    f, e, v, _ = O.evaluate(s, b["pos"], cutoff=cp, pme=pm, bonded=True, virial=True)
    fr, er, vr = O.ref_evaluate(s, b["pos"], cutoff=cp, pme=pm, bonded=True, virial=True)
    assert np.sqrt(((f - fr) ** 2).sum() / (fr ** 2).sum()) < 1e-12
    np.testing.assert_allclose(e, er, rtol=1e-12, atol=1e-9)
    assert np.abs(v - vr).max() < 1e-8 * np.abs(vr).max()


def charged_box(nw=216, seed=13):
    """A water box with a net charge: the first water's hydrogens lose their charge
    (total charge -0.834 e)."""
    b = dict(W.water_box(nw, seed=seed))
    q = b["charge"].copy()
    q[1] = q[2] = 0.0
    b["charge"] = q
    return b


def test_charged_box_charged_term():
    """The charged-system term of NonbondedPMEwaldSystemForce::initialize
    (mdl/interface/force/nonbonded/NonbondedPMEwaldSystemForce.h:555-575): -pi (sum q)^2 /
    (2 V alpha^2), present only when |sum q * 0.00268283| > 1e-5."""
    b = charged_box()
    s = O.System(b)
    pm = O.pme_params((20, 20, 20), 8.0)
    _, _, _, info = O.evaluate(s, b["pos"], pme=pm)
    qs, a, V = b["charge"].sum(), info["alpha"], np.prod(b["box"])
    assert abs(qs * 0.00268283) > 1e-5
    assert info["terms"][4] == pytest.approx(-np.pi * qs * qs / (2 * V * a * a), rel=1e-14)
    _, _, _, info0 = O.evaluate(O.System(W.water_box(216, seed=13)), b["pos"], pme=pm)
    assert info0["terms"][4] == 0.0


@needs_ref
def test_oracle_matches_reference_charged_box():
    b = charged_box()
    s = O.System(b)
    pm = O.pme_params((20, 20, 20), 8.0)
    f, e, v, _ = O.evaluate(s, b["pos"], pme=pm, virial=True)
    fr, er, vr = O.ref_evaluate(s, b["pos"], pme=pm, virial=True)
    assert np.sqrt(((f - fr) ** 2).sum() / (fr ** 2).sum()) < 1e-12
    assert abs(e[0] - er[0]) < 1e-12 * abs(er[0])
    assert np.abs(v - vr).max() < 1e-8
