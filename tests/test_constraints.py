"""SHAKE / RATTLE on the CPU: the host constraint-list builder and the oracle's constrained
leapfrog against the reference's own LeapfrogIntegrator, ModifierShake and ModifierRattle.

Golden fixture (tests/golden/water64_rigid_ref.npz, made by make_golden_constraints.py from the
reference compiled in place): 64 rigid TIP3P waters, no force terms, 2 fs steps, four modifier
settings.  Tolerance: exact equality (the restatement performs the reference's operations in
its order, and no force term enters)."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from protomol3_b200 import constraints as CS
from protomol3_b200 import waterbox as W

GOLD = os.path.join(os.path.dirname(__file__), "golden", "water64_rigid_ref.npz")
CASES = ("sr", "s", "r", "tight")


def _opt(a):
    return None if a[1] == 0 else (float(a[0]), int(a[1]))


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def test_fixture_inputs_are_the_generator_output(gold):
    box = W.water_box(64, seed=7)
    assert np.array_equal(box["pos"], gold["pos0"]) and np.array_equal(box["vel"], gold["vel0"])


def test_constraint_list_matches_reference_builder(gold):
    a1, a2, ln = CS.rattle_shake_constraints(W.water_box(64, seed=7))
    assert np.array_equal(a1, gold["con_a1"]) and np.array_equal(a2, gold["con_a2"])
    assert np.array_equal(ln, gold["con_len"])
    assert len(a1) == 3 * 64  # every water rigid: H-H, H1-O, H2-O


@pytest.mark.parametrize("case", CASES)
def test_oracle_equals_reference_run(gold, case):
    box = W.water_box(64, seed=7)
    cons = CS.rattle_shake_constraints(box)
    vir = np.zeros(9)
    pos, vel, _, _ = O.leapfrog_constrained(O.System(box), gold["pos0"], gold["vel0"], float(gold["dt"]),
                                            int(gold[case + "_steps"]), cons,
                                            shake=_opt(gold[case + "_shake"]),
                                            rattle=_opt(gold[case + "_rattle"]), rattle_virial=vir)
    assert np.array_equal(pos, gold[case + "_pos"])
    assert np.array_equal(vel, gold[case + "_vel"])
    # the constraint virial the reference's energies hold after the run: the last RATTLE's
    # (ModifierRattle.cpp:58; SHAKE's terms, ModifierShake.cpp:65-68, are cleared by the force
    # evaluation after each drift, so a SHAKE-only run reports none)
    assert np.array_equal(vir, gold[case + "_virial"])


def test_oracle_langevin_equals_reference_run(gold):
    """LangevinLeapfrogIntegrator with SHAKE and RATTLE at temperature 0 (gamma 50/ps): the
    oracle's restatement equals the reference's run bit for bit."""
    box = W.water_box(64, seed=7)
    cons = CS.rattle_shake_constraints(box)
    vir = np.zeros(9)
    pos, vel, _, _ = O.langevin_constrained(O.System(box), gold["pos0"], gold["vel0"], float(gold["dt"]),
                                            int(gold["lv_steps"]), cons, 0.0, float(gold["lv_gamma"]),
                                            rattle_virial=vir)
    assert np.array_equal(pos, gold["lv_pos"])
    assert np.array_equal(vel, gold["lv_vel"])
    assert np.array_equal(vir, gold["lv_virial"])


def test_planted_mistake_is_caught(gold):
    """A rest length off by one part in 10^12 in the oracle's input must break exact equality."""
    box = W.water_box(64, seed=7)
    a1, a2, ln = CS.rattle_shake_constraints(box)
    ln = ln.copy()
    ln[0] *= 1 + 1e-12
    pos, vel, _, _ = O.leapfrog_constrained(O.System(box), gold["pos0"], gold["vel0"], 2.0, 20, (a1, a2, ln))
    assert not np.array_equal(pos, gold["sr_pos"])


def test_constraints_hold_after_the_run(gold):
    """Rigid geometry within the SHAKE tolerance: mean |d^2 - l^2| / (2 l^2) <= 1e-5."""
    a1, a2, ln = gold["con_a1"], gold["con_a2"], gold["con_len"]
    p = gold["sr_pos"].reshape(-1, 3)
    d2 = ((p[a2] - p[a1]) ** 2).sum(1)
    assert np.mean(np.abs(d2 - ln ** 2) / (2 * ln ** 2)) <= 1e-5
    # RATTLE: bond vectors and relative velocities orthogonal within its tolerance
    v = gold["sr_vel"].reshape(-1, 3)
    assert np.mean(np.abs(((p[a1] - p[a2]) * (v[a1] - v[a2])).sum(1))) <= 1e-5


def test_builder_adds_other_hydrogen_bonds_with_all():
    """Non-water X-H bonds join the list only with ``all`` (TopologyUtilities.cpp:754-772)."""
    topo = {"elem": "CHHHOHH", "bonds": np.array([[0, 1], [0, 2], [0, 3], [4, 5], [4, 6]]),
            "bond_r0": np.array([1.09, 1.1, 1.11, 0.9572, 0.9572]),
            "angles": np.array([[5, 4, 6], [1, 0, 2]]), "angle_theta0": np.array([1.8242, 1.9])}
    a1, a2, ln = CS.rattle_shake_constraints(topo, all_bonds=True)
    assert list(zip(a1, a2)) == [(5, 6), (5, 4), (6, 4), (0, 1), (0, 2), (0, 3)]
    a1, a2, ln = CS.rattle_shake_constraints(topo, all_bonds=False)
    assert list(zip(a1, a2)) == [(5, 6), (5, 4), (6, 4)]


@pytest.mark.skipif(not O.ref_md_available(), reason="reference integrator not compiled here")
def test_oracle_equals_live_reference_on_another_box():
    box = W.water_box(100, seed=11)
    system = O.System(box)
    pos_r, vel_r, cons_r = O.ref_leapfrog_constrained(system, box["elem"], box["pos"], box["vel"], 1.5, 12)
    cons = CS.rattle_shake_constraints(box)
    assert all(np.array_equal(x, y) for x, y in zip(cons, cons_r))
    pos, vel, _, _ = O.leapfrog_constrained(system, box["pos"], box["vel"], 1.5, 12, cons)
    assert np.array_equal(pos, pos_r) and np.array_equal(vel, vel_r)
