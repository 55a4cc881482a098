"""The oracle's integrators against ProtoMol's own LeapfrogIntegrator and
LangevinLeapfrogIntegrator, run with force terms (golden fixture tests/golden/water216_md_ref.npz,
made by tests/golden/make_golden_md.py from the reference compiled in place; and the compiled
reference itself, oracle/_ref, where it is present).

The system is the 216-water plain-method workload: LJ + Coulomb cutoff with C2 switching
7 -> 8 A, bonds and angles, 1 fs.  Two FP64 programs that sum the same forces in different orders
follow the same trajectory only for a while: water is chaotic, and the oracle's and the
reference's positions, equal to 1e-15 after one step, differ by ~1e-9 A after 100 steps and by
whole angstroms after 300.  So trajectories are compared over the first 100 steps with bounds
that grow with the step, and the 1,000-step run is compared step by step: the forces and
energies of both programs on the reference's own positions of every step.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")
# max |x - x_ref| (A) allowed after k steps of a free-running FP64 trajectory; measured 7e-15,
# 1.4e-12 and 1.0e-9 for the oracle at 10, 50 and 100 steps
TRAJ_TOL = {10: 1e-12, 50: 1e-10, 100: 1e-8}


def load():
    return dict(np.load(os.path.join(GOLD, "water216_md_ref.npz")))


def system(d):
    from protomol3_b200 import waterbox as W
    box = W.water_box(216, seed=1234)
    assert np.array_equal(box["pos"], d["pos0"]) and np.array_equal(box["vel"], d["vel0"])
    return box, O.System(box)


def cutoff():
    return O.cutoff_params(lj=("C2", 7.0, 8.0), coul=("C2", 7.0, 8.0))


def rel(a, b):
    return np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum())


def test_leapfrog_run1_steps_match_reference():
    """LeapfrogIntegrator stepped by run(1): energies of every step and positions/velocities
    after 10, 50 and 100 steps."""
    d = load()
    box, s = system(d)
    pos, vel = box["pos"].copy(), box["vel"].copy()
    f0, e0, _, _ = O.evaluate(s, pos, cutoff=cutoff(), bonded=True)
    assert rel(f0, d["lf_forces"][0]) < 1e-13
    np.testing.assert_allclose(e0, d["lf_energies"][0], rtol=1e-13)
    keep = list(d["lf_keep"])
    for k in range(1, 101):
        pos, vel, f, e = O.leapfrog(s, pos, vel, 1.0, 1, cutoff=cutoff())
        np.testing.assert_allclose(e, d["lf_energies"][k], rtol=1e-10, atol=1e-9)
        if k in keep:
            j = keep.index(k)
            assert np.abs(pos - d["lf_pos"][j]).max() < TRAJ_TOL[k]
            assert np.abs(vel - d["lf_vel"][j]).max() < TRAJ_TOL[k] * 10
    assert rel(f, d["lf_forces"][1]) < 1e-7


@pytest.mark.parametrize("gamma", [1.0, 50.0])
def test_langevin_zero_temperature_matches_reference(gamma):
    """LangevinLeapfrogIntegrator (integrator/base/LangevinLeapfrogIntegrator.cpp:44-71) at
    T = 0, where its noise term vanishes: vdt, fdt, ndt and the gamma units of the oracle's
    restatement against the reference's own run, 100 steps."""
    d = load()
    box, s = system(d)
    pre = "lv%d_" % int(gamma)
    keep = list(d["lv_keep"])
    pos, vel = box["pos"].copy(), box["vel"].copy()
    for k in range(1, 101):
        pos, vel, f, e = O.langevin(s, pos, vel, 1.0, 1, 0.0, gamma, first_step=k - 1, cutoff=cutoff())
        np.testing.assert_allclose(e, d[pre + "energies"][k], rtol=1e-10, atol=1e-9)
        if k in keep:
            j = keep.index(k)
            assert np.abs(pos - d[pre + "pos"][j]).max() < TRAJ_TOL[k]
            assert np.abs(vel - d[pre + "vel"][j]).max() < TRAJ_TOL[k] * 10


def test_langevin_friction_is_felt():
    """The 50/ps run loses kinetic energy to friction faster than the 1/ps run (the fixture's
    two runs differ as the friction says), and the oracle follows each."""
    d = load()
    box, s = system(d)
    m = box["mass"][:, None]
    ke = {}
    for g in (1.0, 50.0):
        v = d["lv%d_vel" % int(g)][-1]
        ke[g] = 0.5 * (m * v * v).sum()
    assert ke[50.0] < 0.9 * ke[1.0]


def test_langevin_small_gamma_approaches_leapfrog():
    """As gamma -> 0 the Langevin half kick becomes the leapfrog half kick: the velocity gap
    after 20 steps shrinks in proportion to gamma."""
    d = load()
    box, s = system(d)
    pl, vl = box["pos"].copy(), box["vel"].copy()
    for _ in range(20):
        pl, vl, _, _ = O.leapfrog(s, pl, vl, 1.0, 1, cutoff=cutoff())
    gaps = []
    for g in (1e-2, 1e-3):
        p, v, _, _ = O.langevin(s, box["pos"], box["vel"], 1.0, 20, 0.0, g, cutoff=cutoff())
        gaps.append(rel(v, vl))
    # friction removes about gamma x elapsed time of the velocity: 1e-2/ps x 20 fs = 2e-4
    assert gaps[0] < 1e-3 and 5 < gaps[0] / gaps[1] < 20


def test_langevin_noise_stream():
    """The counter-based Gaussian stream: zero mean, unit variance, uncorrelated components,
    different for another atom, half-kick index or seed, and the same for the same counter."""
    g = np.array([O.gauss3(11, i, j) for i in range(400) for j in range(50)]).reshape(-1, 3)
    assert abs(g.mean()) < 0.02 and abs(g.var() - 1) < 0.03
    assert abs(np.corrcoef(g.T)[0, 1]) < 0.03
    assert np.array_equal(O.gauss3(11, 5, 7), O.gauss3(11, 5, 7))
    for other in (O.gauss3(11, 6, 7), O.gauss3(11, 5, 8), O.gauss3(12, 5, 7)):
        assert not np.array_equal(other, O.gauss3(11, 5, 7))


@pytest.mark.skipif(not O.ref_md_available(), reason="reference not compiled (oracle/_ref)")
def test_oracle_forces_on_every_step_of_reference_run():
    """All 1,000 steps of the reference's leapfrog run: on the reference's own positions of
    every step, the oracle's forces and energies equal the reference's (1e-12)."""
    d = load()
    box, s = system(d)
    r = O.ref_md_run(s, box["pos"], box["vel"], 1.0, 1000, cutoff=cutoff(), bonded=True,
                     keep=("energies", "pos", "forces"))
    np.testing.assert_array_equal(r["energies"], d["lf_energies"])
    for k in range(1001):
        f, e, _, _ = O.evaluate(s, r["pos"][k], cutoff=cutoff(), bonded=True)
        assert rel(f, r["forces"][k]) < 1e-12, k
        np.testing.assert_allclose(e, r["energies"][k], rtol=1e-12, atol=1e-10)
