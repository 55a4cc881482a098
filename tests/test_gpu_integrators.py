"""Device integrators against the oracle, step by step, and against ProtoMol's own integrators
(golden fixture tests/golden/water216_md_ref.npz, from the reference compiled in place).

The plain-method workload: 216 TIP3P waters in an 18.62 A box, LJ + Coulomb cutoff with C2
switching 7 -> 8 A (`force LennardJones Coulomb -algorithm NonbondedCutoff`), bonds and angles,
leapfrog 1 fs, 1,000 steps stepped by run(1) as ProtoMolApp steps with outputfreq 1, FP64.

Water is chaotic: two FP64 programs whose forces differ in the last bits follow the same
trajectory for about 100 steps only (the oracle and the reference: 1e-15 A after one step,
1e-9 A after 100, angstroms after 300).  So every one of the 1,000 steps is compared from the
same state: the device's step k -> k+1 against the oracle's step from the device's state k
(positions, velocities, forces and energies to 1e-12 relative), and the device's first 100 steps
against the reference's own run with bounds that grow with the step.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from protomol3_b200 import forces as F
from protomol3_b200 import waterbox as W

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
STEP_TOL = 1e-12                               # one step from the same state, relative RMS
E_ATOL = 648 * 2.0 ** -31                      # energies: fixed-point accumulation, 2^-32 per term
TRAJ_TOL = {10: 1e-11, 50: 1e-9, 100: 1e-7}    # free-running max |x - x_ref| (A), FP64


def rel(a, b):
    return np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum())


def setup(precision="fp64", **integ):
    box = W.water_box(216, seed=1234)
    topo = F.Topology(box, precision)
    fl = [F.BondedSystemForce(), F.NonbondedCutoffSystemForce(lj=("C2", 7.0, 8.0), coulomb=("C2", 7.0, 8.0))]
    md = F.Integrator(topo, fl, timestep=1.0, **integ)
    md.set_state(box["pos"], box["vel"])
    return box, O.System(box), topo, md


def cutoff():
    return O.cutoff_params(lj=("C2", 7.0, 8.0), coul=("C2", 7.0, 8.0))


def test_water216_leapfrog_1000_steps_per_step_fp64():
    d = dict(np.load(os.path.join(GOLD, "water216_md_ref.npz")))
    box, s, topo, md = setup()
    keep = list(d["lf_keep"])
    f0 = md.forces_now()
    assert rel(f0, d["lf_forces"][0]) < STEP_TOL
    pos, vel = md.state()
    for k in range(1, 1001):
        md.run(1)
        p, v = md.state()
        f = md.forces_now()
        e, _ = md.energies()
        po, vo, fo, eo = O.leapfrog(s, pos, vel, 1.0, 1, cutoff=cutoff())
        err = max(rel(p, po), rel(v, vo), rel(f, fo))
        assert err < STEP_TOL, (k, rel(p, po), rel(v, vo), rel(f, fo))
        np.testing.assert_allclose(e[0, :4], eo, rtol=STEP_TOL, atol=E_ATOL)
        if k <= 100:
            np.testing.assert_allclose(e[0, :4], d["lf_energies"][k], rtol=1e-9, atol=E_ATOL)
        if k in keep:
            j = keep.index(k)
            assert np.abs(p - d["lf_pos"][j]).max() < TRAJ_TOL[k], k
            assert np.abs(v - d["lf_vel"][j]).max() < 10 * TRAJ_TOL[k], k
        if k == 100:
            assert rel(f, d["lf_forces"][1]) < 1e-6
        pos, vel = p, v
    md.close()
    topo.close()


@pytest.mark.parametrize("gamma", [1.0, 50.0])
def test_langevin_zero_temperature_vs_reference_and_oracle(gamma):
    """LangevinLeapfrogIntegrator at T = 0 (noise term exactly zero): 100 steps, every step
    against the oracle from the same state, and the trajectory against the reference's own."""
    d = dict(np.load(os.path.join(GOLD, "water216_md_ref.npz")))
    box, s, topo, md = setup(kind="langevin", temperature=0.0, gamma=gamma, seed=5)
    pre = "lv%d_" % int(gamma)
    keep = list(d["lv_keep"])
    pos, vel = md.state()
    for k in range(1, 101):
        md.run(1)
        p, v = md.state()
        e, _ = md.energies()
        po, vo, fo, eo = O.langevin(s, pos, vel, 1.0, 1, 0.0, gamma, seed=5, first_step=k - 1,
                                    cutoff=cutoff())
        assert rel(p, po) < STEP_TOL and rel(v, vo) < STEP_TOL, k
        np.testing.assert_allclose(e[0, :4], d[pre + "energies"][k], rtol=1e-9, atol=E_ATOL)
        if k in keep:
            j = keep.index(k)
            assert np.abs(p - d[pre + "pos"][j]).max() < TRAJ_TOL[k], k
        pos, vel = p, v
    md.close()
    topo.close()


def test_langevin_300K_noise_matches_oracle_stream():
    """At 300 K (gamma 1/ps) the device's noise is the oracle's restated counter-based stream:
    every one of 50 steps, from the same state, agrees to 1e-12; a run of 5 steps in one call
    agrees with five single steps."""
    box, s, topo, md = setup(kind="langevin", temperature=300.0, gamma=1.0, seed=99)
    pos, vel = md.state()
    for k in range(1, 51):
        md.run(1)
        p, v = md.state()
        po, vo, _, _ = O.langevin(s, pos, vel, 1.0, 1, 300.0, 1.0, seed=99, first_step=k - 1,
                                  cutoff=cutoff())
        assert rel(p, po) < STEP_TOL and rel(v, vo) < STEP_TOL, k
        pos, vel = p, v
    md.run(5)
    p, v = md.state()
    po, vo, _, _ = O.langevin(s, pos, vel, 1.0, 5, 300.0, 1.0, seed=99, first_step=50, cutoff=cutoff())
    assert rel(p, po) < 1e-11 and rel(v, vo) < 1e-11
    md.close()
    topo.close()


def test_langevin_small_gamma_approaches_leapfrog_on_device():
    """gamma -> 0 at T = 0: the device's Langevin run tends to its leapfrog run (gap after 20
    steps proportional to gamma)."""
    box, s, topo, md = setup()
    md.run(20)
    _, vl = md.state()
    md.close()
    topo.close()
    gaps = []
    for g in (1e-2, 1e-3):
        box, s, topo, md = setup(kind="langevin", temperature=0.0, gamma=g)
        for _ in range(20):
            md.run(1)
        gaps.append(rel(md.state()[1], vl))
        md.close()
        topo.close()
    assert gaps[0] < 1e-3 and 5 < gaps[0] / gaps[1] < 20
