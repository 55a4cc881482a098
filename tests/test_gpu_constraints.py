"""SHAKE / RATTLE on the device (two-pass group kernels of pmb_md.cu) against the reference's
own integrator and modifiers (golden fixture) and the oracle's restatement.

With no force terms every operation is the reference's, in its order, so the device state must
equal the reference's bit for bit; with forces, the fixed-point force accumulation separates
the trajectories by rounding only (tolerance 1e-9 A on positions after 10 steps)."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from protomol3_b200 import _lib as L
from protomol3_b200 import constraints as CS
from protomol3_b200 import forces as F
from protomol3_b200 import waterbox as W

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden", "water64_rigid_ref.npz")


def _opt(a):
    return None if a[1] == 0 else (float(a[0]), int(a[1]))


def _device_run(box, cons, dt, steps, shake, rattle, precision="fp64", forces=(), chunks=None,
                use_graph=True, **integ):
    topo = F.Topology(box, precision)
    md = F.Integrator(topo, list(forces), timestep=dt, use_graph=use_graph, **integ)
    md.set_constraints(cons, shake=shake is not None, shake_epsilon=(shake or (0, 0))[0],
                       shake_max_iter=(shake or (0, 0))[1], rattle=rattle is not None,
                       rattle_epsilon=(rattle or (0, 0))[0], rattle_max_iter=(rattle or (0, 0))[1])
    md.set_state(box["pos"], box["vel"])
    for n in (chunks or [steps]):
        md.run(n)
    pos, vel = md.state()
    sweeps = md.constraint_sweeps()
    md.close()
    topo.close()
    return pos, vel, sweeps


@pytest.mark.parametrize("case", ["sr", "s", "r", "tight"])
def test_device_equals_reference_golden(case):
    g = np.load(GOLD)
    box = W.water_box(64, seed=7)
    cons = CS.rattle_shake_constraints(box)
    pos, vel, _ = _device_run(box, cons, float(g["dt"]), int(g[case + "_steps"]),
                              _opt(g[case + "_shake"]), _opt(g[case + "_rattle"]))
    assert np.array_equal(pos, g[case + "_pos"])
    assert np.array_equal(vel, g[case + "_vel"])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_equals_oracle_many_groups(precision):
    """2,000 waters (63 warps of groups), runs split over several calls (the closing RATTLE of
    each call, then the next call's opening half kick), with and without the CUDA graph."""
    box = W.water_box(2000, seed=21)
    cons = CS.rattle_shake_constraints(box)
    ref_pos, ref_vel, _, _ = O.leapfrog_constrained(O.System(box), box["pos"], box["vel"], 2.0, 4, cons)
    ref_pos, ref_vel, _, _ = O.leapfrog_constrained(O.System(box), ref_pos, ref_vel, 2.0, 6, cons,
                                                    last_pos=ref_pos)
    for graph in (True, False):
        pos, vel, sweeps = _device_run(box, cons, 2.0, 10, (1e-5, 30), (1e-5, 30), precision,
                                       chunks=[4, 6], use_graph=graph)
        assert np.array_equal(pos, ref_pos) and np.array_equal(vel, ref_vel)
        assert 1 <= sweeps[0] <= 31 and 1 <= sweeps[1] <= 31


def test_device_second_round_when_the_sweep_count_jumps():
    """The first scan of an application covers up to two sweeps more than the last one took;
    velocities scaled up between two runs make the next applications need more, which the
    second round supplies.  Still the oracle's result exactly."""
    box = W.water_box(500, seed=33)
    cons = CS.rattle_shake_constraints(box)
    topo = F.Topology(box, "fp64")
    md = F.Integrator(topo, [], timestep=2.0)
    md.set_constraints(cons)
    md.set_state(box["pos"], box["vel"])
    md.run(3)
    p1, v1 = md.state()
    k1 = md.constraint_sweeps()
    md.set_state(p1, 6.0 * v1)
    md.run(3)
    p2, v2 = md.state()
    k2 = md.constraint_sweeps()
    md.close()
    topo.close()
    r1, w1, _, _ = O.leapfrog_constrained(O.System(box), box["pos"], box["vel"], 2.0, 3, cons)
    r2, w2, _, _ = O.leapfrog_constrained(O.System(box), r1, 6.0 * w1, 2.0, 3, cons, last_pos=r1)
    assert np.array_equal(p1, r1) and np.array_equal(v1, w1)
    assert np.array_equal(p2, r2) and np.array_equal(v2, w2)
    assert k2[0] > k1[0] + 2 or k2[1] > k1[1] + 2, (k1, k2)


def test_device_general_groups():
    """Groups other than single waters take the general kernel: every tenth water is linked to
    the next one by an extra H-O bond, which joins the two into one group of 6 atoms and 7
    constraints.  Still the oracle's result exactly."""
    box = dict(W.water_box(300, seed=5))
    extra = np.array([[3 * w + 2, 3 * w + 3] for w in range(0, 290, 10)], np.int32)
    box["bonds"] = np.concatenate([box["bonds"], extra])
    p = box["pos"].reshape(-1, 3)
    box["bond_r0"] = np.concatenate([box["bond_r0"], np.linalg.norm(p[extra[:, 0]] - p[extra[:, 1]], axis=1)])
    box["bond_k"] = np.concatenate([box["bond_k"], np.zeros(len(extra))])
    cons = CS.rattle_shake_constraints(box)
    assert len(cons[0]) == 3 * 300 + len(extra)
    ref_pos, ref_vel, _, _ = O.leapfrog_constrained(O.System(box), box["pos"], box["vel"], 1.0, 8, cons)
    pos, vel, _ = _device_run(box, cons, 1.0, 8, (1e-5, 30), (1e-5, 30))
    assert np.array_equal(pos, ref_pos) and np.array_equal(vel, ref_vel)


def test_device_with_forces_close_to_oracle():
    """Bonded + LJ/Coulomb C2 cutoff forces, FP64 path, 10 steps of 2 fs on 216 rigid waters."""
    box = W.water_box(216, seed=9)
    cons = CS.rattle_shake_constraints(box)
    cp = O.cutoff_params(lj=("C2", 7.0, 8.0), coul=("C2", 7.0, 8.0))
    ref_pos, ref_vel, _, _ = O.leapfrog_constrained(O.System(box), box["pos"], box["vel"], 2.0, 10, cons,
                                                    cutoff=cp, bonded=True)
    forces = [F.BondedSystemForce(),
              F.NonbondedCutoffSystemForce(lj=("C2", 7.0, 8.0), coulomb=("C2", 7.0, 8.0))]
    pos, vel, _ = _device_run(box, cons, 2.0, 10, (1e-5, 30), (1e-5, 30), "fp64", forces)
    assert np.abs(pos - ref_pos).max() < 1e-9
    assert np.abs(vel - ref_vel).max() < 1e-9


def test_langevin_with_constraints_equals_reference_golden():
    """SHAKE after the drift and RATTLE after the closing half kick of the LangevinLeapfrogIntegrator
    (temperature 0, gamma 50/ps): the reference's own run (golden case lv).  The friction factor
    exp(-gamma h / 2) comes from the device's exp, which may differ from the host's in the last
    bit, so equality is to 1e-13 rather than bit for bit."""
    g = np.load(GOLD)
    box = W.water_box(64, seed=7)
    cons = CS.rattle_shake_constraints(box)
    pos, vel, _ = _device_run(box, cons, float(g["dt"]), int(g["lv_steps"]), (1e-5, 30), (1e-5, 30),
                              kind="langevin", temperature=0.0, gamma=float(g["lv_gamma"]), seed=3)
    assert np.abs(pos - g["lv_pos"]).max() < 1e-13
    assert np.abs(vel - g["lv_vel"]).max() < 1e-13 * max(1.0, np.abs(g["lv_vel"]).max())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_langevin_with_constraints_and_noise_equals_oracle(precision):
    """Rigid water under Langevin at 300 K (gamma 1/ps, 2 fs) with forces, runs split over
    calls: against the oracle with the same counter-based noise, step for step."""
    box = W.water_box(216, seed=8)
    cons = CS.rattle_shake_constraints(box)
    forces = [F.BondedSystemForce(),
              F.NonbondedCutoffSystemForce(lj=("C2", 7.0, 8.0), coulomb=("C2", 7.0, 8.0))]
    s = O.System(box)
    cp = O.cutoff_params(lj=("C2", 7.0, 8.0), coul=("C2", 7.0, 8.0))
    topo = F.Topology(box, precision)
    md = F.Integrator(topo, forces, timestep=2.0, kind="langevin", temperature=300.0, gamma=1.0, seed=21)
    md.set_constraints(cons)
    md.set_state(box["pos"], box["vel"])
    pos, vel = box["pos"].copy(), box["vel"].copy()
    tol = 1e-11 if precision == "fp64" else 1e-5
    for k in range(10):
        md.run(1)
        p, v = md.state()
        po, vo, _, _ = O.langevin_constrained(s, pos, vel, 2.0, 1, cons, 300.0, 1.0, seed=21, first_step=k,
                                              cutoff=cp, bonded=True, last_pos=pos)
        assert np.abs(p - po).max() < tol and np.abs(v - vo).max() < tol * 100, k
        pos, vel = p, v
    a1, a2, ln = cons
    d2 = ((pos[a2] - pos[a1]) ** 2).sum(1)
    assert np.mean(np.abs(d2 - ln ** 2) / (2 * ln ** 2)) <= 1e-5
    md.close()
    topo.close()


@pytest.mark.parametrize("case", ["sr", "r", "tight", "s", "lv"])
def test_rattle_constraint_virial_equals_reference(case):
    """With the virial on, the run's energies hold after run(n) what the reference's do: the
    virial of the last RATTLE application (ModifierRattle.cpp:58; no force terms here), and none
    for SHAKE alone (its terms are cleared by the force evaluation after each drift)."""
    g = np.load(GOLD)
    box = W.water_box(64, seed=7)
    cons = CS.rattle_shake_constraints(box)
    topo = F.Topology(box, "fp64")
    if case == "lv":
        md = F.Integrator(topo, [], timestep=float(g["dt"]), kind="langevin", temperature=0.0,
                          gamma=float(g["lv_gamma"]), seed=3)
        shake, rattle, steps = (1e-5, 30), (1e-5, 30), int(g["lv_steps"])
    else:
        md = F.Integrator(topo, [], timestep=float(g["dt"]))
        shake, rattle, steps = _opt(g[case + "_shake"]), _opt(g[case + "_rattle"]), int(g[case + "_steps"])
    md.set_virial(True)
    md.set_constraints(cons, shake=shake is not None, shake_epsilon=(shake or (0, 0))[0],
                       shake_max_iter=(shake or (0, 0))[1], rattle=rattle is not None,
                       rattle_epsilon=(rattle or (0, 0))[0], rattle_max_iter=(rattle or (0, 0))[1])
    md.set_state(box["pos"], box["vel"])
    md.run(steps)
    e, _ = md.energies()
    vir = e[0, L.E_VIRIAL:L.E_VIRIAL + 9]
    ref = g[case + "_virial"]
    assert np.abs(vir - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max()) + 64 * 2.0 ** -31
    md.close()
    topo.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_md_force_virial_equals_evaluation(precision):
    """Without constraints the run's virial after a step is the force virial of the step's
    evaluation: the same as pmb_evaluate's at the run's positions."""
    box = W.water_box(216, seed=12)
    fl = [F.BondedSystemForce(), F.NonbondedCutoffSystemForce(lj=("C2", 7.0, 8.0)),
          F.NonbondedPMEwaldSystemForce((20, 20, 20), 8.0)]
    topo = F.Topology(box, precision)
    md = F.Integrator(topo, fl, timestep=1.0)
    md.set_virial(True)
    md.set_state(box["pos"], box["vel"])
    md.run(3)
    e, _ = md.energies()
    pos, _ = md.state()
    t2 = F.Topology(box, precision)
    f = np.zeros((t2.n_atoms, 3))
    ss = F.ScalarStructure(1, virial=True)
    F.evaluate_all(t2, [F.BondedSystemForce(), F.NonbondedCutoffSystemForce(lj=("C2", 7.0, 8.0)),
                        F.NonbondedPMEwaldSystemForce((20, 20, 20), 8.0)], pos, f, ss)
    tol = 1e-9 if precision == "fp64" else 1e-5
    v, vr = e[0, L.E_VIRIAL:L.E_VIRIAL + 9], ss.virial().ravel()
    assert np.abs(v - vr).max() <= tol * np.abs(vr).max() * 10
    np.testing.assert_allclose(e[0, :4], ss.table[0, :4], rtol=tol, atol=216 * 3 * 2.0 ** -31)
    for m, t in ((md, topo),):
        m.close()
        t.close()
    t2.close()
