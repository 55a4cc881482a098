"""Device MD beyond single steps: NVE reproducibility and energy conservation of the mixed
path, and the Langevin integrator's seeded noise and thermostat
(integrator/leapfrog/LangevinLeapfrogIntegrator.cpp:44-71)."""
import numpy as np
import pytest

from protomol3_b200 import forces as F
from protomol3_b200 import waterbox as W

pytestmark = pytest.mark.gpu
BOLTZMANN = 0.001987191  # kcal/mol/K (PMConstants.cpp)


def _forces(box, rc=10.0, switchon=8.0):
    grid = W.pme_grid_for(box["box"][0])
    return [F.BondedSystemForce(), F.NonbondedCutoffSystemForce(lj=("C2", switchon, rc)),
            F.NonbondedPMEwaldSystemForce((grid,) * 3, rc)]


def _run(box, precision, steps, chunk, **integ):
    topo = F.Topology(box, precision)
    md = F.Integrator(topo, _forces(box), timestep=1.0, **integ)
    md.set_state(box["pos"], box["vel"])
    etot, kin = [], []
    for k in range(0, steps + 1, chunk):
        if k:
            md.run(chunk)
        e, kk = md.energies()
        etot.append(e[0, :4].sum() + kk[0])
        kin.append(kk[0])
    pos, vel = md.state()
    md.close()
    topo.close()
    return np.array(etot), np.array(kin), pos, vel


def test_nve_mixed_bit_identical_and_energy_conserving():
    """Two mixed-precision NVE runs of 600 steps give bit-identical positions and velocities
    (fixed-point accumulation, deterministic lists); the total energy stays within 0.02 kcal/mol
    per degree of freedom of its start, and its drift is of the size of the FP64 path's."""
    box = W.water_box(1000, seed=77)
    e1, _, p1, v1 = _run(box, "mixed", 600, 100)
    e2, _, p2, v2 = _run(box, "mixed", 600, 100)
    assert np.array_equal(p1, p2) and np.array_equal(v1, v2)
    assert np.array_equal(e1, e2)
    ndof = 3 * len(box["charge"]) - 3
    e64, _, _, _ = _run(box, "fp64", 600, 100)
    assert np.abs(e1 - e1[0]).max() / ndof < 0.02
    assert np.abs(e64 - e64[0]).max() / ndof < 0.02
    assert abs(e1[-1] - e1[0]) <= 2.0 * abs(e64[-1] - e64[0]) + 0.002 * ndof
    # (the mixed and FP64 trajectories themselves separate within a fraction of a picosecond,
    # as any two trajectories of a chaotic system do; only statistics are compared)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_langevin_seeded_and_thermostatted(precision):
    """Same seed: identical trajectories; another seed: a different one; a 216-water box started
    at 150 K relaxes to the 300 K bath (gamma = 10/ps) within 2% over 1.5 ps of averaging."""
    box = dict(W.water_box(216, seed=3, temperature=150.0))
    kw = dict(kind="langevin", temperature=300.0, gamma=10.0)
    _, k1, p1, _ = _run(box, precision, 2500, 100, seed=11, **kw)
    _, _, p2, _ = _run(box, precision, 200, 100, seed=11, **kw)
    _, _, p3, _ = _run(box, precision, 200, 100, seed=12, **kw)
    _, _, p1s, _ = _run(box, precision, 200, 100, seed=11, **kw)
    assert np.array_equal(p2, p1s)
    assert not np.array_equal(p2, p3)
    ndof = 3 * len(box["charge"])
    temp = 2.0 * k1 / (ndof * BOLTZMANN)
    assert temp[0] < 200.0
    assert abs(temp[10:].mean() - 300.0) < 0.02 * 300.0 + 3 * temp[10:].std() / np.sqrt(len(temp) - 10)
