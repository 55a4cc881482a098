"""Checkpoints of device-resident MD state (OutputCheckpoint, output/OutputCheckpoint.cpp:58-178;
CheckpointModule, module/CheckpointModule.cpp:30-48) and force / minimal-image output from a run.

Tolerances: a run restored from an exact checkpoint continues bit for bit (array equality of
positions, velocities and energies), in the same run object or in a new system of the same
boxes; without the list's reference positions the restored run is rebuilt at the checkpoint's
positions and agrees to the rounding of the arithmetic, which the chaotic dynamics amplifies
(bounds below).  Files: the reference's layouts (golden water27_ref.chk from
CheckpointConfigWriter; XYZ form pinned in tests/test_output.py)."""
import os

import numpy as np
import pytest

from protomol3_b200 import forces as F
from protomol3_b200 import waterbox as W

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def make(box, precision, **integ):
    topo = F.Topology(box, precision)
    g = W.pme_grid_for(box["box"][0])
    fl = [F.BondedSystemForce(), F.NonbondedCutoffSystemForce(lj=("C2", 7.5, 9.0)),
          F.NonbondedPMEwaldSystemForce((g, g, g), 9.0)]
    return topo, F.Integrator(topo, fl, timestep=1.0, **integ)


def finish(md, n):
    md.run(n)
    pos, vel = md.state()
    e, k = md.energies()
    return pos, vel, e, k


@pytest.mark.parametrize("precision,kind", [("mixed", "langevin"), ("fp64", "leapfrog"), ("mixed", "leapfrog")])
def test_restored_run_continues_bit_for_bit(precision, kind):
    """60 steps straight, against 30 steps, a checkpoint, and 30 steps of a new system restored
    from it (and of the first run restored in place).  The lattice start moves atoms fast, so
    the list is rebuilt several times on both sides of the checkpoint."""
    box = W.water_box(500, seed=12)
    integ = dict(kind=kind, temperature=300.0, gamma=1.0, seed=77) if kind == "langevin" else {}
    topo, md = make(box, precision, **integ)
    md.set_state(box["pos"], box["vel"])
    md.run(30)
    ck = md.checkpoint()
    assert ck["step"] == 30
    b0 = topo.list_builds()
    ref = finish(md, 30)
    assert topo.list_builds() > b0  # rebuilds after the checkpoint too
    # a new system of the same box
    topo2, md2 = make(box, precision, **integ)
    md2.restore(ck)
    got = finish(md2, 30)
    for a, b in zip(ref, got):
        assert np.array_equal(a, b)
    assert md2.checkpoint()["step"] == 60
    # the first run, rewound to the checkpoint
    md.restore(ck)
    again = finish(md, 30)
    for a, b in zip(ref, again):
        assert np.array_equal(a, b)
    # without the list's reference positions: a fresh list, equal to rounding
    topo3, md3 = make(box, precision, **integ)
    md3.restore(ck, exact=False)
    loose = finish(md3, 30)
    tol = 1e-7 if precision == "fp64" else 1e-3
    assert np.abs(loose[0] - ref[0]).max() < tol
    for t, m in ((topo, md), (topo2, md2), (topo3, md3)):
        m.close()
        t.close()


def test_checkpoint_files_in_the_reference_layout(tmp_path):
    """pos_base<id>.pos / vel_base<id>.vel hold the checkpoint's positions and velocities in the
    XYZ form (15 significant digits), the checkpoint file has CheckpointConfigWriter's sections
    (golden water27_ref.chk) with this library's noise state under #Random, and the previous
    checkpoint's files are removed."""
    box = W.water_box(216, seed=9)
    topo, md = make(box, "mixed", kind="langevin", temperature=300.0, gamma=1.0, seed=5)
    md.set_state(box["pos"], box["vel"])
    names = ["OH2", "H1", "H2"] * 216
    md.run(10)
    md.write_checkpoint(tmp_path / "run.chk", 2, tmp_path / "w.", tmp_path / "v.", names, first_step=1000)
    md.run(5)
    md.write_checkpoint(tmp_path / "run.chk", 3, tmp_path / "w.", tmp_path / "v.", names, first_step=1000)
    assert not (tmp_path / "w.2.pos").exists() and not (tmp_path / "v.2.vel").exists()
    ck = md.checkpoint()
    for fname, arr in (("w.3.pos", ck["positions"]), ("v.3.vel", ck["velocities"])):
        lines = (tmp_path / fname).read_text().splitlines()
        assert int(lines[0]) == 648
        vals = np.array([[float(x) for x in ln.split()[1:]] for ln in lines[1:]])
        assert [ln.split("\t")[0] for ln in lines[1:]] == names
        np.testing.assert_allclose(vals, arr, rtol=1e-14, atol=1e-14)
        mine = F.Trajectory.xyz(tmp_path / ("again_" + fname), names)
        mine.write(arr)
        mine.close()
        assert (tmp_path / fname).read_bytes() == (tmp_path / ("again_" + fname)).read_bytes()
    got = (tmp_path / "run.chk").read_text().split("\n")
    gold = open(os.path.join(GOLD, "water27_ref.chk")).read().split("\n")
    assert len(got) == len(gold)
    assert got[0] == gold[0] == "!Checkpoint File!"
    assert [got[k] for k in (1, 3, 5, 7)] == [gold[k] for k in (1, 3, 5, 7)] == ["#ID", "#Step", "#Random", "#Integrator"]
    assert got[2] == "3" and got[4] == "1015" and got[8:] == gold[8:]
    assert got[6] == "philox4x32-10 5 30"  # seed, half kicks drawn (2 per step)
    # a run given its noise stream (a system moved from another run): the stream's seed and the
    # half kicks drawn on it, not the run's own
    md.set_box_noise(seeds=[9], steps=[100])
    md.run(4)
    md.write_checkpoint(tmp_path / "run.chk", 4, tmp_path / "w.", tmp_path / "v.", names)
    assert (tmp_path / "run.chk").read_text().split("\n")[6] == "philox4x32-10 9 208"
    md.close()
    topo.close()


def test_force_frames_and_device_minimal_image(tmp_path):
    """Force frames (OutputXYZTrajectoryForce) hold the run's forces of the last evaluation;
    minimal-image DCD frames taken off the device equal those written from host positions."""
    box = W.water_box(216, seed=9)
    topo, md = make(box, "fp64")
    md.set_state(box["pos"], box["vel"])
    names = ["OH2", "H1", "H2"] * 216
    ft = F.Trajectory.xyz_trajectory(tmp_path / "f.xyz", names)
    dev = F.Trajectory.dcd(tmp_path / "dev.dcd", 648)
    host = F.Trajectory.dcd(tmp_path / "host.dcd", 648)
    for t in (dev, host):
        t.set_minimal_image(box["mass"], box["molecule"], box["bonds"], box["box"], box["box"] * 0.5)
    forces = []
    for _ in range(3):
        md.run(40)
        md.write_force_frame(ft)
        md.write_frame(dev)
        forces.append(md.forces_now())
        host.write(md.state()[0])
    for t in (ft, dev, host):
        t.close()
    assert (tmp_path / "dev.dcd").read_bytes()[180:] == (tmp_path / "host.dcd").read_bytes()[180:]
    lines = (tmp_path / "f.xyz").read_text().splitlines()
    assert lines[0].strip() == "3" and len(lines[0]) == 19
    for k in range(3):
        blk = lines[1 + k * 649: 1 + (k + 1) * 649]
        assert int(blk[0]) == 648
        vals = np.array([[float(x) for x in ln.split()[1:]] for ln in blk[1:]])
        np.testing.assert_allclose(vals, forces[k], rtol=1e-14, atol=1e-13)
    md.close()
    topo.close()
