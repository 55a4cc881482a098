"""Trajectory frames taken off a device MD run (asynchronous copy into pinned staging buffers and
a writer thread) against the same frames written from host positions.  The mixed path is
deterministic, so a second run gives the positions of every frame bit for bit.  Tolerance: byte
equality except the DCD's first title line (it names the file)."""
import numpy as np
import pytest

from protomol3_b200 import forces as F
from protomol3_b200 import waterbox as W

pytestmark = pytest.mark.gpu
TITLE = slice(100, 180)


def _md(box):
    topo = F.Topology(box, "mixed")
    grid = W.pme_grid_for(box["box"][0])
    fl = [F.BondedSystemForce(), F.NonbondedCutoffSystemForce(lj=("C2", 7.0, 8.0)),
          F.NonbondedPMEwaldSystemForce((grid,) * 3, 8.0)]
    md = F.Integrator(topo, fl, timestep=1.0)
    md.set_state(box["pos"], box["vel"])
    return topo, md


def test_device_frames_equal_host_frames(tmp_path):
    box = W.water_box(216, seed=12)
    n = len(box["charge"])
    names = ["OH2", "H1", "H2"] * 216
    # frames off the device, several in flight at once (one step apart, no waits in between)
    topo, md = _md(box)
    dcd = F.Trajectory.dcd(tmp_path / "dev.dcd", n, first_step=0)
    xyz = F.Trajectory.xyz(tmp_path / "dev.xyz", names)
    for _ in range(12):
        md.run(1)
        md.write_frame(dcd)
        md.write_frame(xyz)
    dcd.flush()
    assert dcd.frames() == 12 and xyz.frames() == 12
    dcd.close()
    xyz.close()
    md.close()
    topo.close()
    # the same run again, positions through the host
    topo, md = _md(box)
    dcd = F.Trajectory.dcd(tmp_path / "host.dcd", n, first_step=0)
    xyz = F.Trajectory.xyz(tmp_path / "host.xyz", names)
    for _ in range(12):
        md.run(1)
        pos, _ = md.state()
        dcd.write(pos)
        xyz.write(pos)
    dcd.close()
    xyz.close()
    md.close()
    topo.close()
    a, b = (tmp_path / "dev.dcd").read_bytes(), (tmp_path / "host.dcd").read_bytes()
    assert len(a) == len(b) and a[:TITLE.start] == b[:TITLE.start] and a[TITLE.stop:] == b[TITLE.stop:]
    assert (tmp_path / "dev.xyz").read_bytes() == (tmp_path / "host.xyz").read_bytes()


def test_frame_atom_count_must_match(tmp_path):
    box = W.water_box(27, seed=2)
    topo, md = _md(box)
    t = F.Trajectory.dcd(tmp_path / "bad.dcd", 80)
    with pytest.raises(RuntimeError):
        md.write_frame(t)
    t.close()
    md.close()
    topo.close()
