"""Trajectory files against the reference's own writers (CPU: frames from host positions).

Golden files (tests/golden/water27_ref.{dcd,xyz}, made by make_golden_output.py with the
reference's DCDTrajectoryWriter and XYZWriter compiled in place): 27 TIP3P waters, three frames.
Tolerance: byte equality, except the 80 bytes of the DCD's first title line, which name the file
and the writer's build."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from protomol3_b200 import forces as F

GOLD = os.path.join(os.path.dirname(__file__), "golden")
TITLE = slice(100, 180)


def _frames():
    return np.load(os.path.join(GOLD, "water27_frames.npz"))["frames"]


def _names():
    return ["OH2", "H1", "H2"] * 27


def _same_but_title(a, b):
    return len(a) == len(b) and a[:TITLE.start] == b[:TITLE.start] and a[TITLE.stop:] == b[TITLE.stop:]


def test_dcd_matches_reference_writer(tmp_path):
    fr = _frames()
    t = F.Trajectory.dcd(tmp_path / "w.dcd", fr.shape[1])
    for f in fr:
        t.write(f)
    assert t.frames() == 3
    t.close()
    mine = (tmp_path / "w.dcd").read_bytes()
    gold = open(os.path.join(GOLD, "water27_ref.dcd"), "rb").read()
    assert _same_but_title(mine, gold)
    assert mine[TITLE].startswith(b"Remarks: File '")


def test_xyz_matches_reference_writer(tmp_path):
    fr = _frames()
    t = F.Trajectory.xyz(tmp_path / "w.xyz", _names())
    for f in fr:  # every frame rewrites the file: the last one stays
        t.write(f)
    t.close()
    assert (tmp_path / "w.xyz").read_bytes() == open(os.path.join(GOLD, "water27_ref.xyz"), "rb").read()


def test_dcd_big_endian_is_the_byte_swap(tmp_path):
    fr = _frames()
    for little in (True, False):
        t = F.Trajectory.dcd(tmp_path / ("e%d.dcd" % little), fr.shape[1], little_endian=little)
        for f in fr:
            t.write(f)
        t.close()
    le = (tmp_path / "e1.dcd").read_bytes()
    be = (tmp_path / "e0.dcd").read_bytes()
    # the frame records: int32 markers and float32 values, each word byte-swapped
    off = len(le) - 3 * (81 * 4 + 8) * 3
    w_le = np.frombuffer(le[off:], "<u4")
    w_be = np.frombuffer(be[off:], ">u4")
    assert np.array_equal(w_le, w_be)


def test_dcd_comment_lengthens_the_title(tmp_path):
    t = F.Trajectory.dcd(tmp_path / "c.dcd", 81, comment="x" * 100)
    t.write(_frames()[0])
    t.close()
    d = (tmp_path / "c.dcd").read_bytes()
    n2 = int(np.frombuffer(d[96:100], "<i4")[0])
    assert n2 == 3 and int(np.frombuffer(d[92:96], "<i4")[0]) == 3 * 80 + 4


def test_bad_arguments_raise(tmp_path):
    with pytest.raises(RuntimeError):
        F.Trajectory.dcd("", 10)
    t = F.Trajectory.dcd(tmp_path / "x.dcd", 81)
    with pytest.raises(ValueError):
        t.write(np.zeros((80, 3)))
    t.close()
    with pytest.raises(RuntimeError):
        F.Trajectory.dcd(tmp_path / "no" / "such" / "dir.dcd", 81).write(_frames()[0])


@pytest.mark.skipif(not O.ref_md_available(), reason="reference writers not compiled here")
def test_live_reference_writers_on_another_case(tmp_path, monkeypatch):
    rng = np.random.default_rng(5)
    fr = rng.uniform(-50, 50, (4, 10, 3))
    monkeypatch.chdir(tmp_path)
    O.ref_write_dcd("r.dcd", fr, first_step=7)
    t = F.Trajectory.dcd("m.dcd", 10, first_step=7)
    for f in fr:
        t.write(f)
    t.close()
    a, b = open("r.dcd", "rb").read(), open("m.dcd", "rb").read()
    assert _same_but_title(a, b)
    names = ["C%d" % i for i in range(10)]
    O.ref_write_xyz("r.xyz", fr[0], names)
    t = F.Trajectory.xyz("m.xyz", names)
    t.write(fr[0])
    t.close()
    assert open("r.xyz", "rb").read() == open("m.xyz", "rb").read()


def test_xyz_trajectory_matches_reference_writer(tmp_path):
    """XYZTrajectoryWriter as OutputXYZTrajectoryForce writes it: a frame-count line rewritten
    with every frame, the frames appended (golden water27_ref_traj.xyz)."""
    fr = _frames()
    t = F.Trajectory.xyz_trajectory(tmp_path / "t.xyz", _names())
    for f in fr:
        t.write(f)
    assert t.frames() == 3
    t.close()
    assert (tmp_path / "t.xyz").read_bytes() == open(os.path.join(GOLD, "water27_ref_traj.xyz"), "rb").read()


def test_dcd_minimal_image_matches_reference(tmp_path):
    """OutputDCDTrajectory's minimal-image option: frames whose atoms were scattered over
    periodic images come out as the reference's SemiGenericTopology::minimalImage writes them
    (golden water27_ref_min.dcd), byte for byte but the first title line."""
    from protomol3_b200 import waterbox as W
    d = np.load(os.path.join(GOLD, "water27_frames.npz"))
    box = W.water_box(27, seed=3)
    t = F.Trajectory.dcd(tmp_path / "m.dcd", 81)
    t.set_minimal_image(box["mass"], box["molecule"], box["bonds"], box["box"], d["origin"])
    for f in d["scrambled"]:
        t.write(f)
    t.close()
    mine = (tmp_path / "m.dcd").read_bytes()
    gold = open(os.path.join(GOLD, "water27_ref_min.dcd"), "rb").read()
    assert _same_but_title(mine, gold)
    # and the scrambling was undone: every water whole, its centre of mass inside the box
    plain = F.Trajectory.dcd(tmp_path / "p.dcd", 81)
    for f in d["scrambled"]:
        plain.write(f)
    plain.close()
    assert (tmp_path / "p.dcd").read_bytes()[200:] != mine[200:]


def test_minimal_image_refuses_bad_input(tmp_path):
    from protomol3_b200 import waterbox as W
    box = W.water_box(27, seed=3)
    t = F.Trajectory.dcd(tmp_path / "m.dcd", 81)
    bad = box["bonds"].copy()
    bad[0] = (0, 5)  # atoms of two waters
    with pytest.raises(RuntimeError):
        t.set_minimal_image(box["mass"], box["molecule"], bad, box["box"])
    x = F.Trajectory.xyz(tmp_path / "x.xyz", _names())
    with pytest.raises(RuntimeError):
        x.set_minimal_image(box["mass"], box["molecule"], box["bonds"], box["box"])
    t.close()
    x.close()
