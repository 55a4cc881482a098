"""Build the golden files that pin the trajectory writers to ProtoMol's own.

Run in a container that holds the ProtoMol 3 source tree, after ``make -C oracle ref`` has
compiled the reference's DCDTrajectoryWriter and XYZWriter in place into
``oracle/_ref/libpmref_md.so``:

    python tests/golden/make_golden_output.py

It writes next to this script, for a seeded box of 27 TIP3P waters (``protomol3_b200.waterbox``,
seed 3) and three frames (its positions shifted by 0, 0.25 and 0.5 A along x):

* ``water27_ref.dcd``: the DCD file as OutputDCDTrajectory writes it (timestep argument 1.0,
  first step 0), one ``write`` per frame;
* ``water27_ref.xyz``: the XYZ file of the last frame with names OH2/H1/H2;
* ``water27_ref_traj.xyz``: the three frames through XYZTrajectoryWriter, as
  OutputXYZTrajectoryForce writes it (a frame-count line, then the frames);
* ``water27_ref_min.dcd``: the minimal-image DCD (OutputDCDTrajectory with minimalImage) of three
  scrambled frames, every atom of the frames moved by a seeded whole number of box edges per
  axis (molecules split over images, centres far outside the box); molecules are the waters with
  their two O-H bonds as pairs, box origin at the box centre;
* ``water27_ref.chk``: a checkpoint file of CheckpointConfigWriter (ID 3, step 1500) with the
  reference's Random and a LeapfrogIntegrator;
* ``water27_frames.npz``: the three frames, the scrambled frames and the box origin.

The first title line of a DCD file names the file and the writer's build date, so tests compare
every byte but those 80.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402
from protomol3_b200 import waterbox as W  # noqa: E402


def frames():
    box = W.water_box(27, seed=3)
    return np.stack([box["pos"] + np.array([0.25 * k, 0.0, 0.0]) for k in range(3)])


def names():
    return ["OH2", "H1", "H2"] * 27


def scrambled(fr, edge):
    rng = np.random.default_rng(27)
    return np.stack([f + rng.integers(-2, 3, size=f.shape) * edge for f in fr])


def main():
    if not O.ref_md_available():
        raise SystemExit("oracle/_ref/libpmref_md.so is missing: run make -C oracle ref first")
    fr = frames()
    box = W.water_box(27, seed=3)
    edge = box["box"][0]
    sc = scrambled(fr, edge)
    origin = box["box"] * 0.5
    os.chdir(HERE)  # relative names: the DCD title records the name it was given
    O.ref_write_dcd("water27_ref.dcd", fr)
    O.ref_write_xyz("water27_ref.xyz", fr[-1], names())
    O.ref_write_xyz_trajectory("water27_ref_traj.xyz", fr, names())
    O.ref_write_dcd_minimal("water27_ref_min.dcd", O.System(box), sc, box["bonds"], origin)
    O.ref_write_checkpoint_config("water27_ref.chk", 3, 1500)
    np.savez_compressed("water27_frames.npz", frames=fr, scrambled=sc, origin=origin)


if __name__ == "__main__":
    main()
