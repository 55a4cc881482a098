"""Build the golden fixture that pins the vacuum cutoff forces to ProtoMol's own.

Run in a container that holds the ProtoMol 3 source tree, after ``make -C oracle ref`` has
compiled the reference's cutoff forces with VacuumBoundaryConditions in place
(``oracle/_ref/libpmref_md.so``, harness ``oracle/ref_vacuum.cpp``):

    python tests/golden/make_golden_vacuum.py [--ref <ProtoMol 3 tree>]

It writes ``vacuum_ref.npz`` next to this script with two inputs and the reference's forces and
energies for each force set:

* ``ala``: the alanine dipeptide of the reference's vacuum ConfigTests
  (``protomol-test/ConfigTests/data/alanine.{psf,pdb,par}``, exclusion scheme scaled1-4,
  topology conventions as in make_golden.py), with the LJ settings of C2Test (C2, 8 -> 10 A) and
  C1Test (C1, 10 A), a plain 10 A Coulomb cutoff, and LJ C2 with Coulomb C2 together;
* ``drop``: a droplet of TIP3P water (the waters of a seeded 1,000-water box,
  ``protomol3_b200.waterbox`` seed 8, whose oxygen lies within 14 A of the box centre), LJ C2
  8 -> 10 A with Coulomb C1 10 A.

Those ConfigTests also run dihedral and improper terms and all-pairs Coulomb, which this path does
not have, so their trajectories are not reproduced here; the force sets above are the
reference's vacuum cutoff forces on their inputs.
"""
import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, HERE)

from make_golden import build_topology, parse_par, parse_pdb_xyz, parse_psf  # noqa: E402
from oracle import oracle as O  # noqa: E402
from protomol3_b200 import waterbox as W  # noqa: E402

SETS = {"lj_c2": (("C2", 8.0, 10.0), None), "lj_c1": (("C1", 0.0, 10.0), None),
        "coul_cut": (None, ("cutoff", 0.0, 10.0)), "lj_c2_coul_c2": (("C2", 8.0, 10.0), ("C2", 8.0, 10.0))}


def droplet():
    box = W.water_box(1000, seed=8)
    c = box["box"] / 2
    pos = box["pos"].reshape(-1, 3, 3)
    keep = np.where(np.linalg.norm(pos[:, 0] - c, axis=1) < 14.0)[0]
    sub = W.water_box(len(keep), seed=8)  # same per-water topology, renumbered
    sub = dict(sub)
    sub["pos"] = pos[keep].reshape(-1, 3)
    sub["vel"] = box["vel"].reshape(-1, 3, 3)[keep].reshape(-1, 3)
    return sub


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("PROTOMOL3_REF"),
                    help="ProtoMol 3 source tree (default: $PROTOMOL3_REF)")
    ref = ap.parse_args().ref
    if not ref:
        raise SystemExit("pass --ref <ProtoMol 3 tree> or set PROTOMOL3_REF")
    if not O.ref_md_available():
        raise SystemExit("oracle/_ref/libpmref_md.so is missing: run make -C oracle ref first")
    d = os.path.join(ref, "protomol-test/ConfigTests/data")
    ala = build_topology(parse_psf(os.path.join(d, "alanine.psf")), parse_par(os.path.join(d, "alanine.par")),
                         "scaled1-4")
    ala["pos"] = parse_pdb_xyz(os.path.join(d, "alanine.pdb"))
    ala["coulomb_scaling"] = 1.0
    out = {}
    for tag, topo, sets in (("ala", ala, SETS), ("drop", droplet(), {"lj_c2_coul_c1": (("C2", 8.0, 10.0), ("C1", 0.0, 10.0))})):
        topo = dict(topo, box=np.array([1000.0, 1000.0, 1000.0]))  # unused by the vacuum forces
        s = O.System(topo)
        for k in ("type", "charge", "mass", "lj", "excl_pairs", "excl_kind", "molecule", "pos"):
            out[tag + "_" + k] = np.asarray(topo[k])
        for name, (lj, coul) in sets.items():
            f, e, v = O.ref_evaluate_vacuum(s, topo["pos"], O.cutoff_params(lj=lj, coul=coul))
            out["%s_%s_forces" % (tag, name)] = f
            out["%s_%s_energies" % (tag, name)] = e
            out["%s_%s_virial" % (tag, name)] = v
    np.savez_compressed(os.path.join(HERE, "vacuum_ref.npz"), **out)


if __name__ == "__main__":
    main()
