"""Build the golden fixture that pins the exact Ewald reciprocal check path to ProtoMol's own.

Run in a container that holds the ProtoMol 3 source tree, after ``make -C oracle ref`` has
compiled NonbondedFullEwaldSystemForce in place (``oracle/_ref/libpmref_md.so``, harness
``oracle/ref_ewald.cpp``):

    python tests/golden/make_golden_ewald.py

It writes ``ewald_ref.npz`` next to this script: the reference's reciprocal-only Ewald forces,
Coulomb energy and virial for two seeded TIP3P boxes (``protomol3_b200.waterbox``):

* ``w216``: 216 waters (18.6 A), the reference's default alpha (-1) and accuracy 1e-6;
* ``w500``: 500 waters, alpha 0.35 and accuracy 1e-5, with the virial.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402
from protomol3_b200 import waterbox as W  # noqa: E402

CASES = {"w216": (216, 4, -1.0, 1e-6), "w500": (500, 6, 0.35, 1e-5)}


def main():
    if not O.ref_md_available():
        raise SystemExit("oracle/_ref/libpmref_md.so is missing: run make -C oracle ref first")
    out = {}
    for tag, (nw, seed, alpha, acc) in CASES.items():
        box = W.water_box(nw, seed=seed)
        f, e, v = O.ref_ewald_reciprocal(O.System(box), box["pos"], alpha, acc, virial=True)
        out[tag + "_forces"], out[tag + "_energy"], out[tag + "_virial"] = f, e, v
        out[tag + "_pos"] = box["pos"]
    np.savez_compressed(os.path.join(HERE, "ewald_ref.npz"), **out)


if __name__ == "__main__":
    main()
