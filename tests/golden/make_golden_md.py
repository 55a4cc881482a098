"""Build the golden fixture that pins the integrators to ProtoMol's own LeapfrogIntegrator and
LangevinLeapfrogIntegrator, run with force terms.

Run in a container that holds the ProtoMol 3 source tree, after ``make -C oracle ref`` has
compiled the reference's integrators and forces in place into ``oracle/_ref/``:

    python tests/golden/make_golden_md.py

It writes ``water216_md_ref.npz`` next to this script.  The system is the 216-water TIP3P box
of the one-GPU plain-method workload (``protomol3_b200.waterbox``, seed 1234, 18.62 A edge) with
the reference's ``force LennardJones Coulomb -algorithm NonbondedCutoff`` (C2 switching 7 -> 8 A
for both, module/NonbondedCutoffForceModule.cpp:58-88) plus the bond and angle forces.  The
reference steps by run(1), as ProtoMolApp does with outputfreq 1:

* ``lf_*``: LeapfrogIntegrator, 1 fs, 1,000 steps: the energies of every step (Coulomb, LJ,
  bond, angle), positions and velocities after steps 10, 50 and 100, forces at steps 0 and 100;
* ``lv1_*`` / ``lv50_*``: LangevinLeapfrogIntegrator at temperature 0 (the noise term is then
  exactly zero, so the run does not depend on the reference's serial random generator) with
  gamma 1/ps and 50/ps, 1 fs, 100 steps: energies of every step, positions and velocities after
  steps 10 and 100.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from protomol3_b200 import waterbox as W  # noqa: E402

LF_STEPS, LF_KEEP, LF_FORCES = 1000, (10, 50, 100), (0, 100)
LV_STEPS, LV_KEEP, LV_GAMMAS = 100, (10, 100), (1.0, 50.0)


def cutoff():
    return O.cutoff_params(lj=("C2", 7.0, 8.0), coul=("C2", 7.0, 8.0))


def main():
    if not O.ref_md_available():
        raise SystemExit("oracle/_ref/libpmref_md.so is missing: run make -C oracle ref first")
    box = W.water_box(216, seed=1234)
    system = O.System(box)
    out = {"pos0": box["pos"], "vel0": box["vel"], "dt": 1.0}
    r = O.ref_md_run(system, box["pos"], box["vel"], 1.0, LF_STEPS, cutoff=cutoff(), bonded=True,
                     keep=("energies", "pos", "vel", "forces"))
    out["lf_energies"] = r["energies"]
    out["lf_keep"] = np.array(LF_KEEP)
    out["lf_pos"] = r["pos"][list(LF_KEEP)]
    out["lf_vel"] = r["vel"][list(LF_KEEP)]
    out["lf_force_steps"] = np.array(LF_FORCES)
    out["lf_forces"] = r["forces"][list(LF_FORCES)]
    for g in LV_GAMMAS:
        r = O.ref_md_run(system, box["pos"], box["vel"], 1.0, LV_STEPS, cutoff=cutoff(), bonded=True,
                         langevin=(0.0, g, 1234), keep=("energies", "pos", "vel"))
        k = "lv%d_" % int(g)
        out[k + "energies"] = r["energies"]
        out[k + "pos"] = r["pos"][list(LV_KEEP)]
        out[k + "vel"] = r["vel"][list(LV_KEEP)]
    out["lv_keep"] = np.array(LV_KEEP)
    out["lv_gammas"] = np.array(LV_GAMMAS)
    np.savez_compressed(os.path.join(HERE, "water216_md_ref.npz"), **out)


if __name__ == "__main__":
    main()
