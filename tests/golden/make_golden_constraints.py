"""Build the golden fixture that pins SHAKE/RATTLE to ProtoMol's own integrator and modifiers.

Run in a container that holds the ProtoMol 3 source tree, after ``make -C oracle ref`` has
compiled the reference's LeapfrogIntegrator, ModifierShake, ModifierRattle and constraint-list
builder in place into ``oracle/_ref/libpmref_md.so``:

    python tests/golden/make_golden_constraints.py

It writes ``water64_rigid_ref.npz`` next to this script: a seeded box of 64 TIP3P waters (the
generator of ``protomol3_b200.waterbox``, seed 7), the reference's constraint list for it, and
the positions and velocities after ``LeapfrogIntegrator::run(n)`` with no force terms at a 2 fs
step, for four modifier settings (``shake``/``rattle`` with their epsilon and max_iter):

* ``sr``: SHAKE and RATTLE at the defaults (1e-5, 30), 20 steps;
* ``s``: SHAKE alone, 20 steps;
* ``r``: RATTLE alone, 20 steps;
* ``tight``: SHAKE (1e-8, 5) and RATTLE (1e-9, 3), 15 steps, where max_iter ends every
  application before convergence;
* ``lv``: the LangevinLeapfrogIntegrator at temperature 0 (noise term exactly zero) with
  gamma 50/ps, SHAKE and RATTLE at the defaults, 20 steps.

Every case also keeps ``<case>_virial``: the virial the reference's energies hold after the run
(ScalarStructure with virial on; with no force terms, the last RATTLE application's terms).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from protomol3_b200 import waterbox as W  # noqa: E402

CASES = {"sr": ((1e-5, 30), (1e-5, 30), 20), "s": ((1e-5, 30), None, 20),
         "r": (None, (1e-5, 30), 20), "tight": ((1e-8, 5), (1e-9, 3), 15)}


def main():
    if not O.ref_md_available():
        raise SystemExit("oracle/_ref/libpmref_md.so is missing: run make -C oracle ref first")
    box = W.water_box(64, seed=7)
    system = O.System(box)
    out = {"pos0": box["pos"], "vel0": box["vel"], "dt": 2.0}
    for name, (shake, rattle, steps) in CASES.items():
        vir = np.zeros(9)
        pos, vel, cons = O.ref_leapfrog_constrained(system, box["elem"], box["pos"], box["vel"],
                                                    2.0, steps, shake=shake, rattle=rattle, virial=vir)
        out[name + "_pos"], out[name + "_vel"], out[name + "_virial"] = pos, vel, vir
        out[name + "_steps"] = steps
        out[name + "_shake"] = np.array(shake if shake else (0.0, 0))
        out[name + "_rattle"] = np.array(rattle if rattle else (0.0, 0))
        out["con_a1"], out["con_a2"], out["con_len"] = cons
    vir = np.zeros(9)
    pos, vel, cons = O.ref_leapfrog_constrained(system, box["elem"], box["pos"], box["vel"], 2.0, 20,
                                                shake=(1e-5, 30), rattle=(1e-5, 30), langevin=(0.0, 50.0, 1234),
                                                virial=vir)
    out["lv_pos"], out["lv_vel"], out["lv_steps"], out["lv_gamma"], out["lv_virial"] = pos, vel, 20, 50.0, vir
    np.savez_compressed(os.path.join(HERE, "water64_rigid_ref.npz"), **out)


if __name__ == "__main__":
    main()
