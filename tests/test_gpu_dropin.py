"""Drop-in parity: a .conf force definition made by the reference's own ForceFactory into the
ProtoMol plugin classes (protomol3_b200/protomol/B200SystemForces.h) and evaluated through
SystemForce::evaluate on the reference's own Topology, against the reference's CPU force
(oracle/_ref/libpmref.so) on the same topology and positions.

Tolerances: fp64 1e-9 relative RMS force, 1e-9 relative energy; mixed 1e-5."""
import ctypes as C
import os

import numpy as np
import pytest

from oracle import oracle as O
from protomol3_b200 import waterbox as W

pytestmark = pytest.mark.gpu
LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                   "libdropin.so")
TOL = {"fp64": 1e-9, "mixed": 1e-5}
PME = "Coulomb -algorithm PMEwaldB200 -real -reciprocal -correction -interpolation BSpline"


def _dropin(system, pos, definition, repeat=1):
    if not os.path.exists(LIB) or not O.ref_available():
        pytest.skip("drop-in harness not built (needs the reference sources)")
    L = C.CDLL(LIB)
    L.dropin_eval.argtypes = [C.c_void_p, C.c_char_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                              C.c_char_p, C.c_int]
    r = O._ref_input(system, np.ascontiguousarray(pos, np.float64), 5.0)
    n = system.n
    f, e, v = np.zeros((n, 3)), np.zeros(2), np.zeros(9)
    msg = C.create_string_buffer(2048)
    rc = L.dropin_eval(C.addressof(r), definition.encode(), repeat, f.ctypes.data, e.ctypes.data,
                       v.ctypes.data, msg, len(msg))
    assert rc == 0, msg.value.decode()
    return f, e, v, msg.value.decode()


def _rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_pme_through_the_reference_factory(precision):
    b = W.water_box(216, seed=5)
    s = O.System(b)
    f, e, v, made = _dropin(s, b["pos"], PME + " -gridsize 20 20 20 -cutoff 8 -precision " + precision,
                            repeat=2)
    assert made.startswith(PME)
    fr, er, vr = O.ref_evaluate(s, b["pos"], pme=O.pme_params((20, 20, 20), 8.0), virial=True)
    assert _rel(f, fr) < TOL[precision]
    # Coulomb is real + reciprocal + intra-molecular + self, terms that cancel (here 28 + 351 +
    # 16,246 - 16,663 = -39): the real and reciprocal terms are computed in the tested precision
    # and judged against their magnitudes; the correction and self terms are FP64 in both
    # precisions (1e-12 of theirs); plus the fixed-point resolution
    _, _, _, info = O.evaluate(s, b["pos"], pme=O.pme_params((20, 20, 20), 8.0))
    t = np.abs(info["terms"])
    assert abs(e[0] - er[0]) <= TOL[precision] * (t[0] + t[1]) + 1e-12 * (t[2] + t[3]) + s.n * 2.0 ** -31
    np.testing.assert_allclose(v, vr, rtol=0, atol=10 * TOL[precision] * np.abs(vr).max() + 1e-6)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cutoff_lj_coulomb_through_the_reference_factory(precision):
    b = W.water_box(216, seed=3)
    s = O.System(b)
    f, e, v, made = _dropin(s, b["pos"], "LennardJones Coulomb -algorithm NonbondedCutoffB200 "
                            "-switchingFunction C2 -switchingFunction C2 -switchon 7 -cutoff 8 "
                            "-precision " + precision)
    assert "NonbondedCutoffB200" in made
    fr, er, vr = O.ref_evaluate(s, b["pos"], cutoff=O.cutoff_params(lj=("C2", 7.0, 8.0),
                                                                     coul=("C2", 7.0, 8.0)), virial=True)
    assert _rel(f, fr) < TOL[precision]
    for k in (0, 1):
        assert abs(e[k] - er[k]) < TOL[precision] * abs(er[k]) + 1e-6
