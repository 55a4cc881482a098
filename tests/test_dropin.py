"""The ProtoMol plugin classes (protomol3_b200/protomol/B200SystemForces.h) inside the
reference's own ForceFactory (factory/ForceFactory.cpp, compiled from the reference sources into
oracle/_ref/libdropin.so by tests/dropin/Makefile): .conf force definitions resolve to the B200
forces with the reference's parameter parsing and checks.  No device is needed to make a force."""
import ctypes as C
import os

import pytest

LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                   "libdropin.so")
pytestmark = pytest.mark.skipif(not os.path.exists(LIB), reason="drop-in harness not built "
                                "(needs the reference sources)")


def _make(definition):
    L = C.CDLL(LIB)
    L.dropin_make.argtypes = [C.c_char_p, C.c_char_p, C.c_int]
    buf = C.create_string_buffer(4096)
    rc = L.dropin_make(definition.encode(), buf, len(buf))
    return rc, buf.value.decode()


PME = "Coulomb -algorithm PMEwaldB200 -real -reciprocal -correction -interpolation BSpline"


@pytest.mark.parametrize("definition,id_part,params", [
    (PME + " -gridsize 20 20 20 -cutoff 8 -precision mixed",
     PME, ["-gridsize=20", "=20", "-cutoff=8", "-order=4", "-accuracy=1e-06", "-alpha=-1", "-precision=mixed"]),
    (PME + " -switchingFunction C1 -gridsize 24 24 24 -cutoff 9",
     PME + " -switchingFunction C1", ["-gridsize=24", "-cutoff=9", "-precision=fp64"]),
    ("LennardJones Coulomb -algorithm NonbondedCutoffB200 -switchingFunction C2 -switchingFunction C1 "
     "-switchon 0.1 -cutoff 6.5",
     "LennardJones Coulomb -switchingFunction C2 -switchingFunction C1 -algorithm NonbondedCutoffB200",
     ["-switchon=0.1", "-cutoff=6.5", "-precision=fp64"]),
    ("LennardJones -algorithm NonbondedCutoffB200 -switchingFunction C2 -switchon 8 -cutoff 10 -precision mixed",
     "LennardJones -switchingFunction C2 -algorithm NonbondedCutoffB200", ["-switchon=8", "-cutoff=10",
                                                                          "-precision=mixed"]),
])
def test_factory_makes_b200_forces(definition, id_part, params):
    rc, msg = _make(definition)
    assert rc == 0, msg
    assert msg.startswith(id_part)
    for p in params:
        assert p in msg.split(), (p, msg)


@pytest.mark.parametrize("definition", [
    PME + " -gridsize 20 20 20 -cutoff 8 -order 5",       # the reference's doMake: order even
    PME + " -gridsize 20 20 20 -cutoff 8 -order 24",      # order <= grid
    PME + " -gridsize 20 20 20 -cutoff 8 -precision fp16",
])
def test_factory_rejects_what_the_reference_rejects(definition):
    """The rejection goes through the reference's `report << error`, which aborts and leaves the
    process-wide report stream in its error state; so each case runs in a child process."""
    import subprocess
    import sys
    code = ("import sys; sys.path.insert(0, %r); import test_dropin as T; "
            "rc, msg = T._make(%r); print('RC', rc)" % (os.path.dirname(os.path.abspath(__file__)), definition))
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    rcs = [ln.split()[1] for ln in out.stdout.splitlines() if ln.startswith("RC")]
    assert rcs and rcs[0] != "0", out.stdout + out.stderr
