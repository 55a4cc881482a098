"""CPU-side checks of the C ABI library and the host mirror (no GPU work is launched here)."""
import os
import re

import numpy as np
import pytest

from protomol3_b200 import _lib as L
from protomol3_b200 import forces as F
from protomol3_b200 import waterbox as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "pmb200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pmb_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = L.lib()
    names = header_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    # and the ctypes prototypes cover the header exactly
    assert sorted(p[0] for p in L._PROTOS) == names


def test_no_device_is_reported_not_faked():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    assert L.lib().pmb_device_count() == 0
    topo = F.Topology(W.water_box(10), "mixed")
    with pytest.raises(L.PMBError) as ei:
        topo.system()
    assert "no CUDA device" in str(ei.value)


def test_force_factory_parses_reference_definitions():
    f = F.ForceFactory.make("LennardJones Coulomb -algorithm NonbondedCutoff -switchingFunction C2 "
                            "-switchingFunction C1 -switchon 0.1 -cutoff 6.5")
    assert isinstance(f, F.NonbondedCutoffSystemForce)
    assert (f.desc.lj, f.desc.lj_switch, f.desc.lj_switchon, f.desc.lj_cutoff) == (1, 2, 0.1, 6.5)
    assert (f.desc.coulomb, f.desc.coulomb_switch, f.desc.coulomb_cutoff) == (1, 1, 6.5)
    p = F.ForceFactory.make("Coulomb -algorithm PMEwald -real -reciprocal -correction "
                            "-interpolation BSpline -gridsize 96 96 96 -cutoff 10 -order 4 -accuracy 1e-6")
    assert isinstance(p, F.NonbondedPMEwaldSystemForce)
    assert list(p.desc.grid) == [96, 96, 96] and p.desc.cutoff == 10 and p.desc.order == 4
    assert (p.desc.real, p.desc.reciprocal, p.desc.correction) == (1, 1, 1)
    r = F.ForceFactory.make("Coulomb -algorithm PMEwald -real -gridsize 8 8 8 -cutoff 6")
    assert (r.desc.real, r.desc.reciprocal, r.desc.correction) == (1, 0, 0)
    assert isinstance(F.ForceFactory.make("Bond, Angle"), F.BondedSystemForce)
    for bad in ("LennardJones -algorithm NonbondedCutoff -switchingFunction C9 -cutoff 8",
                "Coulomb -algorithm PMEwald -gridsize 8 8 -cutoff 6",
                "Dihedral", "LennardJones -algorithm FullEwald"):
        with pytest.raises(ValueError):
            F.ForceFactory.make(bad)


def test_water_box_generator():
    b = W.water_box(216, seed=1234)
    assert len(b["charge"]) == 648
    assert abs(b["box"][0] - 18.62) < 0.01
    assert abs(b["charge"].sum()) < 1e-9
    pos = b["pos"].reshape(-1, 3, 3)
    roh = np.linalg.norm(pos[:, 1] - pos[:, 0], axis=1)
    assert np.allclose(roh, 0.9572)
    mom = (b["vel"] * b["mass"][:, None]).sum(0)
    assert np.abs(mom).max() < 1e-9
    assert W.fft_friendly(97) == 100 and W.fft_friendly(96) == 96
    assert W.pme_grid_for(99.34) == 100
