"""Allocation-free NonbondedCutoff entry point (pmb_cutoff_evaluate_static) against the allocating
one (pmb_evaluate_device) on the same device positions, two calls in a row, plus its refusals.

The allocation-free pass always computes in FP64 (all pairs, no neighbour list), so against an
FP64 system it agrees to FP64 rounding (sums in another order; forces of pmb_evaluate_device pass
through 2^-40 fixed point) and against a mixed-precision system to the mixed tolerance.
"""
import ctypes as C
import os

import numpy as np
import pytest

from protomol3_b200 import _lib as L
from protomol3_b200 import forces as F
from protomol3_b200 import waterbox as W

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL = {"fp64": 1e-9, "mixed": 1e-5}


def _golden(name, edge):
    d = dict(np.load(os.path.join(GOLD, name)))
    d["box"] = np.array([edge, edge, edge])
    return d


def _case(name):
    if name == "water423_lj_c2_coulomb_c1":
        return ([_golden("water423_periodic.npz", 28.0)],
                F.NonbondedCutoffSystemForce(lj=("C2", 0.1, 6.5), coulomb=("C1", 0.0, 6.5)))
    if name == "pentane320_lj_c2":
        return ([_golden("pentane320_periodic.npz", 23.0)],
                F.NonbondedCutoffSystemForce(lj=("C2", 8.0, 9.0)))
    # two boxes of different sizes in one system
    return ([_golden("water423_periodic.npz", 28.0), W.water_box(100, seed=7)],
            F.NonbondedCutoffSystemForce(lj=("Cutoff", 0.0, 6.0), coulomb=("C2", 4.0, 6.0)))


CASES = ["water423_lj_c2_coulomb_c1", "pentane320_lj_c2", "two_boxes_lj_cutoff_coulomb_c2"]


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _rel_rms(f, ref):
    return float(np.sqrt(((f - ref) ** 2).sum() / (ref ** 2).sum()))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case", CASES)
def test_static_matches_evaluate_device(case, precision):
    import torch
    boxes, force = _case(case)
    topo = F.Topology(boxes, precision)
    h = force.handle(topo)
    n, nb = topo.n_atoms, topo.n_boxes
    dev = torch.device("cuda")
    pos = torch.tensor(topo.positions(), dtype=torch.float64, device=dev)
    f_ref = torch.zeros((n, 3), dtype=torch.float64, device=dev)
    e_ref = torch.zeros(nb * L.E_STRIDE, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    fs = (C.c_void_p * 1)(h)
    L.check(L.lib().pmb_evaluate_device(topo.system(), fs, 1, _ptr(pos), _ptr(f_ref), _ptr(e_ref), 1))
    if L.lib().pmb_system_check(topo.system()) == L.PMB_ERR_CAPACITY:  # lists enlarged: repeat
        L.check(L.lib().pmb_evaluate_device(topo.system(), fs, 1, _ptr(pos), _ptr(f_ref), _ptr(e_ref), 1))
        L.check(L.lib().pmb_system_check(topo.system()))
    torch.cuda.synchronize()
    fr = f_ref.cpu().numpy()
    er = e_ref.cpu().numpy().reshape(nb, L.E_STRIDE)
    tol = TOL[precision]
    for _ in range(2):
        f = torch.full((n, 3), float("nan"), dtype=torch.float64, device=dev)
        e = torch.full((nb * L.E_STRIDE,), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        L.check(L.lib().pmb_cutoff_evaluate_static(h, _ptr(pos), _ptr(f), _ptr(e), 1))
        torch.cuda.synchronize()
        fa = f.cpu().numpy()
        ea = e.cpu().numpy().reshape(nb, L.E_STRIDE)
        assert np.isfinite(fa).all() and np.isfinite(ea).all()
        assert _rel_rms(fa, fr) < tol
        for b in range(nb):
            nab = len(boxes[b]["charge"])
            for slot in (L.E_COULOMB, L.E_LJ):
                assert abs(ea[b, slot] - er[b, slot]) <= tol * abs(er[b, slot]) + nab * 2.0 ** -31
            # virial judged against the magnitude of the tensor (small off-diagonal elements
            # carry the absolute error of the large diagonal ones)
            va, vr = ea[b, L.E_VIRIAL:L.E_VIRIAL + 9], er[b, L.E_VIRIAL:L.E_VIRIAL + 9]
            assert np.abs(va - vr).max() <= 10 * tol * np.abs(vr).max() + 1e-6
            assert ea[b, L.E_BOND] == 0.0 and ea[b, L.E_ANGLE] == 0.0


def test_static_rejects_more_boxes_than_its_scratch():
    import torch
    box = W.water_box(1, seed=3, edge=20.0)
    topo = F.Topology([box] * (L.STATIC_MAX_BOXES + 1), "fp64")
    force = F.NonbondedCutoffSystemForce(lj=("C2", 5.0, 6.0))
    h = force.handle(topo)
    pos = torch.tensor(topo.positions(), dtype=torch.float64, device="cuda")
    f = torch.full((topo.n_atoms, 3), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = L.lib().pmb_cutoff_evaluate_static(h, _ptr(pos), _ptr(f), None, 0)
    assert rc == L.PMB_ERR_CAPACITY
    assert "PMB_STATIC_MAX_BOXES" in L.last_error()
    torch.cuda.synchronize()
    assert np.isnan(f.cpu().numpy()).all()  # nothing ran


def test_static_rejects_pme():
    import torch
    box = W.water_box(64, seed=5)
    topo = F.Topology(box, "fp64")
    pme = F.NonbondedPMEwaldSystemForce(gridsize=(16, 16, 16), cutoff=6.0)
    h = pme.handle(topo)
    pos = torch.tensor(topo.positions(), dtype=torch.float64, device="cuda")
    f = torch.zeros((topo.n_atoms, 3), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    assert L.lib().pmb_cutoff_evaluate_static(h, _ptr(pos), _ptr(f), None, 0) == L.PMB_ERR_UNSUPPORTED


def test_static_first_on_a_fresh_system_and_allocates_nothing():
    """The use the entry point exists for: the first evaluation of a newly made system, with no
    neighbour list allocated yet.  It matches pmb_evaluate_device called afterwards, and once one
    call has run, further calls leave the device's free memory exactly as it was."""
    import torch
    boxes, force = _case("two_boxes_lj_cutoff_coulomb_c2")
    topo = F.Topology(boxes, "fp64")
    h = force.handle(topo)
    n, nb = topo.n_atoms, topo.n_boxes
    dev = torch.device("cuda")
    pos = torch.tensor(topo.positions(), dtype=torch.float64, device=dev)
    f = torch.full((n, 3), float("nan"), dtype=torch.float64, device=dev)
    e = torch.full((nb * L.E_STRIDE,), float("nan"), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    L.check(L.lib().pmb_cutoff_evaluate_static(h, _ptr(pos), _ptr(f), _ptr(e), 1))
    torch.cuda.synchronize()
    fa, ea = f.cpu().numpy(), e.cpu().numpy().reshape(nb, L.E_STRIDE)
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        L.check(L.lib().pmb_cutoff_evaluate_static(h, _ptr(pos), _ptr(f), _ptr(e), 1))
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert np.array_equal(f.cpu().numpy(), fa)
    f_ref = torch.zeros((n, 3), dtype=torch.float64, device=dev)
    e_ref = torch.zeros(nb * L.E_STRIDE, dtype=torch.float64, device=dev)
    fs = (C.c_void_p * 1)(h)
    L.check(L.lib().pmb_evaluate_device(topo.system(), fs, 1, _ptr(pos), _ptr(f_ref), _ptr(e_ref), 1))
    if L.lib().pmb_system_check(topo.system()) == L.PMB_ERR_CAPACITY:
        L.check(L.lib().pmb_evaluate_device(topo.system(), fs, 1, _ptr(pos), _ptr(f_ref), _ptr(e_ref), 1))
        L.check(L.lib().pmb_system_check(topo.system()))
    torch.cuda.synchronize()
    fr, er = f_ref.cpu().numpy(), e_ref.cpu().numpy().reshape(nb, L.E_STRIDE)
    assert _rel_rms(fa, fr) < TOL["fp64"]
    for b in range(nb):
        nab = len(boxes[b]["charge"])
        for slot in (L.E_COULOMB, L.E_LJ):
            assert abs(ea[b, slot] - er[b, slot]) <= TOL["fp64"] * abs(er[b, slot]) + nab * 2.0 ** -31
