"""Parity of the CUDA path (through the C ABI) with the CPU oracle and the golden vectors.

Tolerances:
  * FP64 path: relative RMS force error <= 1e-9 and relative energy error <= 1e-9 against the
    FP64 oracle (only summation order and fixed-point accumulation at 2^-40 differ);
  * mixed path: relative RMS force error <= 1e-5 (the target stated for the mixed precision path)
    and relative energy error <= 1e-5;
  * golden water_CHARMM_PERIODIC_L trajectory: absolute 1e-5, ProtoMol's own test tolerance
    (test/test.py:14).
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from protomol3_b200 import forces as F
from protomol3_b200 import waterbox as W

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL = {"fp64": 1e-9, "mixed": 1e-5}


def rel_rms(f, ref):
    return float(np.sqrt(((f - ref) ** 2).sum() / (ref ** 2).sum()))


def energy_ok(e, ref, scale, precision, n_atoms):
    """Energies are totals of terms that cancel (Coulomb: real + reciprocal + intra + self), so the
    error is judged against ``scale`` = the magnitude of the terms computed in the tested precision.
    Fixed-point accumulation adds at most 2^-33 kcal/mol per contribution (FP64 allowance)."""
    return abs(e - ref) <= TOL[precision] * scale + n_atoms * 2.0 ** -31


def gpu_eval(box, force_list, precision, virial=False, positions=None):
    topo = F.Topology(box, precision)
    pos = topo.positions() if positions is None else positions
    frc = np.zeros((topo.n_atoms, 3))
    e = F.ScalarStructure(topo.n_boxes, virial=virial)
    F.evaluate_all(topo, force_list, pos, frc, e)
    return frc, e, topo


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cutoff_golden_water423(precision):
    d = dict(np.load(os.path.join(GOLD, "water423_periodic.npz")))
    d["box"] = np.array([28.0, 28.0, 28.0])
    cut = F.ForceFactory.make("LennardJones Coulomb -algorithm NonbondedCutoff "
                              "-switchingFunction C2 -switchingFunction C1 -switchon 0.1 -cutoff 6.5")
    f, e, _ = gpu_eval(d, [cut, F.BondedSystemForce()], precision, virial=True)
    s = O.System(d)
    fo, eo, vo, _ = O.evaluate(s, d["pos"], cutoff=O.cutoff_params(lj=("C2", 0.1, 6.5),
                                                                   coul=("C1", 0.0, 6.5)),
                               bonded=True, virial=True)
    assert rel_rms(f, fo) < TOL[precision]
    for slot, k in ((F.ScalarStructure.LENNARDJONES, O.E_LJ), (F.ScalarStructure.COULOMB, O.E_COULOMB),
                    (F.ScalarStructure.BOND, O.E_BOND), (F.ScalarStructure.ANGLE, O.E_ANGLE)):
        assert abs(e[slot] - eo[k]) <= TOL[precision] * abs(eo[k]) + 1e-9
    np.testing.assert_allclose(e.virial().ravel(), vo, rtol=10 * TOL[precision], atol=1e-6)
    # and against the reference's own golden step-0 forces (absolute 1e-5)
    if precision == "fp64":
        assert np.abs(f - d["exp_forces0"]).max() < 1e-5


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_pentane_lj_energy(precision):
    d = dict(np.load(os.path.join(GOLD, "pentane320_periodic.npz")))
    lj = F.NonbondedCutoffSystemForce(lj=("C2", 8.0, 9.0))
    f, e, _ = gpu_eval(d, [lj], precision)
    assert abs(e[F.ScalarStructure.LENNARDJONES] - d["exp_lj_energy0"]) < (1e-5 if precision == "fp64" else 1e-3)
    fo, eo, _, _ = O.evaluate(O.System(d), d["pos"], cutoff=O.cutoff_params(lj=("C2", 8.0, 9.0)))
    assert rel_rms(f, fo) < TOL[precision]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("nw,grid,rc", [(216, 20, 8.0), (60, 12, 9.0), (500, 24, 9.0)])
def test_pme_vs_oracle(precision, nw, grid, rc):
    b = W.water_box(nw, seed=5)
    pme = F.NonbondedPMEwaldSystemForce((grid,) * 3, rc)
    f, e, topo = gpu_eval(b, [pme], precision, virial=True)
    fo, eo, vo, info = O.evaluate(O.System(b), b["pos"], pme=O.pme_params((grid,) * 3, rc), virial=True)
    assert abs(pme.alpha(topo) - info["alpha"]) < 1e-15
    assert rel_rms(f, fo) < TOL[precision]
    real, recip = info["terms"][0], info["terms"][1]
    assert energy_ok(e[F.ScalarStructure.COULOMB], eo[O.E_COULOMB], abs(real) + abs(recip),
                     precision, topo.n_atoms)
    np.testing.assert_allclose(e.virial().ravel(), vo, rtol=0, atol=TOL[precision] * np.abs(vo).max() * 10)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("grid,order", [((25, 18, 32), 6), ((27, 16, 30), 8), ((64, 96, 40), 4),
                                        ((32, 160, 96), 4), ((128, 32, 32), 4), ((40, 64, 160), 4),
                                        ((96, 128, 128), 4)])
def test_pme_anisotropic_grid_and_order(precision, grid, order):
    """Grid lengths of pure radix 5, 3 and 2 in different dimensions and interpolation orders
    other than 4 (the generic spread/gather instance); lengths of 32 R points (R = 1 to 5) take
    the warp-shuffle transforms in that dimension, the others the shared-memory ones."""
    b = W.water_box(216, seed=11)
    pme = F.NonbondedPMEwaldSystemForce(grid, 8.0, order=order)
    f, e, topo = gpu_eval(b, [pme], precision, virial=True)
    fo, eo, vo, info = O.evaluate(O.System(b), b["pos"], pme=O.pme_params(grid, 8.0, order=order),
                                  virial=True)
    assert rel_rms(f, fo) < TOL[precision]
    real, recip = info["terms"][0], info["terms"][1]
    assert energy_ok(e[F.ScalarStructure.COULOMB], eo[O.E_COULOMB], abs(real) + abs(recip),
                     precision, topo.n_atoms)
    np.testing.assert_allclose(e.virial().ravel(), vo, rtol=0, atol=TOL[precision] * np.abs(vo).max() * 10)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_lj_plus_pme_fused(precision):
    """LJ C2 8->10 with PME real space 10 A, the config-2 force set, on a 1,000-water box."""
    b = W.water_box(1000, seed=9)
    grid = W.pme_grid_for(b["box"][0])
    lj = F.ForceFactory.make("LennardJones -algorithm NonbondedCutoff -switchingFunction C2 "
                             "-switchon 8 -cutoff 10")
    pme = F.ForceFactory.make("Coulomb -algorithm PMEwald -real -reciprocal -correction "
                              "-interpolation BSpline -gridsize %d %d %d -cutoff 10 -order 4 "
                              "-accuracy 1e-6" % (grid, grid, grid))
    f, e, topo = gpu_eval(b, [lj, pme, F.BondedSystemForce()], precision)
    s = O.System(b)
    fo, eo, _, info = O.evaluate(s, b["pos"], cutoff=O.cutoff_params(lj=("C2", 8.0, 10.0)),
                                 pme=O.pme_params((grid,) * 3, 10.0), bonded=True)
    assert rel_rms(f, fo) < TOL[precision]
    assert energy_ok(e[F.ScalarStructure.LENNARDJONES], eo[O.E_LJ], abs(eo[O.E_LJ]), precision,
                     topo.n_atoms)
    assert energy_ok(e[F.ScalarStructure.COULOMB], eo[O.E_COULOMB],
                     abs(info["terms"][0]) + abs(info["terms"][1]), precision, topo.n_atoms)


def test_mixed_bit_reproducible():
    b = W.water_box(2000, seed=21)
    grid = W.pme_grid_for(b["box"][0])
    fl = [F.NonbondedCutoffSystemForce(lj=("C2", 8.0, 10.0)),
          F.NonbondedPMEwaldSystemForce((grid,) * 3, 10.0), F.BondedSystemForce()]
    topo = F.Topology(b, "mixed")
    outs = []
    for _ in range(3):
        frc = np.zeros((topo.n_atoms, 3))
        e = F.ScalarStructure(1)
        F.evaluate_all(topo, fl, topo.positions(), frc, e)
        outs.append((frc.copy(), e.table.copy()))
    for frc, et in outs[1:]:
        assert np.array_equal(frc, outs[0][0])
        assert np.array_equal(et, outs[0][1])


def test_leapfrog_golden_trajectory_fp64():
    """200 leapfrog steps of water_CHARMM_PERIODIC_L on the device vs the reference's output."""
    d = dict(np.load(os.path.join(GOLD, "water423_periodic.npz")))
    topo = F.Topology(d, "fp64")
    cut = F.NonbondedCutoffSystemForce(lj=("C2", 0.1, 6.5), coulomb=("C1", 0.0, 6.5))
    md = F.Integrator(topo, [F.BondedSystemForce(), cut], timestep=0.5)
    md.set_state(d["pos"], d["vel"])
    assert np.abs(md.forces_now() - d["exp_forces0"]).max() < 1e-5
    md.run(200)
    pos, vel = md.state()
    assert np.abs(pos - d["exp_pos"]).max() < 1e-5
    assert np.abs(vel - d["exp_vel"]).max() < 1e-5
    assert np.abs(md.forces_now() - d["exp_forces_end"]).max() < 1e-5
    e, _ = md.energies()
    row = d["exp_energy"][1]
    np.testing.assert_allclose(e[0, [2, 3, 1, 0]], row[[5, 6, 9, 10]], rtol=1e-7, atol=1e-4)


@pytest.mark.parametrize("graph", [True, False])
def test_leapfrog_matches_oracle_pme(graph):
    b = W.water_box(216, seed=2)
    topo = F.Topology(b, "fp64")
    fl = [F.BondedSystemForce(), F.NonbondedCutoffSystemForce(lj=("C2", 7.0, 8.0)),
          F.NonbondedPMEwaldSystemForce((20, 20, 20), 8.0)]
    md = F.Integrator(topo, fl, timestep=1.0, use_graph=graph)
    md.set_state(b["pos"], b["vel"])
    md.run(20)
    pos, vel = md.state()
    po, vo, _, _ = O.leapfrog(O.System(b), b["pos"], b["vel"], 1.0, 20,
                              cutoff=O.cutoff_params(lj=("C2", 7.0, 8.0)),
                              pme=O.pme_params((20, 20, 20), 8.0))
    assert np.abs(pos - po).max() < 1e-8
    assert np.abs(vel - vo).max() < 1e-8


@pytest.fixture(scope="module")
def water98k():
    """The full 98,304-atom box (32,768 waters, 96^3 grid, rc 10, LJ C2 8->10) and the oracle's
    forces, energies and terms on it (computed once for both precisions)."""
    b = W.water_box(32768, seed=1234)
    fo, eo, _, info = O.evaluate(O.System(b), b["pos"], cutoff=O.cutoff_params(lj=("C2", 8.0, 10.0)),
                                 pme=O.pme_params((96, 96, 96), 10.0))
    return b, fo, eo, info


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_water98k_size_vs_oracle(water98k, precision):
    """The plain FP64 path (the drop-in) and the mixed path at full size, against the oracle."""
    b, fo, eo, info = water98k
    lj = F.NonbondedCutoffSystemForce(lj=("C2", 8.0, 10.0))
    pme = F.NonbondedPMEwaldSystemForce((96, 96, 96), 10.0)
    f, e, topo = gpu_eval(b, [lj, pme], precision)
    assert rel_rms(f, fo) < TOL[precision]
    assert energy_ok(e[F.ScalarStructure.COULOMB], eo[O.E_COULOMB],
                     abs(info["terms"][0]) + abs(info["terms"][1]), precision, topo.n_atoms)
    assert energy_ok(e[F.ScalarStructure.LENNARDJONES], eo[O.E_LJ], abs(eo[O.E_LJ]), precision,
                     topo.n_atoms)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batched_ensemble_subset_vs_oracle(precision):
    """Boxes of the ensemble workload (LJ C2 7.5 -> 9 A, PME rc 9 A at ~1 A grid spacing,
    order 4, bonded) advanced as one batched system, each compared with the oracle evaluated on
    that box alone.  Four of the six are under twice the cutoff (100-190 waters, 14.4-17.8 A),
    where the reference's cutoff LJ takes a single minimal image (force/OneAtomPair.h:55-57) and
    PME's real term sums lattice images."""
    boxes = [W.water_box(n, seed=60 + n) for n in (100, 120, 150, 190, 450, 1300)]
    grids = [W.pme_grid_for(b["box"][0]) for b in boxes]
    fl = [F.NonbondedCutoffSystemForce(lj=("C2", 7.5, 9.0)),
          F.NonbondedPMEwaldSystemForce((0, 0, 0), 9.0, box_grids=[[g] * 3 for g in grids]),
          F.BondedSystemForce()]
    fb, eb, topo = gpu_eval(boxes, fl, precision, virial=True)
    off = 0
    for k, (b, g) in enumerate(zip(boxes, grids)):
        n = len(b["charge"])
        fo, eo, vo, info = O.evaluate(O.System(b), b["pos"], cutoff=O.cutoff_params(lj=("C2", 7.5, 9.0)),
                                      pme=O.pme_params((g,) * 3, 9.0), bonded=True, virial=True)
        assert rel_rms(fb[off:off + n], fo) < TOL[precision], k
        assert energy_ok(eb.table[k, F.ScalarStructure.LENNARDJONES], eo[O.E_LJ], abs(eo[O.E_LJ]),
                         precision, n), k
        assert energy_ok(eb.table[k, F.ScalarStructure.COULOMB], eo[O.E_COULOMB],
                         abs(info["terms"][0]) + abs(info["terms"][1]), precision, n), k
        for slot, j in ((F.ScalarStructure.BOND, O.E_BOND), (F.ScalarStructure.ANGLE, O.E_ANGLE)):
            assert abs(eb.table[k, slot] - eo[j]) <= 1e-9 * abs(eo[j]) + n * 2.0 ** -31, k
        np.testing.assert_allclose(eb.virial(k).ravel(), vo, rtol=0,
                                   atol=10 * TOL[precision] * np.abs(vo).max(), err_msg=str(k))
        off += n


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_pme_charged_box_vs_oracle(precision):
    """A box with a net charge of -0.834 e: the charged-system energy
    -pi (sum q)^2 / (2 V alpha^2) of NonbondedPMEwaldSystemForce.h:555-575 enters the Coulomb
    energy (oracle pinned to the compiled reference in tests/test_oracle.py)."""
    b = dict(W.water_box(216, seed=13))
    q = b["charge"].copy()
    q[1] = q[2] = 0.0
    b["charge"] = q
    pme = F.NonbondedPMEwaldSystemForce((20, 20, 20), 8.0)
    f, e, topo = gpu_eval(b, [pme], precision, virial=True)
    fo, eo, vo, info = O.evaluate(O.System(b), b["pos"], pme=O.pme_params((20, 20, 20), 8.0), virial=True)
    # the charged term is present: -pi (sum q)^2 / (2 V alpha^2) = -0.36 kcal/mol here
    assert info["terms"][4] < -0.3
    assert rel_rms(f, fo) < TOL[precision]
    assert energy_ok(e[F.ScalarStructure.COULOMB], eo[O.E_COULOMB],
                     abs(info["terms"][0]) + abs(info["terms"][1]), precision, topo.n_atoms)
    np.testing.assert_allclose(e.virial().ravel(), vo, rtol=0, atol=TOL[precision] * np.abs(vo).max() * 10)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_list_reuse_with_skin_matches_rebuild_every_step(precision):
    """A Verlet skin changes which pairs are tested, never which are evaluated."""
    b = W.water_box(1500, seed=41)
    grid = W.pme_grid_for(b["box"][0])

    def run(skin):
        topo = F.Topology(b, precision)
        topo.set_skin(skin)
        fl = [F.BondedSystemForce(), F.NonbondedCutoffSystemForce(lj=("C2", 8.0, 10.0)),
              F.NonbondedPMEwaldSystemForce((grid,) * 3, 10.0)]
        md = F.Integrator(topo, fl, timestep=1.0)
        md.set_state(b["pos"], b["vel"])
        md.run(40)
        pos, vel = md.state()
        return pos, md.forces_now()
    p0, f0 = run(0.0)
    p1, f1 = run(0.6)
    # FP64: only summation order differs; FP32: per-tile rounding differences grow along the
    # (chaotic) trajectory, so the bound is the size of that growth after 40 steps
    tol = 1e-9 if precision == "fp64" else 2e-3
    assert np.abs(p1 - p0).max() < tol
    assert rel_rms(f1, f0) < (1e-9 if precision == "fp64" else 1e-3)


def test_profile_needs_positions():
    """pmb_profile on a system that never received positions is an error, not a silent run on
    uninitialised device memory; with positions it reports every pipeline stage."""
    from protomol3_b200 import _lib as L
    b = W.water_box(216, seed=4)
    topo = F.Topology(b, "mixed")
    fl = [F.NonbondedCutoffSystemForce(lj=("C2", 7.0, 8.0)),
          F.NonbondedPMEwaldSystemForce((20, 20, 20), 8.0), F.BondedSystemForce()]
    with pytest.raises(L.PMBError) as err:
        F.profile(topo, fl, nrep=2)
    assert err.value.code == L.PMB_ERR_STATE
    st = F.profile(topo, fl, positions=topo.positions(), nrep=2)
    for stage in ("nblist", "pair", "pme_spread", "pme_fft", "pme_gather", "bonded"):
        assert stage in st and st[stage] >= 0.0



def pinned_array(shape, fill):
    """A numpy view of page-locked host memory (what a caller gets from cudaMallocHost)."""
    import torch
    a = torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()
    a[...] = fill
    return a


@pytest.mark.parametrize("pinned_positions", [False, True])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("n_waters", [216, 27000])
def test_page_locked_force_array_gets_the_same_sum(precision, n_waters, pinned_positions):
    """A page-locked force array is added to on the device and copied back into directly (with
    page-locked positions too, every copy is a node of the evaluation's graph); a pageable one
    receives the forces in a host staging buffer and is added to on the host.  Both add the same
    two doubles per component, so the results are equal bit for bit, evaluation after evaluation
    (the graphed evaluation is replayed), and the energies too."""
    b = W.water_box(n_waters, seed=11)
    edge = b["box"][0]
    grid = W.pme_grid_for(edge)
    fl = [F.NonbondedCutoffSystemForce(lj=("C2", 7.0, 8.0)),
          F.NonbondedPMEwaldSystemForce((grid,) * 3, 8.0), F.BondedSystemForce()]
    topo = F.Topology(b, precision)
    rng = np.random.default_rng(3)
    pos = b["pos"].copy()
    pb = pinned_array(pos.shape, pos) if pinned_positions else None
    for it in range(3):
        start = rng.normal(size=(topo.n_atoms, 3))
        fa, fb = start.copy(), pinned_array((topo.n_atoms, 3), start)
        ea, eb = F.ScalarStructure(1, virial=True), F.ScalarStructure(1, virial=True)
        F.evaluate_all(topo, fl, pos, fa, ea)
        if pb is not None:
            pb[...] = pos
        F.evaluate_all(topo, fl, pos if pb is None else pb, fb, eb)
        assert np.array_equal(fa, fb)
        assert np.array_equal(ea.table, eb.table)
        assert not np.array_equal(fa, start)
        pos = pos + rng.uniform(-0.02, 0.02, pos.shape)
    topo.close()


def test_systems_with_page_locked_evaluations_free_their_device_memory():
    """A system that added forces to a page-locked array on the device (which needs a device copy
    of the array) gives every byte back when it is destroyed: eight systems of 60,000 atoms made,
    evaluated and destroyed one after another leave the device's free memory where the first left
    it (each one's copy of the forces alone is 1.44 MB)."""
    import torch
    b = W.water_box(20000, seed=12)
    fl = [F.NonbondedCutoffSystemForce(lj=("C2", 7.0, 8.0))]

    def cycle():
        topo = F.Topology(b, "mixed")
        frc = pinned_array((topo.n_atoms, 3), 0.0)
        F.evaluate_all(topo, fl, b["pos"], frc, F.ScalarStructure(1))
        assert np.abs(frc).max() > 0
        topo.close()
    cycle()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(8):
        cycle()
    torch.cuda.synchronize()
    assert free0 - torch.cuda.mem_get_info()[0] <= 4 << 20


@pytest.mark.parametrize("pinned", [False, True, "both"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_non_finite_position_is_an_error_and_changes_nothing(precision, pinned):
    """A NaN or infinite position gives PMB_ERR_NUMERIC and leaves the caller's forces and
    energies as they were, whether the list kernels saw it on the device (pair and PME forces) or
    the host did (bonded terms alone, no list), and whether the force array is pageable or
    page-locked (added to on the device), with the positions page-locked as well ("both": every
    copy inside the evaluation's graph); the next finite evaluation is right again."""
    from protomol3_b200 import _lib as L
    b = dict(W.water_box(216, seed=4))
    # off the waters' rest geometry, so that the bonded forces are not zero
    b["pos"] = b["pos"] + np.random.default_rng(4).uniform(-0.05, 0.05, b["pos"].shape)
    fl = [F.NonbondedCutoffSystemForce(lj=("C2", 7.0, 8.0)),
          F.NonbondedPMEwaldSystemForce((20, 20, 20), 8.0), F.BondedSystemForce()]
    for forces, bad in ((fl, np.nan), (fl, np.inf), ([F.BondedSystemForce()], -np.inf)):
        topo = F.Topology(b, precision)
        pos = pinned_array(b["pos"].shape, b["pos"]) if pinned == "both" else b["pos"].copy()
        pos[5, 1] = bad
        frc = pinned_array((topo.n_atoms, 3), 7.0) if pinned else np.full((topo.n_atoms, 3), 7.0)
        e = F.ScalarStructure(1)
        with pytest.raises(L.PMBError) as err:
            F.evaluate_all(topo, forces, pos, frc, e)
        assert err.value.code == L.PMB_ERR_NUMERIC
        assert (frc == 7.0).all() and (e.table == 0).all()
        frc[:] = 0.0
        F.evaluate_all(topo, forces, b["pos"], frc, e)
        fo = np.zeros_like(frc)
        for fc in forces:
            if isinstance(fc, F.BondedSystemForce):
                fo += O.evaluate(O.System(b), b["pos"], bonded=True)[0]
            elif isinstance(fc, F.NonbondedCutoffSystemForce):
                fo += O.evaluate(O.System(b), b["pos"], cutoff=O.cutoff_params(lj=("C2", 7.0, 8.0)))[0]
            else:
                fo += O.evaluate(O.System(b), b["pos"], pme=O.pme_params((20, 20, 20), 8.0))[0]
        assert rel_rms(frc, fo) < TOL[precision]
        topo.close()


def test_list_tiles_cover_every_pair_within_the_cutoff():
    """pmb_system_list_tiles: the list's pair slots (256 per tile) hold every pair within the
    cutoff (the pairs are listed once each) and no more than a few times their number."""
    b = W.water_box(500, seed=21)
    rc = 9.0
    topo = F.Topology(b, "mixed")
    assert topo.list_tiles() == 0  # no list yet
    f = np.zeros((topo.n_atoms, 3))
    F.evaluate_all(topo, [F.NonbondedCutoffSystemForce(lj=("C2", 7.5, rc))], b["pos"], f, F.ScalarStructure(1))
    slots = 256 * topo.list_tiles()
    L = b["box"][0]
    x = b["pos"]
    d = x[:, None, :] - x[None, :, :]
    d -= L * np.rint(d / L)
    r2 = (d ** 2).sum(-1)
    pairs = int(((r2 <= rc * rc).sum() - len(x)) // 2)
    assert pairs <= slots <= 4 * pairs, (pairs, slots)
    topo.close()
