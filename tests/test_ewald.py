"""The exact Ewald reciprocal sum on the CPU: a numpy restatement of
NonbondedFullEwaldSystemForce::reciprocalTerm (force/nonbonded/NonbondedFullEwaldSystemForce.h:
873-1083, k-vectors and default alpha of initialize :590-660), test infrastructure only, against
the reference's own result (golden fixture tests/golden/ewald_ref.npz, made by
make_golden_ewald.py).  Tolerance: 1e-10 relative (the reference forms the sines and cosines by
recurrences, the restatement directly)."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from protomol3_b200 import waterbox as W

GOLD = os.path.join(os.path.dirname(__file__), "golden", "ewald_ref.npz")
CASES = {"w216": (216, 4, -1.0, 1e-6), "w500": (500, 6, 0.35, 1e-5)}


def ewald_reciprocal(box, alpha, accuracy):
    pos, q = box["pos"], box["charge"]
    lx, ly, lz = box["box"]
    V = lx * ly * lz
    lr = np.array([(ly * lz) / (lx * (ly * lz)), (lz * lx) / (ly * (lz * lx)), (lx * ly) / (lz * (lx * ly))])
    a = alpha if alpha > 0 else np.sqrt(np.pi) * (5.5 * len(q) / V ** 2) ** (1.0 / 6.0)
    kc = 2.0 * a * np.sqrt(-np.log(accuracy))
    hmax = [int(np.floor(kc / (2 * np.pi) * L)) for L in (lx, ly, lz)]
    ks = []
    for h in range(0, hmax[0] + 1):
        for k in range(0 if h == 0 else -hmax[1], hmax[1] + 1):
            for l in range(1 if h == 0 and k == 0 else -hmax[2], hmax[2] + 1):
                kv = 2.0 * np.pi * np.array([h, k, l]) * lr
                if kv @ kv < kc * kc:
                    ks.append(kv)
    ks = np.array(ks)
    k2 = (ks ** 2).sum(1)
    b = 1.0 / k2 * np.exp(-k2 / (a * a) / 4.0)
    ph = pos @ ks.T
    sn, cs = q[:, None] * np.sin(ph), q[:, None] * np.cos(ph)
    S, C = sn.sum(0), cs.sum(0)
    e = b * (S * S + C * C)
    f = (8.0 * np.pi / V * b * (sn * C - cs * S)) @ ks
    c = 2.0 * (1.0 / k2 + 1.0 / (4 * a * a))
    vir = np.einsum("k,kij->ij", e, np.eye(3)[None] - c[:, None, None] * ks[:, :, None] * ks[:, None, :])
    return f, 4.0 * np.pi / V * e.sum(), 4.0 * np.pi / V * vir.ravel()


@pytest.mark.parametrize("tag", list(CASES))
def test_restatement_equals_reference(tag):
    g = np.load(GOLD)
    nw, seed, alpha, acc = CASES[tag]
    box = W.water_box(nw, seed=seed)
    assert np.array_equal(box["pos"], g[tag + "_pos"])
    f, e, v = ewald_reciprocal(box, alpha, acc)
    ref = g[tag + "_forces"]
    assert np.sqrt(((f - ref) ** 2).sum() / (ref ** 2).sum()) < 1e-10
    assert abs(e - g[tag + "_energy"]) < 1e-10 * abs(g[tag + "_energy"])
    assert np.allclose(v, g[tag + "_virial"], rtol=1e-9, atol=1e-9)


@pytest.mark.skipif(not O.ref_md_available(), reason="reference Ewald sum not compiled here")
def test_live_reference_equals_fixture():
    g = np.load(GOLD)
    box = W.water_box(216, seed=4)
    f, e, v = O.ref_ewald_reciprocal(O.System(box), box["pos"], -1.0, 1e-6, virial=True)
    assert np.array_equal(f, g["w216_forces"]) and e == g["w216_energy"]
