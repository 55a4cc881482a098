"""Seeded synthetic periodic boxes of flexible TIP3P water.

The generator produces the inputs the benchmark and the parity tests run on:

* geometry and force-field constants are CHARMM TIP3 values as they appear in ProtoMol's
  ``par_all27_prot_lipid.inp`` (bond OT-HT 450 kcal/mol/A^2 at 0.9572 A, angle HT-OT-HT
  55 kcal/mol/rad^2 at 104.52 deg, OT eps -0.1521 Rmin/2 1.7682, HT eps -0.046 Rmin/2 0.2245)
  and charges O -0.834 / H +0.417, masses 15.9994 / 1.008;
* molecules sit on a cubic lattice with uniform jitter of +-0.1 lattice spacing and a uniform
  random orientation (random unit quaternion), edge L = (29.915 * n_waters)^(1/3) A
  (1.0 g/cm^3);
* velocities are Maxwell-Boltzmann at the requested temperature with the centre-of-mass
  motion removed, in ProtoMol's internal units (A per internal time unit, where one internal
  time unit is 48.88821290839616 fs; base/PMConstants.cpp:53).

The topology dict uses the reference's conventions (scaled charge = e * 18.2226123264,
CHARMM mixing for the LJ table, exclusion scheme scaled1-4 which makes the three intra-water
pairs FULL exclusions) so the same dict feeds the CUDA path, the CPU oracle and the
compiled-reference harness.
"""
import numpy as np

SQRTCOULOMBCONSTANT = 18.2226123264
BOLTZMANN = 0.001987191
TIMEFACTOR = 48.88821290839616
VOLUME_PER_WATER = 29.915

OT_EPS, OT_RMIN2 = -0.1521, 1.7682
HT_EPS, HT_RMIN2 = -0.046, 0.2245
ROH, THETA_HOH = 0.9572, 104.52
MASS_O, MASS_H = 15.9994, 1.008
Q_O, Q_H = -0.834, 0.417


def lj_table():
    par = [(OT_EPS, OT_RMIN2), (HT_EPS, HT_RMIN2)]
    lj = np.zeros((2, 2, 4))
    for i, (ei, ri) in enumerate(par):
        for j, (ej, rj) in enumerate(par):
            r, e = ri + rj, np.sqrt(ei * ej)
            lj[i, j] = (r ** 12 * e, 2 * r ** 6 * e, r ** 12 * e, 2 * r ** 6 * e)
    return lj


def box_edge(n_waters):
    return (VOLUME_PER_WATER * n_waters) ** (1.0 / 3.0)


def _random_rotations(rng, n):
    u = rng.random((n, 3))
    q = np.stack([np.sqrt(1 - u[:, 0]) * np.sin(2 * np.pi * u[:, 1]),
                  np.sqrt(1 - u[:, 0]) * np.cos(2 * np.pi * u[:, 1]),
                  np.sqrt(u[:, 0]) * np.sin(2 * np.pi * u[:, 2]),
                  np.sqrt(u[:, 0]) * np.cos(2 * np.pi * u[:, 2])], axis=1)
    x, y, z, w = q.T
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1)], 1)


def water_box(n_waters, seed=1234, temperature=300.0, edge=None):
    """Topology + state dict for ``n_waters`` flexible TIP3P waters (3 atoms each)."""
    rng = np.random.default_rng(seed)
    L = box_edge(n_waters) if edge is None else float(edge)
    m = int(np.ceil(n_waters ** (1.0 / 3.0) - 1e-9))
    spacing = L / m
    sites = np.stack(np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij"),
                     -1).reshape(-1, 3)
    sites = sites[rng.permutation(len(sites))[:n_waters]]
    centres = (sites + 0.5) * spacing + rng.uniform(-0.1, 0.1, (n_waters, 3)) * spacing
    half = np.deg2rad(THETA_HOH) / 2
    body = np.array([[0.0, 0.0, 0.0],
                     [ROH * np.sin(half), 0.0, ROH * np.cos(half)],
                     [-ROH * np.sin(half), 0.0, ROH * np.cos(half)]])
    com = (body * np.array([MASS_O, MASS_H, MASS_H])[:, None]).sum(0) / (MASS_O + 2 * MASS_H)
    body = body - com
    rot = _random_rotations(rng, n_waters)
    pos = (centres[:, None, :] + np.einsum("nij,aj->nai", rot, body)).reshape(-1, 3)
    n = 3 * n_waters
    mass = np.tile([MASS_O, MASS_H, MASS_H], n_waters)
    # Maxwell-Boltzmann in internal units: sigma_v = sqrt(kT/m) (kcal/mol/amu)^(1/2) = A/tu
    vel = rng.standard_normal((n, 3)) * np.sqrt(BOLTZMANN * temperature / mass)[:, None]
    vel -= (vel * mass[:, None]).sum(0) / mass.sum()
    w = np.arange(n_waters, dtype=np.int32)
    o, h1, h2 = 3 * w, 3 * w + 1, 3 * w + 2
    excl = np.stack([np.stack([o, h1], 1), np.stack([o, h2], 1), np.stack([h1, h2], 1)],
                    1).reshape(-1, 2)
    return dict(
        n=n, box=np.array([L, L, L]), origin=np.zeros(3), pos=pos, vel=vel, mass=mass,
        charge=np.tile([Q_O, Q_H, Q_H], n_waters) * SQRTCOULOMBCONSTANT,
        type=np.tile(np.array([0, 1, 1], np.int32), n_waters),
        molecule=np.repeat(w, 3).astype(np.int32), lj=lj_table(),
        excl_pairs=excl.astype(np.int32), excl_kind=np.full(len(excl), 2, np.int32),
        bonds=np.stack([np.stack([o, h1], 1), np.stack([o, h2], 1)], 1).reshape(-1, 2).astype(np.int32),
        bond_k=np.full(2 * n_waters, 450.0), bond_r0=np.full(2 * n_waters, ROH),
        angles=np.stack([h1, o, h2], 1).astype(np.int32),
        angle_k=np.full(n_waters, 55.0), angle_theta0=np.full(n_waters, np.deg2rad(THETA_HOH)),
        ub_k=np.zeros(n_waters), ub_r0=np.zeros(n_waters), coulomb_scaling=1.0,
        elem="OHH" * n_waters, seed=seed)


def fft_friendly(n):
    """Smallest integer >= n whose prime factors are all 2, 3 or 5."""
    n = max(int(np.ceil(n)), 1)
    while True:
        m = n
        for p in (2, 3, 5):
            while m % p == 0:
                m //= p
        if m == 1:
            return n
        n += 1


def pme_grid_for(edge, spacing=1.0, minimum=8):
    """PME grid edge at about ``spacing`` A rounded up to a 2/3/5-smooth size."""
    return fft_friendly(max(minimum, edge / spacing))


def ensemble(n_boxes=256, lo=100, hi=2000, seed=4321, temperature=300.0):
    """Independent water boxes of uneven size: water counts uniform on [lo, hi], each box at
    1.0 g/cm^3 with its own seed.  Returns (boxes, PME grid edge per box at ~1 A spacing)."""
    rng = np.random.default_rng(seed)
    counts = rng.integers(lo, hi + 1, size=n_boxes)
    boxes = [water_box(int(n), seed=seed + 1 + k, temperature=temperature)
             for k, n in enumerate(counts)]
    grids = [pme_grid_for(b["box"][0]) for b in boxes]
    return boxes, grids
