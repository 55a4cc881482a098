"""Build the golden fixtures that pin the CPU oracle to ProtoMol's own regression data.

Run once in a container that holds the ProtoMol 3 source tree (read as text only; nothing of
the reference is executed):

    python tests/golden/make_golden.py [--ref <ProtoMol 3 tree>]

It writes two small ``.npz`` fixtures next to this script:

``water423_periodic.npz``
    ``test/tests/water_CHARMM_PERIODIC_L.conf``: 141 flexible TIP3 waters in a 28 A periodic box,
    Bond + Angle, Coulomb cutoff 6.5 A with C1 switching, Lennard-Jones cutoff 6.5 A with C2
    switching (switchon 0.1), leapfrog 0.5 fs for 200 steps.  Inputs come from
    ``test/tests/data/water_423.{psf,pos.pdb,vel.pdb}`` and ``par_all27_prot_lipid.inp``; the
    expected outputs are ``test/tests/expected/water_CHARMM_PERIODIC_L.{forces,pos,vel,energy}``
    (forces at step 0 and step 200, final positions and velocities, all-energies rows at
    t = 0 fs and t = 100 fs).  ProtoMol compares these at an absolute tolerance of 1e-5
    (test/test.py:14).

``pentane320_periodic.npz``
    ``protomol-test/ConfigTests/data/EnergiesTest.conf``: 64 united-atom n-pentanes in a 23 A
    periodic box, exclusion scheme 1-4, Lennard-Jones cutoff 9 A with C2 switching from 8 A.
    Only the step-0 row of ``EnergiesTest.energies.orig`` depends on the initial coordinates
    alone, so the fixture keeps its Lennard-Jones energy (-340.57666) as the pin.

Conventions follow the reference's topology builder:
  * scaled charge = charge * 18.2226123264 (BuildTopology.cpp:92, PMConstants.cpp:67);
  * CHARMM mixing A = (Ri+Rj)^12 sqrt(ei ej), B = 2 (Ri+Rj)^6 sqrt(ei ej) with R = Rmin/2
    (BuildTopology.cpp:663-673);
  * exclusions: bonds and angle ends FULL, dihedral ends FULL for "1-4" or MODIFIED for
    "scaled1-4" (BuildTopology.cpp:1103-1158);
  * PDB velocities are divided by 20.45482706 (IOModule.cpp:126, PMConstants.cpp:71);
  * angles are converted with degree * pi / 180 (MathUtilities.h:126-128).
"""
import argparse
import os
import struct

import numpy as np

SQRTCOULOMBCONSTANT = 18.2226123264
PDBVELSCALINGFACTOR = 20.45482706
HERE = os.path.dirname(os.path.abspath(__file__))


def parse_psf(path):
    lines = open(path).read().splitlines()
    out = {"atoms": [], "bonds": [], "angles": [], "dihedrals": []}
    i = 0
    while i < len(lines):
        ln = lines[i]
        if "!NATOM" in ln:
            n = int(ln.split()[0])
            for k in range(n):
                t = lines[i + 1 + k].split()
                # index seg resid resname name type charge mass
                out["atoms"].append((t[4], t[5], float(t[6]), float(t[7]), int(t[2])))
            i += n
        for key, tag, width in (("bonds", "!NBOND", 2), ("angles", "!NTHETA", 3),
                                ("dihedrals", "!NPHI", 4)):
            if tag in ln:
                n = int(ln.split()[0])
                vals = []
                j = i + 1
                while len(vals) < n * width:
                    vals.extend(int(v) - 1 for v in lines[j].split())
                    j += 1
                out[key] = [tuple(vals[k * width:(k + 1) * width]) for k in range(n)]
                i = j - 1
        i += 1
    return out


def parse_par(path):
    """Minimal CHARMM28 parameter reader: BONDS, ANGLES (with Urey-Bradley), NONBONDED."""
    sec = None
    bonds, angles, nonb = {}, {}, {}
    for raw in open(path):
        ln = raw.split("!")[0].strip()
        if not ln or ln.startswith("*"):
            continue
        head = ln.split()[0].upper()
        if head in ("BONDS", "ANGLES", "DIHEDRALS", "IMPROPER", "NONBONDED", "NBFIX",
                    "HBOND", "END", "CMAP"):
            sec = head
            continue
        if head.startswith("CUTNB") or head.startswith("NBXMOD"):
            continue
        t = ln.split()
        try:
            if sec == "BONDS":
                bonds[(t[0], t[1])] = (float(t[2]), float(t[3]))
            elif sec == "ANGLES":
                ub = (float(t[5]), float(t[6])) if len(t) >= 7 else (0.0, 0.0)
                angles[(t[0], t[1], t[2])] = (float(t[3]), float(t[4])) + ub
            elif sec == "NONBONDED":
                eps, rmin = float(t[2]), float(t[3])
                eps14, rmin14 = (float(t[5]), float(t[6])) if len(t) >= 7 else (eps, rmin)
                nonb[t[0]] = (eps, rmin, eps14, rmin14)
        except (ValueError, IndexError):
            continue
    return bonds, angles, nonb


def lookup(table, key):
    if key in table:
        return table[key]
    rev = tuple(reversed(key))
    if rev in table:
        return table[rev]
    raise KeyError(key)


def build_topology(psf, par, exclude):
    bonds_p, angles_p, nonb = par
    names = [a[1] for a in psf["atoms"]]
    type_names = []
    for t in names:
        if t not in type_names:
            type_names.append(t)
    types = np.array([type_names.index(t) for t in names], np.int32)
    charge = np.array([a[2] for a in psf["atoms"]]) * SQRTCOULOMBCONSTANT
    mass = np.array([a[3] for a in psf["atoms"]])
    nt = len(type_names)
    lj = np.zeros((nt, nt, 4))
    for i, ti in enumerate(type_names):
        ei, ri, e14i, r14i = nonb[ti]
        for j, tj in enumerate(type_names):
            ej, rj, e14j, r14j = nonb[tj]
            r, e = ri + rj, np.sqrt(ei * ej)
            r14, e14 = r14i + r14j, np.sqrt(e14i * e14j)
            lj[i, j] = (r ** 12 * e, 2 * r ** 6 * e, r14 ** 12 * e14, 2 * r14 ** 6 * e14)
    bonds = np.array(psf["bonds"], np.int32).reshape(-1, 2)
    bond_par = np.array([lookup(bonds_p, (names[a], names[b])) for a, b in bonds]).reshape(-1, 2)
    angles = np.array(psf["angles"], np.int32).reshape(-1, 3)
    ang_par = np.array([lookup(angles_p, (names[a], names[b], names[c]))
                        for a, b, c in angles]).reshape(-1, 4)
    ang_par[:, 1] = ang_par[:, 1] * np.pi / 180.0
    excl = {}
    for a, b in bonds:
        excl[(min(a, b), max(a, b))] = 2
    for a, _, c in angles:
        excl[(min(a, c), max(a, c))] = 2
    if exclude in ("1-4", "scaled1-4"):
        for a, _, _, d in psf["dihedrals"]:
            key = (min(a, d), max(a, d))
            excl.setdefault(key, 2 if exclude == "1-4" else 1)
    keys = sorted(excl)
    excl_pairs = np.array(keys, np.int32).reshape(-1, 2)
    excl_kind = np.array([excl[k] for k in keys], np.int32)
    # molecules = connected components of the bond graph (BuildTopology.cpp:1032-1064)
    parent = list(range(len(names)))

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x
    for a, b in bonds:
        parent[find(a)] = find(b)
    roots, mol = {}, []
    for i in range(len(names)):
        mol.append(roots.setdefault(find(i), len(roots)))
    return dict(type=types, charge=charge, mass=mass, lj=lj, bonds=bonds,
                bond_k=bond_par[:, 0], bond_r0=bond_par[:, 1], angles=angles,
                angle_k=ang_par[:, 0], angle_theta0=ang_par[:, 1], ub_k=ang_par[:, 2],
                ub_r0=ang_par[:, 3], excl_pairs=excl_pairs, excl_kind=excl_kind,
                molecule=np.array(mol, np.int32))


def parse_pdb_xyz(path):
    xyz = []
    for ln in open(path):
        if ln.startswith("ATOM") or ln.startswith("HETATM"):
            xyz.append((float(ln[30:38]), float(ln[38:46]), float(ln[46:54])))
    return np.array(xyz)


def parse_xyz_frames(path):
    lines = open(path).read().splitlines()
    pos = 0
    nframes = 1
    first = lines[0].split()
    if len(lines) > 1 and len(lines[1].split()) == 1:
        nframes = int(first[0])
        pos = 1
    frames = []
    for _ in range(nframes):
        n = int(lines[pos].split()[0])
        frames.append(np.array([[float(v) for v in lines[pos + 1 + k].split()[1:4]]
                                for k in range(n)]))
        pos += 1 + n
    return frames


def parse_energies(path):
    return np.array([[float(v) for v in ln.split()] for ln in open(path) if ln.strip()])


def read_xyzbin(path):
    raw = open(path, "rb").read()
    n = struct.unpack("<i", raw[:4])[0]
    return np.frombuffer(raw[4:4 + 24 * n], "<f8").reshape(n, 3).copy()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("PROTOMOL3_REF"),
                    help="ProtoMol 3 source tree (default: $PROTOMOL3_REF)")
    ref = ap.parse_args().ref
    if not ref:
        raise SystemExit("pass --ref <ProtoMol 3 tree> or set PROTOMOL3_REF")

    d = os.path.join(ref, "test/tests/data")
    e = os.path.join(ref, "test/tests/expected")
    psf = parse_psf(os.path.join(d, "water_423.psf"))
    par = parse_par(os.path.join(d, "par_all27_prot_lipid.inp"))
    topo = build_topology(psf, par, "scaled1-4")
    pos = parse_pdb_xyz(os.path.join(d, "water_423.pos.pdb"))
    vel = parse_pdb_xyz(os.path.join(d, "water_423.vel.pdb")) / PDBVELSCALINGFACTOR
    forces = parse_xyz_frames(os.path.join(e, "water_CHARMM_PERIODIC_L.forces"))
    np.savez_compressed(
        os.path.join(HERE, "water423_periodic.npz"), **topo,
        pos=pos, vel=vel, box=np.array([28.0, 28.0, 28.0]), origin=np.zeros(3),
        dt=0.5, nsteps=200, coul_cutoff=6.5, lj_cutoff=6.5, lj_switchon=0.1,
        exp_forces0=forces[0], exp_forces_end=forces[-1],
        exp_pos=parse_xyz_frames(os.path.join(e, "water_CHARMM_PERIODIC_L.pos"))[0],
        exp_vel=parse_xyz_frames(os.path.join(e, "water_CHARMM_PERIODIC_L.vel"))[0],
        exp_energy=parse_energies(os.path.join(e, "water_CHARMM_PERIODIC_L.energy")))

    d2 = os.path.join(ref, "protomol-test/ConfigTests/data")
    psf2 = parse_psf(os.path.join(d2, "VelacTest.psf"))
    par2 = parse_par(os.path.join(d2, "VelacTest.par"))
    topo2 = build_topology(psf2, par2, "1-4")
    en2 = parse_energies(os.path.join(d2, "EnergiesTest.energies.orig"))
    np.savez_compressed(
        os.path.join(HERE, "pentane320_periodic.npz"), **topo2,
        pos=read_xyzbin(os.path.join(d2, "VelacTest.coor")),
        box=np.array([23.0, 23.0, 23.0]), origin=np.array([6.8, 7.3, 8.2]),
        lj_cutoff=9.0, lj_switchon=8.0, exp_lj_energy0=en2[0, 9])
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    main()
