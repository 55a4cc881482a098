"""SHAKE/RATTLE constraint lists on the host, in the reference's order.

``rattle_shake_constraints`` restates ``buildRattleShakeBondConstraintList``
(protomol/topology/TopologyUtilities.cpp:695-775): for every angle whose three atoms are two
hydrogens and one oxygen (by the first letter of the atom names), in angle order, the H-H distance
from the law of cosines over the two O-H rest lengths and the rest angle, then H1-O and H2-O; with
``all``, every other bond with a hydrogen, in bond order.  That makes each water rigid (3
constraints on 3 atoms) and leaves the other angles free.  The list feeds
``forces.Integrator.set_constraints``.
"""
import math

import numpy as np


def rattle_shake_constraints(topo, all_bonds=True):
    """(atom1, atom2, rest_length) arrays for a topology dict with ``elem`` (first letter of each
    atom's name), ``bonds``, ``bond_r0``, ``angles`` and ``angle_theta0``."""
    elem = topo["elem"]
    bonds = np.asarray(topo["bonds"], np.int64).reshape(-1, 2)
    r0 = np.asarray(topo["bond_r0"], np.float64)
    angles = np.asarray(topo["angles"], np.int64).reshape(-1, 3)
    theta0 = np.asarray(topo["angle_theta0"], np.float64)
    n = len(elem)
    mybonds = [[] for _ in range(n)]
    for k, (a, b) in enumerate(bonds):
        mybonds[a].append(k)
        mybonds[b].append(k)
    a1, a2, ln = [], [], []
    water_bonds = []
    for i, atoms in enumerate(angles):
        hyd, oxy, ato = [], 0, 0
        for a in atoms:
            if elem[a] == "H":
                hyd.append(int(a))
            if elem[a] == "O":
                ato = int(a)
                oxy += 1
        if len(hyd) == 2 and oxy == 1:
            b = float(r0[mybonds[hyd[0]][0]])  # a hydrogen has one bond
            c = float(r0[mybonds[hyd[1]][0]])
            alpha = float(theta0[i])
            a1 += [hyd[0], hyd[0], hyd[1]]
            a2 += [hyd[1], ato, ato]
            ln += [math.sqrt(b * b + c * c - 2 * b * c * math.cos(alpha)), b, c]
            water_bonds += [mybonds[hyd[0]][0], mybonds[hyd[1]][0]]
    water_bonds.sort()
    if all_bonds:
        # the bonds already constrained through a water are skipped by walking the sorted list of
        # their indices alongside the bond index, as the reference does
        used = 0
        for i in range(len(bonds)):
            if water_bonds and water_bonds[used] == i:
                if used < len(water_bonds) - 1:
                    used += 1
            elif elem[bonds[i][0]] == "H" or elem[bonds[i][1]] == "H":
                a1.append(int(bonds[i][0]))
                a2.append(int(bonds[i][1]))
                ln.append(float(r0[i]))
    return (np.array(a1, np.int32), np.array(a2, np.int32), np.array(ln, np.float64))
