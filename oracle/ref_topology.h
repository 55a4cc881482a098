// Test infrastructure (oracle): the input structs of the reference harnesses and an in-memory
// Topology<PeriodicBoundaryConditions, CubicCellManager> built from them, shared by
// ref_harness.cpp (the reference's own forces) and the drop-in harness of the ProtoMol plugin.
// Include after the ProtoMol topology headers, inside no namespace.
#ifndef PMB_ORACLE_REF_TOPOLOGY_H
#define PMB_ORACLE_REF_TOPOLOGY_H

extern "C" {

struct ref_input {
  int n, ntypes;
  const double *pos, *charge, *mass;
  const int *type, *molecule;
  const double *lj;  // [nt*nt*4]
  int nexcl;
  const int *excl_pairs, *excl_kind;
  int nbonds;
  const int *bonds;
  const double *bond_k, *bond_r0;
  int nangles;
  const int *angles;
  const double *angle_k, *angle_theta0, *ub_k, *ub_r0;
  double box[3], origin[3];
  double cellsize, coulomb_scaling;
};

struct ref_cutoff {
  int do_lj, lj_switch;  // 0 cutoff, 1 C1, 2 C2
  double lj_switchon, lj_cutoff;
  int do_coul, coul_switch;
  double coul_switchon, coul_cutoff;
};

struct ref_pme {
  int nx, ny, nz, order;
  double cutoff, accuracy, alpha;
  int real_switch;  // 0 cutoff, 1 C1
};

}  // extern "C"

// The atoms, parameters, exclusions, bonds and angles of any Topology<BC, CubicCellManager>.
template <class T>
static inline void fill_topo(T *t, const ref_input *in);

#ifndef PMB_REF_VACUUM
static inline Topo *make_topo(const ref_input *in) {
  Topo *t = new Topo(in->coulomb_scaling, ExclusionType(ExclusionType::ONE4),
                     PBC(Vector3D(in->box[0], 0, 0), Vector3D(0, in->box[1], 0),
                         Vector3D(0, 0, in->box[2]),
                         Vector3D(in->origin[0], in->origin[1], in->origin[2])),
                     CubicCellManager(in->cellsize), 16.0f);
  fill_topo(t, in);
  return t;
}
#endif

template <class T>
static inline void fill_topo(T *t, const ref_input *in) {
  t->atoms.resize(in->n);
  int nmol = 0;
  for (int i = 0; i < in->n; i++) {
    t->atoms[i].type = in->type[i];
    t->atoms[i].scaledCharge = in->charge[i];
    t->atoms[i].scaledMass = in->mass ? in->mass[i] : 1.0;
    t->atoms[i].molecule = in->molecule[i];
    if (in->molecule[i] + 1 > nmol) nmol = in->molecule[i] + 1;
  }
  t->molecules.resize(nmol);
  t->atomTypes.resize(in->ntypes);
  t->lennardJonesParameters.resize(in->ntypes);
  for (int a = 0; a < in->ntypes; a++)
    for (int b = a; b < in->ntypes; b++) {
      const double *p = in->lj + 4 * (a * in->ntypes + b);
      t->lennardJonesParameters.set(a, b, LennardJonesParameters(p[0], p[1], p[2], p[3]));
    }
  t->exclusions.resize(in->n);
  for (int k = 0; k < in->nexcl; k++)
    t->exclusions.add(in->excl_pairs[2 * k], in->excl_pairs[2 * k + 1],
                      in->excl_kind[k] == 1 ? EXCLUSION_MODIFIED : EXCLUSION_FULL);
  t->exclusions.optimize();
  for (int k = 0; k < in->nbonds; k++) {
    Bond b;
    b.atom1 = in->bonds[2 * k];
    b.atom2 = in->bonds[2 * k + 1];
    b.springConstant = in->bond_k[k];
    b.restLength = in->bond_r0[k];
    t->bonds.push_back(b);
  }
  for (int k = 0; k < in->nangles; k++) {
    Angle a;
    a.atom1 = in->angles[3 * k];
    a.atom2 = in->angles[3 * k + 1];
    a.atom3 = in->angles[3 * k + 2];
    a.forceConstant = in->angle_k[k];
    a.restAngle = in->angle_theta0[k];
    a.ureyBradleyConstant = in->ub_k[k];
    a.ureyBradleyRestLength = in->ub_r0[k];
    t->angles.push_back(a);
  }
}

#endif
