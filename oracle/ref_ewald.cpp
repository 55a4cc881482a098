// Test-infrastructure harness: ProtoMol 3's exact Ewald sum with only the reciprocal term,
//   NonbondedFullEwaldSystemForce<PeriodicBoundaryConditions, CubicCellManager, false, true,
//       false, CutoffSwitchingFunction>(alpha, accuracy, expansion factor 0)
// (force/nonbonded/NonbondedFullEwaldSystemForce.h), compiled from the reference sources by
// oracle/Makefile, so tests can compare the library's Ewald check path with it.
#include <protomol/base/Report.h>
using namespace ProtoMol::Report;

#include <protomol/force/nonbonded/NonbondedFullEwaldSystemForce.h>
#include <protomol/switch/CutoffSwitchingFunction.h>
#include <protomol/topology/CellListEnumeratorPeriodicBoundaries.h>
#include <protomol/topology/CubicCellManager.h>
#include <protomol/topology/PeriodicBoundaryConditions.h>
#include <protomol/topology/Topology.h>
#include <protomol/type/ScalarStructure.h>
#include <protomol/type/Vector3DBlock.h>

using namespace ProtoMol;

typedef PeriodicBoundaryConditions PBC;
typedef Topology<PBC, CubicCellManager> Topo;
#include "ref_topology.h"

extern "C" int ref_ewald_reciprocal(const ref_input *in, double alpha, double accuracy, double *forces,
                                    double *energies, double *virial) {
  Topo *t = make_topo(in);
  NonbondedFullEwaldSystemForce<PBC, CubicCellManager, false, true, false, CutoffSwitchingFunction> f(alpha, accuracy,
                                                                                                     0.0);
  Vector3DBlock pos(in->n), frc(in->n);
  for (int i = 0; i < in->n; i++) {
    pos[i] = Vector3D(in->pos[3 * i], in->pos[3 * i + 1], in->pos[3 * i + 2]);
    frc[i] = Vector3D(0, 0, 0);
  }
  ScalarStructure e;
  e.clear();
  e.molecularVirial(false);
  e.virial(virial != 0);
  f.evaluate(t, &pos, &frc, &e);
  for (int i = 0; i < in->n; i++)
    for (int k = 0; k < 3; k++) forces[3 * i + k] += frc[i].c[k];
  energies[0] += e[ScalarStructure::COULOMB];
  if (virial)
    for (int k = 0; k < 9; k++) virial[k] += e[(ScalarStructure::Index)(ScalarStructure::VIRIALXX + k)];
  delete t;
  return 0;
}
