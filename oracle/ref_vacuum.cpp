// Test-infrastructure harness: ProtoMol 3's cutoff forces with VacuumBoundaryConditions (no
// periodic images; cell pairs from CellListEnumerator_standard), compiled from the reference
// sources by oracle/Makefile, for the vacuum force sets of its ConfigTests
// (protomol-test/ConfigTests/data/{C1Test,C2Test,CoulombForceCutoffTest}.conf: boundaryConditions
// vacuum, cellManager Cubic).
//   NonbondedCutoffSystemForce<CubicCellManager, OneAtomPairTwo<VacuumBoundaryConditions, Switch,
//       LennardJonesForce, Switch, CoulombForce>>  and the OneAtomPair forms with one potential
//   (module/NonbondedCutoffForceModule.cpp registers them for vacuum as for periodic boxes)
#include <protomol/base/Report.h>
using namespace ProtoMol::Report;

#include <protomol/force/CoulombForce.h>
#include <protomol/force/LennardJonesForce.h>
#include <protomol/force/OneAtomPair.h>
#include <protomol/force/OneAtomPairTwo.h>
#include <protomol/force/nonbonded/NonbondedCutoffSystemForce.h>
#include <protomol/switch/C1SwitchingFunction.h>
#include <protomol/switch/C2SwitchingFunction.h>
#include <protomol/switch/CutoffSwitchingFunction.h>
#include <protomol/topology/CellListEnumeratorStandard.h>
#include <protomol/topology/CubicCellManager.h>
#include <protomol/topology/Topology.h>
#include <protomol/topology/VacuumBoundaryConditions.h>
#include <protomol/type/ScalarStructure.h>
#include <protomol/type/Vector3DBlock.h>

using namespace ProtoMol;

typedef VacuumBoundaryConditions VBC;
typedef Topology<VBC, CubicCellManager> Topo;
#define PMB_REF_VACUUM
#include "ref_topology.h"

namespace {

template <class SA, class SB>
SystemForce *vac_two(const ref_cutoff *c, SA sa, SB sb) {
  typedef OneAtomPairTwo<VBC, SA, LennardJonesForce, SB, CoulombForce> OAP;
  double rc = c->lj_cutoff > c->coul_cutoff ? c->lj_cutoff : c->coul_cutoff;
  return new NonbondedCutoffSystemForce<CubicCellManager, OAP>(rc, OAP(LennardJonesForce(), sa, CoulombForce(), sb));
}

template <class S, class F>
SystemForce *vac_one(double rc, S s) {
  typedef OneAtomPair<VBC, S, F> OAP;
  return new NonbondedCutoffSystemForce<CubicCellManager, OAP>(rc, OAP(F(), s));
}

template <class S>
SystemForce *vac_with_coul(const ref_cutoff *c, S sa) {
  switch (c->coul_switch) {
    case 1: return vac_two(c, sa, C1SwitchingFunction(c->coul_cutoff));
    case 2: return vac_two(c, sa, C2SwitchingFunction(c->coul_switchon, c->coul_cutoff));
    default: return vac_two(c, sa, CutoffSwitchingFunction(c->coul_cutoff));
  }
}

template <class F>
SystemForce *vac_single(int sw, double on, double rc) {
  if (sw == 2) return vac_one<C2SwitchingFunction, F>(rc, C2SwitchingFunction(on, rc));
  if (sw == 1) return vac_one<C1SwitchingFunction, F>(rc, C1SwitchingFunction(rc));
  return vac_one<CutoffSwitchingFunction, F>(rc, CutoffSwitchingFunction(rc));
}

}  // namespace

extern "C" int ref_cutoff_eval_vacuum(const ref_input *in, const ref_cutoff *c, double *forces,
                                      double *energies, double *virial) {
  Topo *t = new Topo(in->coulomb_scaling, ExclusionType(ExclusionType::ONE4), VBC(),
                     CubicCellManager(in->cellsize), 16.0f);
  fill_topo(t, in);
  SystemForce *f = 0;
  if (c->do_lj && c->do_coul) {
    switch (c->lj_switch) {
      case 1: f = vac_with_coul(c, C1SwitchingFunction(c->lj_cutoff)); break;
      case 2: f = vac_with_coul(c, C2SwitchingFunction(c->lj_switchon, c->lj_cutoff)); break;
      default: f = vac_with_coul(c, CutoffSwitchingFunction(c->lj_cutoff)); break;
    }
  } else if (c->do_lj) {
    f = vac_single<LennardJonesForce>(c->lj_switch, c->lj_switchon, c->lj_cutoff);
  } else if (c->do_coul) {
    f = vac_single<CoulombForce>(c->coul_switch, c->coul_switchon, c->coul_cutoff);
  }
  if (f) {
    Vector3DBlock pos(in->n), frc(in->n);
    for (int i = 0; i < in->n; i++) {
      pos[i] = Vector3D(in->pos[3 * i], in->pos[3 * i + 1], in->pos[3 * i + 2]);
      frc[i] = Vector3D(0, 0, 0);
    }
    ScalarStructure e;
    e.clear();
    e.molecularVirial(false);
    e.virial(virial != 0);
    t->uncacheCellList();
    f->evaluate(t, &pos, &frc, &e);
    for (int i = 0; i < in->n; i++)
      for (int k = 0; k < 3; k++) forces[3 * i + k] += frc[i].c[k];
    energies[0] += e[ScalarStructure::COULOMB];
    energies[1] += e[ScalarStructure::LENNARDJONES];
    if (virial)
      for (int k = 0; k < 9; k++) virial[k] += e[(ScalarStructure::Index)(ScalarStructure::VIRIALXX + k)];
  }
  delete f;
  delete t;
  return 0;
}
