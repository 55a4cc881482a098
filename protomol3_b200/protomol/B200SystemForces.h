/* -*- c++ -*- */
// ProtoMol 3 plugin classes for libpmb200: SystemForce subclasses that a ProtoMol build registers
// in its ForceFactory beside the CPU forces (force/system/SystemForce.h:32-52;
// factory/ForceFactory.h; module registration as in module/Module.h:28), so that a .conf selects
// them by name:
//
//   force Coulomb -algorithm PMEwaldB200 -real -reciprocal -correction -interpolation BSpline
//         -gridsize 96 96 96 -cutoff 10 -order 4 -accuracy 1e-6 -alpha -1 -precision mixed
//   force LennardJones -switchingFunction C2 -algorithm NonbondedCutoffB200 -switchon 8
//         -cutoff 10 -precision fp64
//
// Each force owns a device system built from the topology at its first evaluate; evaluate() is
// SystemForce::evaluate: forces and the ScalarStructure energies are accumulated into (+=), as
// ForceGroup requires (force/ForceGroup.cpp:65-69).  Errors of the C ABI become THROW.
//
// Header only, C++98 like the rest of ProtoMol.  Include it where the ProtoMol headers and
// include/pmb200.h are on the include path, and link libpmb200.so.
#ifndef PMB200_PROTOMOL_B200SYSTEMFORCES_H
#define PMB200_PROTOMOL_B200SYSTEMFORCES_H

#include <protomol/base/Exception.h>
#include <protomol/base/Report.h>
#include <protomol/config/Parameter.h>
#include <protomol/config/Value.h>
#include <protomol/factory/ForceFactory.h>
#include <protomol/force/system/SystemForce.h>
#include <protomol/topology/CubicCellManager.h>
#include <protomol/topology/ExclusionTable.h>
#include <protomol/topology/PeriodicBoundaryConditions.h>
#include <protomol/topology/Topology.h>
#include <protomol/type/ScalarStructure.h>
#include <protomol/type/Vector3DBlock.h>

#include <cstring>
#include <string>
#include <vector>

#include "pmb200.h"

namespace ProtoMol {
namespace B200 {

typedef Topology<PeriodicBoundaryConditions, CubicCellManager> PeriodicTopology;

inline std::string switchName(int kind) {
  return kind == PMB_SWITCH_C1 ? "C1" : (kind == PMB_SWITCH_C2 ? "C2" : "Cutoff");
}

inline int precisionFromName(const std::string &p) {
  if (p == "mixed") return PMB_MIXED;
  if (p == "fp64") return PMB_FP64;
  return -1;
}

inline std::string precisionName(int p) { return p == PMB_MIXED ? "mixed" : "fp64"; }

inline void check(int status) {
  if (status != PMB_OK) THROW(std::string("libpmb200: ") + pmb_last_error());
}

// The parts of the topology the force path reads (GenericTopology.h:142-164), as one box.
inline pmb_system *buildSystem(const GenericTopology *g, int precision) {
  const PeriodicTopology *t = dynamic_cast<const PeriodicTopology *>(g);
  if (t == NULL)
    THROW("B200 forces need Topology<PeriodicBoundaryConditions, CubicCellManager>");
  const unsigned int n = g->atoms.size();
  std::vector<double> charge(n), mass(n);
  std::vector<int> type(n), molecule(n);
  for (unsigned int i = 0; i < n; i++) {
    charge[i] = g->atoms[i].scaledCharge;
    mass[i] = g->atoms[i].scaledMass;
    type[i] = g->atoms[i].type;
    molecule[i] = g->atoms[i].molecule;
  }
  const int nt = g->lennardJonesParameters.size();
  std::vector<double> lj(4 * nt * nt);
  for (int a = 0; a < nt; a++)
    for (int b = 0; b < nt; b++) {
      const LennardJonesParameters &p = g->lennardJonesParameters(a, b);
      double *o = &lj[4 * (a * nt + b)];
      o[0] = p.A; o[1] = p.B; o[2] = p.A14; o[3] = p.B14;
    }
  const std::vector<ExclusionPair> &table = g->exclusions.getTable();
  std::vector<int> pairs, kind;
  for (unsigned int k = 0; k < table.size(); k++) {
    if (table[k].excl == EXCLUSION_NONE) continue;
    pairs.push_back(table[k].a1);
    pairs.push_back(table[k].a2);
    kind.push_back(table[k].excl == EXCLUSION_MODIFIED ? 1 : 2);
  }
  const PeriodicBoundaryConditions &bc = t->boundaryConditions;
  const Vector3D e1 = bc.e1(), e2 = bc.e2(), e3 = bc.e3();
  if (e1.c[1] != 0.0 || e1.c[2] != 0.0 || e2.c[0] != 0.0 || e2.c[2] != 0.0 || e3.c[0] != 0.0 ||
      e3.c[1] != 0.0)
    THROW("B200 forces need an orthogonal periodic box");
  pmb_box_desc d;
  std::memset(&d, 0, sizeof(d));
  d.n_atoms = (int)n;
  d.n_types = nt;
  d.charge = n ? &charge[0] : NULL;
  d.mass = n ? &mass[0] : NULL;
  d.type = n ? &type[0] : NULL;
  d.molecule = n ? &molecule[0] : NULL;
  d.lj = nt ? &lj[0] : NULL;
  d.n_excl = (int)kind.size();
  d.excl_pairs = kind.empty() ? NULL : &pairs[0];
  d.excl_kind = kind.empty() ? NULL : &kind[0];
  d.box[0] = e1.c[0];
  d.box[1] = e2.c[1];
  d.box[2] = e3.c[2];
  d.coulomb_scaling = g->coulombScalingFactor;
  pmb_system *s = pmb_system_create(&d, 1, precision);
  if (s == NULL) THROW(std::string("libpmb200: ") + pmb_last_error());
  return s;
}

// Adds the device energies of one box to the ScalarStructure slots (ScalarStructure.h:26-54).
inline void addEnergies(const double *e, ScalarStructure *energies, bool lj, bool coulomb) {
  if (lj) (*energies)[ScalarStructure::LENNARDJONES] += e[PMB_E_LJ];
  if (coulomb) (*energies)[ScalarStructure::COULOMB] += e[PMB_E_COULOMB];
  if (energies->virial())
    for (int k = 0; k < 9; k++)
      (*energies)[(ScalarStructure::Index)(ScalarStructure::VIRIALXX + k)] += e[PMB_E_VIRIAL + k];
}

// A force's device state: the system (built at the first evaluate) and the force handle.
class DeviceForce {
 public:
  DeviceForce() : sys(NULL), force(NULL), natoms(0) {}
  ~DeviceForce() { release(); }
  void release() {
    if (force) pmb_force_destroy(force);
    if (sys) pmb_system_destroy(sys);
    force = NULL;
    sys = NULL;
  }
  // Evaluates desc on the topology's atoms; builds the device system on first use (and again
  // if the number of atoms changed).
  void evaluate(const GenericTopology *topo, const pmb_force_desc &desc, int precision,
                const Vector3DBlock *positions, Vector3DBlock *forces, double *e, bool virial) {
    if (sys == NULL || natoms != positions->size()) {
      release();
      sys = buildSystem(topo, precision);
      force = pmb_force_create(sys, &desc);
      if (force == NULL) THROW(std::string("libpmb200: ") + pmb_last_error());
      natoms = positions->size();
    }
    check(pmb_force_evaluate(force, positions->c, forces->c, e, virial ? 1 : 0));
  }

 private:
  DeviceForce(const DeviceForce &);
  DeviceForce &operator=(const DeviceForce &);
  pmb_system *sys;
  pmb_force *force;
  unsigned int natoms;
};

// Coulomb -algorithm PMEwaldB200 -real -reciprocal -correction -interpolation BSpline
// [-switchingFunction C1]: the replacement of NonbondedPMEwaldSystemForce<PBC, CubicCellManager,
// true, true, true, BSpline, Cutoff|C1> with the same parameters (NonbondedPMEwaldSystemForce.h:
// 1003-1014, checks of doMake :1026-1058) plus -precision.  RSW: real-space switch.
template <int RSW>
class NonbondedPMEwaldB200SystemForce : public SystemForce {
 public:
  NonbondedPMEwaldB200SystemForce()
      : nx(0), ny(0), nz(0), order(4), cutoff(0.0), accuracy(1e-6), alpha(-1.0), precision(PMB_FP64) {}
  NonbondedPMEwaldB200SystemForce(int nx_, int ny_, int nz_, Real rc, int order_, Real acc,
                                  Real alpha_, int precision_)
      : nx(nx_), ny(ny_), nz(nz_), order(order_), cutoff(rc), accuracy(acc), alpha(alpha_),
        precision(precision_) {}

  using SystemForce::evaluate;
  virtual void evaluate(const GenericTopology *topo, const Vector3DBlock *positions,
                        Vector3DBlock *forces, ScalarStructure *energies) {
    pmb_force_desc d;
    std::memset(&d, 0, sizeof(d));
    d.kind = PMB_FORCE_PME;
    d.grid[0] = nx; d.grid[1] = ny; d.grid[2] = nz;
    d.order = order;
    d.cutoff = cutoff;
    d.accuracy = accuracy;
    d.alpha = alpha;
    d.real_switch = RSW;
    d.real = d.reciprocal = d.correction = 1;
    double e[PMB_E_STRIDE] = {0};
    dev.evaluate(topo, d, precision, positions, forces, e, energies->virial());
    addEnergies(e, energies, false, true);
  }

  virtual std::string getKeyword() const { return "PMEwaldB200"; }
  virtual std::string getIdNoAlias() const {
    return std::string("Coulomb -algorithm ") + getKeyword() +
           " -real -reciprocal -correction -interpolation BSpline" +
           (RSW == PMB_SWITCH_C1 ? std::string(" -switchingFunction C1") : std::string(""));
  }
  virtual void getParameters(std::vector<Parameter> &p) const {
    p.push_back(Parameter("-gridsize", Value(nx, ConstraintValueType::Positive())));
    p.push_back(Parameter("", Value(ny, ConstraintValueType::Positive())));
    p.push_back(Parameter("", Value(nz, ConstraintValueType::Positive())));
    p.push_back(Parameter("-cutoff", Value(cutoff, ConstraintValueType::Positive()), Text("Rc cutoff")));
    p.push_back(Parameter("-order", Value(order, ConstraintValueType::Positive()), 4, Text("interpolation")));
    p.push_back(Parameter("-accuracy", Value(accuracy, ConstraintValueType::Positive()), (Real)(1.e-6)));
    p.push_back(Parameter("-alpha", Value(alpha), (Real)-1.0, Text("splitting")));
    p.push_back(Parameter("-precision", Value(precisionName(precision), ConstraintValueType::NotEmpty()),
                          std::string("fp64"), Text("fp64 (the drop-in path) or mixed")));
  }

 private:
  virtual Force *doMake(const std::vector<Value> &values) const {
    const int gx = values[0], gy = values[1], gz = values[2], ord = values[4];
    const Real rc = values[3], acc = values[5], a = values[6];
    const int prec = precisionFromName(values[7].getString());
    std::string err;
    if (ord < 2 || (ord % 2) != 0 || !values[4].valid())
      err += " order (=" + values[4].getString() + ") > 1 and even.";
    if (!values[0].valid() || !values[1].valid() || !values[2].valid() || gx < ord || gy < ord || gz < ord)
      err += " order <= nx, ny, nz.";
    if (rc <= 0.0 || !values[3].valid()) err += " cutoff (=" + values[3].getString() + ") > 0.";
    if (acc <= 0.0 || !values[5].valid()) err += " accuracy (=" + values[5].getString() + ") > 0.";
    if (!values[6].valid()) err += " alpha '" + values[6].getString() + "' not valid.";
    if (prec < 0) err += " precision '" + values[7].getString() + "' is fp64 or mixed.";
    if (!err.empty()) {
      Report::report << Report::error << "force " << getKeyword() << ":" << err << Report::endr;
      return NULL;
    }
    return new NonbondedPMEwaldB200SystemForce(gx, gy, gz, rc, ord, acc, a, prec);
  }

  int nx, ny, nz, order;
  Real cutoff, accuracy, alpha;
  int precision;
  DeviceForce dev;
};

// The parameters of one switching function (switch/C1SwitchingFunction.cpp:18-22,
// C2SwitchingFunction.cpp:20-28, CutoffSwitchingFunction.h:47-51).
inline void switchParameters(int kind, Real switchon, Real cutoff, std::vector<Parameter> &p) {
  if (kind == PMB_SWITCH_C2)
    p.push_back(Parameter("-switchon", Value(switchon, ConstraintValueType::NotNegative()), Text("switchon distance")));
  p.push_back(Parameter("-cutoff", Value(cutoff, ConstraintValueType::Positive()), Text("cutoff distance")));
}
inline int switchParameterCount(int kind) { return kind == PMB_SWITCH_C2 ? 2 : 1; }

// LennardJones [Coulomb] -switchingFunction A [-switchingFunction B]
// -algorithm NonbondedCutoffB200: the replacement of NonbondedCutoffSystemForce<CubicCellManager,
// OneAtomPair(Two)<PBC, A, LennardJonesForce [, B, CoulombForce]>> (NonbondedCutoffForce.h:
// 68-91, OneAtomPairTwo.h:130-160).  LSW / CSW: switch of each potential, -1 = potential absent.
template <int LSW, int CSW>
class NonbondedCutoffB200SystemForce : public SystemForce {
 public:
  NonbondedCutoffB200SystemForce()
      : ljOn(0.0), ljCut(0.0), cOn(0.0), cCut(0.0), cutoff(0.0), precision(PMB_FP64) {}
  NonbondedCutoffB200SystemForce(Real ljOn_, Real ljCut_, Real cOn_, Real cCut_, Real cutoff_, int precision_)
      : ljOn(ljOn_), ljCut(ljCut_), cOn(cOn_), cCut(cCut_), cutoff(cutoff_), precision(precision_) {}

  using SystemForce::evaluate;
  virtual void evaluate(const GenericTopology *topo, const Vector3DBlock *positions,
                        Vector3DBlock *forces, ScalarStructure *energies) {
    pmb_force_desc d;
    std::memset(&d, 0, sizeof(d));
    d.kind = PMB_FORCE_CUTOFF;
    if (LSW >= 0) {
      d.lj = 1;
      d.lj_switch = LSW;
      d.lj_switchon = ljOn;
      d.lj_cutoff = ljCut;
    }
    if (CSW >= 0) {
      d.coulomb = 1;
      d.coulomb_switch = CSW;
      d.coulomb_switchon = cOn;
      d.coulomb_cutoff = cCut;
    }
    double e[PMB_E_STRIDE] = {0};
    dev.evaluate(topo, d, precision, positions, forces, e, energies->virial());
    addEnergies(e, energies, LSW >= 0, CSW >= 0);
  }

  virtual std::string getKeyword() const { return "NonbondedCutoffB200"; }
  virtual std::string getIdNoAlias() const {
    std::string id;
    if (LSW >= 0) id += "LennardJones";
    if (CSW >= 0) id += std::string(id.empty() ? "" : " ") + "Coulomb";
    if (LSW >= 0) id += " -switchingFunction " + switchName(LSW);
    if (CSW >= 0) id += " -switchingFunction " + switchName(CSW);
    return id + " -algorithm " + getKeyword();
  }
  virtual void getParameters(std::vector<Parameter> &p) const {
    if (LSW >= 0) switchParameters(LSW, ljOn, ljCut, p);
    if (CSW >= 0) switchParameters(CSW, cOn, cCut, p);
    p.push_back(Parameter("-cutoff", Value(cutoff, ConstraintValueType::Positive()), Text("algorithm cutoff")));
    p.push_back(Parameter("-precision", Value(precisionName(precision), ConstraintValueType::NotEmpty()),
                          std::string("fp64"), Text("fp64 (the drop-in path) or mixed")));
  }

 private:
  virtual Force *doMake(const std::vector<Value> &v) const {
    unsigned int k = 0;
    Real lo = 0.0, lc = 0.0, co = 0.0, cc = 0.0;
    std::string err;
    if (LSW >= 0) {
      if (LSW == PMB_SWITCH_C2) lo = v[k++];
      lc = v[k++];
      if (LSW == PMB_SWITCH_C2 && !(lo >= 0.0 && lo < lc)) err += " LennardJones: 0 <= switchon < cutoff.";
    }
    if (CSW >= 0) {
      if (CSW == PMB_SWITCH_C2) co = v[k++];
      cc = v[k++];
      if (CSW == PMB_SWITCH_C2 && !(co >= 0.0 && co < cc)) err += " Coulomb: 0 <= switchon < cutoff.";
    }
    const Real rc = v[k++];
    const int prec = precisionFromName(v[k].getString());
    if (!(rc > 0.0)) err += " cutoff > 0.";
    if (prec < 0) err += " precision '" + v[k].getString() + "' is fp64 or mixed.";
    if (!err.empty()) {
      Report::report << Report::error << "force " << getIdNoAlias() << ":" << err << Report::endr;
      return NULL;
    }
    return new NonbondedCutoffB200SystemForce(lo, lc, co, cc, rc, prec);
  }

  Real ljOn, ljCut, cOn, cCut, cutoff;
  int precision;
  DeviceForce dev;
};

// Registers the B200 forces in a force factory: PME with a cutoff or C1 real-space switch, one
// potential with each switching function, and the two-potential sets the reference registers
// (LennardJones C2 with Coulomb C1 or C2, module/NonbondedCutoffForceModule.cpp:74-80; other
// orders of the same switches are not distinguishable by the factory's id matching).
inline void registerForces(ForceFactory &f) {
  f.reg(new NonbondedPMEwaldB200SystemForce<PMB_SWITCH_CUTOFF>());
  f.reg(new NonbondedPMEwaldB200SystemForce<PMB_SWITCH_C1>());
  f.reg(new NonbondedCutoffB200SystemForce<PMB_SWITCH_CUTOFF, -1>());
  f.reg(new NonbondedCutoffB200SystemForce<PMB_SWITCH_C1, -1>());
  f.reg(new NonbondedCutoffB200SystemForce<PMB_SWITCH_C2, -1>());
  f.reg(new NonbondedCutoffB200SystemForce<-1, PMB_SWITCH_CUTOFF>());
  f.reg(new NonbondedCutoffB200SystemForce<-1, PMB_SWITCH_C1>());
  f.reg(new NonbondedCutoffB200SystemForce<-1, PMB_SWITCH_C2>());
  f.reg(new NonbondedCutoffB200SystemForce<PMB_SWITCH_C2, PMB_SWITCH_C1>());
  f.reg(new NonbondedCutoffB200SystemForce<PMB_SWITCH_C2, PMB_SWITCH_C2>());
}

}  // namespace B200
}  // namespace ProtoMol
#endif  // PMB200_PROTOMOL_B200SYSTEMFORCES_H
