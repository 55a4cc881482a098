// Test infrastructure: the ProtoMol plugin classes of protomol3_b200/protomol/B200SystemForces.h
// made by the reference's own ForceFactory from a .conf force definition and evaluated through
// SystemForce::evaluate on the reference's own Topology<PeriodicBoundaryConditions,
// CubicCellManager> (built by oracle/ref_topology.h).  The parity test compares the result with
// the reference's CPU forces (oracle/ref_harness.cpp) on the same input.
#include <protomol/base/Report.h>
using namespace ProtoMol::Report;

#include <protomol/base/Exception.h>
#include <protomol/factory/ForceFactory.h>
#include <protomol/force/system/SystemForce.h>
#include <protomol/topology/CubicCellManager.h>
#include <protomol/topology/PeriodicBoundaryConditions.h>
#include <protomol/topology/Topology.h>
#include <protomol/type/ScalarStructure.h>
#include <protomol/type/Vector3DBlock.h>

#include <cstring>
#include <string>

#include "protomol3_b200/protomol/B200SystemForces.h"

using namespace ProtoMol;

typedef PeriodicBoundaryConditions PBC;
typedef Topology<PBC, CubicCellManager> Topo;

#include "ref_topology.h"

static void put(char *msg, int len, const std::string &s) {
  if (msg && len > 0) {
    std::strncpy(msg, s.c_str(), (size_t)len - 1);
    msg[len - 1] = 0;
  }
}

// Makes `definition` (e.g. "Coulomb -algorithm PMEwaldB200 -real -reciprocal -correction
// -interpolation BSpline -gridsize 20 20 20 -cutoff 8 -precision mixed") through a ForceFactory
// holding the B200 prototypes, evaluates it `repeat` times on the same positions (forces and
// energies of the last evaluation returned), and reports the made force's id in msg.
extern "C" int dropin_eval(const ref_input *in, const char *definition, int repeat, double *forces,
                           double *energies, double *virial, char *msg, int msglen) {
  try {
    Topo *t = make_topo(in);
    ForceFactory factory;
    B200::registerForces(factory);
    Force *f = factory.make(definition);
    SystemForce *sf = dynamic_cast<SystemForce *>(f);
    if (sf == NULL) {
      put(msg, msglen, "the factory made no system force");
      delete t;
      return 1;
    }
    Vector3DBlock pos(in->n), frc(in->n);
    ScalarStructure e;
    for (int r = 0; r < (repeat > 0 ? repeat : 1); r++) {
      for (int i = 0; i < in->n; i++) {
        pos[i] = Vector3D(in->pos[3 * i], in->pos[3 * i + 1], in->pos[3 * i + 2]);
        frc[i] = Vector3D(0, 0, 0);
      }
      e.clear();
      e.molecularVirial(false);
      e.virial(virial != NULL);
      sf->evaluate(t, &pos, &frc, &e);
    }
    for (int i = 0; i < in->n; i++)
      for (int k = 0; k < 3; k++) forces[3 * i + k] = frc[i].c[k];
    energies[0] = e[ScalarStructure::COULOMB];
    energies[1] = e[ScalarStructure::LENNARDJONES];
    if (virial)
      for (int k = 0; k < 9; k++) virial[k] = e[(ScalarStructure::Index)(ScalarStructure::VIRIALXX + k)];
    put(msg, msglen, f->getId());
    delete f;
    delete t;
    return 0;
  } catch (const Exception &ex) {
    put(msg, msglen, ex.getMessage());
    return 2;
  }
}

// Makes `definition` through the factory without evaluating it (no device needed): 0 and the
// made force's id with its parameters in msg, or 1 when the factory rejects the definition.
extern "C" int dropin_make(const char *definition, char *msg, int msglen) {
  try {
    ForceFactory factory;
    B200::registerForces(factory);
    Force *f = factory.make(definition);
    if (f == NULL) {
      put(msg, msglen, "rejected");
      return 1;
    }
    std::vector<Parameter> p;
    f->getParameters(p);
    std::string s = f->getId();
    for (unsigned int i = 0; i < p.size(); i++)
      s += " " + p[i].keyword + "=" + p[i].value.getString();
    put(msg, msglen, s);
    delete f;
    return 0;
  } catch (const Exception &ex) {
    put(msg, msglen, ex.getMessage());
    return 2;
  }
}
