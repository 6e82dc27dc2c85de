// ProtoMol module that puts the libpmgpu forces behind ProtoMol's own
// force-module API, so a .conf selects them with the usual grammar:
//
//   force LennardJones Coulomb -algorithm NonbondedCutoffGPU -cutoff 8
//         -ljswitch C2 -ljswitchon 7 -coulombswitch C2 -coulombswitchon 7
//   force LennardJones -algorithm NonbondedCutoffGPU -cutoff 9 -ljswitch C2 -ljswitchon 8
//   force Coulomb -algorithm PMEwaldGPU -alpha 0.35 -cutoff 9 -order 4 -gridsize 64
//   force Dihedral -algorithm TorsionGPU
//
// Each force is a SystemForce (force/system/SystemForce.h:16-85) whose
// evaluate() adds its forces into the caller's Vector3DBlock and its
// energies (and virial when requested) into the ScalarStructure, exactly
// the contract of the CPU forces it replaces.  All GPU forces of one
// topology share one pmgpu system, built on first use from the topology
// ProtoMol made (atoms, LJ table, exclusion table, periodic box, torsions).
// Registration follows module/BondedForcesModule.cpp: a Module whose
// registerForces() hands exemplars to app->forceFactory.
#include "PmgpuForceModule.h"

#include <protomol/ProtoMolApp.h>
#include <protomol/base/Exception.h>
#include <protomol/base/StringUtilities.h>
#include <protomol/config/Parameter.h>
#include <protomol/config/Value.h>
#include <protomol/force/system/SystemForce.h>
#include <protomol/topology/GenericTopology.h>
#include <protomol/topology/PeriodicBoundaryConditions.h>
#include <protomol/topology/SemiGenericTopology.h>
#include <protomol/type/ScalarStructure.h>
#include <protomol/type/Vector3DBlock.h>

#include <map>
#include <string>
#include <vector>

#include "pmgpu.h"

using namespace std;
using namespace ProtoMol;

namespace {

void check(int rc, const string &what) {
  if (rc != PMGPU_OK) THROW(what + ": " + pmgpu_last_error());
}

// One device context and one pmgpu system per ProtoMol topology.
struct Shared {
  pmgpu_context *ctx;
  map<const GenericTopology *, pmgpu_system *> systems;
  Shared() : ctx(0) {}
};
Shared &shared() {
  static Shared s;
  return s;
}

pmgpu_system *systemFor(const GenericTopology *topo) {
  Shared &sh = shared();
  map<const GenericTopology *, pmgpu_system *>::iterator it = sh.systems.find(topo);
  if (it != sh.systems.end()) return it->second;
  if (!sh.ctx) check(pmgpu_context_create(0, &sh.ctx), "pmgpu context");
  const int n = (int)topo->atoms.size();
  vector<double> q(n), m(n);
  vector<int> type(n), mol(n), water(n);
  for (int i = 0; i < n; i++) {
    const Atom &a = topo->atoms[i];
    q[i] = a.scaledCharge;
    m[i] = a.scaledMass;
    type[i] = a.type;
    mol[i] = a.molecule;
    water[i] = topo->molecules[a.molecule].water ? 1 : 0;
  }
  const int nt = (int)topo->lennardJonesParameters.size();
  vector<double> lj(4 * (size_t)nt * nt);
  for (int i = 0; i < nt; i++)
    for (int j = 0; j < nt; j++) {
      const LennardJonesParameters &p = topo->lennardJonesParameters(i, j);
      double *d = &lj[4 * ((size_t)i * nt + j)];
      d[0] = p.A;
      d[1] = p.B;
      d[2] = p.A14;
      d[3] = p.B14;
    }
  // exclusions: the pair forces use ExclusionTable::check(), the Ewald
  // correction iterates getTable()
  const vector<ExclusionPair> &ex = topo->exclusions.getTable();
  vector<int> excl(3 * ex.size()), table_class(ex.size());
  for (size_t k = 0; k < ex.size(); k++) {
    excl[3 * k] = ex[k].a1;
    excl[3 * k + 1] = ex[k].a2;
    excl[3 * k + 2] = (int)topo->exclusions.check(ex[k].a1, ex[k].a2);
    table_class[k] = (int)ex[k].excl;
  }
  vector<int> tors;
  vector<double> tprm;
  for (size_t k = 0; k < topo->dihedrals.size(); k++) {
    const Torsion &t = topo->dihedrals[k];
    for (int j = 0; j < t.multiplicity; j++) {
      tors.push_back(t.atom1);
      tors.push_back(t.atom2);
      tors.push_back(t.atom3);
      tors.push_back(t.atom4);
      tprm.push_back(t.forceConstant[j]);
      tprm.push_back((double)t.periodicity[j]);
      tprm.push_back(t.phaseShift[j]);
    }
  }
  pmgpu_topology t = pmgpu_topology();
  t.n_atoms = n;
  t.charge = &q[0];
  t.mass = &m[0];
  t.type = &type[0];
  t.molecule = &mol[0];
  t.n_types = nt;
  t.lj = lj.empty() ? 0 : &lj[0];
  t.n_exclusions = (int)ex.size();
  t.exclusions = excl.empty() ? 0 : &excl[0];
  t.exclusion_table_class = table_class.empty() ? 0 : &table_class[0];
  t.coulomb_scaling = topo->coulombScalingFactor;
  t.water = &water[0];
  t.gb_obc[0] = 1.0;
  t.gb_obc[1] = 0.8;
  t.gb_obc[2] = 4.85;
  t.n_dihedrals = (int)tors.size() / 4;
  t.dihedral_atoms = tors.empty() ? 0 : &tors[0];
  t.dihedral_params = tprm.empty() ? 0 : &tprm[0];
  const SemiGenericTopology<PeriodicBoundaryConditions> *pt =
      dynamic_cast<const SemiGenericTopology<PeriodicBoundaryConditions> *>(topo);
  if (pt) {
    const PeriodicBoundaryConditions &bc = pt->boundaryConditions;
    t.periodic = 1;
    for (int c = 0; c < 3; c++) {
      t.box[c] = bc.e1().c[c];
      t.box[3 + c] = bc.e2().c[c];
      t.box[6 + c] = bc.e3().c[c];
      t.box[9 + c] = bc.origin().c[c];
    }
  }
  pmgpu_system *s = 0;
  check(pmgpu_system_create(sh.ctx, &t, PMGPU_PREC_MIXED, &s), "pmgpu system");
  sh.systems[topo] = s;
  return s;
}

int switchKind(const string &name) {
  if (equalNocase(name, "C1")) return PMGPU_SW_C1;
  if (equalNocase(name, "C2")) return PMGPU_SW_C2;
  if (equalNocase(name, "Cutoff")) return PMGPU_SW_CUTOFF;
  if (equalNocase(name, "Universal")) return PMGPU_SW_UNIVERSAL;
  THROW("unknown switching function '" + name + "' (C1, C2, Cutoff)");
  return PMGPU_SW_CUTOFF;
}

// Common part of the GPU system forces: the force id inside the shared
// pmgpu system, made on first evaluation, and the ADD of forces, energies
// and virial into ProtoMol's containers.
class PmgpuSystemForce : public SystemForce {
 public:
  PmgpuSystemForce() : myId(-1), mySystem(0) {}
  using SystemForce::evaluate;
  virtual void evaluate(const GenericTopology *topo, const Vector3DBlock *positions,
                        Vector3DBlock *forces, ScalarStructure *energies) {
    pmgpu_system *s = systemFor(topo);
    if (s != mySystem || myId < 0) {
      mySystem = s;
      myId = addTo(s, topo);
    }
    double e[PMGPU_E_COUNT] = {0, 0, 0, 0, 0, 0, 0};
    double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const bool vir = energies->virial();
    check(pmgpu_force_evaluate(s, myId, positions->c, forces->c, e, vir ? v : 0),
          getIdNoAlias());
    (*energies)[ScalarStructure::COULOMB] += e[PMGPU_E_COULOMB];
    (*energies)[ScalarStructure::LENNARDJONES] += e[PMGPU_E_LENNARDJONES];
    (*energies)[ScalarStructure::DIHEDRAL] += e[PMGPU_E_DIHEDRAL];
    (*energies)[ScalarStructure::IMPROPER] += e[PMGPU_E_IMPROPER];
    if (vir)
      for (int k = 0; k < 9; k++)
        (*energies)[(ScalarStructure::Index)(ScalarStructure::VIRIALXX + k)] += v[k];
  }
  virtual void parallelEvaluate(const GenericTopology *topo, const Vector3DBlock *positions,
                                Vector3DBlock *forces, ScalarStructure *energies) {
    evaluate(topo, positions, forces, energies);
  }
  virtual unsigned int numberOfBlocks(const GenericTopology *, const Vector3DBlock *) {
    return 1;
  }

 protected:
  virtual int addTo(pmgpu_system *s, const GenericTopology *topo) const = 0;
  int myId;
  pmgpu_system *mySystem;
};

// NonbondedCutoff (module/NonbondedCutoffForceModule.cpp:40-201) on the GPU.
class CutoffGpuForce : public PmgpuSystemForce {
 public:
  CutoffGpuForce(const string &keyword, bool lj, bool coul)
      : myKeyword(keyword), myLJ(lj), myCoul(coul), myCutoff(8.0), myLJSwitch("C2"),
        myLJSwitchOn(0.0), myCoulSwitch("C2"), myCoulSwitchOn(0.0) {}
  virtual string getKeyword() const { return myKeyword; }
  virtual string getIdNoAlias() const { return myKeyword + " -algorithm NonbondedCutoffGPU"; }
  virtual void getParameters(vector<Parameter> &p) const {
    p.push_back(Parameter("-cutoff", Value(myCutoff, ConstraintValueType::Positive()), 8.0));
    p.push_back(Parameter("-ljswitch", Value(myLJSwitch), string("C2")));
    p.push_back(Parameter("-ljswitchon", Value(myLJSwitchOn), 0.0));
    p.push_back(Parameter("-coulombswitch", Value(myCoulSwitch), string("C2")));
    p.push_back(Parameter("-coulombswitchon", Value(myCoulSwitchOn), 0.0));
  }

 private:
  virtual Force *doMake(const vector<Value> &values) const {
    CutoffGpuForce *f = new CutoffGpuForce(myKeyword, myLJ, myCoul);
    f->myCutoff = values[0];
    f->myLJSwitch = values[1].getString();
    f->myLJSwitchOn = values[2];
    f->myCoulSwitch = values[3].getString();
    f->myCoulSwitchOn = values[4];
    return f;
  }
  virtual int addTo(pmgpu_system *s, const GenericTopology *topo) const {
    pmgpu_switch lj = {switchKind(myLJSwitch), myCutoff, myLJSwitchOn, 0.0, 0.0};
    pmgpu_switch co = {switchKind(myCoulSwitch), myCutoff, myCoulSwitchOn, 0.0, 0.0};
    int id = -1;
    check(pmgpu_force_cutoff_add(s, myLJ ? &lj : 0, myCoul ? &co : 0, myCutoff,
                                 0.0, &id),
          getIdNoAlias());
    return id;
  }
  string myKeyword;
  bool myLJ, myCoul;
  Real myCutoff;
  string myLJSwitch;
  Real myLJSwitchOn;
  string myCoulSwitch;
  Real myCoulSwitchOn;
};

// Ewald Coulomb (NonbondedFullEwaldSystemForce, -real -reciprocal
// -correction) with the reciprocal term as smooth PME.
class PmeGpuForce : public PmgpuSystemForce {
 public:
  PmeGpuForce() : myAlpha(0.35), myCutoff(9.0), myOrder(4), myGrid(64) {}
  virtual string getKeyword() const { return "Coulomb"; }
  virtual string getIdNoAlias() const { return "Coulomb -algorithm PMEwaldGPU"; }
  virtual void getParameters(vector<Parameter> &p) const {
    p.push_back(Parameter("-alpha", Value(myAlpha, ConstraintValueType::Positive()), 0.35));
    p.push_back(Parameter("-cutoff", Value(myCutoff, ConstraintValueType::Positive()), 9.0));
    p.push_back(Parameter("-order", Value(myOrder, ConstraintValueType::Positive()), 4));
    p.push_back(Parameter("-gridsize", Value(myGrid, ConstraintValueType::Positive()), 64));
  }

 private:
  virtual Force *doMake(const vector<Value> &values) const {
    PmeGpuForce *f = new PmeGpuForce();
    f->myAlpha = values[0];
    f->myCutoff = values[1];
    f->myOrder = values[2];
    f->myGrid = values[3];
    return f;
  }
  virtual int addTo(pmgpu_system *s, const GenericTopology *topo) const {
    const int grid[3] = {myGrid, myGrid, myGrid};
    int id = -1;
    check(pmgpu_force_pme_add(s, myAlpha, myCutoff, myOrder, grid, PMGPU_EWALD_ALL, 0,
                              0.0, &id),
          getIdNoAlias());
    return id;
  }
  Real myAlpha, myCutoff;
  int myOrder, myGrid;
};

// Dihedral torsions (force/bonded/DihedralSystemForce.h) on the GPU.
class TorsionGpuForce : public PmgpuSystemForce {
 public:
  virtual string getKeyword() const { return "Dihedral"; }
  virtual string getIdNoAlias() const { return "Dihedral -algorithm TorsionGPU"; }
  virtual void getParameters(vector<Parameter> &) const {}

 private:
  virtual Force *doMake(const vector<Value> &) const { return new TorsionGpuForce(); }
  virtual int addTo(pmgpu_system *s, const GenericTopology *) const {
    int id = -1;
    check(pmgpu_force_torsion_add(s, 1, 0, &id), getIdNoAlias());
    return id;
  }
};

}  // namespace

void PmgpuForceModule::registerForces(ProtoMolApp *app) {
  ForceFactory &f = app->forceFactory;
  f.registerExemplar(new CutoffGpuForce("LennardJones Coulomb", true, true));
  f.registerExemplar(new CutoffGpuForce("LennardJones", true, false));
  f.registerExemplar(new CutoffGpuForce("Coulomb", false, true));
  f.registerExemplar(new PmeGpuForce());
  f.registerExemplar(new TorsionGpuForce());
}
