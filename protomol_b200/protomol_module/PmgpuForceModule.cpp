// ProtoMol module that puts libpmgpu behind ProtoMol's own force and
// integrator factories, so a .conf selects the device path with the
// reference grammar, the algorithm name carrying a GPU suffix:
//
//   force LennardJones Coulomb -algorithm NonbondedCutoffGPU
//         -switchingFunction C2 -switchon 7 -cutoff 8
//         -switchingFunction C1 -cutoff 8 -cutoff 8
//   force Coulomb -algorithm PMEwaldGPU -alpha 0.35 -cutoff 9 -order 4 -gridsize 64
//   force GBBornRadii -algorithm NonbondedSimpleFullGPU
//   force GBPartialSum -algorithm NonbondedSimpleFullGPU
//   force GBForce -algorithm NonbondedSimpleFullGPU -soluteDielec 1 -solventDielec 78.5
//   force LennardJones -algorithm NonbondedSimpleFullGPU
//   force Dihedral -algorithm TorsionGPU
//   Integrator { level 0 LeapfrogGPU { timestep 1 force ... } }
//   Integrator { level 0 LangevinLeapfrogGPU { timestep 1 temperature 300
//                gamma 5 seed 1234 force ... } }
//
// Forces.  Each GPU force is a SystemForce (force/system/SystemForce.h:16-85)
// whose evaluate() adds its forces into the caller's Vector3DBlock and its
// energies (and virial when asked) into the ScalarStructure, the contract of
// the CPU forces it replaces; driven by a CPU integrator, positions go to
// the device and forces come back every evaluation.  The cutoff forces are
// registered per switching-function combination with the parameter lists of
// their CPU counterparts (OneAtomPair(Two)::getParameters, then the
// algorithm -cutoff, force/nonbonded/NonbondedCutoffForce.h:85-91), so the
// factory (factory/ForceFactory.cpp:21-242) reads the same lines.
//
// Integrators.  LeapfrogGPU and LangevinLeapfrogGPU are STSIntegrators
// whose run(n) (integrator/leapfrog/LeapfrogIntegrator.cpp:89-104 and
// StandardIntegrator.cpp:27-37 with LangevinLeapfrogIntegrator's half
// kicks) runs all n steps on the device: positions, velocities and forces
// stay resident, and only at the end of run(n) (ProtoMolApp::step hands
// run() the steps up to the next output, ProtoMolApp.cpp:486-498) are
// positions, velocities, forces and energies written back to the app for
// the outputs and checkpoints.  While ProtoMol writes those outputs the
// device already runs the next segment, started at the end of run(n) on the
// guess that it has as many steps; the next run() takes it when it does and
// the host left the state alone, and discards it (pmgpu_run_discard)
// otherwise.  Every force of their force group must have
// a device form: the GPU forces above, and the CPU Bond, Angle, Dihedral and
// Improper forces, which they map to the device's bonded terms.
//
// All GPU forces and integrators of one topology share one pmgpu system,
// built on first use from the topology ProtoMol made.  Registration follows
// module/BondedForcesModule.cpp and module/LeapfrogModule.cpp:18-24.
#include "PmgpuForceModule.h"

#include <protomol/ProtoMolApp.h>
#include <protomol/base/Exception.h>
#include <protomol/base/PMConstants.h>
#include <protomol/base/StringUtilities.h>
#include <protomol/config/Parameter.h>
#include <protomol/config/Value.h>
#include <protomol/force/ForceGroup.h>
#include <protomol/force/system/SystemForce.h>
#include <protomol/integrator/STSIntegrator.h>
#include <protomol/topology/GenericTopology.h>
#include <protomol/topology/PeriodicBoundaryConditions.h>
#include <protomol/topology/SemiGenericTopology.h>
#include <protomol/type/ScalarStructure.h>
#include <protomol/type/Vector3DBlock.h>

#include <cstdlib>
#include <cstring>
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

// The pmgpu topology of a ProtoMol topology: atoms (scaled charges and
// masses), the LJ table, the exclusion table (the class check() returns for
// the pair forces, the class the table holds for the Ewald correction),
// bonds, angles, torsions (one term per multiplicity), GB atom parameters
// and OBC constants, and the periodic box.
pmgpu_system *systemFor(const GenericTopology *topo) {
  Shared &sh = shared();
  map<const GenericTopology *, pmgpu_system *>::iterator it = sh.systems.find(topo);
  if (it != sh.systems.end()) return it->second;
  if (!sh.ctx) check(pmgpu_context_create(0, &sh.ctx), "pmgpu context");
  const int n = (int)topo->atoms.size();
  vector<double> q(n), m(n), vdwr(n), scale(n), offset(n);
  vector<int> type(n), mol(n), water(n);
  bool gb = n > 0;
  for (int i = 0; i < n; i++) {
    const Atom &a = topo->atoms[i];
    q[i] = a.scaledCharge;
    m[i] = a.scaledMass;
    type[i] = a.type;
    mol[i] = a.molecule;
    water[i] = topo->molecules[a.molecule].water ? 1 : 0;
    if (a.myGBSA_T) {
      vdwr[i] = a.myGBSA_T->vanDerWaalRadius;
      scale[i] = a.myGBSA_T->scalingFactor;
      offset[i] = a.myGBSA_T->offsetRadius;
    } else {
      gb = false;
    }
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
  const vector<ExclusionPair> &ex = topo->exclusions.getTable();
  vector<int> excl(3 * ex.size() + 3), table_class(ex.size() + 1);
  for (size_t k = 0; k < ex.size(); k++) {
    excl[3 * k] = ex[k].a1;
    excl[3 * k + 1] = ex[k].a2;
    excl[3 * k + 2] = (int)topo->exclusions.check(ex[k].a1, ex[k].a2);
    table_class[k] = (int)ex[k].excl;
  }
  vector<int> bonds, angles;
  vector<double> bprm, aprm;
  for (size_t k = 0; k < topo->bonds.size(); k++) {
    const Bond &b = topo->bonds[k];
    bonds.push_back(b.atom1);
    bonds.push_back(b.atom2);
    bprm.push_back(b.springConstant);
    bprm.push_back(b.restLength);
  }
  for (size_t k = 0; k < topo->angles.size(); k++) {
    const Angle &a = topo->angles[k];
    angles.push_back(a.atom1);
    angles.push_back(a.atom2);
    angles.push_back(a.atom3);
    aprm.push_back(a.forceConstant);
    aprm.push_back(a.restAngle);
    aprm.push_back(a.ureyBradleyConstant);
    aprm.push_back(a.ureyBradleyRestLength);
  }
  vector<int> tors[2];
  vector<double> tprm[2];
  for (int kind = 0; kind < 2; kind++) {
    const vector<Torsion> &list = kind == 0 ? topo->dihedrals : topo->impropers;
    for (size_t k = 0; k < list.size(); k++) {
      const Torsion &t = list[k];
      for (int j = 0; j < t.multiplicity; j++) {
        tors[kind].push_back(t.atom1);
        tors[kind].push_back(t.atom2);
        tors[kind].push_back(t.atom3);
        tors[kind].push_back(t.atom4);
        tprm[kind].push_back(t.forceConstant[j]);
        tprm[kind].push_back((double)t.periodicity[j]);
        tprm[kind].push_back(t.phaseShift[j]);
      }
    }
  }
  // SCPISM data as the topology builder formed it (BuildTopology.cpp:757-818)
  vector<double> scp[6];
  vector<int> scpi[3];
  if (topo->doSCPISM) {
    for (int k = 0; k < 6; k++) scp[k].resize(n);
    for (int k = 0; k < 3; k++) scpi[k].resize(n);
    for (int i = 0; i < n; i++) {
      const Atom &at = topo->atoms[i];
      const SCPISMAtomTypeParameters *tp = topo->atomTypes[at.type].mySCPISM_T;
      scp[0][i] = at.mySCPISM_A->sqrtalphaSCPISM;
      scp[1][i] = tp->alpha;
      scp[2][i] = at.mySCPISM_A->zeta;
      scp[3][i] = at.mySCPISM_A->eta;
      scp[4][i] = tp->C_i;
      scp[5][i] = tp->g_i;
      scpi[0][i] = (int)tp->isHbonded;
      scpi[1][i] = at.residue_seq;
      scpi[2][i] = at.name == "HN" ? 1 : (at.name == "O" ? 2 : 0);
    }
  }
  pmgpu_topology t;
  memset(&t, 0, sizeof(t));
  if (topo->doSCPISM && n) {
    t.scpism_sqrtalpha = &scp[0][0];
    t.scpism_alpha = &scp[1][0];
    t.scpism_zeta = &scp[2][0];
    t.scpism_eta = &scp[3][0];
    t.scpism_c = &scp[4][0];
    t.scpism_g = &scp[5][0];
    t.scpism_hbond = &scpi[0][0];
    t.scpism_residue = &scpi[1][0];
    t.scpism_name = &scpi[2][0];
  }
  t.n_atoms = n;
  t.charge = n ? &q[0] : 0;
  t.mass = n ? &m[0] : 0;
  t.type = n ? &type[0] : 0;
  t.molecule = n ? &mol[0] : 0;
  t.n_types = nt;
  t.lj = lj.empty() ? 0 : &lj[0];
  t.n_exclusions = (int)ex.size();
  t.exclusions = &excl[0];
  t.exclusion_table_class = &table_class[0];
  t.coulomb_scaling = topo->coulombScalingFactor;
  t.n_bonds = (int)topo->bonds.size();
  t.bond_atoms = bonds.empty() ? 0 : &bonds[0];
  t.bond_params = bprm.empty() ? 0 : &bprm[0];
  t.n_angles = (int)topo->angles.size();
  t.angle_atoms = angles.empty() ? 0 : &angles[0];
  t.angle_params = aprm.empty() ? 0 : &aprm[0];
  if (gb) {
    t.gb_vdwr = &vdwr[0];
    t.gb_scale = &scale[0];
    t.gb_offset = &offset[0];
  }
  t.water = n ? &water[0] : 0;
  // OBC constants as ProtoMolApp sets them for doGBSAObc (ProtoMolApp.cpp:285-299)
  t.gb_obc[0] = topo->alphaObc;
  t.gb_obc[1] = topo->betaObc;
  t.gb_obc[2] = topo->gammaObc;
  t.n_dihedrals = (int)tors[0].size() / 4;
  t.dihedral_atoms = tors[0].empty() ? 0 : &tors[0][0];
  t.dihedral_params = tprm[0].empty() ? 0 : &tprm[0][0];
  t.n_impropers = (int)tors[1].size() / 4;
  t.improper_atoms = tors[1].empty() ? 0 : &tors[1][0];
  t.improper_params = tprm[1].empty() ? 0 : &tprm[1][0];
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

// Adds the device's energies (ScalarStructure slots COULOMB .. OTHER) and
// virial into ProtoMol's ScalarStructure.
void addEnergies(ScalarStructure *energies, const double *e, const double *v) {
  static const ScalarStructure::Index slot[PMGPU_E_COUNT] = {
      ScalarStructure::COULOMB, ScalarStructure::LENNARDJONES, ScalarStructure::BOND,
      ScalarStructure::ANGLE, ScalarStructure::DIHEDRAL, ScalarStructure::IMPROPER,
      ScalarStructure::OTHER};
  for (int k = 0; k < PMGPU_E_COUNT; k++) (*energies)[slot[k]] += e[k];
  if (v)
    for (int k = 0; k < 9; k++)
      (*energies)[(ScalarStructure::Index)(ScalarStructure::VIRIALXX + k)] += v[k];
}

// Common part of the GPU system forces: the force id inside the shared
// pmgpu system (attach() makes it once per system) and the ADD of forces,
// energies and virial into ProtoMol's containers.
class PmgpuSystemForce : public SystemForce {
 public:
  PmgpuSystemForce() : myId(-1), mySystem(0) {}
  // The force's id in s (-1: a pass that runs inside another force).
  int attach(pmgpu_system *s, const GenericTopology *topo) {
    if (s != mySystem) {
      mySystem = s;
      myId = addTo(s, topo);
    }
    return myId;
  }
  using SystemForce::evaluate;
  virtual void evaluate(const GenericTopology *topo, const Vector3DBlock *positions,
                        Vector3DBlock *forces, ScalarStructure *energies) {
    const int id = attach(systemFor(topo), topo);
    if (id < 0) return;
    double e[PMGPU_E_COUNT] = {0, 0, 0, 0, 0, 0, 0};
    double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const bool vir = energies->virial();
    check(pmgpu_force_evaluate(mySystem, id, positions->c, forces->c, e, vir ? v : 0),
          getIdNoAlias());
    addEnergies(energies, e, vir ? v : 0);
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

// ---------------------------------------------------------------- switches
// A switching function's kind and the parameters its CPU counterpart reads,
// in its order (switch/C1SwitchingFunction.cpp:18-22,
// C2SwitchingFunction.cpp:20-28, CnSwitchingFunction.cpp:64-79,
// CutoffSwitchingFunction.h:47-51).
enum { P_N = 0, P_SWITCHON, P_SWITCHOFF, P_CUTOFF };
struct SwitchSpec {
  const char *name;
  int kind;
  int nparams;
  int params[4];
};
const SwitchSpec kC1 = {"C1", PMGPU_SW_C1, 1, {P_CUTOFF}};
const SwitchSpec kC2 = {"C2", PMGPU_SW_C2, 2, {P_SWITCHON, P_CUTOFF}};
const SwitchSpec kCn = {"Cn", PMGPU_SW_CN, 4, {P_N, P_SWITCHON, P_SWITCHOFF, P_CUTOFF}};
const SwitchSpec kCutoff = {"Cutoff", PMGPU_SW_CUTOFF, 1, {P_CUTOFF}};
// CmpCnCnSwitchingFunction.cpp:27-45 (its id is spelled "ComplimentCnCn")
const SwitchSpec kCmpCnCn = {"ComplimentCnCn", PMGPU_SW_CMPCNCN, 4,
                             {P_SWITCHON, P_SWITCHOFF, P_CUTOFF, P_N}};
// ComplementSwitchingFunction.h:48-60: "Complement" + the function's id and
// its parameters
const SwitchSpec kCompC1 = {"ComplementC1", PMGPU_SW_C1 | PMGPU_SW_COMPLEMENT, 1, {P_CUTOFF}};
const SwitchSpec kCompC2 = {"ComplementC2", PMGPU_SW_C2 | PMGPU_SW_COMPLEMENT, 2,
                            {P_SWITCHON, P_CUTOFF}};
const SwitchSpec kCompCn = {"ComplementCn", PMGPU_SW_CN | PMGPU_SW_COMPLEMENT, 4,
                            {P_N, P_SWITCHON, P_SWITCHOFF, P_CUTOFF}};

void switchParameters(const SwitchSpec &sw, const pmgpu_switch &v, vector<Parameter> &p) {
  for (int k = 0; k < sw.nparams; k++) switch (sw.params[k]) {
      case P_N:
        p.push_back(Parameter("-n", Value(v.order, ConstraintValueType::Positive())));
        break;
      case P_SWITCHON:
        p.push_back(Parameter("-switchon", Value(v.switchon, ConstraintValueType::NotNegative())));
        break;
      case P_SWITCHOFF:
        p.push_back(Parameter("-switchoff", Value(v.switchoff,
                                                  ConstraintValueType::NotNegative()), 0.0));
        break;
      default:
        p.push_back(Parameter("-cutoff", Value(v.cutoff, ConstraintValueType::Positive())));
        break;
    }
}

// Reads the switch's values from values[*at...], advancing *at.
pmgpu_switch switchMake(const SwitchSpec &sw, const vector<Value> &values, size_t *at) {
  pmgpu_switch s;
  s.kind = sw.kind;
  s.cutoff = s.switchon = s.switchoff = s.order = 0.0;
  for (int k = 0; k < sw.nparams; k++) {
    Real x = 0;
    values[(*at)++].get(x);
    switch (sw.params[k]) {
      case P_N: s.order = x; break;
      case P_SWITCHON: s.switchon = x; break;
      case P_SWITCHOFF: s.switchoff = x; break;
      default: s.cutoff = x; break;
    }
  }
  return s;
}

// ---------------------------------------------------------------- forces
// NonbondedCutoff (module/NonbondedCutoffForceModule.cpp:55-96) on the GPU:
// LennardJones and/or Coulomb, one switching function each; with full set,
// the NonbondedFull lattice sum (module/NonbondedFullForceModule.cpp:39-46,
// force/nonbonded/NonbondedFullSystemForce.h, which adds -blocksize).
class CutoffGpuForce : public PmgpuSystemForce {
 public:
  CutoffGpuForce(bool lj, bool coul, const SwitchSpec &a, const SwitchSpec *b, bool full = false)
      : myLJ(lj), myCoul(coul), mySwA(a), mySwB(b ? *b : a), myTwo(b != 0), myFull(full),
        myCutoff(8.0), myBlock(64) {
    memset(&myA, 0, sizeof(myA));
    memset(&myB, 0, sizeof(myB));
  }
  virtual string getKeyword() const { return myFull ? "NonbondedFullGPU" : "NonbondedCutoffGPU"; }
  virtual string getIdNoAlias() const {
    string id = myTwo ? "LennardJones Coulomb" : (myLJ ? "LennardJones" : "Coulomb");
    id += string(" -switchingFunction ") + mySwA.name;
    if (myTwo) id += string(" -switchingFunction ") + mySwB.name;
    return id + " -algorithm " + getKeyword();
  }
  virtual void getParameters(vector<Parameter> &p) const {
    switchParameters(mySwA, myA, p);
    if (myTwo) switchParameters(mySwB, myB, p);
    p.push_back(Parameter("-cutoff", Value(myCutoff, ConstraintValueType::Positive())));
    if (myFull)
      p.push_back(Parameter("-blocksize", Value(myBlock, ConstraintValueType::Positive()), 64));
  }

 private:
  virtual Force *doMake(const vector<Value> &values) const {
    CutoffGpuForce *f = new CutoffGpuForce(myLJ, myCoul, mySwA, myTwo ? &mySwB : 0, myFull);
    size_t at = 0;
    f->myA = switchMake(mySwA, values, &at);
    if (myTwo) f->myB = switchMake(mySwB, values, &at);
    values[at++].get(f->myCutoff);
    if (myFull) values[at].get(f->myBlock);  // read and ignored: the device tiles its own way
    return f;
  }
  virtual int addTo(pmgpu_system *s, const GenericTopology *) const {
    const pmgpu_switch *lj = myLJ ? &myA : 0;
    const pmgpu_switch *co = myCoul ? (myTwo ? &myB : &myA) : 0;
    int id = -1;
    if (myFull)
      check(pmgpu_force_full_add(s, lj, co, myCutoff, 0.0, &id), getIdNoAlias());
    else
      check(pmgpu_force_cutoff_add(s, lj, co, myCutoff, 0.0, &id), getIdNoAlias());
    return id;
  }
  bool myLJ, myCoul;
  SwitchSpec mySwA, mySwB;
  bool myTwo, myFull;
  pmgpu_switch myA, myB;
  Real myCutoff;
  int myBlock;
};

// Ewald Coulomb (NonbondedFullEwaldSystemForce, -real -reciprocal
// -correction) with the reciprocal term as smooth PME.
class PmeGpuForce : public PmgpuSystemForce {
 public:
  PmeGpuForce() : myAlpha(0.35), myCutoff(9.0), myOrder(4), myGrid(64) {}
  virtual string getKeyword() const { return "PMEwaldGPU"; }
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
  virtual int addTo(pmgpu_system *s, const GenericTopology *) const {
    const int grid[3] = {myGrid, myGrid, myGrid};
    int id = -1;
    check(pmgpu_force_pme_add(s, myAlpha, myCutoff, myOrder, grid, PMGPU_EWALD_ALL, 0, 0.0, &id),
          getIdNoAlias());
    return id;
  }
  Real myAlpha, myCutoff;
  int myOrder, myGrid;
};

// NonbondedSimpleFull LennardJones / Coulomb (vacuum all pairs,
// module/NonbondedSimpleFullForceModule.cpp) on the GPU; -blocksize is read
// and ignored, as the device tiles its own way
// (NonbondedSimpleFullSystemForce.h:93-99).
class SimpleFullGpuForce : public PmgpuSystemForce {
 public:
  SimpleFullGpuForce(bool lj, bool coul) : myLJ(lj), myCoul(coul), myBlock(64) {}
  virtual string getKeyword() const { return "NonbondedSimpleFullGPU"; }
  virtual string getIdNoAlias() const {
    return string(myLJ && myCoul ? "LennardJones Coulomb" : (myLJ ? "LennardJones" : "Coulomb")) +
           " -algorithm " + getKeyword();
  }
  virtual void getParameters(vector<Parameter> &p) const {
    p.push_back(Parameter("-blocksize", Value(myBlock, ConstraintValueType::Positive()), 64));
  }

 private:
  virtual Force *doMake(const vector<Value> &values) const {
    SimpleFullGpuForce *f = new SimpleFullGpuForce(myLJ, myCoul);
    f->myBlock = values[0];
    return f;
  }
  virtual int addTo(pmgpu_system *s, const GenericTopology *) const {
    int id = -1;
    const int rc = pmgpu_force_simplefull_add(s, myLJ ? 1 : 0, myCoul ? 1 : 0, &id);
    if (rc == PMGPU_ERR_UNSUPPORTED) {
      // a periodic box: every pair's minimal image, Universal switching
      pmgpu_switch u;
      memset(&u, 0, sizeof(u));
      u.kind = PMGPU_SW_UNIVERSAL;
      check(pmgpu_force_simplefull_switched_add(s, myLJ ? &u : 0, myCoul ? &u : 0, &id),
            getIdNoAlias());
      return id;
    }
    check(rc, getIdNoAlias());
    return id;
  }
  bool myLJ, myCoul;
  int myBlock;
};

// NonbondedSimpleFull with switching functions (module/
// NonbondedSimpleFullForceModule.cpp:55-199: C1, C2, Cn and the Complement
// of C1, C2 and Cn, one or two terms), vacuum or periodic.
class SimpleFullSwGpuForce : public PmgpuSystemForce {
 public:
  SimpleFullSwGpuForce(bool lj, bool coul, const SwitchSpec &a, const SwitchSpec *b)
      : myLJ(lj), myCoul(coul), mySwA(a), mySwB(b ? *b : a), myTwo(b != 0), myBlock(64) {
    memset(&myA, 0, sizeof(myA));
    memset(&myB, 0, sizeof(myB));
  }
  virtual string getKeyword() const { return "NonbondedSimpleFullGPU"; }
  virtual string getIdNoAlias() const {
    string id = myTwo ? "LennardJones Coulomb" : (myLJ ? "LennardJones" : "Coulomb");
    id += string(" -switchingFunction ") + mySwA.name;
    if (myTwo) id += string(" -switchingFunction ") + mySwB.name;
    return id + " -algorithm " + getKeyword();
  }
  virtual void getParameters(vector<Parameter> &p) const {
    switchParameters(mySwA, myA, p);
    if (myTwo) switchParameters(mySwB, myB, p);
    p.push_back(Parameter("-blocksize", Value(myBlock, ConstraintValueType::Positive()), 64));
  }

 private:
  virtual Force *doMake(const vector<Value> &values) const {
    SimpleFullSwGpuForce *f = new SimpleFullSwGpuForce(myLJ, myCoul, mySwA, myTwo ? &mySwB : 0);
    size_t at = 0;
    f->myA = switchMake(mySwA, values, &at);
    if (myTwo) f->myB = switchMake(mySwB, values, &at);
    values[at].get(f->myBlock);
    return f;
  }
  virtual int addTo(pmgpu_system *s, const GenericTopology *) const {
    const pmgpu_switch *lj = myLJ ? &myA : 0;
    const pmgpu_switch *co = myCoul ? (myTwo ? &myB : &myA) : 0;
    int id = -1;
    check(pmgpu_force_simplefull_switched_add(s, lj, co, &id), getIdNoAlias());
    return id;
  }
  bool myLJ, myCoul;
  SwitchSpec mySwA, mySwB;
  bool myTwo;
  pmgpu_switch myA, myB;
  int myBlock;
};

// The OBC GB chain (force/GB/GBBornRadii.cpp, GBPartialSum.cpp, GBForce.cpp,
// GBACEForce.cpp) as NonbondedSimpleFull forces.  The device runs the
// passes inside GBForce's (and GBACEForce's) evaluation, so GBBornRadii and
// GBPartialSum only keep their places in the force list (they add no force
// and no energy in the reference either); GBForce and GBACEForce add their
// forces and energies (COULOMB).
class GbGpuForce : public PmgpuSystemForce {
 public:
  explicit GbGpuForce(const string &keyword)
      : myKeyword(keyword), mySolute(1.0), mySolvent(80.0), mySigma(2.26 / 418.4),
        myRho(1.4), myBlock(64) {}
  virtual string getKeyword() const { return "NonbondedSimpleFullGPU"; }
  virtual string getIdNoAlias() const { return myKeyword + " -algorithm " + getKeyword(); }
  virtual void getParameters(vector<Parameter> &p) const {
    if (myKeyword == "GBForce") {
      p.push_back(Parameter("-soluteDielec",
                            Value(mySolute, ConstraintValueType::NoConstraints()), 1.0));
      p.push_back(Parameter("-solventDielec",
                            Value(mySolvent, ConstraintValueType::NoConstraints()), 80.0));
    } else if (myKeyword == "GBACEForce") {
      // GBACEForce::getParameters (force/GB/GBACEForce.cpp:224-230)
      p.push_back(Parameter("-solvationparam",
                            Value(mySigma, ConstraintValueType::NoConstraints()), 2.26 / 418.4));
      p.push_back(Parameter("-watersphereradius",
                            Value(myRho, ConstraintValueType::NoConstraints()), 1.4));
    }
    p.push_back(Parameter("-blocksize", Value(myBlock, ConstraintValueType::Positive()), 64));
  }

 private:
  virtual Force *doMake(const vector<Value> &values) const {
    GbGpuForce *f = new GbGpuForce(myKeyword);
    size_t at = 0;
    if (myKeyword == "GBForce") {
      f->mySolute = values[at++];
      f->mySolvent = values[at++];
    } else if (myKeyword == "GBACEForce") {
      f->mySigma = values[at++];
      f->myRho = values[at++];
    }
    f->myBlock = values[at];
    return f;
  }
  virtual int addTo(pmgpu_system *s, const GenericTopology *) const {
    int id = -1;
    if (myKeyword == "GBForce")
      check(pmgpu_force_gb_add(s, mySolute, mySolvent, &id), getIdNoAlias());
    else if (myKeyword == "GBACEForce")
      check(pmgpu_force_gbace_add(s, mySigma, myRho, &id), getIdNoAlias());
    return id;
  }
  string myKeyword;
  Real mySolute, mySolvent, mySigma, myRho;
  int myBlock;
};

// LennardJones and/or CoulombSCPISM (force/coulomb/CoulombSCPISMForce.h)
// on NonbondedCutoff or NonbondedSimpleFull (module/NonbondedCutoffForce
// Module.cpp:91-107, :150-160; NonbondedSimpleFullForceModule.cpp:104-116)
// on the GPU: the parameters in the reference's order, each force's own
// (-D for CoulombSCPISM) before its switch's, then the algorithm's.
class ScpismGpuForce : public PmgpuSystemForce {
 public:
  ScpismGpuForce(bool simpleFull, const SwitchSpec *lj, const SwitchSpec &coul)
      : myFull(simpleFull), myTwo(lj != 0), mySwA(lj ? *lj : coul), mySwB(coul), myD(80.0),
        myCutoff(8.0), myBlock(64) {
    memset(&myA, 0, sizeof(myA));
    memset(&myB, 0, sizeof(myB));
  }
  virtual string getKeyword() const {
    return myFull ? "NonbondedSimpleFullGPU" : "NonbondedCutoffGPU";
  }
  virtual string getIdNoAlias() const {
    string id = myTwo ? "LennardJones CoulombSCPISM" : "CoulombSCPISM";
    if (myTwo) id += string(" -switchingFunction ") + mySwA.name;
    id += string(" -switchingFunction ") + mySwB.name;
    return id + " -algorithm " + getKeyword();
  }
  virtual void getParameters(vector<Parameter> &p) const {
    if (myTwo) switchParameters(mySwA, myA, p);
    p.push_back(Parameter("-D", Value(myD, ConstraintValueType::NotNegative()), 80.0));
    switchParameters(mySwB, myB, p);
    if (myFull)
      p.push_back(Parameter("-blocksize", Value(myBlock, ConstraintValueType::Positive()), 64));
    else
      p.push_back(Parameter("-cutoff", Value(myCutoff, ConstraintValueType::Positive())));
  }

 private:
  virtual Force *doMake(const vector<Value> &values) const {
    ScpismGpuForce *f = new ScpismGpuForce(myFull, myTwo ? &mySwA : 0, mySwB);
    size_t at = 0;
    if (myTwo) f->myA = switchMake(mySwA, values, &at);
    values[at++].get(f->myD);
    f->myB = switchMake(mySwB, values, &at);
    if (myFull)
      values[at].get(f->myBlock);
    else
      values[at].get(f->myCutoff);
    return f;
  }
  virtual int addTo(pmgpu_system *s, const GenericTopology *) const {
    int id = -1;
    check(pmgpu_force_scpism_add(s, myTwo ? &myA : 0, &myB, myD, &id), getIdNoAlias());
    return id;
  }
  bool myFull, myTwo;
  SwitchSpec mySwA, mySwB;
  pmgpu_switch myA, myB;
  Real myD, myCutoff;
  int myBlock;
};

// BornRadii and BornSelf (force/born/BornRadii.h, BornSelfForce.h) with
// the Cutoff switch on NonbondedCutoff.  The device runs both passes in
// BornSelf's evaluation: BornRadii only records its -bornswitch and cutoff
// for the BornSelf line that follows it (it adds no force or energy in the
// reference either).
map<pmgpu_system *, pair<int, Real> > &bornRadiiSettings() {
  static map<pmgpu_system *, pair<int, Real> > m;
  return m;
}

class BornGpuForce : public PmgpuSystemForce {
 public:
  explicit BornGpuForce(bool self)
      : mySelf(self), mySwitch(3), myD(80.0), mySwCutoff(5.0), myCutoff(5.0) {}
  virtual string getKeyword() const { return "NonbondedCutoffGPU"; }
  virtual string getIdNoAlias() const {
    return string(mySelf ? "BornSelf" : "BornRadii") +
           " -switchingFunction Cutoff -algorithm NonbondedCutoffGPU";
  }
  virtual void getParameters(vector<Parameter> &p) const {
    // BornRadii.cpp:9-13, BornSelfForce.cpp:8-16, then the Cutoff switch
    // and the algorithm's cutoff
    p.push_back(Parameter("-bornswitch", Value(mySwitch, ConstraintValueType::NotNegative()), 3));
    if (mySelf) p.push_back(Parameter("-D", Value(myD, ConstraintValueType::NotNegative()), 80.0));
    p.push_back(Parameter("-cutoff", Value(mySwCutoff, ConstraintValueType::Positive())));
    p.push_back(Parameter("-cutoff", Value(myCutoff, ConstraintValueType::Positive())));
  }

 private:
  virtual Force *doMake(const vector<Value> &values) const {
    BornGpuForce *f = new BornGpuForce(mySelf);
    size_t at = 0;
    values[at++].get(f->mySwitch);
    if (mySelf) values[at++].get(f->myD);
    values[at++].get(f->mySwCutoff);
    values[at].get(f->myCutoff);
    return f;
  }
  virtual int addTo(pmgpu_system *s, const GenericTopology *) const {
    if (!mySelf) {
      bornRadiiSettings()[s] = make_pair(mySwitch, mySwCutoff);
      return -1;
    }
    pair<int, Real> r(3, 5.0);
    if (bornRadiiSettings().count(s)) r = bornRadiiSettings()[s];
    int id = -1;
    check(pmgpu_force_born_add(s, r.first, r.second, mySwitch, mySwCutoff, myD, &id),
          getIdNoAlias());
    return id;
  }
  bool mySelf;
  int mySwitch;
  Real myD, mySwCutoff, myCutoff;
};

// Dihedral / Improper torsions (force/bonded/DihedralSystemForce.h,
// ImproperSystemForce.h; MTorsionSystemForce) on the GPU.
class TorsionGpuForce : public PmgpuSystemForce {
 public:
  explicit TorsionGpuForce(bool dihedral) : myDihedral(dihedral) {}
  virtual string getKeyword() const { return "TorsionGPU"; }
  virtual string getIdNoAlias() const {
    return string(myDihedral ? "Dihedral" : "Improper") + " -algorithm TorsionGPU";
  }
  virtual void getParameters(vector<Parameter> &) const {}

 private:
  virtual Force *doMake(const vector<Value> &) const { return new TorsionGpuForce(myDihedral); }
  virtual int addTo(pmgpu_system *s, const GenericTopology *) const {
    int id = -1;
    check(pmgpu_force_torsion_add(s, myDihedral ? 1 : 0, myDihedral ? 0 : 1, &id),
          getIdNoAlias());
    return id;
  }
  bool myDihedral;
};

// ------------------------------------------------------------ integrators
// Leapfrog / LangevinLeapfrog with every step on the device.
class DeviceIntegrator : public STSIntegrator {
 public:
  DeviceIntegrator(int kind, Real timestep, Real temperature, Real gamma, int seed,
                   ForceGroup *fg)
      : STSIntegrator(timestep, fg), myKind(kind), myTemperature(temperature),
        myGamma(gamma), mySeed(seed), mySystem(0), mySpeculated(0) {}

  virtual void initialize(ProtoMolApp *app) {
    STSIntegrator::initialize(app);
    if (mySystem && mySpeculated) check(pmgpu_run_discard(mySystem), getIdNoAlias());
    mySpeculated = 0;
    mySystem = systemFor(app->topology);
    // every force of the group gets its device form; only those run
    const vector<Force *> forces = myForcesToEvaluate->getForces();
    vector<int> ids;
    for (size_t k = 0; k < forces.size(); k++) {
      PmgpuSystemForce *g = dynamic_cast<PmgpuSystemForce *>(forces[k]);
      int id = -1;
      if (g) {
        id = g->attach(mySystem, app->topology);
      } else {
        const string kw = forces[k]->getKeyword();
        if (equalNocase(kw, "Bond") || equalNocase(kw, "Angle"))
          check(pmgpu_force_bonded_add(mySystem, equalNocase(kw, "Bond"), equalNocase(kw, "Angle"),
                                       &id), kw);
        else if (equalNocase(kw, "Dihedral") || equalNocase(kw, "Improper"))
          check(pmgpu_force_torsion_add(mySystem, equalNocase(kw, "Dihedral"),
                                        equalNocase(kw, "Improper"), &id), kw);
        else
          THROW(getIdNoAlias() + ": force '" + forces[k]->getId() +
                "' has no device form (use a GPU algorithm)");
      }
      if (id >= 0) ids.push_back(id);
    }
    // forces attached to the system by other integrators stay off here
    pmgpu_stats st;
    for (int id = 0; pmgpu_force_stats(mySystem, id, &st) == PMGPU_OK; id++) {
      bool mine = false;
      for (size_t k = 0; k < ids.size(); k++) mine = mine || ids[k] == id;
      check(pmgpu_force_set_enabled(mySystem, id, mine ? 1 : 0), getIdNoAlias());
    }
    myHostPos.clear();
    myHostVel.clear();
    // Integrator::initialize evaluates the initial forces (and energies)
    upload();
    double e[PMGPU_E_COUNT];
    check(pmgpu_evaluate(mySystem, e, 0), getIdNoAlias());
    download(e);
  }

  virtual long run(const long numTimesteps) {
    if (numTimesteps < 1) return 0;
    pmgpu_integrator it;
    it.kind = myKind;
    it.timestep_fs = getTimestep();
    it.temperature = myTemperature;
    it.gamma_ps = myGamma;
    it.seed = (uint64_t)mySeed;
    // the segment started at the end of the last run() is these steps if it
    // has as many and the host left the state as it was handed over
    if (mySpeculated == numTimesteps && hostUnchanged()) {
      check(pmgpu_run_wait(mySystem), getIdNoAlias());
    } else {
      if (mySpeculated) check(pmgpu_run_discard(mySystem), getIdNoAlias());
      upload();
      check(pmgpu_run(mySystem, &it, numTimesteps), getIdNoAlias());
    }
    mySpeculated = 0;
    // the simulated time the outputs report, advanced by the steps taken
    // (as the reference's own device integrator does,
    // integrator/openMM/OpenMMIntegrator.cpp:688)
    app->topology->time += numTimesteps * getTimestep();
    double e[PMGPU_E_COUNT];
    check(pmgpu_system_get_energies(mySystem, e, 0), getIdNoAlias());
    download(e);
    // ProtoMolApp::step writes its outputs from the state just handed back
    // before it asks for the next steps (ProtoMolApp.cpp:474-500): the next
    // segment, guessed to be as long as this one, runs on the device
    // meanwhile.  Only when this integrator is the application's (no other
    // integrator touches the system between the calls), not past lastStep,
    // and unless PMGPU_OVERLAP=0.
    const long next = app->currentStep + numTimesteps;
    if (overlapEnabled() && app->integrator == this &&
        (app->lastStep < 0 || next + numTimesteps <= app->lastStep)) {
      check(pmgpu_run_async(mySystem, &it, numTimesteps), getIdNoAlias());
      mySpeculated = numTimesteps;
    }
    return numTimesteps;
  }

  virtual void getParameters(vector<Parameter> &parameters) const {
    STSIntegrator::getParameters(parameters);
    if (myKind == PMGPU_INT_LANGEVIN_LEAPFROG) {
      // LangevinLeapfrogIntegrator::getParameters (integrator/base/
      // LangevinLeapfrogIntegrator.cpp:74-85)
      parameters.push_back(Parameter("temperature",
                                     Value(myTemperature, ConstraintValueType::NotNegative())));
      parameters.push_back(Parameter("gamma", Value(myGamma, ConstraintValueType::NotNegative())));
      parameters.push_back(Parameter("seed", Value(mySeed, ConstraintValueType::NotNegative()),
                                     1234));
    }
  }
  virtual string getIdNoAlias() const {
    return myKind == PMGPU_INT_LEAPFROG ? "LeapfrogGPU" : "LangevinLeapfrogGPU";
  }

 private:
  virtual STSIntegrator *doMake(const vector<Value> &values, ForceGroup *fg) const {
    if (myKind == PMGPU_INT_LEAPFROG) return new DeviceIntegrator(myKind, values[0], 0, 0, 0, fg);
    return new DeviceIntegrator(myKind, values[0], values[1], values[2], values[3], fg);
  }

  static bool overlapEnabled() {
    const char *v = getenv("PMGPU_OVERLAP");
    return !(v && v[0] == '0');
  }
  bool hostUnchanged() const {
    const size_t n3 = 3 * app->positions.size();
    return myHostPos.size() == n3 && myHostVel.size() == n3 &&
           memcmp(&myHostPos[0], app->positions.c, n3 * sizeof(double)) == 0 &&
           memcmp(&myHostVel[0], app->velocities.c, n3 * sizeof(double)) == 0;
  }
  // Positions and velocities go to the device only when the host changed
  // them since the last download (a modifier, a restart, the first call).
  void upload() {
    const size_t n3 = 3 * app->positions.size();
    const double *x = app->positions.c, *v = app->velocities.c;
    if (myHostPos.size() != n3 || memcmp(&myHostPos[0], x, n3 * sizeof(double)) != 0)
      check(pmgpu_system_set_positions(mySystem, x), getIdNoAlias());
    if (myHostVel.size() != n3 || memcmp(&myHostVel[0], v, n3 * sizeof(double)) != 0)
      check(pmgpu_system_set_velocities(mySystem, v), getIdNoAlias());
  }
  // The state at the end of a run() (or the initial evaluation) back in the
  // app: positions, velocities, this integrator's forces and the energies.
  void download(const double *e) {
    const size_t n3 = 3 * app->positions.size();
    check(pmgpu_system_get_positions(mySystem, app->positions.c), getIdNoAlias());
    check(pmgpu_system_get_velocities(mySystem, app->velocities.c), getIdNoAlias());
    check(pmgpu_system_get_forces(mySystem, myForces->c), getIdNoAlias());
    myHostPos.assign(app->positions.c, app->positions.c + n3);
    myHostVel.assign(app->velocities.c, app->velocities.c + n3);
    app->energies.clear();
    addEnergies(&app->energies, e, 0);
  }

  int myKind;
  Real myTemperature, myGamma;
  int mySeed;
  pmgpu_system *mySystem;
  vector<double> myHostPos, myHostVel;
  long mySpeculated;  // steps of the segment started ahead of the next run() (0: none)
};

}  // namespace

void PmgpuForceModule::registerForces(ProtoMolApp *app) {
  ForceFactory &f = app->forceFactory;
  // the switching-function combinations the reference registers for
  // NonbondedCutoff (module/NonbondedCutoffForceModule.cpp:55-96), plus Cutoff
  const SwitchSpec singles[] = {kC1, kC2, kCn, kCutoff, kCmpCnCn};
  for (int k = 0; k < 5; k++) {
    f.registerExemplar(new CutoffGpuForce(true, false, singles[k], 0));
    f.registerExemplar(new CutoffGpuForce(false, true, singles[k], 0));
  }
  const SwitchSpec pairs[][2] = {{kC2, kC1}, {kC2, kC2}, {kC2, kCn}, {kCn, kCn}, {kCn, kC2},
                                 {kCutoff, kCutoff}, {kC2, kCutoff}, {kCmpCnCn, kCmpCnCn}};
  for (int k = 0; k < 8; k++)
    f.registerExemplar(new CutoffGpuForce(true, true, pairs[k][0], &pairs[k][1]));
  // NonbondedFull: one term, C1, C2, Cn or CmpCnCn
  // (module/NonbondedFullForceModule.cpp:39-46)
  const SwitchSpec fulls[] = {kC1, kC2, kCn, kCmpCnCn};
  for (int k = 0; k < 4; k++) {
    f.registerExemplar(new CutoffGpuForce(true, false, fulls[k], 0, true));
    f.registerExemplar(new CutoffGpuForce(false, true, fulls[k], 0, true));
  }
  // NonbondedSimpleFull with switching functions
  const SwitchSpec sf_coul[] = {kC1, kC2, kCompC1, kCompC2, kCompCn};
  for (int k = 0; k < 5; k++) f.registerExemplar(new SimpleFullSwGpuForce(false, true, sf_coul[k], 0));
  const SwitchSpec sf_lj[] = {kC2, kCn, kCompC1, kCompC2, kCompCn};
  for (int k = 0; k < 5; k++) f.registerExemplar(new SimpleFullSwGpuForce(true, false, sf_lj[k], 0));
  const SwitchSpec sf_pairs[][2] = {{kCompC2, kCompC1}, {kCompCn, kCompC1}, {kC2, kC1},
                                    {kC2, kC2}, {kCn, kCn}};
  for (int k = 0; k < 5; k++)
    f.registerExemplar(new SimpleFullSwGpuForce(true, true, sf_pairs[k][0], &sf_pairs[k][1]));
  f.registerExemplar(new PmeGpuForce());
  f.registerExemplar(new SimpleFullGpuForce(true, false));
  f.registerExemplar(new SimpleFullGpuForce(false, true));
  f.registerExemplar(new SimpleFullGpuForce(true, true));
  f.registerExemplar(new GbGpuForce("GBBornRadii"));
  f.registerExemplar(new GbGpuForce("GBPartialSum"));
  f.registerExemplar(new GbGpuForce("GBForce"));
  f.registerExemplar(new GbGpuForce("GBACEForce"));
  f.registerExemplar(new TorsionGpuForce(true));
  f.registerExemplar(new TorsionGpuForce(false));
  // SCPISM (module/NonbondedCutoffForceModule.cpp:91-160,
  // NonbondedSimpleFullForceModule.cpp:104-116)
  const SwitchSpec scp[] = {kC1, kC2, kCn, kCmpCnCn};
  for (int k = 0; k < 4; k++) {
    f.registerExemplar(new ScpismGpuForce(false, 0, scp[k]));
    f.registerExemplar(new ScpismGpuForce(true, 0, scp[k]));
  }
  const SwitchSpec scp_pairs[][2] = {{kC2, kC1}, {kC2, kC2}, {kCn, kCn}, {kCmpCnCn, kC1},
                                     {kCn, kC2}};
  for (int k = 0; k < 5; k++) {
    f.registerExemplar(new ScpismGpuForce(false, &scp_pairs[k][0], scp_pairs[k][1]));
    f.registerExemplar(new ScpismGpuForce(true, &scp_pairs[k][0], scp_pairs[k][1]));
  }
  f.registerExemplar(new BornGpuForce(false));
  f.registerExemplar(new BornGpuForce(true));
}

void PmgpuForceModule::init(ProtoMolApp *app) {
  app->integratorFactory.registerExemplar(
      new DeviceIntegrator(PMGPU_INT_LEAPFROG, 1.0, 0, 0, 0, 0));
  app->integratorFactory.registerExemplar(
      new DeviceIntegrator(PMGPU_INT_LANGEVIN_LEAPFROG, 1.0, 300.0, 5.0, 1234, 0));
}
