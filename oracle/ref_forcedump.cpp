// Test-infrastructure driver linked against the unmodified ProtoMol library
// (oracle/_ref/libProtoMol.a).  It loads a .conf exactly as the ProtoMol
// executable does (protomol/main.cpp:13-34: ModuleManager, configure,
// build), then evaluates a caller-supplied sequence of force definitions
// through ProtoMol's own ForceFactory (factory/ForceFactory.cpp:21-242) and
// SystemForce::preProcess/evaluate/postProcess (the order used by
// ForceGroup::evaluateSystemForces, force/ForceGroup.cpp:54-72).  For every
// force it writes the FP64 forces, the ScalarStructure energies and the
// atomic virial.  It also writes the built topology (charges, masses, types,
// molecules, LJ table, exclusion table, boundary box, GB atom parameters) so
// that the oracle restatement and the CUDA path can be fed the identical
// system.  Nothing here is part of the product.
//
//   pm_forcedump <conf> <out.txt> [--steps N] "<force def>" ["<force def>" ...]
//
// With --steps N the conf's own integrator is first advanced N steps
// (ProtoMolApp::step) and the dump is taken at the resulting positions.
#include <protomol/ProtoMolApp.h>
#include <protomol/base/ModuleManager.h>
#include <protomol/base/Exception.h>
#include <protomol/force/system/SystemForce.h>
#include <protomol/topology/GenericTopology.h>
#include <protomol/topology/SemiGenericTopology.h>
#include <protomol/topology/PeriodicBoundaryConditions.h>
#include <protomol/topology/VacuumBoundaryConditions.h>
#include <protomol/type/ScalarStructure.h>
#include <protomol/type/Vector3DBlock.h>
#include <protomol/config/Value.h>
#include <protomol/config/ValueType.h>
#include <sstream>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

using namespace std;
using namespace ProtoMol;

extern void moduleInitFunction(ModuleManager *);

static void putv(FILE *f, const char *key, const vector<double> &v) {
  fprintf(f, "%s %lu", key, (unsigned long)v.size());
  for (size_t i = 0; i < v.size(); i++) fprintf(f, " %.17g", v[i]);
  fprintf(f, "\n");
}
static void puti(FILE *f, const char *key, const vector<long> &v) {
  fprintf(f, "%s %lu", key, (unsigned long)v.size());
  for (size_t i = 0; i < v.size(); i++) fprintf(f, " %ld", v[i]);
  fprintf(f, "\n");
}

int main(int argc, char *argv[]) {
  if (argc < 3) {
    fprintf(stderr, "usage: %s conf out.txt [--steps N] force...\n", argv[0]);
    return 2;
  }
  try {
    string conf = argv[1];
    string out = argv[2];
    int a = 3;
    long steps = 0;
    if (a + 1 < argc && strcmp(argv[a], "--steps") == 0) {
      steps = atol(argv[a + 1]);
      a += 2;
    }
    vector<string> defs;
    for (; a < argc; a++) defs.push_back(argv[a]);

    ModuleManager modManager;
    moduleInitFunction(&modManager);
    ProtoMolApp app(&modManager);
    vector<string> args;
    args.push_back("pm_forcedump");
    args.push_back(conf);
    if (!app.configure(args)) return 3;
    app.build();
    if (steps > 0) app.step(steps);
    // ProtoMolApp::build drops the force exemplars once the integrator is
    // made (ProtoMolApp.cpp:462); register them again for our own makes.
    modManager.registerForces(&app);

    GenericTopology *topo = app.topology;
    const unsigned n = topo->atoms.size();
    FILE *f = fopen(out.c_str(), "w");
    if (!f) { perror("open"); return 4; }

    fprintf(f, "natoms 1 %u\n", n);
    vector<double> q(n), m(n), vdw(n), sf(n), off(n);
    vector<long> type(n), mol(n), water(n);
    for (unsigned i = 0; i < n; i++) {
      const Atom &at = topo->atoms[i];
      q[i] = at.scaledCharge;
      m[i] = at.scaledMass;
      type[i] = at.type;
      mol[i] = at.molecule;
      water[i] = topo->molecules[at.molecule].water ? 1 : 0;
      if (at.myGBSA_T) {
        vdw[i] = at.myGBSA_T->vanDerWaalRadius;
        sf[i] = at.myGBSA_T->scalingFactor;
        off[i] = at.myGBSA_T->offsetRadius;
      }
    }
    putv(f, "charge", q);
    putv(f, "mass", m);
    puti(f, "type", type);
    puti(f, "molecule", mol);
    puti(f, "water", water);
    if (topo->doGBSAOpenMM) {
      putv(f, "gb_vdwr", vdw);
      putv(f, "gb_scale", sf);
      putv(f, "gb_offset", off);
      vector<double> obc(3);
      obc[0] = topo->alphaObc; obc[1] = topo->betaObc; obc[2] = topo->gammaObc;
      putv(f, "gb_obc", obc);
    }
    if (topo->doSCPISM) {
      // SCPISM data as the topology builder forms it (topology/
      // BuildTopology.cpp:757-818): per atom its type's alpha, C_i, g_i and
      // H-bond class, its own sqrt(alpha), zeta and eta, its residue and
      // whether its name is HN (1) or O (2) (force/born/BornRadii.h:56-58)
      vector<double> sa(n), al(n), ze(n), et(n), ci(n), gi(n);
      vector<long> hb(n), res(n), nm(n);
      for (unsigned i = 0; i < n; i++) {
        const Atom &at = topo->atoms[i];
        const SCPISMAtomTypeParameters *t = topo->atomTypes[at.type].mySCPISM_T;
        sa[i] = at.mySCPISM_A->sqrtalphaSCPISM;
        al[i] = t->alpha;
        ze[i] = at.mySCPISM_A->zeta;
        et[i] = at.mySCPISM_A->eta;
        ci[i] = t->C_i;
        gi[i] = t->g_i;
        hb[i] = (long)t->isHbonded;
        res[i] = at.residue_seq;
        nm[i] = at.name == "HN" ? 1 : (at.name == "O" ? 2 : 0);
      }
      putv(f, "scp_sqrtalpha", sa);
      putv(f, "scp_alpha", al);
      putv(f, "scp_zeta", ze);
      putv(f, "scp_eta", et);
      putv(f, "scp_c", ci);
      putv(f, "scp_g", gi);
      puti(f, "scp_hbond", hb);
      puti(f, "scp_residue", res);
      puti(f, "scp_name", nm);
    }
    // Type names, used only by tests that re-derive GB scaling factors.
    fprintf(f, "typenames %lu", (unsigned long)topo->atomTypes.size());
    for (size_t t = 0; t < topo->atomTypes.size(); t++)
      fprintf(f, " %s", topo->atomTypes[t].name.c_str());
    fprintf(f, "\n");

    const int nt = topo->lennardJonesParameters.size();
    vector<double> lj(4 * nt * nt);
    for (int i = 0; i < nt; i++)
      for (int j = 0; j < nt; j++) {
        const LennardJonesParameters &p = topo->lennardJonesParameters(i, j);
        double *d = &lj[4 * (i * nt + j)];
        d[0] = p.A; d[1] = p.B; d[2] = p.A14; d[3] = p.B14;
      }
    fprintf(f, "ntypes 1 %d\n", nt);
    putv(f, "lj", lj);

    const vector<ExclusionPair> &ex = topo->exclusions.getTable();
    vector<long> exv(3 * ex.size());
    for (size_t k = 0; k < ex.size(); k++) {
      exv[3 * k] = ex[k].a1;
      exv[3 * k + 1] = ex[k].a2;
      exv[3 * k + 2] = (long)ex[k].excl;
    }
    puti(f, "exclusions", exv);
    // ExclusionTable::check keeps the class of the LAST add() of a pair while
    // getTable() keeps the FIRST (ExclusionTable.cpp:103-118 dedupes by atom
    // pair only); pair forces use check(), the Ewald correction the table.
    vector<long> chk(ex.size());
    for (size_t k = 0; k < ex.size(); k++)
      chk[k] = (long)topo->exclusions.check(ex[k].a1, ex[k].a2);
    puti(f, "exclusions_check", chk);
    // Harmonic bonds and angles (topology/Bond.h, topology/Angle.h).
    vector<long> bidx, aidx;
    vector<double> bprm, aprm;
    for (size_t k = 0; k < topo->bonds.size(); k++) {
      bidx.push_back(topo->bonds[k].atom1);
      bidx.push_back(topo->bonds[k].atom2);
      bprm.push_back(topo->bonds[k].springConstant);
      bprm.push_back(topo->bonds[k].restLength);
    }
    for (size_t k = 0; k < topo->angles.size(); k++) {
      aidx.push_back(topo->angles[k].atom1);
      aidx.push_back(topo->angles[k].atom2);
      aidx.push_back(topo->angles[k].atom3);
      aprm.push_back(topo->angles[k].forceConstant);
      aprm.push_back(topo->angles[k].restAngle);
      aprm.push_back(topo->angles[k].ureyBradleyConstant);
      aprm.push_back(topo->angles[k].ureyBradleyRestLength);
    }
    puti(f, "bonds", bidx);
    putv(f, "bond_params", bprm);
    puti(f, "angles", aidx);
    putv(f, "angle_params", aprm);
    // Torsions (topology/Torsion.h): one row per term (atoms, k, n, delta),
    // a torsion of multiplicity m giving m rows.
    for (int kind = 0; kind < 2; kind++) {
      const std::vector<Torsion> &ts = kind == 0 ? topo->dihedrals : topo->impropers;
      std::vector<long> tidx;
      std::vector<double> tprm;
      for (size_t k = 0; k < ts.size(); k++)
        for (int m = 0; m < ts[k].multiplicity; m++) {
          tidx.push_back(ts[k].atom1);
          tidx.push_back(ts[k].atom2);
          tidx.push_back(ts[k].atom3);
          tidx.push_back(ts[k].atom4);
          tprm.push_back(ts[k].forceConstant[m]);
          tprm.push_back((double)ts[k].periodicity[m]);
          tprm.push_back(ts[k].phaseShift[m]);
        }
      puti(f, kind == 0 ? "dihedrals" : "impropers", tidx);
      putv(f, kind == 0 ? "dihedral_params" : "improper_params", tprm);
    }
    vector<double> csf(1, topo->coulombScalingFactor);
    putv(f, "coulomb_scaling", csf);

    const SemiGenericTopology<PeriodicBoundaryConditions> *pt =
      dynamic_cast<const SemiGenericTopology<PeriodicBoundaryConditions> *>(topo);
    vector<double> box(12, 0.0);
    if (pt) {
      const PeriodicBoundaryConditions &bc = pt->boundaryConditions;
      for (int c = 0; c < 3; c++) {
        box[c] = bc.e1().c[c];
        box[3 + c] = bc.e2().c[c];
        box[6 + c] = bc.e3().c[c];
        box[9 + c] = bc.origin().c[c];
      }
    }
    fprintf(f, "periodic 1 %d\n", pt ? 1 : 0);
    putv(f, "box", box);

    vector<double> pos(3 * n), vel(3 * n);
    for (unsigned i = 0; i < n; i++)
      for (int c = 0; c < 3; c++) {
        pos[3 * i + c] = app.positions[i].c[c];
        vel[3 * i + c] = app.velocities[i].c[c];
      }
    putv(f, "positions", pos);
    putv(f, "velocities", vel);

    for (size_t d = 0; d < defs.size(); d++) {
      // Same tokenisation the integrator factory applies to a conf's
      // force lines (factory/IntegratorFactory.cpp:120-124).
      stringstream ssf("force " + defs[d]);
      Value fv(ValueType::Force(""));
      ssf >> fv;
      Force *force = app.forceFactory.make(fv.getString());
      SystemForce *sys = dynamic_cast<SystemForce *>(force);
      if (!sys) {
        fprintf(stderr, "not a SystemForce: %s\n", defs[d].c_str());
        return 5;
      }
      Vector3DBlock forces;
      forces.resize(n);
      forces.zero();
      ScalarStructure energies;
      energies.virial(true);
      energies.clear();
      topo->uncacheCellList();
      sys->preProcess(topo, &app.positions);
      sys->evaluate(topo, &app.positions, &forces, &energies);
      sys->postProcess(topo, &energies, &forces);

      fprintf(f, "force 1 %lu\n", (unsigned long)d);
      fprintf(f, "forcedef 1 %s\n", defs[d].c_str());
      // The prototype the factory resolved the line to, with its values.
      {
        vector<Parameter> prm;
        force->getParameters(prm);
        string id = force->getIdNoAlias();
        for (size_t k = 0; k < prm.size(); k++)
          id += " " + prm[k].keyword + "=" + prm[k].value.getString();
        fprintf(f, "forceid 1 %s\n", id.c_str());
      }
      vector<double> fo(3 * n);
      for (unsigned i = 0; i < n; i++)
        for (int c = 0; c < 3; c++) fo[3 * i + c] = forces[i].c[c];
      putv(f, "forces", fo);
      vector<double> en(ScalarStructure::LAST);
      for (int k = 0; k < (int)ScalarStructure::LAST; k++)
        en[k] = energies[(ScalarStructure::Index)k];
      putv(f, "energies", en);
      // Not deleted: GB forces share per-atom state through the topology
      // and the process exits right after.
    }
    fclose(f);
    return 0;
  } catch (const Exception &e) {
    cerr << "ERROR: " << e << endl;
  }
  return 1;
}
