/* FP64 CPU restatement of ProtoMol's nonbonded hot path.  TEST
 * INFRASTRUCTURE ONLY: this is the checker that the CUDA library is compared
 * against, never a code path of the product.  Every function cites the
 * reference file:line it restates (paths relative to the ProtoMol tree).
 *
 * Parity pins: tests/test_oracle_pins.py checks these functions against the
 * ProtoMol reference itself (forces/energies dumped by oracle/_ref/pm_forcedump
 * and committed under tests/golden/) and against the reference's own golden
 * test outputs.
 */
#ifndef PMORACLE_H
#define PMORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

/* Exclusion classes, topology/ExclusionTable.h:19-23. */
enum { ORC_EXCL_NONE = 0, ORC_EXCL_MODIFIED = 1, ORC_EXCL_FULL = 2 };

/* Switching functions (the switch/ directory). */
enum { ORC_SW_UNIVERSAL = 0, ORC_SW_CUTOFF = 1, ORC_SW_C1 = 2, ORC_SW_C2 = 3,
       ORC_SW_CN = 4, ORC_SW_CMPCNCN = 5 };
/* Flag OR'd into a C1, C2 or Cn kind: ComplementSwitchingFunction of it
 * (switch/ComplementSwitchingFunction.h:14-74). */
enum { ORC_SW_COMPLEMENT = 16 };
/* Potentials (CoulombSCPISM: force/coulomb/CoulombSCPISMForce.h). */
enum { ORC_POT_COULOMB = 0, ORC_POT_LJ = 1, ORC_POT_SCPISM = 2 };

/* SCPISM per-atom data as ProtoMol's topology builder forms it
 * (topology/BuildTopology.cpp:757-818): the atom's type's alpha, C_i, g_i
 * and H-bond class (0 none, 1 polar H, 2 acceptor; topology/AtomType.h:10),
 * the atom's sqrt(alpha), zeta and eta, its residue number, whether its
 * name is HN (1) or O (2), and whether its molecule is water. */
typedef struct {
  const double *sqrtalpha, *alpha, *zeta, *eta, *c, *g;
  const int *hbond, *residue, *name, *water;
} orc_scpism;

typedef struct {
  int kind;
  double cutoff;    /* -cutoff */
  double switchon;  /* -switchon (C2, Cn) */
  double switchoff; /* -switchoff (Cn: 0 = use cutoff; CmpCnCn: the middle
                       distance, switchon < switchoff < cutoff) */
  double order;     /* -n (Cn) */
} orc_switch;

typedef struct {
  int n;
  const double *pos;      /* 3n, AoS like Vector3DBlock */
  const double *charge;   /* n, scaled charge (q * 18.2226123264) */
  const int *type;        /* n */
  const int *molecule;    /* n */
  int ntypes;
  const double *lj;       /* 4*ntypes*ntypes: A, B, A14, B14 */
  int nexcl;
  const int *excl;        /* 3*nexcl: a1, a2, class as ExclusionTable::check
                             returns it (the last add() of the pair) */
  const int *excl_table_class; /* nexcl or NULL: class as getTable() keeps it
                             (the first add()); used by the Ewald correction */
  double coulomb_scaling; /* coulombScalingFactor */
  int periodic;
  double box[12];         /* e1, e2, e3, origin (orthogonal boxes only) */
} orc_system;

/* ProtoMol cell assignment (topology/Topology.h:44-86,
 * topology/CubicCellManager.cpp:40-65, topology/ArrayCellListStructure.cpp:22-48).
 * Writes the integer cell (x,y,z) of every atom and the cell-array dims. */
int orc_cell_assign(const orc_system *s, double cellsize, int *cell_xyz,
                    int *dims);

/* The unordered atom pairs the NonbondedCutoff driver hands to
 * doOneAtomPair and that survive the rough cutoff test and the FULL
 * exclusion (force/nonbonded/NonbondedCutoffForce.h:37-54,
 * force/OneAtomPairTwo.h:30-55), in the reference's enumeration order.
 * pairs_out gets (i, j, class) triples; returns the count (may exceed cap,
 * in which case only cap triples are written). */
long orc_cutoff_pairs(const orc_system *s, double cellsize, double alg_cutoff,
                      double pair_cutoff, int *pairs_out, long cap);

/* NonbondedCutoffSystemForce with OneAtomPair (nterms = 1) or
 * OneAtomPairTwo (nterms = 2) of Coulomb / LennardJones.  Adds into
 * forces (3n).  energies[0] += Coulomb, energies[1] += LennardJones;
 * virial (9, row major) += atomic virial. */
int orc_cutoff_force(const orc_system *s, double cellsize, double alg_cutoff,
                     int nterms, const int *potentials, const orc_switch *sw,
                     double *forces, double *energies, double *virial);

/* NonbondedSimpleFullSystemForce, vacuum, OneAtomPair with the given
 * switch (force/nonbonded/NonbondedSimpleFullSystemForce.h:125-150). */
int orc_simplefull_force(const orc_system *s, int potential,
                         const orc_switch *sw, double *forces,
                         double *energies, double *virial);

/* NonbondedSimpleFullSystemForce with OneAtomPair (nterms = 1) or
 * OneAtomPairTwo (nterms = 2), vacuum or periodic (minimal image). */
int orc_simplefull_force_n(const orc_system *s, int nterms, const int *potentials,
                           const orc_switch *sw, double *forces, double *energies,
                           double *virial);

/* LennardJones and/or CoulombSCPISM (-D dielectric) over every pair within
 * the larger switch cutoff, OneAtomPair / OneAtomPairTwo
 * (force/coulomb/CoulombSCPISMForce.h), vacuum or the periodic minimal
 * image: the pair set of NonbondedCutoff and of NonbondedSimpleFull with a
 * cutoff switch alike. */
int orc_scpism_pair_force(const orc_system *s, const orc_scpism *p, double D, int nterms,
                          const int *potentials, const orc_switch *sw, double *forces,
                          double *energies, double *virial);

/* BornRadii then BornSelf (force/born/BornRadii.h, force/born/
 * BornSelfForce.h) over the pairs within each force's cutoff switch
 * (OneAtomPair with the Cutoff switch): the Born radii (written to
 * born_out if not NULL), the BornSelf pair forces and the self energies of
 * the atoms that took part in a pair (energies[0], COULOMB). */
int orc_born_force(const orc_system *s, const orc_scpism *p, int radii_bornswitch,
                   double radii_cutoff, int self_bornswitch, double self_cutoff, double D,
                   double *born_out, double *forces, double *energies, double *virial);

/* NonbondedFullSystemForce (lattice sum, force/nonbonded/
 * NonbondedFullSystemForce.h:38-62) with OneAtomPairFull
 * (force/OneAtomPairFull.h:35-135): every pair i <= j in blocks of 64, the
 * minimal image with the pair's exclusion class and every lattice image
 * (|L| <= 2 alg_cutoff) with none; an atom's own images add half their
 * energy and no force.  Periodic boxes only. */
int orc_full_force(const orc_system *s, int potential, const orc_switch *sw,
                   double alg_cutoff, double *forces, double *energies, double *virial);

/* NonbondedFullEwaldSystemForce parameters, derived exactly as in
 * force/nonbonded/NonbondedFullEwaldSystemForce.h:598-620. */
typedef struct {
  double alpha, accuracy, rc, kc;
  int exact_erf; /* 0: A&S poly5 (default build); 1: USE_EWALD_EXACT_ERF */
} orc_ewald;
void orc_ewald_setup(const orc_system *s, double alpha, double accuracy,
                     int exact_erf, orc_ewald *out);

/* Terms of NonbondedFullEwaldSystemForce::evaluate (:324-398).  Each adds
 * into forces and writes its own energy (and adds virial). */
int orc_ewald_real(const orc_system *s, const orc_ewald *e, double cellsize,
                   double *forces, double *energy, double *virial);
int orc_ewald_reciprocal(const orc_system *s, const orc_ewald *e,
                         double *forces, double *energy, double *virial);
int orc_ewald_correction(const orc_system *s, const orc_ewald *e,
                         double *forces, double *energy, double *virial);
/* Point self energy and charged-system energy (:694-714). */
void orc_ewald_self(const orc_system *s, const orc_ewald *e, double *self,
                    double *charged);

/* Smooth PME reciprocal term (Essmann et al., J. Chem. Phys. 103, 8577
 * (1995)), FP64, with a direct (non-FFT) evaluation of the structure factor
 * on the mesh: used to pin the FFT-based restatements at small sizes. */

/* GB (OBC) in the vacuum all-pairs driver: GBBornRadii
 * (force/GB/GBBornRadii.cpp:15-173), GBPartialSum
 * (force/GB/GBPartialSum.cpp:11-57), GBForce (force/GB/GBForce.cpp:14-242).
 * water[i] != 0 marks atoms of water molecules (skipped by GBBornRadii).
 * Outputs: born (n), forces (3n, added), energy (GB pair + self). */
typedef struct {
  const double *vdwr;    /* n, vanDerWaalRadius */
  const double *scale;   /* n, scalingFactor S */
  const double *offset;  /* n, offsetRadius (0.09) */
  const int *water;      /* n */
  double alpha_obc, beta_obc, gamma_obc;
  double solute_dielec, solvent_dielec;
} orc_gb;
/* GBACEForce (ACE nonpolar term on the GBBornRadii radii): forces ADDED,
 * energy set. */
int orc_gbace_force(const orc_system *s, const orc_gb *g, double sigma, double rho_s,
                    double *forces, double *energy);
int orc_gb_force(const orc_system *s, const orc_gb *g, double *born,
                 double *forces, double *energy);

/* Integrator updates (FP64), h = timestep[fs] * INV_TIMEFACTOR.
 * Leapfrog (integrator/leapfrog/LeapfrogIntegrator.cpp:33-104):
 *   first step: v += F*h/2/m; x += v*h; F = f(x); then per step
 *   v += F*h/m; x += v*h; F = f(x); last: v += F*h/2/m.
 * These expose the single operations; the drivers live in Python. */
/* Torsions (MTorsionSystemForce::calcTorsion, force/bonded/
 * MTorsionSystemForce.h:40-204): nt terms, atoms 4 per term, params 3 per
 * term (k, periodicity n, phase delta [rad]); n > 0 is the cosine form
 * k (1 + cos(n phi + delta)), n == 0 the harmonic k (phi - delta)^2.
 * Forces are added; energy and virial (may be NULL) are set. */
/* Harmonic bonds (2 atoms; k, r0) and angles with Urey-Bradley (3 atoms;
 * k_theta, theta0 [rad], k_ub, r_ub): forces ADDED, energy and virial set. */
int orc_bond_force(const orc_system *s, int nb, const int *atoms, const double *params,
                   double *forces, double *energy, double *virial);
int orc_angle_force(const orc_system *s, int na, const int *atoms, const double *params,
                    double *forces, double *energy, double *virial);
int orc_torsion_force(const orc_system *s, int nt, const int *atoms,
                      const double *params, double *forces, double *energy,
                      double *virial);

void orc_kick(int n, const double *mass, const double *forces, double h,
              double *vel);
void orc_drift(int n, const double *vel, double h, double *pos);
/* LangevinLeapfrog half kick with a caller-supplied Gaussian stream
 * (integrator/base/LangevinLeapfrogIntegrator.cpp:44-71); gauss holds 3n
 * numbers per atom in (x, y, z) order. */
void orc_langevin_half_kick(int n, const double *mass, const double *forces,
                            double timestep_fs, double gamma_ps,
                            double temperature, const double *gauss,
                            double *vel);

#ifdef __cplusplus
}
#endif
#endif
