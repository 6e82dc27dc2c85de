/*
 * pmgpu -- B200 (sm_100a) implementation of ProtoMol's nonbonded hot path
 * behind a plain C ABI: cutoff Lennard-Jones + Coulomb over a device-built
 * cell list with ProtoMol's switching functions, Ewald real space + PME
 * reciprocal space + exclusion/self corrections, OBC generalized Born, the
 * harmonic bonds/angles needed to integrate flexible water, and
 * device-resident leapfrog / Langevin-leapfrog integration.
 *
 * Every entry point returns a status code (PMGPU_OK == 0); the message of
 * the last failure on the calling thread is available from
 * pmgpu_last_error().  No entry point takes or returns a torch or CUDA
 * runtime type: host arrays are plain pointers with explicit sizes, in
 * ProtoMol's own layouts (Vector3DBlock = double[3N] x,y,z per atom;
 * ScalarStructure energies indexed as in type/ScalarStructure.h:26-67).
 *
 * Reference interfaces each entry point replaces (paths inside ProtoMol):
 *   SystemForce::evaluate(topo, positions, forces, energies)
 *       force/system/SystemForce.h:32-35           -> pmgpu_force_evaluate
 *   ForceFactory::make(<force line>) for NonbondedCutoff / FullEwald /
 *       NonbondedSimpleFull GB* forces
 *       factory/ForceFactory.cpp:21-242            -> pmgpu_force_*_add
 *   Integrator::run(n) of Leapfrog / LangevinLeapfrog
 *       integrator/leapfrog/LeapfrogIntegrator.cpp:89-104,
 *       integrator/StandardIntegrator.cpp:27-37    -> pmgpu_run
 *   GenericTopology (atoms, LJ table, exclusions, boundary conditions)
 *       topology/GenericTopology.h:120-165         -> pmgpu_topology
 */
#ifndef PMGPU_H
#define PMGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PMGPU_ABI_VERSION 2

/* ---- status codes ------------------------------------------------- */
enum {
  PMGPU_OK = 0,
  PMGPU_ERR_ARG = 1,          /* invalid argument / configuration */
  PMGPU_ERR_CUDA = 2,         /* CUDA runtime or cuFFT failure */
  PMGPU_ERR_OOM = 3,          /* device allocation failed */
  PMGPU_ERR_OVERFLOW = 4,     /* a device capacity (cell, list) overflowed */
  PMGPU_ERR_NAN = 5,          /* non-finite force or energy detected */
  PMGPU_ERR_UNSUPPORTED = 6,  /* configuration outside what is built */
  PMGPU_ERR_STATE = 7         /* call made in the wrong state */
};

/* ---- ProtoMol enumerations ---------------------------------------- */
/* ExclusionClass, topology/ExclusionTable.h:19-23 */
enum { PMGPU_EXCL_NONE = 0, PMGPU_EXCL_MODIFIED = 1, PMGPU_EXCL_FULL = 2 };

/* Switching functions, switch/{Universal,Cutoff,C1,C2,Cn,CmpCnCn}
 * SwitchingFunction.  PMGPU_SW_COMPLEMENT OR'd into C1, C2 or Cn is the
 * ComplementSwitchingFunction of that function
 * (switch/ComplementSwitchingFunction.h:14-74: 1 - S, no cutoff), which
 * ProtoMol registers on the all-pairs path only. */
enum {
  PMGPU_SW_UNIVERSAL = 0,
  PMGPU_SW_CUTOFF = 1,
  PMGPU_SW_C1 = 2,
  PMGPU_SW_C2 = 3,
  PMGPU_SW_CN = 4,
  PMGPU_SW_CMPCNCN = 5,
  PMGPU_SW_COMPLEMENT = 16
};

/* Energy slots written by pmgpu_evaluate / pmgpu_force_evaluate: the first
 * PMGPU_E_COUNT entries of ProtoMol's ScalarStructure (COULOMB,
 * LENNARDJONES, BOND, ANGLE, DIHEDRAL, IMPROPER, OTHER). */
enum {
  PMGPU_E_COULOMB = 0,
  PMGPU_E_LENNARDJONES = 1,
  PMGPU_E_BOND = 2,
  PMGPU_E_ANGLE = 3,
  PMGPU_E_DIHEDRAL = 4,
  PMGPU_E_IMPROPER = 5,
  PMGPU_E_OTHER = 6,
  PMGPU_E_COUNT = 7
};

/* Arithmetic of the pair kernels. */
enum { PMGPU_PREC_MIXED = 0, /* FP32 pair math, FP64 accumulation/updates */
       PMGPU_PREC_DOUBLE = 1 /* FP64 throughout */ };

/* ---- topology ------------------------------------------------------ */
typedef struct {
  int n_atoms;
  const double *charge;     /* n: Atom::scaledCharge (q * 18.2226123264) */
  const double *mass;       /* n: Atom::scaledMass */
  const int *type;          /* n: Atom::type */
  const int *molecule;      /* n: Atom::molecule */
  int n_types;
  const double *lj;         /* n_types^2 * 4: A, B, A14, B14 per type pair
                               (LennardJonesParameterTable) */
  int n_exclusions;
  const int *exclusions;    /* 3 per entry of ExclusionTable::getTable():
                               a1, a2, and the class ExclusionTable::check
                               returns for the pair (used by pair forces) */
  const int *exclusion_table_class; /* n_exclusions or NULL: the class the
                               table entry itself holds, used by the Ewald
                               correction term (NULL: same as above).  The
                               two differ when a pair was added twice with
                               different classes (ExclusionTable.cpp:103-118) */
  double coulomb_scaling;   /* GenericTopology::coulombScalingFactor */
  int periodic;             /* 1: PeriodicBoundaryConditions, 0: vacuum */
  double box[12];           /* e1, e2, e3, origin (orthogonal boxes) */
  /* Harmonic bonds (force/bonded/BondSystemForce.h): i, j and (k, r0). */
  int n_bonds;
  const int *bond_atoms;    /* 2 per bond */
  const double *bond_params;/* 2 per bond: k [kcal/mol/A^2], r0 [A] */
  /* Harmonic angles (force/bonded/AngleSystemForce.h): i, j(center), k
   * and (k_theta, theta0 [rad], k_ub, r_ub). */
  int n_angles;
  const int *angle_atoms;   /* 3 per angle */
  const double *angle_params;/* 4 per angle */
  /* OBC GB atom parameters (GBSAAtomParameters, topology/Atom.h:35-157);
   * may be NULL when no GB force is added. */
  const double *gb_vdwr;    /* vanDerWaalRadius */
  const double *gb_scale;   /* scalingFactor */
  const double *gb_offset;  /* offsetRadius */
  const int *water;         /* 1 if the atom's molecule is a water */
  double gb_obc[3];         /* alphaObc, betaObc, gammaObc */
  /* Torsions (topology/Torsion.h; MTorsionSystemForce): 4 atoms and
   * (k [kcal/mol], periodicity n, phase [rad]) per term, a torsion of
   * multiplicity m given as m terms.  n > 0: k (1 + cos(n phi + phase));
   * n == 0: k (phi - phase)^2.  NULL arrays: none. */
  int n_dihedrals;
  const int *dihedral_atoms;
  const double *dihedral_params;
  int n_impropers;
  const int *improper_atoms;
  const double *improper_params;
  /* SCPISM implicit-solvent data as ProtoMol's topology builder forms it
   * (topology/BuildTopology.cpp:757-818, topology/Atom.h:10-29,
   * topology/AtomType.h:10-21), n each: the atom's sqrt(alpha), its type's
   * alpha, the atom's zeta and eta, its type's C_i and g_i, its type's
   * H-bond class (0 none, 1 polar hydrogen, 2 acceptor), its residue
   * number, and its name class (1 "HN", 2 "O", 0 other; BornRadii.h:56).
   * NULL scpism_alpha: no SCPISM parameters (the SCPISM forces are then
   * refused).  The water flags above mark atoms the SCPISM pair terms skip. */
  const double *scpism_sqrtalpha, *scpism_alpha, *scpism_zeta, *scpism_eta;
  const double *scpism_c, *scpism_g;
  const int *scpism_hbond, *scpism_residue, *scpism_name;
} pmgpu_topology;

typedef struct {
  int kind;         /* PMGPU_SW_* */
  double cutoff;    /* -cutoff */
  double switchon;  /* -switchon (C2, Cn) */
  double switchoff; /* -switchoff (Cn: 0 means "use cutoff"; CmpCnCn: the
                       middle distance, switchon < switchoff <= cutoff) */
  double order;     /* -n (Cn, CmpCnCn) */
} pmgpu_switch;

typedef struct pmgpu_context pmgpu_context;
typedef struct pmgpu_system pmgpu_system;

/* ---- context ------------------------------------------------------- */
int pmgpu_context_create(int device, pmgpu_context **out);
int pmgpu_context_destroy(pmgpu_context *ctx);
/* Message of the last failing call on this thread ("" if none). */
const char *pmgpu_last_error(void);
int pmgpu_abi_version(void);

/* ---- systems ------------------------------------------------------- */
/* Copies the topology to the device; positions/velocities start at zero. */
int pmgpu_system_create(pmgpu_context *ctx, const pmgpu_topology *topo,
                        int precision, pmgpu_system **out);
int pmgpu_system_destroy(pmgpu_system *sys);
/* Host <-> device copies of Vector3DBlock-layout arrays (3n doubles).
 * Positions with a non-finite coordinate are refused with PMGPU_ERR_NAN.
 * New positions are a new configuration: the next evaluation builds every
 * pair list afresh, as for a new system. */
int pmgpu_system_set_positions(pmgpu_system *sys, const double *pos);
int pmgpu_system_get_positions(pmgpu_system *sys, double *pos);
int pmgpu_system_set_velocities(pmgpu_system *sys, const double *vel);
int pmgpu_system_get_velocities(pmgpu_system *sys, double *vel);
/* The step counter that keys the Langevin noise (ProtoMol's current step;
 * a new system starts at 0, every MD step adds one).  With positions,
 * velocities and this counter set, a system continues exactly as a new
 * system made from that state would. */
int pmgpu_system_set_step(pmgpu_system *sys, long long step);
/* Total force of the last evaluation (all enabled terms), 3n doubles. */
int pmgpu_system_get_forces(pmgpu_system *sys, double *forces);
/* Energies (PMGPU_E_COUNT) and atomic virial (9, may be NULL) of the last
 * evaluation. */
int pmgpu_system_get_energies(pmgpu_system *sys, double *energies,
                              double *virial);
/* The CUDA stream (a cudaStream_t) that orders all of this system's work:
 * each evaluation forks its concurrent terms from it onto two internal
 * streams and joins them back before it ends, so work a caller enqueues on
 * this stream after a call sees that call's results. */
void *pmgpu_system_stream(pmgpu_system *sys);
/* Device pointers of the resident state: positions and velocities as
 * double[3n] (Vector3DBlock layout), forces as int64 fixed point
 * [3][n] (x plane, y plane, z plane) with PMGPU_FORCE_SCALE units. */
int pmgpu_system_device_state(pmgpu_system *sys, double **pos, double **vel,
                              long long **force_fixed);
#define PMGPU_FORCE_SCALE 4294967296.0 /* 2^32 per kcal/mol/A */

/* ---- forces (one per ProtoMol `force` line) ------------------------- */
/* NonbondedCutoff with LennardJones and/or Coulomb
 * (module/NonbondedCutoffForceModule.cpp:40-201).  lj_sw / coul_sw may be
 * NULL for an absent term.  cellsize is the topology's cellsize keyword;
 * alg_cutoff is the algorithm's -cutoff. */
int pmgpu_force_cutoff_add(pmgpu_system *sys, const pmgpu_switch *lj_sw,
                           const pmgpu_switch *coul_sw, double alg_cutoff,
                           double cellsize, int *force_id);
/* NonbondedFull (lattice sum) LennardJones and/or Coulomb
 * (force/nonbonded/NonbondedFullSystemForce.h:38-62 with
 * force/OneAtomPairFull.h:35-135; module/NonbondedFullForceModule.cpp:39-46):
 * every periodic image of every pair within the switch cutoff, the
 * minimal image with the pair's exclusion class and the others with none.
 * Switches C1, C2, Cn or CmpCnCn; alg_cutoff (the algorithm's -cutoff,
 * which bounds the lattice) at least the switch cutoffs; periodic boxes
 * with edges longer than the cutoff (PMGPU_ERR_UNSUPPORTED otherwise: an
 * atom's own images then lie within the cutoff). */
int pmgpu_force_full_add(pmgpu_system *sys, const pmgpu_switch *lj_sw,
                         const pmgpu_switch *coul_sw, double alg_cutoff, double cellsize,
                         int *force_id);
/* NonbondedSimpleFull with switching functions: LennardJones and/or
 * Coulomb over every pair i < j (OneAtomPair / OneAtomPairTwo,
 * module/NonbondedSimpleFullForceModule.cpp:55-199), vacuum or the
 * minimal image of a periodic box, switches Universal, C1, C2, Cn or the
 * Complement of C1, C2, Cn.  NULL switch: the term is absent.  The pair
 * arithmetic is FP64 in both precisions. */
int pmgpu_force_simplefull_switched_add(pmgpu_system *sys, const pmgpu_switch *lj_sw,
                                        const pmgpu_switch *coul_sw, int *force_id);
/* LennardJones and/or CoulombSCPISM (force/coulomb/CoulombSCPISMForce.h,
 * -D the bulk dielectric) on NonbondedCutoff or NonbondedSimpleFull
 * (module/NonbondedCutoffForceModule.cpp:91-107, 145-160;
 * module/NonbondedSimpleFullForceModule.cpp:104-116): every pair within the
 * larger switch cutoff, vacuum or the periodic minimal image, which is the
 * pair set of both algorithms; FP64 pair arithmetic.  coul_sw is the
 * CoulombSCPISM term's switch (required), lj_sw NULL for no LJ term. */
int pmgpu_force_scpism_add(pmgpu_system *sys, const pmgpu_switch *lj_sw,
                           const pmgpu_switch *coul_sw, double dielectric, int *force_id);
/* BornRadii followed by BornSelf (force/born/BornRadii.h:33-77,
 * force/born/BornSelfForce.h:31-118, module/NonbondedCutoffForceModule.cpp:
 * 145-148): the SCPISM Born radii over the pairs within radii_cutoff (Born
 * switch radii_bornswitch), then the BornSelf pair forces over the pairs
 * within self_cutoff and the self energy of every atom in such a pair
 * (COULOMB).  FP64. */
int pmgpu_force_born_add(pmgpu_system *sys, int radii_bornswitch, double radii_cutoff,
                         int self_bornswitch, double self_cutoff, double dielectric,
                         int *force_id);
/* NonbondedSimpleFull LennardJones and/or Coulomb (vacuum all pairs with
 * exclusions, module/NonbondedSimpleFullForceModule.cpp). */
int pmgpu_force_simplefull_add(pmgpu_system *sys, int lj, int coulomb,
                               int *force_id);
/* Ewald Coulomb delivered as PME: real space (erfc-screened, cutoff rc),
 * reciprocal space (smooth PME, B-spline order, grid), exclusion
 * correction and self/charged-system terms, selected by flags.  The real
 * term follows NonbondedFullEwaldSystemForce::realTerm (:753-858) with the
 * A&S erfc (exact_erf = 0) or the C library erfc (exact_erf = 1). */
enum { PMGPU_EWALD_REAL = 1, PMGPU_EWALD_RECIPROCAL = 2,
       PMGPU_EWALD_CORRECTION = 4, PMGPU_EWALD_ALL = 7 };
int pmgpu_force_pme_add(pmgpu_system *sys, double alpha, double rc,
                        int order, const int grid[3], int flags,
                        int exact_erf, double cellsize, int *force_id);
/* GBBornRadii + GBPartialSum + GBForce (OBC, vacuum, all pairs),
 * force/GB/GB{BornRadii,PartialSum,Force}.cpp. */
int pmgpu_force_gb_add(pmgpu_system *sys, double solute_dielec,
                       double solvent_dielec, int *force_id);
/* GBACEForce (force/GB/GBACEForce.cpp:17-209): the ACE nonpolar solvation
 * term on the OBC Born radii, vacuum, all pairs; its energy goes to
 * PMGPU_E_COULOMB as in the reference.  solvation_param is -solvationparam
 * [kcal/mol/A^2] (reference default 2.26 / 418.4), water_sphere_radius is
 * -watersphereradius [A] (default 1.4).  Evaluated with a GB force, both
 * share one Born-radius computation. */
int pmgpu_force_gbace_add(pmgpu_system *sys, double solvation_param,
                          double water_sphere_radius, int *force_id);
/* GB forces (the same three passes as pmgpu_force_gb_add) for callers that
 * must not allocate device memory: a host that has given all of HBM to its
 * own pool, a plugin that may only use the buffers it is handed, or a loop
 * that cannot take the device-wide synchronisation cudaMalloc/cudaFree
 * imply.  This entry point has no counterpart in the reference.
 *
 * Every array is device memory on the current device, owned by the caller:
 * pos (3n, Vector3DBlock layout), charge, gb_vdwr, gb_scale, gb_offset (n
 * each), water (n, or NULL), forces (3n, OVERWRITTEN, kcal/mol/A) and
 * energy (1 double, overwritten with the GB energy).  obc is a host array
 * {alpha, beta, gamma}.  stream is a cudaStream_t (NULL: default stream);
 * the call only enqueues work on it.
 *
 * Scratch lives in one statically sized device array inside the library,
 * so n_atoms above PMGPU_GB_STATIC_MAX_ATOMS is rejected with
 * PMGPU_ERR_ARG.  Every call looks up the array's device address in the
 * current context (no allocation; a context made after cudaDeviceReset gets
 * its own array); make the first call on a device before any stream
 * capture, since it may load the library's device code.  All calls on a
 * device share the array and it keeps the
 * previous call's contents (the call clears what must start at zero): two
 * calls whose work overlaps on the GPU race and both results are wrong, so
 * issue them on one stream or otherwise serialise them. */
#define PMGPU_GB_STATIC_MAX_ATOMS 16384
int pmgpu_gb_forces_noalloc(int n_atoms, const double *pos, const double *charge,
                            const double *gb_vdwr, const double *gb_scale,
                            const double *gb_offset, const int *water,
                            const double obc[3], double solute_dielec,
                            double solvent_dielec, int precision,
                            double *forces, double *energy, void *stream);
/* Harmonic bonds and angles of the topology. */
int pmgpu_force_bonded_add(pmgpu_system *sys, int bonds, int angles,
                           int *force_id);
/* Dihedral and/or Improper torsions of the topology
 * (force/bonded/DihedralSystemForce.h, ImproperSystemForce.h); energies go
 * to PMGPU_E_DIHEDRAL / PMGPU_E_IMPROPER. */
int pmgpu_force_torsion_add(pmgpu_system *sys, int dihedrals, int impropers,
                            int *force_id);
int pmgpu_force_set_enabled(pmgpu_system *sys, int force_id, int enabled);

/* Evaluate all enabled forces at the resident positions.  energies (may be
 * NULL) gets PMGPU_E_COUNT values, virial (may be NULL) 9.  With both NULL
 * the evaluation is force-only: it runs the kernels of an inner MD step
 * (including the specialised force-only pair kernels), computes no
 * energies, and pmgpu_system_get_energies then reports zeros; the forces
 * (pmgpu_system_get_forces) are complete. */
int pmgpu_evaluate(pmgpu_system *sys, double *energies, double *virial);

/* ProtoMol SystemForce::evaluate semantics for one force term: uploads
 * positions (3n doubles), evaluates that term only, ADDS its forces into
 * forces (3n doubles) and its energies into energies (ScalarStructure
 * slots, PMGPU_E_COUNT) and, if virial != NULL, its virial (9).  With
 * energies and virial both NULL the term is evaluated force-only, as in
 * pmgpu_evaluate. */
int pmgpu_force_evaluate(pmgpu_system *sys, int force_id, const double *pos,
                         double *forces, double *energies, double *virial);

/* ---- integration ---------------------------------------------------- */
enum { PMGPU_INT_LEAPFROG = 0, PMGPU_INT_LANGEVIN_LEAPFROG = 1 };
typedef struct {
  int kind;              /* PMGPU_INT_* */
  double timestep_fs;    /* -timestep */
  double temperature;    /* LangevinLeapfrog temperature [K] */
  double gamma_ps;       /* LangevinLeapfrog gamma [1/ps] */
  uint64_t seed;         /* counter-based RNG key */
} pmgpu_integrator;

/* Integrator::run(n): n steps on the device, state stays resident.
 * Leapfrog follows LeapfrogIntegrator::run (half kick, drift, forces,
 * (kick, drift, forces)*, half kick); LangevinLeapfrog follows
 * StandardIntegrator::run with LangevinLeapfrogIntegrator::doHalfKick.
 * The first call (and any call after positions are set from the host)
 * evaluates the initial forces first, as Integrator::initialize does. */
int pmgpu_run(pmgpu_system *sys, const pmgpu_integrator *integ, long n_steps);

/* ---- asynchronous segments (serving many systems at once) ----------- */
/* pmgpu_run split in two: pmgpu_run_async enqueues the segment on the
 * system's stream and returns at once; pmgpu_run_wait waits for it and
 * returns what pmgpu_run would have (a list overflow found there re-runs
 * the segment from its start before returning).  pmgpu_run_query sets
 * *done without blocking.  Every other call on the system first waits for
 * a pending segment.  Segments of different systems run concurrently on
 * the device.  No counterpart in the reference (ProtoMol runs one system
 * per process). */
int pmgpu_run_async(pmgpu_system *sys, const pmgpu_integrator *integ, long n_steps);
int pmgpu_run_query(pmgpu_system *sys, int *done);
int pmgpu_run_wait(pmgpu_system *sys);
/* Waits for a pending segment and undoes it: positions, velocities,
 * forces and the step counter return to their values at its start, as if it
 * had not run (pair lists are rebuilt at the next evaluation).  A device
 * integrator starts the segment after an output this way before the host
 * knows it is wanted, so that it runs while the outputs are written, and
 * discards it when the next run() asks for other steps or the host changed
 * the state.  No pending segment: nothing to do. */
int pmgpu_run_discard(pmgpu_system *sys);
/* Free and total device memory of the context's GPU (admission control). */
int pmgpu_mem_info(pmgpu_context *ctx, long long *free_bytes, long long *total_bytes);
/* Estimated device bytes of a periodic system of n_atoms with edges
 * box[3], a pair list of the given reach (cutoff + skin; 0: none) and a
 * PME grid (NULL: none). */
int pmgpu_footprint_estimate(int n_atoms, const double box[3], double reach,
                             const int grid[3], long long *bytes);

/* ---- ensembles ------------------------------------------------------ */
/* Many resident systems advanced together.  Every kernel of an MD step is
 * one launch over all members (a device table of per-member arguments and
 * first-block offsets; each block finds its member by binary search), the
 * members whose PME grids have the same dimensions share one batched FFT
 * plan pair, and the steps of a segment replay as captured CUDA graphs, so
 * the launches per step do not grow with the member count.  A member's
 * launches compute what its own single-system launches compute, in the
 * same fixed-point sums: its trajectory is bitwise the same in any
 * ensemble, alone or beside others, for the same pair-kernel splits.
 *
 * Members: periodic, PMGPU_PREC_MIXED, one context, one cutoff pair list
 * (LennardJones and / or Coulomb or the Ewald real term), at most one PME
 * force, bonded terms; the same force set on every member.  They stay
 * owned by the caller, must outlive the ensemble and must not be used
 * through the single-system calls while an ensemble call runs (every
 * ensemble call is synchronous).  No counterpart in the reference, which
 * runs one system per process. */
typedef struct pmgpu_ensemble pmgpu_ensemble;
int pmgpu_ensemble_create(pmgpu_system *const *members, int n, pmgpu_ensemble **out);
/* Gives the members their own PME grids back and frees the ensemble. */
int pmgpu_ensemble_destroy(pmgpu_ensemble *e);
/* n_steps MD steps of integrator it on every member: for each member the
 * steps pmgpu_run(member, it, n_steps) takes, its energies of the last
 * step then read by pmgpu_system_get_energies.  A pair list that overflows
 * grows and the segment runs again from its start on every member. */
int pmgpu_ensemble_run(pmgpu_ensemble *e, const pmgpu_integrator *it, long n_steps);
/* Pair-kernel splits (the warps each 8-atom i cluster's tiles are divided
 * over in the force-only kernel): splits[k] for member k, 0 the
 * single-system choice.  Changes rounding (not the pair set), so results
 * are bitwise reproducible for a given table. */
int pmgpu_ensemble_set_splits(pmgpu_ensemble *e, const int *splits);
/* Device milliseconds of one force-only pair launch over all members with
 * member k at splits[k] (0: its current choice), averaged over reps
 * launches; the members' state is unchanged.  For autotuning. */
int pmgpu_ensemble_time_pairs(pmgpu_ensemble *e, const int *splits, int reps, double *ms);
typedef struct {
  int members;
  int fft_buckets;         /* distinct PME grids (one batched FFT pair each) */
  long long kernels;       /* own kernel launches of the last run */
  long long graph_replays; /* CUDA graph launches of the last run */
  long long steps;         /* MD steps of the last run */
} pmgpu_ensemble_info;
int pmgpu_ensemble_get_info(pmgpu_ensemble *e, pmgpu_ensemble_info *out);
/* Member k's i-cluster count and the splits its pair launch takes. */
int pmgpu_ensemble_member(pmgpu_ensemble *e, int k, int *clusters, int *splits);

/* ---- diagnostics ---------------------------------------------------- */
/* Measured FP32 FMA throughput of the context's GPU in TFLOP/s (an FMA
 * counts two flops): every SM runs independent FMA chains for about a
 * millisecond.  The compute roofline of the pair kernel is quoted against
 * it.  No counterpart in the reference. */
int pmgpu_fp32_peak(pmgpu_context *ctx, double *tflops);
typedef struct {
  long long pairs_in_cutoff;   /* pairs that passed the cutoff test */
  long long list_entries;      /* tiles in the pair list: (8-atom i cluster,
                                  4-atom j cluster, image) entries */
  long long clusters;          /* 8-atom i-clusters */
  long long list_builds;       /* pair-list builds so far */
  int cells[3];                /* sort-grid dims of the cutoff path */
  int pair_kernel;             /* form of the last pair-kernel launch of the
                                  force's list: PMGPU_PAIRK_* */
  int list_capacity;           /* tiles a list row holds (grows on overflow) */
} pmgpu_stats;
/* Pair-kernel forms: the generic kernel (any terms and switches, energies,
 * virial) and the specialised force-only FP32 kernels of the inner MD steps
 * (every term with one cutoff, box edges at least twice the cutoff). */
enum {
  PMGPU_PAIRK_GENERIC = 0,
  PMGPU_PAIRK_LJC2_EWALD = 1,   /* LJ with C2 switching + Ewald real space */
  PMGPU_PAIRK_LJC2_COULC2 = 2,  /* LJ C2 + Coulomb C2 */
  PMGPU_PAIRK_LJC2_COULC1 = 3   /* LJ C2 + Coulomb C1 */
};
/* Counts from the last evaluation of force_id (pairs_in_cutoff requires
 * the force to have been evaluated with counting on; see
 * pmgpu_set_count_pairs). */
int pmgpu_force_stats(pmgpu_system *sys, int force_id, pmgpu_stats *out);
int pmgpu_set_count_pairs(pmgpu_system *sys, int enabled);

/* Per-phase device timing (CUDA events on the system stream), the
 * counterpart of ProtoMol's TimerStatistic FORCES/INTEGRATOR timers
 * (base/TimerStatistic.h:21-28).  Phases: */
enum {
  PMGPU_PHASE_LIST = 0,       /* cell sort, gather, neighbour-list build */
  PMGPU_PHASE_PAIRS = 1,      /* fused LJ / Coulomb / Ewald real pair kernel */
  PMGPU_PHASE_PME = 2,        /* PME spread + FFTs + convolution + gather */
  PMGPU_PHASE_CORRECTION = 3, /* Ewald exclusion correction */
  PMGPU_PHASE_BONDED = 4,     /* bonds and angles */
  PMGPU_PHASE_GB = 5,         /* GB passes */
  PMGPU_PHASE_SIMPLEFULL = 6, /* vacuum all-pairs LJ / Coulomb */
  PMGPU_PHASE_INTEGRATE = 7,  /* kick / drift updates */
  PMGPU_PHASE_COUNT = 8
};
int pmgpu_profile_enable(pmgpu_system *sys, int enabled);
/* Milliseconds and launch counts per phase accumulated since the last
 * reset (ms and launches hold PMGPU_PHASE_COUNT entries each). */
int pmgpu_profile_read(pmgpu_system *sys, double *ms, long long *launches,
                       int reset);
/* Number of this library's own kernels launched on the system so far
 * (library kernels such as cuFFT's are not counted). */
int pmgpu_kernel_count(pmgpu_system *sys, long long *count);

/* ProtoMol cell assignment (topology/Topology.h:44-86 with
 * CubicCellManager, cellsize given) computed by the device binning kernel
 * on the resident positions: cell_xyz gets 3n ints, dims 3 ints. */
int pmgpu_debug_cell_assign(pmgpu_system *sys, double cellsize,
                            int *cell_xyz, int *dims);
/* Fixes the pair lists' capacity (tiles per list row) of the system's
 * cutoff forces, for testing the growth path: a build that needs more
 * flags the overflow internally, the capacity is grown to what the largest
 * row needed and the evaluation or MD segment is repeated from its start,
 * so results equal those of a list that never overflowed.  No counterpart
 * in the reference (its cell lists have no capacity). */
int pmgpu_debug_set_list_capacity(pmgpu_system *sys, int tiles_per_row);
/* Fixes the atoms a pair-list column bucket holds (rounded up to a
 * multiple of 32, at most 4096) for the system's cutoff forces, for testing
 * the growth path: a build that bins more atoms into one column flags the
 * overflow internally, the buckets grow to the fullest column's count and
 * the evaluation or MD segment is repeated from its start. */
int pmgpu_debug_set_column_capacity(pmgpu_system *sys, int atoms_per_column);
/* Limits the tiles a list row may hold in the next builds to tiles_per_row
 * without touching the current list, positions or forces: the first later
 * build (an MD step's rebuild) that needs more takes the growth path, which
 * lifts the limit.  For testing that path inside MD segments. */
int pmgpu_debug_limit_list_rows(pmgpu_system *sys, int tiles_per_row);
/* The unordered pair set (i < j, original indices) the cutoff force
 * force_id evaluated on its last evaluation: pairs gets 2 ints per pair,
 * up to cap pairs; *count gets the total. */
int pmgpu_debug_pair_set(pmgpu_system *sys, int force_id, int *pairs,
                         long long cap, long long *count);

#ifdef __cplusplus
}
#endif
#endif /* PMGPU_H */
