// Internal declarations shared by the pmgpu translation units.
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>
#include <stdint.h>

#include <algorithm>
#include <mutex>
#include <utility>
#include <string>
#include <vector>

#include "pmgpu.h"

namespace pmgpu {

// ---------------------------------------------------------------- errors
void set_error(const std::string &msg);
int fail(int code, const std::string &msg);

#define PM_CUDA(call)                                                        \
  do {                                                                       \
    cudaError_t e_ = (call);                                                 \
    if (e_ != cudaSuccess)                                                   \
      return ::pmgpu::fail(PMGPU_ERR_CUDA, std::string(#call) + ": " +       \
                                               cudaGetErrorString(e_));      \
  } while (0)

#define PM_CHECK(call)                                                       \
  do {                                                                       \
    int r_ = (call);                                                         \
    if (r_ != PMGPU_OK) return r_;                                           \
  } while (0)

// ------------------------------------------------------------ constants
constexpr double kForceScale = PMGPU_FORCE_SCALE;   // 2^32 per kcal/mol/A
constexpr double kEnergyScale = 4294967296.0;       // 2^32 per kcal/mol
constexpr double kInvTimeFactor = 0.02045482828087295;  // PMConstants.cpp:54
constexpr double kBoltzmann = 0.001987191;              // PMConstants.cpp:70
constexpr double kEpsilon = 1.0e-14;                    // PMConstants.cpp:50
constexpr int kMaxInt2 = 2147483647 / 2;                // PMConstants.cpp:45

// Accumulator slots on the device (int64 fixed point, kEnergyScale).
enum { ACC_COULOMB = 0, ACC_LJ, ACC_BOND, ACC_ANGLE, ACC_DIHEDRAL,
       ACC_IMPROPER, ACC_OTHER, ACC_VIRIAL = 7, ACC_PAIRS = 16,
       ACC_COUNT = 18 };

// Status word bits (device side).
enum { ST_LIST_OVERFLOW = 1, ST_NONFINITE = 2, ST_CELL_OVERFLOW = 4,
       ST_BAD_BOX = 8 };

// Tile layout (uint2, 8 bytes): x = j cluster (bits 0..23) | periodic image
// of the j cluster as three 2-bit fields (sx+1, sy+1, sz+1) at bits 24..29
// | kModFlag (bit 30) when the tile has modified (scaled 1-4) pairs;
// y = interaction mask, bit l for lane l = (i atom l & 7, j atom l >> 3).
// The modified mask of a flagged tile is in a parallel array (tmod) at the
// tile's index; it is read only for flagged tiles.  Fully excluded
// minimal-image pairs are cleared from the interaction mask when the list
// is built.
constexpr uint32_t kJMask = 0xFFFFFFu;
constexpr int kShiftBits = 24;
constexpr uint32_t kShiftMask = 0x3Fu;
constexpr uint32_t kModFlag = 1u << 30;
// j-lane entries (uint2, the force-only kernel's list): for each tile and
// each of its j atoms with at least one pair in the interaction mask,
// x = j slot (bits 0..25) | the tile's image code << 26, y = that j atom's
// byte of the interaction mask | its byte of the modified mask << 8.
// A row holds up to 4 entries per tile of capacity.
constexpr int kJSlotBits = 26;
constexpr uint32_t kJSlotMask = (1u << kJSlotBits) - 1u;
constexpr int kZeroShift = 1 | (1 << 2) | (1 << 4);
__host__ __device__ constexpr int shift_code(int sx, int sy, int sz) {
  return (sx + 1) | ((sy + 1) << 2) | ((sz + 1) << 4);
}
constexpr int kMaxAtoms = 1 << 24;

// Sort grid of the cluster-pair list: xy column width (about the edge of a
// cube holding 8 atoms of condensed matter) and z-bin height.
constexpr double kColumnWidth = 4.4;
constexpr double kZBin = 0.5;

// Warps per block of the tile kernel and of the list build.
constexpr int kPairWarps = 8;
constexpr int kBuildWarps = 8;
// Inner MD steps captured per CUDA graph in pmgpu_run.
constexpr long kGraphSteps = 10;

// Orthogonal periodic box in the exact form ProtoMol's
// PeriodicBoundaryConditions::set computes (PeriodicBoundaryConditions.cpp:32-78).
struct Box {
  int periodic;
  double e[3];        // edge lengths e1.x, e2.y, e3.z
  double er[3];       // e1r.x, e2r.y, e3r.z
  double origin[3];
  double min[3], max[3];
  double H[3], H2[3];
  double D;           // min half edge squared
  double V;
};

// Switching function, FP64 constants as ProtoMol precomputes them.
struct SwitchParams {
  int kind;
  int modify;          // switch value/derivative applied (C1, C2, Cn)
  double cutoff, cutoff2, switchon2;
  double c1a, c1b, c1c;          // C1: 1.5/rc, 0.5/rc^3, 1.5/rc^3
  double s1, s2, s3;             // C2: 1/(rc2-rs2)^3, rc2-3rs2, 4/(rc2-rs2)^3
  int ord_int, ord_idx;          // Cn, CmpCnCn
  double irange[8];
  double compoff, compoff2;      // CmpCnCn: the middle distance (-switchoff)
  double itrange[8];             // CmpCnCn: 1/(switchoff - cutoff)^(k)
  int complement;                // ComplementSwitchingFunction of the kind
  double rough2;                 // rough-test cutoff^2 (MAXREAL for a complement)
};

// Pair-term selection for the fused pair kernel.
enum { TERM_LJ = 1, TERM_COUL = 2, TERM_EWALD = 4 };
// What a pair-kernel launch produces: forces only (inner MD steps),
// forces + FP64 energies, + virial, or + the recorded pair set.
enum { PAIR_FORCE = 0, PAIR_ENERGY = 1, PAIR_VIRIAL = 2, PAIR_RECORD = 3 };

struct PairTerms {
  int mask;                 // TERM_*
  SwitchParams lj_sw, coul_sw;
  double lj_cut2, coul_cut2;   // effective rough-test cutoffs^2
  double ewald_alpha, ewald_rc2;
  int exact_erf;
  double coulomb_scaling;
  int minimal_image;        // cutoff terms see only the minimal image
  const float4 *ewtab = nullptr;  // Ewald real-space force table (see below)
};

// Ewald real-space force table of the FP32 force-only kernel: the pair
// force factor G(r^2) = [erfc(a r)/r + 2a/sqrt(pi) exp(-a^2 r^2)] / r^2 (the
// A&S erfc the reference uses, NonbondedFullEwaldSystemForce.h:753-858,
// MathUtilities.cpp:39-49) as cubics in t over intervals of r^2 that split
// each octave [2^e, 2^(e+1)) into 2^kEwTabSubBits equal parts, for
// e = kEwTabLoExp .. kEwTabLoExp + kEwTabOctaves - 1.  The interval index
// and t are bit fields of the FP32 r^2 (exponent and top mantissa bits; the
// rest of the mantissa).  Interpolation error below 1e-8 relative (FP32
// evaluation about 1e-7, as the analytic FP32 form).
constexpr int kEwTabLoExp = -4;      // r^2 from 1/16 A^2
constexpr int kEwTabOctaves = 11;    // to 128 A^2
constexpr int kEwTabSubBits = 7;
constexpr int kEwTabN = kEwTabOctaves << kEwTabSubBits;
constexpr unsigned kEwTabBase = (unsigned)(127 + kEwTabLoExp) << kEwTabSubBits;

// Device arrays of one cluster-pair list (one per distinct (cutoff, skin)
// in a system).  Atoms are binned into buckets of ncx x ncy columns of the
// xy plane and sorted by z inside a column; every column's atoms are
// contiguous and padded to a whole number of 8-atom clusters (padding
// slots hold no atom).  A per-column index of z bins gives the slot range
// of a z window.  The list holds, per 8-atom i cluster, tiles against
// 4-atom j clusters: each unordered pair within the reach appears in
// exactly one tile (see k_build_tiles).
constexpr int kColCap = 4096;  // atoms per column the in-block sort holds
// Every i cluster's tiles are split over kRowParts rows (the columns of its
// search window dealt round-robin), each built and consumed by its own warp.
constexpr int kRowParts = 4;

struct NeighborList {
  double cutoff = 0, skin = 0, reach = 0;
  int ncx = 0, ncy = 0, nzb = 0, ncol = 0;
  double lo[3] = {0, 0, 0};          // grid corner in the wrapped (xw) frame
  double cs[3] = {0, 0, 0};          // column widths (x, y), z-bin height
  int nkeys = 0;                     // ncol * nzb
  int ns_max = 0;                    // slots incl. padding (multiple of 8)
  int nclusters = 0;                 // ns_max / 8
  int nrows = 0;                     // nclusters * kRowParts tile rows
  int cap = 0;                       // tiles per row
  int cap_set = 0;                   // tiles per row fixed by the caller (0: sized here)
  int bcap = 0;                      // atoms a column bucket holds (multiple of 32, <= kColCap)
  int bcap_set = 0;                  // bucket size fixed by the caller (0: sized here)
  int built = 0;
  int decided = 0;                   // this evaluation's rebuild decision is taken
  // a force-only MD step left its pair forces in d_fslot for the next update
  // kernel to add; until then d_force lacks them (nb_fold_slots adds them)
  int slot_pending = 0;
  int limit = 0;  // tiles a row may hold below cap (a test hook; 0: cap)
  int last_form = PMGPU_PAIRK_GENERIC;  // pair-kernel form of the last launch
  long long builds = 0;
  // device
  unsigned *d_zkey = nullptr;    // n: z above the grid corner (FP32 bits, >= 0)
  int *d_bucket = nullptr;       // ncol buckets of bcap atoms: each column's atoms, any order
  int *d_col_count = nullptr;    // ncol: atoms binned into each column
  int *d_col_base = nullptr;     // ncol + 1: first slot of each column (padded)
  int *d_key_start = nullptr;    // nkeys + 1: first slot of each (column, z bin)
  int *d_sorted = nullptr;       // ns_max: atom of each slot, -1 for padding
  double *d_offset = nullptr;    // 3n: x_build - x_wrapped (original order)
  double *d_xbuild = nullptr;    // 3n
  float4 *d_xhi = nullptr;       // ns_max (x,y,z,q)
  float4 *d_xlo = nullptr;       // ns_max (x,y,z residue, type bits)
  double4 *d_xw = nullptr;       // ns_max FP64 wrapped position + q
  int *d_mol_s = nullptr;        // ns_max molecule of each slot (-1 padding)
  float4 *d_bb = nullptr;        // 2 per 4-atom cluster: lower, upper corner
  long long *d_fslot = nullptr;  // 3 planes of ns_max: pair forces by slot (fixed point)
  int *d_slot_of = nullptr;  // atom -> slot of the current order (rebuild steps write it)
  uint2 *d_tiles = nullptr;      // nrows rows of cap tiles (row r: cluster r / kRowParts)
  unsigned *d_tmod = nullptr;    // modified masks of the flagged tiles, same indexing
  uint2 *d_jlanes = nullptr;     // nrows rows of 4 cap j-lane entries
  int *d_jl_count = nullptr;     // entries per row
  int *d_tile_count = nullptr;   // nrows
  unsigned int *d_maxdisp = nullptr;  // rebuild check: block ticket, max displacement^2 bits
  // rebuild flag, build count, largest row need and largest column count
  // after an overflow
  int *d_rebuild = nullptr;
  // the tile build's row counter and finished-warp count; binning blocks done
  int *d_build_work = nullptr;
};

struct System;

struct Force {
  int kind = 0;     // FK_*
  int enabled = 1;
  int id = 0;
  // cutoff / ewald
  PairTerms terms{};
  double cellsize = 0;
  double alg_cutoff = 0;
  int list_index = -1;
  // ewald
  int ewald_flags = 0;
  double alpha = 0, rc = 0;
  int order = 4;
  int grid[3] = {0, 0, 0};
  double self_energy = 0, charged_energy = 0;
  // pme device state
  cufftHandle plan_r2c = 0, plan_c2r = 0;
  float *d_grid = nullptr;            // real grid (K1*K2*K3)
  long long *d_grid_fixed = nullptr;  // fixed-point spread target
  float2 *d_cgrid = nullptr;          // complex grid (K1*K2*(K3/2+1))
  float *d_influence = nullptr;       // K1*K2*(K3/2+1) influence function
  float4 *d_ewtab = nullptr;          // real-space force table (kEwTabN cubics)
  void *d_fft_work = nullptr;         // cuFFT work area shared by both plans
  size_t fft_work_bytes = 0;
  // simplefull
  int sf_lj = 0, sf_coul = 0;
  // SCPISM: bulk dielectric (-D); Born radii and self-force switches/cutoffs
  double scp_D = 80.0;
  int born_rsw = 3, born_ssw = 3;
  double born_rcut = 5.0, born_scut = 5.0;
  // gb
  double solute = 1.0, solvent = 80.0;
  // gbace (GBACEForce -solvationparam, -watersphereradius)
  double ace_sigma = 0.0, ace_rho = 0.0;
  // bonded
  int bonds = 0, angles = 0;
  int dihedrals = 0, impropers = 0;
  long long last_pairs = 0;
};

enum { FK_CUTOFF = 1, FK_PME = 2, FK_GB = 3, FK_BONDED = 4,
       FK_SIMPLEFULL = 5, FK_TORSION = 6, FK_GBACE = 7,
       FK_SIMPLEFULL_SW = 8 /* switched all pairs: terms.mask, lj_sw, coul_sw */,
       FK_SCPISM = 9 /* LJ + CoulombSCPISM all pairs within the switch cutoffs */,
       FK_BORN = 10 /* SCPISM BornRadii + BornSelf */ };

// Per-phase CUDA-event timing; events are recorded only when enabled and
// summed at the next host synchronisation.
struct Profiler {
  int enabled = 0;
  struct Mark { int phase; cudaEvent_t a, b; };
  std::vector<Mark> pending;
  std::vector<cudaEvent_t> pool;
  double ms[PMGPU_PHASE_COUNT] = {0};
  long long launches[PMGPU_PHASE_COUNT] = {0};
  int open_phase = -1;
  cudaEvent_t open_ev = nullptr;
};
void prof_begin(struct System *s, int phase);
void prof_end(struct System *s);
void prof_collect(struct System *s);

struct System {
  pmgpu_context *ctx = nullptr;
  Profiler prof;
  long long kernels = 0;  // own kernel launches (see pmgpu_kernel_count)
  int device = 0;
  int n = 0;
  int precision = PMGPU_PREC_MIXED;
  Box box{};
  cudaStream_t stream = nullptr;
  cudaStream_t side = nullptr;     // second stream for the non-pair terms
  cudaStream_t side2 = nullptr;    // third stream: short terms beside the PME chain
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_join2 = nullptr;
  // host copies of static topology
  std::vector<double> h_charge, h_mass;
  std::vector<int> h_type, h_mol;
  int ntypes = 0;
  std::vector<double> h_lj;
  std::vector<int> h_excl;  // exclusions as given: a, b, class per entry
  double coulomb_scaling = 1.0;
  // device topology
  double *d_charge = nullptr, *d_mass = nullptr;
  int *d_type = nullptr, *d_mol = nullptr;
  float4 *d_lj32 = nullptr;     // ntypes^2: A, B, A14, B14 (FP32)
  float2 *d_ljab = nullptr;     // ntypes^2 by column: [t2 * ntypes + t1] = A, B of (t1, t2)
  float2 *d_ljcomb = nullptr;   // per type sqrt(epsilon), rmin/2 when the table follows the CHARMM rule
  double4 *d_lj64 = nullptr;    // ntypes^2 (FP64)
  int *d_excl_start = nullptr, *d_excl_partner = nullptr;  // CSR
  int *d_excl_class = nullptr;
  int *d_excl_pairs = nullptr;  // 3 per exclusion (a1, a2, class)
  int2 *d_excl_range = nullptr; // per atom: lowest and highest partner index
  int n_excl = 0;
  int n_bonds = 0, n_angles = 0;
  int *d_bond_atoms = nullptr, *d_angle_atoms = nullptr;
  double *d_bond_params = nullptr, *d_angle_params = nullptr;
  int n_dihedrals = 0, n_impropers = 0;
  int *d_dihedral_atoms = nullptr, *d_improper_atoms = nullptr;
  double *d_dihedral_params = nullptr, *d_improper_params = nullptr;
  // GB
  double *d_gb_vdwr = nullptr, *d_gb_scale = nullptr, *d_gb_offset = nullptr;
  int *d_water = nullptr;
  // SCPISM (pmgpu_topology scpism_*): [6][n] sqrt(alpha), alpha, zeta, eta,
  // C_i, g_i and [3][n] H-bond class, residue, name class; the BornSelf
  // factor and self energy of each atom [2][n] (per evaluation)
  double *d_scp = nullptr;
  int *d_scp_i = nullptr;
  double *d_born_q = nullptr;
  double gb_obc[3] = {1.0, 0.8, 4.85};
  double *d_gb_born = nullptr, *d_gb_psi = nullptr, *d_gb_partial = nullptr;
  long long *d_gb_fixed = nullptr;  // 2n: burial and partial-sum accumulators
  double *d_gb_ace = nullptr;       // n: GBACE pair-force factor per atom
  // dynamic state
  double *d_pos = nullptr;   // 3n AoS
  double *d_vel = nullptr;   // 3n AoS
  long long *d_force = nullptr;  // 3 planes of n, fixed point
  long long *d_acc = nullptr;    // ACC_COUNT fixed point accumulators
  int *d_status = nullptr;
  // simple-full tile masks: per tile pair (I <= J) of 32-atom tiles the
  // index of its masks or -1; per (masks, lane) the bits of excluded (x)
  // and modified (y) partners k of that lane's atom
  int *d_sf_tile = nullptr;
  uint2 *d_sf_bits = nullptr;
  // FP32 pair records of the all-pairs passes (2n, write_pair_record);
  // rec_fresh: this evaluation's update kernel wrote them
  float4 *d_rec = nullptr;
  int rec_fresh = 0;
  // GB FP32 records: static (k_gb_static) and per evaluation (k_gb_radii)
  float4 *d_gb_gst = nullptr, *d_gb_grad = nullptr;
  long long *h_acc = nullptr;    // pinned mirror
  int *h_status = nullptr;       // pinned mirror
  // forces and lists
  std::vector<Force> forces;
  std::vector<NeighborList> lists;
  int count_pairs = 0;
  int forces_valid = 0;   // resident forces correspond to resident positions
  uint64_t step = 0;      // RNG counter (host mirror of *d_step)
  unsigned long long *d_step = nullptr;
  // captured multi-step graphs of pmgpu_run (invalidated by graph_version)
  int graph_version = 0;
  int graphs_disabled = 0;
  struct StepGraph {
    int version = -1;
    long steps = 0;
    pmgpu_integrator key{};
    cudaGraphExec_t exec = nullptr;
    long long kernels = 0;  // own kernels per replay
  } graphs[2];
  struct PendingRun {
    int active = 0;
    pmgpu_integrator integ{};
    long n_steps = 0;
    uint64_t step0 = 0;
    int valid0 = 0;
  } pending;  // segment enqueued by pmgpu_run_async, not yet waited for
  long long last_pairs = 0;
  double last_energy[PMGPU_E_COUNT] = {0, 0, 0, 0, 0, 0, 0};
  double last_virial[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  double *d_stage = nullptr;       // 3n device staging
  void *d_snap = nullptr;          // run() rollback snapshot (pos, vel, force)
  double *h_stage = nullptr;       // 3n pinned host staging
  long long *d_pairbuf = nullptr;  // debug pair-set buffer
  long long pairbuf_cap = 0;
  long long *d_paircount = nullptr;
};

// Device buffers are stream-ordered (cudaMallocAsync / cudaFreeAsync on the
// system's stream): creating and destroying a system never synchronises the
// whole device, so systems served side by side do not stall one another.
// Launches kern on st as a programmatic dependent of the stream's previous
// kernel (see pdl_wait in pm_device.cuh); kern must call pdl_wait() first.
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem,
                              cudaStream_t st, Args... args) {
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}

int dev_alloc(System *s, void **p, size_t bytes);
template <typename T>
inline int dev_alloc(System *s, T **p, size_t bytes) {
  return dev_alloc(s, reinterpret_cast<void **>(p), bytes);
}
void dev_free(System *s, void *p);

// ------------------------------------------------------- batched launches
// One batched launch's arguments: the launch arguments of every member of an
// ensemble and the first block of each member in the grid (first[n] is the
// grid size), copied to the device once; a kernel's batched form finds its
// member by the block index (batch_member in pm_device.cuh).
template <typename A>
struct BatchTable {
  std::vector<A> h;
  std::vector<int> first = std::vector<int>(1, 0);
  A *d = nullptr;
  int *d_first = nullptr;
  size_t cap = 0;
  void clear() {
    h.clear();
    first.assign(1, 0);
  }
  void add(const A &a, int blocks) {
    h.push_back(a);
    first.push_back(first.back() + blocks);
  }
  int total() const { return first.back(); }
  int members() const { return (int)h.size(); }
  // copies the host tables to the device (synchronously: the host vectors
  // may change afterwards)
  cudaError_t upload() {
    if (h.size() > cap) {
      release();
      cap = h.size();
      cudaError_t e = cudaMalloc(&d, sizeof(A) * std::max<size_t>(cap, 1));
      if (e == cudaSuccess) e = cudaMalloc(&d_first, sizeof(int) * (cap + 1));
      if (e != cudaSuccess) return e;
    }
    if (h.empty()) return cudaSuccess;
    cudaError_t e = cudaMemcpy(d, h.data(), sizeof(A) * h.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return e;
    return cudaMemcpy(d_first, first.data(), sizeof(int) * first.size(), cudaMemcpyHostToDevice);
  }
  void release() {
    if (d) cudaFree(d);
    if (d_first) cudaFree(d_first);
    d = nullptr;
    d_first = nullptr;
    cap = 0;
  }
};

// ------------------------------------------------------------ host API of TUs
void box_from_topology(const pmgpu_topology *t, Box *b);
void switch_setup(const pmgpu_switch *in, SwitchParams *o);

// api.cu (shared with the ensemble driver)
// evaluates the enabled forces (only >= 0: that force) at the resident
// positions into the zeroed forces and accumulators; fold = 0 leaves the
// pair forces of a force-only MD step in the list's slot buffer
int evaluate_forces(System *s, int only, int mode, int fold = 1);
int begin_eval(System *s);
// reads the accumulators and the status word after an evaluation or a
// segment (overflow: the lists grow and PMGPU_ERR_OVERFLOW is returned)
int read_results(System *s, int only, double *energies, double *virial, int add,
                 int energies_valid = 1);
// the same on accumulators and status already copied to h_acc / h_status
int take_results(System *s, int only, double *energies, double *virial, int add,
                 int energies_valid = 1);
int run_snapshot(System *s, int restore);
void pair_groups(System *s, std::vector<std::pair<int, PairTerms>> *out);

// batched launches over an ensemble's members (nonbonded.cu, pme.cu,
// bonded_integrate.cu)
struct NbBatch;
struct PmeBatch;
struct BdBatch;
NbBatch *nb_batch_new();
void nb_batch_free(NbBatch *b);
int nb_batch_build(NbBatch *b, System *const *m, int n, const PairTerms *terms,
                   const int *splits);
int nb_batch_time_jl(NbBatch *b, System *const *m, int n, const int *splits, int reps,
                     cudaStream_t st, double *ms);
void nb_batch_member_info(NbBatch *b, int k, int *splits, int *clusters);
int nb_batch_list(NbBatch *b, cudaStream_t st, long long *launched);
int nb_batch_pairs(NbBatch *b, int mode, cudaStream_t st, long long *launched);
void nb_batch_mark(NbBatch *b, System *const *m, int n, int mode);
PmeBatch *pme_batch_new();
void pme_batch_free(PmeBatch *b);
int pme_batch_build(PmeBatch *b, System *const *m, int n, Force *const *fs);
int pme_batch_reciprocal(PmeBatch *b, int em, cudaStream_t st, long long *launched);
int pme_batch_correction(PmeBatch *b, int em, cudaStream_t st, long long *launched);
int pme_batch_buckets(const PmeBatch *b);
BdBatch *bd_batch_new();
void bd_batch_free(BdBatch *b);
int bd_batch_build(BdBatch *b, System *const *m, int n, const pmgpu_integrator *it,
                   const int *bd_flags);
int bd_batch_update(BdBatch *b, int phase, int zero_acc, cudaStream_t st,
                    long long *launched);
int bd_batch_bonded(BdBatch *b, int em, cudaStream_t st, long long *launched);

// nonbonded.cu
int nb_list_init(System *s, NeighborList *nl, double cutoff, double skin,
                 double cellsize_for_debug);
int nb_list_free(System *s, NeighborList *nl);
// Per evaluation: nb_prepare (rebuild decision, conditional sort, gather of
// the slot coordinates), then nb_build (conditional cluster boxes and tile
// build), then nb_pair_forces.
int nb_prepare(System *s, NeighborList *nl, int force_rebuild);
int nb_build(System *s, NeighborList *nl);
// fold: add the slot-ordered pair forces into the atom forces at once;
// 0 (force-only MD steps with one list) leaves them for the next update
// kernel and marks the list slot_pending
int nb_pair_forces(System *s, NeighborList *nl, const PairTerms &t, int mode, int fold);
// adds a pending slot buffer into the atom forces (no-op when none is pending)
int nb_fold_slots(System *s, NeighborList *nl);
int fold_pending_slots(System *s);
int nb_debug_cells(System *s, double cellsize, int *cell_xyz, int *dims);
int nb_simplefull(System *s, int lj, int coul, int em);
int nb_simplefull_sw(System *s, const SwitchParams *lj_sw, const SwitchParams *coul_sw,
                     int em, int scpism = 0, double dielectric = 80.0);
int nb_born(System *s, const Force &f, int em);
// the exclusion tile masks of the FP32 simple-full pass (once per system)
int nb_simplefull_init(System *s);
// Launch shape of the FP32 half all-pairs passes (each unordered pair once,
// forces to both atoms): work items of 32 i atoms x 32 / split j atoms (a
// share of a 32 x 32 tile pair I <= J) in equal shares per block
// (BlockItems); one block per SM (the kernels' register counts admit no
// second).
void halfpairs_grid(int n, int split, int *tiles, long long *items, int *blocks);
// the atoms' FP32 pair records (write_pair_record) from the FP64 positions
int nb_stage_pairs(System *s);
void launch_stage_pairs(int n, const double *pos, const double *charge, const int *type,
                        float4 *rec, cudaStream_t st);

// pme.cu
int pme_init(System *s, Force *f);
int pme_free(System *s, Force *f);
// builds f->d_ewtab for f->alpha (nonbonded.cu)
int ewald_table_build(System *s, Force *f);
int pme_reciprocal(System *s, Force *f, int em);
int ewald_correction(System *s, Force *f, int em);

// gb.cu
int gb_init(System *s);
int gb_forces(System *s, const Force *gb, const Force *ace);

// bonded_integrate.cu
// bonds, angles, dihedrals and impropers (each flag: include that kind) in
// one launch; *launched = 1 when there was any term
int bonded_all(System *s, int bonds, int angles, int dihedrals, int impropers, int em,
               int *launched);
int zero_forces(System *s);
// zero_acc: the update launch also clears the energy accumulators (the
// start of a force evaluation); list: the pair list whose rebuild decision
// the update takes from the drifted positions (or null)
int integrate_kick_drift(System *s, const pmgpu_integrator *it, int phase, int zero_acc = 0,
                         NeighborList *list = nullptr);
struct UpdateArgs;
int update_args(System *s, const pmgpu_integrator *it, int phase, int zero_acc,
                NeighborList *list, UpdateArgs *out);
int update_blocks(const System *s);
int set_device_step(System *s);
int forces_to_host(System *s, double *out, int add);

}  // namespace pmgpu

struct pmgpu_context {
  int device = 0;
  // cuFFT plan pairs (R2C, C2R) of systems that ended, kept for the next
  // system of the same grid: plan creation costs more than a short request
  struct FftPlans {
    int dims[3];
    cufftHandle r2c, c2r;
    size_t work;  // work-area bytes the pair needs
  };
  std::mutex fft_mu;
  std::vector<FftPlans> fft_free;
};
