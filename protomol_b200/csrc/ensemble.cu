// Ensembles: many resident systems advanced together (pmgpu_ensemble_*).
//
// An ensemble step is the single-system MD step (update kernel, then the
// force evaluation at the drifted positions) with every kernel launched
// once over all members: each batched kernel reads a device table of
// per-member arguments and first-block offsets, and a block runs the
// member's own kernel body on the member's own block index.  The PME
// chain runs on a second stream and the short terms (Ewald correction,
// bonded) on a third, beside the list work and the pair kernel, as in the
// single-system evaluation.  Forces and energies are 64-bit fixed-point
// sums, so the order in which blocks of different members (or of one
// member) finish changes nothing: a member's results are bitwise those of
// the same member in any other ensemble with the same pair-kernel splits.
//
// Segment control mirrors pmgpu_run: a snapshot of every member's state,
// the steps (replayed from captured CUDA graphs), one gathered read of all
// members' accumulators and status words, and on a pair-list overflow the
// lists grow, the tables are rebuilt and the segment runs again from the
// snapshot.
#include <cstring>
#include <map>

#include "pm_device.cuh"
#include "pm_internal.cuh"

namespace pmgpu {

// One member's state and its rollback snapshot (the layout of
// run_snapshot: positions, velocities, then fixed-point forces).
struct SnapArgs {
  long long n3;
  double *pos, *vel;
  long long *force;
  double *spos, *svel;
  long long *sforce;
  unsigned long long *step;  // device step counter (Langevin noise)
};

// SAVE: state -> snapshot; otherwise snapshot -> state.  Either way the
// member's device step counter is set to steps0[m], the host counter at the
// start of the segment.
template <bool SAVE>
__global__ void __launch_bounds__(256)
    k_snapshot_batch(const SnapArgs *__restrict__ tab, const int *__restrict__ first, int nm,
                     const unsigned long long *__restrict__ steps0) {
  const int m = batch_member(first, nm, blockIdx.x);
  const Blk b = batch_blk(first, m);
  const SnapArgs a = tab[m];
  for (long long i = (long long)b.x * blockDim.x + threadIdx.x; i < a.n3;
       i += (long long)b.n * blockDim.x) {
    if (SAVE) {
      a.spos[i] = a.pos[i];
      a.svel[i] = a.vel[i];
      a.sforce[i] = a.force[i];
    } else {
      a.pos[i] = a.spos[i];
      a.vel[i] = a.svel[i];
      a.force[i] = a.sforce[i];
    }
  }
  if (b.x == 0 && threadIdx.x == 0) *a.step = steps0[m];
}

// Every member's accumulators and status word into one packed array of
// ACC_COUNT + 1 values per member (one block each), read back in one copy.
struct ResArgs {
  const long long *acc;
  const int *status;
};
__global__ void k_results_batch(const ResArgs *__restrict__ tab, int nm,
                                long long *__restrict__ out) {
  const int m = blockIdx.x;
  if (m >= nm) return;
  const ResArgs a = tab[m];
  long long *o = out + (size_t)m * (ACC_COUNT + 1);
  for (int i = threadIdx.x; i < ACC_COUNT; i += blockDim.x) o[i] = a.acc[i];
  if (threadIdx.x == 0) o[ACC_COUNT] = *a.status;
}

// Segments of up to this many steps replay as one captured graph (first
// step, inner steps, last step and closing half kick); longer segments
// replay graphs of kEnsembleChunk inner steps between an eager first and
// last step.
constexpr long kEnsembleWhole = 64;
constexpr long kEnsembleChunk = 50;

}  // namespace pmgpu

using namespace pmgpu;

struct pmgpu_ensemble {
  int device = 0;
  std::vector<System *> m;
  cudaStream_t st = nullptr, side = nullptr, side2 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_join2 = nullptr;
  NbBatch *nb = nullptr;
  PmeBatch *pme = nullptr;
  BdBatch *bd = nullptr;
  // the force set every member has
  int terms = 0;
  int pme_flags = 0;           // ewald_flags of the PME force (0: none)
  int bd_flags[4] = {0, 0, 0, 0};
  std::vector<Force *> pme_force;
  std::vector<int> splits;     // per member; 0: the single-system choice
  // tables and graphs
  int nb_valid = 0, bd_valid = 0;
  pmgpu_integrator key{};
  std::vector<long long> seen_version;  // members' graph_version at the last build
  long long version = 0;       // bumped by every table rebuild
  struct Graph {
    cudaGraphExec_t exec = nullptr;
    long long version = -1;
    long long kernels = 0;
  };
  std::map<std::pair<long, int>, Graph> graphs;  // (steps, whole segment?)
  int graphs_disabled = 0;
  BatchTable<SnapArgs> snap;
  BatchTable<ResArgs> res;
  long long *d_res = nullptr, *h_res = nullptr;
  unsigned long long *d_steps0 = nullptr, *h_steps0 = nullptr;
  // counters
  long long kernels = 0, replays = 0, last_kernels = 0, last_replays = 0, last_steps = 0;
};

namespace {

int ens_fail(int code, const char *msg) { return fail(code, msg); }

// The force set of a member as the ensemble needs it: the merged terms of
// its one pair-kernel group, its PME force, its bonded flags.
int member_shape(System *s, PairTerms *terms, Force **pme, int bd[4]) {
  if (!s->box.periodic) return ens_fail(PMGPU_ERR_UNSUPPORTED, "ensemble members must be periodic");
  if (s->precision != PMGPU_PREC_MIXED)
    return ens_fail(PMGPU_ERR_UNSUPPORTED, "ensemble members must be mixed precision");
  if (s->n == 0) return ens_fail(PMGPU_ERR_UNSUPPORTED, "ensemble members need atoms");
  if (s->pending.active) return ens_fail(PMGPU_ERR_STATE, "a member has a segment pending");
  if (s->prof.enabled) return ens_fail(PMGPU_ERR_STATE, "a member has profiling on");
  std::vector<std::pair<int, PairTerms>> groups;
  pair_groups(s, &groups);
  if (s->lists.size() != 1 || groups.size() != 1 || groups[0].first != 0)
    return ens_fail(PMGPU_ERR_UNSUPPORTED, "ensemble members need exactly one cutoff pair list");
  *terms = groups[0].second;
  *pme = nullptr;
  bd[0] = bd[1] = bd[2] = bd[3] = 0;
  for (auto &f : s->forces) {
    if (!f.enabled) continue;
    switch (f.kind) {
      case FK_CUTOFF:
        break;
      case FK_PME:
        if (f.ewald_flags & (PMGPU_EWALD_RECIPROCAL | PMGPU_EWALD_CORRECTION)) {
          if (*pme) return ens_fail(PMGPU_ERR_UNSUPPORTED, "ensemble members need one PME force");
          *pme = &f;
        }
        break;
      case FK_BONDED:
        bd[0] |= f.bonds;
        bd[1] |= f.angles;
        break;
      case FK_TORSION:
        bd[2] |= f.dihedrals;
        bd[3] |= f.impropers;
        break;
      default:
        return ens_fail(PMGPU_ERR_UNSUPPORTED,
                        "ensemble members take cutoff, PME and bonded forces only");
    }
  }
  if (*pme && !((*pme)->ewald_flags & PMGPU_EWALD_RECIPROCAL))
    return ens_fail(PMGPU_ERR_UNSUPPORTED, "the ensemble's PME force needs its reciprocal term");
  return PMGPU_OK;
}

int check_shapes(pmgpu_ensemble *e, std::vector<PairTerms> *terms) {
  const int n = (int)e->m.size();
  terms->assign(n, PairTerms());
  for (int k = 0; k < n; k++) {
    Force *pf = nullptr;
    int bd[4];
    PM_CHECK(member_shape(e->m[k], &(*terms)[k], &pf, bd));
    const int flags = pf ? pf->ewald_flags : 0;
    if ((*terms)[k].mask != e->terms || flags != e->pme_flags || pf != e->pme_force[k] ||
        std::memcmp(bd, e->bd_flags, sizeof(bd)) != 0)
      return ens_fail(PMGPU_ERR_UNSUPPORTED, "ensemble members need the same force set");
  }
  return PMGPU_OK;
}

// Forces of members whose resident forces are stale (new positions, a
// first run): the single-system evaluation, pair forces folded at once.
int ensure_forces(pmgpu_ensemble *e) {
  for (System *s : e->m) {
    if (s->forces_valid) continue;
    int r = PMGPU_OK;
    for (int attempt = 0; attempt < 3; attempt++) {
      PM_CHECK(zero_forces(s));
      PM_CHECK(begin_eval(s));
      PM_CHECK(evaluate_forces(s, -1, PAIR_FORCE, 1));
      r = read_results(s, -1, nullptr, nullptr, 0, 0);
      if (r != PMGPU_ERR_OVERFLOW) break;
    }
    PM_CHECK(r);
    s->forces_valid = 1;
  }
  return PMGPU_OK;
}

// (Re)builds the list, pair and update tables when a member's buffers
// changed (list growth, a first run) or the integrator changed.
int ensure_tables(pmgpu_ensemble *e, const pmgpu_integrator *it) {
  const int n = (int)e->m.size();
  bool stale = !e->nb_valid;
  for (int k = 0; k < n; k++) stale |= e->seen_version[k] != e->m[k]->graph_version;
  std::vector<PairTerms> terms;
  if (stale) {
    PM_CHECK(check_shapes(e, &terms));
    PM_CHECK(nb_batch_build(e->nb, e->m.data(), n, terms.data(), e->splits.data()));
    e->nb_valid = 1;
    e->bd_valid = 0;
  }
  const bool same = e->key.kind == it->kind && e->key.timestep_fs == it->timestep_fs &&
                    e->key.temperature == it->temperature && e->key.gamma_ps == it->gamma_ps &&
                    e->key.seed == it->seed;
  if (!e->bd_valid || !same) {
    std::vector<int> flags(4 * (size_t)n);
    for (int k = 0; k < n; k++)
      for (int q = 0; q < 4; q++) flags[4 * k + q] = e->bd_flags[q];
    PM_CHECK(bd_batch_build(e->bd, e->m.data(), n, it, flags.data()));
    e->bd_valid = 1;
    e->key = *it;
    stale = true;
  }
  if (stale) {
    for (int k = 0; k < n; k++) e->seen_version[k] = e->m[k]->graph_version;
    e->version++;
  }
  return PMGPU_OK;
}

// One MD step of every member (one_step + evaluate_forces of each).
int ens_step(pmgpu_ensemble *e, int phase, int mode) {
  long long &kc = e->kernels;
  // the update launch also clears the accumulators and takes the rebuild
  // decision of each member's list
  PM_CHECK(bd_batch_update(e->bd, phase, 1, e->st, &kc));
  const int em = mode == PAIR_FORCE ? 0 : 1;
  PM_CUDA(cudaEventRecord(e->ev_fork, e->st));
  PM_CUDA(cudaStreamWaitEvent(e->side, e->ev_fork, 0));
  PM_CUDA(cudaStreamWaitEvent(e->side2, e->ev_fork, 0));
  if (e->pme_flags & PMGPU_EWALD_RECIPROCAL)
    PM_CHECK(pme_batch_reciprocal(e->pme, em, e->side, &kc));
  if (e->pme_flags & PMGPU_EWALD_CORRECTION)
    PM_CHECK(pme_batch_correction(e->pme, em, e->side2, &kc));
  PM_CHECK(bd_batch_bonded(e->bd, em, e->side2, &kc));
  PM_CHECK(nb_batch_list(e->nb, e->st, &kc));
  PM_CHECK(nb_batch_pairs(e->nb, mode, e->st, &kc));
  PM_CUDA(cudaEventRecord(e->ev_join, e->side));
  PM_CUDA(cudaStreamWaitEvent(e->st, e->ev_join, 0));
  PM_CUDA(cudaEventRecord(e->ev_join2, e->side2));
  PM_CUDA(cudaStreamWaitEvent(e->st, e->ev_join2, 0));
  return PMGPU_OK;
}

// Steps k0..k1-1 of a segment of n steps (the first step takes the
// starting half kick, the last evaluates energies); closing adds the
// segment's closing half kick.
int ens_enqueue(pmgpu_ensemble *e, long k0, long k1, long n, int closing) {
  const bool lang = e->key.kind == PMGPU_INT_LANGEVIN_LEAPFROG;
  for (long k = k0; k < k1; k++) {
    const int phase = lang ? (k == 0 ? 3 : 4) : (k == 0 ? 0 : 1);
    PM_CHECK(ens_step(e, phase, k + 1 == n ? PAIR_ENERGY : PAIR_FORCE));
  }
  if (closing) PM_CHECK(bd_batch_update(e->bd, lang ? 5 : 2, 0, e->st, &e->kernels));
  return PMGPU_OK;
}

// Replays (capturing on first use) the graph of steps k0..k1-1 of a
// segment of n steps; *used = 0 when capture is not possible.
int ens_graph(pmgpu_ensemble *e, long k0, long k1, long n, int closing, int *used) {
  *used = 0;
  const std::pair<long, int> key(closing ? n : k1 - k0, closing);
  pmgpu_ensemble::Graph &g = e->graphs[key];
  if (!g.exec || g.version != e->version) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    g.exec = nullptr;
    const long long k_before = e->kernels;
    if (cudaStreamBeginCapture(e->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      cudaGetLastError();
      e->graphs_disabled = 1;
      return PMGPU_OK;
    }
    int r = ens_enqueue(e, k0, k1, n, closing);
    cudaGraph_t graph = nullptr;
    cudaError_t ec = cudaStreamEndCapture(e->st, &graph);
    const long long per = e->kernels - k_before;
    e->kernels = k_before;
    cudaError_t ei = cudaSuccess;
    if (r == PMGPU_OK && ec == cudaSuccess && graph)
      ei = cudaGraphInstantiate(&g.exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (r != PMGPU_OK || ec != cudaSuccess || !graph || ei != cudaSuccess) {
      if (std::getenv("PMGPU_DEBUG"))
        std::fprintf(stderr, "pmgpu: ensemble graph not used (end capture: %s; instantiate: %s)\n",
                     cudaGetErrorString(ec), cudaGetErrorString(ei));
      cudaGetLastError();
      g.exec = nullptr;
      e->graphs_disabled = 1;
      return PMGPU_OK;
    }
    g.version = e->version;
    g.kernels = per;
  }
  PM_CUDA(cudaGraphLaunch(g.exec, e->st));
  e->kernels += g.kernels;
  e->replays++;
  *used = 1;
  return PMGPU_OK;
}

int ens_segment(pmgpu_ensemble *e, long n) {
  int used = 0;
  if (!e->graphs_disabled && n <= kEnsembleWhole) {
    PM_CHECK(ens_graph(e, 0, n, n, 1, &used));
    if (used) return PMGPU_OK;
  }
  PM_CHECK(ens_enqueue(e, 0, 1, n, 0));
  long k = 1;
  while (k < n - 1) {
    const long g = std::min(kEnsembleChunk, n - 1 - k);
    used = 0;
    if (!e->graphs_disabled) PM_CHECK(ens_graph(e, k, k + g, n, 0, &used));
    if (!used) PM_CHECK(ens_enqueue(e, k, k + g, n, 0));
    k += g;
  }
  return ens_enqueue(e, std::max(k, 1L), n, n, 1);
}

int ens_snapshot(pmgpu_ensemble *e, int save) {
  const int nm = e->snap.members();
  if (save)
    k_snapshot_batch<true><<<e->snap.total(), 256, 0, e->st>>>(e->snap.d, e->snap.d_first, nm,
                                                               e->d_steps0);
  else
    k_snapshot_batch<false><<<e->snap.total(), 256, 0, e->st>>>(e->snap.d, e->snap.d_first, nm,
                                                                e->d_steps0);
  PM_CUDA(cudaGetLastError());
  e->kernels++;
  return PMGPU_OK;
}

// Reads every member's accumulators and status; *overflow is set when a
// list overflowed (that member's lists have grown).
int ens_results(pmgpu_ensemble *e, int *overflow) {
  const int n = (int)e->m.size();
  k_results_batch<<<n, 32, 0, e->st>>>(e->res.d, n, e->d_res);
  PM_CUDA(cudaGetLastError());
  e->kernels++;
  PM_CUDA(cudaMemcpyAsync(e->h_res, e->d_res, sizeof(long long) * (ACC_COUNT + 1) * n,
                          cudaMemcpyDeviceToHost, e->st));
  PM_CUDA(cudaStreamSynchronize(e->st));
  *overflow = 0;
  int err = PMGPU_OK;
  for (int k = 0; k < n; k++) {
    System *s = e->m[k];
    const long long *o = e->h_res + (size_t)k * (ACC_COUNT + 1);
    std::memcpy(s->h_acc, o, sizeof(long long) * ACC_COUNT);
    *s->h_status = (int)o[ACC_COUNT];
    if (!*s->h_status) {
      PM_CHECK(take_results(s, -1, nullptr, nullptr, 0, 1));
      continue;
    }
    const int r = take_results(s, -1, nullptr, nullptr, 0, 1);
    PM_CUDA(cudaStreamSynchronize(s->stream));  // the status reset, a list regrown
    if (r == PMGPU_ERR_OVERFLOW) *overflow = 1;
    else if (err == PMGPU_OK) err = r;
  }
  return err;
}

// Host flags of a member after a segment, as pmgpu_run leaves them.
void mark_members(pmgpu_ensemble *e, long n_steps, int ok) {
  nb_batch_mark(e->nb, e->m.data(), (int)e->m.size(), PAIR_ENERGY);
  for (System *s : e->m) {
    s->step += (uint64_t)n_steps;
    s->forces_valid = ok;
    s->rec_fresh = 0;
    for (auto &nl : s->lists) {
      nl.decided = 0;
      nl.slot_pending = 0;
    }
  }
}

}  // namespace

extern "C" {

int pmgpu_ensemble_create(pmgpu_system *const *members, int n, pmgpu_ensemble **out) {
  if (!members || !out || n < 1) return fail(PMGPU_ERR_ARG, "bad ensemble arguments");
  *out = nullptr;
  auto *e = new pmgpu_ensemble();
  struct Guard {
    pmgpu_ensemble *e;
    ~Guard() {
      if (e) pmgpu_ensemble_destroy(e);
    }
  } guard{e};
  for (int k = 0; k < n; k++) {
    if (!members[k]) return fail(PMGPU_ERR_ARG, "null ensemble member");
    System *s = reinterpret_cast<System *>(members[k]);
    for (System *q : e->m)
      if (q == s) return fail(PMGPU_ERR_ARG, "a system is in the ensemble twice");
    if (k > 0 && (s->ctx != e->m[0]->ctx || s->device != e->m[0]->device))
      return fail(PMGPU_ERR_ARG, "ensemble members must share one context");
    e->m.push_back(s);
  }
  e->device = e->m[0]->device;
  PM_CUDA(cudaSetDevice(e->device));
  // the force set of the first member is the ensemble's
  {
    PairTerms t;
    Force *pf = nullptr;
    PM_CHECK(member_shape(e->m[0], &t, &pf, e->bd_flags));
    e->terms = t.mask;
    e->pme_flags = pf ? pf->ewald_flags : 0;
  }
  e->pme_force.assign(n, nullptr);
  for (int k = 0; k < n; k++) {
    PairTerms t;
    int bd[4];
    PM_CHECK(member_shape(e->m[k], &t, &e->pme_force[k], bd));
  }
  std::vector<PairTerms> terms;
  PM_CHECK(check_shapes(e, &terms));
  for (System *s : e->m) PM_CUDA(cudaStreamSynchronize(s->stream));
  int prio_low = 0, prio_high = 0;
  PM_CUDA(cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high));
  PM_CUDA(cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking));
  PM_CUDA(cudaStreamCreateWithPriority(&e->side, cudaStreamNonBlocking, prio_high));
  PM_CUDA(cudaStreamCreateWithPriority(&e->side2, cudaStreamNonBlocking, prio_low));
  PM_CUDA(cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming));
  PM_CUDA(cudaEventCreateWithFlags(&e->ev_join, cudaEventDisableTiming));
  PM_CUDA(cudaEventCreateWithFlags(&e->ev_join2, cudaEventDisableTiming));
  e->nb = nb_batch_new();
  e->bd = bd_batch_new();
  if (e->pme_flags) {
    e->pme = pme_batch_new();
    PM_CHECK(pme_batch_build(e->pme, e->m.data(), n, e->pme_force.data()));
  }
  e->splits.assign(n, 0);
  e->seen_version.assign(n, -1);
  // rollback snapshots and the gathered results
  for (int k = 0; k < n; k++) {
    System *s = e->m[k];
    const size_t n3 = 3 * (size_t)s->n;
    if (!s->d_snap)
      PM_CHECK(dev_alloc(s, &s->d_snap, n3 * (2 * sizeof(double) + sizeof(long long))));
    double *sp = reinterpret_cast<double *>(s->d_snap);
    e->snap.add(SnapArgs{(long long)n3, s->d_pos, s->d_vel, s->d_force, sp, sp + n3,
                         reinterpret_cast<long long *>(sp + 2 * n3), s->d_step},
                (int)std::min<size_t>((n3 + 255) / 256, 64));
    e->res.add(ResArgs{s->d_acc, s->d_status}, 1);
    PM_CUDA(cudaStreamSynchronize(s->stream));
  }
  PM_CUDA(e->snap.upload());
  PM_CUDA(e->res.upload());
  PM_CUDA(cudaMalloc(&e->d_res, sizeof(long long) * (ACC_COUNT + 1) * n));
  PM_CUDA(cudaMallocHost(&e->h_res, sizeof(long long) * (ACC_COUNT + 1) * n));
  PM_CUDA(cudaMalloc(&e->d_steps0, sizeof(unsigned long long) * n));
  PM_CUDA(cudaMallocHost(&e->h_steps0, sizeof(unsigned long long) * n));
  guard.e = nullptr;
  *out = e;
  return PMGPU_OK;
}

int pmgpu_ensemble_destroy(pmgpu_ensemble *e) {
  if (!e) return PMGPU_OK;
  cudaSetDevice(e->device);
  if (e->st) cudaStreamSynchronize(e->st);
  for (auto &kv : e->graphs)
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
  if (e->pme) pme_batch_free(e->pme);
  if (e->nb) nb_batch_free(e->nb);
  if (e->bd) bd_batch_free(e->bd);
  e->snap.release();
  e->res.release();
  if (e->d_res) cudaFree(e->d_res);
  if (e->h_res) cudaFreeHost(e->h_res);
  if (e->d_steps0) cudaFree(e->d_steps0);
  if (e->h_steps0) cudaFreeHost(e->h_steps0);
  cudaEvent_t evs[] = {e->ev_fork, e->ev_join, e->ev_join2};
  for (auto ev : evs)
    if (ev) cudaEventDestroy(ev);
  cudaStream_t sts[] = {e->st, e->side, e->side2};
  for (auto q : sts)
    if (q) cudaStreamDestroy(q);
  for (System *s : e->m) {
    cudaStreamSynchronize(s->stream);
    s->graph_version++;  // the members' own graphs saw the shared PME grids
  }
  delete e;
  return PMGPU_OK;
}

int pmgpu_ensemble_run(pmgpu_ensemble *e, const pmgpu_integrator *it, long n_steps) {
  if (!e || !it) return fail(PMGPU_ERR_ARG, "null argument");
  if (!(it->timestep_fs > 0)) return fail(PMGPU_ERR_ARG, "timestep must be > 0");
  if (it->kind != PMGPU_INT_LEAPFROG && it->kind != PMGPU_INT_LANGEVIN_LEAPFROG)
    return fail(PMGPU_ERR_ARG, "unknown integrator");
  if (it->kind == PMGPU_INT_LANGEVIN_LEAPFROG && !(it->gamma_ps > 0))
    return fail(PMGPU_ERR_ARG, "LangevinLeapfrog needs gamma > 0");
  PM_CUDA(cudaSetDevice(e->device));
  e->last_kernels = e->last_replays = e->last_steps = 0;
  if (n_steps < 1) return PMGPU_OK;
  for (System *s : e->m)
    if (s->pending.active) return fail(PMGPU_ERR_STATE, "a member has a segment pending");
  PM_CHECK(ensure_forces(e));
  const int n = (int)e->m.size();
  const long long k0 = e->kernels, r0 = e->replays;
  int r = PMGPU_OK;
  for (int attempt = 0; attempt < 3; attempt++) {
    PM_CHECK(ensure_tables(e, it));
    for (int k = 0; k < n; k++) e->h_steps0[k] = e->m[k]->step;
    PM_CUDA(cudaMemcpyAsync(e->d_steps0, e->h_steps0, sizeof(unsigned long long) * n,
                            cudaMemcpyHostToDevice, e->st));
    PM_CHECK(ens_snapshot(e, attempt == 0));
    PM_CHECK(ens_segment(e, n_steps));
    int overflow = 0;
    r = ens_results(e, &overflow);
    if (!overflow) break;
    // grown lists: every member back to the segment start, every list
    // built again there (as the first segment's lists were), new tables
    r = PMGPU_ERR_OVERFLOW;
    e->nb_valid = 0;
    if (attempt < 2) {
      PM_CHECK(ens_snapshot(e, 0));
      PM_CUDA(cudaStreamSynchronize(e->st));
      for (System *s : e->m) {
        for (auto &nl : s->lists) {
          PM_CHECK(nb_prepare(s, &nl, 1));
          PM_CHECK(nb_build(s, &nl));
          s->kernels += 1;  // the tile build (nb_prepare counts its own)
        }
        PM_CUDA(cudaStreamSynchronize(s->stream));
      }
    }
  }
  mark_members(e, n_steps, r == PMGPU_OK);
  e->last_kernels = e->kernels - k0;
  e->last_replays = e->replays - r0;
  e->last_steps = n_steps;
  return r;
}

int pmgpu_ensemble_set_splits(pmgpu_ensemble *e, const int *splits) {
  if (!e || !splits) return fail(PMGPU_ERR_ARG, "null argument");
  for (size_t k = 0; k < e->m.size(); k++) {
    if (splits[k] < 0) return fail(PMGPU_ERR_ARG, "splits must be >= 0");
    e->splits[k] = splits[k];
  }
  e->nb_valid = 0;
  return PMGPU_OK;
}

int pmgpu_ensemble_time_pairs(pmgpu_ensemble *e, const int *splits, int reps, double *ms) {
  if (!e || !splits || !ms || reps < 1) return fail(PMGPU_ERR_ARG, "bad argument");
  PM_CUDA(cudaSetDevice(e->device));
  PM_CHECK(ensure_forces(e));
  if (!e->nb_valid || [&] {
        for (size_t k = 0; k < e->m.size(); k++)
          if (e->seen_version[k] != e->m[k]->graph_version) return true;
        return false;
      }()) {
    std::vector<PairTerms> terms;
    PM_CHECK(check_shapes(e, &terms));
    PM_CHECK(nb_batch_build(e->nb, e->m.data(), (int)e->m.size(), terms.data(),
                            e->splits.data()));
    e->nb_valid = 1;
    e->bd_valid = 0;
  }
  std::vector<int> sp(splits, splits + e->m.size());
  for (size_t k = 0; k < sp.size(); k++)
    if (sp[k] <= 0) sp[k] = e->splits[k];
  return nb_batch_time_jl(e->nb, e->m.data(), (int)e->m.size(), sp.data(), reps, e->st, ms);
}

int pmgpu_ensemble_get_info(pmgpu_ensemble *e, pmgpu_ensemble_info *out) {
  if (!e || !out) return fail(PMGPU_ERR_ARG, "null argument");
  out->members = (int)e->m.size();
  out->fft_buckets = e->pme ? pme_batch_buckets(e->pme) : 0;
  out->kernels = e->last_kernels;
  out->graph_replays = e->last_replays;
  out->steps = e->last_steps;
  return PMGPU_OK;
}

int pmgpu_ensemble_member(pmgpu_ensemble *e, int k, int *clusters, int *splits) {
  if (!e || !clusters || !splits || k < 0 || k >= (int)e->m.size())
    return fail(PMGPU_ERR_ARG, "bad argument");
  PM_CUDA(cudaSetDevice(e->device));
  if (!e->nb_valid) {
    PM_CHECK(ensure_forces(e));
    std::vector<PairTerms> terms;
    PM_CHECK(check_shapes(e, &terms));
    PM_CHECK(nb_batch_build(e->nb, e->m.data(), (int)e->m.size(), terms.data(),
                            e->splits.data()));
    e->nb_valid = 1;
    e->bd_valid = 0;
  }
  nb_batch_member_info(e->nb, k, splits, clusters);
  return PMGPU_OK;
}

}  // extern "C"
