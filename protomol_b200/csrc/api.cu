// The C ABI of libpmgpu (include/pmgpu.h): contexts, systems, forces,
// evaluation and device-resident integration.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "pm_device.cuh"

namespace pmgpu {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }
int fail(int code, const std::string &msg) {
  g_last_error = msg;
  return code;
}

// PeriodicBoundaryConditions::set (PeriodicBoundaryConditions.cpp:32-78),
// orthogonal boxes; the same FP64 expressions so min/max/H/D round alike.
void box_from_topology(const pmgpu_topology *t, Box *b) {
  std::memset(b, 0, sizeof(*b));
  b->periodic = t->periodic;
  if (!t->periodic) return;
  const double *e1 = t->box, *e2 = t->box + 3, *e3 = t->box + 6, *o = t->box + 9;
  auto cross = [](const double *a, const double *c, double *r) {
    r[0] = a[1] * c[2] - a[2] * c[1];
    r[1] = a[2] * c[0] - a[0] * c[2];
    r[2] = a[0] * c[1] - a[1] * c[0];
  };
  auto dot = [](const double *a, const double *c) {
    return a[0] * c[0] + a[1] * c[1] + a[2] * c[2];
  };
  double a1[3], a2[3], a3[3], tt[3];
  cross(e1, e2, tt);
  b->V = std::fabs(dot(tt, e3));
  cross(e2, e3, a1);
  cross(e3, e1, a2);
  cross(e1, e2, a3);
  double d1 = dot(e1, a1), d2 = dot(e2, a2), d3 = dot(e3, a3);
  b->er[0] = a1[0] / d1;
  b->er[1] = a2[1] / d2;
  b->er[2] = a3[2] / d3;
  b->e[0] = e1[0];
  b->e[1] = e2[1];
  b->e[2] = e3[2];
  for (int c = 0; c < 3; c++) {
    double sum = (e1[c] + e2[c]) + e3[c];
    double lo = o[c] - sum * 0.5, hi = o[c] + sum * 0.5;
    b->min[c] = std::min(lo, hi);
    b->max[c] = std::max(lo, hi);
    b->origin[c] = o[c];
  }
  double dx = (e1[0] * 0.5) * (e1[0] * 0.5);
  double dy = (e2[1] * 0.5) * (e2[1] * 0.5);
  double dz = (e3[2] * 0.5) * (e3[2] * 0.5);
  b->D = std::min(dx, std::min(dy, dz));
  for (int c = 0; c < 3; c++) {
    b->H[c] = b->max[c] - b->min[c];
    b->H2[c] = b->H[c] * 0.5;
  }
}

// Switching-function constants exactly as the ProtoMol constructors form
// them (C1SwitchingFunction.cpp:12-17, C2SwitchingFunction.cpp:12-19,
// CnSwitchingFunction.cpp:41-60, CmpCnCnSwitchingFunction.cpp:11-25); a
// complement keeps its function's constants and drops the rough test
// (ComplementSwitchingFunction.h:35-41).
void switch_setup(const pmgpu_switch *in, SwitchParams *o) {
  std::memset(o, 0, sizeof(*o));
  o->kind = in->kind & ~PMGPU_SW_COMPLEMENT;
  double rc = in->cutoff, rs = in->switchon;
  switch (o->kind) {
    case PMGPU_SW_UNIVERSAL:
      o->cutoff = 1e300;
      o->cutoff2 = 1e300;
      break;
    case PMGPU_SW_CUTOFF:
      o->cutoff = rc;
      o->cutoff2 = rc * rc;
      break;
    case PMGPU_SW_C1:
      o->modify = 1;
      o->cutoff = rc;
      o->cutoff2 = rc * rc;
      o->c1a = 1.5 / rc;
      o->c1b = 0.5 / (rc * rc * rc);
      o->c1c = 1.5 / (rc * rc * rc);
      break;
    case PMGPU_SW_C2: {
      o->modify = 1;
      double d = rc * rc - rs * rs;
      o->cutoff = rc;
      o->cutoff2 = rc * rc;
      o->switchon2 = rs * rs;
      o->s1 = 1.0 / (d * d * d);
      o->s2 = rc * rc - 3.0 * rs * rs;
      o->s3 = 4.0 / (d * d * d);
      break;
    }
    case PMGPU_SW_CN: {
      o->modify = 1;
      double mycut = in->switchoff != 0.0 ? in->switchoff : rc;
      o->cutoff = mycut;
      o->cutoff2 = mycut * mycut;
      o->switchon2 = rs * rs;
      o->ord_int = (int)in->order;
      o->ord_idx = o->ord_int - 2;
      if (o->ord_int == 5) o->ord_int = 2;
      o->irange[0] = std::pow(rs - rc, -(o->ord_int + 1));
      for (int i = 1; i < o->ord_int + 1 && i < 8; i++)
        o->irange[i] = o->irange[i - 1] / (rs - rc);
      break;
    }
    case PMGPU_SW_CMPCNCN: {
      o->modify = 1;
      const double so = in->switchoff;
      double ord = in->order;
      if (ord == 5.0) ord = 2.0;  // remapped before the table index is taken
      o->cutoff = rc;
      o->cutoff2 = rc * rc;
      o->switchon2 = rs * rs;
      o->compoff = so;
      o->compoff2 = so * so;
      o->ord_int = (int)ord;
      o->ord_idx = o->ord_int - 2;
      o->irange[0] = 1.0 / std::pow(rs - so, o->ord_int + 1);
      o->itrange[0] = 1.0 / std::pow(so - rc, o->ord_int + 1);
      for (int i = 1; i < o->ord_int + 1 && i < 8; i++) {
        o->irange[i] = o->irange[i - 1] / (rs - so);
        o->itrange[i] = o->itrange[i - 1] / (so - rc);
      }
      break;
    }
  }
  o->rough2 = o->cutoff2;
  if (in->kind & PMGPU_SW_COMPLEMENT) {
    o->modify = 1;
    o->complement = 1;
    o->rough2 = 1e300;  // Constant::MAXREAL
  }
}

static int validate_switch(const pmgpu_switch *sw, const char *what) {
  if (!sw) return PMGPU_OK;
  std::string w(what);
  if (sw->kind & PMGPU_SW_COMPLEMENT)
    return fail(PMGPU_ERR_ARG, w + ": a Complement switch belongs to the all-pairs path");
  switch (sw->kind) {
    case PMGPU_SW_CUTOFF:
    case PMGPU_SW_C1:
      if (!(sw->cutoff > 0)) return fail(PMGPU_ERR_ARG, w + ": cutoff must be > 0");
      return PMGPU_OK;
    case PMGPU_SW_C2:
      // C2SwitchingFunction::make (C2SwitchingFunction.cpp:33-44)
      if (!(sw->switchon >= 0 && sw->cutoff > 0 && sw->switchon < sw->cutoff))
        return fail(PMGPU_ERR_ARG, w + ": C2 needs 0 <= switchon < cutoff");
      return PMGPU_OK;
    case PMGPU_SW_CN:
      // CnSwitchingFunction::make (CnSwitchingFunction.cpp:83-110)
      if (!(sw->switchon >= 0 && sw->cutoff > 0 && sw->switchon < sw->cutoff) ||
          (sw->switchoff > 0 && sw->switchoff != sw->cutoff) || sw->order < 2 ||
          sw->order > 6)
        return fail(PMGPU_ERR_ARG, w + ": Cn needs 0 <= switchon < cutoff, order 2..6");
      return PMGPU_OK;
    case PMGPU_SW_CMPCNCN:
      // CmpCnCnSwitchingFunction::make (CmpCnCnSwitchingFunction.cpp:47-63)
      if (!(sw->switchon >= 0 && sw->cutoff > 0 && sw->switchoff > 0 &&
            sw->switchon < sw->switchoff && sw->switchoff <= sw->cutoff) ||
          sw->order < 2 || sw->order > 6)
        return fail(PMGPU_ERR_ARG, w + ": CmpCnCn needs 0 <= switchon < switchoff <= cutoff, "
                                       "order 2..6");
      return PMGPU_OK;
    case PMGPU_SW_UNIVERSAL:
      return fail(PMGPU_ERR_ARG, w + ": a cutoff force needs a cutoff switching function");
    default:
      return fail(PMGPU_ERR_ARG, w + ": unknown switching function");
  }
}

int dev_alloc(System *s, void **p, size_t bytes) {
  cudaError_t e = cudaMallocAsync(p, std::max<size_t>(bytes, 1), s->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return fail(e == cudaErrorMemoryAllocation ? PMGPU_ERR_OOM : PMGPU_ERR_CUDA,
                std::string("device allocation of ") + std::to_string(bytes) +
                    " bytes: " + cudaGetErrorString(e));
  }
  return PMGPU_OK;
}

void dev_free(System *s, void *p) {
  if (p) cudaFreeAsync(p, s->stream);
}

// Allocates count elements on the system's stream and fills them from h
// (or with zeros).
template <typename T>
static int upload(System *s, T **d, const T *h, size_t count) {
  if (count == 0) count = 1;
  PM_CHECK(dev_alloc(s, d, sizeof(T) * count));
  if (h) PM_CUDA(cudaMemcpyAsync(*d, h, sizeof(T) * count, cudaMemcpyHostToDevice, s->stream));
  else PM_CUDA(cudaMemsetAsync(*d, 0, sizeof(T) * count, s->stream));
  return PMGPU_OK;
}

// ProtoMol fills its LJ table from per-type (epsilon, rmin/2) by the CHARMM
// rule (topology/BuildTopology.cpp:662-672): r = s_i + s_j,
// e = sqrt(e_i e_j), A = e r^12, B = 2 e r^6.  When every normal (A, B)
// entry follows that rule to 1e-10 relative, *out receives the per-type
// (sqrt(e), s) and the FP32 all-pairs kernel computes A and B instead of
// reading the ntypes^2 table.  The 1-4 entries are always read from the
// table.
static bool lj_charmm_rule(const double *lj, int nt, std::vector<float2> *out) {
  if (nt <= 0 || !lj) return false;
  std::vector<double> se(nt), sh(nt);
  for (int t = 0; t < nt; t++) {
    const double A = lj[4 * ((size_t)t * nt + t)], B = lj[4 * ((size_t)t * nt + t) + 1];
    if (A == 0 && B == 0) {
      se[t] = 0;
      sh[t] = 0;
      continue;
    }
    if (!(A > 0 && B > 0)) return false;
    // diagonal: (2 s)^6 = 2 A / B and e = B^2 / (4 A)
    sh[t] = 0.5 * std::pow(2 * A / B, 1.0 / 6.0);
    se[t] = std::sqrt(B * B / (4 * A));
  }
  auto close = [](double got, double want) {
    return std::fabs(got - want) <= 1e-10 * std::max(std::fabs(want), 1e-300);
  };
  for (int t1 = 0; t1 < nt; t1++)
    for (int t2 = 0; t2 < nt; t2++) {
      const double *p = lj + 4 * ((size_t)t1 * nt + t2);
      const double r = sh[t1] + sh[t2], e = se[t1] * se[t2];
      const double r6 = r * r * r * r * r * r;
      if (!close(p[0], e * r6 * r6) || !close(p[1], 2 * e * r6)) return false;
    }
  out->resize(nt);
  for (int t = 0; t < nt; t++) (*out)[t] = make_float2((float)se[t], (float)sh[t]);
  return true;
}

static int system_free(System *s) {
  cudaSetDevice(s->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  for (auto &f : s->forces) pme_free(s, &f);
  for (auto &nl : s->lists) nb_list_free(s, &nl);
  void *ptrs[] = {s->d_charge, s->d_mass, s->d_type, s->d_mol, s->d_lj32, s->d_ljab,
                  s->d_ljcomb, s->d_lj64,
                  s->d_excl_start, s->d_excl_partner, s->d_excl_class, s->d_excl_pairs,
                  s->d_excl_range,
                  s->d_bond_atoms, s->d_angle_atoms, s->d_bond_params, s->d_angle_params,
                  s->d_dihedral_atoms, s->d_dihedral_params, s->d_improper_atoms,
                  s->d_improper_params,
                  s->d_gb_vdwr, s->d_gb_scale, s->d_gb_offset, s->d_water, s->d_gb_born,
                  s->d_gb_psi, s->d_gb_partial, s->d_gb_fixed, s->d_gb_ace, s->d_pos, s->d_vel,
                  s->d_force, s->d_acc, s->d_status, s->d_pairbuf, s->d_paircount,
                  s->d_stage, s->d_snap, s->d_step, s->d_sf_tile, s->d_gb_gst, s->d_gb_grad,
                  s->d_rec, s->d_scp, s->d_scp_i, s->d_born_q,
                  s->d_sf_bits};
  for (auto &g : s->graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  for (void *p : ptrs) dev_free(s, p);
  if (s->stream) cudaStreamSynchronize(s->stream);
  if (s->h_acc) cudaFreeHost(s->h_acc);
  if (s->h_status) cudaFreeHost(s->h_status);
  if (s->h_stage) cudaFreeHost(s->h_stage);
  prof_collect(s);
  for (cudaEvent_t e : s->prof.pool) cudaEventDestroy(e);
  s->prof.pool.clear();
  if (s->side) cudaStreamSynchronize(s->side);
  if (s->ev_fork) cudaEventDestroy(s->ev_fork);
  if (s->side2) cudaStreamSynchronize(s->side2);
  if (s->ev_join) cudaEventDestroy(s->ev_join);
  if (s->ev_join2) cudaEventDestroy(s->ev_join2);
  if (s->side) cudaStreamDestroy(s->side);
  if (s->side2) cudaStreamDestroy(s->side2);
  if (s->stream) cudaStreamDestroy(s->stream);
  return PMGPU_OK;
}

// ------------------------------------------------------------- profiling
static cudaEvent_t prof_event(System *s) {
  Profiler &p = s->prof;
  if (!p.pool.empty()) {
    cudaEvent_t e = p.pool.back();
    p.pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

void prof_begin(System *s, int phase) {
  Profiler &p = s->prof;
  if (!p.enabled) return;
  p.open_phase = phase;
  p.open_ev = prof_event(s);
  cudaEventRecord(p.open_ev, s->stream);
}

void prof_end(System *s) {
  Profiler &p = s->prof;
  if (!p.enabled || p.open_phase < 0) return;
  cudaEvent_t b = prof_event(s);
  cudaEventRecord(b, s->stream);
  p.pending.push_back({p.open_phase, p.open_ev, b});
  p.open_phase = -1;
  // bound the number of outstanding events on long segments
  if (p.pending.size() > 4096) prof_collect(s);
}

void prof_collect(System *s) {
  Profiler &p = s->prof;
  for (auto &m : p.pending) {
    float t = 0.f;
    if (cudaEventSynchronize(m.b) == cudaSuccess && cudaEventElapsedTime(&t, m.a, m.b) == cudaSuccess) {
      p.ms[m.phase] += t;
      p.launches[m.phase] += 1;
    }
    p.pool.push_back(m.a);
    p.pool.push_back(m.b);
  }
  p.pending.clear();
}

// ------------------------------------------------------------ evaluation
struct Launch {
  int list;
  PairTerms terms;
};

static int add_pair_terms(std::vector<Launch> &groups, int list, const PairTerms &t) {
  for (auto &g : groups) {
    if (g.list != list || (g.terms.mask & t.mask)) continue;
    // a lattice sum's cutoff terms (every image) and NonbondedCutoff's
    // (minimal image only) take separate launches
    const bool g_lc = g.terms.mask & (TERM_LJ | TERM_COUL);
    const bool t_lc = t.mask & (TERM_LJ | TERM_COUL);
    if (g_lc && t_lc && g.terms.minimal_image != t.minimal_image) continue;
    if (t.mask & TERM_LJ) {
      g.terms.lj_sw = t.lj_sw;
      g.terms.lj_cut2 = t.lj_cut2;
    }
    if (t.mask & TERM_COUL) {
      g.terms.coul_sw = t.coul_sw;
      g.terms.coul_cut2 = t.coul_cut2;
    }
    if (t.mask & TERM_EWALD) {
      g.terms.ewtab = t.ewtab;
      g.terms.ewald_alpha = t.ewald_alpha;
      g.terms.ewald_rc2 = t.ewald_rc2;
      g.terms.exact_erf = t.exact_erf;
    }
    g.terms.mask |= t.mask;
    if (t_lc) g.terms.minimal_image = t.minimal_image;  // the rule applies to LJ / Coulomb only
    return 0;
  }
  groups.push_back({list, t});
  return 0;
}

// The pair-kernel groups of an evaluation of all enabled forces: the
// (list, merged terms) of each pair-kernel launch.
void pair_groups(System *s, std::vector<std::pair<int, PairTerms>> *out) {
  std::vector<Launch> groups;
  for (auto &f : s->forces) {
    if (!f.enabled) continue;
    if (f.kind == FK_CUTOFF || (f.kind == FK_PME && (f.ewald_flags & PMGPU_EWALD_REAL)))
      add_pair_terms(groups, f.list_index, f.terms);
  }
  out->clear();
  for (auto &g : groups) out->push_back({g.list, g.terms});
}

// Evaluates the enabled forces (or only force `only`) at the resident
// positions, accumulating into the (already zeroed) force planes and
// energy accumulators.  fold = 0 (the force-only steps of an MD run) lets
// the pair forces stay in the list's slot buffer for the next update kernel.
int evaluate_forces(System *s, int only, int mode, int fold) {
  const int want_virial = mode == PAIR_VIRIAL;
  // energy mode of the non-pair terms: 0 forces only (inner MD steps),
  // 1 + energies, 2 + energies and virial
  const int em = mode == PAIR_FORCE ? 0 : (want_virial ? 2 : 1);
  std::vector<Launch> groups;
  std::vector<int> prepared(s->lists.size(), 0);
  int sf_lj = 0, sf_coul = 0, sf_done = 0;
  for (auto &f : s->forces)
    if (f.kind == FK_SIMPLEFULL && f.enabled) {
      sf_lj |= f.sf_lj;
      sf_coul |= f.sf_coul;
    }
  int bd_bonds = 0, bd_angles = 0, bd_dihedrals = 0, bd_impropers = 0, bd_done = 0;
  for (auto &f : s->forces) {
    if (only >= 0 ? f.id != only : !f.enabled) continue;
    if (f.kind == FK_BONDED) {
      bd_bonds |= f.bonds;
      bd_angles |= f.angles;
    } else if (f.kind == FK_TORSION) {
      bd_dihedrals |= f.dihedrals;
      bd_impropers |= f.impropers;
    }
  }
  for (auto &f : s->forces) {
    if (only >= 0 ? f.id != only : !f.enabled) continue;
    if (f.kind == FK_CUTOFF || (f.kind == FK_PME && (f.ewald_flags & PMGPU_EWALD_REAL)))
      add_pair_terms(groups, f.list_index, f.terms);
  }
  // Terms other than the pair kernels (bonded, GB, all-pairs, PME,
  // corrections) only read the positions and add into the fixed-point
  // forces and energies, so they run on the system's second stream beside
  // the list work and the pair kernels, and join before the evaluation ends
  // (not while profiling, which times phases in order).  They start at
  // once, while the list work of the step leaves most of the device idle.
  // The second stream has the higher priority, so its short dependent
  // kernels are not queued behind the pair kernel's blocks.  The PME chain
  // is the longest of them, so the other short terms (bonded, Ewald
  // correction) take a third stream and PME starts at once.
  // the all-pairs passes read the FP32 pair records of the positions,
  // written by this step's update kernel or here
  bool need_rec = false;
  for (auto &f : s->forces) {
    if (only >= 0 ? f.id != only : !f.enabled) continue;
    need_rec |= f.kind == FK_SIMPLEFULL || f.kind == FK_GB || f.kind == FK_GBACE;
  }
  if (need_rec && s->precision == PMGPU_PREC_MIXED && !s->rec_fresh) {
    PM_CHECK(nb_stage_pairs(s));
    s->kernels += s->n > 0;
  }
  s->rec_fresh = 0;
  const bool fork = s->side && !s->prof.enabled;
  const cudaStream_t main_stream = s->stream;
  if (fork) {
    PM_CUDA(cudaEventRecord(s->ev_fork, main_stream));
    PM_CUDA(cudaStreamWaitEvent(s->side, s->ev_fork, 0));
    PM_CUDA(cudaStreamWaitEvent(s->side2, s->ev_fork, 0));
  }
  struct Join {  // back on the main stream, joined, on every exit path
    System *s;
    cudaStream_t main_stream;
    bool on;
    ~Join() {
      s->stream = main_stream;
      // a rebuild decision taken by an update kernel holds for this
      // evaluation only
      for (auto &nl : s->lists) nl.decided = 0;
      if (!on) return;
      cudaEventRecord(s->ev_join, s->side);
      cudaStreamWaitEvent(main_stream, s->ev_join, 0);
      cudaEventRecord(s->ev_join2, s->side2);
      cudaStreamWaitEvent(main_stream, s->ev_join2, 0);
    }
  } join{s, main_stream, fork};
  {
    // GB's passes and the PME chain are long dependent chains and take the
    // second stream; the all-pairs terms go beside them on the main stream,
    // and so do the bonded terms when the main stream has no list work;
    // otherwise the bonded terms and the Ewald correction take the third
    const bool main_idle = s->lists.empty();
    const cudaStream_t short_stream = main_idle ? main_stream : s->side2;
    for (auto &f : s->forces) {
      if (only >= 0 ? f.id != only : !f.enabled) continue;
      if (fork)
        s->stream = f.kind == FK_SIMPLEFULL ? main_stream
                    : f.kind == FK_GB || f.kind == FK_GBACE || f.kind == FK_PME ? s->side
                                                           : short_stream;
      int r = PMGPU_OK;
      switch (f.kind) {
        case FK_PME:
          if (f.ewald_flags & PMGPU_EWALD_CORRECTION) {
            if (fork) s->stream = short_stream;
            prof_begin(s, PMGPU_PHASE_CORRECTION);
            r = ewald_correction(s, &f, em);
            prof_end(s);
            PM_CHECK(r);
            s->kernels += s->n_excl > 0;
            if (fork) s->stream = s->side;
          }
          if (f.ewald_flags & PMGPU_EWALD_RECIPROCAL) {
            prof_begin(s, PMGPU_PHASE_PME);
            r = pme_reciprocal(s, &f, em);
            prof_end(s);
            PM_CHECK(r);
            s->kernels += 4;  // spread, fixed->float, convolve, gather (+ cuFFT)
          }
          break;
        case FK_GB:
        case FK_GBACE: {
          // GBForce and GBACEForce of one evaluation share one chain of
          // passes (the Born radii once), launched at the first of them
          const Force *gb = nullptr, *ace = nullptr;
          for (auto &g : s->forces) {
            if (only >= 0 ? g.id != only : !g.enabled) continue;
            if (g.kind == FK_GB && !gb) gb = &g;
            if (g.kind == FK_GBACE && !ace) ace = &g;
          }
          if (&f != (gb ? gb : ace)) break;
          prof_begin(s, PMGPU_PHASE_GB);
          r = gb_forces(s, gb, ace);
          prof_end(s);
          s->kernels += (s->precision == PMGPU_PREC_MIXED ? 3 : 4) + (gb ? 1 : 0);
          break;
        }
        case FK_BONDED:
        case FK_TORSION: {
          // the bonded terms of every selected force share one launch
          if (bd_done) break;
          bd_done = 1;
          int launched = 0;
          prof_begin(s, PMGPU_PHASE_BONDED);
          r = bonded_all(s, bd_bonds, bd_angles, bd_dihedrals, bd_impropers, em, &launched);
          prof_end(s);
          s->kernels += launched;
          break;
        }
        case FK_SCPISM:
          prof_begin(s, PMGPU_PHASE_SIMPLEFULL);
          r = nb_simplefull_sw(s, (f.terms.mask & TERM_LJ) ? &f.terms.lj_sw : nullptr,
                               &f.terms.coul_sw, em, 1, f.scp_D);
          prof_end(s);
          s->kernels += 1;
          break;
        case FK_BORN:
          prof_begin(s, PMGPU_PHASE_SIMPLEFULL);
          r = nb_born(s, f, em);
          prof_end(s);
          s->kernels += 2;
          break;
        case FK_SIMPLEFULL_SW:
          prof_begin(s, PMGPU_PHASE_SIMPLEFULL);
          r = nb_simplefull_sw(s, (f.terms.mask & TERM_LJ) ? &f.terms.lj_sw : nullptr,
                               (f.terms.mask & TERM_COUL) ? &f.terms.coul_sw : nullptr, em);
          prof_end(s);
          s->kernels += 1;
          break;
        case FK_SIMPLEFULL:
          // all enabled simple-full terms share one all-pairs pass
          if (sf_done) break;
          sf_done = 1;
          prof_begin(s, PMGPU_PHASE_SIMPLEFULL);
          r = nb_simplefull(s, only >= 0 ? f.sf_lj : sf_lj, only >= 0 ? f.sf_coul : sf_coul,
                            em);
          prof_end(s);
          s->kernels += 1;
          break;
        default:
          break;
      }
      PM_CHECK(r);
    }
    s->stream = main_stream;
  }
  // neighbour lists are prepared once per evaluation: the rebuild decision,
  // the (conditional) sort and the per-step gather, then the (conditional)
  // tile build
  for (auto &f : s->forces) {
    if (only >= 0 ? f.id != only : !f.enabled) continue;
    if (f.list_index >= 0 && !prepared[f.list_index]) {
      prof_begin(s, PMGPU_PHASE_LIST);
      int r = nb_prepare(s, &s->lists[f.list_index], 0);
      prof_end(s);
      PM_CHECK(r);  // nb_prepare counts its launches
      prepared[f.list_index] = 1;
    }
  }
  for (size_t k = 0; k < prepared.size(); k++) {
    if (!prepared[k]) continue;
    prof_begin(s, PMGPU_PHASE_LIST);
    int r = nb_build(s, &s->lists[k]);
    prof_end(s);
    PM_CHECK(r);
    s->kernels += 1;  // tiles
  }
  for (auto &g : groups) {
    prof_begin(s, PMGPU_PHASE_PAIRS);
    int r = nb_pair_forces(s, &s->lists[g.list], g.terms, mode, fold);
    prof_end(s);
    PM_CHECK(r);
    s->kernels += 2;  // tiles, slot forces
  }
  return PMGPU_OK;
}

// Constant energy terms (Ewald point self energy and charged-system term,
// NonbondedFullEwaldSystemForce.h:344-353, :694-714) for the selected forces.
static void constant_terms(System *s, int only, double *energies, double *virial) {
  for (auto &f : s->forces) {
    if (only >= 0 ? f.id != only : !f.enabled) continue;
    if (f.kind == FK_PME && (f.ewald_flags & PMGPU_EWALD_CORRECTION)) {
      if (energies) energies[PMGPU_E_COULOMB] += f.self_energy + f.charged_energy;
      if (virial) {
        virial[0] += f.charged_energy;
        virial[4] += f.charged_energy;
        virial[8] += f.charged_energy;
      }
    }
  }
}

// energies_valid = 0: a force-only evaluation, whose energies and virial
// were not computed (recorded as zeros).
int read_results(System *s, int only, double *energies, double *virial, int add,
                 int energies_valid) {
  PM_CUDA(cudaMemcpyAsync(s->h_acc, s->d_acc, sizeof(long long) * ACC_COUNT,
                          cudaMemcpyDeviceToHost, s->stream));
  PM_CUDA(cudaMemcpyAsync(s->h_status, s->d_status, sizeof(int), cudaMemcpyDeviceToHost,
                          s->stream));
  PM_CUDA(cudaStreamSynchronize(s->stream));
  prof_collect(s);
  return take_results(s, only, energies, virial, add, energies_valid);
}

int take_results(System *s, int only, double *energies, double *virial, int add,
                 int energies_valid) {
  int st = *s->h_status;
  if (st) {
    PM_CUDA(cudaMemsetAsync(s->d_status, 0, sizeof(int), s->stream));
    if (st & ST_LIST_OVERFLOW) {
      // Grow every list to at least its largest row's need, and its column
      // buckets to the fullest column's count (fresh build next time); this
      // result is incomplete and no output is touched.
      for (auto &nl : s->lists) {
        int rb[4] = {0, 0, 0, 0};
        PM_CUDA(cudaMemcpyAsync(rb, nl.d_rebuild, sizeof(rb), cudaMemcpyDeviceToHost, s->stream));
        PM_CUDA(cudaStreamSynchronize(s->stream));
        const int need = rb[2] + rb[2] / 4 + 32;
        // a column overflow alone leaves the tile capacity as it is
        const int cap = rb[3] > 0 && rb[2] == 0 ? nl.cap : (std::max(nl.cap * 2, need) + 31) & ~31;
        if (rb[3] > 0) nl.bcap = std::max(nl.bcap, rb[3] + rb[3] / 4 + 32);
        nb_list_free(s, &nl);
        nl.cap = cap;
        nl.cap_set = 0;
        nl.bcap_set = 0;
        nl.limit = 0;
        PM_CHECK(nb_list_init(s, &nl, nl.cutoff, nl.skin, 0));
        s->graph_version++;  // captured graphs hold the old list buffers
      }
      return fail(PMGPU_ERR_OVERFLOW, "neighbour list capacity exceeded; capacity grown");
    }
    if (st & ST_NONFINITE) return fail(PMGPU_ERR_NAN, "non-finite position or force");
    if (st & ST_CELL_OVERFLOW)
      return fail(PMGPU_ERR_UNSUPPORTED, "more atoms in one pair-list column than the sort holds");
  }
  double e[PMGPU_E_COUNT], v[9];
  for (int k = 0; k < PMGPU_E_COUNT; k++) e[k] = (double)s->h_acc[k] / kEnergyScale;
  for (int k = 0; k < 9; k++) v[k] = (double)s->h_acc[ACC_VIRIAL + k] / kEnergyScale;
  if (energies_valid) constant_terms(s, only, e, v);
  else
    for (int k = 0; k < PMGPU_E_COUNT; k++) e[k] = 0.0;
  if (!energies_valid)
    for (int k = 0; k < 9; k++) v[k] = 0.0;
  s->last_pairs = s->h_acc[ACC_PAIRS];
  for (int k = 0; k < PMGPU_E_COUNT; k++) s->last_energy[k] = e[k];
  for (int k = 0; k < 9; k++) s->last_virial[k] = v[k];
  if (energies)
    for (int k = 0; k < PMGPU_E_COUNT; k++) energies[k] = add ? energies[k] + e[k] : e[k];
  if (virial)
    for (int k = 0; k < 9; k++) virial[k] = add ? virial[k] + v[k] : v[k];
  return PMGPU_OK;
}

// Runs fn() and, when a neighbour list overflowed (capacities are then
// doubled by read_results), runs it again; at most three attempts.
template <typename Fn>
static int with_overflow_retry(Fn fn) {
  int r = PMGPU_OK;
  for (int attempt = 0; attempt < 3; attempt++) {
    r = fn();
    if (r != PMGPU_ERR_OVERFLOW) return r;
  }
  return r;
}

// FP32 FMA throughput: every thread advances 8 independent FMA chains (no
// dependence between them, so the pipes stay full); the result is stored
// only under a condition that never holds, so nothing is optimised away.
constexpr int kPeakChains = 8;
__global__ void __launch_bounds__(256) k_fma_peak(int iters, float a, float b, float *sink) {
  float v[kPeakChains];
#pragma unroll
  for (int c = 0; c < kPeakChains; c++) v[c] = (float)(threadIdx.x + c);
  for (int k = 0; k < iters; k++) {
#pragma unroll
    for (int c = 0; c < kPeakChains; c++) v[c] = fmaf(v[c], a, b);
  }
  float t = 0.f;
#pragma unroll
  for (int c = 0; c < kPeakChains; c++) t += v[c];
  if (t == -1.2345f) sink[0] = t;
}

static int fp32_peak(int device, double *tflops) {
  PM_CUDA(cudaSetDevice(device));
  int sms = 148;
  PM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  float *sink = nullptr;
  PM_CUDA(cudaMalloc(&sink, sizeof(float)));
  cudaEvent_t e0, e1;
  PM_CUDA(cudaEventCreate(&e0));
  PM_CUDA(cudaEventCreate(&e1));
  const int blocks = sms * 8, iters = 4096;
  double best = 0.0;
  for (int rep = 0; rep < 4; rep++) {  // the first launch warms up
    PM_CUDA(cudaEventRecord(e0));
    k_fma_peak<<<blocks, 256>>>(iters, 0.999f, 1e-3f, sink);
    PM_CUDA(cudaEventRecord(e1));
    PM_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    PM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    const double flops = 2.0 * kPeakChains * (double)iters * blocks * 256;
    if (rep > 0 && ms > 0.f) best = std::max(best, flops / (ms * 1e-3) / 1e12);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  *tflops = best;
  return PMGPU_OK;
}

int begin_eval(System *s) {
  PM_CUDA(cudaMemsetAsync(s->d_acc, 0, sizeof(long long) * ACC_COUNT, s->stream));
  return PMGPU_OK;
}

}  // namespace pmgpu

using namespace pmgpu;

// ===================================================================== ABI
extern "C" {

static int run_finish(System *s);

const char *pmgpu_last_error(void) { return g_last_error.c_str(); }
int pmgpu_abi_version(void) { return PMGPU_ABI_VERSION; }

int pmgpu_context_create(int device, pmgpu_context **out) {
  if (!out) return fail(PMGPU_ERR_ARG, "null output pointer");
  int count = 0;
  PM_CUDA(cudaGetDeviceCount(&count));
  if (device < 0 || device >= count) return fail(PMGPU_ERR_ARG, "no such CUDA device");
  PM_CUDA(cudaSetDevice(device));
  cudaDeviceProp prop;
  PM_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10)
    return fail(PMGPU_ERR_UNSUPPORTED, "libpmgpu is built for sm_100a (Blackwell B200)");
  // Stream-ordered allocations of freed systems stay in this process's
  // default pool for the next system instead of going back to the driver.
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  auto *c = new pmgpu_context();
  c->device = device;
  *out = c;
  return PMGPU_OK;
}

int pmgpu_context_destroy(pmgpu_context *ctx) {
  if (!ctx) return PMGPU_OK;
  cudaSetDevice(ctx->device);
  for (auto &p : ctx->fft_free) {
    cufftDestroy(p.r2c);
    cufftDestroy(p.c2r);
  }
  delete ctx;
  return PMGPU_OK;
}

int pmgpu_system_create(pmgpu_context *ctx, const pmgpu_topology *t, int precision,
                        pmgpu_system **out) {
  if (!ctx || !t || !out) return fail(PMGPU_ERR_ARG, "null argument");
  if (t->n_atoms < 0 || t->n_atoms >= kMaxAtoms)
    return fail(PMGPU_ERR_ARG, "atom count out of range (0 .. 2^24-1)");
  if (precision != PMGPU_PREC_MIXED && precision != PMGPU_PREC_DOUBLE)
    return fail(PMGPU_ERR_ARG, "precision must be PMGPU_PREC_MIXED or PMGPU_PREC_DOUBLE");
  int n = t->n_atoms;
  if (n > 0 && (!t->charge || !t->mass || !t->type || !t->molecule))
    return fail(PMGPU_ERR_ARG, "charge, mass, type and molecule arrays are required");
  if (t->n_types < 1 || !t->lj) return fail(PMGPU_ERR_ARG, "LJ table required (n_types >= 1)");
  for (int i = 0; i < n; i++)
    if (t->type[i] < 0 || t->type[i] >= t->n_types)
      return fail(PMGPU_ERR_ARG, "atom type index out of range");
  if (t->periodic) {
    const double *b = t->box;
    if (b[1] != 0 || b[2] != 0 || b[3] != 0 || b[5] != 0 || b[6] != 0 || b[7] != 0)
      return fail(PMGPU_ERR_UNSUPPORTED, "only orthogonal periodic boxes are supported");
    if (!(b[0] > 0 && b[4] > 0 && b[8] > 0))
      return fail(PMGPU_ERR_ARG, "box edges must be positive");
  }
  PM_CUDA(cudaSetDevice(ctx->device));
  std::unique_ptr<System> s(new System());
  s->ctx = ctx;
  s->device = ctx->device;
  s->n = n;
  s->precision = precision;
  box_from_topology(t, &s->box);
  s->ntypes = t->n_types;
  s->coulomb_scaling = t->coulomb_scaling;
  PM_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
  int prio_low = 0, prio_high = 0;
  PM_CUDA(cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high));
  PM_CUDA(cudaStreamCreateWithPriority(&s->side, cudaStreamNonBlocking, prio_high));
  PM_CUDA(cudaStreamCreateWithPriority(&s->side2, cudaStreamNonBlocking, prio_low));
  PM_CUDA(cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming));
  PM_CUDA(cudaEventCreateWithFlags(&s->ev_join, cudaEventDisableTiming));
  PM_CUDA(cudaEventCreateWithFlags(&s->ev_join2, cudaEventDisableTiming));
  size_t nn = std::max(1, n);
  PM_CHECK(upload(s.get(), &s->d_charge, t->charge, n));
  PM_CHECK(upload(s.get(), &s->d_mass, t->mass, n));
  PM_CHECK(upload(s.get(), &s->d_type, t->type, n));
  PM_CHECK(upload(s.get(), &s->d_mol, t->molecule, n));
  int nt2 = t->n_types * t->n_types;
  std::vector<float4> lj32(nt2);
  std::vector<double4> lj64(nt2);
  for (int k = 0; k < nt2; k++) {
    const double *p = t->lj + 4 * k;
    lj32[k] = make_float4((float)p[0], (float)p[1], (float)p[2], (float)p[3]);
    lj64[k] = make_double4(p[0], p[1], p[2], p[3]);
  }
  PM_CHECK(upload(s.get(), &s->d_lj32, lj32.data(), nt2));
  std::vector<float2> comb;
  if (lj_charmm_rule(t->lj, t->n_types, &comb)) {
    PM_CHECK(upload(s.get(), &s->d_ljcomb, comb.data(), comb.size()));
  } else {
    // A, B stored by column: a warp whose lanes hold consecutive types of
    // one atom reads the entries of a partner type as one coalesced row
    std::vector<float2> ljab(nt2);
    const int nt = t->n_types;
    for (int t1 = 0; t1 < nt; t1++)
      for (int t2 = 0; t2 < nt; t2++)
        ljab[(size_t)t2 * nt + t1] = make_float2(lj32[(size_t)t1 * nt + t2].x,
                                                 lj32[(size_t)t1 * nt + t2].y);
    PM_CHECK(upload(s.get(), &s->d_ljab, ljab.data(), nt2));
  }
  PM_CHECK(upload(s.get(), &s->d_lj64, lj64.data(), nt2));
  // exclusion table as CSR over both atoms of each pair
  int ne = std::max(0, t->n_exclusions);
  std::vector<int> start(n + 1, 0), partner(2 * (size_t)ne + 1), cls(2 * (size_t)ne + 1);
  for (int k = 0; k < ne; k++) {
    int a = t->exclusions[3 * k], b = t->exclusions[3 * k + 1];
    if (a < 0 || b < 0 || a >= n || b >= n)
      return fail(PMGPU_ERR_ARG, "exclusion atom index out of range");
    start[a + 1]++;
    start[b + 1]++;
  }
  for (int i = 0; i < n; i++) start[i + 1] += start[i];
  std::vector<int> cur(start.begin(), start.end() - 1);
  for (int k = 0; k < ne; k++) {
    int a = t->exclusions[3 * k], b = t->exclusions[3 * k + 1], c = t->exclusions[3 * k + 2];
    partner[cur[a]] = b; cls[cur[a]++] = c;
    partner[cur[b]] = a; cls[cur[b]++] = c;
  }
  // index range of each atom's exclusion partners: pair loops consult the
  // table only for partners inside it
  std::vector<int2> range(std::max(1, n), make_int2(INT_MAX, -1));
  for (int i = 0; i < n; i++)
    for (int k = start[i]; k < start[i + 1]; k++) {
      range[i].x = std::min(range[i].x, partner[k]);
      range[i].y = std::max(range[i].y, partner[k]);
    }
  PM_CHECK(upload(s.get(), &s->d_excl_range, range.data(), (size_t)std::max(1, n)));
  PM_CHECK(upload(s.get(), &s->d_excl_start, start.data(), n + 1));
  PM_CHECK(upload(s.get(), &s->d_excl_partner, partner.data(), 2 * (size_t)ne + 1));
  PM_CHECK(upload(s.get(), &s->d_excl_class, cls.data(), 2 * (size_t)ne + 1));
  // The correction term iterates the table with the class each entry holds.
  std::vector<int> table(3 * (size_t)ne + 3);
  for (int k = 0; k < ne; k++) {
    table[3 * k] = t->exclusions[3 * k];
    table[3 * k + 1] = t->exclusions[3 * k + 1];
    table[3 * k + 2] = t->exclusion_table_class ? t->exclusion_table_class[k]
                                                : t->exclusions[3 * k + 2];
  }
  PM_CHECK(upload(s.get(), &s->d_excl_pairs, table.data(), 3 * (size_t)ne));
  s->n_excl = ne;
  s->h_excl.assign(t->exclusions, t->exclusions + 3 * (size_t)ne);
  s->n_bonds = std::max(0, t->n_bonds);
  s->n_angles = std::max(0, t->n_angles);
  if (s->n_bonds && (!t->bond_atoms || !t->bond_params))
    return fail(PMGPU_ERR_ARG, "bond arrays missing");
  if (s->n_angles && (!t->angle_atoms || !t->angle_params))
    return fail(PMGPU_ERR_ARG, "angle arrays missing");
  PM_CHECK(upload(s.get(), &s->d_bond_atoms, s->n_bonds ? t->bond_atoms : (const int *)nullptr, 2 * (size_t)s->n_bonds));
  PM_CHECK(upload(s.get(), &s->d_bond_params, s->n_bonds ? t->bond_params : (const double *)nullptr, 2 * (size_t)s->n_bonds));
  PM_CHECK(upload(s.get(), &s->d_angle_atoms, s->n_angles ? t->angle_atoms : (const int *)nullptr, 3 * (size_t)s->n_angles));
  PM_CHECK(upload(s.get(), &s->d_angle_params, s->n_angles ? t->angle_params : (const double *)nullptr, 4 * (size_t)s->n_angles));
  s->n_dihedrals = t->dihedral_atoms ? t->n_dihedrals : 0;
  s->n_impropers = t->improper_atoms ? t->n_impropers : 0;
  for (int k = 0; k < 4 * s->n_dihedrals; k++)
    if (t->dihedral_atoms[k] < 0 || t->dihedral_atoms[k] >= n)
      return fail(PMGPU_ERR_ARG, "dihedral atom index out of range");
  for (int k = 0; k < 4 * s->n_impropers; k++)
    if (t->improper_atoms[k] < 0 || t->improper_atoms[k] >= n)
      return fail(PMGPU_ERR_ARG, "improper atom index out of range");
  PM_CHECK(upload(s.get(), &s->d_dihedral_atoms, s->n_dihedrals ? t->dihedral_atoms : (const int *)nullptr, 4 * (size_t)s->n_dihedrals));
  PM_CHECK(upload(s.get(), &s->d_dihedral_params, s->n_dihedrals ? t->dihedral_params : (const double *)nullptr, 3 * (size_t)s->n_dihedrals));
  PM_CHECK(upload(s.get(), &s->d_improper_atoms, s->n_impropers ? t->improper_atoms : (const int *)nullptr, 4 * (size_t)s->n_impropers));
  PM_CHECK(upload(s.get(), &s->d_improper_params, s->n_impropers ? t->improper_params : (const double *)nullptr, 3 * (size_t)s->n_impropers));
  if (t->gb_vdwr && t->gb_scale && t->gb_offset) {
    PM_CHECK(upload(s.get(), &s->d_gb_vdwr, t->gb_vdwr, n));
    PM_CHECK(upload(s.get(), &s->d_gb_scale, t->gb_scale, n));
    PM_CHECK(upload(s.get(), &s->d_gb_offset, t->gb_offset, n));
    for (int k = 0; k < 3; k++) s->gb_obc[k] = t->gb_obc[k];
  }
  if (t->water) PM_CHECK(upload(s.get(), &s->d_water, t->water, n));
  if (t->scpism_alpha) {
    const double *pd[6] = {t->scpism_sqrtalpha, t->scpism_alpha, t->scpism_zeta,
                           t->scpism_eta, t->scpism_c, t->scpism_g};
    const int *pi[3] = {t->scpism_hbond, t->scpism_residue, t->scpism_name};
    for (const double *p : pd)
      if (!p) return fail(PMGPU_ERR_ARG, "SCPISM data given in part");
    for (const int *p : pi)
      if (!p) return fail(PMGPU_ERR_ARG, "SCPISM data given in part");
    std::vector<double> hd(6 * (size_t)nn);
    std::vector<int> hi(3 * (size_t)nn);
    for (int k = 0; k < 6; k++) std::copy(pd[k], pd[k] + n, hd.begin() + (size_t)k * nn);
    for (int k = 0; k < 3; k++) std::copy(pi[k], pi[k] + n, hi.begin() + (size_t)k * nn);
    PM_CHECK(upload(s.get(), &s->d_scp, hd.data(), hd.size()));
    PM_CHECK(upload(s.get(), &s->d_scp_i, hi.data(), hi.size()));
    PM_CHECK(upload(s.get(), &s->d_born_q, (const double *)nullptr, 2 * (size_t)nn));
    PM_CUDA(cudaStreamSynchronize(s->stream));  // the packed host arrays end here
  }
  PM_CHECK(upload(s.get(), &s->d_pos, (const double *)nullptr, 3 * nn));
  PM_CHECK(upload(s.get(), &s->d_vel, (const double *)nullptr, 3 * nn));
  PM_CHECK(upload(s.get(), &s->d_force, (const long long *)nullptr, 3 * nn));
  PM_CHECK(upload(s.get(), &s->d_acc, (const long long *)nullptr, ACC_COUNT));
  PM_CHECK(upload(s.get(), &s->d_status, (const int *)nullptr, 1));
  PM_CHECK(upload(s.get(), &s->d_step, (const unsigned long long *)nullptr, 2));  // step, blocks done
  PM_CHECK(upload(s.get(), &s->d_stage, (const double *)nullptr, 3 * nn));
  PM_CUDA(cudaMallocHost(&s->h_acc, sizeof(long long) * ACC_COUNT));
  PM_CUDA(cudaMallocHost(&s->h_status, sizeof(int)));
  PM_CUDA(cudaMallocHost(&s->h_stage, sizeof(double) * 3 * nn));
  PM_CUDA(cudaStreamSynchronize(s->stream));
  s->h_charge.assign(t->charge, t->charge + n);
  *out = reinterpret_cast<pmgpu_system *>(s.release());
  return PMGPU_OK;
}

int pmgpu_system_destroy(pmgpu_system *h) {
  if (!h) return PMGPU_OK;
  System *s = reinterpret_cast<System *>(h);
  system_free(s);
  delete s;
  return PMGPU_OK;
}

static System *sysp(pmgpu_system *h) { return reinterpret_cast<System *>(h); }

static int copy_in(System *s, double *dst, const double *src) {
  if (!src) return fail(PMGPU_ERR_ARG, "null host array");
  size_t bytes = sizeof(double) * 3 * (size_t)s->n;
  if (!bytes) return PMGPU_OK;
  std::memcpy(s->h_stage, src, bytes);
  PM_CUDA(cudaMemcpyAsync(dst, s->h_stage, bytes, cudaMemcpyHostToDevice, s->stream));
  PM_CUDA(cudaStreamSynchronize(s->stream));
  return PMGPU_OK;
}
static int copy_out(System *s, double *dst, const double *src) {
  if (!dst) return fail(PMGPU_ERR_ARG, "null host array");
  size_t bytes = sizeof(double) * 3 * (size_t)s->n;
  if (!bytes) return PMGPU_OK;
  PM_CUDA(cudaMemcpyAsync(s->h_stage, src, bytes, cudaMemcpyDeviceToHost, s->stream));
  PM_CUDA(cudaStreamSynchronize(s->stream));
  std::memcpy(dst, s->h_stage, bytes);
  return PMGPU_OK;
}

int pmgpu_system_set_positions(pmgpu_system *h, const double *pos) {
  if (!h) return fail(PMGPU_ERR_ARG, "null system");
  System *s = sysp(h);
  if (pos)
    for (size_t k = 0; k < 3 * (size_t)s->n; k++)
      if (!std::isfinite(pos[k]))
        return fail(PMGPU_ERR_NAN, "non-finite position of atom " + std::to_string(k / 3));
  PM_CHECK(run_finish(s));
  PM_CUDA(cudaSetDevice(s->device));
  PM_CHECK(copy_in(s, s->d_pos, pos));
  s->forces_valid = 0;
  for (auto &nl : s->lists) nl.built = 0;  // a fresh build at the next evaluation
  return PMGPU_OK;
}

int pmgpu_system_set_step(pmgpu_system *h, long long step) {
  if (!h) return fail(PMGPU_ERR_ARG, "null system");
  if (step < 0) return fail(PMGPU_ERR_ARG, "step must be >= 0");
  System *s = sysp(h);
  PM_CHECK(run_finish(s));
  s->step = (uint64_t)step;  // the device counter is set at the next run
  return PMGPU_OK;
}
int pmgpu_system_get_positions(pmgpu_system *h, double *pos) {
  if (!h) return fail(PMGPU_ERR_ARG, "null system");
  System *s = sysp(h);
  PM_CHECK(run_finish(s));
  PM_CUDA(cudaSetDevice(s->device));
  return copy_out(s, pos, s->d_pos);
}
int pmgpu_system_set_velocities(pmgpu_system *h, const double *vel) {
  if (!h) return fail(PMGPU_ERR_ARG, "null system");
  System *s = sysp(h);
  PM_CHECK(run_finish(s));
  PM_CUDA(cudaSetDevice(s->device));
  return copy_in(s, s->d_vel, vel);
}
int pmgpu_system_get_velocities(pmgpu_system *h, double *vel) {
  if (!h) return fail(PMGPU_ERR_ARG, "null system");
  System *s = sysp(h);
  PM_CHECK(run_finish(s));
  PM_CUDA(cudaSetDevice(s->device));
  return copy_out(s, vel, s->d_vel);
}

int pmgpu_system_get_forces(pmgpu_system *h, double *forces) {
  if (!h || !forces) return fail(PMGPU_ERR_ARG, "null argument");
  System *s = sysp(h);
  PM_CHECK(run_finish(s));
  PM_CUDA(cudaSetDevice(s->device));
  return forces_to_host(s, forces, 0);
}

int pmgpu_system_get_energies(pmgpu_system *h, double *energies, double *virial) {
  if (!h) return fail(PMGPU_ERR_ARG, "null system");
  System *s = sysp(h);
  PM_CHECK(run_finish(s));
  if (energies)
    for (int k = 0; k < PMGPU_E_COUNT; k++) energies[k] = s->last_energy[k];
  if (virial)
    for (int k = 0; k < 9; k++) virial[k] = s->last_virial[k];
  return PMGPU_OK;
}

void *pmgpu_system_stream(pmgpu_system *h) { return h ? (void *)sysp(h)->stream : nullptr; }

int pmgpu_system_device_state(pmgpu_system *h, double **pos, double **vel,
                              long long **force_fixed) {
  if (!h) return fail(PMGPU_ERR_ARG, "null system");
  System *s = sysp(h);
  if (pos) *pos = s->d_pos;
  if (vel) *vel = s->d_vel;
  if (force_fixed) *force_fixed = s->d_force;
  return PMGPU_OK;
}

// --------------------------------------------------------------- forces
static int list_for(System *s, double cutoff, double skin) {
  for (size_t k = 0; k < s->lists.size(); k++)
    if (s->lists[k].cutoff == cutoff && s->lists[k].skin == skin) return (int)k;
  NeighborList nl;
  int r = nb_list_init(s, &nl, cutoff, skin, 0);
  if (r != PMGPU_OK) {
    nb_list_free(s, &nl);
    return -r;
  }
  s->lists.push_back(nl);
  return (int)s->lists.size() - 1;
}

static int add_force(System *s, Force &f, int *force_id) {
  PM_CHECK(run_finish(s));
  f.id = (int)s->forces.size();
  s->forces.push_back(f);
  if (force_id) *force_id = f.id;
  s->forces_valid = 0;
  s->graph_version++;
  return PMGPU_OK;
}

static double default_skin(const System *s, double cutoff) {
  // A 1.3 A skin: the list is rebuilt on about 18 of 100 steps for liquid
  // (flexible) water at 1 fs, which balances the build against the pairs
  // the skin adds to every step (1.0 and 1.6 A measured within 1 %, 0.7 A
  // 4 % slower); small boxes get a smaller skin so cutoff + skin stays
  // below the box edge.  PMGPU_LIST_SKIN overrides the 1.3 A (a tuning
  // knob: any skin gives the same pair set, only the work split between
  // the list builds and the pair kernel changes).
  double skin = 1.3;
  static const char *env = std::getenv("PMGPU_LIST_SKIN");
  if (env && std::atof(env) >= 0.0) skin = std::atof(env);
  if (s->box.periodic) {
    double emin = std::min(s->box.e[0], std::min(s->box.e[1], s->box.e[2]));
    if (cutoff + skin >= emin) skin = std::max(0.0, 0.5 * (emin - cutoff));
  }
  return skin;
}

// The cutoff terms of NonbondedCutoff (all_images 0) and of the
// NonbondedFull lattice sum (all_images 1) over the cluster-pair list.
static int cutoff_terms_add(pmgpu_system *h, const pmgpu_switch *lj_sw,
                            const pmgpu_switch *coul_sw, double alg_cutoff, double cellsize,
                            int all_images, int *force_id) {
  if (!h) return fail(PMGPU_ERR_ARG, "null system");
  System *s = sysp(h);
  PM_CHECK(run_finish(s));
  PM_CUDA(cudaSetDevice(s->device));
  if (!lj_sw && !coul_sw) return fail(PMGPU_ERR_ARG, "need LennardJones and/or Coulomb");
  PM_CHECK(validate_switch(lj_sw, "LennardJones"));
  PM_CHECK(validate_switch(coul_sw, "Coulomb"));
  if (!(alg_cutoff > 0)) return fail(PMGPU_ERR_ARG, "algorithm cutoff must be > 0");
  if (all_images) {
    if (!s->box.periodic) return fail(PMGPU_ERR_UNSUPPORTED, "NonbondedFull needs a periodic box");
    for (const pmgpu_switch *w : {lj_sw, coul_sw}) {
      if (!w) continue;
      if (w->kind == PMGPU_SW_CUTOFF)
        return fail(PMGPU_ERR_ARG, "NonbondedFull takes C1, C2, Cn or CmpCnCn switching");
      const double wc = (w->kind == PMGPU_SW_CN && w->switchoff > 0) ? w->switchoff : w->cutoff;
      // the lattice holds the vectors up to twice the algorithm cutoff
      // (PeriodicBoundaryConditions.cpp:80-104), which reaches every image
      // inside the switch cutoff only when that is no longer
      if (wc > alg_cutoff)
        return fail(PMGPU_ERR_UNSUPPORTED,
                    "NonbondedFull: switch cutoff beyond the algorithm cutoff");
    }
  }
  Force f;
  f.kind = FK_CUTOFF;
  f.alg_cutoff = alg_cutoff;
  f.cellsize = cellsize;
  f.terms.coulomb_scaling = s->coulomb_scaling;
  // OneAtomPairTwo: rough test with the larger switch cutoff; when any
  // switch modifies (C1/C2/Cn) both terms are switched, which zeroes each
  // beyond its own cutoff (OneAtomPairTwo.h:24-27, :40-45, :66-76).
  double c2max = 0;
  int modify = 0;
  if (lj_sw) {
    switch_setup(lj_sw, &f.terms.lj_sw);
    c2max = std::max(c2max, f.terms.lj_sw.cutoff2);
    modify |= f.terms.lj_sw.modify;
  }
  if (coul_sw) {
    switch_setup(coul_sw, &f.terms.coul_sw);
    c2max = std::max(c2max, f.terms.coul_sw.cutoff2);
    modify |= f.terms.coul_sw.modify;
  }
  if (lj_sw) {
    f.terms.mask |= TERM_LJ;
    f.terms.lj_sw.modify = modify;
    f.terms.lj_cut2 = modify ? f.terms.lj_sw.cutoff2 : c2max;
    if (!lj_sw || !coul_sw) f.terms.lj_cut2 = f.terms.lj_sw.cutoff2;
  }
  if (coul_sw) {
    f.terms.mask |= TERM_COUL;
    f.terms.coul_sw.modify = modify;
    f.terms.coul_cut2 = modify ? f.terms.coul_sw.cutoff2 : c2max;
    if (!lj_sw || !coul_sw) f.terms.coul_cut2 = f.terms.coul_sw.cutoff2;
  }
  double rc = std::sqrt(c2max);
  if (s->box.periodic) {
    double emin = std::min(s->box.e[0], std::min(s->box.e[1], s->box.e[2]));
    if (rc >= emin)
      return fail(PMGPU_ERR_UNSUPPORTED, "cutoff forces need box edges longer than the cutoff");
    // Below twice the cutoff a pair can be inside it under two images; the
    // reference's minimalDifference (PeriodicBoundaryConditions.h:72-110)
    // keeps only the minimal one, and so does the pair kernel.  The
    // lattice sum takes every image (OneAtomPairFull.h:91-132).
    f.terms.minimal_image = all_images ? 0 : 2 * rc > emin;
  }
  int li = list_for(s, rc, default_skin(s, rc));
  if (li < 0) return -li;
  f.list_index = li;
  return add_force(s, f, force_id);
}

int pmgpu_force_cutoff_add(pmgpu_system *h, const pmgpu_switch *lj_sw,
                           const pmgpu_switch *coul_sw, double alg_cutoff,
                           double cellsize, int *force_id) {
  return cutoff_terms_add(h, lj_sw, coul_sw, alg_cutoff, cellsize, 0, force_id);
}

int pmgpu_force_full_add(pmgpu_system *h, const pmgpu_switch *lj_sw,
                         const pmgpu_switch *coul_sw, double alg_cutoff, double cellsize,
                         int *force_id) {
  return cutoff_terms_add(h, lj_sw, coul_sw, alg_cutoff, cellsize, 1, force_id);
}

int pmgpu_force_simplefull_add(pmgpu_system *h, int lj, int coulomb, int *force_id) {
  if (!h) return fail(PMGPU_ERR_ARG, "null system");
  System *s = sysp(h);
  PM_CHECK(run_finish(s));
  if (s->box.periodic)
    return fail(PMGPU_ERR_UNSUPPORTED, "NonbondedSimpleFull is the vacuum all-pairs path");
  if (!lj && !coulomb) return fail(PMGPU_ERR_ARG, "need LennardJones and/or Coulomb");
  if (s->precision == PMGPU_PREC_MIXED) {
    PM_CUDA(cudaSetDevice(s->device));
    PM_CHECK(nb_simplefull_init(s));
  }
  Force f;
  f.kind = FK_SIMPLEFULL;
  f.sf_lj = lj ? 1 : 0;
  f.sf_coul = coulomb ? 1 : 0;
  return add_force(s, f, force_id);
}

int pmgpu_force_simplefull_switched_add(pmgpu_system *h, const pmgpu_switch *lj_sw,
                                        const pmgpu_switch *coul_sw, int *force_id) {
  if (!h) return fail(PMGPU_ERR_ARG, "null system");
  System *s = sysp(h);
  PM_CHECK(run_finish(s));
  PM_CUDA(cudaSetDevice(s->device));
  if (!lj_sw && !coul_sw) return fail(PMGPU_ERR_ARG, "need LennardJones and/or Coulomb");
  for (const pmgpu_switch *w : {lj_sw, coul_sw}) {
    if (!w) continue;
    const int base = w->kind & ~PMGPU_SW_COMPLEMENT;
    if (w->kind & PMGPU_SW_COMPLEMENT) {
      if (base != PMGPU_SW_C1 && base != PMGPU_SW_C2 && base != PMGPU_SW_CN)
        return fail(PMGPU_ERR_ARG, "Complement applies to C1, C2 or Cn");
      pmgpu_switch b = *w;
      b.kind = base;
      PM_CHECK(validate_switch(&b, "Complement switch"));
    } else if (base != PMGPU_SW_UNIVERSAL) {
      PM_CHECK(validate_switch(w, "NonbondedSimpleFull switch"));
    }
  }
  Force f;
  f.kind = FK_SIMPLEFULL_SW;
  // OneAtomPairTwo switches both terms when either switch modifies
  // (OneAtomPairTwo.h:66-76); a single term by its own MODIFY
  int modify = 0;
  if (lj_sw) {
    switch_setup(lj_sw, &f.terms.lj_sw);
    f.terms.mask |= TERM_LJ;
    modify |= f.terms.lj_sw.modify;
  }
  if (coul_sw) {
    switch_setup(coul_sw, &f.terms.coul_sw);
    f.terms.mask |= TERM_COUL;
    modify |= f.terms.coul_sw.modify;
  }
  f.terms.lj_sw.modify = modify;
  f.terms.coul_sw.modify = modify;
  f.terms.coulomb_scaling = s->coulomb_scaling;
  return add_force(s, f, force_id);
}

int pmgpu_force_scpism_add(pmgpu_system *h, const pmgpu_switch *lj_sw,
                           const pmgpu_switch *coul_sw, double dielectric, int *force_id) {
  if (!h) return fail(PMGPU_ERR_ARG, "null system");
  System *s = sysp(h);
  PM_CHECK(run_finish(s));
  PM_CUDA(cudaSetDevice(s->device));
  if (!s->d_scp) return fail(PMGPU_ERR_ARG, "CoulombSCPISM requires SCPISM parameters");
  if (!coul_sw) return fail(PMGPU_ERR_ARG, "CoulombSCPISM needs its switching function");
  if (!(dielectric >= 0)) return fail(PMGPU_ERR_ARG, "-D must be >= 0");
  for (const pmgpu_switch *w : {lj_sw, coul_sw}) {
    if (!w) continue;
    if (w->kind & PMGPU_SW_COMPLEMENT)
      return fail(PMGPU_ERR_ARG, "CoulombSCPISM takes C1, C2, Cn or CmpCnCn switching");
    if (w->kind != PMGPU_SW_UNIVERSAL) PM_CHECK(validate_switch(w, "SCPISM switch"));
  }
  Force f;
  f.kind = FK_SCPISM;
  // OneAtomPairTwo switches both terms when either switch modifies
  // (OneAtomPairTwo.h:66-76); one term by its own MODIFY
  int modify = 0;
  if (lj_sw) {
    switch_setup(lj_sw, &f.terms.lj_sw);
    f.terms.mask |= TERM_LJ;
    modify |= f.terms.lj_sw.modify;
  }
  switch_setup(coul_sw, &f.terms.coul_sw);
  f.terms.mask |= TERM_COUL;
  modify |= f.terms.coul_sw.modify;
  f.terms.lj_sw.modify = modify;
  f.terms.coul_sw.modify = modify;
  f.terms.coulomb_scaling = s->coulomb_scaling;
  f.scp_D = dielectric;
  return add_force(s, f, force_id);
}

int pmgpu_force_born_add(pmgpu_system *h, int radii_bornswitch, double radii_cutoff,
                         int self_bornswitch, double self_cutoff, double dielectric,
                         int *force_id) {
  if (!h) return fail(PMGPU_ERR_ARG, "null system");
  System *s = sysp(h);
  PM_CHECK(run_finish(s));
  PM_CUDA(cudaSetDevice(s->device));
  if (!s->d_scp) return fail(PMGPU_ERR_ARG, "BornRadii / BornSelf require SCPISM parameters");
  if (radii_bornswitch < 0 || self_bornswitch < 0)
    return fail(PMGPU_ERR_ARG, "-bornswitch must be >= 0");
  if (!(radii_cutoff > 0) || !(self_cutoff > 0)) return fail(PMGPU_ERR_ARG, "cutoff must be > 0");
  if (!(dielectric >= 0)) return fail(PMGPU_ERR_ARG, "-D must be >= 0");
  Force f;
  f.kind = FK_BORN;
  f.born_rsw = radii_bornswitch;
  f.born_ssw = self_bornswitch;
  f.born_rcut = radii_cutoff;
  f.born_scut = self_cutoff;
  f.scp_D = dielectric;
  return add_force(s, f, force_id);
}

int pmgpu_force_pme_add(pmgpu_system *h, double alpha, double rc, int order,
                        const int grid[3], int flags, int exact_erf, double cellsize,
                        int *force_id) {
  if (!h) return fail(PMGPU_ERR_ARG, "null system");
  System *s = sysp(h);
  PM_CHECK(run_finish(s));
  PM_CUDA(cudaSetDevice(s->device));
  if (!s->box.periodic) return fail(PMGPU_ERR_UNSUPPORTED, "PME needs a periodic box");
  if (!(alpha > 0)) return fail(PMGPU_ERR_ARG, "alpha must be > 0");
  if ((flags & PMGPU_EWALD_REAL) && !(rc > 0)) return fail(PMGPU_ERR_ARG, "rc must be > 0");
  if (flags & ~PMGPU_EWALD_ALL || !flags) return fail(PMGPU_ERR_ARG, "bad Ewald term flags");
  Force f;
  f.kind = FK_PME;
  f.ewald_flags = flags;
  f.alpha = alpha;
  f.rc = rc;
  f.order = order;
  f.cellsize = cellsize;
  if (grid) for (int a = 0; a < 3; a++) f.grid[a] = grid[a];
  f.terms.coulomb_scaling = s->coulomb_scaling;
  if (flags & PMGPU_EWALD_REAL) {
    f.terms.mask = TERM_EWALD;
    f.terms.ewald_alpha = alpha;
    f.terms.ewald_rc2 = rc * rc;
    f.terms.exact_erf = exact_erf ? 1 : 0;
    if (!exact_erf) {
      PM_CHECK(ewald_table_build(s, &f));
      f.terms.ewtab = f.d_ewtab;
    }
    int li = list_for(s, rc, default_skin(s, rc));
    if (li < 0) return -li;
    f.list_index = li;
  } else {
    // spatial order for spreading still comes from a list when one exists
    f.list_index = s->lists.empty() ? -1 : 0;
  }
  if (flags & PMGPU_EWALD_RECIPROCAL) PM_CHECK(pme_init(s, &f));
  // point self energy and charged-system energy (:694-714)
  double q2 = 0, q = 0;
  for (double c : s->h_charge) q2 += c * c;
  for (double c : s->h_charge) q += c;
  f.self_energy = -q2 * alpha / std::sqrt(M_PI);
  f.charged_energy = 0.0;
  if (std::fabs(q * 0.00268283) > 1.0e-5)
    f.charged_energy = -M_PI / (2.0 * s->box.V * (alpha * alpha)) * q * q;
  return add_force(s, f, force_id);
}

int pmgpu_force_gb_add(pmgpu_system *h, double solute, double solvent, int *force_id) {
  if (!h) return fail(PMGPU_ERR_ARG, "null system");
  System *s = sysp(h);
  PM_CHECK(run_finish(s));
  PM_CUDA(cudaSetDevice(s->device));
  if (s->box.periodic) return fail(PMGPU_ERR_UNSUPPORTED, "GB is the vacuum all-pairs path");
  if (!(solute > 0) || !(solvent > 0)) return fail(PMGPU_ERR_ARG, "dielectrics must be > 0");
  PM_CHECK(gb_init(s));
  Force f;
  f.kind = FK_GB;
  f.solute = solute;
  f.solvent = solvent;
  return add_force(s, f, force_id);
}

int pmgpu_force_gbace_add(pmgpu_system *h, double solvation_param,
                          double water_sphere_radius, int *force_id) {
  if (!h) return fail(PMGPU_ERR_ARG, "null system");
  System *s = sysp(h);
  PM_CHECK(run_finish(s));
  PM_CUDA(cudaSetDevice(s->device));
  if (s->box.periodic) return fail(PMGPU_ERR_UNSUPPORTED, "GBACE is the vacuum all-pairs path");
  if (!std::isfinite(solvation_param) || !std::isfinite(water_sphere_radius))
    return fail(PMGPU_ERR_ARG, "GBACE parameters must be finite");
  PM_CHECK(gb_init(s));
  Force f;
  f.kind = FK_GBACE;
  f.ace_sigma = solvation_param;
  f.ace_rho = water_sphere_radius;
  return add_force(s, f, force_id);
}

int pmgpu_force_bonded_add(pmgpu_system *h, int bonds, int angles, int *force_id) {
  if (!h) return fail(PMGPU_ERR_ARG, "null system");
  Force f;
  f.kind = FK_BONDED;
  f.bonds = bonds ? 1 : 0;
  f.angles = angles ? 1 : 0;
  return add_force(sysp(h), f, force_id);
}

int pmgpu_force_torsion_add(pmgpu_system *h, int dihedrals, int impropers, int *force_id) {
  if (!h) return fail(PMGPU_ERR_ARG, "null system");
  Force f;
  f.kind = FK_TORSION;
  f.dihedrals = dihedrals ? 1 : 0;
  f.impropers = impropers ? 1 : 0;
  return add_force(sysp(h), f, force_id);
}

int pmgpu_force_set_enabled(pmgpu_system *h, int id, int enabled) {
  if (!h) return fail(PMGPU_ERR_ARG, "null system");
  System *s = sysp(h);
  PM_CHECK(run_finish(s));
  if (id < 0 || id >= (int)s->forces.size()) return fail(PMGPU_ERR_ARG, "no such force");
  s->forces[id].enabled = enabled ? 1 : 0;
  s->graph_version++;
  s->forces_valid = 0;
  return PMGPU_OK;
}

int pmgpu_evaluate(pmgpu_system *h, double *energies, double *virial) {
  if (!h) return fail(PMGPU_ERR_ARG, "null system");
  System *s = sysp(h);
  PM_CHECK(run_finish(s));
  PM_CUDA(cudaSetDevice(s->device));
  // no energies and no virial wanted: the force-only kernels of the inner
  // MD steps (the pair kernel's specialised form), forces only
  const int mode = virial ? PAIR_VIRIAL : (energies ? PAIR_ENERGY : PAIR_FORCE);
  int r = with_overflow_retry([&]() {
    PM_CHECK(zero_forces(s));
    PM_CHECK(begin_eval(s));
    PM_CHECK(evaluate_forces(s, -1, mode));
    return read_results(s, -1, energies, virial, 0, mode != PAIR_FORCE);
  });
  s->forces_valid = (r == PMGPU_OK);
  return r;
}

int pmgpu_force_evaluate(pmgpu_system *h, int id, const double *pos, double *forces,
                         double *energies, double *virial) {
  if (!h) return fail(PMGPU_ERR_ARG, "null system");
  System *s = sysp(h);
  PM_CHECK(run_finish(s));
  PM_CUDA(cudaSetDevice(s->device));
  if (id < 0 || id >= (int)s->forces.size()) return fail(PMGPU_ERR_ARG, "no such force");
  if (pos) PM_CHECK(copy_in(s, s->d_pos, pos));
  s->forces_valid = 0;
  const int mode = virial ? PAIR_VIRIAL : (energies ? PAIR_ENERGY : PAIR_FORCE);
  PM_CHECK(with_overflow_retry([&]() {
    PM_CHECK(zero_forces(s));
    PM_CHECK(begin_eval(s));
    PM_CHECK(evaluate_forces(s, id, mode));
    return read_results(s, id, energies, virial, 1, mode != PAIR_FORCE);
  }));
  if (forces) PM_CHECK(forces_to_host(s, forces, 1));
  return PMGPU_OK;
}

// One MD step body: kick + drift (+ device step counter), then the force
// evaluation at the new positions.
static int one_step(System *s, const pmgpu_integrator *it, int phase, int mode) {
  prof_begin(s, PMGPU_PHASE_INTEGRATE);
  // the update launch also starts the evaluation (clears the accumulators)
  // with one pair list, the update also takes its rebuild decision
  NeighborList *nl = s->lists.size() == 1 ? &s->lists[0] : nullptr;
  int ri = integrate_kick_drift(s, it, phase, 1, nl);
  prof_end(s);
  PM_CHECK(ri);
  // the update (which also advances the step counter of the Langevin noise)
  s->kernels += s->n > 0;
  if (s->n == 0) PM_CHECK(begin_eval(s));
  return evaluate_forces(s, -1, mode, mode != PAIR_FORCE);
}

static bool same_integrator(const pmgpu_integrator &a, const pmgpu_integrator &b) {
  return a.kind == b.kind && a.timestep_fs == b.timestep_fs &&
         a.temperature == b.temperature && a.gamma_ps == b.gamma_ps && a.seed == b.seed;
}

// Replays (capturing on first use) a CUDA graph of g inner steps.  *used is
// 0 when capture is not possible, in which case the caller runs eagerly.
static int run_graph(System *s, const pmgpu_integrator *it, long g, int *used) {
  *used = 0;
  System::StepGraph &sg = s->graphs[g == 1 ? 1 : 0];
  const int phase = it->kind == PMGPU_INT_LANGEVIN_LEAPFROG ? 4 : 1;
  if (!(sg.exec && sg.version == s->graph_version && sg.steps == g &&
        same_integrator(sg.key, *it))) {
    if (sg.exec) cudaGraphExecDestroy(sg.exec);
    sg.exec = nullptr;
    long long k0 = s->kernels;
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      cudaGetLastError();
      s->graphs_disabled = 1;
      return PMGPU_OK;
    }
    int r = PMGPU_OK;
    for (long k = 0; k < g && r == PMGPU_OK; k++) r = one_step(s, it, phase, PAIR_FORCE);
    cudaError_t ec = cudaStreamEndCapture(s->stream, &graph);
    const long long per_launch = s->kernels - k0;
    s->kernels = k0;
    cudaError_t ei = cudaSuccess;
    if (r == PMGPU_OK && ec == cudaSuccess && graph)
      ei = cudaGraphInstantiate(&sg.exec, graph, cudaGraphInstantiateFlagUseNodePriority);
    if (r != PMGPU_OK || ec != cudaSuccess || !graph || ei != cudaSuccess) {
      // the reason is kept for pmgpu_last_error and, with PMGPU_DEBUG set,
      // printed; the run continues with eager launches
      if (std::getenv("PMGPU_DEBUG"))
        std::fprintf(stderr, "pmgpu: step graph not used (%s; end capture: %s; instantiate: %s)\n",
                     r != PMGPU_OK ? g_last_error.c_str() : "capture ok",
                     cudaGetErrorString(ec), cudaGetErrorString(ei));
      if (graph) cudaGraphDestroy(graph);
      cudaGetLastError();
      sg.exec = nullptr;
      s->graphs_disabled = 1;  // fall back to eager launches from now on
      return PMGPU_OK;
    }
    cudaGraphDestroy(graph);
    sg.version = s->graph_version;
    sg.steps = g;
    sg.key = *it;
    sg.kernels = per_launch;
  }
  PM_CUDA(cudaGraphLaunch(sg.exec, s->stream));
  s->kernels += sg.kernels;
  *used = 1;
  return PMGPU_OK;
}

// Integrator::run(n) on the device, split into the part that only enqueues
// work on the system's stream (run_enqueue) and the part that waits for it
// and checks the status (run_finish).  Forces of the current positions are
// kept resident between calls (ProtoMol keeps myForces between run calls);
// the first call after positions changed on the host evaluates them, like
// Integrator::initialize (StandardIntegrator.cpp:39-43).
static int check_integrator(const pmgpu_integrator *it) {
  if (!(it->timestep_fs > 0)) return fail(PMGPU_ERR_ARG, "timestep must be > 0");
  if (it->kind != PMGPU_INT_LEAPFROG && it->kind != PMGPU_INT_LANGEVIN_LEAPFROG)
    return fail(PMGPU_ERR_ARG, "unknown integrator");
  if (it->kind == PMGPU_INT_LANGEVIN_LEAPFROG && !(it->gamma_ps > 0))
    return fail(PMGPU_ERR_ARG, "LangevinLeapfrog needs gamma > 0");
  return PMGPU_OK;
}

}  // extern "C"

namespace pmgpu {

// Snapshot of the state a segment starts from: a neighbour list that
// overflows mid-segment is only seen at the end of the segment (no host
// synchronisation per step), and the segment then runs again from here
// with the grown capacity.
int run_snapshot(System *s, int restore) {
  size_t n3 = 3 * (size_t)std::max(1, s->n);
  if (!s->d_snap) PM_CHECK(dev_alloc(s, &s->d_snap, n3 * (2 * sizeof(double) + sizeof(long long))));
  double *snap_pos = reinterpret_cast<double *>(s->d_snap);
  double *snap_vel = snap_pos + n3;
  long long *snap_f = reinterpret_cast<long long *>(snap_vel + n3);
  const cudaMemcpyKind k = cudaMemcpyDeviceToDevice;
  if (!restore) {
    // the snapshot holds complete forces (no pair forces left in a slot buffer)
    PM_CHECK(fold_pending_slots(s));
    PM_CUDA(cudaMemcpyAsync(snap_pos, s->d_pos, n3 * sizeof(double), k, s->stream));
    PM_CUDA(cudaMemcpyAsync(snap_vel, s->d_vel, n3 * sizeof(double), k, s->stream));
    PM_CUDA(cudaMemcpyAsync(snap_f, s->d_force, n3 * sizeof(long long), k, s->stream));
  } else {
    PM_CUDA(cudaMemcpyAsync(s->d_pos, snap_pos, n3 * sizeof(double), k, s->stream));
    PM_CUDA(cudaMemcpyAsync(s->d_vel, snap_vel, n3 * sizeof(double), k, s->stream));
    PM_CUDA(cudaMemcpyAsync(s->d_force, snap_f, n3 * sizeof(long long), k, s->stream));
  }
  return PMGPU_OK;
}

}  // namespace pmgpu

extern "C" {

static int run_enqueue(System *s, const pmgpu_integrator *it, long n_steps) {
  const bool lang = it->kind == PMGPU_INT_LANGEVIN_LEAPFROG;
  PM_CHECK(set_device_step(s));
  if (!s->forces_valid) {
    PM_CHECK(zero_forces(s));
    PM_CHECK(begin_eval(s));
    PM_CHECK(evaluate_forces(s, -1, PAIR_FORCE, 0));
  }
  for (long k = 0; k < n_steps;) {
    // Inner steps (not the first, not the last) replay a captured graph
    // of several steps when possible; the rest run eagerly.
    const long inner_left = (n_steps - 1) - k;
    if (k > 0 && inner_left > 0 && !s->prof.enabled && !s->graphs_disabled) {
      const long g = inner_left >= kGraphSteps ? kGraphSteps : 1;
      int used = 0;
      PM_CHECK(run_graph(s, it, g, &used));
      if (used) {
        s->step += g;
        k += g;
        continue;
      }
    }
    int phase = lang ? (k == 0 ? 3 : 4) : (k == 0 ? 0 : 1);
    PM_CHECK(one_step(s, it, phase, k + 1 == n_steps ? PAIR_ENERGY : PAIR_FORCE));
    s->step++;
    k++;
  }
  prof_begin(s, PMGPU_PHASE_INTEGRATE);
  // the closing half kick also takes the slot forces a force-only
  // evaluation may have left (a run of zero steps)
  int ri = integrate_kick_drift(s, it, lang ? 5 : 2, 0,
                                s->lists.size() == 1 ? &s->lists[0] : nullptr);
  prof_end(s);
  PM_CHECK(ri);
  s->kernels += s->n > 0;
  return PMGPU_OK;
}

static int run_start(System *s, const pmgpu_integrator *it, long n_steps) {
  s->pending.integ = *it;
  s->pending.n_steps = n_steps;
  s->pending.step0 = s->step;
  s->pending.valid0 = s->forces_valid;
  s->pending.active = 1;
  PM_CHECK(run_snapshot(s, 0));
  return run_enqueue(s, it, n_steps);
}

// Waits for the pending segment; on a list overflow (capacity already
// doubled by read_results) restores the snapshot and runs the segment
// again, at most three attempts in all.
static int run_finish(System *s) {
  if (!s->pending.active) return PMGPU_OK;
  PM_CUDA(cudaSetDevice(s->device));
  int r = PMGPU_OK;
  for (int attempt = 0; attempt < 3; attempt++) {
    if (attempt > 0) {
      PM_CHECK(run_snapshot(s, 1));
      s->step = s->pending.step0;
      s->forces_valid = s->pending.valid0;
      PM_CHECK(run_enqueue(s, &s->pending.integ, s->pending.n_steps));
    }
    r = read_results(s, -1, nullptr, nullptr, 0);
    if (r != PMGPU_ERR_OVERFLOW) break;
  }
  s->pending.active = 0;
  s->forces_valid = (r == PMGPU_OK);
  return r;
}

int pmgpu_run(pmgpu_system *h, const pmgpu_integrator *it, long n_steps) {
  if (!h || !it) return fail(PMGPU_ERR_ARG, "null argument");
  System *s = sysp(h);
  PM_CUDA(cudaSetDevice(s->device));
  PM_CHECK(check_integrator(it));
  PM_CHECK(run_finish(s));  // a segment still pending from pmgpu_run_async
  if (n_steps < 1) return PMGPU_OK;
  PM_CHECK(run_start(s, it, n_steps));
  return run_finish(s);
}

int pmgpu_run_async(pmgpu_system *h, const pmgpu_integrator *it, long n_steps) {
  if (!h || !it) return fail(PMGPU_ERR_ARG, "null argument");
  System *s = sysp(h);
  PM_CUDA(cudaSetDevice(s->device));
  PM_CHECK(check_integrator(it));
  if (s->pending.active) return fail(PMGPU_ERR_STATE, "a segment is already pending");
  if (n_steps < 1) return PMGPU_OK;
  return run_start(s, it, n_steps);
}

int pmgpu_run_query(pmgpu_system *h, int *done) {
  if (!h || !done) return fail(PMGPU_ERR_ARG, "null argument");
  System *s = sysp(h);
  if (!s->pending.active) {
    *done = 1;
    return PMGPU_OK;
  }
  PM_CUDA(cudaSetDevice(s->device));
  cudaError_t e = cudaStreamQuery(s->stream);
  if (e == cudaErrorNotReady) {
    *done = 0;
    return PMGPU_OK;
  }
  if (e != cudaSuccess) return fail(PMGPU_ERR_CUDA, cudaGetErrorString(e));
  *done = 1;
  return PMGPU_OK;
}

int pmgpu_run_wait(pmgpu_system *h) {
  if (!h) return fail(PMGPU_ERR_ARG, "null argument");
  System *s = sysp(h);
  PM_CUDA(cudaSetDevice(s->device));
  return run_finish(s);
}

int pmgpu_run_discard(pmgpu_system *h) {
  if (!h) return fail(PMGPU_ERR_ARG, "null argument");
  System *s = sysp(h);
  PM_CUDA(cudaSetDevice(s->device));
  if (!s->pending.active) return PMGPU_OK;
  // the segment's own outcome does not matter: it is undone
  (void)run_finish(s);
  PM_CHECK(run_snapshot(s, 1));
  s->step = s->pending.step0;
  s->forces_valid = s->pending.valid0;
  for (auto &nl : s->lists) nl.built = 0;  // fresh lists, as for new positions
  PM_CUDA(cudaStreamSynchronize(s->stream));
  return PMGPU_OK;
}

int pmgpu_mem_info(pmgpu_context *ctx, long long *free_bytes, long long *total_bytes) {
  if (!ctx || !free_bytes || !total_bytes) return fail(PMGPU_ERR_ARG, "null argument");
  PM_CUDA(cudaSetDevice(ctx->device));
  size_t f = 0, t = 0;
  PM_CUDA(cudaMemGetInfo(&f, &t));
  *free_bytes = (long long)f;
  *total_bytes = (long long)t;
  return PMGPU_OK;
}

// Device bytes a periodic system of n atoms and edge lengths box[3] needs
// with a pair list of the given reach and a PME grid (grid may be NULL):
// the resident state, the sorted coordinates, the list at its initial
// capacity and the PME grids (cuFFT work areas are estimated as one more
// complex grid).
int pmgpu_fp32_peak(pmgpu_context *ctx, double *tflops) {
  if (!ctx || !tflops) return fail(PMGPU_ERR_ARG, "null argument");
  return fp32_peak(ctx->device, tflops);
}

int pmgpu_footprint_estimate(int n_atoms, const double box[3], double reach,
                             const int grid[3], long long *bytes) {
  if (!box || !bytes || n_atoms < 0 || !(reach >= 0)) return fail(PMGPU_ERR_ARG, "bad argument");
  const double n = std::max(1, n_atoms);
  const double V = box[0] * box[1] * box[2];
  double b = n * (24 * 3 + 24 + 24 + 8 + 8 + 8);        // pos, vel, snapshot, force, q, m, ids
  if (reach > 0) {
    // cluster-pair list: padded slots, cluster boxes, sort keys, tile rows
    // (the same sizing as the list set-up)
    const double ncol = std::max(1.0, std::floor(box[0] / kColumnWidth)) *
                        std::max(1.0, std::floor(box[1] / kColumnWidth));
    const double nkeys = ncol * std::max(1.0, std::floor(box[2] / kZBin));
    const double ns = n + 7 * ncol + 8, ncl = ns / 8;
    const double dens = V > 0 ? std::max(n / V, 0.12) : 0.15;
    const double r = reach + 5.0;
    const double cap = 4.18879 * r * r * r * dens / 8.0 / kRowParts * 1.6 + 64;
    b += ns * (16 + 16 + 32 + 4 + 4 + 8 + 24) + n * (4 + 4 + 4 + 24 + 24) + nkeys * 4 + ncol * 16 +
         ncl * kRowParts * (44 * cap + 8);
  }
  if (grid) {
    double G = (double)grid[0] * grid[1] * grid[2];
    double Gc = (double)grid[0] * grid[1] * (grid[2] / 2 + 1);
    b += G * (8 + 4) + Gc * (8 + 4) + Gc * 8;
  }
  *bytes = (long long)(b + (1 << 20));
  return PMGPU_OK;
}

int pmgpu_profile_enable(pmgpu_system *h, int enabled) {
  if (!h) return fail(PMGPU_ERR_ARG, "null system");
  sysp(h)->prof.enabled = enabled ? 1 : 0;
  return PMGPU_OK;
}

int pmgpu_profile_read(pmgpu_system *h, double *ms, long long *launches, int reset) {
  if (!h) return fail(PMGPU_ERR_ARG, "null system");
  System *s = sysp(h);
  PM_CUDA(cudaSetDevice(s->device));
  PM_CUDA(cudaStreamSynchronize(s->stream));
  prof_collect(s);
  for (int k = 0; k < PMGPU_PHASE_COUNT; k++) {
    if (ms) ms[k] = s->prof.ms[k];
    if (launches) launches[k] = s->prof.launches[k];
    if (reset) {
      s->prof.ms[k] = 0;
      s->prof.launches[k] = 0;
    }
  }
  return PMGPU_OK;
}

int pmgpu_kernel_count(pmgpu_system *h, long long *count) {
  if (!h || !count) return fail(PMGPU_ERR_ARG, "null argument");
  *count = sysp(h)->kernels;
  return PMGPU_OK;
}

int pmgpu_set_count_pairs(pmgpu_system *h, int enabled) {
  if (!h) return fail(PMGPU_ERR_ARG, "null system");
  sysp(h)->count_pairs = enabled ? 1 : 0;
  return PMGPU_OK;
}

int pmgpu_force_stats(pmgpu_system *h, int id, pmgpu_stats *out) {
  if (!h || !out) return fail(PMGPU_ERR_ARG, "null argument");
  System *s = sysp(h);
  PM_CHECK(run_finish(s));
  if (id < 0 || id >= (int)s->forces.size()) return fail(PMGPU_ERR_ARG, "no such force");
  std::memset(out, 0, sizeof(*out));
  const Force &f = s->forces[id];
  out->pairs_in_cutoff = s->last_pairs;
  if (f.list_index >= 0) {
    const NeighborList &nl = s->lists[f.list_index];
    out->cells[0] = nl.ncx;
    out->cells[1] = nl.ncy;
    out->cells[2] = nl.nzb;
    out->clusters = nl.nclusters;
    out->pair_kernel = nl.last_form;
    out->list_capacity = nl.cap;
    int rb[2] = {0, 0};
    PM_CUDA(cudaMemcpyAsync(rb, nl.d_rebuild, sizeof(rb), cudaMemcpyDeviceToHost, s->stream));
    PM_CUDA(cudaStreamSynchronize(s->stream));
    out->list_builds = rb[1];
    // list entries: tiles (8 x 4 atom pairs each) over all i clusters
    std::vector<int> cnt(std::max(1, nl.nrows));
    if (nl.nrows) {
      PM_CUDA(cudaMemcpyAsync(cnt.data(), nl.d_tile_count, sizeof(int) * nl.nrows,
                              cudaMemcpyDeviceToHost, s->stream));
      PM_CUDA(cudaStreamSynchronize(s->stream));
      long long tot = 0;
      for (int k = 0; k < nl.nrows; k++) tot += cnt[k];
      out->list_entries = tot;
    }
  }
  return PMGPU_OK;
}

int pmgpu_debug_cell_assign(pmgpu_system *h, double cellsize, int *cell_xyz, int *dims) {
  if (!h || !cell_xyz || !dims) return fail(PMGPU_ERR_ARG, "null argument");
  if (!(cellsize > 0)) return fail(PMGPU_ERR_ARG, "cellsize must be > 0");
  System *s = sysp(h);
  PM_CHECK(run_finish(s));
  PM_CUDA(cudaSetDevice(s->device));
  return nb_debug_cells(s, cellsize, cell_xyz, dims);
}

int pmgpu_debug_set_list_capacity(pmgpu_system *h, int tiles_per_row) {
  if (!h) return fail(PMGPU_ERR_ARG, "null system");
  if (tiles_per_row < 1) return fail(PMGPU_ERR_ARG, "tiles_per_row must be >= 1");
  System *s = sysp(h);
  PM_CHECK(run_finish(s));
  PM_CUDA(cudaSetDevice(s->device));
  for (auto &nl : s->lists) {
    nb_list_free(s, &nl);
    nl.cap = 0;
    nl.cap_set = tiles_per_row;
    PM_CHECK(nb_list_init(s, &nl, nl.cutoff, nl.skin, 0));
  }
  s->graph_version++;
  s->forces_valid = 0;
  return PMGPU_OK;
}

int pmgpu_debug_set_column_capacity(pmgpu_system *h, int atoms_per_column) {
  if (!h) return fail(PMGPU_ERR_ARG, "null system");
  if (atoms_per_column < 1) return fail(PMGPU_ERR_ARG, "atoms_per_column must be >= 1");
  System *s = sysp(h);
  PM_CHECK(run_finish(s));
  PM_CUDA(cudaSetDevice(s->device));
  for (auto &nl : s->lists) {
    nb_list_free(s, &nl);
    nl.bcap = 0;
    nl.bcap_set = atoms_per_column;
    PM_CHECK(nb_list_init(s, &nl, nl.cutoff, nl.skin, 0));
  }
  s->graph_version++;
  s->forces_valid = 0;
  return PMGPU_OK;
}

int pmgpu_debug_limit_list_rows(pmgpu_system *h, int tiles_per_row) {
  if (!h) return fail(PMGPU_ERR_ARG, "null system");
  if (tiles_per_row < 1) return fail(PMGPU_ERR_ARG, "tiles_per_row must be >= 1");
  System *s = sysp(h);
  PM_CHECK(run_finish(s));
  for (auto &nl : s->lists) nl.limit = tiles_per_row;
  s->graph_version++;  // captured graphs hold the build's arguments
  return PMGPU_OK;
}

int pmgpu_debug_pair_set(pmgpu_system *h, int id, int *pairs, long long cap,
                         long long *count) {
  if (!h || !count) return fail(PMGPU_ERR_ARG, "null argument");
  System *s = sysp(h);
  PM_CHECK(run_finish(s));
  PM_CUDA(cudaSetDevice(s->device));
  if (id < 0 || id >= (int)s->forces.size()) return fail(PMGPU_ERR_ARG, "no such force");
  Force &f = s->forces[id];
  if (f.list_index < 0) return fail(PMGPU_ERR_ARG, "force has no pair list");
  long long want = std::max(1LL, cap);
  if (s->pairbuf_cap < want) {
    dev_free(s, s->d_pairbuf);
    PM_CHECK(dev_alloc(s, &s->d_pairbuf, sizeof(long long) * want));
    s->pairbuf_cap = want;
  }
  if (!s->d_paircount) PM_CHECK(dev_alloc(s, &s->d_paircount, sizeof(long long)));
  PM_CUDA(cudaMemsetAsync(s->d_paircount, 0, sizeof(long long), s->stream));
  PM_CHECK(zero_forces(s));
  PM_CHECK(begin_eval(s));
  PM_CHECK(nb_prepare(s, &s->lists[f.list_index], 0));
  PM_CHECK(nb_build(s, &s->lists[f.list_index]));
  PM_CHECK(nb_pair_forces(s, &s->lists[f.list_index], f.terms, PAIR_RECORD, 1));
  long long total = 0;
  PM_CUDA(cudaMemcpyAsync(&total, s->d_paircount, sizeof(long long), cudaMemcpyDeviceToHost,
                          s->stream));
  PM_CUDA(cudaStreamSynchronize(s->stream));
  *count = total;
  long long ncopy = std::min(total, cap);
  if (pairs && ncopy > 0) {
    std::vector<long long> buf(ncopy);
    PM_CUDA(cudaMemcpyAsync(buf.data(), s->d_pairbuf, sizeof(long long) * ncopy,
                            cudaMemcpyDeviceToHost, s->stream));
    PM_CUDA(cudaStreamSynchronize(s->stream));
    for (long long k = 0; k < ncopy; k++) {
      pairs[2 * k] = (int)(buf[k] >> 32);
      pairs[2 * k + 1] = (int)(buf[k] & 0xffffffffLL);
    }
  }
  s->forces_valid = 0;
  return PMGPU_OK;
}

}  // extern "C"
