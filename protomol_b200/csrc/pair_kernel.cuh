// The fused nonbonded pair kernel: Lennard-Jones and Coulomb with
// ProtoMol's switching functions (OneAtomPair / OneAtomPairTwo,
// force/OneAtomPairTwo.h:30-100) and the Ewald real-space term
// (NonbondedFullEwaldSystemForce::realTerm, .h:753-858), over the
// cluster-pair list (8 x 4 atom tiles, one pair per lane, each unordered
// pair listed once).
//
// Arithmetic:
//   * forces: the kernel precision Real (FP32 in the mixed mode) from
//     hi/lo-split FP64 coordinates; pairs whose FP32 distance lies within a
//     relative band of a cutoff are re-tested with the reference's exact
//     FP64 arithmetic, so the accepted pair set is the reference's;
//   * energies and virial: only when requested (ProtoMol's energies are
//     observed at output steps), and then in FP64 from the FP64 wrapped
//     coordinates, because FP32 rounding of large cancelling pair energies
//     alone leaves a relative error near 1e-5 on the Ewald real-space sum;
//   * Cn switching: its polynomial in (r - rc) has large alternating
//     coefficients (switch/CnSwitchingFunction.cpp:9-23), so it is evaluated
//     in FP64 in every mode.
#pragma once

#include "pm_device.cuh"

namespace pmgpu {

template <typename Real>
struct PairArgs {
  Box box;
  int n;
  int ntypes;
  int mask;
  SwitchDev<Real> lj_sw, coul_sw;
  SwitchDev<double> lj_sw64, coul_sw64;
  int lj_modify, coul_modify;
  // rough-test cutoffs^2 (FP64 exact and the kernel-precision band)
  double lj_cut2, coul_cut2, ew_cut2, max_cut2;
  Real lj_lo, lj_hi, coul_lo, coul_hi, ew_lo, ew_hi, max_lo, max_hi;
  int same_cut;          // all active terms share one cutoff
  int minimal_image;     // LJ / Coulomb cutoff terms only for the minimal image
  Real half_edge[3];
  Real alpha, a2pi;
  double alpha64, a2pi64;
  int exact_erf;
  Real csf;  // coulomb scaling factor
  double csf64;
  int cap;              // tiles per row
  int nclusters;        // 8-atom i clusters (kRowParts tile rows each)
  int splits;           // warps per i cluster
  const int *sorted;
  const double *pos;     // raw positions (exact re-test)
  const int *excl_start, *excl_partner, *excl_class;
  const uint2 *tiles;
  const unsigned *tmod;  // modified masks of flagged tiles
  const uint2 *jlanes;   // j-lane entries (force-only kernel)
  const float4 *ewtab;   // Ewald real-space force table (null: analytic)
  const int *jl_count;   // entries per row
  const int *tile_count;
  const float4 *xhi, *xlo;
  const double4 *xw;
  const int *type;
  const float4 *lj32;
  const double4 *lj64;
  long long *fslot;      // 3 planes of ns: forces by list slot (added to the
                         // atoms' forces by k_slot_forces)
  int ns;                // slots (plane stride of fslot)
  long long *acc;
  long long *pairbuf;
  long long pairbuf_cap;
  long long *paircount;
  int count_pairs;       // accumulate the accepted-pair count
  int energy_only;       // energies (and virial) only: the forces come from the
                         // force-only kernel launched beside
};

// Exact FP64 squared distance of the image in hand, formed the way the
// reference forms it: the minimal difference (PeriodicBoundaryConditions.h:
// 72-110) plus a lattice vector (NonbondedFullEwaldSystemForce.h:790-805;
// for orthogonal boxes lattice components are exactly e_c * k_c).  d is the
// kernel's own difference, used only to pick the lattice vector.
template <typename Real>
__device__ __forceinline__ double exact_r2(const PairArgs<Real> &a, int oi, int oj,
                                           double dx, double dy, double dz) {
  double mx, my, mz;
  double r2 = box_mindiff(a.box, a.pos[3 * oi], a.pos[3 * oi + 1], a.pos[3 * oi + 2],
                          a.pos[3 * oj], a.pos[3 * oj + 1], a.pos[3 * oj + 2], mx, my, mz);
  if (!a.box.periodic) return r2;
  double kx = rint((dx - mx) * a.box.er[0]);
  double ky = rint((dy - my) * a.box.er[1]);
  double kz = rint((dz - mz) * a.box.er[2]);
  if (kx == 0.0 && ky == 0.0 && kz == 0.0) return r2;
  return xnorm2(xadd(mx, xmul(a.box.e[0], kx)), xadd(my, xmul(a.box.e[1], ky)),
                xadd(mz, xmul(a.box.e[2], kz)));
}

__device__ __forceinline__ float fast_exp(float x) { return __expf(x); }
__device__ __forceinline__ double fast_exp(double x) { return exp(x); }

template <typename Real>
__device__ __forceinline__ void apply_switch(const SwitchDev<Real> &sw,
                                             const SwitchDev<double> &sw64, Real r2,
                                             Real &ff, Real &en) {
  Real sv, sd;
  // the Cn and CmpCnCn polynomials cancel in FP32: evaluated in FP64
  if (sizeof(Real) == 4 && (sw.kind == PMGPU_SW_CN || sw.kind == PMGPU_SW_CMPCNCN)) {
    double v64, d64;
    switch_eval<double>(sw64, (double)r2, v64, d64);
    sv = (Real)v64;
    sd = (Real)d64;
  } else {
    switch_eval<Real>(sw, r2, sv, sd);
  }
  ff = ff * sv - en * sd;
  en = en * sv;
}

// Compile-time description of a pair-kernel instantiation's switching
// functions and erfc variant; -1 means "read from the arguments at run
// time".  The force-only FP32 kernel of the common configurations is
// specialised so that the per-pair arithmetic carries no run-time dispatch.
constexpr int kSwNone = 9;  // switch not applied (Universal, Cutoff: MODIFY = 0)
template <int LJK, int CK, int EXACT>
struct PairSpec {
  static constexpr int lj = LJK, coul = CK, exact = EXACT;
};
using GenericSpec = PairSpec<-1, -1, -1>;

template <typename Real, int KIND>
__device__ __forceinline__ void switch_k(const SwitchDev<Real> &sw, const SwitchDev<double> &sw64,
                                         int modify, Real r2, Real &ff, Real &en) {
  if (KIND < 0) {
    if (modify) apply_switch<Real>(sw, sw64, r2, ff, en);
  } else if (KIND == PMGPU_SW_C2) {
    // C2SwitchingFunction::operator() (switch/C2SwitchingFunction.h:42-52)
    if (r2 > sw.cutoff2) {
      ff = Real(0);
      en = Real(0);
    } else if (r2 >= sw.switchon2) {
      Real c2 = sw.cutoff2 - r2;
      Real c4 = c2 * (sw.s2 + Real(2) * r2);
      Real val = sw.s1 * (c2 * c4);
      Real der = sw.s3 * (c2 * c2 - c4);
      ff = ff * val - en * der;
      en = en * val;
    }
  } else if (KIND == PMGPU_SW_C1) {
    Real val, der;
    switch_eval<Real>(sw, r2, val, der);
    ff = ff * val - en * der;
    en = en * val;
  }
}

// Per-pair flags of an accepted pair: which terms are inside their cutoff,
// and whether the pair is a modified (scaled 1-4) one.
constexpr int kQLJ = 1, kQCoul = 2, kQEwald = 4, kQModified = 8;

// Pair force, energies of one accepted pair (the terms' arithmetic of
// OneAtomPairTwo::doOneAtomPair, force/OneAtomPairTwo.h:55-100).
// Returns f with F_i -= d * f.
template <typename Real, int TERMS, typename SPEC>
__device__ __forceinline__ Real pair_force(const PairArgs<Real> &a, const Real *ljrow, Real r2,
                                           Real qq, int tj, int flags, Real &en_lj,
                                           Real &en_c) {
  const bool modified = flags & kQModified;
  const Real rinv = rsqrt_nr(r2);
  const Real rinv2 = rinv * rinv;
  Real f = 0;
  if ((TERMS & TERM_LJ) && (flags & kQLJ)) {
    Real A, B;
    if (sizeof(Real) == 4) {
      float4 p = __ldg(reinterpret_cast<const float4 *>(ljrow) + tj);
      A = modified ? p.z : p.x;
      B = modified ? p.w : p.y;
    } else {
      double4 p = reinterpret_cast<const double4 *>(ljrow)[tj];
      A = modified ? p.z : p.x;
      B = modified ? p.w : p.y;
    }
    // LennardJonesForce::operator() (force/LennardJonesForce.h:28-60)
    Real r6 = rinv2 * rinv2 * rinv2;
    Real r6B = B * r6;
    Real r12A = A * r6 * r6;
    Real en = r12A - r6B;
    Real ff = (Real(12) * r12A - Real(6) * r6B) * rinv2;
    switch_k<Real, SPEC::lj>(a.lj_sw, a.lj_sw64, a.lj_modify, r2, ff, en);
    en_lj += en;
    f += ff;
  }
  if (modified) qq *= a.csf;
  if ((TERMS & TERM_COUL) && (flags & kQCoul)) {
    // CoulombForce::operator() (force/CoulombForce.h:29-40)
    Real en = qq * rinv;
    Real ff = en * rinv2;
    switch_k<Real, SPEC::coul>(a.coul_sw, a.coul_sw64, a.coul_modify, r2, ff, en);
    en_c += en;
    f += ff;
  }
  if ((TERMS & TERM_EWALD) && (flags & kQEwald)) {
    // NonbondedFullEwaldSystemForce::realTerm (:820-842)
    Real r = r2 * rinv;
    Real ar = a.alpha * r;
    Real ee = qq * fast_exp(-ar * ar);
    Real en;
    if (SPEC::exact == 0 || (SPEC::exact < 0 && !a.exact_erf))
      en = poly5_fast<Real>(ar) * ee * rinv;  // A&S erfc (MathUtilities.cpp:39-49)
    else
      en = qq * erfc(ar) * rinv;  // USE_EWALD_EXACT_ERF: C library erfc
    f += (en + a.a2pi * ee) * rinv2;
    en_c += en;
  }
  return f;
}

// Switch of a force-only specialised kernel, without branches: the value
// and derivative of every region are formed and the region's selected
// (C2SwitchingFunction.h:42-52, C1SwitchingFunction.h:41-50).  rinv is
// 1/sqrt(r2).
template <typename Real, int KIND>
__device__ __forceinline__ void switch_fast(const SwitchDev<Real> &sw, Real r2, Real rinv,
                                            Real &ff, Real en) {
  if (KIND == PMGPU_SW_C2) {
    // the polynomial is 1 with zero slope at the switch-on distance and 0
    // with zero slope at the cutoff, so r^2 clamped into [rs^2, rc^2] gives
    // every region's value and derivative (to rounding) without selects
    const Real r2c = fmin(fmax(r2, sw.switchon2), sw.cutoff2);
    const Real c2 = sw.cutoff2 - r2c;
    const Real c4 = c2 * (sw.s2 + Real(2) * r2c);
    const Real val = sw.s1 * (c2 * c4);
    const Real der = sw.s3 * (c2 * c2 - c4);
    ff = ff * val - en * der;
  } else if (KIND == PMGPU_SW_C1) {
    const Real d = r2 * rinv;
    const bool off = r2 > sw.cutoff2;
    const Real val = off ? Real(0) : Real(1) - d * (sw.c1a - r2 * sw.c1b);
    const Real der = off ? Real(0) : -sw.c1a * rinv + d * sw.c1c;
    ff = ff * val - en * der;
  }
}

// Pair force of the force-only specialised kernels: every term inside its
// (common) cutoff, no energies, no branches.  Same arithmetic as
// pair_force.  p holds the pair's LJ table entry (A, B, A14, B14).
template <typename Real, int TERMS, typename SPEC, bool MOD, typename P4>
__device__ __forceinline__ Real pair_force_p(const PairArgs<Real> &a, const P4 &p, Real r2,
                                             Real qq, bool modified) {
  const Real rinv = rsqrt_nr(r2);
  const Real rinv2 = rinv * rinv;
  Real f = 0;
  if (TERMS & TERM_LJ) {
    const Real A = MOD && modified ? p.z : p.x;
    const Real B = MOD && modified ? p.w : p.y;
    const Real r6 = rinv2 * rinv2 * rinv2;
    const Real r6B = B * r6;
    const Real r12A = A * r6 * r6;
    Real ff = (Real(12) * r12A - Real(6) * r6B) * rinv2;
    switch_fast<Real, SPEC::lj>(a.lj_sw, r2, rinv, ff, r12A - r6B);
    f += ff;
  }
  if (MOD) qq = modified ? qq * a.csf : qq;
  if (TERMS & TERM_COUL) {
    const Real en = qq * rinv;
    Real ff = en * rinv2;
    switch_fast<Real, SPEC::coul>(a.coul_sw, r2, rinv, ff, en);
    f += ff;
  }
  if (TERMS & TERM_EWALD) {
    const Real ar = a.alpha * (r2 * rinv);
    const Real ee = qq * fast_exp(-ar * ar);
    const Real en = SPEC::exact == 0 ? poly5_fast<Real>(ar) * ee * rinv : qq * erfc(ar) * rinv;
    f += (en + a.a2pi * ee) * rinv2;
  }
  return f;
}

// pair_force_p of the LJ + Ewald real force-only kernel with the Ewald
// factor read from the force table (kEwTabN cubics in shared memory): no
// square root, exponential or erfc per pair.  r2 must lie in the table's
// range [2^kEwTabLoExp, 2^(kEwTabLoExp + kEwTabOctaves)); others read the
// nearest end interval (the callers keep them out of the accepted pairs).
template <typename SPEC, bool MOD>
__device__ __forceinline__ float pair_force_tab(const PairArgs<float> &a, const float4 &p,
                                                float r2, float qq, bool modified,
                                                const float4 *s_ew) {
  const float rinv2 = __fdividef(1.f, r2);
  const float A = MOD && modified ? p.z : p.x;
  const float B = MOD && modified ? p.w : p.y;
  const float r6 = rinv2 * rinv2 * rinv2;
  const float r6B = B * r6;
  const float r12A = A * r6 * r6;
  float ff = (12.f * r12A - 6.f * r6B) * rinv2;
  switch_fast<float, SPEC::lj>(a.lj_sw, r2, 0.f, ff, r12A - r6B);
  if (MOD) qq = modified ? qq * a.csf : qq;
  const unsigned bits = __float_as_uint(r2);
  const int idx = min(max((int)(bits >> (23 - kEwTabSubBits)) - (int)kEwTabBase, 0), kEwTabN - 1);
  const float t =
      __uint_as_float(((bits << kEwTabSubBits) & 0x007FFFFFu) | 0x3F800000u) - 1.f;
  const float4 c = s_ew[idx];
  return fmaf(qq, fmaf(t, fmaf(t, fmaf(t, c.w, c.z), c.y), c.x), ff);
}

template <typename Real, int TERMS, typename SPEC, bool MOD>
__device__ __forceinline__ Real pair_force_fast(const PairArgs<Real> &a, const Real *ljrow,
                                                Real r2, Real qq, int tj, bool modified) {
  if (sizeof(Real) == 4) {
    const float4 p = __ldg(reinterpret_cast<const float4 *>(ljrow) + tj);
    return pair_force_p<Real, TERMS, SPEC, MOD>(a, p, r2, qq, modified);
  }
  const double4 p = reinterpret_cast<const double4 *>(ljrow)[tj];
  return pair_force_p<Real, TERMS, SPEC, MOD>(a, p, r2, qq, modified);
}

// FP64 energies (and, for the virial, the FP64 pair force) of one accepted
// pair from the FP64 wrapped coordinates: the observables of output steps
// in the mixed-precision path.
template <typename Real, int TERMS, bool FORCE64>
__device__ __forceinline__ void pair_energy64(const PairArgs<Real> &a, const double4 &wi,
                                              const double4 &wj, int shift, int ti, int tj,
                                              int flags, double &Elj, double &Ec,
                                              double *V) {
  const int sx = (shift & 3) - 1, sy = ((shift >> 2) & 3) - 1, sz = ((shift >> 4) & 3) - 1;
  double ex = wj.x - (wi.x - sx * a.box.e[0]);
  double ey = wj.y - (wi.y - sy * a.box.e[1]);
  double ez = wj.z - (wi.z - sz * a.box.e[2]);
  double r2e = ex * ex + ey * ey + ez * ez;
  double rr2 = 1.0 / r2e;
  double f = 0.0;
  const bool modified = flags & kQModified;
  if ((TERMS & TERM_LJ) && (flags & kQLJ)) {
    double4 p = a.lj64[ti * a.ntypes + tj];
    double A = modified ? p.z : p.x;
    double B = modified ? p.w : p.y;
    double r6 = rr2 * rr2 * rr2;
    double en = A * r6 * r6 - B * r6;
    double ff = FORCE64 ? (12.0 * A * r6 * r6 - 6.0 * B * r6) * rr2 : 0.0;
    if (a.lj_modify) {
      double sv, sd;
      switch_eval<double>(a.lj_sw64, r2e, sv, sd);
      ff = ff * sv - en * sd;
      en *= sv;
    }
    Elj += en;
    f += ff;
  }
  double qq = wi.w * wj.w;
  if (modified) qq *= a.csf64;
  if ((TERMS & TERM_COUL) && (flags & kQCoul)) {
    double en = qq * sqrt(rr2);
    double ff = en * rr2;
    if (a.coul_modify) {
      double sv, sd;
      switch_eval<double>(a.coul_sw64, r2e, sv, sd);
      ff = ff * sv - en * sd;
      en *= sv;
    }
    Ec += en;
    f += ff;
  }
  if ((TERMS & TERM_EWALD) && (flags & kQEwald)) {
    double r = sqrt(r2e);
    double ar = a.alpha64 * r;
    double ee = qq * exp(-ar * ar);
    double en = !a.exact_erf ? poly5<double>(ar) * ee / r : qq * erfc(ar) / r;
    Ec += en;
    f += (en + a.a2pi64 * ee) * rr2;
  }
  if (FORCE64) {
    // addVirial(fij, d) with fij = d * f (each pair is listed once)
    V[0] += ex * ex * f; V[1] += ex * ey * f; V[2] += ex * ez * f;
    V[3] += ey * ey * f; V[4] += ey * ez * f; V[5] += ez * ez * f;
  }
}

// Registers: the specialised force-only FP32 kernels (the inner MD steps)
// are held to 48 so five blocks fit per SM, the generic force-only FP32
// kernel to 64; energy/virial/record and FP64 variants get more.
template <typename Real, int MODE, typename SPEC>
struct PairOccupancy {
  static constexpr bool fast = MODE == PAIR_FORCE && sizeof(Real) == 4 && SPEC::lj >= 0 &&
                               SPEC::exact >= 0;
  static constexpr int warps = fast ? 40 : ((MODE == PAIR_FORCE && sizeof(Real) == 4) ? 32 : 16);
  static constexpr int blocks = warps / kPairWarps;
};

// Sum of (x, y, z) over the 8 lanes that share lane >> 3, transposed: on
// return lane l holds component (l & 3) of its group's sum (x, y, z, 0).
// Four shuffles instead of nine.
template <typename Real>
__device__ __forceinline__ Real group8_sum3(Real x, Real y, Real z, int lane) {
  const bool b0 = lane & 1, b1 = lane & 2;
  // xor 1: even lanes keep (x, z), odd lanes keep (y, 0)
  const Real k0 = b0 ? y : x, s0 = b0 ? x : y;
  const Real k1 = b0 ? Real(0) : z, s1 = b0 ? z : Real(0);
  const Real r0 = k0 + __shfl_xor_sync(0xffffffffu, s0, 1);
  const Real r1 = k1 + __shfl_xor_sync(0xffffffffu, s1, 1);
  // xor 2: lanes with bit 1 clear keep r0, the others r1
  Real v = (b1 ? r1 : r0) + __shfl_xor_sync(0xffffffffu, b1 ? r0 : r1, 2);
  v += __shfl_xor_sync(0xffffffffu, v, 4);
  return v;
}

__device__ __forceinline__ long long fixed_force(float v) {
  return __float2ll_rn(v * 4294967296.0f);  // exact scaling by 2^32
}
__device__ __forceinline__ long long fixed_force(double v) { return to_fixed(v, kForceScale); }

// One warp per (8-atom i cluster, contiguous share of its tiles).  Lane
// l holds pair (i atom l & 7, j atom l >> 3) of every 8 x 4 tile, so a
// tile's 32 pairs are evaluated at once with no compaction.  The list holds
// each unordered pair once, so the pair force goes to both atoms: i's
// share accumulates in the lane over the warp's tiles, j's share is summed
// over the 8 lanes of the same j atom and added with one fixed-point
// atomic per component.  Energies and virial count every pair once.
// Pairs are accepted by the cutoff tests of the reference (with the exact
// FP64 re-test near a cutoff); the tile mask carries the list's exclusion
// and modified (scaled 1-4) status.
template <typename Real, int TERMS, int MODE, typename SPEC>
__device__ __forceinline__ void pairs_body(const PairArgs<Real> &a, Blk blk) {
  constexpr bool MIXED = sizeof(Real) == 4;
  constexpr bool ENERGY = MODE != PAIR_FORCE;
  constexpr bool VIRIAL = MODE == PAIR_VIRIAL;
  constexpr bool RECORD = MODE == PAIR_RECORD;
  // force-only kernels of a specialised configuration (launched only when
  // every term shares one cutoff and the box holds twice the cutoff): every
  // accepted pair takes every term, evaluated without branches
  constexpr bool FAST = MIXED && MODE == PAIR_FORCE && SPEC::lj >= 0 && SPEC::exact >= 0;
  constexpr unsigned kAll = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int il = lane & 7, jl = lane >> 3;
  const unsigned lanebit = 1u << lane;        // this lane's bit of a tile mask
  const unsigned jbyte = 0xFFu << (8 * jl);   // the 8 lanes of this lane's j atom
  const bool jcomp = il < 3;                  // lane adds j's force component il
  double Elj = 0, Ec = 0;
  double V64[6] = {0, 0, 0, 0, 0, 0};
  Real vxx = 0, vxy = 0, vxz = 0, vyy = 0, vyz = 0, vzz = 0;
  int npairs = 0;
  // work items (i cluster, share of its tiles); the warps of a smaller
  // grid stride over them
  const int nitems = a.nclusters * a.splits;
  for (int gw = blk.x * kPairWarps + (threadIdx.x >> 5); gw < nitems;
       gw += blk.n * kPairWarps) {
  const int ci = gw / a.splits, sp = gw - ci * a.splits;
  // the cluster's tiles are its kRowParts rows read one after the other;
  // this warp takes tiles [t0, t1) of that sequence
  static_assert(kRowParts == 4, "one int4 of row counts per cluster");
  const int4 c4 = *reinterpret_cast<const int4 *>(a.tile_count + kRowParts * ci);
  const int cnt = c4.x + c4.y + c4.z + c4.w;
  const int t0 = (int)((long long)cnt * sp / a.splits);
  const int t1 = (int)((long long)cnt * (sp + 1) / a.splits);
  if (t1 <= t0) continue;
  const int islot = 8 * ci + il;
  const int oi = a.sorted[islot];
  const double4 wi = a.xw[islot];  // energy modes and the FP64 kernel only
  Real xi_h[3], xi_l[3];
  Real qi;
  int ti;
  if (MIXED) {
    const float4 h = a.xhi[islot], l = a.xlo[islot];
    xi_h[0] = h.x; xi_h[1] = h.y; xi_h[2] = h.z; qi = h.w;
    xi_l[0] = l.x; xi_l[1] = l.y; xi_l[2] = l.z; ti = __float_as_int(l.w);
  } else {
    xi_h[0] = wi.x; xi_h[1] = wi.y; xi_h[2] = wi.z; qi = wi.w;
    xi_l[0] = xi_l[1] = xi_l[2] = Real(0);
    ti = oi >= 0 ? a.type[oi] : 0;
  }
  const Real *ljrow = MIXED ? reinterpret_cast<const Real *>(a.lj32 + ti * a.ntypes)
                            : reinterpret_cast<const Real *>(a.lj64 + ti * a.ntypes);
  // i as seen from the tile's image of j (d = xj - (xi - s L))
  int cur = kZeroShift;
  Real xs_h[3] = {xi_h[0], xi_h[1], xi_h[2]};
  Real xs_l[3] = {xi_l[0], xi_l[1], xi_l[2]};
  Real fx = 0, fy = 0, fz = 0;
  constexpr int kAllTerms = ((TERMS & TERM_LJ) ? kQLJ : 0) | ((TERMS & TERM_COUL) ? kQCoul : 0) |
                            ((TERMS & TERM_EWALD) ? kQEwald : 0);
  // tile t0 is index kb of row part p; the warp walks the parts in order
  int p = 0, kb = t0, rowlen = c4.x;
  while (kb >= rowlen) {
    kb -= rowlen;
    p++;
    rowlen = p == 1 ? c4.y : (p == 2 ? c4.z : c4.w);
  }
  for (int left = t1 - t0; left > 0;) {
    const size_t row0 = (size_t)(kRowParts * ci + p) * a.cap;
    const uint2 *row = a.tiles + row0;
    const int ke = min(rowlen, kb + left);
    left -= ke - kb;
  for (int k = kb; k < ke; k++) {
    const uint2 t2 = __ldg(row + k);
    const uint3 tile = make_uint3(t2.x, t2.y,
                                  (t2.x & kModFlag) ? __ldg(a.tmod + row0 + k) : 0u);
    const int hj = (int)(tile.x & kJMask);
    const int sh = (int)((tile.x >> kShiftBits) & kShiftMask);
    if (__any_sync(kAll, sh != cur)) {  // tiles are grouped by image
      const int sx = (sh & 3) - 1, sy = ((sh >> 2) & 3) - 1, sz = ((sh >> 4) & 3) - 1;
      // reloaded rather than held in registers through the loop
      const double4 w = a.xw[islot];
      const double xs64[3] = {w.x - sx * a.box.e[0], w.y - sy * a.box.e[1],
                              w.z - sz * a.box.e[2]};
      for (int c = 0; c < 3; c++) {
        if (MIXED) {
          const float h = (float)xs64[c];
          xs_h[c] = h;
          xs_l[c] = (float)(xs64[c] - (double)h);
        } else {
          xs_h[c] = xs64[c];
        }
      }
      cur = sh;
    }
    const int jslot = 4 * hj + jl;
    const bool live = (tile.y & lanebit) != 0u;
    Real dx, dy, dz, qj;
    int tj = 0;
    if (MIXED) {
      const float4 h = a.xhi[jslot], l = a.xlo[jslot];
      dx = (h.x - xs_h[0]) + (l.x - xs_l[0]);
      dy = (h.y - xs_h[1]) + (l.y - xs_l[1]);
      dz = (h.z - xs_h[2]) + (l.z - xs_l[2]);
      qj = h.w;
      tj = __float_as_int(l.w);
    } else {
      const double4 wj = a.xw[jslot];
      dx = wj.x - xs_h[0];
      dy = wj.y - xs_h[1];
      dz = wj.z - xs_h[2];
      qj = wj.w;
    }
    const Real r2 = dx * dx + dy * dy + dz * dz;
    if constexpr (FAST) {
      bool act = live && r2 <= a.max_lo;
      const bool band = live && !act && r2 <= a.max_hi;
      if (__any_sync(kAll, band)) {
        if (band)
          act = exact_r2(a, oi, a.sorted[jslot], (double)dx, (double)dy, (double)dz) <=
                a.max_cut2;
      }
      const unsigned actm = __ballot_sync(kAll, act);
      if (a.count_pairs) npairs += act;
      if (!actm) continue;
      const Real rr = act ? r2 : Real(1);
      Real f;
      // modified (scaled 1-4) pairs are rare: tiles without any take the
      // path without their selects (the mask is the tile's, so the branch
      // is uniform)
      if (__any_sync(kAll, tile.z != 0u))
        f = pair_force_fast<Real, TERMS, SPEC, true>(a, ljrow, rr, qi * qj, tj,
                                                     (tile.z & lanebit) != 0u);
      else
        f = pair_force_fast<Real, TERMS, SPEC, false>(a, ljrow, rr, qi * qj, tj, false);
      f = act ? f : Real(0);
      const Real jx = dx * f, jy = dy * f, jz = dz * f;
      fx -= jx;
      fy -= jy;
      fz -= jz;
      const Real js = group8_sum3<Real>(jx, jy, jz, lane);
      // address and value formed by every lane, one predicated atomic
      long long *dst = a.fslot + il * a.ns + jslot;
      const long long v = fixed_force(js);
      if (jcomp && (actm & jbyte)) red_add(dst, v);
      continue;
    }
    int flags = 0;
    bool band = false;
    if (live && a.same_cut) {  // every term shares one cutoff
      if (r2 <= a.max_lo) flags = kAllTerms;
      else band = r2 <= a.max_hi;
    } else if (live) {
      if (TERMS & TERM_LJ) {
        if (r2 <= a.lj_lo) flags |= kQLJ;
        else band |= r2 <= a.lj_hi;
      }
      if (TERMS & TERM_COUL) {
        if (r2 <= a.coul_lo) flags |= kQCoul;
        else band |= r2 <= a.coul_hi;
      }
      if (TERMS & TERM_EWALD) {
        if (r2 <= a.ew_lo) flags |= kQEwald;
        else band |= r2 <= a.ew_hi;
      }
    }
    // pairs within a rounding band of a cutoff take the reference's exact
    // FP64 test (rare: a real branch)
    if (__any_sync(kAll, band)) {
      if (band) {
        const double r2x = exact_r2(a, oi, a.sorted[jslot], (double)dx, (double)dy, (double)dz);
        if ((TERMS & TERM_LJ) && r2 > a.lj_lo && r2x <= a.lj_cut2) flags |= kQLJ;
        if ((TERMS & TERM_COUL) && r2 > a.coul_lo && r2x <= a.coul_cut2) flags |= kQCoul;
        if ((TERMS & TERM_EWALD) && r2 > a.ew_lo && r2x <= a.ew_cut2) flags |= kQEwald;
      }
    }
    // boxes below twice the cutoff: cutoff terms take the minimal image only
    // (Ewald real space sums every image, NonbondedFullEwaldSystemForce.h:790)
    if ((TERMS & (TERM_LJ | TERM_COUL)) && a.minimal_image && (flags & (kQLJ | kQCoul)) &&
        !(fabs(dx) <= a.half_edge[0] && fabs(dy) <= a.half_edge[1] &&
          fabs(dz) <= a.half_edge[2]))
      flags &= ~(kQLJ | kQCoul);
    Real jx = 0, jy = 0, jz = 0;
    // an energy-only pass (the forces of the step come from the force-only
    // kernel) skips the FP32 force and the j-force sums
    const bool forces = !(MIXED && ENERGY && a.energy_only);
    if (flags) {
      if ((tile.z >> lane) & 1u) flags |= kQModified;
      if (!MIXED) tj = a.type[a.sorted[jslot]];
      Real en_lj = 0, en_c = 0;
      if (forces) {
        const Real f =
            pair_force<Real, TERMS, SPEC>(a, ljrow, r2, qi * qj, tj, flags, en_lj, en_c);
        jx = dx * f;
        jy = dy * f;
        jz = dz * f;
        fx -= jx;
        fy -= jy;
        fz -= jz;
      }
      npairs++;
      if (ENERGY) {
        if (MIXED) {
          pair_energy64<Real, TERMS, VIRIAL>(a, wi, a.xw[jslot], sh, ti, tj, flags, Elj, Ec,
                                             V64);
        } else {
          Elj += (double)en_lj;
          Ec += (double)en_c;
        }
      }
      if (VIRIAL && !MIXED) {
        // addVirial(fij, d) with fij = d * f
        vxx += dx * jx; vxy += dx * jy; vxz += dx * jz;
        vyy += dy * jy; vyz += dy * jz; vzz += dz * jz;
      }
      if (RECORD) {
        const int oj = a.sorted[jslot];
        if (oi != oj) {
          long long slot = atomicAdd((unsigned long long *)a.paircount, 1ull);
          if (slot < a.pairbuf_cap)
            a.pairbuf[slot] = ((long long)min(oi, oj) << 32) | (unsigned)max(oi, oj);
        }
      }
    }
    // j's share: summed over its 8 lanes, one atomic per component
    if (forces) {
      const unsigned act = __ballot_sync(kAll, flags != 0);
      const Real js = group8_sum3<Real>(jx, jy, jz, lane);
      long long *dst = a.fslot + il * a.ns + jslot;
      const long long v = fixed_force(js);
      if (il < 3 && ((act >> (8 * jl)) & 0xFFu)) red_add(dst, v);
    }
  }
    if (left > 0) {  // next non-empty row part
      do {
        p++;
        rowlen = __ldg(a.tile_count + kRowParts * ci + p);
      } while (rowlen == 0);
      kb = 0;
    }
  }
  // i's share: summed over the 4 j lanes of each i atom
#pragma unroll
  for (int o = 8; o < 32; o <<= 1) {
    fx += __shfl_xor_sync(kAll, fx, o);
    fy += __shfl_xor_sync(kAll, fy, o);
    fz += __shfl_xor_sync(kAll, fz, o);
  }
  if (jl == 0 && oi >= 0 && !a.energy_only) {
    red_add(&a.fslot[islot], fixed_force(fx));
    red_add(&a.fslot[a.ns + islot], fixed_force(fy));
    red_add(&a.fslot[2 * a.ns + islot], fixed_force(fz));
  }
  }  // work items
  if (ENERGY || a.count_pairs) {
    int np = warp_sum(npairs);
    if (lane == 0) red_add(&a.acc[ACC_PAIRS], (long long)np);
  }
  if (ENERGY) {
    double dlj = warp_sum(Elj);
    double dc = warp_sum(Ec);
    double V[6] = {0, 0, 0, 0, 0, 0};
    if (VIRIAL) {
      if (MIXED) {
        for (int q = 0; q < 6; q++) V[q] = warp_sum(V64[q]);
      } else {
        V[0] = warp_sum((double)vxx); V[1] = warp_sum((double)vxy);
        V[2] = warp_sum((double)vxz); V[3] = warp_sum((double)vyy);
        V[4] = warp_sum((double)vyz); V[5] = warp_sum((double)vzz);
      }
    }
    if (lane == 0) {
      if (TERMS & TERM_LJ) red_add(&a.acc[ACC_LJ], to_fixed(dlj, kEnergyScale));
      if (TERMS & (TERM_COUL | TERM_EWALD))
        red_add(&a.acc[ACC_COULOMB], to_fixed(dc, kEnergyScale));
      if (VIRIAL) {
        const int map[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
        for (int q = 0; q < 9; q++)
          red_add(&a.acc[ACC_VIRIAL + q], to_fixed(V[map[q]], kEnergyScale));
      }
    }
  }
}

// The launch arguments of a batched launch's member, copied into shared
// memory by the block (every thread reads them many times).
template <typename A>
__device__ __forceinline__ const A &batch_args_shared(const A *__restrict__ tab, int m,
                                                      unsigned char *raw) {
  static_assert(sizeof(A) % 4 == 0, "argument structs are whole words");
  const int *src = reinterpret_cast<const int *>(tab + m);
  int *dst = reinterpret_cast<int *>(raw);
  for (int k = threadIdx.x; k < (int)(sizeof(A) / 4); k += blockDim.x) dst[k] = __ldg(src + k);
  __syncthreads();
  return *reinterpret_cast<const A *>(raw);
}

template <typename Real, int TERMS, int MODE, typename SPEC>
__global__ void __launch_bounds__(kPairWarps * 32, PairOccupancy<Real, MODE, SPEC>::blocks)
    k_pairs(PairArgs<Real> a) {
  pairs_body<Real, TERMS, MODE, SPEC>(a, own_blk());
}

template <typename Real, int TERMS, int MODE, typename SPEC>
__global__ void __launch_bounds__(kPairWarps * 32, PairOccupancy<Real, MODE, SPEC>::blocks)
    k_pairs_batch(const PairArgs<Real> *__restrict__ tab, const int *__restrict__ first, int nm) {
  __shared__ __align__(16) unsigned char raw[sizeof(PairArgs<Real>)];
  const int m = batch_member(first, nm, blockIdx.x);
  pairs_body<Real, TERMS, MODE, SPEC>(batch_args_shared(tab, m, raw), batch_blk(first, m));
}

// ---------------------------------------------------------------------------
// Force-only FP32 pair kernel of the inner MD steps, j atoms on the lanes.
//
// A warp takes the tiles of its work item (one 8-atom i cluster, a
// contiguous share of its tiles) eight at a time: lane l holds j atom l & 3
// of tile l >> 2 of the batch and evaluates its pairs with the cluster's 8
// i atoms one after another, the i atoms broadcast from shared memory.  A
// lane's j force is complete after those eight pairs and goes out with one
// fixed-point atomic per component.  The i forces stay in registers (8
// atoms x 3 components per lane) over all the tiles of the item and are
// summed over the lanes once, at its end, by transposed butterflies
// (warp_tsum8).  Against one pair per lane per tile (k_pairs) this leaves
// out the per-tile image bookkeeping, the per-tile j-force reduction and the
// tile-wide votes: the work per tile is the pair arithmetic and a few loads.
//
// Coordinates: FP32 vectors from the cluster's first atom, formed in FP64
// from the wrapped FP64 positions with the j atom's periodic image added in
// FP64, so each distance carries one FP32 rounding of vectors no longer
// than the reach plus the cluster extent.  Pairs within the relative band
// of the cutoff take the reference's exact FP64 test after the batch's
// pairs (rare), so the accepted set is the reference's.
constexpr int kJlWarps = 8;
constexpr int kJlMaxTypes = 16;  // LJ tables staged in shared memory up to this many types
constexpr int kJlMaxSplits = 16;  // warps one i cluster's tiles may be divided over
constexpr float kEwTabMin = 1.0f / (1 << -kEwTabLoExp);  // the table's lowest r^2

// The eight pairs of one lane's j atom with the cluster's i atoms (mi: the
// pairs of the list's interaction mask).
template <int TERMS, typename SPEC, bool MOD, bool SMEM_LJ, bool TAB>
__device__ __forceinline__ void jl_pairs8(const PairArgs<float> &a, const float4 *s_lj,
                                          const float4 *s_ew,
                                          const float4 *xi, const int *ti, float rjx, float rjy,
                                          float rjz, float qj, int tj, unsigned mi, unsigned mm,
                                          float (&fi)[8][3], float &fjx, float &fjy, float &fjz,
                                          unsigned &band, int &npairs) {
#pragma unroll
  for (int il = 0; il < 8; il++) {
    const float4 x = xi[il];
    const float dx = rjx - x.x, dy = rjy - x.y, dz = rjz - x.z;
    const float r2 = dx * dx + dy * dy + dz * dz;
    const bool on = (mi >> il) & 1u;
    // (table form: pairs closer than the table's range take the exact path)
    const bool act = on && r2 <= a.max_lo && (!TAB || r2 >= kEwTabMin);
    band |= (on && !act && r2 <= a.max_hi) ? (1u << il) : 0u;
    npairs += act;
    const float rr = act ? r2 : 1.f;
    const float4 p = SMEM_LJ ? s_lj[ti[il] + tj] : __ldg(a.lj32 + ti[il] + tj);
    float f;
    if constexpr (TAB)
      f = pair_force_tab<SPEC, MOD>(a, p, rr, x.w * qj, MOD && ((mm >> il) & 1u), s_ew);
    else
      f = pair_force_p<float, TERMS, SPEC, MOD>(a, p, rr, x.w * qj, MOD && ((mm >> il) & 1u));
    f = act ? f : 0.f;
    fjx = fmaf(dx, f, fjx);
    fjy = fmaf(dy, f, fjy);
    fjz = fmaf(dz, f, fjz);
    fi[il][0] = fmaf(-dx, f, fi[il][0]);
    fi[il][1] = fmaf(-dy, f, fi[il][1]);
    fi[il][2] = fmaf(-dz, f, fi[il][2]);
  }
}

// The j atoms' records of one warp step, staged by cp.async: the FP64
// wrapped position and charge, and the type.
struct JlStage {
  double4 w[32];
  int t[32];
};

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

template <int TERMS, typename SPEC, bool SMEM_LJ, bool TAB>
__device__ __forceinline__ void pairs_jl_body(const PairArgs<float> &a, Blk blk) {
  constexpr unsigned kAll = 0xffffffffu;
  __shared__ float4 s_lj[SMEM_LJ ? kJlMaxTypes * kJlMaxTypes : 1];
  __shared__ float4 s_ew[TAB ? kEwTabN : 1];
  __shared__ float4 s_xi[kJlWarps][8];   // i atoms from the reference point, charge
  __shared__ int s_ti[kJlWarps][8];      // i type * ntypes
  __shared__ int s_oi[kJlWarps][8];      // i atom (-1: padding)
  __shared__ double s_wc[kJlWarps][3];   // reference point (FP64)
  __shared__ JlStage s_js[kJlWarps][2];  // j-atom records of two warp steps
  if (SMEM_LJ)
    for (int k = threadIdx.x; k < a.ntypes * a.ntypes; k += blockDim.x) s_lj[k] = a.lj32[k];
  if (TAB)
    for (int k = threadIdx.x; k < kEwTabN; k += blockDim.x) s_ew[k] = __ldg(a.ewtab + k);
  if (SMEM_LJ || TAB) __syncthreads();
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  int npairs = 0;
  const int nitems = a.nclusters * a.splits;
  const size_t rowcap = 4 * (size_t)a.cap;  // entries per row
  for (int gw = blk.x * kJlWarps + wib; gw < nitems; gw += blk.n * kJlWarps) {
    const int ci = gw / a.splits, sp = gw - ci * a.splits;
    static_assert(kRowParts == 4, "one int4 of row counts per cluster");
    const int4 c4 = *reinterpret_cast<const int4 *>(a.jl_count + kRowParts * ci);
    const int p1 = c4.x, p2 = p1 + c4.y, p3 = p2 + c4.z, cnt = p3 + c4.w;
    const int t0 = (int)((long long)cnt * sp / a.splits);
    const int t1 = (int)((long long)cnt * (sp + 1) / a.splits);
    if (t1 <= t0) continue;
    __syncwarp();  // the previous item's reads of this warp's staging are done
    if (lane < 8) {
      const int islot = 8 * ci + lane;
      const double4 w0 = a.xw[8 * ci];  // a cluster with entries has an atom in its first slot
      const double4 wi = a.xw[islot];
      const int oi = a.sorted[islot];
      s_xi[wib][lane] = make_float4((float)(wi.x - w0.x), (float)(wi.y - w0.y),
                                    (float)(wi.z - w0.z), (float)wi.w);
      s_ti[wib][lane] = (oi >= 0 ? __float_as_int(__ldg(&a.xlo[islot].w)) : 0) * a.ntypes;
      s_oi[wib][lane] = oi;
      if (lane < 3) s_wc[wib][lane] = lane == 0 ? w0.x : (lane == 1 ? w0.y : w0.z);
    }
    __syncwarp();
    const float4 *xi = s_xi[wib];
    const int *ti = s_ti[wib];
    float fi[8][3];
#pragma unroll
    for (int k = 0; k < 8; k++) fi[k][0] = fi[k][1] = fi[k][2] = 0.f;
    // Software pipeline over the warp steps (32 entries each): the entries
    // of step k + 2 are loaded into registers and the j atoms' records of
    // step k + 1 are copied into this lane's shared-memory slot (cp.async)
    // while step k computes, so the dependent loads (entry, then the j
    // atom's record) are in flight during a whole step.  A lane reads only
    // the slot it copied itself.
    auto entry_at = [&](int idx) -> uint2 {
      if (idx >= t1) return make_uint2(0u, 0u);  // mask 0: no entry
      const int p = (idx >= p1) + (idx >= p2) + (idx >= p3);
      const int off = idx - (p == 0 ? 0 : (p == 1 ? p1 : (p == 2 ? p2 : p3)));
      return __ldg(a.jlanes + (size_t)(kRowParts * ci + p) * rowcap + off);
    };
    auto stage = [&](uint2 e, int buf) {
      if (e.y & 0xFFu) {
        const int js = (int)(e.x & kJSlotMask);
        JlStage &g = s_js[wib][buf];
        cp_async16(&g.w[lane], &a.xw[js]);
        cp_async16(reinterpret_cast<char *>(&g.w[lane]) + 16,
                   reinterpret_cast<const char *>(&a.xw[js]) + 16);
        cp_async4(&g.t[lane], &a.xlo[js].w);
      }
      cp_async_commit();
    };
    uint2 ecur = entry_at(t0 + lane), enext = entry_at(t0 + 32 + lane);
    stage(ecur, 0);
    for (int b0 = t0, k = 0; b0 < t1; b0 += 32, k++) {
      stage(enext, (k + 1) & 1);
      const uint2 enext2 = entry_at(b0 + 64 + lane);
      cp_async_wait<1>();  // this step's copies have landed
      unsigned mi = ecur.y & 0xFFu, mm = (ecur.y >> 8) & 0xFFu;
      const int jslot = (int)(ecur.x & kJSlotMask);
      int tj = 0;
      float rjx = 0.f, rjy = 0.f, rjz = 0.f, qj = 0.f;
      if (mi) {
        const JlStage &g = s_js[wib][k & 1];
        const double4 wj = g.w[lane];
        // the j atom in the entry's image (d = xj + s L - xi), from the
        // reference point; the image offsets are exact (-L, 0 or L)
        const int sh = (int)(ecur.x >> kJSlotBits);
        const int sx = sh & 3, sy = (sh >> 2) & 3, sz = (sh >> 4) & 3;
        const double ox = sx == 1 ? 0.0 : (sx == 0 ? -a.box.e[0] : a.box.e[0]);
        const double oy = sy == 1 ? 0.0 : (sy == 0 ? -a.box.e[1] : a.box.e[1]);
        const double oz = sz == 1 ? 0.0 : (sz == 0 ? -a.box.e[2] : a.box.e[2]);
        rjx = (float)((wj.x + ox) - s_wc[wib][0]);
        rjy = (float)((wj.y + oy) - s_wc[wib][1]);
        rjz = (float)((wj.z + oz) - s_wc[wib][2]);
        qj = (float)wj.w;
        tj = g.t[lane];
      }
      ecur = enext;
      enext = enext2;
      float fjx = 0.f, fjy = 0.f, fjz = 0.f;
      unsigned band = 0u;
      // modified (scaled 1-4) pairs are rare: batches without any take the
      // path without their selects
      if (__any_sync(kAll, mm != 0u))
        jl_pairs8<TERMS, SPEC, true, SMEM_LJ, TAB>(a, s_lj, s_ew, xi, ti, rjx, rjy, rjz, qj, tj,
                                                   mi, mm, fi,
                                              fjx, fjy, fjz, band, npairs);
      else
        jl_pairs8<TERMS, SPEC, false, SMEM_LJ, TAB>(a, s_lj, s_ew, xi, ti, rjx, rjy, rjz, qj, tj,
                                                    mi, mm,
                                               fi, fjx, fjy, fjz, band, npairs);
      // pairs within the rounding band of the cutoff: the exact FP64 test
      // (rare; their i forces go out as atomics, so this path keeps none of
      // the register-held sums live)
      if (__any_sync(kAll, band != 0u)) {
        const int oj = band ? a.sorted[jslot] : -1;
        while (band) {
          const int il = __ffs(band) - 1;
          band &= band - 1u;
          const float4 x = xi[il];
          const float dx = rjx - x.x, dy = rjy - x.y, dz = rjz - x.z;
          const float r2 = dx * dx + dy * dy + dz * dz;
          if (exact_r2(a, s_oi[wib][il], oj, (double)dx, (double)dy, (double)dz) > a.max_cut2)
            continue;
          const float4 p = SMEM_LJ ? s_lj[ti[il] + tj] : __ldg(a.lj32 + ti[il] + tj);
          const float f = pair_force_p<float, TERMS, SPEC, true>(a, p, r2, x.w * qj,
                                                                 (mm >> il) & 1u);
          fjx = fmaf(dx, f, fjx);
          fjy = fmaf(dy, f, fjy);
          fjz = fmaf(dz, f, fjz);
          long long *di = a.fslot + 8 * ci + il;
          red_add(di, fixed_force(-dx * f));
          red_add(di + a.ns, fixed_force(-dy * f));
          red_add(di + 2 * (size_t)a.ns, fixed_force(-dz * f));
          npairs++;
        }
      }
      if (mi) {
        long long *dst = a.fslot + jslot;
        red_add(dst, fixed_force(fjx));
        red_add(dst + a.ns, fixed_force(fjy));
        red_add(dst + 2 * (size_t)a.ns, fixed_force(fjz));
      }
    }
    cp_async_wait<0>();  // no copy of this item is left in flight
    // the i forces summed over the lanes: lane l ends with the totals of i
    // atom (l >> 2) & 7 and writes component l & 3
    float sum[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      float v[8];
#pragma unroll
      for (int k = 0; k < 8; k++) v[k] = fi[k][c];
      sum[c] = warp_tsum8(v, lane);
    }
    const int il = (lane >> 2) & 7, comp = lane & 3;
    if (comp < 3 && s_oi[wib][il] >= 0)
      red_add(&a.fslot[(size_t)comp * a.ns + 8 * ci + il],
              fixed_force(comp == 0 ? sum[0] : (comp == 1 ? sum[1] : sum[2])));
  }
  if (a.count_pairs) {
    const int np = warp_sum(npairs);
    if (lane == 0) red_add(&a.acc[ACC_PAIRS], (long long)np);
  }
}

template <int TERMS, typename SPEC, bool SMEM_LJ, bool TAB>
__global__ void __launch_bounds__(kJlWarps * 32, 3) k_pairs_jl(PairArgs<float> a) {
  pairs_jl_body<TERMS, SPEC, SMEM_LJ, TAB>(a, own_blk());
}

template <int TERMS, typename SPEC, bool SMEM_LJ, bool TAB>
__global__ void __launch_bounds__(kJlWarps * 32, 3)
    k_pairs_jl_batch(const PairArgs<float> *__restrict__ tab, const int *__restrict__ first,
                     int nm) {
  __shared__ __align__(16) unsigned char raw[sizeof(PairArgs<float>)];
  const int m = batch_member(first, nm, blockIdx.x);
  pairs_jl_body<TERMS, SPEC, SMEM_LJ, TAB>(batch_args_shared(tab, m, raw),
                                           batch_blk(first, m));
}

// Adds the forces accumulated by list slot into the atoms' forces and
// clears the slot buffer for the next launch.
struct SlotArgs {
  int ns, n;
  const int *sorted;
  long long *fslot, *force;
};
__device__ __forceinline__ void slot_forces_body(const SlotArgs &A, Blk b) {
  const int ns = A.ns, n = A.n;
  const int *__restrict__ sorted = A.sorted;
  long long *__restrict__ fslot = A.fslot;
  long long *__restrict__ force = A.force;
  const int s = b.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  const int i = sorted[s];
  if (i < 0) return;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const long long v = fslot[(size_t)c * ns + s];
    if (v) {
      red_add(&force[(size_t)c * n + i], v);
      fslot[(size_t)c * ns + s] = 0;
    }
  }
}
__global__ void k_slot_forces(SlotArgs a) {
  pdl_wait();  // the predecessor's writes are visible from here on
  slot_forces_body(a, own_blk());
}
__global__ void k_slot_forces_batch(const SlotArgs *__restrict__ tab, const int *__restrict__ first,
                                    int nm) {
  const int m = batch_member(first, nm, blockIdx.x);
  slot_forces_body(tab[m], batch_blk(first, m));
}

}  // namespace pmgpu
