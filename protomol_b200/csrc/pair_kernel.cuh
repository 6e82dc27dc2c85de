// The fused nonbonded pair kernel: Lennard-Jones and Coulomb with
// ProtoMol's switching functions (OneAtomPair / OneAtomPairTwo,
// force/OneAtomPairTwo.h:30-100) and the Ewald real-space term
// (NonbondedFullEwaldSystemForce::realTerm, .h:753-858), over full Verlet
// lists (warp per sorted atom, accepted pairs compacted in shared memory).
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
  double lj_cut2, coul_cut2, ew_cut2;
  Real lj_lo, lj_hi, coul_lo, coul_hi, ew_lo, ew_hi, max_lo, max_hi;
  int same_cut;          // all active terms share one cutoff
  int minimal_image;     // LJ / Coulomb cutoff terms only for the minimal image
  Real half_edge[3];
  Real alpha, a2pi;
  double alpha64, a2pi64;
  int exact_erf;
  Real csf;  // coulomb scaling factor
  double csf64;
  int cap;
  const int *sorted;
  const double *pos;     // raw positions (exact re-test)
  const int *excl_start, *excl_partner, *excl_class;
  const uint32_t *nbr;
  const int *nbr_count;
  const float4 *xhi, *xlo;
  const double4 *xw;
  const int *type;
  const float4 *lj32;
  const double4 *lj64;
  long long *force;      // 3 planes
  long long *acc;
  long long *pairbuf;
  long long pairbuf_cap;
  long long *paircount;
  int count_pairs;       // accumulate the accepted-pair count
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
// rsqrt with one Newton step: the bare MUFU estimate carries a small bias
// that would otherwise show in the summed forces.
__device__ __forceinline__ float rsqrt_nr(float x) {
  float y = rsqrtf(x);
  return y * (1.5f - 0.5f * x * y * y);
}
__device__ __forceinline__ double rsqrt_nr(double x) { return 1.0 / sqrt(x); }

template <typename Real>
__device__ __forceinline__ void apply_switch(const SwitchDev<Real> &sw,
                                             const SwitchDev<double> &sw64, Real r2,
                                             Real &ff, Real &en) {
  Real sv, sd;
  if (sizeof(Real) == 4 && sw.kind == PMGPU_SW_CN) {
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
    // addVirial(fij, d) with fij = d * f, half per visit
    double hf = 0.5 * f;
    V[0] += ex * ex * hf; V[1] += ex * ey * hf; V[2] += ex * ez * hf;
    V[3] += ey * ey * hf; V[4] += ey * ez * hf; V[5] += ez * ez * hf;
  }
}

// One warp per sorted atom i over its full neighbour row.  Phase 1: the 32
// lanes take 32 consecutive entries, form the distance, apply the cutoff
// tests (with the exact FP64 re-test near a cutoff) and compact the accepted
// pairs into a per-warp ring in shared memory.  Phase 2: whenever 32
// accepted pairs are queued, every lane evaluates one of them, so the
// expensive pair arithmetic runs with all lanes busy.  Each unordered pair
// is visited from both ends; forces are written for i only (no atomics on
// j), energies and virial are halved.
constexpr int kQueue = 64;

// Per-warp ring of accepted pairs: (dx, dy, dz, r2) and (j, type j, charge
// j, flags | image << 4).
template <typename Real> struct QueueVec;
template <> struct QueueVec<float> { using T = float4; };
template <> struct QueueVec<double> { using T = double4; };

template <typename Real>
struct PairQueue {
  typename QueueVec<Real>::T d[kPairWarps][kQueue];
  int4 m[kPairWarps][kQueue];
  Real qj[kPairWarps][kQueue];
};

// Registers: the force-only FP32 variant (the inner MD steps) is held to 64
// so four blocks fit per SM; energy/virial/record and FP64 variants get more.
template <typename Real, int MODE>
struct PairOccupancy {
  static constexpr int blocks = (MODE == PAIR_FORCE && sizeof(Real) == 4) ? 4 : 2;
};

template <typename Real, int TERMS, int MODE, typename SPEC>
__global__ void __launch_bounds__(kPairWarps * 32, PairOccupancy<Real, MODE>::blocks)
    k_pairs(PairArgs<Real> a) {
  constexpr bool MIXED = sizeof(Real) == 4;
  constexpr bool ENERGY = MODE != PAIR_FORCE;
  constexpr bool VIRIAL = MODE == PAIR_VIRIAL;
  constexpr bool RECORD = MODE == PAIR_RECORD;
  constexpr unsigned kAll = 0xffffffffu;
  __shared__ PairQueue<Real> Q;
  const int w = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const unsigned lt_mask = (1u << lane) - 1u;
  Real vxx = 0, vxy = 0, vxz = 0, vyy = 0, vyz = 0, vzz = 0;
  double Elj = 0, Ec = 0;
  double V64[6] = {0, 0, 0, 0, 0, 0};
  int npairs = 0;
  // Warps stride over the sorted atoms (the grid may be smaller than one
  // warp per atom, which leaves room on every SM for the work of the other
  // stream); no block-wide barrier below.
  for (int ii = blockIdx.x * kPairWarps + w; ii < a.n; ii += gridDim.x * kPairWarps) {
    const int cnt = a.nbr_count[ii];
    const uint32_t *row = a.nbr + (size_t)ii * a.cap;
    uint32_t e_next = lane < cnt ? __ldg(row + lane) : 0u;
    const int oi = a.sorted[ii];
    const double4 wi = a.xw[ii];
    Real xi_h[3], xi_l[3], qi;
    int ti;
    if (MIXED) {
      float4 h = a.xhi[ii], l = a.xlo[ii];
      xi_h[0] = h.x; xi_h[1] = h.y; xi_h[2] = h.z; qi = h.w;
      xi_l[0] = l.x; xi_l[1] = l.y; xi_l[2] = l.z; ti = __float_as_int(l.w);
    } else {
      xi_h[0] = wi.x; xi_h[1] = wi.y; xi_h[2] = wi.z; qi = wi.w;
      xi_l[0] = xi_l[1] = xi_l[2] = Real(0);
      ti = a.type[oi];
    }
    const Real *ljrow = MIXED ? reinterpret_cast<const Real *>(a.lj32 + ti * a.ntypes)
                              : reinterpret_cast<const Real *>(a.lj64 + ti * a.ntypes);
    // i as seen from the current entry's image of j (d = xj - (xi - s L))
    int cur = kZeroShift;
    Real xs_h[3] = {xi_h[0], xi_h[1], xi_h[2]};
    Real xs_l[3] = {xi_l[0], xi_l[1], xi_l[2]};
    Real fx = 0, fy = 0, fz = 0;
    int head = 0, queued = 0;

    auto process = [&](int p) {
      const auto d = Q.d[w][p];
      const int4 m = Q.m[w][p];
      const int flags = m.w & 15;
      Real en_lj = 0, en_c = 0;
      const Real f = pair_force<Real, TERMS, SPEC>(a, ljrow, d.w, qi * Q.qj[w][p], m.y, flags,
                                             en_lj, en_c);
      fx -= d.x * f;
      fy -= d.y * f;
      fz -= d.z * f;
      npairs++;
      if (ENERGY) {
        if (MIXED) {
          pair_energy64<Real, TERMS, VIRIAL>(a, wi, a.xw[m.x], m.w >> 4, ti, m.y, flags, Elj,
                                             Ec, V64);
        } else {
          Elj += (double)en_lj;
          Ec += (double)en_c;
        }
      }
      if (VIRIAL && !MIXED) {
        // addVirial(fij, d) with fij = d * f, half per visit
        Real hf = Real(0.5) * f;
        vxx += d.x * d.x * hf; vxy += d.x * d.y * hf; vxz += d.x * d.z * hf;
        vyy += d.y * d.y * hf; vyz += d.y * d.z * hf; vzz += d.z * d.z * hf;
      }
      if (RECORD) {
        int oj = a.sorted[m.x];
        if (oi < oj) {
          long long slot = atomicAdd((unsigned long long *)a.paircount, 1ull);
          if (slot < a.pairbuf_cap) a.pairbuf[slot] = ((long long)oi << 32) | (unsigned)oj;
        }
      }
    };

    for (int k0 = 0; k0 < cnt; k0 += 32) {
      const int k = k0 + lane;
      const bool have = k < cnt;
      const uint32_t e = e_next;
      // the next round's entry is fetched while this round computes
      e_next = (k + 32 < cnt) ? __ldg(row + k + 32) : 0u;
      const int j = (int)(e & kJMask);
      const int sh = (int)((e >> kShiftBits) & kShiftMask);
      // image changes are rare (atoms near a face of the box): a real branch
      if (__any_sync(kAll, have && sh != cur)) {
        if (have && sh != cur) {
          const int sx = (sh & 3) - 1, sy = ((sh >> 2) & 3) - 1, sz = ((sh >> 4) & 3) - 1;
          const double xs64[3] = {wi.x - sx * a.box.e[0], wi.y - sy * a.box.e[1],
                                  wi.z - sz * a.box.e[2]};
          for (int c = 0; c < 3; c++) {
            if (MIXED) {
              float h = (float)xs64[c];
              xs_h[c] = h;
              xs_l[c] = (float)(xs64[c] - (double)h);
            } else {
              xs_h[c] = xs64[c];
            }
          }
          cur = sh;
        }
      }
      Real dx, dy, dz, qj;
      int tj = 0;
      if (MIXED) {
        const float4 h = a.xhi[j], l = a.xlo[j];
        dx = (h.x - xs_h[0]) + (l.x - xs_l[0]);
        dy = (h.y - xs_h[1]) + (l.y - xs_l[1]);
        dz = (h.z - xs_h[2]) + (l.z - xs_l[2]);
        qj = h.w;
        tj = __float_as_int(l.w);
      } else {
        const double4 wj = a.xw[j];
        dx = wj.x - xs_h[0];
        dy = wj.y - xs_h[1];
        dz = wj.z - xs_h[2];
        qj = wj.w;
      }
      const Real r2 = dx * dx + dy * dy + dz * dz;
      constexpr int kAllTerms = ((TERMS & TERM_LJ) ? kQLJ : 0) | ((TERMS & TERM_COUL) ? kQCoul : 0) |
                                ((TERMS & TERM_EWALD) ? kQEwald : 0);
      int flags = 0;
      bool band = false;
      if (have && a.same_cut) {  // every term shares one cutoff
        if (r2 <= a.max_lo) flags = kAllTerms;
        else band = r2 <= a.max_hi;
      } else if (have) {
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
          const double r2x = exact_r2(a, oi, a.sorted[j], (double)dx, (double)dy, (double)dz);
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
      const bool pass = flags != 0;
      const unsigned mk = __ballot_sync(kAll, pass);
      if (pass) {
        if (!MIXED) tj = a.type[a.sorted[j]];
        if (e & kModifiedBit) flags |= kQModified;
        const int p = (head + queued + __popc(mk & lt_mask)) & (kQueue - 1);
        typename QueueVec<Real>::T d;
        d.x = dx; d.y = dy; d.z = dz; d.w = r2;
        Q.d[w][p] = d;
        Q.m[w][p] = make_int4(j, tj, 0, flags | (sh << 4));
        Q.qj[w][p] = qj;
      }
      queued += __popc(mk);
      if (queued >= 32) {
        __syncwarp();
        process((head + lane) & (kQueue - 1));
        head += 32;
        queued -= 32;
        __syncwarp();
      }
    }
    if (queued > 0) {
      __syncwarp();
      if (lane < queued) process((head + lane) & (kQueue - 1));
    }
    __syncwarp();  // the ring is refilled by the next atom
    double Fx = warp_sum((double)fx), Fy = warp_sum((double)fy), Fz = warp_sum((double)fz);
    if (lane == 0) {
      red_add(&a.force[oi], to_fixed(Fx, kForceScale));
      red_add(&a.force[a.n + oi], to_fixed(Fy, kForceScale));
      red_add(&a.force[2 * a.n + oi], to_fixed(Fz, kForceScale));
    }
  }
  if (ENERGY || a.count_pairs) {
    int np = warp_sum(npairs);
    if (lane == 0) red_add(&a.acc[ACC_PAIRS], (long long)np);
  }
  if (ENERGY) {
    double dlj = warp_sum(Elj) * 0.5;
    double dc = warp_sum(Ec) * 0.5;
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

}  // namespace pmgpu
