// The fused nonbonded pair kernel: Lennard-Jones and Coulomb with
// ProtoMol's switching functions (OneAtomPair / OneAtomPairTwo,
// force/OneAtomPairTwo.h:30-100) and the Ewald real-space term
// (NonbondedFullEwaldSystemForce::realTerm, .h:753-858), over full Verlet
// lists (thread per sorted atom).
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
  Real lj_lo, lj_hi, coul_lo, coul_hi, ew_lo, ew_hi, max_hi;
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
};

__device__ __forceinline__ int excl_lookup(const int *start, const int *partner,
                                           const int *cls, int oi, int oj) {
  int b = start[oi], e = start[oi + 1];
  for (int k = b; k < e; k++)
    if (partner[k] == oj) return cls[k];
  return PMGPU_EXCL_NONE;
}

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

// Thread per sorted atom i; walks its full neighbour list.  Each unordered
// pair is visited from both ends: forces are written for i only (no atomics
// on j), energies and virial are halved.
// TPA lanes (a warp-aligned tile) share one atom: lane l walks entries
// l, l + TPA, ... of the atom's neighbour row, so 23.5k atoms still fill the
// GPU, and the tile reduces its forces with shuffles at the end.
template <typename Real, int TERMS, int MODE, int TPA>
__global__ void __launch_bounds__(128) k_pairs(PairArgs<Real> a) {
  static_assert(TPA >= 1 && TPA <= 32 && (TPA & (TPA - 1)) == 0, "TPA: power of two");
  constexpr bool MIXED = sizeof(Real) == 4;
  constexpr bool ENERGY = MODE != PAIR_FORCE;
  constexpr bool VIRIAL = MODE == PAIR_VIRIAL;
  constexpr bool RECORD = MODE == PAIR_RECORD;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = gt & (TPA - 1);
  int i = gt / TPA;
  bool valid = i < a.n;
  int ii = valid ? i : 0;
  int oi = a.sorted[ii];
  double4 wi = a.xw[ii];
  double xs64[3] = {wi.x, wi.y, wi.z};
  Real xs_h[3], xs_l[3], qi;
  int ti;
  if (MIXED) {
    float4 h = a.xhi[ii], l = a.xlo[ii];
    xs_h[0] = h.x; xs_h[1] = h.y; xs_h[2] = h.z; qi = h.w;
    xs_l[0] = l.x; xs_l[1] = l.y; xs_l[2] = l.z; ti = __float_as_int(l.w);
  } else {
    xs_h[0] = wi.x; xs_h[1] = wi.y; xs_h[2] = wi.z; qi = wi.w;
    xs_l[0] = xs_l[1] = xs_l[2] = Real(0);
    ti = a.type[oi];
  }
  int cur_shift = kZeroShift;
  Real fx = 0, fy = 0, fz = 0;
  Real vxx = 0, vxy = 0, vxz = 0, vyy = 0, vyz = 0, vzz = 0;
  int npairs = 0;
  int cnt = valid ? a.nbr_count[ii] : 0;
  // Forces are summed in the kernel precision over chunks of kPairChunk
  // neighbours and the chunk sums in FP64.
  constexpr int kPairChunk = 16;
  double Fx = 0, Fy = 0, Fz = 0, Elj = 0, Ec = 0;
  double V[6] = {0, 0, 0, 0, 0, 0};
  const uint32_t *row = a.nbr + (size_t)ii * a.cap;
  for (int k0 = lane; k0 < cnt; k0 += kPairChunk * TPA) {
    const int k1 = min(cnt, k0 + kPairChunk * TPA);
    for (int k = k0; k < k1; k += TPA) {
      uint32_t e = row[k];
      int j = (int)(e & kJMask);
      int sh = (int)((e >> kShiftBits) & 31);
      if (sh != cur_shift) {
        // i moved by minus the j image shift: d = xj - (xi - s L)
        int sx = sh / 9 - 1, sy = (sh / 3) % 3 - 1, sz = sh % 3 - 1;
        xs64[0] = wi.x - sx * a.box.e[0];
        xs64[1] = wi.y - sy * a.box.e[1];
        xs64[2] = wi.z - sz * a.box.e[2];
        if (MIXED) {
          for (int c = 0; c < 3; c++) {
            float h = (float)xs64[c];
            xs_h[c] = h;
            xs_l[c] = (float)(xs64[c] - (double)h);
          }
        } else {
          xs_h[0] = xs64[0]; xs_h[1] = xs64[1]; xs_h[2] = xs64[2];
        }
        cur_shift = sh;
      }
      Real dx, dy, dz, qj;
      int tj;
      double4 wj;
      if (MIXED) {
        float4 h = a.xhi[j], l = a.xlo[j];
        dx = (h.x - xs_h[0]) + (l.x - xs_l[0]);
        dy = (h.y - xs_h[1]) + (l.y - xs_l[1]);
        dz = (h.z - xs_h[2]) + (l.z - xs_l[2]);
        qj = h.w;
        tj = __float_as_int(l.w);
      } else {
        wj = a.xw[j];
        dx = wj.x - xs_h[0];
        dy = wj.y - xs_h[1];
        dz = wj.z - xs_h[2];
        qj = wj.w;
        tj = -1;
      }
      Real r2 = dx * dx + dy * dy + dz * dz;
      if (r2 > a.max_hi) continue;
      int excl = PMGPU_EXCL_NONE;
      int oj = -1;
      if (e & kSameMolBit) {
        oj = a.sorted[j];
        excl = excl_lookup(a.excl_start, a.excl_partner, a.excl_class, oi, oj);
      }
      bool do_lj = false, do_coul = false, do_ew = false;
      double r2x = -1.0;  // exact FP64 r^2 of this image, when needed
      if (TERMS & TERM_LJ) {
        if (r2 <= a.lj_lo) do_lj = true;
        else if (r2 <= a.lj_hi) {
          if (oj < 0) oj = a.sorted[j];
          r2x = exact_r2(a, oi, oj, (double)dx, (double)dy, (double)dz);
          do_lj = r2x <= a.lj_cut2;
        }
      }
      if (TERMS & TERM_COUL) {
        if (r2 <= a.coul_lo) do_coul = true;
        else if (r2 <= a.coul_hi) {
          if (oj < 0) oj = a.sorted[j];
          if (r2x < 0) r2x = exact_r2(a, oi, oj, (double)dx, (double)dy, (double)dz);
          do_coul = r2x <= a.coul_cut2;
        }
      }
      if (TERMS & TERM_EWALD) {
        if (r2 <= a.ew_lo) do_ew = true;
        else if (r2 <= a.ew_hi) {
          if (oj < 0) oj = a.sorted[j];
          if (r2x < 0) r2x = exact_r2(a, oi, oj, (double)dx, (double)dy, (double)dz);
          do_ew = r2x <= a.ew_cut2;
        }
      }
      // FULL exclusions skip the pair (OneAtomPairTwo.h:47-53); in the
      // Ewald real term they skip only the minimal image, which is the entry
      // carrying the same-molecule bit (NonbondedFullEwaldSystemForce.h:795-801).
      if (excl == PMGPU_EXCL_FULL) {
        do_lj = false;
        do_coul = false;
        do_ew = false;
      }
      if (!(do_lj || do_coul || do_ew)) continue;
      if (!MIXED) tj = a.type[a.sorted[j]];
      const Real rinv = rsqrt_nr(r2);
      const Real rinv2 = rinv * rinv;
      Real f = 0;
      Real en_lj = 0, en_c = 0;
      if ((TERMS & TERM_LJ) && do_lj) {
        Real A, B;
        if (MIXED) {
          float4 p = __ldg(&a.lj32[ti * a.ntypes + tj]);
          A = excl == PMGPU_EXCL_MODIFIED ? p.z : p.x;
          B = excl == PMGPU_EXCL_MODIFIED ? p.w : p.y;
        } else {
          double4 p = a.lj64[ti * a.ntypes + tj];
          A = excl == PMGPU_EXCL_MODIFIED ? p.z : p.x;
          B = excl == PMGPU_EXCL_MODIFIED ? p.w : p.y;
        }
        // LennardJonesForce::operator() (force/LennardJonesForce.h:28-60)
        Real r6 = rinv2 * rinv2 * rinv2;
        Real r6B = B * r6;
        Real r12A = A * r6 * r6;
        Real en = r12A - r6B;
        Real ff = (Real(12) * r12A - Real(6) * r6B) * rinv2;
        if (a.lj_modify) apply_switch<Real>(a.lj_sw, a.lj_sw64, r2, ff, en);
        en_lj += en;
        f += ff;
      }
      if ((TERMS & TERM_COUL) && do_coul) {
        // CoulombForce::operator() (force/CoulombForce.h:29-40)
        Real en = qi * qj * rinv;
        if (excl == PMGPU_EXCL_MODIFIED) en *= a.csf;
        Real ff = en * rinv2;
        if (a.coul_modify) apply_switch<Real>(a.coul_sw, a.coul_sw64, r2, ff, en);
        en_c += en;
        f += ff;
      }
      if ((TERMS & TERM_EWALD) && do_ew) {
        Real qq = qi * qj;
        if (excl == PMGPU_EXCL_MODIFIED) qq *= a.csf;
        Real r = r2 * rinv;
        Real ar = a.alpha * r;
        Real ee = qq * fast_exp(-ar * ar);
        Real en;
        if (!a.exact_erf)
          en = poly5<Real>(ar) * ee * rinv;  // A&S erfc (MathUtilities.cpp:39-49)
        else
          en = qq * erfc(ar) * rinv;  // USE_EWALD_EXACT_ERF: C library erfc
        f += (en + a.a2pi * ee) * rinv2;
        en_c += en;
      }
      npairs++;
      fx -= dx * f;
      fy -= dy * f;
      fz -= dz * f;
      if (ENERGY) {
        if (!MIXED) {
          Elj += (double)en_lj;
          Ec += (double)en_c;
        } else {
          // FP64 energy of the same pair from the FP64 wrapped coordinates
          double4 w = a.xw[j];
          double ex = w.x - xs64[0], ey = w.y - xs64[1], ez = w.z - xs64[2];
          double r2e = ex * ex + ey * ey + ez * ez;
          double rr2 = 1.0 / r2e;
          if ((TERMS & TERM_LJ) && do_lj) {
            double4 p = a.lj64[ti * a.ntypes + tj];
            double A = excl == PMGPU_EXCL_MODIFIED ? p.z : p.x;
            double B = excl == PMGPU_EXCL_MODIFIED ? p.w : p.y;
            double r6 = rr2 * rr2 * rr2;
            double en = A * r6 * r6 - B * r6;
            if (a.lj_modify) {
              double sv, sd;
              switch_eval<double>(a.lj_sw64, r2e, sv, sd);
              en *= sv;
            }
            Elj += en;
          }
          double qq = (double)qi * w.w;
          if (excl == PMGPU_EXCL_MODIFIED) qq *= a.csf64;
          if ((TERMS & TERM_COUL) && do_coul) {
            double en = qq * sqrt(rr2);
            if (a.coul_modify) {
              double sv, sd;
              switch_eval<double>(a.coul_sw64, r2e, sv, sd);
              en *= sv;
            }
            Ec += en;
          }
          if ((TERMS & TERM_EWALD) && do_ew) {
            double r = sqrt(r2e);
            double ar = a.alpha64 * r;
            double en = !a.exact_erf ? poly5<double>(ar) * qq * exp(-ar * ar) / r
                                     : qq * erfc(ar) / r;
            Ec += en;
          }
        }
      }
      if (VIRIAL) {
        // addVirial(fij, d) with fij = d * f, half per visit
        Real hf = Real(0.5) * f;
        vxx += dx * dx * hf; vxy += dx * dy * hf; vxz += dx * dz * hf;
        vyy += dy * dy * hf; vyz += dy * dz * hf; vzz += dz * dz * hf;
      }
      if (RECORD) {
        if (oj < 0) oj = a.sorted[j];
        if (oi < oj) {
          long long slot = atomicAdd((unsigned long long *)a.paircount, 1ull);
          if (slot < a.pairbuf_cap) a.pairbuf[slot] = ((long long)oi << 32) | (unsigned)oj;
        }
      }
    }
    Fx += (double)fx; Fy += (double)fy; Fz += (double)fz;
    fx = fy = fz = Real(0);
    if (VIRIAL) {
      V[0] += (double)vxx; V[1] += (double)vxy; V[2] += (double)vxz;
      V[3] += (double)vyy; V[4] += (double)vyz; V[5] += (double)vzz;
      vxx = vxy = vxz = vyy = vyz = vzz = Real(0);
    }
  }
  // reduce the atom's force over its TPA lanes (fixed lane order)
#pragma unroll
  for (int o = TPA / 2; o > 0; o >>= 1) {
    Fx += __shfl_xor_sync(0xffffffffu, Fx, o);
    Fy += __shfl_xor_sync(0xffffffffu, Fy, o);
    Fz += __shfl_xor_sync(0xffffffffu, Fz, o);
  }
  if (valid && lane == 0) {
    red_add(&a.force[oi], to_fixed(Fx, kForceScale));
    red_add(&a.force[a.n + oi], to_fixed(Fy, kForceScale));
    red_add(&a.force[2 * a.n + oi], to_fixed(Fz, kForceScale));
  }
  int np = warp_sum(npairs);
  if (ENERGY) {
    double dlj = warp_sum(Elj) * 0.5;
    double dc = warp_sum(Ec) * 0.5;
    if (VIRIAL)
      for (int q = 0; q < 6; q++) V[q] = warp_sum(V[q]);
    if ((threadIdx.x & 31) == 0) {
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
  if ((threadIdx.x & 31) == 0) red_add(&a.acc[ACC_PAIRS], (long long)np);
}

}  // namespace pmgpu
