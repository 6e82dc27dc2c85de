// Device helpers shared by the pmgpu kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "pm_internal.cuh"

namespace pmgpu {

// ---------------------------------------------------- exact FP64 helpers
// The reference's own x86-64 build rounds every double operation
// separately (no fused multiply-add).  These helpers keep nvcc from
// contracting, so positions, cells and the cutoff test agree bit for bit.
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xnorm2(double x, double y, double z) {
  return xadd(xadd(xmul(x, x), xmul(y, y)), xmul(z, z));
}

// PeriodicBoundaryConditions::minimalDifference(c1, c2, distSquared),
// PeriodicBoundaryConditions.h:72-110 (orthogonal branch); d = c2 - c1.
__device__ __forceinline__ double box_mindiff(const Box &b, double x1, double y1,
                                              double z1, double x2, double y2,
                                              double z2, double &dx, double &dy,
                                              double &dz) {
  dx = xsub(x2, x1);
  dy = xsub(y2, y1);
  dz = xsub(z2, z1);
  double r2 = xnorm2(dx, dy, dz);
  if (!b.periodic) return r2;
  if (r2 > b.D) {
    if (dx < -b.H2[0]) dx = xadd(dx, b.H[0]);
    else if (dx > b.H2[0]) dx = xsub(dx, b.H[0]);
    if (dy < -b.H2[1]) dy = xadd(dy, b.H[1]);
    else if (dy > b.H2[1]) dy = xsub(dy, b.H[1]);
    if (dz < -b.H2[2]) dz = xadd(dz, b.H[2]);
    else if (dz > b.H2[2]) dz = xsub(dz, b.H[2]);
    r2 = xnorm2(dx, dy, dz);
    if (r2 > b.D) {
      dx = xsub(dx, xmul(b.e[0], rint(xmul(b.er[0], dx))));
      dy = xsub(dy, xmul(b.e[1], rint(xmul(b.er[1], dy))));
      dz = xsub(dz, xmul(b.e[2], rint(xmul(b.er[2], dz))));
      r2 = xnorm2(dx, dy, dz);
    }
  }
  return r2;
}

// PeriodicBoundaryConditions::minimalPosition(c), :113-140.
__device__ __forceinline__ void box_minpos(const Box &b, double x, double y,
                                           double z, double &ox, double &oy,
                                           double &oz) {
  if (!b.periodic) {
    ox = x; oy = y; oz = z;
    return;
  }
  ox = xsub(x, b.origin[0]);
  oy = xsub(y, b.origin[1]);
  oz = xsub(z, b.origin[2]);
  if (xnorm2(ox, oy, oz) <= b.D) return;
  if (ox < -b.H2[0]) ox = xadd(ox, b.H[0]);
  else if (ox > b.H2[0]) ox = xsub(ox, b.H[0]);
  if (oy < -b.H2[1]) oy = xadd(oy, b.H[1]);
  else if (oy > b.H2[1]) oy = xsub(oy, b.H[1]);
  if (oz < -b.H2[2]) oz = xadd(oz, b.H[2]);
  else if (oz > b.H2[2]) oz = xsub(oz, b.H[2]);
  if (xnorm2(ox, oy, oz) <= b.D) return;
  ox = xsub(ox, xmul(b.e[0], rint(xmul(b.er[0], ox))));
  oy = xsub(oy, xmul(b.e[1], rint(xmul(b.er[1], oy))));
  oz = xsub(oz, xmul(b.e[2], rint(xmul(b.er[2], oz))));
}

// ------------------------------------------------------------ switching
// Value and derivative-over-distance of ProtoMol's switching functions
// (switch/C1SwitchingFunction.h:41-50, C2SwitchingFunction.h:42-52,
// CnSwitchingFunction.cpp:149-175, CmpCnCnSwitchingFunction.h:45-95,
// CutoffSwitchingFunction.h:41-44, UniversalSwitchingFunction.h:45-48,
// and the complement 1 - S of ComplementSwitchingFunction.h:42-46), in
// the precision Real.
template <typename Real>
struct SwitchDev {
  int kind;
  Real cutoff, cutoff2, switchon2;
  Real c1a, c1b, c1c;
  Real s1, s2, s3;
  int ord_int, ord_idx;
  Real irange[8];
  Real compoff, compoff2;
  Real itrange[8];
  int complement;
};

template <typename Real>
__host__ inline SwitchDev<Real> make_switch_dev(const SwitchParams &p) {
  SwitchDev<Real> d;
  d.kind = p.kind;
  d.cutoff = (Real)p.cutoff;
  d.cutoff2 = (Real)p.cutoff2;
  d.switchon2 = (Real)p.switchon2;
  d.c1a = (Real)p.c1a; d.c1b = (Real)p.c1b; d.c1c = (Real)p.c1c;
  d.s1 = (Real)p.s1; d.s2 = (Real)p.s2; d.s3 = (Real)p.s3;
  d.ord_int = p.ord_int; d.ord_idx = p.ord_idx;
  for (int i = 0; i < 8; i++) d.irange[i] = (Real)p.irange[i];
  d.compoff = (Real)p.compoff;
  d.compoff2 = (Real)p.compoff2;
  for (int i = 0; i < 8; i++) d.itrange[i] = (Real)p.itrange[i];
  d.complement = p.complement;
  return d;
}

// Cn polynomial tables (switch/CnSwitchingFunction.cpp:9-23).
static __constant__ double c_cn_sw[5][7] = {
    {10., -15., 6., 0, 0, 0, 0},
    {35., -84., 70., -20., 0, 0, 0},
    {126., -420., 540., -315., 70., 0, 0},
    {0, 0, 0, 0, 0, 0, 0},
    {1716., -9009., 20020., -24024., 16380., -6006., 924.0}};
static __constant__ double c_cn_dsw[5][7] = {
    {30., -60., 30., 0, 0, 0, 0},
    {140., -420., 420., -140., 0, 0, 0},
    {630., -2520., 3780., -2520., 630., 0, 0},
    {0, 0, 0, 0, 0, 0, 0},
    {12012., -72072., 180180., -240240., 180180., -72072., 12012.0}};

// Programmatic dependent launch.  A kernel started with launch_pdl may begin
// while its predecessor in the stream still runs: pdl_wait() blocks until
// that grid has completed and its memory is visible, so it is the first
// statement of every such kernel.  pdl_trigger() lets the successor's
// launch begin once every block of this grid has triggered or exited, so
// the successor's blocks never hold resources a block of this grid still
// needs.  Both are no-ops for ordinary launches.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;"); }

__device__ __forceinline__ float pm_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double pm_sqrt(double x) { return sqrt(x); }

// rsqrt with one Newton step: the bare MUFU estimate carries a small bias
// that would otherwise show in the summed forces.
__device__ __forceinline__ float rsqrt_nr(float x) {
  float y = rsqrtf(x);
  return y * (1.5f - 0.5f * x * y * y);
}
__device__ __forceinline__ double rsqrt_nr(double x) { return 1.0 / sqrt(x); }

// 1/x from the hardware estimate refined by one Newton step,
// y' = y + y (1 - x y); within about one ulp for normal positive x.
__device__ __forceinline__ float rcp_nr(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return fmaf(y, fmaf(-x, y, 1.0f), y);
}

// Sums v[0..7] over the 32 lanes of a warp by a transposed butterfly
// (9 shuffles): each exchange step hands half of the remaining slots to the
// partner lane, so lane l ends with the total of slot (l >> 2) & 7, as do
// the other three lanes of its quad.  The order of the additions is fixed.
__device__ __forceinline__ float warp_tsum8(const float (&v)[8], int lane) {
  const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
  float a[4], b[2];
#pragma unroll
  for (int m = 0; m < 4; m++)
    a[m] = (b4 ? v[m + 4] : v[m]) + __shfl_xor_sync(0xffffffffu, b4 ? v[m] : v[m + 4], 16);
#pragma unroll
  for (int m = 0; m < 2; m++)
    b[m] = (b3 ? a[m + 2] : a[m]) + __shfl_xor_sync(0xffffffffu, b3 ? a[m] : a[m + 2], 8);
  float c = (b2 ? b[1] : b[0]) + __shfl_xor_sync(0xffffffffu, b2 ? b[0] : b[1], 4);
  c += __shfl_xor_sync(0xffffffffu, c, 2);
  c += __shfl_xor_sync(0xffffffffu, c, 1);
  return c;
}

// The work items of a launch dealt to the blocks round-robin (block b
// takes items b, b + G, b + 2G, ... of G blocks), so every SM gets the same
// number of items and the same mix of cheap and dear ones; inside a block
// the warps take the items of its share from a shared-memory counter, so
// they stay busy to the end of it.  `counter` is a __shared__ int the block
// sets to zero (then synchronises) before the first next().
struct BlockItems {
  int *counter;
  __device__ __forceinline__ long long next(int lane) const {
    int k = 0;
    if (lane == 0) k = atomicAdd(counter, 1);
    return blockIdx.x + (long long)gridDim.x * __shfl_sync(0xffffffffu, k, 0);
  }
};

// Work item w of the half all-pairs sweep: the tile pairs (I, J), I <= J,
// of `tiles` 32-atom tiles, numbered diagonal by diagonal: d = J - I = 0
// holds I = 0..tiles-1, d = 1 holds I = 0..tiles-2, and so on, so that
// w = d tiles - d (d - 1) / 2 + I.  Pairs of nearby tiles, which in a chain
// molecule hold the near (dearer) atom pairs, are spread over the numbers.
__device__ __forceinline__ void tile_pair_of(long long w, int tiles, int *I, int *J) {
  const double t2 = 2.0 * tiles + 1.0;
  int d = (int)((t2 - sqrt(t2 * t2 - 8.0 * (double)w)) * 0.5);
  d = max(0, min(d, tiles - 1));
  auto start = [&](long long q) { return q * tiles - q * (q - 1) / 2; };
  while (d > 0 && start(d) > w) d--;
  while (d + 1 < tiles && start(d + 1) <= w) d++;
  *I = (int)(w - start(d));
  *J = *I + d;
}

// An FP64 coordinate as an FP32 pair: hi = x rounded, lo = x - hi rounded,
// so hi + lo carries 48 significant bits and a difference of two such
// pairs, (hj - hi) + (lj - li), is as good as the FP64 difference rounded
// to FP32.
__device__ __forceinline__ void split_hilo(double x, float &hi, float &lo) {
  hi = (float)x;
  lo = (float)(x - (double)hi);
}

// The FP32 record of atom i read by the all-pairs passes: rec[i] =
// (x_hi, y_hi, z_hi, charge), rec[n + i] = (x_lo, y_lo, z_lo, type bits).
__device__ __forceinline__ void write_pair_record(float4 *rec, int n, int i, double x,
                                                  double y, double z, double q, int type) {
  float4 h, l;
  split_hilo(x, h.x, l.x);
  split_hilo(y, h.y, l.y);
  split_hilo(z, h.z, l.z);
  h.w = (float)q;
  l.w = __int_as_float(type);
  rec[i] = h;
  rec[n + i] = l;
}

template <typename Real>
__device__ __forceinline__ void switch_eval_base(const SwitchDev<Real> &w, Real r2,
                                                 Real &val, Real &der);
template <typename Real>
__device__ __forceinline__ void switch_eval(const SwitchDev<Real> &w, Real r2,
                                            Real &val, Real &der) {
  switch_eval_base<Real>(w, r2, val, der);
  if (w.complement) {
    val = Real(1) - val;
    der = -der;
  }
}

template <typename Real>
__device__ __forceinline__ void switch_eval_base(const SwitchDev<Real> &w, Real r2,
                                                 Real &val, Real &der) {
  switch (w.kind) {
    case PMGPU_SW_C2:
      der = Real(0);
      if (r2 > w.cutoff2) {
        val = Real(0);
      } else if (r2 >= w.switchon2) {
        Real c2 = w.cutoff2 - r2;
        Real c4 = c2 * (w.s2 + Real(2) * r2);
        val = w.s1 * (c2 * c4);
        der = w.s3 * (c2 * c2 - c4);
      } else {
        val = Real(1);
      }
      return;
    case PMGPU_SW_C1: {
      if (r2 > w.cutoff2) {
        val = Real(0);
        der = Real(0);
        return;
      }
      Real d = pm_sqrt(r2);
      val = Real(1) - d * (w.c1a - r2 * w.c1b);
      der = -w.c1a / d + d * w.c1c;
      return;
    }
    case PMGPU_SW_CN:
    case PMGPU_SW_CMPCNCN: {
      // Cn: one polynomial from the switch-on distance to the cutoff.
      // CmpCnCn (CmpCnCnSwitchingFunction.h:45-95): 0 below switchon, a
      // rising polynomial (1 - p) up to switchoff, a falling one (p) to the
      // cutoff; each is the Cn loop with its own offset and range table.
      const bool cmp = w.kind == PMGPU_SW_CMPCNCN;
      der = Real(0);
      val = Real(0);
      if (r2 > w.cutoff2) return;
      if (r2 < w.switchon2) {
        val = cmp ? Real(0) : Real(1);
        return;
      }
      const bool rising = cmp && r2 <= w.compoff2;
      const bool falling = cmp && !rising;
      Real sq = pm_sqrt(r2);
      Real sd = sq - (rising ? w.compoff : w.cutoff);
      Real c;  // c[0] = sd^ordInt
      if (sizeof(Real) == 8) {
        c = (Real)pow((double)sd, (double)w.ord_int);
      } else {
        c = Real(1);
        for (int i = 0; i < w.ord_int; i++) c *= sd;
      }
      for (int i = 0; i < w.ord_int + 1; i++) {
        Real cn = c * sd;                            // c[i+1]
        const Real rg = falling ? w.itrange[i] : w.irange[i];
        val += (Real)c_cn_sw[w.ord_idx][i] * cn * rg;
        der += (Real)c_cn_dsw[w.ord_idx][i] * c * rg;
        c = cn;
      }
      if (rising) {
        val = Real(1) - val;
        der = -der;
      }
      der /= sq;
      return;
    }
    case PMGPU_SW_CUTOFF:
      der = Real(0);
      val = r2 > w.cutoff2 ? Real(0) : Real(1);
      return;
    default:
      val = Real(1);
      der = Real(0);
      return;
  }
}

// A&S 7.1.26 polynomial (base/MathUtilities.cpp:39-49).
template <typename Real>
__device__ __forceinline__ Real poly5(Real ar) {
  Real t = Real(1) / (Real(1) + Real(0.3275911) * ar);
  return t * (Real(0.254829592) +
              t * (Real(-0.284496736) +
                   t * (Real(1.421413741) +
                        t * (Real(-1.453152027) + t * Real(1.061405429)))));
}

// The same polynomial with the reciprocal from the fast hardware
// approximation (about 2 ulp) in FP32; FP64 keeps the exact division.
template <typename Real>
__device__ __forceinline__ Real poly5_fast(Real ar) {
  return poly5<Real>(ar);
}
template <>
__device__ __forceinline__ float poly5_fast<float>(float ar) {
  float t = __fdividef(1.0f, 1.0f + 0.3275911f * ar);
  return t * (0.254829592f +
              t * (-0.284496736f + t * (1.421413741f + t * (-1.453152027f + t * 1.061405429f))));
}

// ----------------------------------------------------------- fixed point
__device__ __forceinline__ long long to_fixed(double v, double scale) {
  return __double2ll_rn(v * scale);
}
__device__ __forceinline__ void red_add(long long *p, long long v) {
  atomicAdd(reinterpret_cast<unsigned long long *>(p),
            static_cast<unsigned long long>(v));
}

// Pair-list rebuild decision, taken on the device by the last block of a
// grid to finish: every thread passes the squared displacement of its atom
// from its position at the last build (0 for no atom); the list is rebuilt
// when it is forced or some atom moved more than half the skin.
// rebuild[0] is the flag, rebuild[1] counts builds; ticket[0] orders the
// blocks, ticket[1] holds the running maximum (FP32 bits).  Every thread of
// the block must call it; blockDim.x is THREADS and nblocks the number of
// blocks of this system's launch.
template <int THREADS>
__device__ __forceinline__ void rebuild_decide(float d2, unsigned *ticket, int *rebuild,
                                               float half_skin2, int force, int nblocks,
                                               unsigned long long *step = nullptr) {
  __shared__ float wmax[THREADS / 32];
  __shared__ bool last;
  if (!(d2 == d2)) d2 = 3.0e38f;  // NaN: rebuild (the binning flags it)
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) d2 = fmaxf(d2, __shfl_xor_sync(0xffffffffu, d2, o));
  if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = d2;
  __syncthreads();
  if (threadIdx.x == 0) {
    float m = wmax[0];
    for (int w = 1; w < THREADS / 32; w++) m = fmaxf(m, wmax[w]);
    if (m > 0.f) atomicMax(&ticket[1], __float_as_uint(m));
    __threadfence();
    last = atomicAdd(&ticket[0], 1u) == (unsigned)nblocks - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    const float m = __uint_as_float(atomicExch(&ticket[1], 0u));
    const int r = force || m > half_skin2;
    rebuild[0] = r;
    if (r) rebuild[1] += 1;
    ticket[0] = 0u;
    // the caller's step counter, when it rides on this ticket (every block
    // has read it before counting itself done)
    if (step) step[0] += 1ull;
  }
}

// ------------------------------------------------------- batched launches
// A kernel body runs either as its own launch (one system) or inside a
// batched launch over the members of an ensemble, one after another in the
// grid.  Blk is the block's index and the block count of its system's part.
struct Blk {
  int x, n;
};
__device__ __forceinline__ Blk own_blk() { return Blk{(int)blockIdx.x, (int)gridDim.x}; }

// The member of a batched launch that block b belongs to: first[m] is the
// first block of member m (first[nm] is the grid size), members with no
// blocks are skipped.
__device__ __forceinline__ int batch_member(const int *__restrict__ first, int nm, int b) {
  int lo = 0, hi = nm;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(first + mid) <= b) lo = mid;
    else hi = mid;
  }
  return lo;
}
__device__ __forceinline__ Blk batch_blk(const int *__restrict__ first, int m) {
  const int f = __ldg(first + m);
  return Blk{(int)blockIdx.x - f, __ldg(first + m + 1) - f};
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace pmgpu
