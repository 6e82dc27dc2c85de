// Nonbonded pair path on the device:
//   * binning of atoms into ProtoMol's cubic cells (same FP64 formula as
//     Topology::updateCellLists / CubicCellManager::findCell) refined by a
//     Morton-ordered 4x4x4 sub-grid, and a deterministic counting sort;
//   * Verlet neighbour lists (thread per sorted atom, full lists with a
//     skin; rebuilt on the device when an atom has moved more than skin/2);
//   * the fused pair kernel: Lennard-Jones and Coulomb with ProtoMol's
//     switching functions, and the Ewald real-space term, in FP32 from
//     hi/lo-split FP64 coordinates, with an FP64 re-test of pairs near the
//     cutoff so the accepted pair set equals the FP64 reference's;
//   * the vacuum all-pairs (NonbondedSimpleFull) LJ / Coulomb kernel.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "pm_device.cuh"

namespace pmgpu {

// ------------------------------------------------------------------ grid
struct GridArgs {
  Box box;
  int n;
  int ncx, ncy, ncz;
  double cs[3];      // coarse cell size vector
  double inv[3];     // 1 / cs
  double delta[3];   // origin - min (ProtoMol Topology.h:58)
  double vmin[3];    // vacuum: grid minimum (positions clamp into the grid)
};

__device__ __forceinline__ int morton3(int x, int y, int z) {
  int m = 0;
#pragma unroll
  for (int b = 0; b < 2; b++) {
    m |= ((x >> b) & 1) << (3 * b + 2);
    m |= ((y >> b) & 1) << (3 * b + 1);
    m |= ((z >> b) & 1) << (3 * b);
  }
  return m;
}

// Cell of one atom: floor((delta + minimalPosition(x)) * inv) per axis
// (Topology.h:67-70, CubicCellManager.cpp:40-44); also returns the wrapped
// position and the fractional position inside the cell.
__device__ __forceinline__ void cell_of(const GridArgs &g, double x, double y,
                                        double z, int c[3], double w[3],
                                        double frac[3]) {
  box_minpos(g.box, x, y, z, w[0], w[1], w[2]);
  for (int a = 0; a < 3; a++) {
    double q;
    if (g.box.periodic)
      q = xmul(xadd(g.delta[a], w[a]), g.inv[a]);
    else
      q = xmul(xsub(w[a], g.vmin[a]), g.inv[a]);
    double f = floor(q);
    c[a] = (int)f;
    frac[a] = q - f;
  }
}

__global__ void k_bin(GridArgs g, const double *__restrict__ pos,
                      const int *__restrict__ rebuild, int *__restrict__ key,
                      int *__restrict__ key_count, double *__restrict__ offset,
                      double *__restrict__ xbuild, int *__restrict__ status) {
  if (!*rebuild) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.n) return;
  double x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
  int c[3];
  double w[3], fr[3];
  cell_of(g, x, y, z, c, w, fr);
  int dims[3] = {g.ncx, g.ncy, g.ncz};
  int f[3];
  for (int a = 0; a < 3; a++) {
    if (c[a] < 0) { c[a] = 0; fr[a] = 0.0; }
    if (c[a] >= dims[a]) { c[a] = dims[a] - 1; fr[a] = 0.999999; }
    int k = (int)(fr[a] * kFine);
    f[a] = k < 0 ? 0 : (k >= kFine ? kFine - 1 : k);
  }
  if (!isfinite(x) || !isfinite(y) || !isfinite(z)) atomicOr(status, ST_NONFINITE);
  int cell = (c[0] * g.ncy + c[1]) * g.ncz + c[2];
  int k = cell * kFine3 + morton3(f[0], f[1], f[2]);
  key[i] = k;
  atomicAdd(&key_count[k], 1);
  offset[3 * i] = x - w[0];
  offset[3 * i + 1] = y - w[1];
  offset[3 * i + 2] = z - w[2];
  xbuild[3 * i] = x;
  xbuild[3 * i + 1] = y;
  xbuild[3 * i + 2] = z;
}

// Single-block exclusive scan of the key counts (nkeys is at most a few
// hundred thousand); also zeroes the scatter cursors.
__global__ void k_scan(const int *__restrict__ rebuild, const int *__restrict__ count,
                       int *__restrict__ start, int *__restrict__ cursor, int nkeys) {
  if (!*rebuild) return;
  __shared__ int warp_tot[32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < nkeys; base += blockDim.x) {
    int i = base + threadIdx.x;
    int v = i < nkeys ? count[i] : 0;
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) warp_tot[wid] = incl;
    __syncthreads();
    if (wid == 0) {
      int nw = blockDim.x >> 5;
      int t = lane < nw ? warp_tot[lane] : 0;
      int ti = t;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int u = __shfl_up_sync(0xffffffffu, ti, o);
        if (lane >= o) ti += u;
      }
      if (lane < nw) warp_tot[lane] = ti - t;  // exclusive warp offsets
    }
    __syncthreads();
    int excl = carry + warp_tot[wid] + incl - v;
    if (i < nkeys) {
      start[i] = excl;
      cursor[i] = 0;
    }
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = excl + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) start[nkeys] = carry;
}

__global__ void k_scatter(const int *__restrict__ rebuild, int n,
                          const int *__restrict__ key, const int *__restrict__ start,
                          int *__restrict__ cursor, int *__restrict__ sorted) {
  if (!*rebuild) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int k = key[i];
  int slot = start[k] + atomicAdd(&cursor[k], 1);
  sorted[slot] = i;
}

// Deterministic order inside each fine cell: ascending atom index (the
// order ProtoMol's linked cell lists have, Topology.h:72-83).
__global__ void k_sort_keys(const int *__restrict__ rebuild, int nkeys,
                            const int *__restrict__ start, int *__restrict__ sorted,
                            int *__restrict__ key_count) {
  if (!*rebuild) return;
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nkeys) return;
  int b = start[k], e = start[k + 1];
  for (int i = b + 1; i < e; i++) {
    int v = sorted[i];
    int j = i - 1;
    while (j >= b && sorted[j] > v) {
      sorted[j + 1] = sorted[j];
      j--;
    }
    sorted[j + 1] = v;
  }
  key_count[k] = 0;  // ready for the next build
}

// Per-step gather of the sorted coordinates: xw = x - offset keeps every
// atom in the image it had at the last build, so list shifts stay valid.
template <bool MIXED>
__global__ void k_gather(int n, const double *__restrict__ pos,
                         const double *__restrict__ offset,
                         const double *__restrict__ xbuild,
                         const int *__restrict__ sorted,
                         const double *__restrict__ charge,
                         const int *__restrict__ type, float4 *__restrict__ xhi,
                         float4 *__restrict__ xlo, double4 *__restrict__ xw,
                         unsigned int *__restrict__ maxdisp) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  float d2 = 0.f;
  if (s < n) {
    int i = sorted[s];
    double x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
    double wx = x - offset[3 * i], wy = y - offset[3 * i + 1], wz = z - offset[3 * i + 2];
    double q = charge[i];
    xw[s] = make_double4(wx, wy, wz, q);
    if (MIXED) {
      float hx = (float)wx, hy = (float)wy, hz = (float)wz;
      xhi[s] = make_float4(hx, hy, hz, (float)q);
      xlo[s] = make_float4((float)(wx - (double)hx), (float)(wy - (double)hy),
                           (float)(wz - (double)hz), __int_as_float(type[i]));
    }
    double dx = x - xbuild[3 * i], dy = y - xbuild[3 * i + 1], dz = z - xbuild[3 * i + 2];
    d2 = (float)(dx * dx + dy * dy + dz * dz);
    if (!(d2 == d2)) d2 = 3.0e38f;  // NaN forces a rebuild / status check
  }
  float m = d2;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m > 0.f) atomicMax(maxdisp, __float_as_uint(m));
}

// Decide whether this step rebuilds the list: first build, forced, or an
// atom moved more than half the skin since the last build.
// rebuild[0] is the flag, rebuild[1] counts builds.
__global__ void k_check_rebuild(unsigned int *maxdisp, int *rebuild, float half_skin2,
                                int force) {
  float m = __uint_as_float(*maxdisp);
  int r = force || (m > half_skin2);
  rebuild[0] = r;
  if (r) {
    *maxdisp = 0u;
    rebuild[1] += 1;
  }
}

// ---------------------------------------------------------- list build
struct BuildArgs {
  Box box;
  int n;
  int ncx, ncy, ncz;
  double reach2;
  int cap;
  int periodic;
};

__global__ void k_build_list(BuildArgs a, const int *__restrict__ rebuild,
                             const int *__restrict__ key, const int *__restrict__ sorted,
                             const int *__restrict__ start, const double4 *__restrict__ xw,
                             const int *__restrict__ mol, uint32_t *__restrict__ nbr,
                             int *__restrict__ nbr_count, int *__restrict__ status) {
  if (!*rebuild) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  int oi = sorted[i];
  double4 pi = xw[i];
  int mi = mol[oi];
  int cell = key[oi] / kFine3;
  int cz = cell % a.ncz, cy = (cell / a.ncz) % a.ncy, cx = cell / (a.ncz * a.ncy);
  int count = 0;
  int dims[3] = {a.ncx, a.ncy, a.ncz};
  // In a non-periodic box, cells beyond the grid do not exist; in a
  // periodic box with fewer than 3 cells per axis the same cell is visited
  // under different images, which is what the Ewald image sum needs.
  for (int ddx = -1; ddx <= 1; ddx++) {
    int nx = cx + ddx, sx = 0;
    if (a.periodic) {
      if (nx < 0) { nx += dims[0]; sx = -1; }
      else if (nx >= dims[0]) { nx -= dims[0]; sx = 1; }
    } else if (nx < 0 || nx >= dims[0]) continue;
    for (int ddy = -1; ddy <= 1; ddy++) {
      int ny = cy + ddy, sy = 0;
      if (a.periodic) {
        if (ny < 0) { ny += dims[1]; sy = -1; }
        else if (ny >= dims[1]) { ny -= dims[1]; sy = 1; }
      } else if (ny < 0 || ny >= dims[1]) continue;
      for (int ddz = -1; ddz <= 1; ddz++) {
        int nz = cz + ddz, sz = 0;
        if (a.periodic) {
          if (nz < 0) { nz += dims[2]; sz = -1; }
          else if (nz >= dims[2]) { nz -= dims[2]; sz = 1; }
        } else if (nz < 0 || nz >= dims[2]) continue;
        // With one or two cells on an axis the -1/0/+1 neighbours name the
        // same cells under different images; every (cell, image) pair is
        // still distinct, and the box edge exceeds the reach, so no pair
        // is visited twice under the same image.
        int shift = (sx + 1) * 9 + (sy + 1) * 3 + (sz + 1);
        double ox = sx * a.box.e[0], oy = sy * a.box.e[1], oz = sz * a.box.e[2];
        int c2 = (nx * dims[1] + ny) * dims[2] + nz;
        int jb = start[c2 * kFine3], je = start[c2 * kFine3 + kFine3];
        for (int j = jb; j < je; j++) {
          if (j == i && shift == kZeroShift) continue;
          double4 pj = xw[j];
          double dx = (pj.x + ox) - pi.x, dy = (pj.y + oy) - pi.y, dz = (pj.z + oz) - pi.z;
          double r2 = dx * dx + dy * dy + dz * dz;
          if (r2 >= a.reach2) continue;
          uint32_t e = (uint32_t)j | ((uint32_t)shift << kShiftBits);
          int oj = sorted[j];
          if (mol[oj] == mi) {
            bool minimal = !a.periodic ||
                           (fabs(dx) <= a.box.H2[0] && fabs(dy) <= a.box.H2[1] &&
                            fabs(dz) <= a.box.H2[2]);
            if (minimal) e |= kSameMolBit;
          }
          if (count < a.cap) nbr[(size_t)count * a.n + i] = e;
          count++;
        }
      }
    }
  }
  if (count > a.cap) {
    atomicOr(status, ST_LIST_OVERFLOW);
    count = a.cap;
  }
  nbr_count[i] = count;
}

// ---------------------------------------------------------- pair kernel
template <typename Real>
struct PairArgs {
  Box box;
  int n;
  int ntypes;
  int mask;
  SwitchDev<Real> lj_sw, coul_sw;
  int lj_modify, coul_modify;
  // rough-test cutoffs^2 (FP64 exact and the FP32 band around them)
  double lj_cut2, coul_cut2, ew_cut2;
  Real lj_lo, lj_hi, coul_lo, coul_hi, ew_lo, ew_hi, max_hi;
  Real alpha, a2pi;
  int exact_erf;
  Real csf;  // coulomb scaling factor
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
// FP32/FP64 difference of the kernel, used only to pick the lattice vector.
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

template <typename Real>
__device__ __forceinline__ Real fast_exp(Real x);
template <>
__device__ __forceinline__ float fast_exp<float>(float x) { return __expf(x); }
template <>
__device__ __forceinline__ double fast_exp<double>(double x) { return exp(x); }
template <typename Real>
__device__ __forceinline__ Real fast_rsqrt(Real x);
template <>
__device__ __forceinline__ float fast_rsqrt<float>(float x) { return rsqrtf(x); }
template <>
__device__ __forceinline__ double fast_rsqrt<double>(double x) { return 1.0 / sqrt(x); }

// Thread per sorted atom i; walks its full neighbour list.  Each unordered
// pair is visited from both ends: forces are written for i only (no
// atomics on j), energies are halved.
template <typename Real, int TERMS, bool VIRIAL, bool RECORD>
__global__ void __launch_bounds__(128)
k_pairs(PairArgs<Real> a) {
  constexpr bool MIXED = sizeof(Real) == 4;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool valid = i < a.n;
  int ii = valid ? i : 0;
  int oi = a.sorted[ii];
  double4 wi = a.xw[ii];
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
  Real fx = 0, fy = 0, fz = 0, elj = 0, ec = 0;
  Real vxx = 0, vxy = 0, vxz = 0, vyy = 0, vyz = 0, vzz = 0;
  int npairs = 0;
  int cnt = valid ? a.nbr_count[ii] : 0;
  for (int k = 0; k < cnt; k++) {
    uint32_t e = a.nbr[(size_t)k * a.n + ii];
    int j = (int)(e & kJMask);
    int sh = (int)((e >> kShiftBits) & 31);
    if (sh != cur_shift) {
      // i coordinates moved by minus the j image shift: d = xj - (xi - s L)
      int sx = sh / 9 - 1, sy = (sh / 3) % 3 - 1, sz = sh % 3 - 1;
      double px = wi.x - sx * a.box.e[0], py = wi.y - sy * a.box.e[1],
             pz = wi.z - sz * a.box.e[2];
      if (MIXED) {
        float hx = (float)px, hy = (float)py, hz = (float)pz;
        xs_h[0] = hx; xs_h[1] = hy; xs_h[2] = hz;
        xs_l[0] = (float)(px - hx); xs_l[1] = (float)(py - hy); xs_l[2] = (float)(pz - hz);
      } else {
        xs_h[0] = px; xs_h[1] = py; xs_h[2] = pz;
      }
      cur_shift = sh;
    }
    Real dx, dy, dz, qj;
    int tj;
    if (MIXED) {
      float4 h = a.xhi[j], l = a.xlo[j];
      dx = (h.x - xs_h[0]) + (l.x - xs_l[0]);
      dy = (h.y - xs_h[1]) + (l.y - xs_l[1]);
      dz = (h.z - xs_h[2]) + (l.z - xs_l[2]);
      qj = h.w;
      tj = __float_as_int(l.w);
    } else {
      double4 w = a.xw[j];
      dx = w.x - xs_h[0];
      dy = w.y - xs_h[1];
      dz = w.z - xs_h[2];
      qj = w.w;
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
    // Ewald real term they skip only the minimal image, which is the
    // entry carrying the same-molecule bit (NonbondedFullEwald...h:795-801).
    if (excl == PMGPU_EXCL_FULL) {
      do_lj = false;
      do_coul = false;
      do_ew = false;
    }
    if (!(do_lj || do_coul || do_ew)) continue;
    if (!MIXED) tj = a.type[a.sorted[j]];
    Real rinv = fast_rsqrt<Real>(r2);
    Real rinv2 = rinv * rinv;
    Real f = 0;
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
      Real r6 = rinv2 * rinv2 * rinv2;
      Real r6B = B * r6;
      Real r12A = A * r6 * r6;
      Real en = r12A - r6B;
      Real ff = (Real(12) * r12A - Real(6) * r6B) * rinv2;
      if (a.lj_modify) {
        Real sv, sd;
        switch_eval<Real>(a.lj_sw, r2, sv, sd);
        ff = ff * sv - en * sd;
        en = en * sv;
      }
      elj += en;
      f += ff;
    }
    if ((TERMS & TERM_COUL) && do_coul) {
      Real en = qi * qj * rinv;
      if (excl == PMGPU_EXCL_MODIFIED) en *= a.csf;
      Real ff = en * rinv2;
      if (a.coul_modify) {
        Real sv, sd;
        switch_eval<Real>(a.coul_sw, r2, sv, sd);
        ff = ff * sv - en * sd;
        en = en * sv;
      }
      ec += en;
      f += ff;
    }
    if ((TERMS & TERM_EWALD) && do_ew) {
      Real qq = qi * qj;
      if (excl == PMGPU_EXCL_MODIFIED) qq *= a.csf;
      Real r = r2 * rinv;
      Real ar = a.alpha * r;
      Real ee = qq * fast_exp<Real>(-ar * ar);
      Real en;
      if (!a.exact_erf) {
        en = poly5<Real>(ar) * ee * rinv;
      } else {
        en = qq * erfc(ar) * rinv;  // USE_EWALD_EXACT_ERF: libm erfc
      }
      Real ff = (en + a.a2pi * ee) * rinv2;
      ec += en;
      f += ff;
    }
    npairs++;
    fx -= dx * f;
    fy -= dy * f;
    fz -= dz * f;
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
  if (valid) {
    red_add(&a.force[oi], to_fixed((double)fx, kForceScale));
    red_add(&a.force[a.n + oi], to_fixed((double)fy, kForceScale));
    red_add(&a.force[2 * a.n + oi], to_fixed((double)fz, kForceScale));
  }
  double dlj = warp_sum((double)elj) * 0.5;
  double dc = warp_sum((double)ec) * 0.5;
  int np = warp_sum(npairs);
  double v[6];
  if (VIRIAL) {
    v[0] = warp_sum((double)vxx); v[1] = warp_sum((double)vxy);
    v[2] = warp_sum((double)vxz); v[3] = warp_sum((double)vyy);
    v[4] = warp_sum((double)vyz); v[5] = warp_sum((double)vzz);
  }
  if ((threadIdx.x & 31) == 0) {
    if (TERMS & TERM_LJ) red_add(&a.acc[ACC_LJ], to_fixed(dlj, kEnergyScale));
    if (TERMS & (TERM_COUL | TERM_EWALD)) red_add(&a.acc[ACC_COULOMB], to_fixed(dc, kEnergyScale));
    red_add(&a.acc[ACC_PAIRS], (long long)np);
    if (VIRIAL) {
      const int map[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
      for (int q = 0; q < 9; q++) red_add(&a.acc[ACC_VIRIAL + q], to_fixed(v[map[q]], kEnergyScale));
    }
  }
}

// ------------------------------------------------------------ host side
int nb_list_init(System *s, NeighborList *nl, double cutoff, double skin, double) {
  nl->cutoff = cutoff;
  nl->skin = skin;
  nl->reach = cutoff + skin;
  int n = s->n;
  const Box &b = s->box;
  if (b.periodic) {
    for (int a = 0; a < 3; a++)
      if (b.e[a] <= nl->reach)
        return fail(PMGPU_ERR_UNSUPPORTED,
                    "box edge must exceed cutoff + list skin on the cell-list path");
    // CubicCellManager::initialize (CubicCellManager.cpp:46-65) and
    // ArrayCellListStructure::initialize (ArrayCellListStructure.cpp:40-42)
    int dims[3];
    for (int a = 0; a < 3; a++) {
      double vd = b.max[a] - b.min[a];
      double f = std::floor(vd / nl->reach);
      nl->cs[a] = vd / std::max(1.0, f);
      dims[a] = std::max(1, (int)std::floor(vd / nl->cs[a] + kEpsilon));
    }
    nl->ncx = dims[0]; nl->ncy = dims[1]; nl->ncz = dims[2];
  } else {
    // Vacuum: a fixed grid over the current bounding box plus a margin of
    // one reach; atoms that later leave it clamp into the edge cells
    // (cells only accelerate the search, they never drop a pair).
    std::vector<double> h(3 * (size_t)std::max(n, 1), 0.0);
    if (n) PM_CUDA(cudaMemcpy(h.data(), s->d_pos, sizeof(double) * 3 * n,
                              cudaMemcpyDeviceToHost));
    double mn[3] = {0, 0, 0}, mx[3] = {0, 0, 0};
    for (int a = 0; a < 3; a++) { mn[a] = h[a]; mx[a] = h[a]; }
    for (int i = 1; i < n; i++)
      for (int a = 0; a < 3; a++) {
        mn[a] = std::min(mn[a], h[3 * i + a]);
        mx[a] = std::max(mx[a], h[3 * i + a]);
      }
    int dims[3];
    for (int a = 0; a < 3; a++) {
      double span = (mx[a] - mn[a]) + 2 * nl->reach;
      dims[a] = std::max(1, std::min(128, (int)std::floor(span / nl->reach)));
      nl->cs[a] = span / dims[a];
      nl->vac_origin[a] = mn[a] - nl->reach;
    }
    nl->ncx = dims[0]; nl->ncy = dims[1]; nl->ncz = dims[2];
  }
  nl->nkeys = nl->ncx * nl->ncy * nl->ncz * kFine3;
  // capacity: expected neighbours in the reach sphere at the mean density,
  // with headroom for local fluctuations (overflow is detected and
  // reported, and the next call doubles the capacity).
  double dens = b.periodic ? n / b.V : 0.15;
  double expect = 4.18879 * nl->reach * nl->reach * nl->reach * dens;
  int cap = (int)(expect * 1.5 + 64);
  cap = std::min(cap, std::max(32, n));
  cap = (cap + 31) & ~31;
  if (nl->cap > cap) cap = nl->cap;
  nl->cap = cap;
  size_t nn = std::max(1, n);
  PM_CUDA(cudaMalloc(&nl->d_key, sizeof(int) * nn));
  PM_CUDA(cudaMalloc(&nl->d_key_count, sizeof(int) * nl->nkeys));
  PM_CUDA(cudaMemset(nl->d_key_count, 0, sizeof(int) * nl->nkeys));
  PM_CUDA(cudaMalloc(&nl->d_key_start, sizeof(int) * (nl->nkeys + 1)));
  PM_CUDA(cudaMalloc(&nl->d_key_cursor, sizeof(int) * nl->nkeys));
  PM_CUDA(cudaMalloc(&nl->d_sorted, sizeof(int) * nn));
  PM_CUDA(cudaMalloc(&nl->d_offset, sizeof(double) * 3 * nn));
  PM_CUDA(cudaMalloc(&nl->d_xbuild, sizeof(double) * 3 * nn));
  PM_CUDA(cudaMalloc(&nl->d_xhi, sizeof(float4) * nn));
  PM_CUDA(cudaMalloc(&nl->d_xlo, sizeof(float4) * nn));
  PM_CUDA(cudaMalloc(&nl->d_xw, sizeof(double4) * nn));
  PM_CUDA(cudaMalloc(&nl->d_nbr, sizeof(uint32_t) * (size_t)cap * nn));
  PM_CUDA(cudaMalloc(&nl->d_nbr_count, sizeof(int) * nn));
  PM_CUDA(cudaMemset(nl->d_nbr_count, 0, sizeof(int) * nn));
  PM_CUDA(cudaMalloc(&nl->d_maxdisp, sizeof(unsigned int)));
  PM_CUDA(cudaMemset(nl->d_maxdisp, 0, sizeof(unsigned int)));
  PM_CUDA(cudaMalloc(&nl->d_rebuild, 2 * sizeof(int)));
  PM_CUDA(cudaMemset(nl->d_rebuild, 0, 2 * sizeof(int)));
  nl->built = 0;
  return PMGPU_OK;
}

int nb_list_free(NeighborList *nl) {
  void *ptrs[] = {nl->d_key, nl->d_key_count, nl->d_key_start, nl->d_key_cursor,
                  nl->d_sorted, nl->d_offset, nl->d_xbuild, nl->d_xhi, nl->d_xlo,
                  nl->d_xw, nl->d_nbr, nl->d_nbr_count, nl->d_maxdisp, nl->d_rebuild};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  nl->d_key = nullptr; nl->d_key_count = nullptr; nl->d_key_start = nullptr;
  nl->d_key_cursor = nullptr; nl->d_sorted = nullptr; nl->d_offset = nullptr;
  nl->d_xbuild = nullptr; nl->d_xhi = nullptr; nl->d_xlo = nullptr;
  nl->d_xw = nullptr; nl->d_nbr = nullptr; nl->d_nbr_count = nullptr;
  nl->d_maxdisp = nullptr; nl->d_rebuild = nullptr;
  return PMGPU_OK;
}

static GridArgs make_grid(const System *s, const NeighborList *nl) {
  GridArgs g;
  g.box = s->box;
  g.n = s->n;
  g.ncx = nl->ncx; g.ncy = nl->ncy; g.ncz = nl->ncz;
  for (int a = 0; a < 3; a++) {
    g.cs[a] = nl->cs[a];
    g.inv[a] = 1.0 / nl->cs[a];
    g.delta[a] = s->box.periodic ? s->box.origin[a] - s->box.min[a] : 0.0;
    g.vmin[a] = s->box.periodic ? 0.0 : nl->vac_origin[a];
  }
  return g;
}

// Sort + (conditional) list build + per-step gather.  Never synchronises
// with the host: the rebuild decision lives in device memory.
int nb_prepare(System *s, NeighborList *nl, int force_rebuild) {
  int n = s->n;
  if (n == 0) return PMGPU_OK;
  cudaStream_t st = s->stream;
  const int T = 256;
  int nb = (n + T - 1) / T;
  int first = !nl->built;
  float hs = (float)(0.5 * nl->skin);
  k_check_rebuild<<<1, 1, 0, st>>>(nl->d_maxdisp, nl->d_rebuild, hs * hs,
                                   (force_rebuild || first) ? 1 : 0);
  GridArgs g = make_grid(s, nl);
  k_bin<<<nb, T, 0, st>>>(g, s->d_pos, nl->d_rebuild, nl->d_key, nl->d_key_count,
                          nl->d_offset, nl->d_xbuild, s->d_status);
  k_scan<<<1, 1024, 0, st>>>(nl->d_rebuild, nl->d_key_count, nl->d_key_start,
                             nl->d_key_cursor, nl->nkeys);
  k_scatter<<<nb, T, 0, st>>>(nl->d_rebuild, n, nl->d_key, nl->d_key_start,
                              nl->d_key_cursor, nl->d_sorted);
  k_sort_keys<<<(nl->nkeys + T - 1) / T, T, 0, st>>>(nl->d_rebuild, nl->nkeys,
                                                    nl->d_key_start, nl->d_sorted,
                                                    nl->d_key_count);
  if (s->precision == PMGPU_PREC_MIXED)
    k_gather<true><<<nb, T, 0, st>>>(n, s->d_pos, nl->d_offset, nl->d_xbuild,
                                     nl->d_sorted, s->d_charge, s->d_type, nl->d_xhi,
                                     nl->d_xlo, nl->d_xw, nl->d_maxdisp);
  else
    k_gather<false><<<nb, T, 0, st>>>(n, s->d_pos, nl->d_offset, nl->d_xbuild,
                                      nl->d_sorted, s->d_charge, s->d_type, nl->d_xhi,
                                      nl->d_xlo, nl->d_xw, nl->d_maxdisp);
  BuildArgs ba;
  ba.box = s->box;
  ba.n = n;
  ba.ncx = nl->ncx; ba.ncy = nl->ncy; ba.ncz = nl->ncz;
  ba.reach2 = nl->reach * nl->reach;
  ba.cap = nl->cap;
  ba.periodic = s->box.periodic;
  k_build_list<<<(n + 127) / 128, 128, 0, st>>>(ba, nl->d_rebuild, nl->d_key,
                                                nl->d_sorted, nl->d_key_start, nl->d_xw,
                                                s->d_mol, nl->d_nbr, nl->d_nbr_count,
                                                s->d_status);
  PM_CUDA(cudaGetLastError());
  nl->built = 1;
  return PMGPU_OK;
}

template <typename Real>
static void fill_pair_args(PairArgs<Real> &a, System *s, NeighborList *nl,
                           const PairTerms &t) {
  a.box = s->box;
  a.n = s->n;
  a.ntypes = s->ntypes;
  a.mask = t.mask;
  a.lj_sw = make_switch_dev<Real>(t.lj_sw);
  a.coul_sw = make_switch_dev<Real>(t.coul_sw);
  a.lj_modify = t.lj_sw.modify;
  a.coul_modify = t.coul_sw.modify;
  // The FP32 squared distance is within ~1e-5 A^2 of the exact one; pairs
  // inside this relative band are re-tested in FP64.
  const double band = sizeof(Real) == 4 ? 4.0e-5 : 1.0e-12;
  a.lj_cut2 = t.lj_cut2;
  a.coul_cut2 = t.coul_cut2;
  a.ew_cut2 = t.ewald_rc2;
  a.lj_lo = (Real)(t.lj_cut2 * (1 - band));
  a.lj_hi = (Real)(t.lj_cut2 * (1 + band));
  a.coul_lo = (Real)(t.coul_cut2 * (1 - band));
  a.coul_hi = (Real)(t.coul_cut2 * (1 + band));
  a.ew_lo = (Real)(t.ewald_rc2 * (1 - band));
  a.ew_hi = (Real)(t.ewald_rc2 * (1 + band));
  double mx = 0;
  if (t.mask & TERM_LJ) mx = std::max(mx, t.lj_cut2);
  if (t.mask & TERM_COUL) mx = std::max(mx, t.coul_cut2);
  if (t.mask & TERM_EWALD) mx = std::max(mx, t.ewald_rc2);
  a.max_hi = (Real)(mx * (1 + band));
  a.alpha = (Real)t.ewald_alpha;
  a.a2pi = (Real)(2.0 * t.ewald_alpha / std::sqrt(M_PI));
  a.exact_erf = t.exact_erf;
  a.csf = (Real)t.coulomb_scaling;
  a.cap = nl->cap;
  a.sorted = nl->d_sorted;
  a.pos = s->d_pos;
  a.excl_start = s->d_excl_start;
  a.excl_partner = s->d_excl_partner;
  a.excl_class = s->d_excl_class;
  a.nbr = nl->d_nbr;
  a.nbr_count = nl->d_nbr_count;
  a.xhi = nl->d_xhi;
  a.xlo = nl->d_xlo;
  a.xw = nl->d_xw;
  a.type = s->d_type;
  a.lj32 = s->d_lj32;
  a.lj64 = s->d_lj64;
  a.force = s->d_force;
  a.acc = s->d_acc;
  a.pairbuf = s->d_pairbuf;
  a.pairbuf_cap = s->pairbuf_cap;
  a.paircount = s->d_paircount;
}

template <typename Real, int TERMS>
static void launch_pairs_t(PairArgs<Real> &a, cudaStream_t st, int virial, int record) {
  int nb = (a.n + 127) / 128;
  if (record)
    k_pairs<Real, TERMS, false, true><<<nb, 128, 0, st>>>(a);
  else if (virial)
    k_pairs<Real, TERMS, true, false><<<nb, 128, 0, st>>>(a);
  else
    k_pairs<Real, TERMS, false, false><<<nb, 128, 0, st>>>(a);
}

template <typename Real>
static int launch_pairs(PairArgs<Real> &a, cudaStream_t st, int virial, int record) {
  switch (a.mask) {
    case TERM_LJ: launch_pairs_t<Real, TERM_LJ>(a, st, virial, record); break;
    case TERM_COUL: launch_pairs_t<Real, TERM_COUL>(a, st, virial, record); break;
    case TERM_LJ | TERM_COUL:
      launch_pairs_t<Real, TERM_LJ | TERM_COUL>(a, st, virial, record); break;
    case TERM_EWALD: launch_pairs_t<Real, TERM_EWALD>(a, st, virial, record); break;
    case TERM_LJ | TERM_EWALD:
      launch_pairs_t<Real, TERM_LJ | TERM_EWALD>(a, st, virial, record); break;
    default:
      return fail(PMGPU_ERR_UNSUPPORTED, "unsupported pair-term combination");
  }
  PM_CUDA(cudaGetLastError());
  return PMGPU_OK;
}

int nb_pair_forces(System *s, NeighborList *nl, const PairTerms &t, int want_virial,
                   int record_pairs) {
  if (s->n == 0) return PMGPU_OK;
  if (s->precision == PMGPU_PREC_MIXED) {
    PairArgs<float> a;
    fill_pair_args<float>(a, s, nl, t);
    return launch_pairs<float>(a, s->stream, want_virial, record_pairs);
  }
  PairArgs<double> a;
  fill_pair_args<double>(a, s, nl, t);
  return launch_pairs<double>(a, s->stream, want_virial, record_pairs);
}

// ProtoMol cell assignment with a given cellsize on the resident positions
// (the same binning kernel the list path runs, fed ProtoMol's own cell
// sizes).  Positions are downloaded only to form the vacuum bounding box,
// exactly as Topology::updateCellLists does (Topology.h:47-53).
__global__ void k_cells_debug(GridArgs g, const double *__restrict__ pos,
                              int *__restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.n) return;
  int c[3];
  double w[3], fr[3];
  cell_of(g, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], c, w, fr);
  out[3 * i] = c[0];
  out[3 * i + 1] = c[1];
  out[3 * i + 2] = c[2];
}

int nb_debug_cells(System *s, double cellsize, int *cell_xyz, int *dims) {
  int n = s->n;
  GridArgs g;
  g.box = s->box;
  g.n = n;
  double mn[3], mx[3];
  if (s->box.periodic) {
    for (int a = 0; a < 3; a++) { mn[a] = s->box.min[a]; mx[a] = s->box.max[a]; }
  } else {
    std::vector<double> h(3 * (size_t)std::max(n, 1), 0.0);
    if (n) PM_CUDA(cudaMemcpy(h.data(), s->d_pos, sizeof(double) * 3 * n,
                              cudaMemcpyDeviceToHost));
    // Vector3DBlock::boundingbox (type/Vector3DBlock.cpp:9-35)
    for (int a = 0; a < 3; a++) mn[a] = mx[a] = h[a];
    for (int i = 1; i < n; i++)
      for (int a = 0; a < 3; a++) {
        double v = h[3 * i + a];
        if (v < mn[a]) mn[a] = v;
        else if (v > mx[a]) mx[a] = v;
      }
  }
  int d[3];
  for (int a = 0; a < 3; a++) {
    double vd = mx[a] - mn[a], cs, vres;
    if (s->box.periodic) {
      double f = std::floor(vd / cellsize);
      cs = vd / std::max(1.0, f);
      vres = vd;
    } else {
      cs = cellsize;
      vres = vd + cellsize;
    }
    d[a] = std::max(1, (int)std::floor(vres / cs + kEpsilon));
    g.cs[a] = cs;
    g.inv[a] = 1.0 / cs;
    g.delta[a] = s->box.periodic ? s->box.origin[a] - mn[a] : 0.0;
    g.vmin[a] = s->box.periodic ? 0.0 : mn[a];
  }
  g.ncx = d[0]; g.ncy = d[1]; g.ncz = d[2];
  int *dout = nullptr;
  PM_CUDA(cudaMalloc(&dout, sizeof(int) * 3 * std::max(n, 1)));
  if (n) k_cells_debug<<<(n + 255) / 256, 256, 0, s->stream>>>(g, s->d_pos, dout);
  cudaError_t e = cudaMemcpyAsync(cell_xyz, dout, sizeof(int) * 3 * n,
                                  cudaMemcpyDeviceToHost, s->stream);
  cudaError_t e2 = cudaStreamSynchronize(s->stream);
  cudaFree(dout);
  if (e != cudaSuccess || e2 != cudaSuccess)
    return fail(PMGPU_ERR_CUDA, "debug cell assignment failed");
  dims[0] = d[0]; dims[1] = d[1]; dims[2] = d[2];
  return PMGPU_OK;
}

// --------------------------------------------------- NonbondedSimpleFull
// Vacuum all pairs with exclusions (NonbondedSimpleFullSystemForce.h:125-150
// with OneAtomPair<Vacuum, Universal, LennardJones|Coulomb>): block tiles of
// 128 i atoms against j tiles staged in shared memory; every i sees every
// j != i, energies halved.
template <typename Real, bool LJ, bool COUL>
__global__ void __launch_bounds__(128)
k_simplefull(int n, const double *__restrict__ pos, const double *__restrict__ charge,
             const int *__restrict__ type, const int *__restrict__ mol, int ntypes,
             const double4 *__restrict__ lj64, const int *__restrict__ ex_start,
             const int *__restrict__ ex_partner, const int *__restrict__ ex_class,
             Real csf, long long *__restrict__ force, long long *__restrict__ acc,
             int want_virial) {
  __shared__ double sx[128], sy[128], sz[128], sq[128];
  __shared__ int st[128], sm[128];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool valid = i < n;
  double xi = 0, yi = 0, zi = 0, qi = 0;
  int ti = 0, mi = -1;
  if (valid) {
    xi = pos[3 * i]; yi = pos[3 * i + 1]; zi = pos[3 * i + 2];
    qi = charge[i]; ti = type[i]; mi = mol[i];
  }
  Real fx = 0, fy = 0, fz = 0;
  double elj = 0, ec = 0;
  double v[6] = {0, 0, 0, 0, 0, 0};
  for (int base = 0; base < n; base += 128) {
    int j = base + threadIdx.x;
    if (j < n) {
      sx[threadIdx.x] = pos[3 * j]; sy[threadIdx.x] = pos[3 * j + 1];
      sz[threadIdx.x] = pos[3 * j + 2]; sq[threadIdx.x] = charge[j];
      st[threadIdx.x] = type[j]; sm[threadIdx.x] = mol[j];
    }
    __syncthreads();
    int lim = min(128, n - base);
    if (valid) {
      for (int k = 0; k < lim; k++) {
        int jj = base + k;
        if (jj == i) continue;
        int excl = PMGPU_EXCL_NONE;
        if (sm[k] == mi) {
          excl = excl_lookup(ex_start, ex_partner, ex_class, i, jj);
          if (excl == PMGPU_EXCL_FULL) continue;
        }
        Real dx = (Real)(sx[k] - xi), dy = (Real)(sy[k] - yi), dz = (Real)(sz[k] - zi);
        Real r2 = dx * dx + dy * dy + dz * dz;
        Real rr2 = Real(1) / r2;
        Real f = 0;
        if (LJ) {
          double4 p = lj64[ti * ntypes + st[k]];
          Real A = (Real)(excl == PMGPU_EXCL_MODIFIED ? p.z : p.x);
          Real B = (Real)(excl == PMGPU_EXCL_MODIFIED ? p.w : p.y);
          Real r6 = rr2 * rr2 * rr2;
          Real r6B = B * r6, r12A = A * r6 * r6;
          elj += (double)(r12A - r6B);
          f += (Real(12) * r12A - Real(6) * r6B) * rr2;
        }
        if (COUL) {
          Real en = (Real)(qi * sq[k]) * pm_sqrt(rr2);
          if (excl == PMGPU_EXCL_MODIFIED) en *= csf;
          ec += (double)en;
          f += en * rr2;
        }
        fx -= dx * f; fy -= dy * f; fz -= dz * f;
        if (want_virial) {
          double hf = 0.5 * (double)f;
          v[0] += dx * dx * hf; v[1] += dx * dy * hf; v[2] += dx * dz * hf;
          v[3] += dy * dy * hf; v[4] += dy * dz * hf; v[5] += dz * dz * hf;
        }
      }
    }
    __syncthreads();
  }
  if (valid) {
    red_add(&force[i], to_fixed((double)fx, kForceScale));
    red_add(&force[n + i], to_fixed((double)fy, kForceScale));
    red_add(&force[2 * n + i], to_fixed((double)fz, kForceScale));
  }
  elj = warp_sum(elj) * 0.5;
  ec = warp_sum(ec) * 0.5;
  for (int q = 0; q < 6; q++) v[q] = warp_sum(v[q]);
  if ((threadIdx.x & 31) == 0) {
    if (LJ) red_add(&acc[ACC_LJ], to_fixed(elj, kEnergyScale));
    if (COUL) red_add(&acc[ACC_COULOMB], to_fixed(ec, kEnergyScale));
    if (want_virial) {
      const int map[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
      for (int q = 0; q < 9; q++) red_add(&acc[ACC_VIRIAL + q], to_fixed(v[map[q]], kEnergyScale));
    }
  }
}

int nb_simplefull(System *s, int lj, int coul, int want_virial) {
  int n = s->n;
  if (n == 0 || !(lj || coul)) return PMGPU_OK;
  int nb = (n + 127) / 128;
  auto go = [&](auto kern, auto csf) {
    kern<<<nb, 128, 0, s->stream>>>(n, s->d_pos, s->d_charge, s->d_type, s->d_mol,
                                    s->ntypes, s->d_lj64, s->d_excl_start,
                                    s->d_excl_partner, s->d_excl_class, csf, s->d_force,
                                    s->d_acc, want_virial);
  };
  if (s->precision == PMGPU_PREC_MIXED) {
    float csf = (float)s->coulomb_scaling;
    if (lj && coul) go(k_simplefull<float, true, true>, csf);
    else if (lj) go(k_simplefull<float, true, false>, csf);
    else go(k_simplefull<float, false, true>, csf);
  } else {
    double csf = s->coulomb_scaling;
    if (lj && coul) go(k_simplefull<double, true, true>, csf);
    else if (lj) go(k_simplefull<double, true, false>, csf);
    else go(k_simplefull<double, false, true>, csf);
  }
  PM_CUDA(cudaGetLastError());
  return PMGPU_OK;
}

}  // namespace pmgpu
