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

// Sort key of an atom: coarse xy column, then the global fine z layer
// (kFine layers per coarse cell), then a Morton-ordered kFine x kFine xy
// sub-cell.  Every column is one contiguous z-sorted range, so the list
// build reads the atoms of a neighbour column within the reach in z as one
// slice.
__device__ __forceinline__ int morton2(int x, int y) {
  int m = 0;
#pragma unroll
  for (int b = 0; b < 2; b++) {
    m |= ((x >> b) & 1) << (2 * b + 1);
    m |= ((y >> b) & 1) << (2 * b);
  }
  return m;
}
__device__ __forceinline__ int sort_key(int cx, int cy, int layer, int fx, int fy, int ncy,
                                        int nlayers) {
  return ((cx * ncy + cy) * nlayers + layer) * (kFine * kFine) + morton2(fx, fy);
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
  int k = sort_key(c[0], c[1], c[2] * kFine + f[2], f[0], f[1], g.ncy, g.ncz * kFine);
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
// xhi (FP32 position + charge) feeds the list build in both precisions;
// xlo (the FP32 residue + type) only the mixed-precision pair kernel.
template <bool MIXED>
__global__ void k_gather(int n, const double *__restrict__ pos,
                         const double *__restrict__ offset,
                         const double *__restrict__ xbuild,
                         const int *__restrict__ sorted,
                         const double *__restrict__ charge,
                         const int *__restrict__ type, const int *__restrict__ mol,
                         float4 *__restrict__ xhi, float4 *__restrict__ xlo,
                         double4 *__restrict__ xw, int *__restrict__ mol_s,
                         unsigned int *__restrict__ maxdisp) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  float d2 = 0.f;
  if (s < n) {
    int i = sorted[s];
    double x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
    double wx = x - offset[3 * i], wy = y - offset[3 * i + 1], wz = z - offset[3 * i + 2];
    double q = charge[i];
    xw[s] = make_double4(wx, wy, wz, q);
    float hx = (float)wx, hy = (float)wy, hz = (float)wz;
    xhi[s] = make_float4(hx, hy, hz, (float)q);
    if (MIXED)
      xlo[s] = make_float4((float)(wx - (double)hx), (float)(wy - (double)hy),
                           (float)(wz - (double)hz), __int_as_float(type[i]));
    mol_s[s] = mol[i];
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
  float reach2;       // FP32 candidate radius^2 (reach plus a rounding margin)
  float cull2;        // column culling radius^2 (wider margin)
  float cell_lo[3];   // lower corner of cell 0 in the xw frame
  float cs[3];        // coarse cell size
  float inv_layer;    // 1 / fine z-layer thickness
  int nlayers;        // fine z layers per column
  float L[3];         // box edges
  float H2[3];        // half box edges (minimal-image test)
  int cap;
  int periodic;
  const int *excl_start, *excl_partner, *excl_class;
};

__device__ __forceinline__ int excl_class_of(const int *start, const int *partner,
                                             const int *cls, int oi, int oj) {
  int b = start[oi], e = start[oi + 1];
  for (int k = b; k < e; k++)
    if (partner[k] == oj) return cls[k];
  return PMGPU_EXCL_NONE;
}

// One warp per sorted atom: for each of the 9 neighbour columns (skipping
// columns whose xy box lies beyond the reach) the warp reads the slice of
// fine z layers within the reach (split where it wraps through the periodic
// z face), tests 32 candidates at a time in FP32 against (reach + margin)^2
// and compacts passing entries with a warp ballot, so every row is written
// in a fixed (column, layer, index) order.  Exclusions are resolved here
// (ExclusionTable::check, topology/ExclusionTable.h:116-130, consulted only
// for same-molecule minimal-image pairs as in OneAtomPairTwo.h:47-53):
// fully excluded pairs are dropped, modified pairs flagged.
__global__ void __launch_bounds__(kBuildWarps * 32)
k_build_list(BuildArgs a, const int *__restrict__ rebuild, const int *__restrict__ key,
             const int *__restrict__ sorted, const int *__restrict__ start,
             const float4 *__restrict__ xhi, const int *__restrict__ mol_s,
             uint32_t *__restrict__ nbr, int *__restrict__ nbr_count,
             int *__restrict__ status) {
  if (!*rebuild) return;
  const int lane = threadIdx.x & 31;
  const int i = blockIdx.x * kBuildWarps + (threadIdx.x >> 5);
  if (i >= a.n) return;  // whole warps exit together
  const unsigned lt_mask = (1u << lane) - 1u;
  const int oi = sorted[i];
  const float4 pi = xhi[i];
  const int mi = mol_s[i];
  const int col = key[oi] / (a.nlayers * kFine * kFine);
  const int cy = col % a.ncy, cx = col / a.ncy;
  const int nl = a.nlayers;
  uint32_t *row = nbr + (size_t)i * a.cap;
  int count = 0;

  // candidates of one contiguous slice [jb, je) seen under image (sx, sy, sz)
  auto scan = [&](int jb, int je, int sx, int sy, int sz) {
    const uint32_t sbits = (uint32_t)shift_code(sx, sy, sz) << kShiftBits;
    const bool zero = (sx | sy | sz) == 0;
    const float ox = pi.x - sx * a.L[0];
    const float oy = pi.y - sy * a.L[1];
    const float oz = pi.z - sz * a.L[2];
    for (int j0 = jb; j0 < je; j0 += 32) {
      const int j = j0 + lane;
      bool pass = false;
      uint32_t flags = 0;
      if (j < je && !(j == i && zero)) {
        const float4 pj = xhi[j];
        const float dx = pj.x - ox, dy = pj.y - oy, dz = pj.z - oz;
        pass = dx * dx + dy * dy + dz * dz < a.reach2;
        if (pass && mol_s[j] == mi) {
          const bool minimal = !a.periodic || (fabsf(dx) <= a.H2[0] &&
                                               fabsf(dy) <= a.H2[1] && fabsf(dz) <= a.H2[2]);
          if (minimal) {
            const int cls = excl_class_of(a.excl_start, a.excl_partner, a.excl_class, oi,
                                          sorted[j]);
            if (cls == PMGPU_EXCL_FULL) pass = false;
            else if (cls == PMGPU_EXCL_MODIFIED) flags = kModifiedBit;
          }
        }
      }
      const unsigned m = __ballot_sync(0xffffffffu, pass);
      if (pass) {
        const int slot = count + __popc(m & lt_mask);
        if (slot < a.cap) row[slot] = (uint32_t)j | sbits | flags;
      }
      count += __popc(m);
    }
  };
  auto slice = [&](int c2, int l0, int l1) {  // layers l0..l1 of column c2
    const int base = c2 * nl * (kFine * kFine);
    return make_int2(start[base + l0 * (kFine * kFine)],
                     start[base + (l1 + 1) * (kFine * kFine)]);
  };

  // With one or two columns on an axis the -1/0/+1 neighbours name the same
  // columns under different images; every (column, image) pair is distinct
  // and the box edge exceeds the reach, so no pair appears twice under one
  // image.
  for (int ddx = -1; ddx <= 1; ddx++) {
    int nx = cx + ddx, sx = 0;
    if (a.periodic) {
      if (nx < 0) { nx += a.ncx; sx = -1; }
      else if (nx >= a.ncx) { nx -= a.ncx; sx = 1; }
    } else if (nx < 0 || nx >= a.ncx) continue;
    for (int ddy = -1; ddy <= 1; ddy++) {
      int ny = cy + ddy, sy = 0;
      if (a.periodic) {
        if (ny < 0) { ny += a.ncy; sy = -1; }
        else if (ny >= a.ncy) { ny -= a.ncy; sy = 1; }
      } else if (ny < 0 || ny >= a.ncy) continue;
      const int c2 = nx * a.ncy + ny;
      if (!a.periodic) {  // vacuum: atoms may be clamped into edge cells
        int2 r = slice(c2, 0, nl - 1);
        scan(r.x, r.y, 0, 0, 0);
        continue;
      }
      // xy distance from the atom to this column's box (in this image)
      const float lox = a.cell_lo[0] + (cx + ddx) * a.cs[0];
      const float loy = a.cell_lo[1] + (cy + ddy) * a.cs[1];
      const float gx = fmaxf(fmaxf(lox - pi.x, pi.x - (lox + a.cs[0])), 0.f);
      const float gy = fmaxf(fmaxf(loy - pi.y, pi.y - (loy + a.cs[1])), 0.f);
      const float g2 = gx * gx + gy * gy;
      if (g2 > a.cull2) continue;
      const float hz = sqrtf(a.cull2 - g2);  // z half-range of the reach sphere
      const int l0 = (int)floorf((pi.z - hz - a.cell_lo[2]) * a.inv_layer);
      const int l1 = (int)floorf((pi.z + hz - a.cell_lo[2]) * a.inv_layer);
      // layers below 0 are the top of the box seen one box length down
      // (j image sz = -1); layers past the top the bottom one length up
      if (l0 < 0) {
        int2 r = slice(c2, max(nl + l0, 0), nl - 1);
        scan(r.x, r.y, sx, sy, -1);
      }
      {
        int2 r = slice(c2, max(l0, 0), min(l1, nl - 1));
        scan(r.x, r.y, sx, sy, 0);
      }
      if (l1 >= nl) {
        int2 r = slice(c2, 0, min(l1 - nl, nl - 1));
        scan(r.x, r.y, sx, sy, 1);
      }
    }
  }
  if (lane == 0) {
    if (count > a.cap) {
      atomicOr(status, ST_LIST_OVERFLOW);
      count = a.cap;
    }
    nbr_count[i] = count;
  }
}

}  // namespace pmgpu

// ---------------------------------------------------------- pair kernel
#include "pair_kernel.cuh"

namespace pmgpu {

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
    if (n) {
      PM_CUDA(cudaMemcpyAsync(h.data(), s->d_pos, sizeof(double) * 3 * n,
                              cudaMemcpyDeviceToHost, s->stream));
      PM_CUDA(cudaStreamSynchronize(s->stream));
    }
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
  // Condensed matter (liquid water ~0.1 atoms/A^3) bounds the local
  // density even in sparse boxes, where atoms still cluster.
  double dens = b.periodic ? std::max(n / b.V, 0.12) : 0.15;
  double expect = 4.18879 * nl->reach * nl->reach * nl->reach * dens;
  int cap = (int)(expect * 1.5 + 64);
  cap = std::min(cap, std::max(32, n));
  cap = (cap + 31) & ~31;
  if (nl->cap > cap) cap = nl->cap;
  nl->cap = cap;
  size_t nn = std::max(1, n);
  PM_CHECK(dev_alloc(s, &nl->d_key, sizeof(int) * nn));
  PM_CHECK(dev_alloc(s, &nl->d_key_count, sizeof(int) * nl->nkeys));
  PM_CUDA(cudaMemsetAsync(nl->d_key_count, 0, sizeof(int) * nl->nkeys, s->stream));
  PM_CHECK(dev_alloc(s, &nl->d_key_start, sizeof(int) * (nl->nkeys + 1)));
  PM_CHECK(dev_alloc(s, &nl->d_key_cursor, sizeof(int) * nl->nkeys));
  PM_CHECK(dev_alloc(s, &nl->d_sorted, sizeof(int) * nn));
  PM_CHECK(dev_alloc(s, &nl->d_offset, sizeof(double) * 3 * nn));
  PM_CHECK(dev_alloc(s, &nl->d_xbuild, sizeof(double) * 3 * nn));
  PM_CHECK(dev_alloc(s, &nl->d_xhi, sizeof(float4) * nn));
  PM_CHECK(dev_alloc(s, &nl->d_xlo, sizeof(float4) * nn));
  PM_CHECK(dev_alloc(s, &nl->d_xw, sizeof(double4) * nn));
  PM_CHECK(dev_alloc(s, &nl->d_mol_s, sizeof(int) * nn));
  PM_CHECK(dev_alloc(s, &nl->d_nbr, sizeof(uint32_t) * (size_t)cap * nn));
  PM_CHECK(dev_alloc(s, &nl->d_nbr_count, sizeof(int) * nn));
  PM_CUDA(cudaMemsetAsync(nl->d_nbr_count, 0, sizeof(int) * nn, s->stream));
  PM_CHECK(dev_alloc(s, &nl->d_maxdisp, sizeof(unsigned int)));
  PM_CUDA(cudaMemsetAsync(nl->d_maxdisp, 0, sizeof(unsigned int), s->stream));
  PM_CHECK(dev_alloc(s, &nl->d_rebuild, 2 * sizeof(int)));
  PM_CUDA(cudaMemsetAsync(nl->d_rebuild, 0, 2 * sizeof(int), s->stream));
  nl->built = 0;
  return PMGPU_OK;
}

int nb_list_free(System *s, NeighborList *nl) {
  void *ptrs[] = {nl->d_key, nl->d_key_count, nl->d_key_start, nl->d_key_cursor,
                  nl->d_sorted, nl->d_offset, nl->d_xbuild, nl->d_xhi, nl->d_xlo,
                  nl->d_xw, nl->d_nbr, nl->d_nbr_count, nl->d_maxdisp, nl->d_rebuild,
                  nl->d_mol_s};
  for (void *p : ptrs) dev_free(s, p);
  nl->d_key = nullptr; nl->d_key_count = nullptr; nl->d_key_start = nullptr;
  nl->d_key_cursor = nullptr; nl->d_sorted = nullptr; nl->d_offset = nullptr;
  nl->d_xbuild = nullptr; nl->d_xhi = nullptr; nl->d_xlo = nullptr;
  nl->d_xw = nullptr; nl->d_nbr = nullptr; nl->d_nbr_count = nullptr;
  nl->d_maxdisp = nullptr; nl->d_rebuild = nullptr; nl->d_mol_s = nullptr;
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
                                     nl->d_sorted, s->d_charge, s->d_type, s->d_mol,
                                     nl->d_xhi, nl->d_xlo, nl->d_xw, nl->d_mol_s,
                                     nl->d_maxdisp);
  else
    k_gather<false><<<nb, T, 0, st>>>(n, s->d_pos, nl->d_offset, nl->d_xbuild,
                                      nl->d_sorted, s->d_charge, s->d_type, s->d_mol,
                                      nl->d_xhi, nl->d_xlo, nl->d_xw, nl->d_mol_s,
                                      nl->d_maxdisp);
  BuildArgs ba;
  ba.box = s->box;
  ba.n = n;
  ba.ncx = nl->ncx; ba.ncy = nl->ncy; ba.ncz = nl->ncz;
  // FP32 candidate test with a margin well above its rounding error
  const double r1 = nl->reach + 0.01, r2 = nl->reach + 0.05;
  ba.reach2 = (float)(r1 * r1);
  ba.cull2 = (float)(r2 * r2);
  for (int c = 0; c < 3; c++) {
    ba.cell_lo[c] = (float)(s->box.periodic ? s->box.min[c] - s->box.origin[c]
                                            : nl->vac_origin[c]);
    ba.cs[c] = (float)nl->cs[c];
    ba.L[c] = (float)s->box.e[c];
    ba.H2[c] = (float)s->box.H2[c];
  }
  ba.inv_layer = (float)(kFine / nl->cs[2]);
  ba.nlayers = nl->ncz * kFine;
  ba.cap = nl->cap;
  ba.periodic = s->box.periodic;
  ba.excl_start = s->d_excl_start;
  ba.excl_partner = s->d_excl_partner;
  ba.excl_class = s->d_excl_class;
  k_build_list<<<(n + kBuildWarps - 1) / kBuildWarps, kBuildWarps * 32, 0, st>>>(
      ba, nl->d_rebuild, nl->d_key, nl->d_sorted, nl->d_key_start, nl->d_xhi, nl->d_mol_s,
      nl->d_nbr, nl->d_nbr_count, s->d_status);
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
  a.lj_sw64 = make_switch_dev<double>(t.lj_sw);
  a.coul_sw64 = make_switch_dev<double>(t.coul_sw);
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
  a.max_lo = (Real)(mx * (1 - band));
  a.minimal_image = t.minimal_image;
  for (int c = 0; c < 3; c++) a.half_edge[c] = (Real)s->box.H2[c];
  a.same_cut = 1;
  if ((t.mask & TERM_LJ) && t.lj_cut2 != mx) a.same_cut = 0;
  if ((t.mask & TERM_COUL) && t.coul_cut2 != mx) a.same_cut = 0;
  if ((t.mask & TERM_EWALD) && t.ewald_rc2 != mx) a.same_cut = 0;
  a.alpha = (Real)t.ewald_alpha;
  a.a2pi = (Real)(2.0 * t.ewald_alpha / std::sqrt(M_PI));
  a.alpha64 = t.ewald_alpha;
  a.a2pi64 = 2.0 * t.ewald_alpha / std::sqrt(M_PI);
  a.exact_erf = t.exact_erf;
  a.csf = (Real)t.coulomb_scaling;
  a.csf64 = t.coulomb_scaling;
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
  a.count_pairs = s->count_pairs;
}

// Compile-time switch kind of a term for the specialised force-only
// kernel: -2 when the configuration has no specialisation.
static int spec_kind(const SwitchParams &sw) {
  if (!sw.modify) return kSwNone;
  if (sw.kind == PMGPU_SW_C2 || sw.kind == PMGPU_SW_C1) return sw.kind;
  return -2;
}

// Blocks of the pair kernel: one warp per atom, except the force-only FP32
// kernel of the inner MD steps, whose grid is capped at three blocks per SM
// (warps stride over the atoms) so that the PME / bonded chain on the
// system's second stream always finds room beside it.
static int pair_blocks(int n, bool persistent) {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        sms <= 0)
      sms = 148;
  }
  const int nb = (n + kPairWarps - 1) / kPairWarps;
  return persistent ? std::max(1, std::min(nb, 3 * sms)) : nb;
}

template <typename Real, int TERMS, typename SPEC>
static void launch_pairs_spec(PairArgs<Real> &a, cudaStream_t st, int mode) {
  const int T = kPairWarps * 32;
  switch (mode) {
    case PAIR_FORCE:
      k_pairs<Real, TERMS, PAIR_FORCE, SPEC><<<pair_blocks(a.n, sizeof(Real) == 4), T, 0, st>>>(a);
      break;
    case PAIR_ENERGY:
      k_pairs<Real, TERMS, PAIR_ENERGY, SPEC><<<pair_blocks(a.n, false), T, 0, st>>>(a);
      break;
    case PAIR_VIRIAL:
      k_pairs<Real, TERMS, PAIR_VIRIAL, SPEC><<<pair_blocks(a.n, false), T, 0, st>>>(a);
      break;
    default:
      k_pairs<Real, TERMS, PAIR_RECORD, SPEC><<<pair_blocks(a.n, false), T, 0, st>>>(a);
      break;
  }
}

template <typename Real, int TERMS, typename SPEC>
static void launch_force_spec(PairArgs<Real> &a, cudaStream_t st) {
  k_pairs<Real, TERMS, PAIR_FORCE, SPEC><<<pair_blocks(a.n, true), kPairWarps * 32, 0, st>>>(a);
}

template <typename Real, int TERMS>
static void launch_pairs_t(PairArgs<Real> &a, cudaStream_t st, int mode, const PairTerms &t) {
  // specialised force-only FP32 kernels of the common configurations
  if (sizeof(Real) == 4 && mode == PAIR_FORCE) {
    const int lk = spec_kind(t.lj_sw), ck = spec_kind(t.coul_sw);
    if (TERMS == (TERM_LJ | TERM_EWALD) && !t.exact_erf && lk == PMGPU_SW_C2) {
      launch_force_spec<Real, TERM_LJ | TERM_EWALD, PairSpec<PMGPU_SW_C2, -1, 0>>(a, st);
      return;
    }
    if (TERMS == (TERM_LJ | TERM_COUL) && lk == PMGPU_SW_C2 && ck == PMGPU_SW_C2) {
      launch_force_spec<Real, TERM_LJ | TERM_COUL, PairSpec<PMGPU_SW_C2, PMGPU_SW_C2, -1>>(a, st);
      return;
    }
    if (TERMS == (TERM_LJ | TERM_COUL) && lk == PMGPU_SW_C2 && ck == PMGPU_SW_C1) {
      launch_force_spec<Real, TERM_LJ | TERM_COUL, PairSpec<PMGPU_SW_C2, PMGPU_SW_C1, -1>>(a, st);
      return;
    }
  }
  launch_pairs_spec<Real, TERMS, GenericSpec>(a, st, mode);
}

template <typename Real>
static int launch_pairs(PairArgs<Real> &a, cudaStream_t st, int mode, const PairTerms &t) {
  switch (a.mask) {
    case TERM_LJ: launch_pairs_t<Real, TERM_LJ>(a, st, mode, t); break;
    case TERM_COUL: launch_pairs_t<Real, TERM_COUL>(a, st, mode, t); break;
    case TERM_LJ | TERM_COUL: launch_pairs_t<Real, TERM_LJ | TERM_COUL>(a, st, mode, t); break;
    case TERM_EWALD: launch_pairs_t<Real, TERM_EWALD>(a, st, mode, t); break;
    case TERM_LJ | TERM_EWALD: launch_pairs_t<Real, TERM_LJ | TERM_EWALD>(a, st, mode, t); break;
    default:
      return fail(PMGPU_ERR_UNSUPPORTED, "unsupported pair-term combination");
  }
  PM_CUDA(cudaGetLastError());
  return PMGPU_OK;
}

// mode: PAIR_FORCE (forces only), PAIR_ENERGY (+ FP64 energies),
// PAIR_VIRIAL (+ virial), PAIR_RECORD (+ pair-set recording).
int nb_pair_forces(System *s, NeighborList *nl, const PairTerms &t, int mode) {
  if (s->n == 0) return PMGPU_OK;
  if (s->precision == PMGPU_PREC_MIXED) {
    PairArgs<float> a;
    fill_pair_args<float>(a, s, nl, t);
    return launch_pairs<float>(a, s->stream, mode, t);
  }
  PairArgs<double> a;
  fill_pair_args<double>(a, s, nl, t);
  return launch_pairs<double>(a, s->stream, mode, t);
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
    if (n) {
      PM_CUDA(cudaMemcpyAsync(h.data(), s->d_pos, sizeof(double) * 3 * n,
                              cudaMemcpyDeviceToHost, s->stream));
      PM_CUDA(cudaStreamSynchronize(s->stream));
    }
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
  PM_CHECK(dev_alloc(s, &dout, sizeof(int) * 3 * std::max(n, 1)));
  if (n) k_cells_debug<<<(n + 255) / 256, 256, 0, s->stream>>>(g, s->d_pos, dout);
  cudaError_t e = cudaMemcpyAsync(cell_xyz, dout, sizeof(int) * 3 * n,
                                  cudaMemcpyDeviceToHost, s->stream);
  dev_free(s, dout);
  cudaError_t e2 = cudaStreamSynchronize(s->stream);
  if (e != cudaSuccess || e2 != cudaSuccess)
    return fail(PMGPU_ERR_CUDA, "debug cell assignment failed");
  dims[0] = d[0]; dims[1] = d[1]; dims[2] = d[2];
  return PMGPU_OK;
}

// --------------------------------------------------- NonbondedSimpleFull
// Vacuum all pairs with exclusions (NonbondedSimpleFullSystemForce.h:125-150
// with OneAtomPair<Vacuum, Universal, LennardJones|Coulomb>): a 2-D grid of
// (128 i atoms) x (a chunk of j) blocks, j tiles staged in shared memory;
// every i sees every j != i (forces for i only), energies halved.  The
// exclusion table is consulted only for j inside i's partner-index range.
constexpr int kSfTile = 128;

template <typename Real, bool LJ, bool COUL>
__global__ void __launch_bounds__(kSfTile)
k_simplefull(int n, int jchunk, const double *__restrict__ pos,
             const double *__restrict__ charge, const int *__restrict__ type, int ntypes,
             const float4 *__restrict__ lj32, const double4 *__restrict__ lj64,
             const int2 *__restrict__ ex_range, const int *__restrict__ ex_start,
             const int *__restrict__ ex_partner, const int *__restrict__ ex_class, Real csf,
             long long *__restrict__ force, long long *__restrict__ acc, int em) {
  __shared__ double sx[kSfTile], sy[kSfTile], sz[kSfTile], sq[kSfTile];
  __shared__ int st[kSfTile];
  const int i = blockIdx.x * kSfTile + threadIdx.x;
  const bool valid = i < n;
  const int ii = valid ? i : 0;
  const double xi = pos[3 * ii], yi = pos[3 * ii + 1], zi = pos[3 * ii + 2];
  const double qi = charge[ii];
  const int ti = type[ii];
  const int2 er = ex_range[ii];
  Real fx = 0, fy = 0, fz = 0;
  double elj = 0, ec = 0;
  double v[6] = {0, 0, 0, 0, 0, 0};
  const int j0 = blockIdx.y * jchunk, j1 = min(n, j0 + jchunk);
  for (int base = j0; base < j1; base += kSfTile) {
    const int j = base + threadIdx.x;
    if (j < j1) {
      sx[threadIdx.x] = pos[3 * j]; sy[threadIdx.x] = pos[3 * j + 1];
      sz[threadIdx.x] = pos[3 * j + 2]; sq[threadIdx.x] = charge[j];
      st[threadIdx.x] = type[j];
    }
    __syncthreads();
    const int lim = min(kSfTile, j1 - base);
    if (valid) {
      for (int k = 0; k < lim; k++) {
        const int jj = base + k;
        if (jj == i) continue;
        int excl = PMGPU_EXCL_NONE;
        if (jj >= er.x && jj <= er.y) {
          excl = excl_class_of(ex_start, ex_partner, ex_class, i, jj);
          if (excl == PMGPU_EXCL_FULL) continue;
        }
        const Real dx = (Real)(sx[k] - xi), dy = (Real)(sy[k] - yi), dz = (Real)(sz[k] - zi);
        const Real r2 = dx * dx + dy * dy + dz * dz;
        const Real rr2 = Real(1) / r2;
        Real f = 0;
        if (LJ) {
          Real A, B;
          if (sizeof(Real) == 4) {
            const float4 p = __ldg(&lj32[ti * ntypes + st[k]]);
            A = excl == PMGPU_EXCL_MODIFIED ? p.z : p.x;
            B = excl == PMGPU_EXCL_MODIFIED ? p.w : p.y;
          } else {
            const double4 p = lj64[ti * ntypes + st[k]];
            A = excl == PMGPU_EXCL_MODIFIED ? p.z : p.x;
            B = excl == PMGPU_EXCL_MODIFIED ? p.w : p.y;
          }
          const Real r6 = rr2 * rr2 * rr2;
          const Real r6B = B * r6, r12A = A * r6 * r6;
          if (em) elj += (double)(r12A - r6B);
          f += (Real(12) * r12A - Real(6) * r6B) * rr2;
        }
        if (COUL) {
          Real en = (Real)(qi * sq[k]) * pm_sqrt(rr2);
          if (excl == PMGPU_EXCL_MODIFIED) en *= csf;
          if (em) ec += (double)en;
          f += en * rr2;
        }
        fx -= dx * f; fy -= dy * f; fz -= dz * f;
        if (em == 2) {
          const double hf = 0.5 * (double)f;
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
  if (!em) return;
  elj = warp_sum(elj) * 0.5;
  ec = warp_sum(ec) * 0.5;
  if (em == 2)
    for (int q = 0; q < 6; q++) v[q] = warp_sum(v[q]);
  if ((threadIdx.x & 31) == 0) {
    if (LJ) red_add(&acc[ACC_LJ], to_fixed(elj, kEnergyScale));
    if (COUL) red_add(&acc[ACC_COULOMB], to_fixed(ec, kEnergyScale));
    if (em == 2) {
      const int map[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
      for (int q = 0; q < 9; q++) red_add(&acc[ACC_VIRIAL + q], to_fixed(v[map[q]], kEnergyScale));
    }
  }
}

// em: 0 forces only, 1 + energies, 2 + energies and virial.
int nb_simplefull(System *s, int lj, int coul, int em) {
  const int n = s->n;
  if (n == 0 || !(lj || coul)) return PMGPU_OK;
  // enough j chunks for ~2 blocks per SM
  const int iblocks = (n + kSfTile - 1) / kSfTile;
  int chunks = std::max(1, std::min((296 + iblocks - 1) / iblocks, iblocks));
  const int jchunk = ((n + chunks - 1) / chunks + kSfTile - 1) / kSfTile * kSfTile;
  chunks = (n + jchunk - 1) / jchunk;
  const dim3 grid(iblocks, chunks);
  auto go = [&](auto kern, auto csf) {
    kern<<<grid, kSfTile, 0, s->stream>>>(n, jchunk, s->d_pos, s->d_charge, s->d_type,
                                          s->ntypes, s->d_lj32, s->d_lj64, s->d_excl_range,
                                          s->d_excl_start, s->d_excl_partner, s->d_excl_class,
                                          csf, s->d_force, s->d_acc, em);
  };
  if (s->precision == PMGPU_PREC_MIXED) {
    const float csf = (float)s->coulomb_scaling;
    if (lj && coul) go(k_simplefull<float, true, true>, csf);
    else if (lj) go(k_simplefull<float, true, false>, csf);
    else go(k_simplefull<float, false, true>, csf);
  } else {
    const double csf = s->coulomb_scaling;
    if (lj && coul) go(k_simplefull<double, true, true>, csf);
    else if (lj) go(k_simplefull<double, true, false>, csf);
    else go(k_simplefull<double, false, true>, csf);
  }
  PM_CUDA(cudaGetLastError());
  return PMGPU_OK;
}

}  // namespace pmgpu
