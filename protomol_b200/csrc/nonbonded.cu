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
#include <cstdlib>

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

// ------------------------------------------------------ list sort grid
// The cluster-pair list sorts atoms into ncx x ncy columns of the xy plane
// and, within a column, by z (ties by atom index, so the order is
// deterministic).  Eight consecutive atoms of a column then form a compact
// cluster of about kColumnWidth on each side.
struct ListGrid {
  Box box;
  int n, periodic;
  int ncx, ncy, nzb;
  double lo[3];    // grid corner in the wrapped frame
  double inv[3];   // 1 / column width (x, y), 1 / z-bin height
};

// Column layout of a rebuild, by one block once every atom is binned: the
// padded column bases (every column a whole number of 8-atom clusters; a
// column past its bucket counts as a full bucket, and the sort flags it) and
// the slots past the padded total marked empty.
struct ScanArgs {
  int ncol, nkeys, ns_max, bcap;
  int *col_base, *key_start, *sorted;
};

struct BinArgs {
  ListGrid g;
  const double *pos;
  const int *rebuild;
  unsigned *zkey;
  int *col_count, *bucket;
  double *offset, *xbuild;
  int *status;
  unsigned *ticket;  // binning blocks done: the last one lays out the columns
  ScanArgs scan;
};

// Exclusive scan of value(k), k < count, by one block; write(k, prefix)
// receives each prefix and the return value is the total.
template <typename V, typename W>
__device__ int block_scan(int count, V value, W write, int *warp_tot, int *carry) {
  if (threadIdx.x == 0) *carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int base = 0; base < count; base += blockDim.x) {
    const int i = base + threadIdx.x;
    const int v = i < count ? value(i) : 0;
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) warp_tot[wid] = incl;
    __syncthreads();
    if (wid == 0) {
      const int t = lane < nw ? warp_tot[lane] : 0;
      int ti = t;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, ti, o);
        if (lane >= o) ti += u;
      }
      if (lane < nw) warp_tot[lane] = ti - t;
    }
    __syncthreads();
    const int excl = *carry + warp_tot[wid] + incl - v;
    if (i < count) write(i, excl);
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) *carry = excl + v;
    __syncthreads();
  }
  return *carry;
}

__device__ void scan_columns(const ScanArgs &A, const int *col_count) {
  __shared__ int warp_tot[32];
  __shared__ int carry;
  const int bcap = A.bcap;
  int *col_base = A.col_base;
  // the counts come from other blocks' atomics: read them from L2
  const int padded = block_scan(
      A.ncol, [&](int c) { return (min(__ldcg(col_count + c), bcap) + 7) & ~7; },
      [&](int c, int p) { col_base[c] = p; }, warp_tot, &carry);
  if (threadIdx.x == 0) {
    col_base[A.ncol] = padded;
    A.key_start[A.nkeys] = padded;
  }
  for (int s = padded + threadIdx.x; s < A.ns_max; s += blockDim.x) A.sorted[s] = -1;
}

// Rebuild steps: each atom's column (its xy cell of the wrapped position),
// z key and image offset, the atom placed in its column's bucket; the last
// block to finish lays out the columns (scan_columns).
__device__ __forceinline__ void bin_body(const BinArgs &A, Blk b) {
  if (!*A.rebuild) return;
  const ListGrid &g = A.g;
  const double *__restrict__ pos = A.pos;
  const int bcap = A.scan.bcap;
  const int i = b.x * blockDim.x + threadIdx.x;
  const bool valid = i < g.n;
  const unsigned vmask = __ballot_sync(0xffffffffu, valid);
  if (valid) {
    const double x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
    double w[3];
    box_minpos(g.box, x, y, z, w[0], w[1], w[2]);
    const int dims[2] = {g.ncx, g.ncy};
    int c[2];
    const bool finite = isfinite(x) && isfinite(y) && isfinite(z);
    for (int a = 0; a < 2; a++) {
      const double q = finite ? (w[a] - g.lo[a]) * g.inv[a] : 0.0;
      int k = (int)floor(fmin(fmax(q, -1.0), (double)dims[a]));
      c[a] = k < 0 ? 0 : (k >= dims[a] ? dims[a] - 1 : k);
    }
    if (!finite) atomicOr(A.status, ST_NONFINITE);
    const int col = c[0] * g.ncy + c[1];
    // non-negative FP32 bits order like the values
    const float zf = finite ? (float)fmin(fmax(w[2] - g.lo[2], 0.0), 1.0e30) : 0.f;
    A.zkey[i] = __float_as_uint(zf);
    // one atomic per column among the warp's atoms (neighbouring atoms of a
    // molecule share columns); the count it returns places each atom in its
    // column's bucket (the order inside a column is sorted afterwards)
    const unsigned peers = __match_any_sync(vmask, col);
    const int lane = threadIdx.x & 31, leader = __ffs(peers) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(&A.col_count[col], __popc(peers));
    base = __shfl_sync(peers, base, leader);
    const int r = base + __popc(peers & ((1u << lane) - 1u));
    if (r < bcap) A.bucket[(size_t)col * bcap + r] = i;
    A.offset[3 * i] = x - w[0];
    A.offset[3 * i + 1] = y - w[1];
    A.offset[3 * i + 2] = z - w[2];
    A.xbuild[3 * i] = x;
    A.xbuild[3 * i + 1] = y;
    A.xbuild[3 * i + 2] = z;
  }
  __shared__ int last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();  // this block's counts before its ticket
    last = atomicAdd(A.ticket, 1u) == (unsigned)(b.n - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  scan_columns(A.scan, A.col_count);
  if (threadIdx.x == 0) *A.ticket = 0u;  // ready for the next build
}
__global__ void k_bin(BinArgs a) {
  pdl_wait();  // the predecessor's writes are visible from here on
  pdl_trigger();
  bin_body(a, own_blk());
}
__global__ void k_bin_batch(const BinArgs *__restrict__ tab, const int *__restrict__ first,
                            int nm) {
  const int m = batch_member(first, nm, blockIdx.x);
  bin_body(tab[m], batch_blk(first, m));
}

// Slot records of the sorted coordinates: xw = x - offset keeps every atom
// in the image it had at the last build, so tile images stay valid.
// Padding slots get far-away positions and no charge; no tile pairs them.
struct GatherArgs {
  int ns;
  const double *pos, *offset;
  const int *sorted;
  const double *charge;
  const int *type, *mol;
  float4 *xhi, *xlo;
  double4 *xw;
  int *mol_s;
  const int *rebuild;
  float4 *bb;
};

// Slot s's records for atom i (i < 0: padding): the FP64 wrapped position
// and charge, the FP32 high part with the charge and, in mixed precision,
// the FP32 residue with the type bits.  (hx, hy, hz) gets the FP32
// position of an atom.
__device__ __forceinline__ void write_slot(const GatherArgs &A, bool mixed, int s, int i,
                                           float &hx, float &hy, float &hz) {
  if (i < 0) {
    const double far = 1.0e5 + 16.0 * s;
    A.xw[s] = make_double4(far, 1.0e5, 1.0e5, 0.0);
    A.xhi[s] = make_float4((float)far, 1.0e5f, 1.0e5f, 0.f);
    if (mixed) A.xlo[s] = make_float4(0.f, 0.f, 0.f, __int_as_float(0));
    A.mol_s[s] = -1;
    return;
  }
  const double x = A.pos[3 * i], y = A.pos[3 * i + 1], z = A.pos[3 * i + 2];
  const double wx = x - A.offset[3 * i], wy = y - A.offset[3 * i + 1],
               wz = z - A.offset[3 * i + 2];
  const double q = A.charge[i];
  A.xw[s] = make_double4(wx, wy, wz, q);
  hx = (float)wx;
  hy = (float)wy;
  hz = (float)wz;
  A.xhi[s] = make_float4(hx, hy, hz, (float)q);
  if (mixed)
    A.xlo[s] = make_float4((float)(wx - (double)hx), (float)(wy - (double)hy),
                           (float)(wz - (double)hz), __int_as_float(A.type[i]));
  A.mol_s[s] = A.mol[i];
}

// The box of the 4-atom cluster of slots s..s+3 (4 consecutive lanes, the
// whole warp taking part): lower corner with the number of atoms in .w,
// upper corner.
__device__ __forceinline__ void write_cluster_box(float4 *bb, int s, bool in, bool atom,
                                                  float hx, float hy, float hz) {
  float lo[3] = {atom ? hx : 3.0e38f, atom ? hy : 3.0e38f, atom ? hz : 3.0e38f};
  float hi[3] = {atom ? hx : -3.0e38f, atom ? hy : -3.0e38f, atom ? hz : -3.0e38f};
  int m = atom ? 1 : 0;
#pragma unroll
  for (int o = 1; o < 4; o <<= 1) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      lo[c] = fminf(lo[c], __shfl_xor_sync(0xffffffffu, lo[c], o));
      hi[c] = fmaxf(hi[c], __shfl_xor_sync(0xffffffffu, hi[c], o));
    }
    m += __shfl_xor_sync(0xffffffffu, m, o);
  }
  if (in && (s & 3) == 0) {
    bb[2 * (s >> 2)] = make_float4(lo[0], lo[1], lo[2], (float)m);
    bb[2 * (s >> 2) + 1] = make_float4(hi[0], hi[1], hi[2], 0.f);
  }
}

// One block per column: bitonic sort of (z, atom) in shared memory, the
// column's padded slots written in that order, and the column's z-bin
// index (first slot of every bin).  A column above kColCap atoms flags
// ST_CELL_OVERFLOW and is left empty; one above its bucket (but within
// kColCap) flags ST_LIST_OVERFLOW with its count, for the host to grow the
// buckets and repeat the work.  With gather set (the rebuild of an MD step,
// whose update kernel writes the slot records on the other steps) the block
// also writes its slots' records and cluster boxes, and the blocks share
// the empty slots past the last column.
constexpr int kSortThreads = 256;
struct SortArgs {
  const int *rebuild;
  int nzb, ncol, bcap;
  float inv_z;
  int *col_count;
  const int *col_base, *bucket;
  const unsigned *zkey;
  int *sorted, *slot_of, *key_start, *status;
  int *need;  // largest column count past the bucket size
  int gather, mixed;
  GatherArgs g;
};
__device__ __forceinline__ void sort_body(const SortArgs &A, Blk b) {
  const int nzb = A.nzb, bcap = A.bcap;
  const float inv_z = A.inv_z;
  int *__restrict__ col_count = A.col_count;
  const int *__restrict__ col_base = A.col_base;
  const unsigned *__restrict__ zkey = A.zkey;
  int *__restrict__ sorted = A.sorted;
  int *__restrict__ slot_of = A.slot_of;
  int *__restrict__ key_start = A.key_start;
  if (!*A.rebuild) return;
  __shared__ unsigned long long keys[kColCap];
  const int col = b.x;
  int m = col_count[col];
  const int base = col_base[col], pend = col_base[col + 1];
  if (m > kColCap) {
    if (threadIdx.x == 0) atomicOr(A.status, ST_CELL_OVERFLOW);
    m = 0;
  } else if (m > bcap) {
    if (threadIdx.x == 0) {
      atomicOr(A.status, ST_LIST_OVERFLOW);
      atomicMax(A.need, m);
    }
    m = bcap;
  }
  int P = 1;
  while (P < m) P <<= 1;
  const int *__restrict__ bucket = A.bucket + (size_t)col * bcap;
  for (int k = threadIdx.x; k < P; k += kSortThreads) {
    if (k < m) {
      const int i = bucket[k];
      keys[k] = ((unsigned long long)zkey[i] << 32) | (unsigned)i;
    } else {
      keys[k] = ~0ull;
    }
  }
  __syncthreads();
  for (int size = 2; size <= P; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int k = threadIdx.x; k < P; k += kSortThreads) {
        const int l = k ^ stride;
        if (l > k) {
          const unsigned long long x = keys[k], y = keys[l];
          const bool up = (k & size) == 0;
          if ((x > y) == up) {
            keys[k] = y;
            keys[l] = x;
          }
        }
      }
      __syncthreads();
    }
  }
  auto bin_of = [&](int k) {
    const float zf = __uint_as_float((unsigned)(keys[k] >> 32));
    const int q = (int)(zf * inv_z);
    return q < 0 ? 0 : (q >= nzb ? nzb - 1 : q);
  };
  int *ks = key_start + (size_t)col * nzb;
  // the column's slots (a whole number of clusters: warps stay uniform)
  const int len = pend - base;
  for (int k0 = 0; k0 < len; k0 += kSortThreads) {
    const int k = k0 + threadIdx.x;
    const bool in = k < len;
    const int atom = in && k < m ? (int)(keys[k] & 0xffffffffu) : -1;
    if (in) {
      sorted[base + k] = atom;
      if (atom >= 0) slot_of[atom] = base + k;
    }
    if (A.gather) {
      float hx = 0.f, hy = 0.f, hz = 0.f;
      if (in) write_slot(A.g, A.mixed, base + k, atom, hx, hy, hz);
      write_cluster_box(A.g.bb, base + k, in, atom >= 0, hx, hy, hz);
    }
  }
  if (A.gather) {
    // the empty slots past the last column (the padded total is a multiple
    // of 8, so every cluster lies within one warp's lanes)
    const int ns = A.g.ns;
    for (int s0 = col_base[A.ncol] + b.x * kSortThreads; s0 < ns; s0 += b.n * kSortThreads) {
      const int s = s0 + threadIdx.x;
      const bool in = s < ns;
      float hx = 0.f, hy = 0.f, hz = 0.f;
      if (in) write_slot(A.g, A.mixed, s, -1, hx, hy, hz);
      write_cluster_box(A.g.bb, s, in, false, hx, hy, hz);
    }
  }
  for (int k = threadIdx.x; k < m; k += kSortThreads) {
    const int q = bin_of(k), prev = k ? bin_of(k - 1) : -1;
    for (int z = prev + 1; z <= q; z++) ks[z] = base + k;
  }
  const int last = m ? bin_of(m - 1) : -1;
  for (int z = last + 1 + threadIdx.x; z < nzb; z += kSortThreads) ks[z] = base + m;
  __syncthreads();
  if (threadIdx.x == 0) col_count[col] = 0;  // ready for the next build
}
__global__ void __launch_bounds__(kSortThreads) k_sort_cols(SortArgs a) {
  pdl_wait();  // the predecessor's writes are visible from here on
  pdl_trigger();
  sort_body(a, own_blk());
}
__global__ void __launch_bounds__(kSortThreads)
k_sort_cols_batch(const SortArgs *__restrict__ tab, const int *__restrict__ first, int nm) {
  const int m = batch_member(first, nm, blockIdx.x);
  sort_body(tab[m], batch_blk(first, m));
}

// The slot records of every slot (evaluations outside MD steps, and the
// members of an ensemble); the cluster boxes on a rebuild.
template <bool MIXED>
__device__ __forceinline__ void gather_slots_body(const GatherArgs &A, Blk b) {
  const int s = b.x * blockDim.x + threadIdx.x;
  const bool in = s < A.ns;
  const int i = in ? A.sorted[s] : -1;
  float hx = 0.f, hy = 0.f, hz = 0.f;
  if (in) write_slot(A, MIXED, s, i, hx, hy, hz);
  if (*A.rebuild) write_cluster_box(A.bb, s, in, in && i >= 0, hx, hy, hz);
}
template <bool MIXED>
__global__ void k_gather(GatherArgs a) {
  pdl_wait();  // the predecessor's writes are visible from here on
  pdl_trigger();
  gather_slots_body<MIXED>(a, own_blk());
}
template <bool MIXED>
__global__ void k_gather_batch(const GatherArgs *__restrict__ tab, const int *__restrict__ first,
                               int nm) {
  const int m = batch_member(first, nm, blockIdx.x);
  gather_slots_body<MIXED>(tab[m], batch_blk(first, m));
}

// Decides whether this evaluation rebuilds the list (rebuild_decide) from
// the current positions: first build, forced, or an atom lies more than
// half the skin from its position at the last build (so no pair can have
// come from beyond the reach to within the cutoff).  MD steps take the
// decision in the update kernel instead (k_update).
constexpr int kCheckThreads = 256;
__global__ void __launch_bounds__(kCheckThreads)
k_check_rebuild(int n, const double *__restrict__ pos, const double *__restrict__ xbuild,
                unsigned *__restrict__ ticket, int *__restrict__ rebuild, float half_skin2,
                int force) {
  pdl_wait();  // the predecessor's writes are visible from here on
  pdl_trigger();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  float d2 = 0.f;
  if (i < n && !force) {
    const double dx = pos[3 * i] - xbuild[3 * i], dy = pos[3 * i + 1] - xbuild[3 * i + 1],
                 dz = pos[3 * i + 2] - xbuild[3 * i + 2];
    d2 = (float)(dx * dx + dy * dy + dz * dz);
  }
  rebuild_decide<kCheckThreads>(d2, ticket, rebuild, half_skin2, force, (int)gridDim.x);
}

// ---------------------------------------------------------- list build
struct TileBuildArgs {
  int nclusters;     // 8-atom i clusters (kRowParts tile rows each)
  int periodic;
  int ncx, ncy, nzb;
  float lo[3];       // grid corner in the wrapped frame
  float cs[3];       // column widths (x, y), z-bin height
  float L[3];        // box edges
  float H2[3];       // half box edges (minimal-image test)
  float reach2;      // FP32 pair test radius^2 (reach plus a rounding margin)
  float cull;        // cluster / column culling radius (wider margin)
  int cap;           // tiles per row in the buffer (the row stride)
  int limit;         // tiles a row may hold (cap, or a lower test limit)
  const int *excl_start, *excl_partner, *excl_class;
};

__device__ __forceinline__ int excl_class_of(const int *start, const int *partner,
                                             const int *cls, int oi, int oj) {
  int b = start[oi], e = start[oi + 1];
  for (int k = b; k < e; k++)
    if (partner[k] == oj) return cls[k];
  return PMGPU_EXCL_NONE;
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }


// One warp per (8-atom i cluster, row part).  The search window of the
// i cluster is the set of (column, periodic image, z slice) ranges whose
// box lies within the culling radius of the i cluster's box; the 32 lanes
// form 32 of those ranges at a time, and the non-empty ones are dealt
// round-robin over the kRowParts warps of the cluster.  In a range, a
// 4-atom j cluster is a candidate if its box (in that image) lies within
// the radius.  Each unordered pair is listed once: j clusters of a later i
// cluster are taken in every image, those of the same i cluster in the
// zero image (pairs with the i atom before the j atom) and in one half of
// the other images.  Candidates are tested four at a time: lane
// (i atom l & 7, candidate l >> 3) tests its i atom against the
// candidate's 4 j atoms, pairs beyond the reach or with padding are masked
// off, and ExclusionTable::check (topology/ExclusionTable.h:116-130;
// consulted for same-molecule minimal-image pairs as in
// OneAtomPairTwo.h:47-53) clears fully excluded pairs and marks modified
// ones.  Tiles are appended in a fixed order (range, cluster index), so
// the list is deterministic.
struct BuildArgs {
  TileBuildArgs a;
  int *rebuild;
  const int *sorted, *start;
  const float4 *xhi;
  const int *mol_s;
  const float4 *bb;
  uint2 *tiles;
  unsigned *tmod;
  int *tile_count;
  uint2 *jlanes;
  int *jl_count;
  int *status;
  int *work;  // [0] next row, [1] warps done (both back to zero at the end)
};
__device__ __forceinline__ void build_body(const BuildArgs &B, Blk blk) {
  const TileBuildArgs &a = B.a;
  int *__restrict__ rebuild = B.rebuild;
  const int *__restrict__ sorted = B.sorted;
  const int *__restrict__ start = B.start;
  const float4 *__restrict__ xhi = B.xhi;
  const int *__restrict__ mol_s = B.mol_s;
  const float4 *__restrict__ bb = B.bb;
  uint2 *__restrict__ tiles = B.tiles;
  unsigned *__restrict__ tmod = B.tmod;
  int *__restrict__ tile_count = B.tile_count;
  uint2 *__restrict__ jlanes = B.jlanes;
  int *__restrict__ jl_count = B.jl_count;
  int *__restrict__ status = B.status;
  if (!*rebuild) return;
  constexpr unsigned kAll = 0xffffffffu;
  // this warp's staging of candidate j clusters (up to 32 of them)
  __shared__ float4 st_x[kBuildWarps][128];
  __shared__ int4 st_o[kBuildWarps][32], st_m[kBuildWarps][32];
  __shared__ int st_h[kBuildWarps][32], st_c[kBuildWarps][32];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  // the warps of the (resident) grid take the rows one at a time from a
  // counter, so the rows' unequal costs spread over the SMs; the output
  // of a row does not depend on which warp builds it
  int *const work = B.work;
  auto next_row = [&]() {
    int r = 0;
    if (lane == 0) r = atomicAdd(&work[0], 1);
    return __shfl_sync(kAll, r, 0);
  };
  for (int rw = next_row(); rw < a.nclusters * kRowParts; rw = next_row()) {
  const int ci = rw / kRowParts, part = rw - ci * kRowParts;
  const float4 l0 = bb[4 * ci], h0 = bb[4 * ci + 1], l1 = bb[4 * ci + 2], h1 = bb[4 * ci + 3];
  if (l0.w + l1.w == 0.f) {
    if (lane == 0) tile_count[rw] = jl_count[rw] = 0;
    continue;
  }
  float ilo[3] = {fminf(l0.x, l1.x), fminf(l0.y, l1.y), fminf(l0.z, l1.z)};
  float ihi[3] = {fmaxf(h0.x, h1.x), fmaxf(h0.y, h1.y), fmaxf(h0.z, h1.z)};
  // non-finite coordinates (already flagged by the binning), or periodic
  // coordinates outside the box: no tiles, no unbounded window
  bool sane = true;
  for (int c = 0; c < 3; c++) {
    const float span = (c < 2 ? (c ? a.ncy : a.ncx) : a.nzb) * a.cs[c];
    sane = sane && isfinite(ilo[c]) && isfinite(ihi[c]) &&
           (!a.periodic || (fabsf(ilo[c] - a.lo[c]) < 2.f * span &&
                            fabsf(ihi[c] - a.lo[c]) < 2.f * span));
  }
  if (!sane) {
    if (lane == 0) {
      tile_count[rw] = jl_count[rw] = 0;
      atomicOr(status, ST_NONFINITE);
    }
    continue;
  }
  const int il = lane & 7, cq = lane >> 3;
  const int islot = 8 * ci + il;
  const int oi = sorted[islot];
  const bool ilive = oi >= 0;
  const float4 pi = xhi[islot];
  const int mi = mol_s[islot];
  const float R = a.cull, R2 = a.cull * a.cull;
  uint2 *row = tiles + (size_t)rw * a.cap;
  unsigned *rowmod = tmod + (size_t)rw * a.cap;
  int count = 0;

  // the candidate test of up to four staged j clusters (lane (il, cq)
  // tests its i atom against the 4 atoms of staged candidate bq[cq])
  auto test4 = [&](const int (&bq)[4], int ng) {
    const int myb = cq == 0 ? bq[0] : (cq == 1 ? bq[1] : (cq == 2 ? bq[2] : bq[3]));
    const bool cval = cq < ng;
    const int hj = st_h[wib][myb], code = st_c[wib][myb];
    const int sx = (code & 3) - 1, sy = ((code >> 2) & 3) - 1, sz = ((code >> 4) & 3) - 1;
    const float S[3] = {sx * a.L[0], sy * a.L[1], sz * a.L[2]};
    const bool diag = code == kZeroShift && (hj >> 1) == ci;
    const int4 o4 = st_o[wib][myb], m4 = st_m[wib][myb];
    const int oj[4] = {o4.x, o4.y, o4.z, o4.w};
    const int mj[4] = {m4.x, m4.y, m4.z, m4.w};
    bool pass[4], same = false;
    float dd[4][3];
#pragma unroll
    for (int jl = 0; jl < 4; jl++) {
      const float4 pj = st_x[wib][4 * myb + jl];
      dd[jl][0] = pj.x + S[0] - pi.x;
      dd[jl][1] = pj.y + S[1] - pi.y;
      dd[jl][2] = pj.z + S[2] - pi.z;
      const float r2 = dd[jl][0] * dd[jl][0] + dd[jl][1] * dd[jl][1] + dd[jl][2] * dd[jl][2];
      pass[jl] = cval && ilive && oj[jl] >= 0 && r2 < a.reach2 && (!diag || islot < 4 * hj + jl);
      same = same || (pass[jl] && mj[jl] == mi);
    }
    unsigned mb[4] = {0u, 0u, 0u, 0u};
    // same-molecule pairs (few tiles): ExclusionTable lookup
    if (__any_sync(kAll, same)) {
#pragma unroll
      for (int jl = 0; jl < 4; jl++) {
        bool mod = false;
        if (pass[jl] && mj[jl] == mi) {
          const bool minimal = !a.periodic || (fabsf(dd[jl][0]) <= a.H2[0] &&
                                               fabsf(dd[jl][1]) <= a.H2[1] &&
                                               fabsf(dd[jl][2]) <= a.H2[2]);
          if (minimal) {
            const int cls = excl_class_of(a.excl_start, a.excl_partner, a.excl_class, oi, oj[jl]);
            if (cls == PMGPU_EXCL_FULL) pass[jl] = false;
            else if (cls == PMGPU_EXCL_MODIFIED) mod = true;
          }
        }
        mb[jl] = __ballot_sync(kAll, mod);
      }
    }
    unsigned pb[4];
#pragma unroll
    for (int jl = 0; jl < 4; jl++) pb[jl] = __ballot_sync(kAll, pass[jl]);
    // lane q < 4 assembles candidate q's masks (bit il + 8 jl) and writes it
    const int q = lane & 3, sh = 8 * q;
    const unsigned im = ((pb[0] >> sh) & 0xFFu) | (((pb[1] >> sh) & 0xFFu) << 8) |
                        (((pb[2] >> sh) & 0xFFu) << 16) | (((pb[3] >> sh) & 0xFFu) << 24);
    const unsigned mm = ((mb[0] >> sh) & 0xFFu) | (((mb[1] >> sh) & 0xFFu) << 8) |
                        (((mb[2] >> sh) & 0xFFu) << 16) | (((mb[3] >> sh) & 0xFFu) << 24);
    const bool wr = lane < ng && im != 0u;
    const unsigned wm = __ballot_sync(kAll, wr);
    if (wr) {
      const int idx = count + __popc(wm & ((1u << lane) - 1u));
      const int bsel = q == 0 ? bq[0] : (q == 1 ? bq[1] : (q == 2 ? bq[2] : bq[3]));
      if (idx < a.limit) {
        row[idx] = make_uint2((uint32_t)st_h[wib][bsel] |
                                  ((uint32_t)st_c[wib][bsel] << kShiftBits) |
                                  (mm ? kModFlag : 0u),
                              im);
        if (mm) rowmod[idx] = mm;
      }
    }
    count += __popc(wm);
  };

  const int ux0 = (int)floorf((ilo[0] - R - a.lo[0]) / a.cs[0]);
  const int ux1 = (int)floorf((ihi[0] + R - a.lo[0]) / a.cs[0]);
  const int uy0 = (int)floorf((ilo[1] - R - a.lo[1]) / a.cs[1]);
  const int uy1 = (int)floorf((ihi[1] + R - a.lo[1]) / a.cs[1]);
  const int b0 = (int)floorf((ilo[2] - R - a.lo[2]) / a.cs[2]);
  const int b1 = (int)floorf((ihi[2] + R - a.lo[2]) / a.cs[2]);
  // periodic: the box edge exceeds the culling radius, so the window spans
  // images -1, 0, 1 only; vacuum: atoms outside the grid sit in its edge
  // columns and bins, and clamping the window the same way keeps every
  // atom within the reach
  const int vx0 = a.periodic ? ux0 : clampi(ux0, 0, a.ncx - 1);
  const int vy0 = a.periodic ? uy0 : clampi(uy0, 0, a.ncy - 1);
  const int nux = (a.periodic ? ux1 : clampi(ux1, 0, a.ncx - 1)) - vx0 + 1;
  const int nuy = (a.periodic ? uy1 : clampi(uy1, 0, a.ncy - 1)) - vy0 + 1;
  const float inv_nuy = 1.0f / (float)nuy;
  const int total = nux * nuy;
  const int half0 = 8 * ci;  // j clusters of earlier i clusters are never taken
  int deal = 0;
  // Columns of the window, 32 at a time: lane k forms column k's z ranges
  // in images sz = -1, 0, 1 (clipped to the half list) as half-cluster
  // ranges [hs, hs + nh); the non-empty columns are dealt round-robin over
  // the row parts, and this part's ranges are concatenated into one index
  // space that the lanes scan 32 half clusters at a time.
  for (int k0 = 0; k0 < total; k0 += 32) {
    const int k = k0 + lane;
    int hs[3] = {0, 0, 0}, nh[3] = {0, 0, 0}, sxy = 0;
    if (k < total) {
      int ix = (int)(((float)k + 0.5f) * inv_nuy);
      ix = ix * nuy > k ? ix - 1 : (ix * nuy + nuy <= k ? ix + 1 : ix);
      const int iy = k - ix * nuy;
      int col, sx = 0, sy = 0;
      bool near = true;
      if (a.periodic) {
        const int ux = vx0 + ix, uy = vy0 + iy;
        sx = ux < 0 ? -1 : (ux >= a.ncx ? 1 : 0);
        sy = uy < 0 ? -1 : (uy >= a.ncy ? 1 : 0);
        col = (ux - sx * a.ncx) * a.ncy + (uy - sy * a.ncy);
        const float clx = a.lo[0] + ux * a.cs[0], cly = a.lo[1] + uy * a.cs[1];
        const float gx = fmaxf(fmaxf(clx - ihi[0], ilo[0] - (clx + a.cs[0])), 0.f);
        const float gy = fmaxf(fmaxf(cly - ihi[1], ilo[1] - (cly + a.cs[1])), 0.f);
        near = gx * gx + gy * gy <= R2;
      } else {
        col = (vx0 + ix) * a.ncy + (vy0 + iy);
      }
      sxy = (sx + 1) | ((sy + 1) << 2);
      if (near) {
#pragma unroll
        for (int z = 0; z < 3; z++) {
          const int sz = z - 1;
          if (!a.periodic && sz != 0) continue;
          // z bins of the window in image sz (bin z of image sz lies at
          // unwrapped bin z + sz * nzb); vacuum: clamped window
          int zlo, zhi;
          if (a.periodic) {
            zlo = max(b0 - sz * a.nzb, 0);
            zhi = min(b1 - sz * a.nzb, a.nzb - 1);
          } else {
            zlo = clampi(b0, 0, a.nzb - 1);
            zhi = clampi(b1, 0, a.nzb - 1);
          }
          if (zlo > zhi) continue;
          const int rs = max(start[col * a.nzb + zlo], half0);
          const int re = start[col * a.nzb + zhi + 1];
          if (re > rs) {
            hs[z] = rs >> 2;
            nh[z] = ((re - 1) >> 2) - hs[z] + 1;
          }
        }
      }
    }
    const int ncol_h = nh[0] + nh[1] + nh[2];
    const unsigned live = __ballot_sync(kAll, ncol_h > 0);
    const int di = deal + __popc(live & ((1u << lane) - 1u));
    deal += __popc(live);
    const int mine_h = (ncol_h > 0 && di % kRowParts == part) ? ncol_h : 0;
    // inclusive scan of this part's half-cluster counts over the lanes
    int incl = mine_h;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(kAll, incl, o);
      if (lane >= o) incl += t;
    }
    const int off = incl - mine_h;
    const int H = __shfl_sync(kAll, incl, 31);
    for (int base = 0; base < H; base += 32) {
      const int idx = base + lane;
      // the column lane r holding index idx: the last lane with off <= idx
      int r = 0;
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
        const int v = __shfl_sync(kAll, off, r + step);
        if (v <= idx) r += step;
      }
      const int loc = idx - __shfl_sync(kAll, off, r);
      const int n0 = __shfl_sync(kAll, nh[0], r), n1 = __shfl_sync(kAll, nh[1], r);
      const int h0s = __shfl_sync(kAll, hs[0], r), h1s = __shfl_sync(kAll, hs[1], r);
      const int h2s = __shfl_sync(kAll, hs[2], r), cxy = __shfl_sync(kAll, sxy, r);
      int h, z;
      if (loc < n0) {
        h = h0s + loc;
        z = 0;
      } else if (loc < n0 + n1) {
        h = h1s + loc - n0;
        z = 1;
      } else {
        h = h2s + loc - n0 - n1;
        z = 2;
      }
      const int code = cxy | (z << 4);
      bool cand = false;
      if (idx < H) {
        const int parent = h >> 1;
        cand = parent > ci || (parent == ci && code >= kZeroShift);
        if (cand) {
          const float S[3] = {((code & 3) - 1) * a.L[0], (((code >> 2) & 3) - 1) * a.L[1],
                              (z - 1) * a.L[2]};
          const float4 jl4 = bb[2 * h], jh4 = bb[2 * h + 1];
          float g2 = 0.f;
          const float jlo[3] = {jl4.x + S[0], jl4.y + S[1], jl4.z + S[2]};
          const float jhi[3] = {jh4.x + S[0], jh4.y + S[1], jh4.z + S[2]};
#pragma unroll
          for (int c = 0; c < 3; c++) {
            const float g = fmaxf(fmaxf(jlo[c] - ihi[c], ilo[c] - jhi[c]), 0.f);
            g2 += g * g;
          }
          cand = jl4.w > 0.f && g2 <= R2;
        }
      }
      unsigned cm = __ballot_sync(kAll, cand);
      if (!cm) continue;
      // every candidate's lane stages its 4 atoms, cluster and image
      if (cand) {
        const float4 *xs = xhi + 4 * h;
        st_x[wib][4 * lane] = xs[0];
        st_x[wib][4 * lane + 1] = xs[1];
        st_x[wib][4 * lane + 2] = xs[2];
        st_x[wib][4 * lane + 3] = xs[3];
        st_o[wib][lane] = *reinterpret_cast<const int4 *>(sorted + 4 * h);
        st_m[wib][lane] = *reinterpret_cast<const int4 *>(mol_s + 4 * h);
        st_h[wib][lane] = h;
        st_c[wib][lane] = code;
      }
      __syncwarp();
      while (cm) {
        // the next (up to) four candidates, in ascending order
        int bq[4];
        int ng = 0;
#pragma unroll
        for (int q = 0; q < 4; q++) {
          bq[q] = cm ? __ffs(cm) - 1 : 0;
          if (cm) {
            cm &= cm - 1;
            ng = q + 1;
          }
        }
        test4(bq, ng);
      }
      __syncwarp();  // the next batch overwrites the staging
    }
  }
  if (lane == 0) {
    if (count > a.limit) {
      // the row keeps its first limit tiles; the host grows the capacity to
      // at least the largest row's need and repeats the work
      atomicOr(status, ST_LIST_OVERFLOW);
      atomicMax(rebuild + 2, count);
    }
    tile_count[rw] = min(count, a.limit);
  }
  // the row's j-lane entries, in tile order, from the tiles just written
  // (visible to the warp after the __syncwarp)
  __syncwarp();
  {
    const int nt = min(count, a.limit);
    uint2 *erow = jlanes + (size_t)rw * 4 * a.cap;
    int ne = 0;
    for (int k0 = 0; k0 < nt; k0 += 32) {
      const int k = k0 + lane;
      uint2 t = make_uint2(0u, 0u);
      unsigned tz = 0u;
      if (k < nt) {
        t = row[k];
        if (t.x & kModFlag) tz = rowmod[k];
      }
      int nb = 0;
#pragma unroll
      for (int q = 0; q < 4; q++) nb += ((t.y >> (8 * q)) & 0xFFu) != 0u;
      int incl = nb;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(kAll, incl, o);
        if (lane >= o) incl += v;
      }
      int at = ne + incl - nb;
      const uint32_t hj = t.x & kJMask, sh = (t.x >> kShiftBits) & kShiftMask;
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const uint32_t mb = (t.y >> (8 * q)) & 0xFFu;
        if (mb)
          erow[at++] = make_uint2((4u * hj + q) | (sh << kJSlotBits),
                                  mb | (((tz >> (8 * q)) & 0xFFu) << 8));
      }
      ne += __shfl_sync(kAll, incl, 31);
    }
    if (lane == 0) jl_count[rw] = ne;
  }
  __syncwarp();  // the next row reuses the staging
  }  // rows
  // the last warp of the launch to finish sets the counters back to zero
  if (lane == 0) {
    __threadfence();
    if (atomicAdd(&work[1], 1) == blk.n * kBuildWarps - 1) {
      work[0] = 0;
      work[1] = 0;
    }
  }
}
__global__ void __launch_bounds__(kBuildWarps * 32, 3) k_build_tiles(BuildArgs a) {
  pdl_wait();  // the predecessor's writes are visible from here on
  build_body(a, own_blk());
}
__global__ void __launch_bounds__(kBuildWarps * 32, 3)
k_build_tiles_batch(const BuildArgs *__restrict__ tab, const int *__restrict__ first, int nm) {
  const int m = batch_member(first, nm, blockIdx.x);
  build_body(tab[m], batch_blk(first, m));
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
  const int n = s->n;
  const Box &b = s->box;
  double lo[3], span[3];
  if (b.periodic) {
    for (int a = 0; a < 3; a++)
      if (b.e[a] <= nl->reach + 0.1)
        return fail(PMGPU_ERR_UNSUPPORTED,
                    "box edge must exceed cutoff + list skin on the pair-list path");
    for (int a = 0; a < 3; a++) {
      lo[a] = b.min[a] - b.origin[a];
      span[a] = b.max[a] - b.min[a];
    }
  } else {
    // Vacuum: a fixed grid over the current bounding box plus a margin of
    // one reach; atoms that later leave it clamp into the edge columns
    // (the grid only orders atoms; cluster boxes decide the pairs).
    std::vector<double> h(3 * (size_t)std::max(n, 1), 0.0);
    if (n) {
      PM_CUDA(cudaMemcpyAsync(h.data(), s->d_pos, sizeof(double) * 3 * n,
                              cudaMemcpyDeviceToHost, s->stream));
      PM_CUDA(cudaStreamSynchronize(s->stream));
    }
    double mn[3] = {h[0], h[1], h[2]}, mx[3] = {h[0], h[1], h[2]};
    for (int i = 1; i < n; i++)
      for (int a = 0; a < 3; a++) {
        mn[a] = std::min(mn[a], h[3 * i + a]);
        mx[a] = std::max(mx[a], h[3 * i + a]);
      }
    for (int a = 0; a < 3; a++) {
      lo[a] = mn[a] - nl->reach;
      span[a] = (mx[a] - mn[a]) + 2 * nl->reach;
    }
  }
  nl->ncx = std::max(1, std::min(256, (int)std::floor(span[0] / kColumnWidth)));
  nl->ncy = std::max(1, std::min(256, (int)std::floor(span[1] / kColumnWidth)));
  nl->nzb = std::max(1, std::min(1024, (int)std::floor(span[2] / kZBin)));
  nl->cs[0] = span[0] / nl->ncx;
  nl->cs[1] = span[1] / nl->ncy;
  nl->cs[2] = span[2] / nl->nzb;
  for (int a = 0; a < 3; a++) nl->lo[a] = lo[a];
  nl->ncol = nl->ncx * nl->ncy;
  nl->nkeys = nl->ncol * nl->nzb;
  // slots: every column padded to whole 8-atom clusters
  nl->ns_max = ((n + 7 * nl->ncol) + 7) & ~7;
  nl->nclusters = nl->ns_max / 8;
  nl->nrows = nl->nclusters * kRowParts;
  // capacity: j clusters within (reach + cluster extent) of an i cluster at
  // the mean density (condensed matter bounds the local density even in
  // sparse boxes), half of them by the one-tile-per-pair rule, with
  // headroom; an overflow is detected and the capacity doubled
  const double dens = b.periodic ? std::max(n / b.V, 0.12) : 0.15;
  const double r = nl->reach + 5.0;
  const double expect = 4.18879 * r * r * r * dens / 4.0 / 2.0;
  int cap = (int)(expect / kRowParts * 1.6 + 32);
  cap = std::min(cap, std::max(32, nl->ns_max / 4 * 27));
  cap = (cap + 31) & ~31;
  if (nl->cap > cap) cap = nl->cap;
  if (nl->cap_set > 0) cap = nl->cap_set;  // a capacity the caller fixed
  nl->cap = cap;
  // column buckets: four times a column's mean count, at least 256 atoms
  // (vacuum grids are dense in the middle), at most the sort's kColCap; a
  // fuller column flags an overflow and the buckets grow to its count
  int bcap = std::max(256, 4 * ((n + nl->ncol - 1) / nl->ncol));
  if (nl->bcap > bcap) bcap = nl->bcap;
  if (nl->bcap_set > 0) bcap = nl->bcap_set;
  nl->bcap = std::min(kColCap, (bcap + 31) & ~31);
  const size_t nn = std::max(1, n), ns = std::max(8, nl->ns_max);
  PM_CHECK(dev_alloc(s, &nl->d_zkey, sizeof(unsigned) * nn));
  PM_CHECK(dev_alloc(s, &nl->d_bucket, sizeof(int) * (size_t)nl->bcap * nl->ncol));
  PM_CHECK(dev_alloc(s, &nl->d_col_count, sizeof(int) * nl->ncol));
  PM_CUDA(cudaMemsetAsync(nl->d_col_count, 0, sizeof(int) * nl->ncol, s->stream));
  PM_CHECK(dev_alloc(s, &nl->d_col_base, sizeof(int) * (nl->ncol + 1)));
  PM_CHECK(dev_alloc(s, &nl->d_key_start, sizeof(int) * (nl->nkeys + 1)));
  PM_CHECK(dev_alloc(s, &nl->d_sorted, sizeof(int) * ns));
  PM_CHECK(dev_alloc(s, &nl->d_slot_of, sizeof(int) * std::max(1, s->n)));
  PM_CUDA(cudaMemsetAsync(nl->d_sorted, 0xff, sizeof(int) * ns, s->stream));
  PM_CHECK(dev_alloc(s, &nl->d_offset, sizeof(double) * 3 * nn));
  PM_CHECK(dev_alloc(s, &nl->d_xbuild, sizeof(double) * 3 * nn));
  PM_CHECK(dev_alloc(s, &nl->d_xhi, sizeof(float4) * ns));
  PM_CHECK(dev_alloc(s, &nl->d_xlo, sizeof(float4) * ns));
  PM_CHECK(dev_alloc(s, &nl->d_xw, sizeof(double4) * ns));
  PM_CHECK(dev_alloc(s, &nl->d_mol_s, sizeof(int) * ns));
  PM_CHECK(dev_alloc(s, &nl->d_bb, sizeof(float4) * 2 * (ns / 4)));
  PM_CHECK(dev_alloc(s, &nl->d_fslot, sizeof(long long) * 3 * ns));
  PM_CUDA(cudaMemsetAsync(nl->d_fslot, 0, sizeof(long long) * 3 * ns, s->stream));
  PM_CHECK(dev_alloc(s, &nl->d_tiles, sizeof(uint2) * (size_t)cap * nl->nrows));
  PM_CHECK(dev_alloc(s, &nl->d_tmod, sizeof(unsigned) * (size_t)cap * nl->nrows));
  PM_CHECK(dev_alloc(s, &nl->d_jlanes, sizeof(uint2) * 4 * (size_t)cap * nl->nrows));
  PM_CHECK(dev_alloc(s, &nl->d_jl_count, sizeof(int) * std::max(1, nl->nrows)));
  PM_CUDA(cudaMemsetAsync(nl->d_jl_count, 0, sizeof(int) * std::max(1, nl->nrows), s->stream));
  PM_CHECK(dev_alloc(s, &nl->d_tile_count, sizeof(int) * std::max(1, nl->nrows)));
  PM_CUDA(cudaMemsetAsync(nl->d_tile_count, 0, sizeof(int) * std::max(1, nl->nrows),
                          s->stream));
  PM_CHECK(dev_alloc(s, &nl->d_maxdisp, 2 * sizeof(unsigned int)));
  PM_CUDA(cudaMemsetAsync(nl->d_maxdisp, 0, 2 * sizeof(unsigned int), s->stream));
  PM_CHECK(dev_alloc(s, &nl->d_rebuild, 4 * sizeof(int)));
  PM_CUDA(cudaMemsetAsync(nl->d_rebuild, 0, 4 * sizeof(int), s->stream));
  PM_CHECK(dev_alloc(s, &nl->d_build_work, 3 * sizeof(int)));
  PM_CUDA(cudaMemsetAsync(nl->d_build_work, 0, 3 * sizeof(int), s->stream));
  nl->built = 0;
  return PMGPU_OK;
}

int nb_list_free(System *s, NeighborList *nl) {
  void *ptrs[] = {nl->d_zkey, nl->d_bucket, nl->d_col_count, nl->d_col_base,
                  nl->d_key_start, nl->d_sorted,
                  nl->d_offset, nl->d_xbuild, nl->d_xhi, nl->d_xlo, nl->d_xw, nl->d_mol_s,
                  nl->d_bb, nl->d_fslot, nl->d_slot_of, nl->d_tiles, nl->d_tmod,
                  nl->d_jlanes, nl->d_jl_count, nl->d_tile_count, nl->d_maxdisp,
                  nl->d_rebuild, nl->d_build_work};
  for (void *p : ptrs) dev_free(s, p);
  nl->d_build_work = nullptr;
  nl->d_bucket = nl->d_col_count = nullptr;
  nl->d_col_base = nl->d_key_start = nl->d_sorted = nl->d_mol_s = nl->d_tile_count = nullptr;
  nl->d_zkey = nullptr;
  nl->d_rebuild = nullptr;
  nl->d_offset = nl->d_xbuild = nullptr;
  nl->d_xhi = nl->d_xlo = nl->d_bb = nullptr;
  nl->d_xw = nullptr;
  nl->d_tiles = nullptr;
  nl->d_tmod = nullptr;
  nl->d_jlanes = nullptr;
  nl->d_jl_count = nullptr;
  nl->d_fslot = nullptr;
  nl->d_slot_of = nullptr;
  nl->d_maxdisp = nullptr;
  return PMGPU_OK;
}

// Launch arguments of a list's per-step kernels (the sort, the gather and
// the tile build).
struct ListArgs {
  BinArgs bin;
  SortArgs sort;
  GatherArgs gather;
  BuildArgs build;
};

static void list_args(System *s, NeighborList *nl, ListArgs *L) {
  ListGrid g;
  g.box = s->box;
  g.n = s->n;
  g.periodic = s->box.periodic;
  g.ncx = nl->ncx; g.ncy = nl->ncy; g.nzb = nl->nzb;
  for (int a = 0; a < 3; a++) {
    g.lo[a] = nl->lo[a];
    g.inv[a] = 1.0 / nl->cs[a];
  }
  const ScanArgs scan{nl->ncol, nl->nkeys, nl->ns_max, nl->bcap,
                      nl->d_col_base, nl->d_key_start, nl->d_sorted};
  L->bin = BinArgs{g, s->d_pos, nl->d_rebuild, nl->d_zkey, nl->d_col_count, nl->d_bucket,
                   nl->d_offset, nl->d_xbuild, s->d_status, (unsigned *)nl->d_build_work + 2,
                   scan};
  L->gather = GatherArgs{nl->ns_max, s->d_pos, nl->d_offset, nl->d_sorted, s->d_charge,
                         s->d_type, s->d_mol, nl->d_xhi, nl->d_xlo, nl->d_xw, nl->d_mol_s,
                         nl->d_rebuild, nl->d_bb};
  L->sort = SortArgs{nl->d_rebuild, nl->nzb, nl->ncol, nl->bcap, (float)(1.0 / nl->cs[2]),
                     nl->d_col_count, nl->d_col_base, nl->d_bucket, nl->d_zkey, nl->d_sorted,
                     nl->d_slot_of, nl->d_key_start, s->d_status, nl->d_rebuild + 3,
                     0, s->precision == PMGPU_PREC_MIXED ? 1 : 0, L->gather};
  TileBuildArgs ba;
  ba.nclusters = nl->nclusters;
  ba.periodic = s->box.periodic;
  ba.ncx = nl->ncx; ba.ncy = nl->ncy; ba.nzb = nl->nzb;
  for (int c = 0; c < 3; c++) {
    ba.lo[c] = (float)nl->lo[c];
    ba.cs[c] = (float)nl->cs[c];
    ba.L[c] = (float)s->box.e[c];
    ba.H2[c] = (float)s->box.H2[c];
  }
  // FP32 pair test with a margin well above its rounding error; wider for
  // the box culling
  const double r1 = nl->reach + 0.01;
  ba.reach2 = (float)(r1 * r1);
  ba.cull = (float)(nl->reach + 0.05);
  ba.cap = nl->cap;
  ba.limit = nl->limit > 0 ? std::min(nl->limit, nl->cap) : nl->cap;
  ba.excl_start = s->d_excl_start;
  ba.excl_partner = s->d_excl_partner;
  ba.excl_class = s->d_excl_class;
  L->build = BuildArgs{ba, nl->d_rebuild, nl->d_sorted, nl->d_key_start, nl->d_xhi,
                       nl->d_mol_s, nl->d_bb, nl->d_tiles, nl->d_tmod, nl->d_tile_count,
                       nl->d_jlanes, nl->d_jl_count, s->d_status, nl->d_build_work};
}

// Sort + (conditional) list build + per-step gather.  Never synchronises
// with the host: the rebuild decision lives in device memory.
int nb_prepare(System *s, NeighborList *nl, int force_rebuild) {
  const int n = s->n;
  if (n == 0) return PMGPU_OK;
  cudaStream_t st = s->stream;
  const int T = 256;
  const int nb = (n + T - 1) / T, nbs = (nl->ns_max + T - 1) / T;
  const int first = !nl->built;
  const float hs = (float)(0.5 * nl->skin);
  // an MD step's update kernel has taken the decision already, and written
  // the slot records of the drifted positions
  const int updated = nl->decided && !first && !force_rebuild;
  if (!nl->decided || first || force_rebuild) {
    PM_CUDA(launch_pdl(k_check_rebuild, nb, kCheckThreads, 0, st, n, s->d_pos, nl->d_xbuild,
                       nl->d_maxdisp, nl->d_rebuild, hs * hs, (force_rebuild || first) ? 1 : 0));
    s->kernels++;
  }
  nl->decided = 0;
  // each kernel of the chain launches as a programmatic dependent of the
  // one before, so on the steps that keep the list their early exits
  // overlap their launches: the binning (with the column layout), the
  // column sort (with the slot records on an MD step's rebuild) and, outside
  // MD steps, the slot records of every evaluation
  ListArgs la;
  list_args(s, nl, &la);
  la.sort.gather = updated;
  PM_CUDA(launch_pdl(k_bin, nb, T, 0, st, la.bin));
  PM_CUDA(launch_pdl(k_sort_cols, nl->ncol, kSortThreads, 0, st, la.sort));
  s->kernels += 2;
  if (!updated) {
    PM_CUDA(launch_pdl(s->precision == PMGPU_PREC_MIXED ? k_gather<true> : k_gather<false>, nbs,
                       T, 0, st, la.gather));
    s->kernels++;
  }
  PM_CUDA(cudaGetLastError());
  nl->built = 1;  // the slot order exists from here on
  return PMGPU_OK;
}

// The (conditional) tile build of a prepared list (the cluster boxes come
// with the gather).
int nb_build(System *s, NeighborList *nl) {
  if (s->n == 0) return PMGPU_OK;
  cudaStream_t st = s->stream;
  ListArgs la;
  list_args(s, nl, &la);
  // a grid of resident blocks whose warps stride over the rows: cheap to
  // launch on the steps that keep the list
  static int sms = 0;
  if (!sms && (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device) !=
                   cudaSuccess || sms <= 0))
    sms = 148;
  const int nblk = std::max(1, std::min((nl->nrows + kBuildWarps - 1) / kBuildWarps, 3 * sms));
  PM_CUDA(launch_pdl(k_build_tiles, nblk, kBuildWarps * 32, 0, st, la.build));
  PM_CUDA(cudaGetLastError());
  return PMGPU_OK;
}

static int pair_splits(int nclusters);

// The Ewald real-space force factor of one pair in FP64, the reference's
// form with the A&S erfc (MathUtilities.cpp:39-49; Abramowitz & Stegun
// 7.1.26): [erfc(a r)/r + 2a/sqrt(pi) exp(-a^2 r^2)] / r^2.
static double ewald_factor(double alpha, double r2) {
  const double r = std::sqrt(r2), x = alpha * r;
  const double t = 1.0 / (1.0 + 0.3275911 * x);
  const double poly =
      t * (0.254829592 + t * (-0.284496736 + t * (1.421413741 + t * (-1.453152027 +
                                                                    t * 1.061405429))));
  const double ex = std::exp(-x * x);
  return (poly * ex / r + 2.0 * alpha / std::sqrt(M_PI) * ex) / r2;
}

// The cubic of each table interval through the factor at the four
// Chebyshev nodes of the interval (near-minimax), as monomials in t.
int ewald_table_build(System *s, Force *f) {
  std::vector<float4> tab(kEwTabN);
  const int sub = 1 << kEwTabSubBits;
  double tn[4];
  for (int k = 0; k < 4; k++) tn[k] = 0.5 + 0.5 * std::cos((2 * k + 1) * M_PI / 8.0);
  for (int i = 0; i < kEwTabN; i++) {
    const int e = kEwTabLoExp + i / sub, k = i % sub;
    const double a = std::ldexp(1.0 + (double)k / sub, e);
    const double b = std::ldexp(1.0 + (double)(k + 1) / sub, e);
    // Vandermonde system V c = y for c0 + c1 t + c2 t^2 + c3 t^3
    double V[4][5];
    for (int r = 0; r < 4; r++) {
      double tp = 1.0;
      for (int c = 0; c < 4; c++, tp *= tn[r]) V[r][c] = tp;
      V[r][4] = ewald_factor(f->alpha, a + tn[r] * (b - a));
    }
    for (int c = 0; c < 4; c++) {  // Gaussian elimination with partial pivoting
      int pr = c;
      for (int r = c + 1; r < 4; r++)
        if (std::fabs(V[r][c]) > std::fabs(V[pr][c])) pr = r;
      for (int q = 0; q < 5; q++) std::swap(V[c][q], V[pr][q]);
      for (int r = 0; r < 4; r++) {
        if (r == c) continue;
        const double m = V[r][c] / V[c][c];
        for (int q = c; q < 5; q++) V[r][q] -= m * V[c][q];
      }
    }
    tab[i] = make_float4((float)(V[0][4] / V[0][0]), (float)(V[1][4] / V[1][1]),
                         (float)(V[2][4] / V[2][2]), (float)(V[3][4] / V[3][3]));
  }
  if (f->d_ewtab) dev_free(s, f->d_ewtab);
  f->d_ewtab = nullptr;
  PM_CHECK(dev_alloc(s, &f->d_ewtab, sizeof(float4) * kEwTabN));
  PM_CUDA(cudaMemcpyAsync(f->d_ewtab, tab.data(), sizeof(float4) * kEwTabN,
                          cudaMemcpyHostToDevice, s->stream));
  // the host vector goes out of scope: wait for the copy
  PM_CUDA(cudaStreamSynchronize(s->stream));
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
  a.max_cut2 = mx;
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
  a.nclusters = nl->nclusters;
  a.splits = pair_splits(nl->nclusters);
  a.sorted = nl->d_sorted;
  a.pos = s->d_pos;
  a.excl_start = s->d_excl_start;
  a.excl_partner = s->d_excl_partner;
  a.excl_class = s->d_excl_class;
  // the table covers r^2 below 2^(kEwTabLoExp + kEwTabOctaves)
  a.ewtab = sizeof(Real) == 4 && (t.mask & TERM_EWALD) && !t.exact_erf &&
                    a.max_hi < std::ldexp(1.0, kEwTabLoExp + kEwTabOctaves)
                ? t.ewtab
                : nullptr;
  a.tiles = nl->d_tiles;
  a.tmod = nl->d_tmod;
  a.jlanes = nl->d_jlanes;
  a.jl_count = nl->d_jl_count;
  a.tile_count = nl->d_tile_count;
  a.xhi = nl->d_xhi;
  a.xlo = nl->d_xlo;
  a.xw = nl->d_xw;
  a.type = s->d_type;
  a.lj32 = s->d_lj32;
  a.lj64 = s->d_lj64;
  a.fslot = nl->d_fslot;
  a.ns = nl->ns_max;
  a.acc = s->d_acc;
  a.pairbuf = s->d_pairbuf;
  a.pairbuf_cap = s->pairbuf_cap;
  a.paircount = s->d_paircount;
  a.count_pairs = s->count_pairs;
  a.energy_only = 0;
}

// Compile-time switch kind of a term for the specialised force-only
// kernel: -2 when the configuration has no specialisation.
static int spec_kind(const SwitchParams &sw) {
  if (!sw.modify) return kSwNone;
  if (sw.kind == PMGPU_SW_C2 || sw.kind == PMGPU_SW_C1) return sw.kind;
  return -2;
}

// Warps per i cluster of the tile kernel: about four waves of the
// force-only kernel's resident warps (40 per SM), at most 8 per cluster, so blocks that finish early are refilled and the
// tail stays short.  The split depends only on the system, so every launch
// of a system sums its forces in the same order.
static int pair_splits(int nclusters) {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        sms <= 0)
      sms = 148;
  }
  const long long want = 4LL * sms * 40;
  return (int)std::max(1LL, std::min(8LL, (want + nclusters / 2) / std::max(1, nclusters)));
}

template <typename Real, int TERMS, typename SPEC>
static void launch_pairs_spec(PairArgs<Real> &a, cudaStream_t st, int mode) {
  const int T = kPairWarps * 32;
  const int nb = (int)(((long long)a.nclusters * a.splits + kPairWarps - 1) / kPairWarps);
  if (nb == 0) return;
  switch (mode) {
    case PAIR_FORCE: k_pairs<Real, TERMS, PAIR_FORCE, SPEC><<<nb, T, 0, st>>>(a); break;
    case PAIR_ENERGY: k_pairs<Real, TERMS, PAIR_ENERGY, SPEC><<<nb, T, 0, st>>>(a); break;
    case PAIR_VIRIAL: k_pairs<Real, TERMS, PAIR_VIRIAL, SPEC><<<nb, T, 0, st>>>(a); break;
    default: k_pairs<Real, TERMS, PAIR_RECORD, SPEC><<<nb, T, 0, st>>>(a); break;
  }
}

// Work items per i cluster of the j-lane force-only kernel: about three
// waves of its resident warps (3 blocks of 8 warps per SM), at most 8 per
// cluster.  Depends only on the system, so every launch of a system sums
// its forces in the same order.
static int jl_splits(int nclusters) {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        sms <= 0)
      sms = 148;
  }
  static int forced = -1;
  if (forced < 0) {
    const char *e = std::getenv("PMGPU_JL_SPLITS");
    forced = e ? std::max(0, std::atoi(e)) : 0;
  }
  if (forced) return std::min(forced, kJlMaxSplits);
  const long long want = 3LL * sms * 3 * kJlWarps;
  return (int)std::max(1LL, std::min(8LL, (want + nclusters / 2) / std::max(1, nclusters)));
}

// The specialised force-only FP32 kernels: j atoms on the lanes
// (k_pairs_jl), the LJ table in shared memory when it is small.
template <typename Real, int TERMS, typename SPEC>
static void launch_force_spec(PairArgs<Real> &a, cudaStream_t st) {
  if constexpr (sizeof(Real) == 4) {
    a.splits = jl_splits(a.nclusters);
    const long long items = (long long)a.nclusters * a.splits;
    const int nb = (int)((items + kJlWarps - 1) / kJlWarps);
    if (nb == 0) return;
    // the Ewald force table for the LJ + Ewald real form when the list has one
    constexpr bool kTab = TERMS == (TERM_LJ | TERM_EWALD) && SPEC::exact == 0;
    const bool tab = kTab && a.ewtab != nullptr;
    if (a.ntypes <= kJlMaxTypes) {
      if (tab) k_pairs_jl<TERMS, SPEC, true, kTab><<<nb, kJlWarps * 32, 0, st>>>(a);
      else k_pairs_jl<TERMS, SPEC, true, false><<<nb, kJlWarps * 32, 0, st>>>(a);
    } else {
      if (tab) k_pairs_jl<TERMS, SPEC, false, kTab><<<nb, kJlWarps * 32, 0, st>>>(a);
      else k_pairs_jl<TERMS, SPEC, false, false><<<nb, kJlWarps * 32, 0, st>>>(a);
    }
  } else {
    launch_pairs_spec<Real, TERMS, SPEC>(a, st, PAIR_FORCE);
  }
}

// Returns the form launched: PMGPU_PAIRK_GENERIC or one of the specialised
// force-only forms (PMGPU_PAIRK_*).
template <typename Real, int TERMS>
static int launch_pairs_t(PairArgs<Real> &a, cudaStream_t st, int mode, const PairTerms &t) {
  // specialised force-only FP32 kernels of the common configurations
  // (every term with one cutoff, box edges at least twice the cutoff)
  if (sizeof(Real) == 4 && mode != PAIR_RECORD && a.same_cut && !a.minimal_image) {
    const int lk = spec_kind(t.lj_sw), ck = spec_kind(t.coul_sw);
    int form = PMGPU_PAIRK_GENERIC;
    if (TERMS == (TERM_LJ | TERM_EWALD) && !t.exact_erf && lk == PMGPU_SW_C2)
      form = PMGPU_PAIRK_LJC2_EWALD;
    else if (TERMS == (TERM_LJ | TERM_COUL) && lk == PMGPU_SW_C2 && ck == PMGPU_SW_C2)
      form = PMGPU_PAIRK_LJC2_COULC2;
    else if (TERMS == (TERM_LJ | TERM_COUL) && lk == PMGPU_SW_C2 && ck == PMGPU_SW_C1)
      form = PMGPU_PAIRK_LJC2_COULC1;
    if (form != PMGPU_PAIRK_GENERIC) {
      // The forces of every mode come from the specialised kernel, so an
      // energy step's forces equal a force-only step's bit for bit (a run
      // split into several calls, whose energy steps fall elsewhere, gives
      // the same trajectory); energies and virial then come from the
      // generic kernel in its energy-only form.
      PairArgs<Real> fa = a;
      if (mode != PAIR_FORCE) fa.count_pairs = 0;  // the energy pass counts
      if (form == PMGPU_PAIRK_LJC2_EWALD)
        launch_force_spec<Real, TERM_LJ | TERM_EWALD, PairSpec<PMGPU_SW_C2, -1, 0>>(fa, st);
      else if (form == PMGPU_PAIRK_LJC2_COULC2)
        launch_force_spec<Real, TERM_LJ | TERM_COUL, PairSpec<PMGPU_SW_C2, PMGPU_SW_C2, -1>>(fa,
                                                                                          st);
      else
        launch_force_spec<Real, TERM_LJ | TERM_COUL, PairSpec<PMGPU_SW_C2, PMGPU_SW_C1, -1>>(fa,
                                                                                          st);
      if (mode != PAIR_FORCE) {
        PairArgs<Real> ea = a;
        ea.energy_only = 1;
        launch_pairs_spec<Real, TERMS, GenericSpec>(ea, st, mode);
      }
      return form;
    }
  }
  launch_pairs_spec<Real, TERMS, GenericSpec>(a, st, mode);
  return PMGPU_PAIRK_GENERIC;
}

template <typename Real>
static int launch_pairs(PairArgs<Real> &a, cudaStream_t st, int mode, const PairTerms &t,
                        int *form) {
  switch (a.mask) {
    case TERM_LJ: *form = launch_pairs_t<Real, TERM_LJ>(a, st, mode, t); break;
    case TERM_COUL: *form = launch_pairs_t<Real, TERM_COUL>(a, st, mode, t); break;
    case TERM_LJ | TERM_COUL:
      *form = launch_pairs_t<Real, TERM_LJ | TERM_COUL>(a, st, mode, t);
      break;
    case TERM_EWALD: *form = launch_pairs_t<Real, TERM_EWALD>(a, st, mode, t); break;
    case TERM_LJ | TERM_EWALD:
      *form = launch_pairs_t<Real, TERM_LJ | TERM_EWALD>(a, st, mode, t);
      break;
    default:
      return fail(PMGPU_ERR_UNSUPPORTED, "unsupported pair-term combination");
  }
  PM_CUDA(cudaGetLastError());
  return PMGPU_OK;
}

// mode: PAIR_FORCE (forces only), PAIR_ENERGY (+ FP64 energies),
// PAIR_VIRIAL (+ virial), PAIR_RECORD (+ pair-set recording).
int nb_pair_forces(System *s, NeighborList *nl, const PairTerms &t, int mode, int fold) {
  if (s->n == 0) return PMGPU_OK;
  if (s->precision == PMGPU_PREC_MIXED) {
    PairArgs<float> a;
    fill_pair_args<float>(a, s, nl, t);
    PM_CHECK(launch_pairs<float>(a, s->stream, mode, t, &nl->last_form));
  } else {
    PairArgs<double> a;
    fill_pair_args<double>(a, s, nl, t);
    PM_CHECK(launch_pairs<double>(a, s->stream, mode, t, &nl->last_form));
  }
  // In the force-only steps of an MD run with one list the next update
  // kernel adds the slot buffer into the forces itself (and clears it)
  if (!fold && mode == PAIR_FORCE && s->lists.size() == 1) {
    nl->slot_pending = 1;
    return PMGPU_OK;
  }
  nl->slot_pending = 1;
  return nb_fold_slots(s, nl);
}

int nb_fold_slots(System *s, NeighborList *nl) {
  if (!nl->slot_pending || s->n == 0) return PMGPU_OK;
  PM_CUDA(launch_pdl(k_slot_forces, (nl->ns_max + 255) / 256, 256, 0, s->stream,
                     SlotArgs{nl->ns_max, s->n, nl->d_sorted, nl->d_fslot, s->d_force}));
  PM_CUDA(cudaGetLastError());
  nl->slot_pending = 0;
  return PMGPU_OK;
}

int fold_pending_slots(System *s) {
  for (auto &nl : s->lists) PM_CHECK(nb_fold_slots(s, &nl));
  return PMGPU_OK;
}

// ---------------------------------------------------------------- batches
// The list and pair kernels of an ensemble's members as batched launches:
// one launch per kernel over every member's part (each member with the
// arguments and grid its own launch would have), so a member's results are
// those of its own launches.
struct NbBatch {
  BatchTable<BinArgs> bin;
  BatchTable<SortArgs> sort;
  BatchTable<GatherArgs> gather;
  BatchTable<BuildArgs> build;
  int terms = 0;
  int form = PMGPU_PAIRK_GENERIC;  // the specialised form of the jl members
  int smem_lj = 1;
  int tab = 1;                         // every jl member has the Ewald force table
  BatchTable<PairArgs<float>> jl;      // members with the specialised force-only form
  BatchTable<PairArgs<float>> gforce;  // members without one (force-only, generic kernel)
  BatchTable<PairArgs<float>> energy;  // every member on energy steps
  BatchTable<SlotArgs> slots;
  std::vector<int> has_form;           // per member: 1 if in jl
  std::vector<PairArgs<float>> base;   // per member: its force-only pair arguments
  BatchTable<PairArgs<float>> probe;   // a timing launch (nb_batch_time_jl)
};

NbBatch *nb_batch_new() { return new NbBatch(); }
void nb_batch_free(NbBatch *b) {
  if (!b) return;
  b->bin.release(); b->sort.release();
  b->gather.release(); b->build.release(); b->jl.release(); b->gforce.release();
  b->energy.release(); b->slots.release(); b->probe.release();
  delete b;
}

// The specialised force-only form a member's pair launch takes
// (launch_pairs_t), or PMGPU_PAIRK_GENERIC.
static int special_form(const PairArgs<float> &a, const PairTerms &t) {
  if (!a.same_cut || a.minimal_image) return PMGPU_PAIRK_GENERIC;
  const int lk = spec_kind(t.lj_sw), ck = spec_kind(t.coul_sw);
  if (t.mask == (TERM_LJ | TERM_EWALD) && !t.exact_erf && lk == PMGPU_SW_C2)
    return PMGPU_PAIRK_LJC2_EWALD;
  if (t.mask == (TERM_LJ | TERM_COUL) && lk == PMGPU_SW_C2 && ck == PMGPU_SW_C2)
    return PMGPU_PAIRK_LJC2_COULC2;
  if (t.mask == (TERM_LJ | TERM_COUL) && lk == PMGPU_SW_C2 && ck == PMGPU_SW_C1)
    return PMGPU_PAIRK_LJC2_COULC1;
  return PMGPU_PAIRK_GENERIC;
}

// splits[k] > 0 sets member k's jl splits (the tiles of each i cluster
// divided over that many warps), 0 or splits == NULL the single-system
// choice.
int nb_batch_build(NbBatch *b, System *const *m, int n, const PairTerms *terms,
                   const int *splits) {
  static int sms = 0;
  if (!sms && (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m[0]->device) !=
                   cudaSuccess || sms <= 0))
    sms = 148;
  b->bin.clear(); b->sort.clear(); b->gather.clear();
  b->build.clear(); b->jl.clear(); b->gforce.clear(); b->energy.clear(); b->slots.clear();
  b->has_form.assign(n, 0);
  b->base.assign(n, PairArgs<float>());
  b->terms = terms[0].mask;
  b->form = PMGPU_PAIRK_GENERIC;
  b->smem_lj = 1;
  b->tab = 1;
  for (int k = 0; k < n; k++) {
    System *s = m[k];
    NeighborList *nl = &s->lists[0];
    if (s->precision != PMGPU_PREC_MIXED || terms[k].mask != b->terms)
      return fail(PMGPU_ERR_UNSUPPORTED, "ensemble members need one precision and one force set");
    ListArgs la;
    list_args(s, nl, &la);
    const int T = 256;
    const int nb = (s->n + T - 1) / T, nbs = (nl->ns_max + T - 1) / T;
    b->bin.add(la.bin, std::max(1, nb));  // its last block lays out the columns
    b->sort.add(la.sort, nl->ncol);
    b->gather.add(la.gather, nbs);
    b->build.add(la.build, std::max(1, std::min((nl->nrows + kBuildWarps - 1) / kBuildWarps,
                                                3 * sms)));
    PairArgs<float> a;
    fill_pair_args<float>(a, s, nl, terms[k]);
    a.count_pairs = 0;
    const int form = special_form(a, terms[k]);
    if (form != PMGPU_PAIRK_GENERIC) {
      if (b->form != PMGPU_PAIRK_GENERIC && b->form != form)
        return fail(PMGPU_ERR_UNSUPPORTED, "ensemble members need one pair-kernel form");
      b->form = form;
      b->smem_lj = b->smem_lj && a.ntypes <= kJlMaxTypes;
      b->tab = b->tab && a.ewtab != nullptr;
      PairArgs<float> fa = a;
      fa.splits = splits && splits[k] > 0 ? std::min(splits[k], kJlMaxSplits)
                                          : jl_splits(fa.nclusters);
      b->base[k] = fa;
      b->jl.add(fa, (int)(((long long)fa.nclusters * fa.splits + kJlWarps - 1) / kJlWarps));
      b->has_form[k] = 1;
    } else {
      b->gforce.add(a, (int)(((long long)a.nclusters * a.splits + kPairWarps - 1) / kPairWarps));
    }
    PairArgs<float> ea = a;
    ea.energy_only = form != PMGPU_PAIRK_GENERIC;
    b->energy.add(ea, (int)(((long long)a.nclusters * a.splits + kPairWarps - 1) / kPairWarps));
    b->slots.add(SlotArgs{nl->ns_max, s->n, nl->d_sorted, nl->d_fslot, s->d_force},
                 (nl->ns_max + 255) / 256);
  }
  BatchTable<PairArgs<float>> *pt[] = {&b->jl, &b->gforce, &b->energy};
  PM_CUDA(b->bin.upload());
  PM_CUDA(b->sort.upload());
  PM_CUDA(b->gather.upload());
  PM_CUDA(b->build.upload());
  for (auto *t : pt) PM_CUDA(t->upload());
  PM_CUDA(b->slots.upload());
  return PMGPU_OK;
}

// The (conditional) sort, the per-step gather and the (conditional) tile
// build of every member (nb_prepare after an update's rebuild decision,
// then nb_build).
int nb_batch_list(NbBatch *b, cudaStream_t st, long long *launched) {
  const int nm = b->bin.members();
  if (!nm) return PMGPU_OK;
  *launched += 4;
  k_bin_batch<<<b->bin.total(), 256, 0, st>>>(b->bin.d, b->bin.d_first, nm);
  k_sort_cols_batch<<<b->sort.total(), kSortThreads, 0, st>>>(b->sort.d, b->sort.d_first, nm);
  k_gather_batch<true><<<b->gather.total(), 256, 0, st>>>(b->gather.d, b->gather.d_first, nm);
  k_build_tiles_batch<<<b->build.total(), kBuildWarps * 32, 0, st>>>(b->build.d,
                                                                      b->build.d_first, nm);
  PM_CUDA(cudaGetLastError());
  return PMGPU_OK;
}

template <int TERMS>
static int launch_generic_batch(BatchTable<PairArgs<float>> &t, int mode, cudaStream_t st) {
  if (!t.members() || !t.total()) return 0;
  const int T = kPairWarps * 32;
  if (mode == PAIR_FORCE)
    k_pairs_batch<float, TERMS, PAIR_FORCE, GenericSpec><<<t.total(), T, 0, st>>>(t.d, t.d_first,
                                                                                   t.members());
  else
    k_pairs_batch<float, TERMS, PAIR_ENERGY, GenericSpec><<<t.total(), T, 0, st>>>(
        t.d, t.d_first, t.members());
  return 1;
}

static int generic_batch(BatchTable<PairArgs<float>> &t, int terms, int mode, cudaStream_t st) {
  switch (terms) {
    case TERM_LJ: return launch_generic_batch<TERM_LJ>(t, mode, st);
    case TERM_COUL: return launch_generic_batch<TERM_COUL>(t, mode, st);
    case TERM_LJ | TERM_COUL: return launch_generic_batch<TERM_LJ | TERM_COUL>(t, mode, st);
    case TERM_EWALD: return launch_generic_batch<TERM_EWALD>(t, mode, st);
    default: return launch_generic_batch<TERM_LJ | TERM_EWALD>(t, mode, st);
  }
}

template <int TERMS, typename SPEC>
static void jl_batch(NbBatch *b, BatchTable<PairArgs<float>> &t, cudaStream_t st) {
  constexpr bool kTab = TERMS == (TERM_LJ | TERM_EWALD) && SPEC::exact == 0;
  const int g = t.total(), nm = t.members(), T = kJlWarps * 32;
  if (kTab && b->tab) {
    if (b->smem_lj) k_pairs_jl_batch<TERMS, SPEC, true, kTab><<<g, T, 0, st>>>(t.d, t.d_first, nm);
    else k_pairs_jl_batch<TERMS, SPEC, false, kTab><<<g, T, 0, st>>>(t.d, t.d_first, nm);
  } else {
    if (b->smem_lj) k_pairs_jl_batch<TERMS, SPEC, true, false><<<g, T, 0, st>>>(t.d, t.d_first, nm);
    else k_pairs_jl_batch<TERMS, SPEC, false, false><<<g, T, 0, st>>>(t.d, t.d_first, nm);
  }
}

// The pair forces of every member: force-only (the inner MD steps; the
// slot-ordered forces stay for the next update kernel) or with energies
// (the last step; the slot forces are folded in), as nb_pair_forces does
// for each member.
static int jl_form(NbBatch *b, BatchTable<PairArgs<float>> &t, cudaStream_t st) {
  if (!t.members() || !t.total()) return 0;
  switch (b->form) {
    case PMGPU_PAIRK_LJC2_EWALD:
      jl_batch<TERM_LJ | TERM_EWALD, PairSpec<PMGPU_SW_C2, -1, 0>>(b, t, st);
      break;
    case PMGPU_PAIRK_LJC2_COULC2:
      jl_batch<TERM_LJ | TERM_COUL, PairSpec<PMGPU_SW_C2, PMGPU_SW_C2, -1>>(b, t, st);
      break;
    default:
      jl_batch<TERM_LJ | TERM_COUL, PairSpec<PMGPU_SW_C2, PMGPU_SW_C1, -1>>(b, t, st);
      break;
  }
  return 1;
}

int nb_batch_pairs(NbBatch *b, int mode, cudaStream_t st, long long *launched) {
  *launched += jl_form(b, b->jl, st);
  if (mode == PAIR_FORCE) {
    *launched += generic_batch(b->gforce, b->terms, PAIR_FORCE, st);
  } else {
    *launched += generic_batch(b->energy, b->terms, PAIR_ENERGY, st);
    if (b->slots.total()) {
      k_slot_forces_batch<<<b->slots.total(), 256, 0, st>>>(b->slots.d, b->slots.d_first,
                                                           b->slots.members());
      *launched += 1;
    }
  }
  PM_CUDA(cudaGetLastError());
  return PMGPU_OK;
}

// Device milliseconds of one force-only jl launch over every member with
// the specialised form, member k with splits[k] warps per i cluster (0:
// the single-system choice), averaged over reps launches after one warm-up
// launch.  The launches add into the members' slot buffers, which are
// cleared again, so the members' state is unchanged; the members' lists
// must be built and their slot buffers empty.
int nb_batch_time_jl(NbBatch *b, System *const *m, int n, const int *splits, int reps,
                     cudaStream_t st, double *ms) {
  *ms = 0.0;
  b->probe.clear();
  for (int k = 0; k < n && k < (int)b->has_form.size(); k++) {
    if (!b->has_form[k]) continue;
    PairArgs<float> a = b->base[k];
    a.splits = splits[k] > 0 ? std::min(splits[k], kJlMaxSplits) : jl_splits(a.nclusters);
    b->probe.add(a, (int)(((long long)a.nclusters * a.splits + kJlWarps - 1) / kJlWarps));
  }
  if (!b->probe.members()) return PMGPU_OK;
  PM_CUDA(b->probe.upload());
  cudaEvent_t e0, e1;
  PM_CUDA(cudaEventCreate(&e0));
  PM_CUDA(cudaEventCreate(&e1));
  jl_form(b, b->probe, st);
  cudaEventRecord(e0, st);
  for (int r = 0; r < reps; r++) jl_form(b, b->probe, st);
  cudaEventRecord(e1, st);
  cudaError_t err = cudaEventSynchronize(e1);
  float t = 0.f;
  if (err == cudaSuccess) err = cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  PM_CUDA(err);
  PM_CUDA(cudaGetLastError());
  for (int k = 0; k < n && k < (int)b->has_form.size(); k++) {
    if (!b->has_form[k]) continue;
    NeighborList &nl = m[k]->lists[0];
    PM_CUDA(cudaMemsetAsync(nl.d_fslot, 0, sizeof(long long) * 3 * (size_t)nl.ns_max, st));
  }
  PM_CUDA(cudaStreamSynchronize(st));
  *ms = reps > 0 ? t / reps : 0.0;
  return PMGPU_OK;
}

// The jl splits member k takes (its own choice when splits[k] is 0) and
// its i-cluster count; -1 / 0 for a member without the specialised form.
void nb_batch_member_info(NbBatch *b, int k, int *splits, int *clusters) {
  const bool f = k >= 0 && k < (int)b->has_form.size() && b->has_form[k];
  *splits = f ? b->base[k].splits : -1;
  *clusters = f ? b->base[k].nclusters : 0;
}

// Host-side state of the members after a batched step's list and pair
// work, as nb_prepare / nb_pair_forces leave it.
void nb_batch_mark(NbBatch *b, System *const *m, int n, int mode) {
  for (int k = 0; k < n; k++) {
    NeighborList &nl = m[k]->lists[0];
    nl.built = 1;
    nl.decided = 0;
    nl.slot_pending = mode == PAIR_FORCE;
    nl.last_form = b->has_form[k] ? b->form : PMGPU_PAIRK_GENERIC;
  }
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

// NonbondedSimpleFull with switching functions: OneAtomPair /
// OneAtomPairTwo (force/OneAtomPair.h:47-107, force/OneAtomPairTwo.h:30-100)
// over every pair, vacuum or the minimal image of a periodic box, the
// Complement switches included.  FP64 pair arithmetic in both precisions.
// Same decomposition as k_simplefull: every i sees every j != i and keeps
// only its own force; energies and virial are halved at the end.
struct SfSwArgs {
  int n, jchunk;
  const double *pos, *charge;
  const int *type, *mol;
  int ntypes;
  const double4 *lj64;
  const int2 *ex_range;
  const int *ex_start, *ex_partner, *ex_class;
  double csf;
  Box box;
  SwitchDev<double> lj_sw, coul_sw;
  int lj, coul, modify;
  double rough2;  // the larger rough-test cutoff^2
  long long *force, *acc;
  int em;  // 0 forces, 1 + energies, 2 + virial
  // the Coulomb term as CoulombSCPISM (scpism 1): bulk dielectric, each
  // atom's sqrt(alpha) and water flag (null: no water)
  int scpism;
  double D;
  const double *sqrtalpha;
  const int *water;
};

// CoulombSCPISMForce::operator() (force/coulomb/CoulombSCPISMForce.h:33-71)
// for the pair (i, j) at 1/r^2 = rr2: the Coulomb energy over the
// distance-dependent dielectric and its force over r.
__device__ __forceinline__ void scpism_pair(double qq, double sai, double saj, double D,
                                            double rr2, double &e, double &f) {
  const double rDist = sqrt(rr2);
  const double Dist = 1.0 / rDist;
  const double alpha_ij = sai * saj;
  const double Dp1 = D + 1.0, rDp1 = 1.0 / Dp1, k = (D - 1.0) * 0.5;
  const double DiElec = Dp1 / (1.0 + k * exp(-alpha_ij * Dist)) - 1.0;
  const double rDiElec = 1.0 / DiElec;
  e = qq * rDist * rDiElec;
  const double drDiElec = alpha_ij * rDp1 * (1.0 + DiElec) * (D - DiElec);
  f = (rDiElec * drDiElec + rDist) * e * rDist;
}

__global__ void __launch_bounds__(kSfTile) k_simplefull_sw(SfSwArgs a) {
  __shared__ double sx[kSfTile], sy[kSfTile], sz[kSfTile], sq[kSfTile];
  __shared__ int st[kSfTile], sm[kSfTile];
  const int i = blockIdx.x * kSfTile + threadIdx.x;
  const bool valid = i < a.n;
  const int ii = valid ? i : 0;
  const double xi = a.pos[3 * ii], yi = a.pos[3 * ii + 1], zi = a.pos[3 * ii + 2];
  const double qi = a.charge[ii];
  const int ti = a.type[ii], mi = a.mol[ii];
  const int2 er = a.ex_range[ii];
  double fx = 0, fy = 0, fz = 0, elj = 0, ec = 0;
  double v[6] = {0, 0, 0, 0, 0, 0};
  const int j0 = blockIdx.y * a.jchunk, j1 = min(a.n, j0 + a.jchunk);
  for (int base = j0; base < j1; base += kSfTile) {
    const int j = base + threadIdx.x;
    if (j < j1) {
      sx[threadIdx.x] = a.pos[3 * j];
      sy[threadIdx.x] = a.pos[3 * j + 1];
      sz[threadIdx.x] = a.pos[3 * j + 2];
      sq[threadIdx.x] = a.charge[j];
      st[threadIdx.x] = a.type[j];
      sm[threadIdx.x] = a.mol[j];
    }
    __syncthreads();
    const int lim = min(kSfTile, j1 - base);
    if (valid) {
      for (int k = 0; k < lim; k++) {
        const int jj = base + k;
        if (jj == i) continue;
        double dx, dy, dz;
        // minimalDifference(x_i, x_j): d = x_j - x_i
        const double r2 = box_mindiff(a.box, xi, yi, zi, sx[k], sy[k], sz[k], dx, dy, dz);
        if (r2 > a.rough2) continue;
        // the exclusion table only for atoms of one molecule
        int excl = PMGPU_EXCL_NONE;
        if (sm[k] == mi && jj >= er.x && jj <= er.y) {
          excl = excl_class_of(a.ex_start, a.ex_partner, a.ex_class, i, jj);
          if (excl == PMGPU_EXCL_FULL) continue;
        }
        const double rr2 = 1.0 / r2;
        double f = 0;
        if (a.lj) {
          const double4 p = a.lj64[ti * a.ntypes + st[k]];
          const double A = excl == PMGPU_EXCL_MODIFIED ? p.z : p.x;
          const double B = excl == PMGPU_EXCL_MODIFIED ? p.w : p.y;
          const double r6 = rr2 * rr2 * rr2;
          const double r6B = B * r6, r12A = A * r6 * r6;
          double e = r12A - r6B, ff = 12.0 * r12A * rr2 - 6.0 * r6B * rr2;
          if (a.modify) {
            double sv, sd;
            switch_eval<double>(a.lj_sw, r2, sv, sd);
            ff = ff * sv - e * sd;
            e = e * sv;
          }
          elj += e;
          f += ff;
        }
        if (a.coul) {
          double e, ff;
          if (a.scpism) {
            if (a.water && (a.water[i] || a.water[jj])) {
              e = ff = 0.0;  // no contribution from water (CoulombSCPISMForce.h:38-40)
            } else {
              scpism_pair(qi * sq[k], a.sqrtalpha[i], a.sqrtalpha[jj], a.D, rr2, e, ff);
              if (excl == PMGPU_EXCL_MODIFIED) {
                e *= a.csf;
                ff *= a.csf;
              }
            }
          } else {
            e = qi * sq[k] * sqrt(rr2);
            if (excl == PMGPU_EXCL_MODIFIED) e *= a.csf;
            ff = e * rr2;
          }
          if (a.modify) {
            double sv, sd;
            switch_eval<double>(a.coul_sw, r2, sv, sd);
            ff = ff * sv - e * sd;
            e = e * sv;
          }
          ec += e;
          f += ff;
        }
        fx -= dx * f;
        fy -= dy * f;
        fz -= dz * f;
        if (a.em == 2) {
          const double hf = 0.5 * f;
          v[0] += dx * dx * hf; v[1] += dx * dy * hf; v[2] += dx * dz * hf;
          v[3] += dy * dy * hf; v[4] += dy * dz * hf; v[5] += dz * dz * hf;
        }
      }
    }
    __syncthreads();
  }
  if (valid) {
    red_add(&a.force[i], to_fixed(fx, kForceScale));
    red_add(&a.force[a.n + i], to_fixed(fy, kForceScale));
    red_add(&a.force[2 * a.n + i], to_fixed(fz, kForceScale));
  }
  if (!a.em) return;
  elj = warp_sum(elj) * 0.5;
  ec = warp_sum(ec) * 0.5;
  if (a.em == 2)
    for (int q = 0; q < 6; q++) v[q] = warp_sum(v[q]);
  if ((threadIdx.x & 31) == 0) {
    if (a.lj) red_add(&a.acc[ACC_LJ], to_fixed(elj, kEnergyScale));
    if (a.coul) red_add(&a.acc[ACC_COULOMB], to_fixed(ec, kEnergyScale));
    if (a.em == 2) {
      const int map[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
      for (int q = 0; q < 9; q++)
        red_add(&a.acc[ACC_VIRIAL + q], to_fixed(v[map[q]], kEnergyScale));
    }
  }
}

// The FP32 pass over each unordered pair once, as the reference visits
// i < j (NonbondedSimpleFullSystemForce.h:125-150): a warp takes 32 x 32
// tile pairs (I, J), I <= J, of its block's share (BlockItems), lane l
// holding atom 32 I + l; the J atoms sit in the warp's shared-memory slice
// and are broadcast one at a time.  The force on i accumulates in the lane, the opposite force on
// each j is summed over the lanes by warp_tsum8 per eight j atoms.  Which
// pairs of a tile are excluded or modified comes from the tile's masks
// (sf_tile, sf_bits), read once per tile; on the diagonal tile only j > i
// counts.  Energies and virial (EM 1, 2) are not halved.
constexpr int kSfWarps = 16;

template <bool LJ, bool COUL, bool COMB, int EM>
__global__ void __launch_bounds__(kSfWarps * 32, 1)
k_simplefull_half(int n, int tiles, long long items,
                  const float4 *__restrict__ rec, int ntypes, const float2 *__restrict__ ljab,
                  const float2 *__restrict__ ljcomb, const float4 *__restrict__ lj32,
                  const int *__restrict__ sf_tile, const uint2 *__restrict__ sf_bits, float csf,
                  long long *__restrict__ force, long long *__restrict__ acc) {
  __shared__ float4 sh[kSfWarps][32], sl[kSfWarps][32];
  __shared__ float2 sc[kSfWarps][COMB ? 32 : 1];
  const int lane = threadIdx.x & 31, wb = threadIdx.x >> 5;
  double elj = 0, ec = 0;
  double v[6] = {0, 0, 0, 0, 0, 0};
  __shared__ int counter;
  if (threadIdx.x == 0) counter = 0;
  __syncthreads();
  const BlockItems queue{&counter};
  long long w;
  for (w = queue.next(lane); w < items; w = queue.next(lane)) {
    int I, J;
    tile_pair_of(w, tiles, &I, &J);
    const int i = I * 32 + lane;
    const bool vi = i < n;
    const int ii = vi ? i : 0;
    const float4 hi = rec[ii], li = rec[n + ii];
    const float xh = hi.x, yh = hi.y, zh = hi.z, xl = li.x, yl = li.y, zl = li.z;
    const float qi = hi.w;
    const int ti = __float_as_int(li.w);
    const float2 ci = COMB ? ljcomb[ti] : make_float2(0.f, 0.f);
    // skip: excluded pairs, partners past the end, j <= i on the diagonal
    unsigned skip = 0u, mod = 0u;
    const int q = sf_tile[w];
    if (q >= 0) {
      const uint2 b = sf_bits[32 * q + lane];
      skip = b.x;
      mod = b.y;
    }
    const int jn = n - J * 32;
    if (jn < 32) skip |= ~0u << jn;
    if (I == J) skip |= (2u << lane) - 1u;
    if (!vi) skip = ~0u;
    {
      const int j = J * 32 + lane;
      const int jj = j < n ? j : 0;
      const float4 l = rec[n + jj];
      sh[wb][lane] = rec[jj];
      sl[wb][lane] = l;
      if (COMB) sc[wb][lane] = ljcomb[__float_as_int(l.w)];
    }
    __syncwarp();
    float fx = 0, fy = 0, fz = 0;
#pragma unroll 1
    for (int g = 0; g < 4; g++) {
      float gx[8], gy[8], gz[8];
      float2 tab[8], m14[8];
      if (LJ && !COMB) {
#pragma unroll
        for (int u = 0; u < 8; u++)
          tab[u] = __ldg(&ljab[__float_as_int(sl[wb][g * 8 + u].w) * ntypes + ti]);
      }
      // the modified (1-4) parameters of this group, loaded together
      const unsigned gmod = LJ ? (mod >> (8 * g)) & 0xffu : 0u;
      if (gmod) {
#pragma unroll
        for (int u = 0; u < 8; u++) {
          m14[u] = make_float2(0.f, 0.f);
          if ((gmod >> u) & 1u) {
            const float4 m = __ldg(&lj32[ti * ntypes + __float_as_int(sl[wb][g * 8 + u].w)]);
            m14[u] = make_float2(m.z, m.w);
          }
        }
      }
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int k = g * 8 + u;
        const float4 h = sh[wb][k], l = sl[wb][k];
        const float dx = (h.x - xh) + (l.x - xl);
        const float dy = (h.y - yh) + (l.y - yl);
        const float dz = (h.z - zh) + (l.z - zl);
        const bool use = !((skip >> k) & 1u);
        const bool modified = (mod >> k) & 1u;
        const float r2 = use ? dx * dx + dy * dy + dz * dz : 1.0f;
        const float rinv = rsqrt_nr(r2);
        const float rr2 = rinv * rinv;
        float f = 0;
        if (LJ) {
          float A, B;
          if (COMB) {
            const float2 cj = sc[wb][k];
            const float rm = ci.y + cj.y, e = ci.x * cj.x;
            const float rm2 = rm * rm, rm6 = rm2 * rm2 * rm2;
            B = 2.0f * e * rm6;
            A = e * rm6 * rm6;
          } else {
            A = tab[u].x;
            B = tab[u].y;
          }
          if (gmod && modified) {
            A = m14[u].x;
            B = m14[u].y;
          }
          const float r6 = rr2 * rr2 * rr2;
          const float r6B = B * r6, r12A = A * r6 * r6;
          if (EM && use) elj += (double)(r12A - r6B);
          f += (12.0f * r12A - 6.0f * r6B) * rr2;
        }
        if (COUL) {
          float en = qi * h.w * rinv;
          if (modified) en *= csf;
          if (EM && use) ec += (double)en;
          f += en * rr2;
        }
        f = use ? f : 0.0f;
        fx -= dx * f; fy -= dy * f; fz -= dz * f;
        gx[u] = dx * f; gy[u] = dy * f; gz[u] = dz * f;
        if (EM == 2) {
          const double df = (double)f;
          v[0] += dx * dx * df; v[1] += dx * dy * df; v[2] += dx * dz * df;
          v[3] += dy * dy * df; v[4] += dy * dz * df; v[5] += dz * dz * df;
        }
      }
      const float sx = warp_tsum8(gx, lane), sy = warp_tsum8(gy, lane),
                  sz = warp_tsum8(gz, lane);
      const int jt = J * 32 + g * 8 + (lane >> 2);
      if ((lane & 3) == 0 && jt < n) {
        red_add(&force[jt], to_fixed((double)sx, kForceScale));
        red_add(&force[n + jt], to_fixed((double)sy, kForceScale));
        red_add(&force[2 * n + jt], to_fixed((double)sz, kForceScale));
      }
    }
    if (vi) {
      red_add(&force[i], to_fixed((double)fx, kForceScale));
      red_add(&force[n + i], to_fixed((double)fy, kForceScale));
      red_add(&force[2 * n + i], to_fixed((double)fz, kForceScale));
    }
    __syncwarp();
  }
  if (!EM) return;
  elj = warp_sum(elj);
  ec = warp_sum(ec);
  if (EM == 2)
    for (int q = 0; q < 6; q++) v[q] = warp_sum(v[q]);
  if (lane == 0) {
    if (LJ) red_add(&acc[ACC_LJ], to_fixed(elj, kEnergyScale));
    if (COUL) red_add(&acc[ACC_COULOMB], to_fixed(ec, kEnergyScale));
    if (EM == 2) {
      const int map[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
      for (int q = 0; q < 9; q++) red_add(&acc[ACC_VIRIAL + q], to_fixed(v[map[q]], kEnergyScale));
    }
  }
}

__global__ void k_stage_pairs(int n, const double *__restrict__ pos,
                              const double *__restrict__ charge, const int *__restrict__ type,
                              float4 *__restrict__ rec) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  write_pair_record(rec, n, i, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], charge[i],
                    type ? type[i] : 0);
}

void launch_stage_pairs(int n, const double *pos, const double *charge, const int *type,
                        float4 *rec, cudaStream_t st) {
  if (n > 0) k_stage_pairs<<<(n + 255) / 256, 256, 0, st>>>(n, pos, charge, type, rec);
}

int nb_stage_pairs(System *s) {
  if (!s->d_rec) return PMGPU_OK;
  launch_stage_pairs(s->n, s->d_pos, s->d_charge, s->d_type, s->d_rec, s->stream);
  PM_CUDA(cudaGetLastError());
  return PMGPU_OK;
}

int nb_simplefull_init(System *s) {
  if (!s->d_rec) PM_CHECK(dev_alloc(s, &s->d_rec, sizeof(float4) * 2 * std::max(1, s->n)));
  if (s->d_sf_tile) return PMGPU_OK;
  const int n = s->n, T = (n + 31) / 32;
  const long long items = (long long)T * (T + 1) / 2;
  std::vector<int> tile((size_t)std::max(1LL, items), -1);
  std::vector<uint2> bits;
  std::vector<unsigned> seen;
  // tile pair numbers as tile_pair_of counts them, diagonal by diagonal
  auto dstart = [&](long long d) { return d * T - d * (d - 1) / 2; };
  const size_t ne = s->h_excl.size() / 3;
  for (size_t e = 0; e < ne; e++) {
    const int a = s->h_excl[3 * e], b = s->h_excl[3 * e + 1], c = s->h_excl[3 * e + 2];
    if (a == b) continue;
    const int lo = std::min(a, b), hi = std::max(a, b);
    const long long w = dstart(hi / 32 - lo / 32) + lo / 32;
    if (tile[w] < 0) {
      tile[w] = (int)(bits.size() / 32);
      bits.resize(bits.size() + 32, make_uint2(0u, 0u));
      seen.resize(seen.size() + 32, 0u);
    }
    // the first entry of a pair decides its class, as a scan of the
    // exclusion table in order would
    const size_t idx = 32 * (size_t)tile[w] + (lo & 31);
    const unsigned bit = 1u << (hi & 31);
    if (seen[idx] & bit) continue;
    seen[idx] |= bit;
    if (c == PMGPU_EXCL_FULL) bits[idx].x |= bit;
    else if (c == PMGPU_EXCL_MODIFIED) bits[idx].y |= bit;
  }
  if (bits.empty()) bits.assign(32, make_uint2(0u, 0u));
  PM_CHECK(dev_alloc(s, &s->d_sf_tile, sizeof(int) * tile.size()));
  PM_CHECK(dev_alloc(s, &s->d_sf_bits, sizeof(uint2) * bits.size()));
  PM_CUDA(cudaMemcpyAsync(s->d_sf_tile, tile.data(), sizeof(int) * tile.size(),
                          cudaMemcpyHostToDevice, s->stream));
  PM_CUDA(cudaMemcpyAsync(s->d_sf_bits, bits.data(), sizeof(uint2) * bits.size(),
                          cudaMemcpyHostToDevice, s->stream));
  PM_CUDA(cudaStreamSynchronize(s->stream));
  return PMGPU_OK;
}

void halfpairs_grid(int n, int split, int *tiles, long long *items, int *blocks) {
  static int sms[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  int &m = sms[dev & 63];
  if (m <= 0 && (cudaDeviceGetAttribute(&m, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
                 m <= 0))
    m = 148;
  const int t = (n + 31) / 32;
  *tiles = t;
  *items = (long long)t * (t + 1) / 2 * split;
  *blocks = (int)std::max(1LL, std::min(*items, (long long)m));
}

// The switched all-pairs form (k_simplefull_sw); lj_sw / coul_sw NULL for
// an absent term.  em as nb_simplefull.
int nb_simplefull_sw(System *s, const SwitchParams *lj_sw, const SwitchParams *coul_sw,
                     int em, int scpism, double dielectric) {
  const int n = s->n;
  if (n == 0 || !(lj_sw || coul_sw)) return PMGPU_OK;
  const int iblocks = (n + kSfTile - 1) / kSfTile;
  int chunks = std::max(1, std::min((296 + iblocks - 1) / iblocks, iblocks));
  const int jchunk = ((n + chunks - 1) / chunks + kSfTile - 1) / kSfTile * kSfTile;
  chunks = (n + jchunk - 1) / jchunk;
  SfSwArgs a;
  a.n = n;
  a.jchunk = jchunk;
  a.pos = s->d_pos;
  a.charge = s->d_charge;
  a.type = s->d_type;
  a.mol = s->d_mol;
  a.ntypes = s->ntypes;
  a.lj64 = s->d_lj64;
  a.ex_range = s->d_excl_range;
  a.ex_start = s->d_excl_start;
  a.ex_partner = s->d_excl_partner;
  a.ex_class = s->d_excl_class;
  a.csf = s->coulomb_scaling;
  a.box = s->box;
  SwitchParams none{};
  a.lj_sw = make_switch_dev<double>(lj_sw ? *lj_sw : none);
  a.coul_sw = make_switch_dev<double>(coul_sw ? *coul_sw : none);
  a.lj = lj_sw != nullptr;
  a.coul = coul_sw != nullptr;
  a.modify = (lj_sw && lj_sw->modify) || (coul_sw && coul_sw->modify);
  a.rough2 = std::max(lj_sw ? lj_sw->rough2 : 0.0, coul_sw ? coul_sw->rough2 : 0.0);
  a.force = s->d_force;
  a.acc = s->d_acc;
  a.em = em;
  a.scpism = scpism;
  a.D = dielectric;
  a.sqrtalpha = s->d_scp;  // plane 0 of the SCPISM data
  a.water = s->d_water;
  k_simplefull_sw<<<dim3(iblocks, chunks), kSfTile, 0, s->stream>>>(a);
  PM_CUDA(cudaGetLastError());
  return PMGPU_OK;
}

// ------------------------------------------------ SCPISM Born radii/self
// BornRadii and BornSelf (force/born/BornRadii.h:33-77, force/born/
// BornSelfForce.h:31-118) as two all-pairs passes in FP64, one thread per
// atom visiting every other atom: the first forms each atom's Born radius
// and from it the atom's BornSelf factor and self energy, the second the
// pair forces (each atom keeps its own; energies and virial halved where a
// pair is seen twice).  Pairs are those the reference's OneAtomPair with
// the Cutoff switch evaluates: within the force's cutoff and not fully
// excluded (the exclusion table only for atoms of one molecule).
struct BornArgs {
  int n;
  const double *pos, *charge;
  const int *mol, *water;
  const double *scp;   // [6][n] sqrt(alpha), alpha, zeta, eta, C_i, g_i
  const int *scp_i;    // [3][n] H-bond class, residue, name class
  const int2 *ex_range;
  const int *ex_start, *ex_partner, *ex_class;
  Box box;
  int rsw, ssw;
  double rcut2, scut2, D;
  double *born_q;      // [2][n] BornSelf factor, self energy
  long long *force, *acc;
  int em;
};

// BornSwitch::switchValue / switchDerivative (force/born/BornSwitch.h:33-68).
__device__ __forceinline__ double born_switch(int sw, double r) {
  if (r >= 5.0) return 0.0;
  if (sw == 3) {
    const double f = 1 - .0016 * r * r * r * r;
    return f * f * f * f;
  }
  if (sw == 1) {
    const double f = 1 - .04 * r * r;
    return f * f;
  }
  if (sw == 2) {
    const double f = 1 - 0.008 * r * r * r;
    return f * f * f;
  }
  return 1.0;
}
__device__ __forceinline__ double born_switch_d(int sw, double r) {
  if (r >= 5.0) return 0.0;
  if (sw == 3) {
    const double f = 1 - .0016 * r * r * r * r;
    return -16 * .0016 * r * r * r * f * f * f;
  }
  if (sw == 1) return -0.16 * (1 - 0.04 * r * r) * r;
  if (sw == 2) return -9 * .008 * r * r * (1 - .008 * r * r * r) * (1 - .008 * r * r * r);
  return 0.0;
}

// The polar-hydrogen factor g_p' g_q of atom p against atom q: p a polar
// H, q an acceptor in another residue; g_p' = -0.378 for an HN against an
// O (BornRadii.h:45-58).
__device__ __forceinline__ bool born_polar(const BornArgs &a, int p, int q, double &gg) {
  const int n = a.n;
  if (!(a.scp_i[p] == 1 && a.scp_i[q] == 2 && a.scp_i[n + p] != a.scp_i[n + q])) return false;
  const double gp = (a.scp_i[2 * n + p] == 1 && a.scp_i[2 * n + q] == 2) ? -0.378
                                                                           : a.scp[5 * n + p];
  gg = gp * a.scp[5 * n + q];
  return true;
}

__device__ __forceinline__ int born_excl(const BornArgs &a, int i, int j, int2 er) {
  if (a.mol[i] != a.mol[j] || j < er.x || j > er.y) return PMGPU_EXCL_NONE;
  return excl_class_of(a.ex_start, a.ex_partner, a.ex_class, i, j);
}

constexpr int kBornThreads = 128;
constexpr double kBornPolarE = 0.80;  // the polar H+ exponent (BornRadii.h:51)

__global__ void __launch_bounds__(kBornThreads) k_born_radii(BornArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const int n = a.n;
  const double xi = a.pos[3 * i], yi = a.pos[3 * i + 1], zi = a.pos[3 * i + 2];
  const double eta = a.scp[3 * n + i], C = a.scp[4 * n + i];
  const int2 er = a.ex_range[i];
  const bool wi = a.water && a.water[i];
  double R = a.scp[2 * n + i];  // preForce: the radius starts at zeta
  for (int j = 0; j < n; j++) {
    if (j == i) continue;
    double dx, dy, dz;
    const double r2 = box_mindiff(a.box, xi, yi, zi, a.pos[3 * j], a.pos[3 * j + 1],
                                  a.pos[3 * j + 2], dx, dy, dz);
    if (r2 > a.rcut2) continue;
    if (born_excl(a, i, j, er) == PMGPU_EXCL_FULL) continue;
    if (wi || (a.water && a.water[j])) continue;
    const double dist = sqrt(r2);
    const double f = born_switch(a.rsw, dist);
    R += eta * f * exp(-C * dist);
    double gg;
    if (born_polar(a, i, j, gg)) R += gg * f * exp(-kBornPolarE * dist);
  }
  // BornSelfForce.h:76-88: the solvation factor, its derivative, the
  // atom's force factor and self energy
  const double D = a.D, K = (D - 1.0) / 2, alpha = a.scp[n + i], q = a.charge[i];
  const double Ds = (1.0 + D) / (1 + K * exp(-alpha * R)) - 1.0;
  const double rDs = 1.0 / Ds, rR = 1.0 / R;
  const double dDs = alpha * (1.0 / (1.0 + D)) * (1 + Ds) * (D - Ds);
  a.born_q[i] = -0.5 * q * q * rR * rR * (1.0 - rDs - R * rDs * rDs * dDs);
  a.born_q[n + i] = 0.5 * q * q * rR * (rDs - 1);
}

__global__ void __launch_bounds__(kBornThreads) k_born_self(BornArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < a.n;
  const int n = a.n;
  double fx = 0, fy = 0, fz = 0, e = 0;
  double v[6] = {0, 0, 0, 0, 0, 0};
  if (valid) {
    const double xi = a.pos[3 * i], yi = a.pos[3 * i + 1], zi = a.pos[3 * i + 2];
    const double eta = a.scp[3 * n + i], C = a.scp[4 * n + i], Qi = a.born_q[i];
    const int2 er = a.ex_range[i];
    bool used = false;
    for (int j = 0; j < n; j++) {
      if (j == i) continue;
      double dx, dy, dz;
      const double r2 = box_mindiff(a.box, xi, yi, zi, a.pos[3 * j], a.pos[3 * j + 1],
                                    a.pos[3 * j + 2], dx, dy, dz);
      if (r2 > a.scut2) continue;
      if (born_excl(a, i, j, er) == PMGPU_EXCL_FULL) continue;
      const double dist = sqrt(r2), rDist = 1.0 / dist;
      const double f = born_switch(a.ssw, dist), fp = born_switch_d(a.ssw, dist);
      double gg;
      double dRij = eta * (fp - f * C) * exp(-C * dist);
      if (born_polar(a, i, j, gg)) dRij += gg * (fp - f * kBornPolarE) * exp(-kBornPolarE * dist);
      const double etaj = a.scp[3 * n + j], Cj = a.scp[4 * n + j];
      double dRji = etaj * (fp - f * Cj) * exp(-Cj * dist);
      if (born_polar(a, j, i, gg)) dRji += gg * (fp - f * kBornPolarE) * exp(-kBornPolarE * dist);
      const double force = (Qi * dRij + a.born_q[j] * dRji) * rDist;
      // fij = d force on the pair, F_i -= fij (d = x_j - x_i)
      fx -= dx * force;
      fy -= dy * force;
      fz -= dz * force;
      used = true;
      if (a.em == 2) {
        const double hf = 0.5 * force;
        v[0] += dx * dx * hf; v[1] += dx * dy * hf; v[2] += dx * dz * hf;
        v[3] += dy * dy * hf; v[4] += dy * dz * hf; v[5] += dz * dz * hf;
      }
    }
    // the self energy of every atom that took part in a pair
    // (BornSelfForce.h:108-117, postProcess :128-135)
    if (used) e = a.born_q[n + i];
    red_add(&a.force[i], to_fixed(fx, kForceScale));
    red_add(&a.force[n + i], to_fixed(fy, kForceScale));
    red_add(&a.force[2 * n + i], to_fixed(fz, kForceScale));
  }
  if (!a.em) return;
  e = warp_sum(e);
  if (a.em == 2)
    for (int q = 0; q < 6; q++) v[q] = warp_sum(v[q]);
  if ((threadIdx.x & 31) == 0) {
    red_add(&a.acc[ACC_COULOMB], to_fixed(e, kEnergyScale));
    if (a.em == 2) {
      const int map[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
      for (int q = 0; q < 9; q++)
        red_add(&a.acc[ACC_VIRIAL + q], to_fixed(v[map[q]], kEnergyScale));
    }
  }
}

int nb_born(System *s, const Force &f, int em) {
  const int n = s->n;
  if (n == 0) return PMGPU_OK;
  BornArgs a;
  a.n = n;
  a.pos = s->d_pos;
  a.charge = s->d_charge;
  a.mol = s->d_mol;
  a.water = s->d_water;
  a.scp = s->d_scp;
  a.scp_i = s->d_scp_i;
  a.ex_range = s->d_excl_range;
  a.ex_start = s->d_excl_start;
  a.ex_partner = s->d_excl_partner;
  a.ex_class = s->d_excl_class;
  a.box = s->box;
  a.rsw = f.born_rsw;
  a.ssw = f.born_ssw;
  a.rcut2 = f.born_rcut * f.born_rcut;
  a.scut2 = f.born_scut * f.born_scut;
  a.D = f.scp_D;
  a.born_q = s->d_born_q;
  a.force = s->d_force;
  a.acc = s->d_acc;
  a.em = em;
  const int nb = (n + kBornThreads - 1) / kBornThreads;
  k_born_radii<<<nb, kBornThreads, 0, s->stream>>>(a);
  k_born_self<<<nb, kBornThreads, 0, s->stream>>>(a);
  PM_CUDA(cudaGetLastError());
  return PMGPU_OK;
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
    int tiles, blocks;
    long long items;
    halfpairs_grid(n, 1, &tiles, &items, &blocks);
    PM_CHECK(nb_simplefull_init(s));
    auto go32 = [&](auto kern) {
      kern<<<blocks, kSfWarps * 32, 0, s->stream>>>(
          n, tiles, items, s->d_rec, s->ntypes, s->d_ljab,
          s->d_ljcomb, s->d_lj32, s->d_sf_tile, s->d_sf_bits, (float)s->coulomb_scaling,
          s->d_force, s->d_acc);
    };
    auto by_em = [&](auto k0, auto k1, auto k2) {
      if (em == 0) go32(k0);
      else if (em == 1) go32(k1);
      else go32(k2);
    };
    const bool comb = s->d_ljcomb != nullptr;
    if (lj && coul) {
      if (comb) by_em(k_simplefull_half<true, true, true, 0>, k_simplefull_half<true, true, true, 1>,
                      k_simplefull_half<true, true, true, 2>);
      else by_em(k_simplefull_half<true, true, false, 0>, k_simplefull_half<true, true, false, 1>,
                 k_simplefull_half<true, true, false, 2>);
    } else if (lj) {
      if (comb) by_em(k_simplefull_half<true, false, true, 0>,
                      k_simplefull_half<true, false, true, 1>,
                      k_simplefull_half<true, false, true, 2>);
      else by_em(k_simplefull_half<true, false, false, 0>, k_simplefull_half<true, false, false, 1>,
                 k_simplefull_half<true, false, false, 2>);
    } else {
      by_em(k_simplefull_half<false, true, false, 0>, k_simplefull_half<false, true, false, 1>,
            k_simplefull_half<false, true, false, 2>);
    }
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
