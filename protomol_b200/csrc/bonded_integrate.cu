// Harmonic bonds and angles (FP64), the device-resident leapfrog and
// Langevin-leapfrog updates (FP64), and fixed-point force conversion.
#include <cmath>

#include "pm_device.cuh"

namespace pmgpu {

// BondSystemForce::calcBond (force/bonded/BondSystemForce.h:89-124).
__device__ __forceinline__ void bond_term(int b, const Box &box, int nb,
                                          const int *__restrict__ atoms,
                                          const double *__restrict__ prm,
                                          const double *__restrict__ pos, int n,
                                          long long *__restrict__ force,
                                          long long *__restrict__ acc, int em) {
  double e = 0, v[6] = {0, 0, 0, 0, 0, 0};
  if (b < nb) {
    int a1 = atoms[2 * b], a2 = atoms[2 * b + 1];
    double k = prm[2 * b], r0 = prm[2 * b + 1];
    double dx, dy, dz;
    // r12 = minimalDifference(atom2, atom1): vector from atom 2 to atom 1
    box_mindiff(box, pos[3 * a2], pos[3 * a2 + 1], pos[3 * a2 + 2], pos[3 * a1],
                pos[3 * a1 + 1], pos[3 * a1 + 2], dx, dy, dz);
    double r = sqrt(dx * dx + dy * dy + dz * dz);
    double dp = 2.0 * k * (r - r0);
    double g = -dp / r;
    double fx = dx * g, fy = dy * g, fz = dz * g;
    red_add(&force[a1], to_fixed(fx, kForceScale));
    red_add(&force[n + a1], to_fixed(fy, kForceScale));
    red_add(&force[2 * n + a1], to_fixed(fz, kForceScale));
    red_add(&force[a2], to_fixed(-fx, kForceScale));
    red_add(&force[n + a2], to_fixed(-fy, kForceScale));
    red_add(&force[2 * n + a2], to_fixed(-fz, kForceScale));
    e = k * (r - r0) * (r - r0);
    if (em == 2) {
      v[0] = fx * dx; v[1] = fx * dy; v[2] = fx * dz;
      v[3] = fy * dy; v[4] = fy * dz; v[5] = fz * dz;
    }
  }
  if (!em) return;
  e = warp_sum(e);
  if (em == 2)
    for (int q = 0; q < 6; q++) v[q] = warp_sum(v[q]);
  if ((threadIdx.x & 31) == 0) {
    red_add(&acc[ACC_BOND], to_fixed(e, kEnergyScale));
    if (em == 2) {
      const int map[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
      for (int q = 0; q < 9; q++) red_add(&acc[ACC_VIRIAL + q], to_fixed(v[map[q]], kEnergyScale));
    }
  }
}

// AngleSystemForce::calcAngle (force/bonded/AngleSystemForce.h:86-171),
// harmonic angle plus Urey-Bradley.
__device__ __forceinline__ void angle_term(int t, const Box &box, int na,
                                           const int *__restrict__ atoms,
                                           const double *__restrict__ prm,
                                           const double *__restrict__ pos, int n,
                                           long long *__restrict__ force,
                                           long long *__restrict__ acc, int em) {
  double e = 0, v[6] = {0, 0, 0, 0, 0, 0};
  if (t < na) {
    int a1 = atoms[3 * t], a2 = atoms[3 * t + 1], a3 = atoms[3 * t + 2];
    double kt = prm[4 * t], t0 = prm[4 * t + 1], kub = prm[4 * t + 2], rub = prm[4 * t + 3];
    double r12[3], r32[3], r13[3];
    box_mindiff(box, pos[3 * a2], pos[3 * a2 + 1], pos[3 * a2 + 2], pos[3 * a1],
                pos[3 * a1 + 1], pos[3 * a1 + 2], r12[0], r12[1], r12[2]);
    box_mindiff(box, pos[3 * a2], pos[3 * a2 + 1], pos[3 * a2 + 2], pos[3 * a3],
                pos[3 * a3 + 1], pos[3 * a3 + 2], r32[0], r32[1], r32[2]);
    box_mindiff(box, pos[3 * a3], pos[3 * a3 + 1], pos[3 * a3 + 2], pos[3 * a1],
                pos[3 * a1 + 1], pos[3 * a1 + 2], r13[0], r13[1], r13[2]);
    double d12 = sqrt(r12[0] * r12[0] + r12[1] * r12[1] + r12[2] * r12[2]);
    double d32 = sqrt(r32[0] * r32[0] + r32[1] * r32[1] + r32[2] * r32[2]);
    double d13 = sqrt(r13[0] * r13[0] + r13[1] * r13[1] + r13[2] * r13[2]);
    double cx = r12[1] * r32[2] - r12[2] * r32[1];
    double cy = r12[2] * r32[0] - r12[0] * r32[2];
    double cz = r12[0] * r32[1] - r12[1] * r32[0];
    double theta = atan2(sqrt(cx * cx + cy * cy + cz * cz),
                         r12[0] * r32[0] + r12[1] * r32[1] + r12[2] * r32[2]);
    double st = sin(theta), ct = cos(theta);
    double dpdt = 2.0 * kt * (theta - t0);
    double f1[3], f3[3];
    double ub = 2.0 * kub * (d13 - rub);
    for (int c = 0; c < 3; c++) {
      double dr12 = r12[c] / d12, dr32 = r32[c] / d32, dr13 = r13[c] / d13;
      double dth1 = (dr12 * ct - dr32) / (st * d12);
      double dth3 = (dr32 * ct - dr12) / (st * d32);
      double ub1 = dr13 * ub;
      f1[c] = -dth1 * dpdt - ub1;
      f3[c] = -dth3 * dpdt + ub1;
    }
    for (int c = 0; c < 3; c++) {
      red_add(&force[c * n + a1], to_fixed(f1[c], kForceScale));
      red_add(&force[c * n + a3], to_fixed(f3[c], kForceScale));
      red_add(&force[c * n + a2], to_fixed(-f1[c] - f3[c], kForceScale));
    }
    e = kt * (theta - t0) * (theta - t0) + kub * (d13 - rub) * (d13 - rub);
    if (em == 2) {
      v[0] = f1[0] * r12[0] + f3[0] * r32[0];
      v[1] = f1[0] * r12[1] + f3[0] * r32[1];
      v[2] = f1[0] * r12[2] + f3[0] * r32[2];
      v[3] = f1[1] * r12[1] + f3[1] * r32[1];
      v[4] = f1[1] * r12[2] + f3[1] * r32[2];
      v[5] = f1[2] * r12[2] + f3[2] * r32[2];
    }
  }
  if (!em) return;
  e = warp_sum(e);
  if (em == 2)
    for (int q = 0; q < 6; q++) v[q] = warp_sum(v[q]);
  if ((threadIdx.x & 31) == 0) {
    red_add(&acc[ACC_ANGLE], to_fixed(e, kEnergyScale));
    if (em == 2) {
      const int map[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
      for (int q = 0; q < 9; q++) red_add(&acc[ACC_VIRIAL + q], to_fixed(v[map[q]], kEnergyScale));
    }
  }
}

__device__ __forceinline__ void dcross(const double *u, const double *v, double *o) {
  o[0] = u[1] * v[2] - u[2] * v[1];
  o[1] = u[2] * v[0] - u[0] * v[2];
  o[2] = u[0] * v[1] - u[1] * v[0];
}
__device__ __forceinline__ double ddot(const double *u, const double *v) {
  return u[0] * v[0] + u[1] * v[1] + u[2] * v[2];
}

// MTorsionSystemForce::calcTorsion (force/bonded/MTorsionSystemForce.h:40-204),
// one term per thread: the dihedral angle from the normals of the (1,2,3)
// and (2,3,4) planes; the gradient goes through d cos(phi) when
// |sin phi| > 0.1 and through d sin(phi) otherwise.  params: k,
// periodicity n, phase delta; n > 0 cosine form, n == 0 harmonic.
__device__ __forceinline__ void torsion_term(int t, const Box &box, int nt,
                                             const int *__restrict__ atoms,
                                             const double *__restrict__ prm,
                                             const double *__restrict__ pos, int n,
                                             long long *__restrict__ force,
                                             long long *__restrict__ acc, int slot, int em) {
  double e = 0, v[6] = {0, 0, 0, 0, 0, 0};
  if (t < nt) {
    const int a1 = atoms[4 * t], a2 = atoms[4 * t + 1], a3 = atoms[4 * t + 2],
              a4 = atoms[4 * t + 3];
    const double k = prm[3 * t], delta = prm[3 * t + 2];
    const int per = (int)prm[3 * t + 1];
    double r12[3], r23[3], r34[3];
    box_mindiff(box, pos[3 * a2], pos[3 * a2 + 1], pos[3 * a2 + 2], pos[3 * a1],
                pos[3 * a1 + 1], pos[3 * a1 + 2], r12[0], r12[1], r12[2]);
    box_mindiff(box, pos[3 * a3], pos[3 * a3 + 1], pos[3 * a3 + 2], pos[3 * a2],
                pos[3 * a2 + 1], pos[3 * a2 + 2], r23[0], r23[1], r23[2]);
    box_mindiff(box, pos[3 * a4], pos[3 * a4 + 1], pos[3 * a4 + 2], pos[3 * a3],
                pos[3 * a3 + 1], pos[3 * a3 + 2], r34[0], r34[1], r34[2]);
    double na[3], nb[3], nc[3];
    dcross(r12, r23, na);
    dcross(r23, r34, nb);
    dcross(r23, na, nc);
    const double ia = 1.0 / sqrt(ddot(na, na)), ib = 1.0 / sqrt(ddot(nb, nb)),
                 ic = 1.0 / sqrt(ddot(nc, nc));
    for (int c = 0; c < 3; c++) {
      na[c] *= ia;
      nb[c] *= ib;
      nc[c] *= ic;
    }
    const double cphi = ddot(na, nb), sphi = ddot(nc, nb);
    const double phi = -atan2(sphi, cphi);
    double dvdphi;
    if (per > 0) {
      dvdphi = -per * k * sin(per * phi + delta);
      e = k * (1.0 + cos(per * phi + delta));
    } else {
      double diff = phi - delta;
      if (diff < -M_PI) diff += 2 * M_PI;
      else if (diff > M_PI) diff -= 2 * M_PI;
      dvdphi = 2.0 * k * diff;
      e = k * diff * diff;
    }
    double f1[3], f2[3], f3[3], t1[3], t2[3];
    if (fabs(sphi) > 0.1) {
      double ga[3], gb[3];
      const double g = dvdphi / sphi;
      for (int c = 0; c < 3; c++) {
        ga[c] = (na[c] * cphi - nb[c]) * ia;
        gb[c] = (nb[c] * cphi - na[c]) * ib;
      }
      dcross(r23, ga, t1);
      dcross(gb, r23, t2);
      for (int c = 0; c < 3; c++) {
        f1[c] = g * t1[c];
        f3[c] = g * t2[c];
      }
      dcross(ga, r12, t1);
      dcross(r34, gb, t2);
      for (int c = 0; c < 3; c++) f2[c] = g * (t1[c] + t2[c]);
    } else {
      double gc[3], gb[3];
      const double g = -dvdphi / cphi;
      for (int c = 0; c < 3; c++) {
        gc[c] = (nc[c] * sphi - nb[c]) * ic;
        gb[c] = (nb[c] * sphi - nc[c]) * ib;
      }
      const double r23sq = ddot(r23, r23), r23gc = ddot(r23, gc);
      for (int c = 0; c < 3; c++) f1[c] = g * (r23sq * gc[c] - r23[c] * r23gc);
      dcross(gb, r23, t1);
      for (int c = 0; c < 3; c++) f3[c] = g * t1[c];
      for (int c = 0; c < 3; c++) {
        const int c1 = (c + 1) % 3, c2 = (c + 2) % 3;
        f2[c] = g * (-(r23[c1] * r12[c1] + r23[c2] * r12[c2]) * gc[c] +
                     (2.0 * r23[c] * r12[c1] - r12[c] * r23[c1]) * gc[c1] +
                     (2.0 * r23[c] * r12[c2] - r12[c] * r23[c2]) * gc[c2] +
                     gb[c2] * r34[c1] - gb[c1] * r34[c2]);
      }
    }
    for (int c = 0; c < 3; c++) {
      red_add(&force[c * n + a1], to_fixed(f1[c], kForceScale));
      red_add(&force[c * n + a2], to_fixed(f2[c] - f1[c], kForceScale));
      red_add(&force[c * n + a3], to_fixed(f3[c] - f2[c], kForceScale));
      red_add(&force[c * n + a4], to_fixed(-f3[c], kForceScale));
    }
    if (em == 2) {
      // upper triangle (xx, xy, xz, yy, yz, zz), mirrored below
      int q = 0;
      for (int i = 0; i < 3; i++)
        for (int j = i; j < 3; j++) v[q++] = f1[i] * r12[j] + f2[i] * r23[j] + f3[i] * r34[j];
    }
  }
  if (!em) return;
  e = warp_sum(e);
  if (em == 2)
    for (int q = 0; q < 6; q++) v[q] = warp_sum(v[q]);
  if ((threadIdx.x & 31) == 0) {
    red_add(&acc[slot], to_fixed(e, kEnergyScale));
    if (em == 2) {
      const int map[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
      for (int q = 0; q < 9; q++) red_add(&acc[ACC_VIRIAL + q], to_fixed(v[map[q]], kEnergyScale));
    }
  }
}

// All bonded terms of an evaluation in one launch: whole 128-thread blocks
// of bonds, then angles, dihedrals and impropers, so every warp holds one
// kind of term (its energy reduction stays per warp).
constexpr int kBondedThreads = 128;
struct BondedLaunch {
  int nb, na, nd, ni;          // terms of each kind in this launch (0: none)
  int bb, ab, db;              // blocks of bonds, angles, dihedrals
};

struct BondedArgs {
  BondedLaunch L;
  Box box;
  const int *bond_atoms;
  const double *bond_prm;
  const int *angle_atoms;
  const double *angle_prm;
  const int *dih_atoms;
  const double *dih_prm;
  const int *imp_atoms;
  const double *imp_prm;
  const double *pos;
  int n;
  long long *force, *acc;
  int em;
};

__device__ __forceinline__ void bonded_body(const BondedArgs &A, Blk b) {
  const BondedLaunch &L = A.L;
  const Box &box = A.box;
  const int n = A.n, em = A.em;
  const double *__restrict__ pos = A.pos;
  long long *__restrict__ force = A.force;
  long long *__restrict__ acc = A.acc;
  const int *__restrict__ bond_atoms = A.bond_atoms;
  const double *__restrict__ bond_prm = A.bond_prm;
  const int *__restrict__ angle_atoms = A.angle_atoms;
  const double *__restrict__ angle_prm = A.angle_prm;
  const int *__restrict__ dih_atoms = A.dih_atoms;
  const double *__restrict__ dih_prm = A.dih_prm;
  const int *__restrict__ imp_atoms = A.imp_atoms;
  const double *__restrict__ imp_prm = A.imp_prm;
  int blk = b.x;
  if (blk < L.bb) {
    bond_term(blk * kBondedThreads + threadIdx.x, box, L.nb, bond_atoms, bond_prm, pos, n,
              force, acc, em);
    return;
  }
  blk -= L.bb;
  if (blk < L.ab) {
    angle_term(blk * kBondedThreads + threadIdx.x, box, L.na, angle_atoms, angle_prm, pos, n,
               force, acc, em);
    return;
  }
  blk -= L.ab;
  if (blk < L.db) {
    torsion_term(blk * kBondedThreads + threadIdx.x, box, L.nd, dih_atoms, dih_prm, pos, n,
                 force, acc, ACC_DIHEDRAL, em);
    return;
  }
  blk -= L.db;
  torsion_term(blk * kBondedThreads + threadIdx.x, box, L.ni, imp_atoms, imp_prm, pos, n, force,
               acc, ACC_IMPROPER, em);
}

__global__ void __launch_bounds__(kBondedThreads) k_bonded(BondedArgs a) {
  bonded_body(a, own_blk());
}

__global__ void __launch_bounds__(kBondedThreads)
k_bonded_batch(const BondedArgs *__restrict__ tab, const int *__restrict__ first, int nm) {
  const int m = batch_member(first, nm, blockIdx.x);
  bonded_body(tab[m], batch_blk(first, m));
}

// The bonded terms' launch arguments of a system (blocks: its grid size).
static BondedArgs bonded_args(System *s, int bonds, int angles, int dihedrals, int impropers,
                              int em, int *blocks) {
  BondedArgs a;
  BondedLaunch &L = a.L;
  L.nb = bonds ? s->n_bonds : 0;
  L.na = angles ? s->n_angles : 0;
  L.nd = dihedrals ? s->n_dihedrals : 0;
  L.ni = impropers ? s->n_impropers : 0;
  auto nbk = [](int k) { return (k + kBondedThreads - 1) / kBondedThreads; };
  L.bb = nbk(L.nb);
  L.ab = nbk(L.na);
  L.db = nbk(L.nd);
  *blocks = L.bb + L.ab + L.db + nbk(L.ni);
  a.box = s->box;
  a.bond_atoms = s->d_bond_atoms;
  a.bond_prm = s->d_bond_params;
  a.angle_atoms = s->d_angle_atoms;
  a.angle_prm = s->d_angle_params;
  a.dih_atoms = s->d_dihedral_atoms;
  a.dih_prm = s->d_dihedral_params;
  a.imp_atoms = s->d_improper_atoms;
  a.imp_prm = s->d_improper_params;
  a.pos = s->d_pos;
  a.n = s->n;
  a.force = s->d_force;
  a.acc = s->d_acc;
  a.em = em;
  return a;
}

int bonded_all(System *s, int bonds, int angles, int dihedrals, int impropers, int em,
               int *launched) {
  int total = 0;
  const BondedArgs a = bonded_args(s, bonds, angles, dihedrals, impropers, em, &total);
  *launched = total > 0;
  if (!total) return PMGPU_OK;
  k_bonded<<<total, kBondedThreads, 0, s->stream>>>(a);
  PM_CUDA(cudaGetLastError());
  return PMGPU_OK;
}

int zero_forces(System *s) {
  // a slot buffer still pending holds stale pair forces: fold (and clear) it
  // before the forces are zeroed, so the next pair launch starts from zero
  PM_CHECK(fold_pending_slots(s));
  PM_CUDA(cudaMemsetAsync(s->d_force, 0, sizeof(long long) * 3 * (size_t)s->n, s->stream));
  return PMGPU_OK;
}

// ------------------------------------------------------------------ RNG
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC'11): counter-based, so the Langevin noise of atom i
// at half-kick h of step s is a pure function of (seed, s, h, i) and can be
// replayed or checkpointed by the step counter alone.
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; r++) {
    uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
    uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    k.x += W0;
    k.y += W1;
  }
  return c;
}

__device__ __forceinline__ float u01f(uint32_t a) {
  // 24-bit uniform in (0, 1]
  return (float)((a >> 8) + 1u) * (1.0f / 16777216.0f);
}

// Three standard normal variates for (atom, step, half) from one Philox
// block: Box-Muller on two uniform pairs, in FP32 (the variates scale the
// FP64 velocity update; 24-bit uniforms bound them at 5.8 sigma).
__device__ __forceinline__ void gauss3(uint64_t seed, uint64_t step, int half, int atom,
                                       double g[3]) {
  const uint4 c = make_uint4((uint32_t)atom, (uint32_t)step, (uint32_t)(step >> 32),
                             (uint32_t)half);
  const uint2 k = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
  const uint4 r = philox4x32_10(c, k);
  float s, co;
  const float rad = sqrtf(-2.0f * logf(u01f(r.x)));
  sincospif(2.0f * u01f(r.y), &s, &co);
  g[0] = (double)(rad * co);
  g[1] = (double)(rad * s);
  const float rad2 = sqrtf(-2.0f * logf(u01f(r.z)));
  g[2] = (double)(rad2 * cospif(2.0f * u01f(r.w)));
}

// ------------------------------------------------------------ integrator
struct UpdateArgs {
  int n;
  int kicks;          // 0, 1 or 2 kicks with the resident forces
  int langevin;
  double coef;        // leapfrog: kick coefficient (h or h/2)
  double h;           // drift step (timestep * INV_TIMEFACTOR)
  int drift;
  int zero_force;
  // Langevin (LangevinLeapfrogIntegrator.cpp:44-71)
  double vdt, fdt, ndt, fc;
  uint64_t seed;
  // (step, half) of each kick's noise: step = step_ptr[0] + kstep_off[k].  The
  // step counter lives in device memory so captured graphs stay valid; with
  // step_inc the last block of the launch advances it (step_ptr[1] counts
  // the blocks done).
  unsigned long long *step_ptr;
  int step_inc;
  int kstep_off[2];
  int khalf[2];
  long long *acc_zero;  // energy accumulators cleared by this launch (or null)
  // the pair list's rebuild decision from the drifted positions (xbuild null:
  // none); see rebuild_decide
  const double *xbuild;
  unsigned *ticket;
  int *rebuild;
  float half_skin2;
  // the FP32 pair records of the drifted positions (null: none)
  float4 *rec;
  const double *charge;
  const int *type;
  // the pair list's slot-ordered force buffer left by a force-only step
  // (null: none): added into the forces here and cleared
  long long *fslot;
  const int *slot_of;
  int ns;
  // the pair list's slot records of the drifted positions (xw null: none),
  // written through the current slot order: the list's gather then only
  // redoes them when the list is rebuilt
  double4 *xw;
  float4 *xhi, *xlo;
  const double *offset;
  int mixed;
  // the system's state
  const double *mass;
  double *pos, *vel;
  long long *force;
  int *status;
};

__global__ void k_step_set(unsigned long long *step, unsigned long long v) { *step = v; }

int set_device_step(System *s) {
  k_step_set<<<1, 1, 0, s->stream>>>(s->d_step, (unsigned long long)s->step);
  PM_CUDA(cudaGetLastError());
  return PMGPU_OK;
}

constexpr int kUpdateThreads = 64;  // small blocks: the update is latency-bound FP64 work
__device__ __forceinline__ void update_body(const UpdateArgs &a, Blk blk) {
  const double *__restrict__ mass = a.mass;
  double *__restrict__ pos = a.pos;
  double *__restrict__ vel = a.vel;
  long long *__restrict__ force = a.force;
  int *__restrict__ status = a.status;
  const int i = blk.x * blockDim.x + threadIdx.x;
  const bool valid = i < a.n;
  float d2 = 0.f;
  double v[3] = {0, 0, 0}, x[3] = {0, 0, 0};
  long long Fx[3] = {0, 0, 0};
  int slot = -1;
  if (valid) {
    for (int c = 0; c < 3; c++) Fx[c] = force[c * a.n + i];
    if (a.fslot) {
      slot = a.slot_of[i];
      if (slot >= 0)
        for (int c = 0; c < 3; c++) Fx[c] += a.fslot[(size_t)c * a.ns + slot];
    }
    double F[3];
    for (int c = 0; c < 3; c++) F[c] = (double)Fx[c] * (1.0 / kForceScale);
    double m = mass[i];
    for (int c = 0; c < 3; c++) v[c] = vel[3 * i + c];
    for (int k = 0; k < a.kicks; k++) {
      if (a.langevin) {
        double g[3];
        gauss3(a.seed, *a.step_ptr + (long long)a.kstep_off[k], a.khalf[k], i, g);
        double sq = sqrt(a.fc / m);
        for (int c = 0; c < 3; c++)
          v[c] = xadd(xadd(xmul(v[c], a.vdt), xmul(F[c], a.fdt) / m),
                      xmul(xmul(g[c], sq), a.ndt));
      } else {
        // StandardIntegrator::doHalfKick / LeapfrogIntegrator::doKickdoDrift
        for (int c = 0; c < 3; c++) v[c] = xadd(v[c], xmul(F[c], a.coef) / m);
      }
    }
    if (a.drift) {
      double dd = 0.0;
      for (int c = 0; c < 3; c++) {
        x[c] = xadd(pos[3 * i + c], xmul(v[c], a.h));
        if (a.xbuild) {
          const double e = x[c] - a.xbuild[3 * i + c];
          dd += e * e;
        }
      }
      d2 = (float)dd;
    }
  }
  // The grid-wide decisions come before this thread's stores, so the fences
  // they take wait for no stores of the update.
  // with a rebuild decision to take, the step counter advances on its
  // ticket (one grid-wide ticket instead of two)
  if (a.xbuild)
    rebuild_decide<kUpdateThreads>(d2, a.ticket, a.rebuild, a.half_skin2, 0, blk.n,
                                   a.step_inc ? a.step_ptr : nullptr);
  if (a.step_inc && !a.xbuild) {
    // every block has read the counter before it counts itself done
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      last = atomicAdd(&a.step_ptr[1], 1ull) == (unsigned long long)blk.n - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
      a.step_ptr[1] = 0ull;
      a.step_ptr[0] += 1ull;
    }
  }
  if (a.acc_zero && i < ACC_COUNT) a.acc_zero[i] = 0;
  if (!valid) return;
  for (int c = 0; c < 3; c++) vel[3 * i + c] = v[c];
  if (a.drift) {
    for (int c = 0; c < 3; c++) {
      pos[3 * i + c] = x[c];
      if (!isfinite(x[c])) atomicOr(status, ST_NONFINITE);
    }
    if (a.rec) write_pair_record(a.rec, a.n, i, x[0], x[1], x[2], a.charge[i], a.type[i]);
    if (a.xw && slot >= 0) {
      // the wrapped position x - (x_build - x_wrapped at the build), as the
      // gather forms it, and its FP32 hi/lo split
      const double wx = x[0] - a.offset[3 * i], wy = x[1] - a.offset[3 * i + 1],
                   wz = x[2] - a.offset[3 * i + 2];
      const double q = a.charge[i];
      a.xw[slot] = make_double4(wx, wy, wz, q);
      const float hx = (float)wx, hy = (float)wy, hz = (float)wz;
      a.xhi[slot] = make_float4(hx, hy, hz, (float)q);
      if (a.mixed)
        a.xlo[slot] = make_float4((float)(wx - (double)hx), (float)(wy - (double)hy),
                                  (float)(wz - (double)hz), __int_as_float(a.type[i]));
    }
  }
  if (slot >= 0)
    for (int c = 0; c < 3; c++) a.fslot[(size_t)c * a.ns + slot] = 0;
  if (a.zero_force)
    for (int c = 0; c < 3; c++) force[c * a.n + i] = 0;
  else if (a.fslot)
    for (int c = 0; c < 3; c++) force[c * a.n + i] = Fx[c];
}

__global__ void __launch_bounds__(kUpdateThreads) k_update(UpdateArgs a) {
  pdl_trigger();  // the list kernels after it may launch; they wait for this grid
  update_body(a, own_blk());
}

__global__ void __launch_bounds__(kUpdateThreads)
k_update_batch(const UpdateArgs *__restrict__ tab, const int *__restrict__ first, int nm) {
  const int m = batch_member(first, nm, blockIdx.x);
  update_body(tab[m], batch_blk(first, m));
}

// phase: 0 = leapfrog first (half kick + drift), 1 = leapfrog middle (kick +
// drift), 2 = leapfrog last (half kick), 3 = Langevin half kick + drift,
// 4 = Langevin two half kicks (end of step s, start of step s+1) + drift,
// 5 = Langevin closing half kick.
int update_args(System *s, const pmgpu_integrator *it, int phase, int zero_acc,
                NeighborList *list, UpdateArgs *out) {
  UpdateArgs &a = *out;
  a.n = s->n;
  a.h = it->timestep_fs * kInvTimeFactor;
  a.langevin = it->kind == PMGPU_INT_LANGEVIN_LEAPFROG;
  a.seed = it->seed;
  // StandardIntegrator::run gives every step two half kicks; the noise of
  // kick (step, half) is Philox(seed; atom, step, half).
  a.step_ptr = s->d_step;
  // only the Langevin noise reads the device step counter (every run sets
  // it from the host counter first); it advances after the drift of a step
  a.step_inc = a.langevin && s->n > 0;
  a.acc_zero = zero_acc ? s->d_acc : nullptr;
  a.xbuild = nullptr;
  a.ticket = nullptr;
  a.rebuild = nullptr;
  a.half_skin2 = 0.f;
  a.kstep_off[0] = 0; a.khalf[0] = 0;
  a.kstep_off[1] = 0; a.khalf[1] = 0;
  a.vdt = a.fdt = a.ndt = a.fc = 0;
  if (a.langevin) {
    double gamma = it->gamma_ps / (1000 * kInvTimeFactor);
    double dt = a.h;
    a.fdt = (1.0 - exp(-0.5 * gamma * dt)) / gamma;
    a.vdt = exp(-0.5 * gamma * dt);
    a.ndt = sqrt((1.0 - exp(-gamma * dt)) / (2.0 * gamma));
    a.fc = 2 * kBoltzmann * it->temperature * gamma;
  }
  switch (phase) {
    case 0: a.kicks = 1; a.coef = 0.5 * a.h; a.drift = 1; a.zero_force = 1; break;
    case 1: a.kicks = 1; a.coef = a.h; a.drift = 1; a.zero_force = 1; break;
    case 2: a.kicks = 1; a.coef = 0.5 * a.h; a.drift = 0; a.zero_force = 0; break;
    case 3:  // first half kick of step st, drift
      a.kicks = 1; a.coef = 0; a.drift = 1; a.zero_force = 1;
      break;
    case 4:  // second half kick of step st-1, first half kick of step st
      a.kicks = 2; a.coef = 0; a.drift = 1; a.zero_force = 1;
      a.kstep_off[0] = -1; a.khalf[0] = 1;
      break;
    case 5:  // second half kick of step st-1
      a.kicks = 1; a.coef = 0; a.drift = 0; a.zero_force = 0;
      a.kstep_off[0] = -1; a.khalf[0] = 1;
      break;
    default: return fail(PMGPU_ERR_ARG, "bad integrator phase");
  }
  a.step_inc = a.step_inc && a.drift;
  // the pair records of the all-pairs passes, from the drifted positions
  a.rec = a.drift && s->d_rec && s->precision == PMGPU_PREC_MIXED ? s->d_rec : nullptr;
  a.charge = s->d_charge;
  a.type = s->d_type;
  s->rec_fresh = a.rec != nullptr;
  a.fslot = nullptr;
  a.slot_of = nullptr;
  a.ns = 0;
  a.xw = nullptr;
  a.xhi = a.xlo = nullptr;
  a.offset = nullptr;
  a.mixed = s->precision == PMGPU_PREC_MIXED;
  if (list && list->built && s->n) {
    a.fslot = list->d_fslot;
    a.slot_of = list->d_slot_of;
    a.ns = list->ns_max;
    list->slot_pending = 0;  // this launch adds the slot buffer and clears it
  }
  if (list && list->built && a.drift && s->n) {
    const float hs = (float)(0.5 * list->skin);
    a.xbuild = list->d_xbuild;
    a.ticket = list->d_maxdisp;
    a.rebuild = list->d_rebuild;
    a.half_skin2 = hs * hs;
    a.xw = list->d_xw;
    a.xhi = list->d_xhi;
    a.xlo = list->d_xlo;
    a.offset = list->d_offset;
    list->decided = 1;  // the decision and the slot records of this step are taken
  }
  a.mass = s->d_mass;
  a.pos = s->d_pos;
  a.vel = s->d_vel;
  a.force = s->d_force;
  a.status = s->d_status;
  return PMGPU_OK;
}

int update_blocks(const System *s) { return (s->n + kUpdateThreads - 1) / kUpdateThreads; }

int integrate_kick_drift(System *s, const pmgpu_integrator *it, int phase, int zero_acc,
                         NeighborList *list) {
  UpdateArgs a;
  PM_CHECK(update_args(s, it, phase, zero_acc, list, &a));
  if (s->n)
    k_update<<<update_blocks(s), kUpdateThreads, 0, s->stream>>>(a);
  PM_CUDA(cudaGetLastError());
  return PMGPU_OK;
}

__global__ void k_forces_to_aos(int n, const long long *__restrict__ force,
                                double *__restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int c = 0; c < 3; c++) out[3 * i + c] = (double)force[c * n + i] * (1.0 / kForceScale);
}

int forces_to_host(System *s, double *out, int add) {
  int n = s->n;
  if (n == 0) return PMGPU_OK;
  // pair forces a force-only step left in a slot buffer belong to d_force
  PM_CHECK(fold_pending_slots(s));
  double *d_tmp = nullptr;
  PM_CUDA(cudaMallocAsync(&d_tmp, sizeof(double) * 3 * n, s->stream));
  k_forces_to_aos<<<(n + 255) / 256, 256, 0, s->stream>>>(n, s->d_force, d_tmp);
  std::vector<double> h(3 * (size_t)n);
  cudaError_t e1 = cudaMemcpyAsync(h.data(), d_tmp, sizeof(double) * 3 * n,
                                   cudaMemcpyDeviceToHost, s->stream);
  cudaFreeAsync(d_tmp, s->stream);
  cudaError_t e2 = cudaStreamSynchronize(s->stream);
  if (e1 != cudaSuccess || e2 != cudaSuccess)
    return fail(PMGPU_ERR_CUDA, std::string("force download: ") +
                                    cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
  if (add)
    for (size_t k = 0; k < h.size(); k++) out[k] += h[k];
  else
    for (size_t k = 0; k < h.size(); k++) out[k] = h[k];
  return PMGPU_OK;
}

// ---------------------------------------------------------------- batches
// The update kernel (every phase of an integrator) and the bonded terms of
// an ensemble's members as batched launches.
struct BdBatch {
  BatchTable<UpdateArgs> upd[6][2];  // [phase][clears the accumulators]
  BatchTable<BondedArgs> bonded[2];  // [energies]
  pmgpu_integrator key{};
};

BdBatch *bd_batch_new() { return new BdBatch(); }
void bd_batch_free(BdBatch *b) {
  if (!b) return;
  for (auto &p : b->upd)
    for (auto &t : p) t.release();
  for (auto &t : b->bonded) t.release();
  delete b;
}

// Update tables of integrator it for every phase (with and without the
// accumulator clear) and the bonded tables.  Builds host-side flags as
// integrate_kick_drift would, so a member's list state matches.
int bd_batch_build(BdBatch *b, System *const *m, int n, const pmgpu_integrator *it,
                   const int *bd_flags) {
  b->key = *it;
  const int first_phase = it->kind == PMGPU_INT_LANGEVIN_LEAPFROG ? 3 : 0;
  for (int ph = 0; ph < 6; ph++)
    for (int z = 0; z < 2; z++) {
      BatchTable<UpdateArgs> &t = b->upd[ph][z];
      t.clear();
      if (ph < first_phase || ph >= first_phase + 3) continue;
      for (int k = 0; k < n; k++) {
        UpdateArgs a;
        // update_args marks the list as decided and its slot buffer as taken;
        // those flags are set again by every step of the batched run
        PM_CHECK(update_args(m[k], it, ph, z, &m[k]->lists[0], &a));
        t.add(a, update_blocks(m[k]));
      }
      PM_CUDA(t.upload());
    }
  for (int e = 0; e < 2; e++) {
    BatchTable<BondedArgs> &t = b->bonded[e];
    t.clear();
    for (int k = 0; k < n; k++) {
      int blocks = 0;
      const int *f = bd_flags + 4 * k;
      const BondedArgs a = bonded_args(m[k], f[0], f[1], f[2], f[3], e, &blocks);
      t.add(a, blocks);
    }
    PM_CUDA(t.upload());
  }
  return PMGPU_OK;
}

int bd_batch_update(BdBatch *b, int phase, int zero_acc, cudaStream_t st, long long *launched) {
  BatchTable<UpdateArgs> &t = b->upd[phase][zero_acc ? 1 : 0];
  if (!t.members() || !t.total()) return PMGPU_OK;
  *launched += 1;
  k_update_batch<<<t.total(), kUpdateThreads, 0, st>>>(t.d, t.d_first, t.members());
  PM_CUDA(cudaGetLastError());
  return PMGPU_OK;
}

int bd_batch_bonded(BdBatch *b, int em, cudaStream_t st, long long *launched) {
  BatchTable<BondedArgs> &t = b->bonded[em ? 1 : 0];
  if (!t.members() || !t.total()) return PMGPU_OK;
  *launched += 1;
  k_bonded_batch<<<t.total(), kBondedThreads, 0, st>>>(t.d, t.d_first, t.members());
  PM_CUDA(cudaGetLastError());
  return PMGPU_OK;
}

}  // namespace pmgpu
