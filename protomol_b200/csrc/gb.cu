// OBC generalized Born in the vacuum all-pairs form:
//   GBBornRadii  (force/GB/GBBornRadii.cpp:15-173): burial integrals -> psi
//                -> Born radius through tanh(alpha psi - beta psi^2 + gamma psi^3)
//   GBPartialSum (force/GB/GBPartialSum.cpp:11-42): per-atom chain-rule sums
//   GBForce      (force/GB/GBForce.cpp:14-242): pair + self energies, forces
// The reference stores six N x N scratch arrays (distij, L, U, expTerm,
// filTerm, partialTerm, topology/Atom.h:35-157); here every pass recomputes
// what it needs in registers.  Each pass is a thread-per-i kernel over a
// 2-D grid (i blocks x j chunks) with j tiles in shared memory, and per-atom
// sums reduced in int64 fixed point, so results are order independent.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>

#include "pm_device.cuh"

namespace pmgpu {

constexpr double kGbScale = 1099511627776.0;  // 2^40 for per-atom GB sums
constexpr int kGbTile = 64;

// 2-D launch shape of the all-pairs passes: enough j chunks (whole tiles)
// that about eight blocks land on every SM.
static void gb_grid(int n, dim3 *grid, int *jchunk) {
  const int iblocks = (n + kGbTile - 1) / kGbTile;
  int chunks = std::max(1, std::min((148 * 8 + iblocks - 1) / iblocks, iblocks));
  *jchunk = ((n + chunks - 1) / chunks + kGbTile - 1) / kGbTile * kGbTile;
  chunks = (n + *jchunk - 1) / *jchunk;
  *grid = dim3(iblocks, chunks);
}

struct GbArgs {
  int n;
  const double *pos, *charge, *vdwr, *scale, *offset;
  const int *water;
  double alpha, beta, gamma;
  double dielec;  // 1/solute - 1/solvent
  long long *burial_fx, *partial_fx;  // fixed-point accumulators
  double *born, *partial;
  double *psi;  // per atom dR/d(burial sum) factor of the force pass
  long long *force, *acc;
  // FP32 passes: pair records (write_pair_record), static records
  // (k_gb_static) and the per-evaluation radius records (born, 1 / born,
  // dR/d(burial sum), q^2 / (2 born^2)) from k_gb_radii
  const float4 *rec, *gst;
  float4 *grad;
  // GBACEForce (null: off): per atom the factor A_i = c1 c_i R_i^-7 dR_i/dI
  // of the ACE pair force, and its energy parameters
  double *ace;
  double ace_sigma, ace_rho;
  int partial_pass;  // GBForce on: the partial sums are formed
};

// GBACEForce's pi (GBACEForce.cpp:6): the reference's constant, not M_PI.
constexpr double kAcePi = 3.14169;

template <typename Real>
__device__ __forceinline__ Real gb_burial_term(Real dist, Real oi, Real oj, Real Sj) {
  // term_i of GBBornRadii::operator() (GBBornRadii.cpp:60-85)
  Real L, U;
  Real sjoj = Sj * oj;
  if (oi >= dist + sjoj) {
    L = Real(1);
    U = Real(1);
  } else {
    Real a = fabs(dist - sjoj);
    L = oi > a ? oi : a;
    U = dist + sjoj;
  }
  Real C = (oi < sjoj - dist) ? Real(2) * (Real(1) / oi - Real(1) / L) : Real(0);
  Real iL = Real(1) / L, iU = Real(1) / U;
  return (iL - iU) + (dist / Real(4)) * (iU * iU - iL * iL) +
         (Real(1) / (Real(2) * dist)) * log(L / U) +
         ((sjoj * sjoj) / (Real(4) * dist)) * (iL * iL - iU * iU) + C;
}

template <typename Real>
__global__ void __launch_bounds__(kGbTile) k_gb_burial(GbArgs a, int jchunk) {
  __shared__ double sx[kGbTile], sy[kGbTile], sz[kGbTile], so[kGbTile], ss[kGbTile];
  __shared__ int sw[kGbTile];
  int i = blockIdx.x * kGbTile + threadIdx.x;
  bool valid = i < a.n;
  int ii = valid ? i : 0;
  double xi = a.pos[3 * ii], yi = a.pos[3 * ii + 1], zi = a.pos[3 * ii + 2];
  Real oi = (Real)(a.vdwr[ii] - a.offset[ii]);
  int wi = a.water ? a.water[ii] : 0;
  double acc = 0.0;
  int j0 = blockIdx.y * jchunk, j1 = min(a.n, j0 + jchunk);
  for (int base = j0; base < j1; base += kGbTile) {
    int j = base + threadIdx.x;
    if (j < j1) {
      sx[threadIdx.x] = a.pos[3 * j]; sy[threadIdx.x] = a.pos[3 * j + 1];
      sz[threadIdx.x] = a.pos[3 * j + 2];
      so[threadIdx.x] = a.vdwr[j] - a.offset[j];
      ss[threadIdx.x] = a.scale[j];
      sw[threadIdx.x] = a.water ? a.water[j] : 0;
    }
    __syncthreads();
    int lim = min(kGbTile, j1 - base);
    if (valid && !wi) {
      Real part = 0;
      for (int k = 0; k < lim; k++) {
        if (base + k == i || sw[k]) continue;
        Real dx = (Real)(sx[k] - xi), dy = (Real)(sy[k] - yi), dz = (Real)(sz[k] - zi);
        Real dist = pm_sqrt(dx * dx + dy * dy + dz * dz);
        part += gb_burial_term<Real>(dist, oi, (Real)so[k], (Real)ss[k]);
      }
      acc += (double)part;
    }
    __syncthreads();
  }
  if (valid && !wi && acc != 0.0) red_add(&a.burial_fx[i], to_fixed(acc, kGbScale));
}

// GBBornRadii::postProcess (GBBornRadii.cpp:145-173) and the GB self
// energy of GBForce (GBForce.cpp:56-63, summed in postProcess :230-242).
__global__ void k_gb_radii(GbArgs a) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double self = 0.0;
  if (i < a.n) {
    // the reciprocals of the static radii do not wait for the burial sum
    const double ri = a.vdwr[i];
    const double oi = ri - a.offset[i];
    const double iri = 1 / ri, ioi = 1 / oi;
    const double q = a.charge[i];
    double burial = (double)a.burial_fx[i] * (1.0 / kGbScale);
    double psi = 0.5 * burial * oi;
    double tp = a.alpha * psi - a.beta * psi * psi + a.gamma * psi * psi * psi;
    double th = tanh(tp);
    double inv = ioi - iri * th;  // 1 / R_i
    double born = 1 / inv;
    // dR_i/d(burial sum) (GBForce.cpp:108-118 without the pair factor dBT):
    // R_i^2 rho~_i (1 - tanh^2) (alpha - 2 beta psi + 3 gamma psi^2) / rho_i
    double td = a.alpha - 2.0 * a.beta * psi + 3.0 * a.gamma * psi * psi;
    const double dfac = born * born * oi * (1.0 - th * th) * td * iri;
    a.psi[i] = dfac;
    a.born[i] = born;
    if (a.ace) {
      // GBACEForce: c1 c_i R^-7 dR/dI (the pair force's per-atom factor,
      // GBACEForce.cpp:164-205) and the atom's ACE energy
      // 4 pi sigma (r + rho_s)^2 (r / R)^6 (:51-62)
      const double rr = (ri + a.ace_rho) * (ri + a.ace_rho);
      const double x = ri * inv, x2 = x * x, x6 = x2 * x2 * x2;
      a.ace[i] = 24.0 * kAcePi * a.ace_sigma * rr * x6 * inv * dfac;
      if (a.n > 1) self += 4.0 * kAcePi * a.ace_sigma * rr * x6;
    }
    if (a.grad)
      a.grad[i] = make_float4((float)born, (float)inv, (float)dfac, (float)(0.5 * q * q * inv * inv));
    a.burial_fx[i] = 0;
    a.partial_fx[i] = 0;
    if (a.n > 1) self += -0.5 * (q * q) * inv * a.dielec;
  }
  self = warp_sum(self);
  if ((threadIdx.x & 31) == 0) red_add(&a.acc[ACC_COULOMB], to_fixed(self, kEnergyScale));
}

template <typename Real>
__global__ void __launch_bounds__(kGbTile) k_gb_partial(GbArgs a, int jchunk) {
  __shared__ double sx[kGbTile], sy[kGbTile], sz[kGbTile], sb[kGbTile], sq[kGbTile];
  int i = blockIdx.x * kGbTile + threadIdx.x;
  bool valid = i < a.n;
  int ii = valid ? i : 0;
  double xi = a.pos[3 * ii], yi = a.pos[3 * ii + 1], zi = a.pos[3 * ii + 2];
  Real bi = (Real)a.born[ii], qi = (Real)a.charge[ii];
  double acc = 0.0;
  int j0 = blockIdx.y * jchunk, j1 = min(a.n, j0 + jchunk);
  for (int base = j0; base < j1; base += kGbTile) {
    int j = base + threadIdx.x;
    if (j < j1) {
      sx[threadIdx.x] = a.pos[3 * j]; sy[threadIdx.x] = a.pos[3 * j + 1];
      sz[threadIdx.x] = a.pos[3 * j + 2];
      sb[threadIdx.x] = a.born[j];
      sq[threadIdx.x] = a.charge[j];
    }
    __syncthreads();
    int lim = min(kGbTile, j1 - base);
    if (valid) {
      Real part = 0;
      for (int k = 0; k < lim; k++) {
        if (base + k == i) continue;
        Real dx = (Real)(sx[k] - xi), dy = (Real)(sy[k] - yi), dz = (Real)(sz[k] - zi);
        Real r2 = dx * dx + dy * dy + dz * dz;
        Real bj = (Real)sb[k];
        Real ex = exp(-r2 / (Real(4) * bi * bj));
        Real fil = pm_sqrt(r2 + bi * bj * ex);
        Real p = qi * (Real)sq[k] * (Real(1) / (fil * fil)) * Real(0.5) * (Real(1) / fil) * ex;
        part += p * (bj + r2 / (Real(4) * bi));  // aTerm, GBPartialSum.cpp:33
      }
      acc += (double)part;
    }
    __syncthreads();
  }
  if (valid && acc != 0.0) red_add(&a.partial_fx[i], to_fixed(acc, kGbScale));
}

__global__ void k_gb_partial_fin(GbArgs a) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.n) a.partial[i] = (double)a.partial_fx[i] * (1.0 / kGbScale);
}

// dBT/dr of GBForce::operator() (GBForce.cpp:70-124) for the "i sees j"
// direction; dR_i/dr is this times the per-atom factor k_gb_radii stores.
template <typename Real>
__device__ __forceinline__ Real gb_dBT(Real dist, Real oi, Real oj, Real Sj) {
  Real sjoj = Sj * oj;
  Real L, U;
  if (oi >= dist + sjoj) {
    L = 1; U = 1;
  } else {
    Real a = fabs(dist - sjoj);
    L = oi > a ? oi : a;
    U = dist + sjoj;
  }
  Real iL = Real(1) / L, iU = Real(1) / U;
  Real dL = (oi <= (dist - sjoj)) ? Real(1) : Real(0);
  Real dU = (oi < (dist + sjoj)) ? Real(1) : Real(0);
  Real dC = (oi <= (sjoj - dist)) ? Real(2) * iL * iL * dL : Real(0);
  Real Sjt = sjoj / dist;
  Real iL2 = iL * iL, iU2 = iU * iU;
  return Real(-0.5) * dL * iL2 + Real(0.5) * dU * iU2 + Real(0.125) * (iU2 - iL2) +
         Real(0.125) * dist * (Real(2) * iL2 * iL * dL - Real(2) * iU2 * iU * dU) -
         Real(0.25) * (Real(1) / (dist * dist)) * log(L / U) +
         (U / (Real(4) * dist * L)) * (iU * dL - (L * iU2) * dU) -
         Real(0.125) * (Sjt * Sjt) * (iL2 - iU2) +
         Real(0.25) * ((sjoj * sjoj) / dist) * iU2 * iU * dU -
         Real(0.25) * ((sjoj * sjoj) / dist) * iL2 * iL * dL + dC;
}

template <typename Real>
__global__ void __launch_bounds__(kGbTile) k_gb_force(GbArgs a, int jchunk) {
  __shared__ double sx[kGbTile], sy[kGbTile], sz[kGbTile], sb[kGbTile], sq[kGbTile];
  __shared__ double so[kGbTile], ss[kGbTile], sp[kGbTile], spart[kGbTile], sa[kGbTile];
  int i = blockIdx.x * kGbTile + threadIdx.x;
  bool valid = i < a.n;
  int ii = valid ? i : 0;
  double xi = a.pos[3 * ii], yi = a.pos[3 * ii + 1], zi = a.pos[3 * ii + 2];
  Real bi = (Real)a.born[ii], qi = (Real)a.charge[ii];
  Real oi = (Real)(a.vdwr[ii] - a.offset[ii]);
  Real Si = (Real)a.scale[ii], dfac_i = (Real)a.psi[ii];
  Real part_i = (Real)a.partial[ii];
  const Real ace_i = a.ace ? (Real)a.ace[ii] : Real(0);
  const Real d = (Real)a.dielec;
  Real fx = 0, fy = 0, fz = 0;
  double epair = 0.0;
  int j0 = blockIdx.y * jchunk, j1 = min(a.n, j0 + jchunk);
  for (int base = j0; base < j1; base += kGbTile) {
    int j = base + threadIdx.x;
    if (j < j1) {
      sx[threadIdx.x] = a.pos[3 * j]; sy[threadIdx.x] = a.pos[3 * j + 1];
      sz[threadIdx.x] = a.pos[3 * j + 2];
      sb[threadIdx.x] = a.born[j]; sq[threadIdx.x] = a.charge[j];
      so[threadIdx.x] = a.vdwr[j] - a.offset[j];
      ss[threadIdx.x] = a.scale[j]; sp[threadIdx.x] = a.psi[j];
      spart[threadIdx.x] = a.partial[j];
      sa[threadIdx.x] = a.ace ? a.ace[j] : 0.0;
    }
    __syncthreads();
    int lim = min(kGbTile, j1 - base);
    if (valid) {
      Real ep = 0;
      for (int k = 0; k < lim; k++) {
        if (base + k == i) continue;
        Real dx = (Real)(sx[k] - xi), dy = (Real)(sy[k] - yi), dz = (Real)(sz[k] - zi);
        Real r2 = dx * dx + dy * dy + dz * dz;
        Real dist = pm_sqrt(r2);
        Real idist = Real(1) / dist;
        Real bj = (Real)sb[k], qj = (Real)sq[k];
        Real oj = (Real)so[k], Sj = (Real)ss[k];
        Real ex = exp(-r2 / (Real(4) * bi * bj));
        Real fGB = pm_sqrt(r2 + bi * bj * ex);
        ep += -(qi * qj) / fGB;
        const Real bti = gb_dBT<Real>(dist, oi, oj, Sj);
        const Real btj = gb_dBT<Real>(dist, oj, oi, Si);
        Real dRi = dfac_i * bti;
        Real dRj = (Real)sp[k] * btj;
        Real pref = qi * qj * (Real(1) / (fGB * fGB)) * Real(0.5) * (Real(1) / fGB);
        // partialTerm[i][j] and [j][i] (GBPartialSum.cpp:33-41)
        Real ptij = pref * ex * (bj + r2 / (Real(4) * bi));
        Real ptji = pref * ex * (bi + r2 / (Real(4) * bj));
        Real f = -pref * ((Real(2) * dist - Real(0.5) * ex * dist) +
                          ex * dRi * (bj + r2 / (Real(4) * bi)) +
                          ex * dRj * (bi + r2 / (Real(4) * bj))) * idist;
        f -= Real(0.5) * qi * qi * dRi / (bi * bi) * idist;
        f -= Real(0.5) * qj * qj * dRj / (bj * bj) * idist;
        f -= (part_i - ptij) * (dRi * idist);
        f -= ((Real)spart[k] - ptji) * (dRj * idist);
        // GBForce scaled by the dielectric factor, plus GBACEForce
        f = f * d + (ace_i * bti + (Real)sa[k] * btj) * idist;
        fx -= dx * f; fy -= dy * f; fz -= dz * f;
      }
      epair += (double)ep;
    }
    __syncthreads();
  }
  if (valid) {
    red_add(&a.force[i], to_fixed((double)fx, kForceScale));
    red_add(&a.force[a.n + i], to_fixed((double)fy, kForceScale));
    red_add(&a.force[2 * a.n + i], to_fixed((double)fz, kForceScale));
  }
  epair = warp_sum(epair) * 0.5 * a.dielec;
  if ((threadIdx.x & 31) == 0) red_add(&a.acc[ACC_COULOMB], to_fixed(epair, kEnergyScale));
}

// ---------------------------------------------------------------------
// FP32 forms of the three all-pairs passes, each over every unordered pair
// once in 32 x 32 tile pairs (see k_gb_burial_half).  Atom records are
// staged with hi/lo FP32 coordinates, so the pair loops take no FP64
// operation or conversion; reciprocals come from the hardware estimate plus
// one Newton step and every distance from one rsqrt; pairs outside the
// half set are masked rather than skipped.

// Far pairs.  When d - s >= o_i (s = S_j o_j), L = d - s and U = d + s,
// dL = dU = 1 and dC = 0, and with t = s / d the closed forms reduce to odd
// power series (their Taylor expansions in t, all terms of one sign):
//   term  = (1/d)   sum_k 2k/(2k+1)        t^(2k+1)
//   dBT   = -(1/d^2) sum_k 2k(k+1)/(2k+1)  t^(2k+1),   k = 1, 2, ...
// For t <= 1/4 eight terms leave a relative truncation below 2e-9, and
// unlike the closed forms, whose terms cancel to O(t^3) of their size, the
// series keeps full FP32 precision.  It needs no reciprocal or logarithm.
constexpr float kGbFarT = 0.25f;

__device__ __forceinline__ bool gb_far(float dist, float oi, float sjoj) {
  return dist - sjoj >= oi && sjoj <= kGbFarT * dist;
}

// sum_{k=1..8} 2k/(2k+1) u^(k-1)
__device__ __forceinline__ float gb_series_term(float u) {
  float p = 16.0f / 17.0f;
  p = fmaf(p, u, 14.0f / 15.0f);
  p = fmaf(p, u, 12.0f / 13.0f);
  p = fmaf(p, u, 10.0f / 11.0f);
  p = fmaf(p, u, 8.0f / 9.0f);
  p = fmaf(p, u, 6.0f / 7.0f);
  p = fmaf(p, u, 4.0f / 5.0f);
  return fmaf(p, u, 2.0f / 3.0f);
}

// sum_{k=1..8} 2k(k+1)/(2k+1) u^(k-1)
__device__ __forceinline__ float gb_series_dbt(float u) {
  float p = 144.0f / 17.0f;
  p = fmaf(p, u, 112.0f / 15.0f);
  p = fmaf(p, u, 84.0f / 13.0f);
  p = fmaf(p, u, 60.0f / 11.0f);
  p = fmaf(p, u, 40.0f / 9.0f);
  p = fmaf(p, u, 24.0f / 7.0f);
  p = fmaf(p, u, 12.0f / 5.0f);
  return fmaf(p, u, 4.0f / 3.0f);
}

// burial term of the "i sees j" direction given dist and 1/dist
__device__ __forceinline__ float gb_burial_term_f32(float dist, float idist, float oi,
                                                   float ioi, float sjoj) {
  if (gb_far(dist, oi, sjoj)) {
    const float t = sjoj * idist, u = t * t;
    return idist * (t * u) * gb_series_term(u);
  }
  float L, U;
  if (oi >= dist + sjoj) {
    L = 1.0f;
    U = 1.0f;
  } else {
    const float a = fabsf(dist - sjoj);
    L = oi > a ? oi : a;
    U = dist + sjoj;
  }
  const float iL = rcp_nr(L), iU = rcp_nr(U);
  const float C = (oi < sjoj - dist) ? 2.0f * (ioi - iL) : 0.0f;
  const float iL2 = iL * iL, iU2 = iU * iU;
  return (iL - iU) + (0.25f * dist) * (iU2 - iL2) + (0.5f * idist) * logf(L * iU) +
         (0.25f * sjoj * sjoj * idist) * (iL2 - iU2) + C;
}

// dBT/dr of the "i sees j" direction (same terms as gb_dBT above)
__device__ __forceinline__ float gb_dBT_f32(float dist, float idist, float oi, float sjoj) {
  if (gb_far(dist, oi, sjoj)) {
    const float t = sjoj * idist, u = t * t;
    return -(idist * idist) * (t * u) * gb_series_dbt(u);
  }
  float L, U;
  if (oi >= dist + sjoj) {
    L = 1.0f;
    U = 1.0f;
  } else {
    const float a = fabsf(dist - sjoj);
    L = oi > a ? oi : a;
    U = dist + sjoj;
  }
  const float iL = rcp_nr(L), iU = rcp_nr(U);
  const float dL = (oi <= (dist - sjoj)) ? 1.0f : 0.0f;
  const float dU = (oi < (dist + sjoj)) ? 1.0f : 0.0f;
  const float iL2 = iL * iL, iU2 = iU * iU;
  const float dC = (oi <= (sjoj - dist)) ? 2.0f * iL2 * dL : 0.0f;
  const float Sjt = sjoj * idist;
  const float s2d = sjoj * sjoj * idist;
  return -0.5f * dL * iL2 + 0.5f * dU * iU2 + 0.125f * (iU2 - iL2) +
         0.125f * dist * (2.0f * iL2 * iL * dL - 2.0f * iU2 * iU * dU) -
         0.25f * (idist * idist) * logf(L * iU) +
         (0.25f * U * idist * iL) * (iU * dL - (L * iU2) * dU) -
         0.125f * (Sjt * Sjt) * (iL2 - iU2) + 0.25f * s2d * iU2 * iU * dU -
         0.25f * s2d * iL2 * iL * dL + dC;
}

// Burial sums over each unordered pair once, both directions per pair: a
// warp takes halves (16 j atoms) of 32 x 32 tile pairs (I, J), I <= J, from
// its block's share (near tile pairs, which take the closed form, cost
// several times more than far ones, so the finer items spread them); the
// "i sees j" term adds to i in the lane, the "j sees i" term to j through
// warp_tsum8.  Water atoms neither receive nor give burial.
template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32, 1)
k_gb_burial_half(GbArgs a, int tiles, long long items) {
  // per j: (x_hi, y_hi, z_hi, rho~) | (x_lo, y_lo, z_lo, S rho~) | (1 / rho~, water)
  __shared__ float4 sh[WARPS][32], sl[WARPS][32];
  __shared__ float2 sg[WARPS][32];
  const int lane = threadIdx.x & 31, wb = threadIdx.x >> 5;
  __shared__ int counter;
  if (threadIdx.x == 0) counter = 0;
  __syncthreads();
  const BlockItems queue{&counter};
  long long w;
  for (w = queue.next(lane); w < items; w = queue.next(lane)) {
    int I, J;
    tile_pair_of(w >> 1, tiles, &I, &J);
    const int g0 = 2 * (int)(w & 1);
    const int i = I * 32 + lane;
    const bool vi = i < a.n;
    const int ii = vi ? i : 0;
    const float4 hi = a.rec[ii], li = a.rec[a.n + ii], gi = a.gst[ii];
    const bool ai = vi && gi.w == 0.0f;
    {
      const int j = J * 32 + lane;
      const int jj = j < a.n ? j : 0;
      const float4 g = a.gst[jj], h = a.rec[jj], l = a.rec[a.n + jj];
      sh[wb][lane] = make_float4(h.x, h.y, h.z, g.x);
      sl[wb][lane] = make_float4(l.x, l.y, l.z, g.y);
      // past the end: unused, like water
      sg[wb][lane] = make_float2(g.z, j < a.n ? g.w : 1.0f);
    }
    __syncwarp();
    float bsum = 0;
#pragma unroll 1
    for (int g = g0; g < g0 + 2; g++) {
      float gb[8];
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int k = g * 8 + u;
        const float4 h = sh[wb][k], l = sl[wb][k];
        const float2 gj = sg[wb][k];
        const bool use = ai && gj.y == 0.0f && (I < J || k > lane);
        const float dx = (h.x - hi.x) + (l.x - li.x);
        const float dy = (h.y - hi.y) + (l.y - li.y);
        const float dz = (h.z - hi.z) + (l.z - li.z);
        const float r2 = use ? dx * dx + dy * dy + dz * dz : 1.0f;
        const float idist = rsqrt_nr(r2);
        const float dist = r2 * idist;
        const float tij = gb_burial_term_f32(dist, idist, gi.x, gi.z, l.w);
        const float tji = gb_burial_term_f32(dist, idist, h.w, gj.x, gi.y);
        bsum += use ? tij : 0.0f;
        gb[u] = use ? tji : 0.0f;
      }
      const float sb = warp_tsum8(gb, lane);
      const int jt = J * 32 + g * 8 + (lane >> 2);
      if ((lane & 3) == 0 && jt < a.n) red_add(&a.burial_fx[jt], to_fixed((double)sb, kGbScale));
    }
    if (ai) red_add(&a.burial_fx[i], to_fixed((double)bsum, kGbScale));
    __syncwarp();
  }
}

// Partial sums over each unordered pair once (same tiling):
// partialTerm[i][j] adds to i in the lane and partialTerm[j][i] to j
// through warp_tsum8.
template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32, 1)
k_gb_partial_half(GbArgs a, int tiles, long long items) {
  __shared__ float4 sh[WARPS][32], sl[WARPS][32], sr[WARPS][32];
  const int lane = threadIdx.x & 31, wb = threadIdx.x >> 5;
  __shared__ int counter;
  if (threadIdx.x == 0) counter = 0;
  __syncthreads();
  const BlockItems queue{&counter};
  long long w;
  for (w = queue.next(lane); w < items; w = queue.next(lane)) {
    int I, J;
    tile_pair_of(w, tiles, &I, &J);
    const int i = I * 32 + lane;
    const bool vi = i < a.n;
    const int ii = vi ? i : 0;
    const float4 hi = a.rec[ii], li = a.rec[a.n + ii], ri = a.grad[ii];
    const float q4bi = 0.25f * ri.y;
    {
      const int j = J * 32 + lane;
      const int jj = j < a.n ? j : 0;
      sh[wb][lane] = a.rec[jj];
      sl[wb][lane] = a.rec[a.n + jj];
      sr[wb][lane] = a.grad[jj];
    }
    __syncwarp();
    const int jn = a.n - J * 32;
    float pi = 0;
#pragma unroll 1
    for (int g = 0; g < 4; g++) {
      float gp[8];
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int k = g * 8 + u;
        const float4 h = sh[wb][k], l = sl[wb][k], rj = sr[wb][k];
        const bool use = vi && k < jn && (I < J || k > lane);
        const float dx = (h.x - hi.x) + (l.x - li.x);
        const float dy = (h.y - hi.y) + (l.y - li.y);
        const float dz = (h.z - hi.z) + (l.z - li.z);
        const float r2 = use ? dx * dx + dy * dy + dz * dz : 1.0f;
        const float bj = rj.x, bb = ri.x * bj;
        const float ex = __expf(-r2 * (q4bi * rj.y));
        const float ifil = rsqrt_nr(r2 + bb * ex);
        const float p = 0.5f * hi.w * h.w * (ifil * ifil * ifil) * ex;
        // aTerm of both directions (GBPartialSum.cpp:33)
        pi += use ? p * (bj + r2 * q4bi) : 0.0f;
        gp[u] = use ? p * (ri.x + 0.25f * r2 * rj.y) : 0.0f;
      }
      const float sp = warp_tsum8(gp, lane);
      const int jt = J * 32 + g * 8 + (lane >> 2);
      if ((lane & 3) == 0 && jt < a.n) red_add(&a.partial_fx[jt], to_fixed((double)sp, kGbScale));
    }
    if (vi) red_add(&a.partial_fx[i], to_fixed((double)pi, kGbScale));
    __syncwarp();
  }
}

// Forces and pair energy over each unordered pair once (same tiling); the
// pair force of GBForce::operator() is symmetric in i and j, so j receives
// its opposite through warp_tsum8.  Work items are halves of tile pairs
// (16 j atoms), so the warps of a block share this heaviest pass finely.
//
// GBForce::operator() (GBForce.cpp:70-124) forms the pair force as
//   -pref (2 d - ex d / 2 + ex dR_i a_ij + ex dR_j a_ji) / d
//   - [q_i^2 / 2R_i^2 + (P_i - pt_ij)] dR_i / d - [same for j] dR_j / d
// with pt_ij = pref ex a_ij the pair's own term of the partial sum P_i.
// The pt_ij terms cancel exactly, leaving
//   -pref (2 - ex / 2) - (D_i dBT_ij + D_j dBT_ji) / d,
//   D_i = (q_i^2 / 2R_i^2 + P_i) dR_i/dI_i,
// a per-atom factor formed once per item; the FP64 pass keeps the
// reference's grouping.
template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32, 1)
k_gb_force_half(GbArgs a, int tiles, long long items) {
  // per j: (x_hi, y_hi, z_hi, q) | (x_lo, y_lo, z_lo, R) | (1 / R, D, rho~, S rho~)
  __shared__ float4 sh[WARPS][32], sl[WARPS][32], sr[WARPS][32];
  const int lane = threadIdx.x & 31, wb = threadIdx.x >> 5;
  __shared__ int counter;
  if (threadIdx.x == 0) counter = 0;
  __syncthreads();
  const BlockItems queue{&counter};
  const double d = a.dielec;
  double epair = 0.0;
  long long w;
  for (w = queue.next(lane); w < items; w = queue.next(lane)) {
    int I, J;
    tile_pair_of(w >> 1, tiles, &I, &J);
    const int g0 = 2 * (int)(w & 1);
    const int i = I * 32 + lane;
    const bool vi = i < a.n;
    const int ii = vi ? i : 0;
    const float4 hi = a.rec[ii], li = a.rec[a.n + ii], gi = a.gst[ii], ri = a.grad[ii];
    // D_i scaled by the dielectric factor, less the ACE factor A_i
    const float Di = (float)(d * ((double)ri.w + (double)a.partial_fx[ii] * (1.0 / kGbScale)) *
                                 (double)ri.z -
                             (a.ace ? a.ace[ii] : 0.0));
    const float q4bi = 0.25f * ri.y;
    const float qd = (float)d;
    {
      const int j = J * 32 + lane;
      const int jj = j < a.n ? j : 0;
      const float4 l = a.rec[a.n + jj], g = a.gst[jj], r = a.grad[jj];
      const double Dj =
          d * ((double)r.w + (double)a.partial_fx[jj] * (1.0 / kGbScale)) * (double)r.z -
          (a.ace ? a.ace[jj] : 0.0);
      sh[wb][lane] = a.rec[jj];
      sl[wb][lane] = make_float4(l.x, l.y, l.z, r.x);
      sr[wb][lane] = make_float4(r.y, (float)Dj, g.x, g.y);
    }
    __syncwarp();
    const int jn = a.n - J * 32;
    float fx = 0, fy = 0, fz = 0, ep = 0;
#pragma unroll 1
    for (int gq = g0; gq < g0 + 2; gq++) {
      float gx[8], gy[8], gz[8];
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int k = gq * 8 + u;
        const float4 h = sh[wb][k], l = sl[wb][k], rj = sr[wb][k];
        const bool use = vi && k < jn && (I < J || k > lane);
        const float dx = (h.x - hi.x) + (l.x - li.x);
        const float dy = (h.y - hi.y) + (l.y - li.y);
        const float dz = (h.z - hi.z) + (l.z - li.z);
        const float r2 = use ? dx * dx + dy * dy + dz * dz : 1.0f;
        const float idist = rsqrt_nr(r2);
        const float dist = r2 * idist;
        const float ex = __expf(-r2 * (q4bi * rj.x));
        const float ifgb = rsqrt_nr(r2 + ri.x * l.w * ex);
        const float qq = hi.w * h.w;
        const float pref = 0.5f * (qq * qd) * (ifgb * ifgb * ifgb);
        const float bti = gb_dBT_f32(dist, idist, gi.x, rj.w);
        const float btj = gb_dBT_f32(dist, idist, rj.z, gi.y);
        float f = -pref * (2.0f - 0.5f * ex) - idist * (Di * bti + rj.y * btj);
        f = use ? f : 0.0f;
        ep += use ? -qq * ifgb : 0.0f;
        fx -= dx * f; fy -= dy * f; fz -= dz * f;
        gx[u] = dx * f; gy[u] = dy * f; gz[u] = dz * f;
      }
      const float sx = warp_tsum8(gx, lane), sy = warp_tsum8(gy, lane),
                  sz = warp_tsum8(gz, lane);
      const int jt = J * 32 + gq * 8 + (lane >> 2);
      if ((lane & 3) == 0 && jt < a.n) {
        red_add(&a.force[jt], to_fixed((double)sx, kForceScale));
        red_add(&a.force[a.n + jt], to_fixed((double)sy, kForceScale));
        red_add(&a.force[2 * a.n + jt], to_fixed((double)sz, kForceScale));
      }
    }
    if (vi) {
      red_add(&a.force[i], to_fixed((double)fx, kForceScale));
      red_add(&a.force[a.n + i], to_fixed((double)fy, kForceScale));
      red_add(&a.force[2 * a.n + i], to_fixed((double)fz, kForceScale));
    }
    epair += (double)ep;
    __syncwarp();
  }
  epair = warp_sum(epair) * d;
  if (lane == 0 && epair != 0.0) red_add(&a.acc[ACC_COULOMB], to_fixed(epair, kEnergyScale));
}

// Static FP32 record of the GB passes: (rho~ = vdwr - offset, S rho~,
// 1 / rho~, 1 for water else 0).
__global__ void k_gb_static(int n, const double *__restrict__ vdwr,
                            const double *__restrict__ scale, const double *__restrict__ offset,
                            const int *__restrict__ water, float4 *__restrict__ gst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double o = vdwr[i] - offset[i];
  gst[i] = make_float4((float)o, (float)(scale[i] * o), (float)(1.0 / o),
                       water && water[i] ? 1.0f : 0.0f);
}

// The FP32 chain: burial sums, Born radii, partial sums, forces (the
// partial sums stay in their fixed-point accumulators).  a.rec holds the
// atoms' pair records and a.gst the static GB records.
static void gb_passes_f32(const GbArgs &a, cudaStream_t st) {
  // one block per SM (the register counts admit no second), so every SM
  // holds the same number of warps and the queue balances the items
  int tiles, blocks, blocks2;
  long long items, items2;
  halfpairs_grid(a.n, 1, &tiles, &items, &blocks);
  halfpairs_grid(a.n, 2, &tiles, &items2, &blocks2);
  k_gb_burial_half<32><<<blocks2, 32 * 32, 0, st>>>(a, tiles, items2);
  // one-warp blocks: they fit beside a resident simple-full block
  k_gb_radii<<<(a.n + 31) / 32, 32, 0, st>>>(a);
  if (a.partial_pass) k_gb_partial_half<16><<<blocks, 16 * 32, 0, st>>>(a, tiles, items);
  k_gb_force_half<16><<<blocks2, 16 * 32, 0, st>>>(a, tiles, items2);
}

int gb_init(System *s) {
  int n = std::max(1, s->n);
  if (!s->d_gb_vdwr) return fail(PMGPU_ERR_ARG, "GB force needs gb_vdwr/gb_scale/gb_offset");
  if (!s->d_gb_born) {
    PM_CHECK(dev_alloc(s, &s->d_gb_born, sizeof(double) * n));
    PM_CHECK(dev_alloc(s, &s->d_gb_psi, sizeof(double) * n));
    PM_CHECK(dev_alloc(s, &s->d_gb_partial, sizeof(double) * n));
    PM_CHECK(dev_alloc(s, &s->d_gb_fixed, sizeof(long long) * 2 * n));
    PM_CHECK(dev_alloc(s, &s->d_gb_ace, sizeof(double) * n));
    PM_CUDA(cudaMemsetAsync(s->d_gb_fixed, 0, sizeof(long long) * 2 * n, s->stream));
  }
  if (s->precision == PMGPU_PREC_MIXED && !s->d_gb_gst) {
    if (!s->d_rec) PM_CHECK(dev_alloc(s, &s->d_rec, sizeof(float4) * 2 * n));
    PM_CHECK(dev_alloc(s, &s->d_gb_gst, sizeof(float4) * n));
    PM_CHECK(dev_alloc(s, &s->d_gb_grad, sizeof(float4) * n));
    if (s->n > 0)
      k_gb_static<<<(s->n + 127) / 128, 128, 0, s->stream>>>(
          s->n, s->d_gb_vdwr, s->d_gb_scale, s->d_gb_offset, s->d_water, s->d_gb_gst);
    PM_CUDA(cudaGetLastError());
  }
  return PMGPU_OK;
}

// gb: the GBForce term (null: none), ace: the GBACEForce term (null: none);
// with both, one chain of passes serves both (the Born radii once, the ACE
// pair force folded into the GB force pass).
int gb_forces(System *s, const Force *gb, const Force *ace) {
  int n = s->n;
  if (n == 0 || (!gb && !ace)) return PMGPU_OK;
  GbArgs a;
  a.n = n;
  a.pos = s->d_pos;
  a.charge = s->d_charge;
  a.vdwr = s->d_gb_vdwr;
  a.scale = s->d_gb_scale;
  a.offset = s->d_gb_offset;
  a.water = s->d_water;
  a.alpha = s->gb_obc[0];
  a.beta = s->gb_obc[1];
  a.gamma = s->gb_obc[2];
  a.dielec = gb ? (1 / gb->solute) - (1 / gb->solvent) : 0.0;
  a.partial_pass = gb != nullptr;
  a.ace = ace ? s->d_gb_ace : nullptr;
  a.ace_sigma = ace ? ace->ace_sigma : 0.0;
  a.ace_rho = ace ? ace->ace_rho : 0.0;
  a.burial_fx = s->d_gb_fixed;
  a.partial_fx = s->d_gb_fixed + n;
  a.born = s->d_gb_born;
  a.psi = s->d_gb_psi;
  a.partial = s->d_gb_partial;
  a.force = s->d_force;
  a.acc = s->d_acc;
  a.rec = s->d_rec;
  a.gst = s->d_gb_gst;
  a.grad = s->d_gb_grad;
  dim3 grid;
  int jchunk;
  gb_grid(n, &grid, &jchunk);
  cudaStream_t st = s->stream;
  if (s->precision == PMGPU_PREC_MIXED) {
    gb_passes_f32(a, st);
  } else {
    k_gb_burial<double><<<grid, kGbTile, 0, st>>>(a, jchunk);
    k_gb_radii<<<(n + 127) / 128, 128, 0, st>>>(a);
    if (a.partial_pass) k_gb_partial<double><<<grid, kGbTile, 0, st>>>(a, jchunk);
    k_gb_partial_fin<<<(n + 127) / 128, 128, 0, st>>>(a);
    k_gb_force<double><<<grid, kGbTile, 0, st>>>(a, jchunk);
  }
  PM_CUDA(cudaGetLastError());
  return PMGPU_OK;
}

}  // namespace pmgpu

// ---------------------------------------------------------------------------
// GB forces without any device allocation.
//
// Some callers cannot allocate device memory at the moment they need GB
// forces: a host program that has handed all of HBM to its own pool
// allocator, a plugin that only ever receives buffers from its host and must
// not grow the device footprint, or a loop that cannot afford the implicit
// device-wide synchronisation that cudaMalloc/cudaFree bring.  For them this
// path keeps its scratch (Born radii, psi, partial sums and the fixed-point
// accumulators) in one statically sized __device__ array that lives as long
// as the library is loaded.  The price is a hard size limit and a single
// shared scratch: every call on a device uses the same array, so two calls
// whose kernels overlap on the GPU (different streams, or different host
// threads on one device) race on it and both results are garbage.  Callers
// serialise their calls, for instance by issuing them all on one stream.
// ---------------------------------------------------------------------------
namespace pmgpu {
namespace {

constexpr int kGbStaticMaxAtoms = PMGPU_GB_STATIC_MAX_ATOMS;
constexpr int kGbStaticAccWords = 32;
static_assert(ACC_COUNT <= kGbStaticAccWords, "accumulator block too small");
// per atom: born, psi, partial (double), burial and partial sums (int64),
// three force planes (int64); then the energy/virial accumulator block;
// then the FP32 records: pair records (2 float4 per atom), static and radius
// records (1 float4 each)
constexpr size_t kGbStaticWords = 16 * (size_t)kGbStaticMaxAtoms + kGbStaticAccWords;

// In host code this name is only a stand-in for the symbol; the device
// address comes from cudaGetSymbolAddress.
static __device__ __align__(256) long long g_gb_scratch[kGbStaticWords];

// Device address of g_gb_scratch in the current context, looked up on every
// call (a lookup, no allocation), so a context created after a
// cudaDeviceReset gets its own copy's address.
int gb_scratch_address(long long **out) {
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_gb_scratch);
  if (e != cudaSuccess || !p)
    return fail(PMGPU_ERR_CUDA, std::string("cudaGetSymbolAddress(GB scratch): ") +
                                    cudaGetErrorString(e));
  *out = static_cast<long long *>(p);
  return PMGPU_OK;
}

// The caller's arrays must be device (or managed) memory of the current
// device: a host pointer here would fault inside the kernels.
int check_device_ptr(const void *p, const char *what) {
  if (!p) return fail(PMGPU_ERR_ARG, std::string(what) + " is NULL");
  cudaPointerAttributes at;
  cudaError_t e = cudaPointerGetAttributes(&at, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(PMGPU_ERR_ARG, std::string(what) + " is not a CUDA pointer");
  }
  if (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged)
    return fail(PMGPU_ERR_ARG, std::string(what) + " is not device memory");
  int dev = -1;
  PM_CUDA(cudaGetDevice(&dev));
  if (at.type == cudaMemoryTypeDevice && at.device != dev)
    return fail(PMGPU_ERR_ARG, std::string(what) + " lives on another device");
  return PMGPU_OK;
}

__global__ void k_gb_static_out(int n, const long long *__restrict__ force,
                                const long long *__restrict__ acc, double *__restrict__ out,
                                double *__restrict__ energy) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n)
    for (int c = 0; c < 3; c++) out[3 * i + c] = (double)force[c * n + i] * (1.0 / kForceScale);
  if (i == 0) *energy = (double)acc[ACC_COULOMB] / kEnergyScale;
}

}  // namespace
}  // namespace pmgpu

extern "C" int pmgpu_gb_forces_noalloc(int n_atoms, const double *pos, const double *charge,
                                       const double *gb_vdwr, const double *gb_scale,
                                       const double *gb_offset, const int *water,
                                       const double obc[3], double solute_dielec,
                                       double solvent_dielec, int precision, double *forces,
                                       double *energy, void *stream) {
  using namespace pmgpu;
  const int n = n_atoms;
  if (n < 0) return fail(PMGPU_ERR_ARG, "n_atoms < 0");
  if (n > kGbStaticMaxAtoms)
    return fail(PMGPU_ERR_ARG, "n_atoms = " + std::to_string(n) +
                                   " exceeds the static GB scratch limit of " +
                                   std::to_string(kGbStaticMaxAtoms) + " atoms");
  if (precision != PMGPU_PREC_MIXED && precision != PMGPU_PREC_DOUBLE)
    return fail(PMGPU_ERR_ARG, "precision must be PMGPU_PREC_MIXED or PMGPU_PREC_DOUBLE");
  if (!obc) return fail(PMGPU_ERR_ARG, "obc is NULL");
  if (!(solute_dielec != 0.0) || !(solvent_dielec != 0.0))
    return fail(PMGPU_ERR_ARG, "dielectric constants must be non-zero");
  PM_CHECK(check_device_ptr(energy, "energy"));
  long long *scratch = nullptr;
  PM_CHECK(gb_scratch_address(&scratch));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (n == 0) {
    PM_CUDA(cudaMemsetAsync(energy, 0, sizeof(double), st));
    return PMGPU_OK;
  }
  PM_CHECK(check_device_ptr(pos, "pos"));
  PM_CHECK(check_device_ptr(charge, "charge"));
  PM_CHECK(check_device_ptr(gb_vdwr, "gb_vdwr"));
  PM_CHECK(check_device_ptr(gb_scale, "gb_scale"));
  PM_CHECK(check_device_ptr(gb_offset, "gb_offset"));
  PM_CHECK(check_device_ptr(forces, "forces"));
  if (water) PM_CHECK(check_device_ptr(water, "water"));

  // carve the scratch for this n; what accumulates starts at zero
  GbArgs a;
  a.n = n;
  a.pos = pos;
  a.charge = charge;
  a.vdwr = gb_vdwr;
  a.scale = gb_scale;
  a.offset = gb_offset;
  a.water = water;
  a.alpha = obc[0];
  a.beta = obc[1];
  a.gamma = obc[2];
  a.dielec = (1 / solute_dielec) - (1 / solvent_dielec);
  a.partial_pass = 1;
  a.ace = nullptr;
  a.ace_sigma = a.ace_rho = 0.0;
  a.born = reinterpret_cast<double *>(scratch);
  a.psi = reinterpret_cast<double *>(scratch + n);
  a.partial = reinterpret_cast<double *>(scratch + 2 * (size_t)n);
  a.burial_fx = scratch + 3 * (size_t)n;
  a.partial_fx = scratch + 4 * (size_t)n;
  a.force = scratch + 5 * (size_t)n;
  a.acc = scratch + 8 * (size_t)n;
  float4 *rec = reinterpret_cast<float4 *>(a.acc + kGbStaticAccWords);
  float4 *gst = rec + 2 * (size_t)n;
  float4 *grad = gst + n;
  a.rec = rec;
  a.gst = gst;
  a.grad = grad;
  PM_CUDA(cudaMemsetAsync(a.burial_fx, 0, sizeof(long long) * (5 * (size_t)n + kGbStaticAccWords),
                          st));

  dim3 grid;
  int jchunk;
  gb_grid(n, &grid, &jchunk);
  if (precision == PMGPU_PREC_MIXED) {
    launch_stage_pairs(n, pos, charge, nullptr, rec, st);
    k_gb_static<<<(n + 127) / 128, 128, 0, st>>>(n, gb_vdwr, gb_scale, gb_offset, water, gst);
    gb_passes_f32(a, st);
  } else {
    k_gb_burial<double><<<grid, kGbTile, 0, st>>>(a, jchunk);
    k_gb_radii<<<(n + 127) / 128, 128, 0, st>>>(a);
    k_gb_partial<double><<<grid, kGbTile, 0, st>>>(a, jchunk);
    k_gb_partial_fin<<<(n + 127) / 128, 128, 0, st>>>(a);
    k_gb_force<double><<<grid, kGbTile, 0, st>>>(a, jchunk);
  }
  k_gb_static_out<<<(n + 255) / 256, 256, 0, st>>>(n, a.force, a.acc, forces, energy);
  PM_CUDA(cudaGetLastError());
  return PMGPU_OK;
}
