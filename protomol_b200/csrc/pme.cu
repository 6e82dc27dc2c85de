// Ewald Coulomb delivered as smooth PME (Essmann et al., J. Chem. Phys.
// 103, 8577 (1995)) plus the two O(exclusions) / O(1) terms of ProtoMol's
// NonbondedFullEwaldSystemForce:
//   * spread: cardinal B-spline (order p) charge spreading into an int64
//     fixed-point grid (order independent, bit reproducible);
//   * 3-D real-to-complex FFT (cuFFT, same stream), convolution with the
//     influence function exp(-pi^2 m^2/alpha^2)/(pi V m^2) |b(m)|^2 with the
//     energy and virial reduced on the way, complex-to-real FFT;
//   * gather: forces from the B-spline derivatives;
//   * correctionTerm (NonbondedFullEwaldSystemForce.h:1092-1131) in FP64.
// The reciprocal energy matches the reference's convention
// E = (4 pi / V) sum_{half space k} exp(-k^2/4a^2)/k^2 |S(k)|^2 (:1013-1054).
#include <algorithm>
#include <cmath>
#include <vector>

#include "pm_device.cuh"

namespace pmgpu {

constexpr int kMaxOrder = 8;
constexpr double kGridScale = 4294967296.0;  // 2^32 per (scaled) charge

struct PmeArgs {
  Box box;
  int n;
  int K[3];
  int order;
  double inv_L[3];
  const double *pos, *charge;
  long long *grid_fixed;  // spread target (int64 fixed point)
  const float *phi;       // potential grid the gather reads
  long long *force;
};

// B-spline weights M_p(fr + k), k = 0..p-1, and their derivatives with
// respect to u, by the Cox-de Boor recursion of the cardinal B-spline
// (fully unrolled for a compile-time order, so the weights stay in
// registers).
template <int P>
__device__ __forceinline__ void bspline(float fr, float *th, float *dth) {
  float m[P];
  m[0] = fr;
  m[1] = 1.f - fr;
#pragma unroll
  for (int k = 2; k < P; k++) m[k] = 0.f;
#pragma unroll
  for (int n = 3; n <= P; n++) {
    if (n == P) {
      // derivative of M_p from M_{p-1}
      dth[0] = m[0];
#pragma unroll
      for (int k = 1; k < P; k++) dth[k] = m[k] - m[k - 1];
    }
    const float div = 1.f / (float)(n - 1);
    float prev = 0.f;
#pragma unroll
    for (int k = 0; k < n; k++) {
      float cur = k < n - 1 ? m[k] : 0.f;
      float x = fr + (float)k;
      m[k] = div * (x * cur + ((float)n - x) * prev);
      prev = cur;
    }
  }
  if (P == 2) {
    dth[0] = 1.f;
    dth[1] = -1.f;
  }
#pragma unroll
  for (int k = 0; k < P; k++) th[k] = m[k];
}

// Grid coordinate of one atom along one axis: u = K * (frac), with frac
// taken from the minimal-image position so it lies in [0, 1].
__device__ __forceinline__ void grid_coord(const PmeArgs &a, int axis, double w,
                                           int &iu, float &fr) {
  double f = (w - a.box.min[axis] + a.box.origin[axis]) * a.inv_L[axis];
  f -= floor(f);
  double u = f * a.K[axis];
  double fl = floor(u);
  iu = (int)fl;
  fr = (float)(u - fl);
  if (iu >= a.K[axis]) iu -= a.K[axis];
}

// Spread: L lanes per atom (L = order rounded up to a power of two); lane
// kx < P adds the P^2 points of its x plane.
template <int P, int L>
__device__ __forceinline__ void spread_body(const PmeArgs &a, Blk b) {
  const double *__restrict__ pos = a.pos;
  const double *__restrict__ charge = a.charge;
  long long *__restrict__ grid = a.grid_fixed;
  const int gt = b.x * blockDim.x + threadIdx.x;
  const int t = gt / L, kx = gt & (L - 1);
  if (t >= a.n || kx >= P) return;
  const int i = t;
  double wx, wy, wz;
  box_minpos(a.box, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], wx, wy, wz);
  int iu[3];
  float fr[3];
  grid_coord(a, 0, wx, iu[0], fr[0]);
  grid_coord(a, 1, wy, iu[1], fr[1]);
  grid_coord(a, 2, wz, iu[2], fr[2]);
  float thx[P], thy[P], thz[P], d[P];
  bspline<P>(fr[0], thx, d);
  bspline<P>(fr[1], thy, d);
  bspline<P>(fr[2], thz, d);
  // this lane's x weight without a dynamically indexed array
  float tx = thx[0];
#pragma unroll
  for (int k = 1; k < P; k++)
    if (kx == k) tx = thx[k];
  int gx = iu[0] - kx;
  if (gx < 0) gx += a.K[0];
  const double qx = charge[i] * (double)tx;
#pragma unroll
  for (int ky = 0; ky < P; ky++) {
    int gy = iu[1] - ky;
    if (gy < 0) gy += a.K[1];
    const double qxy = qx * (double)thy[ky];
    long long *row = grid + ((size_t)gx * a.K[1] + gy) * a.K[2];
#pragma unroll
    for (int kz = 0; kz < P; kz++) {
      int gz = iu[2] - kz;
      if (gz < 0) gz += a.K[2];
      red_add(&row[gz], to_fixed(qxy * (double)thz[kz], kGridScale));
    }
  }
}

template <int P, int L>
__global__ void __launch_bounds__(128) k_pme_spread(PmeArgs a) {
  spread_body<P, L>(a, own_blk());
}
template <int P, int L>
__global__ void __launch_bounds__(128)
k_pme_spread_batch(const PmeArgs *__restrict__ tab, const int *__restrict__ first, int nm) {
  const int m = batch_member(first, nm, blockIdx.x);
  spread_body<P, L>(tab[m], batch_blk(first, m));
}

// Converts the fixed-point charge grid to FP32 and clears it for the next
// spread (the grid is zero at allocation and after every conversion, so no
// separate clearing pass is needed).
struct GridConvArgs {
  int total;
  long long *g;
  float *out;
};
__device__ __forceinline__ void fixed_to_float_body(const GridConvArgs &a, Blk b) {
  int i = b.x * blockDim.x + threadIdx.x;
  if (i < a.total) {
    a.out[i] = (float)((double)a.g[i] * (1.0 / kGridScale));
    a.g[i] = 0;
  }
}
__global__ void k_pme_fixed_to_float(GridConvArgs a) { fixed_to_float_body(a, own_blk()); }
__global__ void k_pme_fixed_to_float_batch(const GridConvArgs *__restrict__ tab,
                                           const int *__restrict__ first, int nm) {
  const int m = batch_member(first, nm, blockIdx.x);
  fixed_to_float_body(tab[m], batch_blk(first, m));
}

// Multiply by the influence function (precomputed for the box:
// exp(-pi^2 m^2/alpha^2)/(pi V m^2) |b(m)|^2, zero at m = 0); with em >= 1
// reduce the energy, with em == 2 also the virial.
// m index convention: m in [0, K/2] -> m, (K/2, K) -> m - K.
struct ConvolveArgs {
  int K0, K1, K2;
  double L0, L1, L2, alpha;
  const float *infl;
  float2 *c;
  long long *acc;
  int em;
};
__device__ __forceinline__ void convolve_body(const ConvolveArgs &A, Blk b) {
  const int K0 = A.K0, K1 = A.K1, K2 = A.K2, em = A.em;
  const double L0 = A.L0, L1 = A.L1, L2 = A.L2, alpha = A.alpha;
  const float *__restrict__ infl = A.infl;
  float2 *__restrict__ c = A.c;
  long long *__restrict__ acc = A.acc;
  const int Kh = K2 / 2 + 1;
  const int total = K0 * K1 * Kh;
  const int idx = b.x * blockDim.x + threadIdx.x;
  double e = 0, v[6] = {0, 0, 0, 0, 0, 0};
  if (idx < total) {
    const float g = infl[idx];
    const float2 f = c[idx];
    c[idx] = make_float2(g * f.x, g * f.y);
    if (em) {
      const int mz = idx % Kh;
      const double w = (mz == 0 || (K2 % 2 == 0 && mz == K2 / 2)) ? 1.0 : 2.0;
      const double f2 = (double)f.x * f.x + (double)f.y * f.y;
      const double emode = 0.5 * w * (double)g * f2;
      e = emode;
      if (em == 2 && g != 0.f) {
        const int my_ = (idx / Kh) % K1, mx_ = idx / (Kh * K1);
        const int mx = mx_ <= K0 / 2 ? mx_ : mx_ - K0;
        const int my = my_ <= K1 / 2 ? my_ : my_ - K1;
        const double hx = mx / L0, hy = my / L1, hz = mz / L2;
        const double h2 = hx * hx + hy * hy + hz * hz;
        const double pa = M_PI * M_PI / (alpha * alpha);
        const double cc = 2.0 * (1.0 / h2 + pa);
        v[0] = emode * (1.0 - cc * hx * hx);
        v[1] = -emode * cc * hx * hy;
        v[2] = -emode * cc * hx * hz;
        v[3] = emode * (1.0 - cc * hy * hy);
        v[4] = -emode * cc * hy * hz;
        v[5] = emode * (1.0 - cc * hz * hz);
      }
    }
  }
  if (!em) return;
  e = warp_sum(e);
  if (em == 2)
    for (int q = 0; q < 6; q++) v[q] = warp_sum(v[q]);
  if ((threadIdx.x & 31) == 0) {
    red_add(&acc[ACC_COULOMB], to_fixed(e, kEnergyScale));
    if (em == 2) {
      const int map[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
      for (int q = 0; q < 9; q++) red_add(&acc[ACC_VIRIAL + q], to_fixed(v[map[q]], kEnergyScale));
    }
  }
}
__global__ void k_pme_convolve(ConvolveArgs a) { convolve_body(a, own_blk()); }
__global__ void k_pme_convolve_batch(const ConvolveArgs *__restrict__ tab,
                                     const int *__restrict__ first, int nm) {
  const int m = batch_member(first, nm, blockIdx.x);
  convolve_body(tab[m], batch_blk(first, m));
}

// Gather: L lanes per atom, lane kx < P sums its x plane; the partial
// forces are reduced over the lanes with shuffles.
template <int P, int L>
__device__ __forceinline__ void gather_body(const PmeArgs &a, Blk b) {
  const double *__restrict__ pos = a.pos;
  const double *__restrict__ charge = a.charge;
  const float *__restrict__ phi = a.phi;
  long long *__restrict__ force = a.force;
  const int gt = b.x * blockDim.x + threadIdx.x;
  const int t = gt / L, kx = gt & (L - 1);
  const int i = t;
  const bool valid = t < a.n;
  float sx = 0.f, sy = 0.f, sz = 0.f;
  if (valid) {
    double wx, wy, wz;
    box_minpos(a.box, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], wx, wy, wz);
    int iu[3];
    float fr[3];
    grid_coord(a, 0, wx, iu[0], fr[0]);
    grid_coord(a, 1, wy, iu[1], fr[1]);
    grid_coord(a, 2, wz, iu[2], fr[2]);
    float thx[P], dthx[P], thy[P], dthy[P], thz[P], dthz[P];
    bspline<P>(fr[0], thx, dthx);
    bspline<P>(fr[1], thy, dthy);
    bspline<P>(fr[2], thz, dthz);
    if (kx < P) {
      float tx = thx[0], dtx = dthx[0];
#pragma unroll
      for (int k = 1; k < P; k++)
        if (kx == k) {
          tx = thx[k];
          dtx = dthx[k];
        }
      int gx = iu[0] - kx;
      if (gx < 0) gx += a.K[0];
#pragma unroll
      for (int ky = 0; ky < P; ky++) {
        int gy = iu[1] - ky;
        if (gy < 0) gy += a.K[1];
        const float *row = phi + ((size_t)gx * a.K[1] + gy) * a.K[2];
        const float txy = tx * thy[ky];
        const float dxy = dtx * thy[ky];
        const float txdy = tx * dthy[ky];
#pragma unroll
        for (int kz = 0; kz < P; kz++) {
          int gz = iu[2] - kz;
          if (gz < 0) gz += a.K[2];
          const float v = __ldg(&row[gz]);
          sx += dxy * thz[kz] * v;
          sy += txdy * thz[kz] * v;
          sz += txy * dthz[kz] * v;
        }
      }
    }
  }
#pragma unroll
  for (int o = L / 2; o > 0; o >>= 1) {
    sx += __shfl_xor_sync(0xffffffffu, sx, o);
    sy += __shfl_xor_sync(0xffffffffu, sy, o);
    sz += __shfl_xor_sync(0xffffffffu, sz, o);
  }
  if (valid && kx == 0) {
    const double q = charge[i];
    red_add(&force[i], to_fixed(-q * (double)sx * a.K[0] * a.inv_L[0], kForceScale));
    red_add(&force[a.n + i], to_fixed(-q * (double)sy * a.K[1] * a.inv_L[1], kForceScale));
    red_add(&force[2 * a.n + i], to_fixed(-q * (double)sz * a.K[2] * a.inv_L[2], kForceScale));
  }
}

template <int P, int L>
__global__ void __launch_bounds__(128) k_pme_gather(PmeArgs a) {
  gather_body<P, L>(a, own_blk());
}
template <int P, int L>
__global__ void __launch_bounds__(128)
k_pme_gather_batch(const PmeArgs *__restrict__ tab, const int *__restrict__ first, int nm) {
  const int m = batch_member(first, nm, blockIdx.x);
  gather_body<P, L>(tab[m], batch_blk(first, m));
}

// correctionTerm, NonbondedFullEwaldSystemForce.h:1092-1131, FP64.
struct CorrectionArgs {
  Box box;
  int nexcl;
  const int *ex;
  const double *pos, *charge;
  double alpha, csf;
  int n;
  long long *force, *acc;
  int em;
};
__device__ __forceinline__ void correction_body(const CorrectionArgs &A, Blk b) {
  const Box &box = A.box;
  const int nexcl = A.nexcl, n = A.n, em = A.em;
  const double alpha = A.alpha, csf = A.csf;
  const int *__restrict__ ex = A.ex;
  const double *__restrict__ pos = A.pos;
  const double *__restrict__ charge = A.charge;
  long long *__restrict__ force = A.force;
  long long *__restrict__ acc = A.acc;
  int k = b.x * blockDim.x + threadIdx.x;
  double e = 0, v[6] = {0, 0, 0, 0, 0, 0};
  if (k < nexcl) {
    int a1 = ex[3 * k], a2 = ex[3 * k + 1], cl = ex[3 * k + 2];
    double dx, dy, dz;
    double r2 = box_mindiff(box, pos[3 * a1], pos[3 * a1 + 1], pos[3 * a1 + 2],
                            pos[3 * a2], pos[3 * a2 + 1], pos[3 * a2 + 2], dx, dy, dz);
    double qq = charge[a1] * charge[a2];
    if (cl == PMGPU_EXCL_MODIFIED) qq *= 1 - csf;
    double r = sqrt(r2);
    double rr = 1 / r;
    // the reference's erf() here is the C library's (bit-exact against it)
    double ee = erf(alpha * r) * rr;
    e = -qq * ee;
    double a2pi = 2.0 * alpha / sqrt(M_PI);
    double g = qq * (a2pi * exp(-(alpha * alpha) * r2) - ee) * rr * rr;
    double fx = dx * g, fy = dy * g, fz = dz * g;
    red_add(&force[a1], to_fixed(-fx, kForceScale));
    red_add(&force[n + a1], to_fixed(-fy, kForceScale));
    red_add(&force[2 * n + a1], to_fixed(-fz, kForceScale));
    red_add(&force[a2], to_fixed(fx, kForceScale));
    red_add(&force[n + a2], to_fixed(fy, kForceScale));
    red_add(&force[2 * n + a2], to_fixed(fz, kForceScale));
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
    red_add(&acc[ACC_COULOMB], to_fixed(e, kEnergyScale));
    if (em == 2) {
      const int map[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
      for (int q = 0; q < 9; q++) red_add(&acc[ACC_VIRIAL + q], to_fixed(v[map[q]], kEnergyScale));
    }
  }
}

__global__ void k_ewald_correction(CorrectionArgs a) { correction_body(a, own_blk()); }
__global__ void k_ewald_correction_batch(const CorrectionArgs *__restrict__ tab,
                                         const int *__restrict__ first, int nm) {
  const int m = batch_member(first, nm, blockIdx.x);
  correction_body(tab[m], batch_blk(first, m));
}

// ------------------------------------------------------------ host side
// |b(m)|^2 = 1 / |sum_{k=0}^{p-2} M_p(k+1) exp(2 pi i m k / K)|^2
// (Essmann et al. eq. 4.4), with the usual fix for the zero of the
// denominator at odd orders (average of the neighbours).
static void bspline_moduli(int K, int p, std::vector<float> &out) {
  std::vector<double> M(p + 1, 0.0);
  // M_p at integer points 1..p-1 by the recursion on a unit fractional part
  std::vector<double> m(p, 0.0);
  m[0] = 0.0;  // fr = 0
  m[1] = 1.0;
  for (int n = 3; n <= p; n++) {
    double prev = 0.0;
    for (int k = 0; k < n; k++) {
      double cur = k < n - 1 ? m[k] : 0.0;
      double x = (double)k;
      m[k] = (x * cur + ((double)n - x) * prev) / (double)(n - 1);
      prev = cur;
    }
  }
  // m[k] = M_p(k) for k = 0..p-1
  std::vector<double> mod(K);
  for (int i = 0; i < K; i++) {
    double sr = 0, si = 0;
    for (int k = 0; k < p - 1; k++) {
      double arg = 2.0 * M_PI * i * k / K;
      sr += m[k + 1] * cos(arg);
      si += m[k + 1] * sin(arg);
    }
    mod[i] = sr * sr + si * si;
  }
  for (int i = 0; i < K; i++)
    if (mod[i] < 1e-7) mod[i] = 0.5 * (mod[(i - 1 + K) % K] + mod[(i + 1) % K]);
  out.resize(K);
  for (int i = 0; i < K; i++) out[i] = (float)(1.0 / mod[i]);
}

int pme_init(System *s, Force *f) {
  if (!s->box.periodic) return fail(PMGPU_ERR_UNSUPPORTED, "PME needs a periodic box");
  if (f->order < 2 || f->order > kMaxOrder)
    return fail(PMGPU_ERR_ARG, "PME order must be in [2, 8]");
  for (int a = 0; a < 3; a++)
    if (f->grid[a] < f->order || f->grid[a] > 1024)
      return fail(PMGPU_ERR_ARG, "PME grid dimension out of range");
  if (!(f->ewald_flags & PMGPU_EWALD_RECIPROCAL)) return PMGPU_OK;
  int K0 = f->grid[0], K1 = f->grid[1], K2 = f->grid[2];
  size_t nreal = (size_t)K0 * K1 * K2;
  size_t ncplx = (size_t)K0 * K1 * (K2 / 2 + 1);
  PM_CHECK(dev_alloc(s, &f->d_grid, sizeof(float) * nreal));
  PM_CHECK(dev_alloc(s, &f->d_grid_fixed, sizeof(long long) * nreal));
  PM_CUDA(cudaMemsetAsync(f->d_grid_fixed, 0, sizeof(long long) * nreal, s->stream));
  PM_CHECK(dev_alloc(s, &f->d_cgrid, sizeof(float2) * ncplx));
  {
    // influence function of the box (fixed for the life of the system)
    std::vector<float> bm[3];
    for (int a = 0; a < 3; a++) bspline_moduli(f->grid[a], f->order, bm[a]);
    const int Kh = K2 / 2 + 1;
    const double L0 = s->box.e[0], L1 = s->box.e[1], L2 = s->box.e[2], V = s->box.V;
    const double pa = M_PI * M_PI / (f->alpha * f->alpha);
    std::vector<float> g(ncplx);
    for (int mx_ = 0; mx_ < K0; mx_++)
      for (int my_ = 0; my_ < K1; my_++)
        for (int mz = 0; mz < Kh; mz++) {
          const int mx = mx_ <= K0 / 2 ? mx_ : mx_ - K0;
          const int my = my_ <= K1 / 2 ? my_ : my_ - K1;
          const size_t idx = ((size_t)mx_ * K1 + my_) * Kh + mz;
          if (mx == 0 && my == 0 && mz == 0) {
            g[idx] = 0.f;
            continue;
          }
          const double hx = mx / L0, hy = my / L1, hz = mz / L2;
          const double h2 = hx * hx + hy * hy + hz * hz;
          g[idx] = (float)(std::exp(-pa * h2) / (M_PI * V * h2) * (double)bm[0][mx_] *
                           (double)bm[1][my_] * (double)bm[2][mz]);
        }
    PM_CHECK(dev_alloc(s, &f->d_influence, sizeof(float) * ncplx));
    PM_CUDA(cudaMemcpyAsync(f->d_influence, g.data(), sizeof(float) * ncplx,
                            cudaMemcpyHostToDevice, s->stream));
    PM_CUDA(cudaStreamSynchronize(s->stream));
  }
  // cuFFT plans without their own work area: one stream-ordered work area
  // serves both (they run back to back on the system's stream).  A pair
  // left by an ended system of the same grid is taken from the context
  // first.
  size_t ws_r2c = 0, ws_c2r = 0;
  bool reused = false;
  {
    std::lock_guard<std::mutex> lock(s->ctx->fft_mu);
    auto &pool = s->ctx->fft_free;
    for (size_t k = 0; k < pool.size(); k++)
      if (pool[k].dims[0] == K0 && pool[k].dims[1] == K1 && pool[k].dims[2] == K2) {
        f->plan_r2c = pool[k].r2c;
        f->plan_c2r = pool[k].c2r;
        ws_r2c = ws_c2r = pool[k].work;
        pool.erase(pool.begin() + k);
        reused = true;
        break;
      }
  }
  if (!reused &&
      (cufftCreate(&f->plan_r2c) != CUFFT_SUCCESS || cufftCreate(&f->plan_c2r) != CUFFT_SUCCESS ||
       cufftSetAutoAllocation(f->plan_r2c, 0) != CUFFT_SUCCESS ||
       cufftSetAutoAllocation(f->plan_c2r, 0) != CUFFT_SUCCESS ||
       cufftMakePlan3d(f->plan_r2c, K0, K1, K2, CUFFT_R2C, &ws_r2c) != CUFFT_SUCCESS ||
       cufftMakePlan3d(f->plan_c2r, K0, K1, K2, CUFFT_C2R, &ws_c2r) != CUFFT_SUCCESS))
    return fail(PMGPU_ERR_CUDA, "cuFFT plan creation failed");
  f->fft_work_bytes = std::max(ws_r2c, ws_c2r);
  PM_CHECK(dev_alloc(s, &f->d_fft_work, f->fft_work_bytes));
  if (cufftSetWorkArea(f->plan_r2c, f->d_fft_work) != CUFFT_SUCCESS ||
      cufftSetWorkArea(f->plan_c2r, f->d_fft_work) != CUFFT_SUCCESS ||
      cufftSetStream(f->plan_r2c, s->stream) != CUFFT_SUCCESS ||
      cufftSetStream(f->plan_c2r, s->stream) != CUFFT_SUCCESS)
    return fail(PMGPU_ERR_CUDA, "cuFFT work area / stream set-up failed");
  return PMGPU_OK;
}

int pme_free(System *s, Force *f) {
  if (f->plan_r2c && f->plan_c2r && s->ctx) {
    // back to the context for the next system of this grid (its next user
    // sets the work area and the stream again)
    std::lock_guard<std::mutex> lock(s->ctx->fft_mu);
    s->ctx->fft_free.push_back(
        {{f->grid[0], f->grid[1], f->grid[2]}, f->plan_r2c, f->plan_c2r, f->fft_work_bytes});
  } else {
    if (f->plan_r2c) cufftDestroy(f->plan_r2c);
    if (f->plan_c2r) cufftDestroy(f->plan_c2r);
  }
  f->plan_r2c = f->plan_c2r = 0;
  void *ptrs[] = {f->d_grid, f->d_grid_fixed, f->d_cgrid, f->d_influence, f->d_fft_work,
                  f->d_ewtab};
  for (void *p : ptrs) dev_free(s, p);
  f->d_grid = nullptr; f->d_grid_fixed = nullptr; f->d_cgrid = nullptr;
  f->d_influence = nullptr;
  f->d_ewtab = nullptr;
  f->terms.ewtab = nullptr;
  f->d_fft_work = nullptr;
  return PMGPU_OK;
}

template <int P>
static void launch_spread_gather(const PmeArgs &a, System *s, Force *f,
                                 int gather) {
  constexpr int L = P <= 4 ? 4 : 8;
  const int nb = (int)(((long long)a.n * L + 127) / 128);
  if (!gather)
    k_pme_spread<P, L><<<nb, 128, 0, s->stream>>>(a);
  else
    k_pme_gather<P, L><<<nb, 128, 0, s->stream>>>(a);
}

static void spread_gather(const PmeArgs &a, System *s, Force *f,
                          int gather) {
  switch (f->order) {
    case 2: launch_spread_gather<2>(a, s, f, gather); break;
    case 3: launch_spread_gather<3>(a, s, f, gather); break;
    case 4: launch_spread_gather<4>(a, s, f, gather); break;
    case 5: launch_spread_gather<5>(a, s, f, gather); break;
    case 6: launch_spread_gather<6>(a, s, f, gather); break;
    case 7: launch_spread_gather<7>(a, s, f, gather); break;
    default: launch_spread_gather<8>(a, s, f, gather); break;
  }
}

// em: 0 forces only, 1 + energy, 2 + energy and virial.
int pme_reciprocal(System *s, Force *f, int em) {
  int n = s->n;
  if (n == 0) return PMGPU_OK;
  PmeArgs a;
  a.box = s->box;
  a.n = n;
  for (int d = 0; d < 3; d++) {
    a.K[d] = f->grid[d];
    a.inv_L[d] = 1.0 / s->box.e[d];
  }
  a.order = f->order;
  a.pos = s->d_pos;
  a.charge = s->d_charge;
  a.grid_fixed = f->d_grid_fixed;
  a.phi = f->d_grid;
  a.force = s->d_force;
  int K0 = f->grid[0], K1 = f->grid[1], K2 = f->grid[2];
  size_t nreal = (size_t)K0 * K1 * K2;
  size_t ncplx = (size_t)K0 * K1 * (K2 / 2 + 1);
  // Atoms are spread and gathered in their own order: PME does not wait for
  // the pair list's sort, so it runs beside the list work of a step.  The
  // plans run on whichever stream this evaluation uses.
  if (cufftSetStream(f->plan_r2c, s->stream) != CUFFT_SUCCESS ||
      cufftSetStream(f->plan_c2r, s->stream) != CUFFT_SUCCESS)
    return fail(PMGPU_ERR_CUDA, "cufftSetStream failed");
  spread_gather(a, s, f, 0);
  k_pme_fixed_to_float<<<(int)((nreal + 255) / 256), 256, 0, s->stream>>>(
      GridConvArgs{(int)nreal, f->d_grid_fixed, f->d_grid});
  if (cufftExecR2C(f->plan_r2c, f->d_grid, (cufftComplex *)f->d_cgrid) != CUFFT_SUCCESS)
    return fail(PMGPU_ERR_CUDA, "cufftExecR2C failed");
  k_pme_convolve<<<(int)((ncplx + 255) / 256), 256, 0, s->stream>>>(
      ConvolveArgs{K0, K1, K2, s->box.e[0], s->box.e[1], s->box.e[2], f->alpha, f->d_influence,
                   f->d_cgrid, s->d_acc, em});
  if (cufftExecC2R(f->plan_c2r, (cufftComplex *)f->d_cgrid, f->d_grid) != CUFFT_SUCCESS)
    return fail(PMGPU_ERR_CUDA, "cufftExecC2R failed");
  spread_gather(a, s, f, 1);
  PM_CUDA(cudaGetLastError());
  return PMGPU_OK;
}

int ewald_correction(System *s, Force *f, int em) {
  if (s->n_excl == 0) return PMGPU_OK;
  k_ewald_correction<<<(s->n_excl + 127) / 128, 128, 0, s->stream>>>(
      CorrectionArgs{s->box, s->n_excl, s->d_excl_pairs, s->d_pos, s->d_charge, f->alpha,
                     s->coulomb_scaling, s->n, s->d_force, s->d_acc, em});
  PM_CUDA(cudaGetLastError());
  return PMGPU_OK;
}

// ---------------------------------------------------------------- batches
// The PME chain and the Ewald correction of an ensemble's members as
// batched launches.  Members whose grids have the same dimensions form a
// bucket: their real and complex grids are slices of one buffer, and one
// batched cuFFT plan pair transforms the bucket at once.
struct PmeBucket {
  int K[3];
  std::vector<int> members;
  cufftHandle r2c = 0, c2r = 0;
  float *grid = nullptr;
  float2 *cgrid = nullptr;
};
struct PmeBatch {
  int order = 4;
  BatchTable<PmeArgs> atoms;  // spread and gather
  BatchTable<GridConvArgs> conv;
  BatchTable<ConvolveArgs> convolve[2];
  BatchTable<CorrectionArgs> corr[2];
  std::vector<PmeBucket> buckets;
  std::vector<System *> sys;
  std::vector<Force *> forces;
};

PmeBatch *pme_batch_new() { return new PmeBatch(); }

// Gives every member its own grids again and frees the buckets.
void pme_batch_free(PmeBatch *b) {
  if (!b) return;
  for (auto &bk : b->buckets) {
    for (int k : bk.members) {
      System *s = b->sys[k];
      Force *f = b->forces[k];
      const size_t nreal = (size_t)f->grid[0] * f->grid[1] * f->grid[2];
      const size_t ncplx = (size_t)f->grid[0] * f->grid[1] * (f->grid[2] / 2 + 1);
      f->d_grid = nullptr;
      f->d_cgrid = nullptr;
      dev_alloc(s, &f->d_grid, sizeof(float) * nreal);
      dev_alloc(s, &f->d_cgrid, sizeof(float2) * ncplx);
      s->graph_version++;  // graphs captured with the bucket's grids
    }
    if (bk.r2c) cufftDestroy(bk.r2c);
    if (bk.c2r) cufftDestroy(bk.c2r);
    if (bk.grid) cudaFree(bk.grid);
    if (bk.cgrid) cudaFree(bk.cgrid);
  }
  b->atoms.release();
  b->conv.release();
  for (int e = 0; e < 2; e++) {
    b->convolve[e].release();
    b->corr[e].release();
  }
  delete b;
}

int pme_batch_build(PmeBatch *b, System *const *m, int n, Force *const *fs) {
  b->sys.assign(m, m + n);
  b->forces.assign(fs, fs + n);
  b->order = fs[0]->order;
  // buckets by grid dimensions
  std::vector<int> bucket_of(n, -1);
  for (int k = 0; k < n; k++) {
    const Force *f = fs[k];
    if (f->order != b->order || !(f->ewald_flags & PMGPU_EWALD_RECIPROCAL))
      return fail(PMGPU_ERR_UNSUPPORTED, "ensemble members need one PME order");
    int found = -1;
    for (size_t q = 0; q < b->buckets.size(); q++)
      if (b->buckets[q].K[0] == f->grid[0] && b->buckets[q].K[1] == f->grid[1] &&
          b->buckets[q].K[2] == f->grid[2])
        found = (int)q;
    if (found < 0) {
      b->buckets.push_back(PmeBucket());
      found = (int)b->buckets.size() - 1;
      for (int a = 0; a < 3; a++) b->buckets[found].K[a] = f->grid[a];
    }
    b->buckets[found].members.push_back(k);
    bucket_of[k] = found;
  }
  for (auto &bk : b->buckets) {
    const int B = (int)bk.members.size();
    const size_t G = (size_t)bk.K[0] * bk.K[1] * bk.K[2];
    const size_t Gc = (size_t)bk.K[0] * bk.K[1] * (bk.K[2] / 2 + 1);
    PM_CUDA(cudaMalloc(&bk.grid, sizeof(float) * G * B));
    PM_CUDA(cudaMalloc(&bk.cgrid, sizeof(float2) * Gc * B));
    int dims[3] = {bk.K[0], bk.K[1], bk.K[2]};
    if (cufftPlanMany(&bk.r2c, 3, dims, nullptr, 1, (int)G, nullptr, 1, (int)Gc, CUFFT_R2C, B) !=
            CUFFT_SUCCESS ||
        cufftPlanMany(&bk.c2r, 3, dims, nullptr, 1, (int)Gc, nullptr, 1, (int)G, CUFFT_C2R, B) !=
            CUFFT_SUCCESS)
      return fail(PMGPU_ERR_CUDA, "batched cuFFT plan creation failed");
    for (int q = 0; q < B; q++) {
      System *s = m[bk.members[q]];
      Force *f = fs[bk.members[q]];
      PM_CUDA(cudaStreamSynchronize(s->stream));
      dev_free(s, f->d_grid);
      dev_free(s, f->d_cgrid);
      f->d_grid = bk.grid + G * q;
      f->d_cgrid = bk.cgrid + Gc * q;
      s->graph_version++;  // graphs captured with the member's own grids
    }
  }
  // argument tables in member order
  b->atoms.clear();
  b->conv.clear();
  for (int e = 0; e < 2; e++) {
    b->convolve[e].clear();
    b->corr[e].clear();
  }
  int L = b->order <= 4 ? 4 : 8;
  for (int k = 0; k < n; k++) {
    System *s = m[k];
    Force *f = fs[k];
    PmeArgs a;
    a.box = s->box;
    a.n = s->n;
    for (int d = 0; d < 3; d++) {
      a.K[d] = f->grid[d];
      a.inv_L[d] = 1.0 / s->box.e[d];
    }
    a.order = f->order;
    a.pos = s->d_pos;
    a.charge = s->d_charge;
    a.grid_fixed = f->d_grid_fixed;
    a.phi = f->d_grid;
    a.force = s->d_force;
    b->atoms.add(a, (int)(((long long)s->n * L + 127) / 128));
    const size_t nreal = (size_t)f->grid[0] * f->grid[1] * f->grid[2];
    const size_t ncplx = (size_t)f->grid[0] * f->grid[1] * (f->grid[2] / 2 + 1);
    b->conv.add(GridConvArgs{(int)nreal, f->d_grid_fixed, f->d_grid}, (int)((nreal + 255) / 256));
    for (int e = 0; e < 2; e++) {
      b->convolve[e].add(ConvolveArgs{f->grid[0], f->grid[1], f->grid[2], s->box.e[0],
                                      s->box.e[1], s->box.e[2], f->alpha, f->d_influence,
                                      f->d_cgrid, s->d_acc, e},
                         (int)((ncplx + 255) / 256));
      b->corr[e].add(CorrectionArgs{s->box, s->n_excl, s->d_excl_pairs, s->d_pos, s->d_charge,
                                    f->alpha, s->coulomb_scaling, s->n, s->d_force, s->d_acc, e},
                     (s->n_excl + 127) / 128);
    }
  }
  PM_CUDA(b->atoms.upload());
  PM_CUDA(b->conv.upload());
  for (int e = 0; e < 2; e++) {
    PM_CUDA(b->convolve[e].upload());
    PM_CUDA(b->corr[e].upload());
  }
  return PMGPU_OK;
}

template <int P>
static void pme_batch_atoms(PmeBatch *b, int gather, cudaStream_t st) {
  constexpr int L = P <= 4 ? 4 : 8;
  BatchTable<PmeArgs> &t = b->atoms;
  if (!t.total()) return;
  if (!gather)
    k_pme_spread_batch<P, L><<<t.total(), 128, 0, st>>>(t.d, t.d_first, t.members());
  else
    k_pme_gather_batch<P, L><<<t.total(), 128, 0, st>>>(t.d, t.d_first, t.members());
}

static void pme_batch_sg(PmeBatch *b, int gather, cudaStream_t st) {
  switch (b->order) {
    case 2: pme_batch_atoms<2>(b, gather, st); break;
    case 3: pme_batch_atoms<3>(b, gather, st); break;
    case 4: pme_batch_atoms<4>(b, gather, st); break;
    case 5: pme_batch_atoms<5>(b, gather, st); break;
    case 6: pme_batch_atoms<6>(b, gather, st); break;
    case 7: pme_batch_atoms<7>(b, gather, st); break;
    default: pme_batch_atoms<8>(b, gather, st); break;
  }
}

// The reciprocal term of every member (pme_reciprocal of each), em as
// there.
int pme_batch_reciprocal(PmeBatch *b, int em, cudaStream_t st, long long *launched) {
  const int nm = b->atoms.members();
  if (!nm) return PMGPU_OK;
  *launched += 4;  // spread, fixed->float, convolve, gather (+ cuFFT's)
  pme_batch_sg(b, 0, st);
  k_pme_fixed_to_float_batch<<<b->conv.total(), 256, 0, st>>>(b->conv.d, b->conv.d_first, nm);
  for (auto &bk : b->buckets) {
    if (cufftSetStream(bk.r2c, st) != CUFFT_SUCCESS ||
        cufftExecR2C(bk.r2c, bk.grid, (cufftComplex *)bk.cgrid) != CUFFT_SUCCESS)
      return fail(PMGPU_ERR_CUDA, "batched cufftExecR2C failed");
  }
  BatchTable<ConvolveArgs> &cv = b->convolve[em ? 1 : 0];
  k_pme_convolve_batch<<<cv.total(), 256, 0, st>>>(cv.d, cv.d_first, nm);
  for (auto &bk : b->buckets) {
    if (cufftSetStream(bk.c2r, st) != CUFFT_SUCCESS ||
        cufftExecC2R(bk.c2r, (cufftComplex *)bk.cgrid, bk.grid) != CUFFT_SUCCESS)
      return fail(PMGPU_ERR_CUDA, "batched cufftExecC2R failed");
  }
  pme_batch_sg(b, 1, st);
  PM_CUDA(cudaGetLastError());
  return PMGPU_OK;
}

int pme_batch_buckets(const PmeBatch *b) { return (int)b->buckets.size(); }

int pme_batch_correction(PmeBatch *b, int em, cudaStream_t st, long long *launched) {
  BatchTable<CorrectionArgs> &t = b->corr[em ? 1 : 0];
  if (!t.members() || !t.total()) return PMGPU_OK;
  *launched += 1;
  k_ewald_correction_batch<<<t.total(), 128, 0, st>>>(t.d, t.d_first, t.members());
  PM_CUDA(cudaGetLastError());
  return PMGPU_OK;
}

}  // namespace pmgpu
