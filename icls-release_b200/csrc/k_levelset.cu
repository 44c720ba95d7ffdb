// k_levelset.cu — level-set kernels of the ICLS hot path (FP64, -fmad=false).
//
//   tube_construction  levelset.f90:87-197
//   HOUC5_nb/WENO5_nb  hyperPDE.f90:397-800, fused with RK_nb
//                      levelset.f90:342-367 and boundsls bound.f90:386-483
//   ls_reinit          levelset.f90:619-882 with WENO5_reinit/WENO5_deri
//                      hyperPDE.f90:2646-2746, 2932-3197
//   inflation          levelset.f90:407-582
//   update_materials   misc.f90:79-290 with Heaviside 'trig' misc.f90:297-464
//
// Halo handling: instead of a separate boundsls pass, every output cell of
// the (-2:i1+2,-2:j1+2,-2:k1+2) array is computed from its periodic source
// column (I,J) = wrap(i,j); the wall rows k=0 and k=k1 evaluate the two
// interior values they extrapolate from.  This reproduces boundsls
// (z-extrapolation, then periodic x, then periodic y) exactly, because the
// inputs already satisfy the periodic halo invariant.
#include "ctx.h"

namespace icls {

namespace {

constexpr int NT = 256;

inline unsigned nblocks(long long n, int nt = NT) { return (unsigned)((n + nt - 1) / nt); }

__device__ __forceinline__ double clipNB(double x, double NB) {
  return x > NB ? NB : (x < -NB ? -NB : x);
}

__device__ __forceinline__ void decodeL(const Params& p, long long n, int& i, int& j, int& k) {
  i = (int)(n % p.nLx) - 2;
  long long r = n / p.nLx;
  j = (int)(r % p.nLy) - 2;
  k = (int)(r / p.nLy) - 2;
}
__device__ __forceinline__ void decodeC(const Params& p, long long n, int& i, int& j, int& k) {
  i = (int)(n % p.nCx);
  long long r = n / p.nCx;
  j = (int)(r % p.nCy);
  k = (int)(r / p.nCy);
}
__device__ __forceinline__ bool interior(const Params& p, int i, int j, int k) {
  return i >= 1 && i <= p.imax && j >= 1 && j <= p.jmax && k >= 1 && k <= p.kmax;
}

// ---------------------------------------------------------------- tube
__global__ void __launch_bounds__(NT) k_tube(Params p, const double* __restrict__ in,
                                             double* __restrict__ out, uint8_t* __restrict__ mask,
                                             long long* __restrict__ cnt) {
  const long long n = blockIdx.x * (long long)NT + threadIdx.x;
  int m = 0;
  if (n < p.nL) {
    int i, j, k;
    decodeL(p, n, i, j, k);
    const int I = wrapx(p, i), J = wrapy(p, j);
    const double NB = p.NB;
    double val;
    if (k == 0)
      val = 2. * clipNB(in[idxL(p, I, J, 1)], NB) - clipNB(in[idxL(p, I, J, 2)], NB);
    else if (k == p.k1)
      val = 2. * clipNB(in[idxL(p, I, J, p.kmax)], NB) - clipNB(in[idxL(p, I, J, p.kmax - 1)], NB);
    else
      val = clipNB(in[idxL(p, I, J, k)], NB);
    out[n] = val;
    if (interior(p, i, j, k)) {
      const double c0 = clipNB(in[n], NB);
      if (fabs(c0) < NB) {
        m = 1;
      } else {
        double xs = 0., ys = 0., zs = 0.;
        for (int d = -2; d <= 2; ++d) xs += fabs(clipNB(in[idxL(p, i + d, j, k)], NB)) - NB;
        for (int d = -2; d <= 2; ++d) ys += fabs(clipNB(in[idxL(p, i, j + d, k)], NB)) - NB;
        for (int d = -2; d <= 2; ++d) zs += fabs(clipNB(in[idxL(p, i, j, k + d)], NB)) - NB;
        m = (xs == 0. && ys == 0. && zs == 0.) ? 0 : 1;
      }
      mask[idxI(p, i, j, k)] = (uint8_t)m;
    }
  }
  int bs = block_sum<int, NT>(m);
  if (threadIdx.x == 0 && bs) atomicAdd((unsigned long long*)cnt, (unsigned long long)bs);
}

// ------------------------------------------------------- advection RHS
// dfdt of HOUC5_nb (hyperPDE.f90:397-495) or WENO5_nb (503-800) at (i,j,k)
template <int SCHEME>
__device__ __forceinline__ double adv_rhs(const Params& p, const double* __restrict__ phi,
                                          double vu, double vv, double vw, int i, int j, int k) {
  const double dx = p.dx, dy = p.dy, dz = p.dz;
  const long long c = idxL(p, i, j, k);
  const long long sx = 1, sy = p.nLx, sz = (long long)p.nLx * p.nLy;
#define PH(o) phi[c + (o)]
  double udfdx, vdfdy, wdfdz, dfx, dfy, dfz;
  if (SCHEME == ICLS_HOUC5) {
    if (p.TwoD) {
      udfdx = 0.;
    } else {
      if (vu >= 0.)
        dfx = houc5_pos(PH(-3 * sx), PH(-2 * sx), PH(-sx), PH(0), PH(sx), PH(2 * sx));
      else
        dfx = houc5_neg(PH(3 * sx), PH(2 * sx), PH(sx), PH(0), PH(-sx), PH(-2 * sx));
      udfdx = -(vu * dfx / dx);
    }
    if (vv >= 0.)
      dfy = houc5_pos(PH(-3 * sy), PH(-2 * sy), PH(-sy), PH(0), PH(sy), PH(2 * sy));
    else
      dfy = houc5_neg(PH(3 * sy), PH(2 * sy), PH(sy), PH(0), PH(-sy), PH(-2 * sy));
    vdfdy = -(vv * dfy / dy);
  } else {
    if (p.TwoD) {
      udfdx = 0.;
    } else {
      if (vu >= 0.)
        dfx = weno5((PH(-2 * sx) - PH(-3 * sx)) / dx, (PH(-sx) - PH(-2 * sx)) / dx, (PH(0) - PH(-sx)) / dx,
                    (PH(sx) - PH(0)) / dx, (PH(2 * sx) - PH(sx)) / dx);
      else
        dfx = weno5((PH(3 * sx) - PH(2 * sx)) / dx, (PH(2 * sx) - PH(sx)) / dx, (PH(sx) - PH(0)) / dx,
                    (PH(0) - PH(-sx)) / dx, (PH(-sx) - PH(-2 * sx)) / dx);
      udfdx = -(vu * dfx);
    }
    // y uses dx, as in the reference (hyperPDE.f90:622-626)
    if (vv >= 0.)
      dfy = weno5((PH(-2 * sy) - PH(-3 * sy)) / dx, (PH(-sy) - PH(-2 * sy)) / dx, (PH(0) - PH(-sy)) / dx,
                  (PH(sy) - PH(0)) / dx, (PH(2 * sy) - PH(sy)) / dx);
    else
      dfy = weno5((PH(3 * sy) - PH(2 * sy)) / dx, (PH(2 * sy) - PH(sy)) / dx, (PH(sy) - PH(0)) / dx,
                  (PH(0) - PH(-sy)) / dx, (PH(-sy) - PH(-2 * sy)) / dx);
    vdfdy = -(vv * dfy);
  }
  if (k > 2 && k < p.kmax - 1) {
    if (SCHEME == ICLS_HOUC5) {
      if (vw >= 0.)
        dfz = houc5_pos(PH(-3 * sz), PH(-2 * sz), PH(-sz), PH(0), PH(sz), PH(2 * sz));
      else
        dfz = houc5_neg(PH(3 * sz), PH(2 * sz), PH(sz), PH(0), PH(-sz), PH(-2 * sz));
      wdfdz = -(vw * dfz / dz);
    } else {
      if (vw >= 0.)
        dfz = weno5((PH(-2 * sz) - PH(-3 * sz)) / dz, (PH(-sz) - PH(-2 * sz)) / dz, (PH(0) - PH(-sz)) / dz,
                    (PH(sz) - PH(0)) / dz, (PH(2 * sz) - PH(sz)) / dz);
      else
        dfz = weno5((PH(3 * sz) - PH(2 * sz)) / dz, (PH(2 * sz) - PH(sz)) / dz, (PH(sz) - PH(0)) / dz,
                    (PH(0) - PH(-sz)) / dz, (PH(-sz) - PH(-2 * sz)) / dz);
      wdfdz = -(vw * dfz);
    }
  } else if (k == 2 || k == p.kmax - 1) {  // HOUC3 near the walls
    if (vw >= 0.)
      dfz = (((1. / 6.) * PH(-2 * sz) - PH(-sz)) + (1. / 2.) * PH(0)) + (1. / 3.) * PH(sz);
    else
      dfz = ((-((1. / 6.) * PH(2 * sz)) + PH(sz)) - (1. / 2.) * PH(0)) - (1. / 3.) * PH(-sz);
    wdfdz = -(vw * dfz / dz);
  } else {  // first-order upwinding at k=1,kmax
    if (vw >= 0.) dfz = PH(0) - PH(-sz);
    else dfz = PH(sz) - PH(0);
    wdfdz = -(vw * dfz / dz);
  }
#undef PH
  return (udfdx + vdfdy) + wdfdz;
}

// RK_nb value of one cell: phi_in (+ factor*dt*dfdt on the band)
template <int SCHEME>
__device__ __forceinline__ double adv_val(const Params& p, int stage1, const double* __restrict__ phi0,
                                          const double* __restrict__ phis, double a, double b, double fdt,
                                          const double* __restrict__ vu, const double* __restrict__ vv,
                                          const double* __restrict__ vw, const uint8_t* __restrict__ mask,
                                          int I, int J, int k) {
  const long long n = idxL(p, I, J, k);
  double v = stage1 ? phi0[n] : a * phi0[n] + b * phis[n];
  if (k >= 1 && k <= p.kmax) {
    const long long q = idxI(p, I, J, k);
    if (mask[q]) v = v + fdt * adv_rhs<SCHEME>(p, phis, vu[q], vv[q], vw[q], I, J, k);
  }
  return v;
}

template <int SCHEME>
__global__ void __launch_bounds__(NT) k_adv_stage(Params p, int stage1, const double* __restrict__ phi0,
                                                  const double* __restrict__ phis, double a, double b,
                                                  double fdt, const double* __restrict__ vu,
                                                  const double* __restrict__ vv, const double* __restrict__ vw,
                                                  const uint8_t* __restrict__ mask, double* __restrict__ out) {
  const long long n = blockIdx.x * (long long)NT + threadIdx.x;
  if (n >= p.nL) return;
  int i, j, k;
  decodeL(p, n, i, j, k);
  const int I = wrapx(p, i), J = wrapy(p, j);
  double val;
  if (k == 0)
    val = 2. * adv_val<SCHEME>(p, stage1, phi0, phis, a, b, fdt, vu, vv, vw, mask, I, J, 1) -
          adv_val<SCHEME>(p, stage1, phi0, phis, a, b, fdt, vu, vv, vw, mask, I, J, 2);
  else if (k == p.k1)
    val = 2. * adv_val<SCHEME>(p, stage1, phi0, phis, a, b, fdt, vu, vv, vw, mask, I, J, p.kmax) -
          adv_val<SCHEME>(p, stage1, phi0, phis, a, b, fdt, vu, vv, vw, mask, I, J, p.kmax - 1);
  else
    val = adv_val<SCHEME>(p, stage1, phi0, phis, a, b, fdt, vu, vv, vw, mask, I, J, k);
  out[n] = val;
}

// ------------------------------------------------------------ reinit
// sgn(phi_0) of ls_reinit (levelset.f90:668-678)
__device__ __forceinline__ double reinit_sgn(const Params& p, double p0) {
  if (p0 < -p.dz) return -1.;
  if (p0 > p.dz) return 1.;
  return p0 / sqrt(p0 * p0 + p.dz * p.dz);
}

// RHS of WENO5_reinit at an interior cell (hyperPDE.f90:2646-2746)
__device__ __forceinline__ double reinit_rhs(const Params& p, const double* __restrict__ phi,
                                             const double* __restrict__ orig, int i, int j, int k) {
  const long long c = idxL(p, i, j, k);
  if (!(fabs(phi[c]) < p.NB + p.dz)) return 0.;
  const double dx = p.dx, dz = p.dz;
  const long long sx = 1, sy = p.nLx, sz = (long long)p.nLx * p.nLy;
#define PH(o) phi[c + (o)]
  double A = 0., B = 0., C, D, E, F;
  if (!p.TwoD) {
    A = weno5((PH(-2 * sx) - PH(-3 * sx)) / dx, (PH(-sx) - PH(-2 * sx)) / dx, (PH(0) - PH(-sx)) / dx,
              (PH(sx) - PH(0)) / dx, (PH(2 * sx) - PH(sx)) / dx);
    B = weno5((PH(3 * sx) - PH(2 * sx)) / dx, (PH(2 * sx) - PH(sx)) / dx, (PH(sx) - PH(0)) / dx,
              (PH(0) - PH(-sx)) / dx, (PH(-sx) - PH(-2 * sx)) / dx);
  }
  C = weno5((PH(-2 * sy) - PH(-3 * sy)) / dx, (PH(-sy) - PH(-2 * sy)) / dx, (PH(0) - PH(-sy)) / dx,
            (PH(sy) - PH(0)) / dx, (PH(2 * sy) - PH(sy)) / dx);
  D = weno5((PH(3 * sy) - PH(2 * sy)) / dx, (PH(2 * sy) - PH(sy)) / dx, (PH(sy) - PH(0)) / dx,
            (PH(0) - PH(-sy)) / dx, (PH(-sy) - PH(-2 * sy)) / dx);
  if (k >= 3 && k <= p.kmax - 2) {
    E = weno5((PH(-2 * sz) - PH(-3 * sz)) / dz, (PH(-sz) - PH(-2 * sz)) / dz, (PH(0) - PH(-sz)) / dz,
              (PH(sz) - PH(0)) / dz, (PH(2 * sz) - PH(sz)) / dz);
    F = weno5((PH(3 * sz) - PH(2 * sz)) / dz, (PH(2 * sz) - PH(sz)) / dz, (PH(sz) - PH(0)) / dz,
              (PH(0) - PH(-sz)) / dz, (PH(-sz) - PH(-2 * sz)) / dz);
  } else {
    E = (PH(0) - PH(-sz)) / dz;
    F = (PH(sz) - PH(0)) / dz;
  }
#undef PH
  const double s = reinit_sgn(p, orig[c]);
  double dydx, dydy, dydz;
  if (p.TwoD) {
    dydx = 0.;
  } else {
    if ((B * s < 0.) && ((A + B) * s < 0.)) dydx = B;
    else if ((A * s > 0.) && ((A + B) * s > 0.)) dydx = A;
    else dydx = 0.5 * (A + B);
  }
  if ((D * s < 0.) && ((C + D) * s < 0.)) dydy = D;
  else if ((C * s > 0.) && ((C + D) * s > 0.)) dydy = C;
  else dydy = 0.5 * (C + D);
  if ((F * s < 0.) && ((E + F) * s < 0.)) dydz = F;
  else if ((E * s > 0.) && ((E + F) * s > 0.)) dydz = E;
  else dydz = 0.5 * (E + F);
  return s * (1. - sqrt((dydx * dydx + dydy * dydy) + dydz * dydz));
}

// one SSP-RK3 stage value of ls_reinit (levelset.f90:800-810)
__device__ __forceinline__ double reinit_val(const Params& p, int stage, const double* __restrict__ phi0,
                                             const double* __restrict__ phis, const double* __restrict__ orig,
                                             double dtau, int I, int J, int k) {
  const long long n = idxL(p, I, J, k);
  const double rhs = (k >= 1 && k <= p.kmax) ? reinit_rhs(p, phis, orig, I, J, k) : 0.;
  if (stage == 1) return phi0[n] + dtau * rhs;
  if (stage == 2) return 3. / 4. * phi0[n] + 1. / 4. * (phis[n] + dtau * rhs);
  return 1. / 3. * phi0[n] + 2. / 3. * (phis[n] + dtau * rhs);
}

__global__ void __launch_bounds__(NT) k_reinit_stage(Params p, int stage, const double* __restrict__ phi0,
                                                     const double* __restrict__ phis,
                                                     const double* __restrict__ orig, double dtau,
                                                     double* __restrict__ out, int check_done,
                                                     DevScalars* __restrict__ dsc) {
  const long long n = blockIdx.x * (long long)NT + threadIdx.x;
  const int done = check_done ? dsc->reinit_done : 0;
  if (done) {
    // an iteration after convergence is the identity (levelset.f90:833-835)
    if (stage == 3 && n < p.nL) out[n] = phi0[n];
    return;
  }
  if (stage == 1 && n == 0) dsc->residual = 0.;
  double r = 0.;
  if (n < p.nL) {
    int i, j, k;
    decodeL(p, n, i, j, k);
    const int I = wrapx(p, i), J = wrapy(p, j);
    double val;
    if (k == 0)
      val = 2. * reinit_val(p, stage, phi0, phis, orig, dtau, I, J, 1) -
            reinit_val(p, stage, phi0, phis, orig, dtau, I, J, 2);
    else if (k == p.k1)
      val = 2. * reinit_val(p, stage, phi0, phis, orig, dtau, I, J, p.kmax) -
            reinit_val(p, stage, phi0, phis, orig, dtau, I, J, p.kmax - 1);
    else
      val = reinit_val(p, stage, phi0, phis, orig, dtau, I, J, k);
    out[n] = val;
    if (stage == 3) r = fabs(val - phi0[n]);
  }
  if (stage == 3) {
    double bm = block_max<double, NT>(r);
    if (threadIdx.x == 0) atomic_max_nonneg(&dsc->residual, bm);
  }
}

__global__ void k_reinit_reset(DevScalars* dsc, int maxiter) {
  dsc->reinit_done = 0;
  dsc->reinit_iters = maxiter;
  dsc->residual = 0.;
}
__global__ void k_reinit_check(DevScalars* dsc, int it, int maxiter, double thr) {
  if (dsc->reinit_done) return;
  if (dsc->residual < thr) {
    dsc->reinit_done = 1;
    dsc->reinit_iters = it;
  } else {
    dsc->reinit_iters = maxiter;
  }
}

// --------------------------------------------------------- Heaviside
__device__ __forceinline__ double heav_trig(const Params& p, double phi, double eps) {
  if (phi < -eps) return 0.;
  if (phi < eps) return (.5 + .5 * phi / eps) + .5 / p.pi * sin(p.pi * phi / eps);
  return 1.;
}
__device__ __forceinline__ double dirac_trig(const Params& p, double phi, double eps) {
  if (phi < -eps) return 0.;
  if (phi < eps) return .5 / eps + .5 / eps * cos(p.pi * phi / eps);
  return 0.;
}

// jiemian = min(jiemian, H_l) over shape C, partial sums of H_l over the
// interior (misc.f90:110-141).  Fixed grid: deterministic partials.
__global__ void __launch_bounds__(kRedThreads) k_heaviside_drop(Params p, const double* __restrict__ phi,
                                                                int first, double* __restrict__ jiemian,
                                                                double* __restrict__ partial) {
  const double eps = 1.5 * p.dz;
  double s = 0.;
  for (long long n = blockIdx.x * (long long)kRedThreads + threadIdx.x; n < p.nC;
       n += (long long)gridDim.x * kRedThreads) {
    int i, j, k;
    decodeC(p, n, i, j, k);
    const double H = heav_trig(p, phi[idxL(p, i, j, k)], eps);
    jiemian[n] = first ? H : fmin(jiemian[n], H);
    if (interior(p, i, j, k)) s += H;
  }
  double bs = block_sum<double, kRedThreads>(s);
  if (threadIdx.x == 0) partial[blockIdx.x] = bs;
}

// volume(l) and rho_avr from the partial sums (misc.f90:139-173)
__global__ void k_volumes(Params p, const double* __restrict__ partials, int nblk, double* __restrict__ vol,
                          DevScalars* __restrict__ dsc) {
  const double N = (1. * p.imax * p.jmax) * p.kmax;
  for (int l = threadIdx.x; l < p.L; l += blockDim.x) {
    double s = 0.;
    for (int b = 0; b < nblk; ++b) s += partials[(long long)l * nblk + b];
    vol[l] = 1. - s / N;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double sv = 0.;
    for (int l = 0; l < p.L; ++l) sv += vol[l];
    dsc->rho_avr = p.rho1 * (1. - sv) + p.rho2 * sv;
  }
}

// miu, rho (shape C) and the face densities (misc.f90:121-172)
__global__ void __launch_bounds__(NT) k_materials_final(Params p, const double* __restrict__ jiemian,
                                                        double* __restrict__ miu, double* __restrict__ rho,
                                                        double* __restrict__ rho_u, double* __restrict__ rho_v,
                                                        double* __restrict__ rho_w) {
  const long long n = blockIdx.x * (long long)NT + threadIdx.x;
  if (n >= p.nC) return;
  int i, j, k;
  decodeC(p, n, i, j, k);
  const double J0 = jiemian[n];
  miu[n] = p.miu1 * J0 + p.miu2 * (1. - J0);
  const double r0 = p.rho1 * J0 + p.rho2 * (1. - J0);
  rho[n] = r0;
  if (interior(p, i, j, k)) {
    const long long q = idxI(p, i, j, k);
    if (p.rho1 == p.rho2) {
      rho_u[q] = p.rho1; rho_v[q] = p.rho1; rho_w[q] = p.rho1;
    } else {
      const double Jx = jiemian[n + 1], Jy = jiemian[n + p.nCx], Jz = jiemian[n + (long long)p.nCx * p.nCy];
      const double rx = p.rho1 * Jx + p.rho2 * (1. - Jx);
      const double ry = p.rho1 * Jy + p.rho2 * (1. - Jy);
      const double rz = p.rho1 * Jz + p.rho2 * (1. - Jz);
      rho_u[q] = (r0 + rx) / 2.;
      rho_v[q] = (r0 + ry) / 2.;
      rho_w[q] = (r0 + rz) / 2.;
    }
  }
}

// ------------------------------------------------------------ inflation
// dheav with boundp semantics (shape C) and the area/volume partial sums
// (levelset.f90:493-507, 525)
__global__ void __launch_bounds__(kRedThreads) k_inflate_sums(Params p, const double* __restrict__ phi,
                                                              const double* __restrict__ kappa,
                                                              const double* __restrict__ nrm_m,
                                                              double* __restrict__ dheav,
                                                              double* __restrict__ part_area,
                                                              double* __restrict__ part_heav) {
  const double s1 = 1.5 * p.dz;
  double sa = 0., sh = 0.;
  for (long long n = blockIdx.x * (long long)kRedThreads + threadIdx.x; n < p.nC;
       n += (long long)gridDim.x * kRedThreads) {
    int i, j, k;
    decodeC(p, n, i, j, k);
    const int I = wrapx(p, i), J = wrapy(p, j);
    const int K = k == 0 ? 1 : (k == p.k1 ? p.kmax : k);
    dheav[n] = heav_trig(p, phi[idxL(p, I, J, K)], s1);
    if (interior(p, i, j, k)) {
      const double ph = phi[idxL(p, i, j, k)];
      const double H = heav_trig(p, ph, s1);
      const double del = dirac_trig(p, ph, s1);
      const double m = nrm_m[idxI(p, i, j, k)];
      sa += p.ispeed_curv ? (del * kappa[n]) * m : del * m;
      sh += H;
    }
  }
  double ba = block_sum<double, kRedThreads>(sa);
  double bh = block_sum<double, kRedThreads>(sh);
  if (threadIdx.x == 0) {
    part_area[blockIdx.x] = ba;
    part_heav[blockIdx.x] = bh;
  }
}

__global__ void k_inflate_final(Params p, const double* __restrict__ part_area,
                                const double* __restrict__ part_heav, int nblk, int l, double istep_dt,
                                double* __restrict__ vol, const double* __restrict__ vol0,
                                double* __restrict__ maxchk, DevScalars* __restrict__ dsc) {
  if (threadIdx.x != 0) return;
  double sa = 0., sh = 0.;
  for (int b = 0; b < nblk; ++b) { sa += part_area[b]; sh += part_heav[b]; }
  double area = sa * p.dx * p.dy * p.dz;
  if (p.TwoD) area = area / p.lx;
  const double volume = 1. - sh / ((1. * p.imax * p.jmax) * p.kmax);
  vol[l] = volume;
  double loss_rate = p.lx * p.ly * p.lz * (volume - vol0[l]) / istep_dt;
  if (p.TwoD) loss_rate = loss_rate / p.lx;
  const double temp = loss_rate / area;
  dsc->inflate_temp = temp;
  dsc->area = area;
  dsc->heav_sum = sh;
  maxchk[l] = temp / (1.5 * p.dz);
}

// u_lc, v_lc, w_lc of levelset.f90:527-548, with u_l,v_l,w_l of 530-532
// after bounduvw evaluated on the fly
__device__ __forceinline__ double infl_face(const Params& p, const double* __restrict__ dheav, double temp,
                                            int axis, int i, int j, int k) {
  const long long n = idxC(p, i, j, k);
  if (axis == 0) return -(temp * (dheav[n + 1] - dheav[n]) / p.dx);
  if (axis == 1) return -(temp * (dheav[n + p.nCx] - dheav[n]) / p.dy);
  return -(temp * (dheav[n + (long long)p.nCx * p.nCy] - dheav[n]) / p.dz);
}
__global__ void __launch_bounds__(NT) k_inflate_vel(Params p, const double* __restrict__ dheav,
                                                    const double* __restrict__ kappa,
                                                    const DevScalars* __restrict__ dsc,
                                                    double* __restrict__ ulc, double* __restrict__ vlc,
                                                    double* __restrict__ wlc) {
  const long long q = blockIdx.x * (long long)NT + threadIdx.x;
  if (q >= p.nI) return;
  const int i = (int)(q % p.imax) + 1;
  const long long r = q / p.imax;
  const int j = (int)(r % p.jmax) + 1;
  const int k = (int)(r / p.jmax) + 1;
  const double temp = dsc->inflate_temp;
  const double ul_m = infl_face(p, dheav, temp, 0, wrapx(p, i - 1), j, k);
  const double ul_0 = infl_face(p, dheav, temp, 0, i, j, k);
  const double vl_m = infl_face(p, dheav, temp, 1, i, wrapy(p, j - 1), k);
  const double vl_0 = infl_face(p, dheav, temp, 1, i, j, k);
  const double wl_m = (k == 1) ? 0. : infl_face(p, dheav, temp, 2, i, j, k - 1);
  const double wl_0 = (k == p.kmax) ? 0. : infl_face(p, dheav, temp, 2, i, j, k);
  double a = (ul_m + ul_0) / 2., b = (vl_m + vl_0) / 2., c = (wl_m + wl_0) / 2.;
  if (p.ispeed_curv) {
    const double kp = kappa[idxC(p, i, j, k)];
    a = a * kp; b = b * kp; c = c * kp;
  }
  ulc[q] = a; vlc[q] = b; wlc[q] = c;
}

// boundmls, extrap='line' (bound.f90:518-~657): three wall layers by
// repeated linear extrapolation from the interior column, then the periodic
// copies.  Reads only interior cells, writes only the others.
__global__ void __launch_bounds__(NT) k_boundmls(Params p, double* __restrict__ y) {
  const long long n = blockIdx.x * (long long)NT + threadIdx.x;
  if (n >= p.nL) return;
  int i, j, k;
  decodeL(p, n, i, j, k);
  const int I = wrapx(p, i), J = wrapy(p, j);
  if (k >= 1 && k <= p.kmax) {
    if (I != i || J != j) y[n] = y[idxL(p, I, J, k)];
    return;
  }
  if (k <= 0) {
    const double y1 = y[idxL(p, I, J, 1)], y2 = y[idxL(p, I, J, 2)];
    const double y0 = 2. * y1 - y2;
    const double ym1 = 2. * y0 - y1;
    const double ym2 = 2. * ym1 - y0;
    y[n] = (k == 0) ? y0 : (k == -1 ? ym1 : ym2);
  } else {
    const double yk = y[idxL(p, I, J, p.kmax)], ykm = y[idxL(p, I, J, p.kmax - 1)];
    const double y0 = 2. * yk - ykm;
    const double yp1 = 2. * y0 - yk;
    const double yp2 = 2. * yp1 - y0;
    y[n] = (k == p.k1) ? y0 : (k == p.k1 + 1 ? yp1 : yp2);
  }
}

__global__ void k_copy(double* __restrict__ dst, const double* __restrict__ src, long long n) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    dst[q] = src[q];
}

}  // namespace

// ================================================================ launchers
void launch_tube(Ctx& c, const double* in, double* out, long long* cnt) {
  Scope sc_(c.prof, c.s, "tube", 1);
  k_tube<<<nblocks(c.P.nL), NT, 0, c.s>>>(c.P, in, out, c.mask, cnt);
}

void launch_adv_stage(Ctx& c, int scheme, int stage1, const double* phi0, const double* phis, double a,
                      double b, double fdt, const double* vu, const double* vv, const double* vw, double* out) {
  Scope sc_(c.prof, c.s, "adv_stage", 1);
  if (scheme == ICLS_HOUC5)
    k_adv_stage<ICLS_HOUC5><<<nblocks(c.P.nL), NT, 0, c.s>>>(c.P, stage1, phi0, phis, a, b, fdt, vu, vv, vw,
                                                            c.mask, out);
  else
    k_adv_stage<ICLS_WENO5><<<nblocks(c.P.nL), NT, 0, c.s>>>(c.P, stage1, phi0, phis, a, b, fdt, vu, vv, vw,
                                                            c.mask, out);
}

void launch_reinit_stage(Ctx& c, int stage, const double* phi0, const double* phis, const double* orig,
                         double dtau, double* out, int check_done) {
  Scope sc_(c.prof, c.s, "reinit_stage", 1);
  k_reinit_stage<<<nblocks(c.P.nL), NT, 0, c.s>>>(c.P, stage, phi0, phis, orig, dtau, out, check_done, c.dsc);
}
void launch_reinit_check(Ctx& c, int it, int maxiter, double thr) {
  Scope sc_(c.prof, c.s, "reinit_check", 1);
  k_reinit_check<<<1, 1, 0, c.s>>>(c.dsc, it, maxiter, thr);
}
void launch_reinit_reset(Ctx& c, int maxiter) {
  Scope sc_(c.prof, c.s, "reinit_reset", 1); k_reinit_reset<<<1, 1, 0, c.s>>>(c.dsc, maxiter); }

void launch_heaviside_drop(Ctx& c, const double* phi, int l, int first) {
  Scope sc_(c.prof, c.s, "heaviside_drop", 1);
  k_heaviside_drop<<<kRedBlocks, kRedThreads, 0, c.s>>>(c.P, phi, first, c.jiemian,
                                                        c.partials + (long long)l * kRedBlocks);
}

void launch_materials_final(Ctx& c) {
  Scope sc_(c.prof, c.s, "materials_final", 2);
  k_volumes<<<1, 256, 0, c.s>>>(c.P, c.partials, kRedBlocks, c.dvol, c.dsc);
  k_materials_final<<<nblocks(c.P.nC), NT, 0, c.s>>>(c.P, c.jiemian, c.miu, c.rho, c.rho_u, c.rho_v, c.rho_w);
}

void launch_inflate_sums(Ctx& c, const double* phi, int l) {
  Scope sc_(c.prof, c.s, "inflate_sums", 2);
  double* pa = c.partials;
  double* ph = c.partials + kRedBlocks;
  k_inflate_sums<<<kRedBlocks, kRedThreads, 0, c.s>>>(c.P, phi, c.kappa, c.nrm_m, c.dheav, pa, ph);
  k_inflate_final<<<1, 32, 0, c.s>>>(c.P, pa, ph, kRedBlocks, l, (double)c.cfg.inflate_step * c.dt, c.dvol,
                                     c.dvol0, c.dmaxchk, c.dsc);
}

void launch_inflate_vel(Ctx& c) {
  Scope sc_(c.prof, c.s, "inflate_vel", 1);
  k_inflate_vel<<<nblocks(c.P.nI), NT, 0, c.s>>>(c.P, c.dheav, c.kappa, c.dsc, c.ulc, c.vlc, c.wlc);
}

void launch_boundmls(Ctx& c, double* phi) {
  Scope sc_(c.prof, c.s, "boundmls", 1); k_boundmls<<<nblocks(c.P.nL), NT, 0, c.s>>>(c.P, phi); }

void launch_copy(Ctx& c, double* dst, const double* src, long long n) {
  Scope sc_(c.prof, c.s, "copy", 1);
  k_copy<<<1184, 256, 0, c.s>>>(dst, src, n);
}

}  // namespace icls
