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
//
// Sweep boxes: after tube_construction clips the level set to +-6dz, every
// cell outside a drop's band holds the same far-field value, and every
// kernel maps a uniform neighbourhood to a uniform value (the stencils of a
// constant field are exactly zero).  Each per-drop kernel therefore sweeps
// only a box around the band (Box3 compute region) and writes the
// far-field value, replayed on the host with the same arithmetic, into a
// 3-cell apron around it; reads never leave the box plus apron.  Full axes
// (band near a periodic seam or a wall) fall back to the whole index range.
#include <climits>

#include "ctx.h"

namespace icls {

namespace {

constexpr int NT = 256;

__device__ __forceinline__ double clipNB(double x, double NB) {
  return x > NB ? NB : (x < -NB ? -NB : x);
}
__device__ __forceinline__ bool interior(const Params& p, int i, int j, int k) {
  return i >= 1 && i <= p.imax && j >= 1 && j <= p.jmax && k >= 1 && k <= p.kmax;
}
__device__ __forceinline__ void decode_box(const int* r0, const int* r1, int q, int& i, int& j, int& k) {
  const int nx = r1[0] - r0[0] + 1, ny = r1[1] - r0[1] + 1;
  i = r0[0] + q % nx;
  const int r = q / nx;
  j = r0[1] + r % ny;
  k = r0[2] + r / ny;
}

// ---------------------------------------------------------------- tube
// in is valid on vin's write region; elsewhere it holds bgin, except the
// ghost rows k<0, k>k1 (never touched by the reinitialisation RHS), which
// hold bgg.  Writes b's write region; the band mask for computed interior
// cells; the band count; the bounding box of computed cells whose clipped
// value is not +NB.
__global__ void __launch_bounds__(NT) k_tube(Params p, Box3 b, Box3 vin, double bgin, double bgg,
                                             const double* __restrict__ in, double* __restrict__ out,
                                             uint8_t* __restrict__ mask, long long* __restrict__ cnt,
                                             int* __restrict__ bbox) {
  int i, j, k;
  const bool ok = cell3(b.w0, b.w1, i, j, k);
  const double NB = p.NB;
  int m = 0;
  int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
  auto rd = [&](int a, int bb, int cc) -> double {
    return in_write(vin, a, bb, cc) ? in[idxL(p, a, bb, cc)] : ((cc < 0 || cc > p.k1) ? bgg : bgin);
  };
  if (ok) {
    const long long n = idxL(p, i, j, k);
    double val;
    if (!in_compute(b, i, j, k)) {
      val = clipNB((k < 0 || k > p.k1) ? bgg : bgin, NB);
    } else {
      const int I = wrapx(p, i), J = wrapy(p, j);
      if (k == 0)
        val = 2. * clipNB(rd(I, J, 1), NB) - clipNB(rd(I, J, 2), NB);
      else if (k == p.k1)
        val = 2. * clipNB(rd(I, J, p.kmax), NB) - clipNB(rd(I, J, p.kmax - 1), NB);
      else
        val = clipNB(rd(I, J, k), NB);
      if (interior(p, i, j, k)) {
        const double c0 = clipNB(rd(i, j, k), NB);
        if (fabs(c0) < NB) {
          m = 1;
        } else {
          double xs = 0., ys = 0., zs = 0.;
          for (int d = -2; d <= 2; ++d) xs += fabs(clipNB(rd(i + d, j, k), NB)) - NB;
          for (int d = -2; d <= 2; ++d) ys += fabs(clipNB(rd(i, j + d, k), NB)) - NB;
          for (int d = -2; d <= 2; ++d) zs += fabs(clipNB(rd(i, j, k + d), NB)) - NB;
          m = (xs == 0. && ys == 0. && zs == 0.) ? 0 : 1;
        }
        mask[idxI(p, i, j, k)] = (uint8_t)m;
      }
      if (val != NB) {
        lo[0] = hi[0] = i; lo[1] = hi[1] = j; lo[2] = hi[2] = k;
      }
    }
    out[n] = val;
  }
  int bs = block_sum<int, BX * BY>(m);
  if (flat_tid() == 0 && bs) atomicAdd((unsigned long long*)cnt, (unsigned long long)bs);
  for (int a = 0; a < 3; ++a) {
    int l = lo[a], h = hi[a];
    for (int o = 16; o > 0; o >>= 1) {
      l = min(l, __shfl_down_sync(0xffffffffu, l, o));
      h = max(h, __shfl_down_sync(0xffffffffu, h, o));
    }
    if ((flat_tid() & 31) == 0 && l != INT_MAX) {
      atomicMin(&bbox[a], l);
      atomicMax(&bbox[3 + a], h);
    }
  }
}

// ------------------------------------------------------- advection RHS
// dfdt of HOUC5_nb (hyperPDE.f90:397-495) or WENO5_nb (503-800) at (i,j,k)
template <int SCHEME>
__device__ __forceinline__ double adv_rhs(const Params& p, const double* __restrict__ phi,
                                          double vu, double vv, double vw, int i, int j, int k) {
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
      udfdx = -divx(p, vu * dfx);
    }
    if (vv >= 0.)
      dfy = houc5_pos(PH(-3 * sy), PH(-2 * sy), PH(-sy), PH(0), PH(sy), PH(2 * sy));
    else
      dfy = houc5_neg(PH(3 * sy), PH(2 * sy), PH(sy), PH(0), PH(-sy), PH(-2 * sy));
    vdfdy = -divy(p, vv * dfy);
  } else {
    if (p.TwoD) {
      udfdx = 0.;
    } else {
      if (vu >= 0.)
        dfx = weno5(divx(p, PH(-2 * sx) - PH(-3 * sx)), divx(p, PH(-sx) - PH(-2 * sx)), divx(p, PH(0) - PH(-sx)),
                    divx(p, PH(sx) - PH(0)), divx(p, PH(2 * sx) - PH(sx)));
      else
        dfx = weno5(divx(p, PH(3 * sx) - PH(2 * sx)), divx(p, PH(2 * sx) - PH(sx)), divx(p, PH(sx) - PH(0)),
                    divx(p, PH(0) - PH(-sx)), divx(p, PH(-sx) - PH(-2 * sx)));
      udfdx = -(vu * dfx);
    }
    // y uses dx, as in the reference (hyperPDE.f90:622-626)
    if (vv >= 0.)
      dfy = weno5(divx(p, PH(-2 * sy) - PH(-3 * sy)), divx(p, PH(-sy) - PH(-2 * sy)), divx(p, PH(0) - PH(-sy)),
                  divx(p, PH(sy) - PH(0)), divx(p, PH(2 * sy) - PH(sy)));
    else
      dfy = weno5(divx(p, PH(3 * sy) - PH(2 * sy)), divx(p, PH(2 * sy) - PH(sy)), divx(p, PH(sy) - PH(0)),
                  divx(p, PH(0) - PH(-sy)), divx(p, PH(-sy) - PH(-2 * sy)));
    vdfdy = -(vv * dfy);
  }
  if (k > 2 && k < p.kmax - 1) {
    if (SCHEME == ICLS_HOUC5) {
      if (vw >= 0.)
        dfz = houc5_pos(PH(-3 * sz), PH(-2 * sz), PH(-sz), PH(0), PH(sz), PH(2 * sz));
      else
        dfz = houc5_neg(PH(3 * sz), PH(2 * sz), PH(sz), PH(0), PH(-sz), PH(-2 * sz));
      wdfdz = -divz(p, vw * dfz);
    } else {
      if (vw >= 0.)
        dfz = weno5(divz(p, PH(-2 * sz) - PH(-3 * sz)), divz(p, PH(-sz) - PH(-2 * sz)), divz(p, PH(0) - PH(-sz)),
                    divz(p, PH(sz) - PH(0)), divz(p, PH(2 * sz) - PH(sz)));
      else
        dfz = weno5(divz(p, PH(3 * sz) - PH(2 * sz)), divz(p, PH(2 * sz) - PH(sz)), divz(p, PH(sz) - PH(0)),
                    divz(p, PH(0) - PH(-sz)), divz(p, PH(-sz) - PH(-2 * sz)));
      wdfdz = -(vw * dfz);
    }
  } else if (k == 2 || k == p.kmax - 1) {  // HOUC3 near the walls
    if (vw >= 0.)
      dfz = (((1. / 6.) * PH(-2 * sz) - PH(-sz)) + (1. / 2.) * PH(0)) + (1. / 3.) * PH(sz);
    else
      dfz = ((-((1. / 6.) * PH(2 * sz)) + PH(sz)) - (1. / 2.) * PH(0)) - (1. / 3.) * PH(-sz);
    wdfdz = -divz(p, vw * dfz);
  } else {  // first-order upwinding at k=1,kmax
    if (vw >= 0.) dfz = PH(0) - PH(-sz);
    else dfz = PH(sz) - PH(0);
    wdfdz = -divz(p, vw * dfz);
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
__global__ void __launch_bounds__(NT) k_adv_stage(Params p, Box3 b, double bg_out, double bgg_out, int stage1,
                                                  const double* __restrict__ phi0, const double* __restrict__ phis,
                                                  double a, double bb, double fdt, const double* __restrict__ vu,
                                                  const double* __restrict__ vv, const double* __restrict__ vw,
                                                  const uint8_t* __restrict__ mask, double* __restrict__ out) {
  int i, j, k;
  if (!cell3(b.w0, b.w1, i, j, k)) return;
  const long long n = idxL(p, i, j, k);
  if (!in_compute(b, i, j, k)) {
    out[n] = (k < 0 || k > p.k1) ? bgg_out : bg_out;
    return;
  }
  const int I = wrapx(p, i), J = wrapy(p, j);
  double val;
  if (k == 0)
    val = 2. * adv_val<SCHEME>(p, stage1, phi0, phis, a, bb, fdt, vu, vv, vw, mask, I, J, 1) -
          adv_val<SCHEME>(p, stage1, phi0, phis, a, bb, fdt, vu, vv, vw, mask, I, J, 2);
  else if (k == p.k1)
    val = 2. * adv_val<SCHEME>(p, stage1, phi0, phis, a, bb, fdt, vu, vv, vw, mask, I, J, p.kmax) -
          adv_val<SCHEME>(p, stage1, phi0, phis, a, bb, fdt, vu, vv, vw, mask, I, J, p.kmax - 1);
  else
    val = adv_val<SCHEME>(p, stage1, phi0, phis, a, bb, fdt, vu, vv, vw, mask, I, J, k);
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
  const long long sx = 1, sy = p.nLx, sz = (long long)p.nLx * p.nLy;
#define PH(o) phi[c + (o)]
  double A = 0., B = 0., C, D, E, F;
  if (!p.TwoD) {
    A = weno5(divx(p, PH(-2 * sx) - PH(-3 * sx)), divx(p, PH(-sx) - PH(-2 * sx)), divx(p, PH(0) - PH(-sx)),
              divx(p, PH(sx) - PH(0)), divx(p, PH(2 * sx) - PH(sx)));
    B = weno5(divx(p, PH(3 * sx) - PH(2 * sx)), divx(p, PH(2 * sx) - PH(sx)), divx(p, PH(sx) - PH(0)),
              divx(p, PH(0) - PH(-sx)), divx(p, PH(-sx) - PH(-2 * sx)));
  }
  C = weno5(divx(p, PH(-2 * sy) - PH(-3 * sy)), divx(p, PH(-sy) - PH(-2 * sy)), divx(p, PH(0) - PH(-sy)),
            divx(p, PH(sy) - PH(0)), divx(p, PH(2 * sy) - PH(sy)));
  D = weno5(divx(p, PH(3 * sy) - PH(2 * sy)), divx(p, PH(2 * sy) - PH(sy)), divx(p, PH(sy) - PH(0)),
            divx(p, PH(0) - PH(-sy)), divx(p, PH(-sy) - PH(-2 * sy)));
  if (k >= 3 && k <= p.kmax - 2) {
    E = weno5(divz(p, PH(-2 * sz) - PH(-3 * sz)), divz(p, PH(-sz) - PH(-2 * sz)), divz(p, PH(0) - PH(-sz)),
              divz(p, PH(sz) - PH(0)), divz(p, PH(2 * sz) - PH(sz)));
    F = weno5(divz(p, PH(3 * sz) - PH(2 * sz)), divz(p, PH(2 * sz) - PH(sz)), divz(p, PH(sz) - PH(0)),
              divz(p, PH(0) - PH(-sz)), divz(p, PH(-sz) - PH(-2 * sz)));
  } else {
    E = divz(p, PH(0) - PH(-sz));
    F = divz(p, PH(sz) - PH(0));
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

__global__ void __launch_bounds__(NT) k_reinit_stage(Params p, Box3 b, double bg_out, double bgg_out, int stage,
                                                     const double* __restrict__ phi0,
                                                     const double* __restrict__ phis,
                                                     const double* __restrict__ orig, double dtau,
                                                     double* __restrict__ out, DevScalars* __restrict__ dsc) {
  const int done = dsc->reinit_done;
  int i, j, k;
  const bool ok = cell3(b.w0, b.w1, i, j, k);
  if (done) {
    // an iteration after convergence is the identity (levelset.f90:833-835)
    if (stage == 3 && ok) out[idxL(p, i, j, k)] = phi0[idxL(p, i, j, k)];
    return;
  }
  if (stage == 1 && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && flat_tid() == 0) dsc->residual = 0.;
  double r = 0.;
  if (ok) {
    const long long n = idxL(p, i, j, k);
    double val;
    if (!in_compute(b, i, j, k)) {
      val = (k < 0 || k > p.k1) ? bgg_out : bg_out;
    } else {
      const int I = wrapx(p, i), J = wrapy(p, j);
      if (k == 0)
        val = 2. * reinit_val(p, stage, phi0, phis, orig, dtau, I, J, 1) -
              reinit_val(p, stage, phi0, phis, orig, dtau, I, J, 2);
      else if (k == p.k1)
        val = 2. * reinit_val(p, stage, phi0, phis, orig, dtau, I, J, p.kmax) -
              reinit_val(p, stage, phi0, phis, orig, dtau, I, J, p.kmax - 1);
      else
        val = reinit_val(p, stage, phi0, phis, orig, dtau, I, J, k);
      if (stage == 3) r = fabs(val - phi0[n]);
    }
    out[n] = val;
  }
  if (stage == 3) {
    double bm = block_max<double, BX * BY>(r);
    if (flat_tid() == 0) atomic_max_nonneg(&dsc->residual, bm);
  }
}

__global__ void k_reinit_reset(DevScalars* dsc, int maxiter) {
  dsc->reinit_done = 0;
  dsc->reinit_iters = maxiter;
  dsc->residual = 0.;
}
// far: |change| of the far-field cells outside the box (0 when none)
__global__ void k_reinit_check(DevScalars* dsc, int it, int maxiter, double thr, double far) {
  if (dsc->reinit_done) return;
  if (far > dsc->residual) dsc->residual = far;
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

// jiemian = min(jiemian, H_l) over the region r (shape C coordinates),
// partial sums of H_l over its interior cells (misc.f90:110-141).  Fixed
// grid: deterministic partials.
__global__ void __launch_bounds__(kRedThreads) k_heaviside_drop(Params p, Box3 r, const double* __restrict__ phi,
                                                                int first, double* __restrict__ jiemian,
                                                                double* __restrict__ partial) {
  const double eps = 1.5 * p.dz;
  const int n = (r.c1[0] - r.c0[0] + 1) * (r.c1[1] - r.c0[1] + 1) * (r.c1[2] - r.c0[2] + 1);
  double s = 0.;
  for (int q = blockIdx.x * kRedThreads + threadIdx.x; q < n; q += gridDim.x * kRedThreads) {
    int i, j, k;
    decode_box(r.c0, r.c1, q, i, j, k);
    const double H = heav_trig(p, phi[idxL(p, i, j, k)], eps);
    const long long c = idxC(p, i, j, k);
    jiemian[c] = first ? H : fmin(jiemian[c], H);
    if (interior(p, i, j, k)) s += H;
  }
  double bs = block_sum<double, kRedThreads>(s);
  if (threadIdx.x == 0) partial[blockIdx.x] = bs;
}

// volume(l) and rho_avr from the partial sums (misc.f90:139-173); outside[l]
// interior cells of drop l lie in its far field, where H = 1
struct PerDrop {
  double v[kMaxDropsParam];
};
__global__ void k_volumes(Params p, const double* __restrict__ partials, int nblk, PerDrop outside,
                          double* __restrict__ vol, DevScalars* __restrict__ dsc) {
  const double N = (1. * p.imax * p.jmax) * p.kmax;
  for (int l = threadIdx.x; l < p.L; l += blockDim.x) {
    double s = 0.;
    for (int b = 0; b < nblk; ++b) s += partials[(long long)l * nblk + b];
    s += outside.v[l];
    vol[l] = 1. - s / N;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double sv = 0.;
    for (int l = 0; l < p.L; ++l) sv += vol[l];
    dsc->rho_avr = p.rho1 * (1. - sv) + p.rho2 * sv;
  }
}

__global__ void __launch_bounds__(NT) k_fill(double* __restrict__ a, long long n, double v) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    a[q] = v;
}

// miu, rho (shape C) and the face densities (misc.f90:121-172)
__global__ void __launch_bounds__(NT) k_materials_final(Params p, const double* __restrict__ jiemian,
                                                        double* __restrict__ miu, double* __restrict__ rho,
                                                        double* __restrict__ rho_u, double* __restrict__ rho_v,
                                                        double* __restrict__ rho_w) {
  const int r0[3] = {0, 0, 0}, r1[3] = {p.i1, p.j1, p.k1};
  int i, j, k;
  if (!cell3(r0, r1, i, j, k)) return;
  const long long n = idxC(p, i, j, k);
  const double J0 = jiemian[n];
  miu[n] = p.miu1 * J0 + p.miu2 * (1. - J0);
  const double r0v = p.rho1 * J0 + p.rho2 * (1. - J0);
  rho[n] = r0v;
  if (interior(p, i, j, k)) {
    const long long q = idxI(p, i, j, k);
    if (p.rho1 == p.rho2) {
      rho_u[q] = p.rho1; rho_v[q] = p.rho1; rho_w[q] = p.rho1;
    } else {
      const double Jx = jiemian[n + 1], Jy = jiemian[n + p.nCx], Jz = jiemian[n + (long long)p.nCx * p.nCy];
      const double rx = p.rho1 * Jx + p.rho2 * (1. - Jx);
      const double ry = p.rho1 * Jy + p.rho2 * (1. - Jy);
      const double rz = p.rho1 * Jz + p.rho2 * (1. - Jz);
      rho_u[q] = (r0v + rx) / 2.;
      rho_v[q] = (r0v + ry) / 2.;
      rho_w[q] = (r0v + rz) / 2.;
    }
  }
}

// ------------------------------------------------------------ inflation
// dheav with boundp semantics over the region r (shape C), the far-field
// value 1 on its apron, and the area/volume partial sums over the interior
// computed cells (levelset.f90:493-507, 525)
__global__ void __launch_bounds__(kRedThreads) k_inflate_sums(Params p, Box3 r, const double* __restrict__ phi,
                                                              const double* __restrict__ kappa,
                                                              const double* __restrict__ nrm_m,
                                                              double* __restrict__ dheav,
                                                              double* __restrict__ part_area,
                                                              double* __restrict__ part_heav) {
  const double s1 = 1.5 * p.dz;
  const int n = (r.w1[0] - r.w0[0] + 1) * (r.w1[1] - r.w0[1] + 1) * (r.w1[2] - r.w0[2] + 1);
  double sa = 0., sh = 0.;
  for (int q = blockIdx.x * kRedThreads + threadIdx.x; q < n; q += gridDim.x * kRedThreads) {
    int i, j, k;
    decode_box(r.w0, r.w1, q, i, j, k);
    const long long c = idxC(p, i, j, k);
    if (!in_compute(r, i, j, k)) {
      dheav[c] = 1.;
      continue;
    }
    const int I = wrapx(p, i), J = wrapy(p, j);
    const int K = k == 0 ? 1 : (k == p.k1 ? p.kmax : k);
    dheav[c] = heav_trig(p, phi[idxL(p, I, J, K)], s1);
    if (interior(p, i, j, k)) {
      const double ph = phi[idxL(p, i, j, k)];
      const double H = heav_trig(p, ph, s1);
      const double del = dirac_trig(p, ph, s1);
      const double m = nrm_m[idxI(p, i, j, k)];
      sa += p.ispeed_curv ? (del * kappa[c]) * m : del * m;
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
                                double outside, double* __restrict__ vol, const double* __restrict__ vol0,
                                double* __restrict__ maxchk, DevScalars* __restrict__ dsc) {
  if (threadIdx.x != 0) return;
  double sa = 0., sh = 0.;
  for (int b = 0; b < nblk; ++b) { sa += part_area[b]; sh += part_heav[b]; }
  sh += outside;
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
// after bounduvw evaluated on the fly; computed interior cells of r
__device__ __forceinline__ double infl_face(const Params& p, const double* __restrict__ dheav, double temp,
                                            int axis, int i, int j, int k) {
  const long long n = idxC(p, i, j, k);
  if (axis == 0) return -divx(p, temp * (dheav[n + 1] - dheav[n]));
  if (axis == 1) return -divy(p, temp * (dheav[n + p.nCx] - dheav[n]));
  return -divz(p, temp * (dheav[n + (long long)p.nCx * p.nCy] - dheav[n]));
}
__global__ void __launch_bounds__(NT) k_inflate_vel(Params p, Box3 r, const double* __restrict__ dheav,
                                                    const double* __restrict__ kappa,
                                                    const DevScalars* __restrict__ dsc,
                                                    double* __restrict__ ulc, double* __restrict__ vlc,
                                                    double* __restrict__ wlc) {
  int i, j, k;
  if (!cell3(r.c0, r.c1, i, j, k)) return;
  if (!interior(p, i, j, k)) return;
  const long long q = idxI(p, i, j, k);
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
  const int r0[3] = {-2, -2, -2}, r1[3] = {p.i1 + 2, p.j1 + 2, p.k1 + 2};
  int i, j, k;
  if (!cell3(r0, r1, i, j, k)) return;
  const long long n = idxL(p, i, j, k);
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

// far-field value into every cell outside the write region of b (makes a
// drop's stored array valid everywhere, e.g. before a download)
__global__ void __launch_bounds__(NT) k_materialize(Params p, Box3 b, double bg, double bgg, double* __restrict__ y) {
  const int r0[3] = {-2, -2, -2}, r1[3] = {p.i1 + 2, p.j1 + 2, p.k1 + 2};
  int i, j, k;
  if (!cell3(r0, r1, i, j, k)) return;
  if (!in_write(b, i, j, k)) y[idxL(p, i, j, k)] = (k < 0 || k > p.k1) ? bgg : bg;
}

__global__ void k_copy(double* __restrict__ dst, const double* __restrict__ src, long long n) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    dst[q] = src[q];
}

const dim3 kBlock(BX, BY, 1);

}  // namespace

dim3 grid_of(const int* r0, const int* r1) {
  const int nx = r1[0] - r0[0] + 1, ny = r1[1] - r0[1] + 1, nz = r1[2] - r0[2] + 1;
  return dim3((unsigned)((nx + BX - 1) / BX), (unsigned)((ny + BY - 1) / BY), (unsigned)nz);
}

Box3 full_box(const Params& P) {
  Box3 b;
  const int n[3] = {P.imax, P.jmax, P.kmax};
  for (int a = 0; a < 3; ++a) {
    b.c0[a] = b.w0[a] = -2;
    b.c1[a] = b.w1[a] = n[a] + 3;
  }
  return b;
}

// the shape-C part of a level-set box, apron of width `ap` on partial axes
Box3 c_region(const Params& P, const Box3& b, int ap) {
  const int n[3] = {P.imax, P.jmax, P.kmax};
  Box3 r;
  for (int a = 0; a < 3; ++a) {
    const bool full = (b.c0[a] <= -2 && b.c1[a] >= n[a] + 3);
    if (full) {
      r.c0[a] = r.w0[a] = 0;
      r.c1[a] = r.w1[a] = n[a] + 1;
    } else {
      r.c0[a] = b.c0[a];
      r.c1[a] = b.c1[a];
      r.w0[a] = std::max(0, b.c0[a] - ap);
      r.w1[a] = std::min(n[a] + 1, b.c1[a] + ap);
    }
  }
  return r;
}

// ================================================================ launchers
void launch_tube(Ctx& c, const Box3& b, const Box3& vin, double bgin, double bgg, const double* in, double* out,
                 long long* cnt, int* bbox) {
  Scope sc_(c.prof, c.s, "tube", 1);
  k_tube<<<grid_of(b.w0, b.w1), kBlock, 0, c.s>>>(c.P, b, vin, bgin, bgg, in, out, c.mask, cnt, bbox);
}

void launch_adv_stage(Ctx& c, const Box3& b, double bg_out, double bgg_out, int scheme, int stage1,
                      const double* phi0, const double* phis, double a, double bb, double fdt, const double* vu,
                      const double* vv, const double* vw, double* out) {
  Scope sc_(c.prof, c.s, "adv_stage", 1);
  if (scheme == ICLS_HOUC5)
    k_adv_stage<ICLS_HOUC5><<<grid_of(b.w0, b.w1), kBlock, 0, c.s>>>(c.P, b, bg_out, bgg_out, stage1, phi0, phis,
                                                                     a, bb, fdt, vu, vv, vw, c.mask, out);
  else
    k_adv_stage<ICLS_WENO5><<<grid_of(b.w0, b.w1), kBlock, 0, c.s>>>(c.P, b, bg_out, bgg_out, stage1, phi0, phis,
                                                                     a, bb, fdt, vu, vv, vw, c.mask, out);
}

void launch_reinit_stage(Ctx& c, const Box3& b, double bg_out, double bgg_out, int stage, const double* phi0,
                         const double* phis, const double* orig, double dtau, double* out) {
  Scope sc_(c.prof, c.s, "reinit_stage", 1);
  k_reinit_stage<<<grid_of(b.w0, b.w1), kBlock, 0, c.s>>>(c.P, b, bg_out, bgg_out, stage, phi0, phis, orig, dtau,
                                                          out, c.dsc);
}
void launch_reinit_check(Ctx& c, int it, int maxiter, double thr, double far) {
  Scope sc_(c.prof, c.s, "reinit_check", 1);
  k_reinit_check<<<1, 1, 0, c.s>>>(c.dsc, it, maxiter, thr, far);
}
void launch_reinit_reset(Ctx& c, int maxiter) {
  Scope sc_(c.prof, c.s, "reinit_reset", 1);
  k_reinit_reset<<<1, 1, 0, c.s>>>(c.dsc, maxiter);
}

void launch_heaviside_drop(Ctx& c, const Box3& b, const double* phi, int l, int first) {
  Scope sc_(c.prof, c.s, "heaviside_drop", 1);
  const Box3 r = c_region(c.P, b, 0);
  k_heaviside_drop<<<kRedBlocks, kRedThreads, 0, c.s>>>(c.P, r, phi, first, c.jiemian,
                                                        c.partials + (long long)l * kRedBlocks);
}

void launch_fill(Ctx& c, double* a, long long n, double v) {
  Scope sc_(c.prof, c.s, "fill", 1);
  k_fill<<<1184, NT, 0, c.s>>>(a, n, v);
}

void launch_materials_final(Ctx& c, const double* outside) {
  Scope sc_(c.prof, c.s, "materials_final", 2);
  PerDrop o;
  for (int l = 0; l < kMaxDropsParam; ++l) o.v[l] = (l < c.P.L) ? outside[l] : 0.;
  k_volumes<<<1, 256, 0, c.s>>>(c.P, c.partials, kRedBlocks, o, c.dvol, c.dsc);
  const int r0[3] = {0, 0, 0}, r1[3] = {c.P.i1, c.P.j1, c.P.k1};
  k_materials_final<<<grid_of(r0, r1), kBlock, 0, c.s>>>(c.P, c.jiemian, c.miu, c.rho, c.rho_u, c.rho_v, c.rho_w);
}

void launch_inflate_sums(Ctx& c, const Box3& b, const double* phi, int l, double outside) {
  Scope sc_(c.prof, c.s, "inflate_sums", 2);
  double* pa = c.partials;
  double* ph = c.partials + kRedBlocks;
  const Box3 r = c_region(c.P, b, 1);
  k_inflate_sums<<<kRedBlocks, kRedThreads, 0, c.s>>>(c.P, r, phi, c.kappa, c.nrm_m, c.dheav, pa, ph);
  k_inflate_final<<<1, 32, 0, c.s>>>(c.P, pa, ph, kRedBlocks, l, (double)c.cfg.inflate_step * c.dt, outside,
                                     c.dvol, c.dvol0, c.dmaxchk, c.dsc);
}

void launch_inflate_vel(Ctx& c, const Box3& b) {
  Scope sc_(c.prof, c.s, "inflate_vel", 1);
  const Box3 r = c_region(c.P, b, 0);
  k_inflate_vel<<<grid_of(r.c0, r.c1), kBlock, 0, c.s>>>(c.P, r, c.dheav, c.kappa, c.dsc, c.ulc, c.vlc, c.wlc);
}

void launch_boundmls(Ctx& c, double* phi) {
  Scope sc_(c.prof, c.s, "boundmls", 1);
  const int r0[3] = {-2, -2, -2}, r1[3] = {c.P.i1 + 2, c.P.j1 + 2, c.P.k1 + 2};
  k_boundmls<<<grid_of(r0, r1), kBlock, 0, c.s>>>(c.P, phi);
}

void launch_materialize(Ctx& c, const Box3& b, double bg, double bgg, double* phi) {
  Scope sc_(c.prof, c.s, "materialize", 1);
  const int r0[3] = {-2, -2, -2}, r1[3] = {c.P.i1 + 2, c.P.j1 + 2, c.P.k1 + 2};
  k_materialize<<<grid_of(r0, r1), kBlock, 0, c.s>>>(c.P, b, bg, bgg, phi);
}

void launch_copy(Ctx& c, double* dst, const double* src, long long n) {
  Scope sc_(c.prof, c.s, "copy", 1);
  k_copy<<<1184, 256, 0, c.s>>>(dst, src, n);
}

}  // namespace icls
