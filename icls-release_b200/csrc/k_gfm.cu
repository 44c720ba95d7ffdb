// k_gfm.cu — interface curvature and ghost-fluid pressure jumps (FP64,
// -fmad=false).
//
//   get_curvature  interface.f90:20-119   (10x27 least-squares fit)
//   re_curvature   interface.f90:186-218
//   icurvature     interface.f90:126-179
//   gfm4p jumps    gfm.f90:95-238
//   ipot           interface.f90:225-277
//
// The 10x27 pseudo-inverse (init.f90:1587-1723) lives in constant memory:
// every thread of a warp reads the same coefficient, which the constant
// cache broadcasts.
#include <algorithm>

#include "ctx.h"

namespace icls {

__constant__ double cP[270];

namespace {

constexpr int NT = 256;


// curvature at an interior cell (interface.f90:57-111); m = |grad phi| or 1
__device__ __forceinline__ double curvature_at(const Params& p, const double* __restrict__ phi, int i, int j,
                                               int k, double& m) {
  const long long c = idxL(p, i, j, k);
  m = 1.;
  if (!(fabs(phi[c]) <= p.NB - 1. * p.dz)) return 0.;
  double s27[27];
  int n = 0;
  const long long sy = p.nLx, sz = (long long)p.nLx * p.nLy;
#pragma unroll
  for (int dk = -1; dk <= 1; ++dk)
#pragma unroll
    for (int dj = -1; dj <= 1; ++dj)
#pragma unroll
      for (int di = -1; di <= 1; ++di) s27[n++] = phi[c + di + dj * sy + dk * sz];
  double x[10];
#pragma unroll
  for (int r = 1; r < 10; ++r) {
    double s = 0.;
#pragma unroll
    for (int q = 0; q < 27; ++q) s = s + cP[r * 27 + q] * s27[q];
    x[r] = s;
  }
  const double dphidx = x[1], dphidy = x[2], dphidz = x[3];
  const double d2phidx = x[4], d2phidy = x[5], d2phidz = x[6];
  const double d2phidxdy = x[7], d2phidxdz = x[8], d2phidydz = x[9];
  const double norm_val = sqrt((dphidx * dphidx + dphidy * dphidy) + dphidz * dphidz);
  m = norm_val;
  double cv;
  if (norm_val < 0.9) {
    cv = 0.;
  } else {
    const double n3 = norm_val * norm_val * norm_val;
    const double term1 = ((d2phidx + d2phidy) + d2phidz) / norm_val;
    double term2 = (dphidx * dphidx * d2phidx + dphidy * dphidy * d2phidy) + dphidz * dphidz * d2phidz;
    term2 = term2 / n3;
    double term3 = (dphidx * dphidy * d2phidxdy + dphidx * dphidz * d2phidxdz) + dphidy * dphidz * d2phidydz;
    term3 = 2. * term3 / n3;
    cv = -((term1 - term2) - term3);
  }
  const double max_kappa = 1. / p.dz;
  if (cv < -max_kappa) cv = -max_kappa;
  else if (cv > max_kappa) cv = max_kappa;
  else if (fabs(cv) < 1e-9) cv = 0.;
  return cv;
}

// get_curvature + boundc over a drop's region of shape C: wall rows stay 0,
// halos are the periodic copies (bound.f90:292-305), the apron (far field,
// |phi| > 5dz) is 0.
__global__ void __launch_bounds__(NT) k_curvature(Params p, Box3 r, const double* __restrict__ phi,
                                                  double* __restrict__ curv, double* __restrict__ nrm_m) {
  int i, j, k;
  if (!cell3(r.w0, r.w1, i, j, k)) return;
  const long long n = idxC(p, i, j, k);
  if (k == 0 || k == p.k1 || !in_compute(r, i, j, k)) { curv[n] = 0.; return; }
  const int I = wrapx(p, i), J = wrapy(p, j);
  double m;
  curv[n] = curvature_at(p, phi, I, J, k, m);
  if (I == i && J == j && nrm_m) nrm_m[idxI(p, i, j, k)] = m;
}

// re_curvature + boundc (interface.f90:186-218) over a drop's region
__global__ void __launch_bounds__(NT) k_recurvature(Params p, Box3 r, const double* __restrict__ phi,
                                                    const double* __restrict__ cin, double* __restrict__ out) {
  int i, j, k;
  if (!cell3(r.w0, r.w1, i, j, k)) return;
  const long long n = idxC(p, i, j, k);
  if (k == 0 || k == p.k1 || !in_compute(r, i, j, k)) { out[n] = 0.; return; }
  const int I = wrapx(p, i), J = wrapy(p, j);
  double acc = 0.;
  if (fabs(phi[idxL(p, I, J, k)]) < 2. * p.dz) {
    const long long c = idxC(p, I, J, k), sy = p.nCx, sz = (long long)p.nCx * p.nCy;
    int q = 0;
#pragma unroll
    for (int dk = -1; dk <= 1; ++dk)
#pragma unroll
      for (int dj = -1; dj <= 1; ++dj)
#pragma unroll
        for (int di = -1; di <= 1; ++di) acc = acc + cP[q++] * cin[c + di + dj * sy + dk * sz];
  }
  out[n] = acc;
}

// icurvature, 3-D and TwoD branches (interface.f90:126-179)
__device__ __forceinline__ double icurvature(const Params& p, int nb, double ph0, double phn, double cv0,
                                             double cvn) {
  double sp = 0.;
  if (cv0 < 0.) sp = -1.;
  if (cv0 > 0.) sp = 1.;
  const double eps_0 = sp * ph0, eps_nb = sp * phn;
  if (p.TwoD) {
    if (cv0 * cvn > 0.) {
      const double r_0 = -1. / cv0 + eps_0;
      const double r_nb = -1. / cvn + eps_nb;
      const double r_i = (r_0 + r_nb) / 2.;
      return -1. / r_i;
    }
    return 0.;
  }
  if (cv0 * cvn > 0.) {
    const double a1 = eps_nb * cv0;
    const double a2 = eps_0 * cvn;
    return (a1 - a2) / (eps_nb - eps_0);
  }
  return 0.;
  (void)nb;
}

// a/(h*h) as the reference evaluates jump/dx**2 (gfm.f90:191)
__device__ __forceinline__ double div2(const Params& p, double a, double h, double rh) {
  return p.pow2 ? a * (rh * rh) : a / (h * h);
}

// jumps of one axis: jp(-1) + jp(0) + jp(1) and the + face jump
__device__ __forceinline__ double axis_jump(const Params& p, const double* __restrict__ phi,
                                            const double* __restrict__ cv, long long cl, long long sl,
                                            long long cc, long long sc, double& pface) {
  const double ph0 = phi[cl], phm = phi[cl - sl], php = phi[cl + sl];
  const double c0 = cv[cc], cm = cv[cc - sc], cpp = cv[cc + sc];
  double jm = 0., jp = 0.;
  pface = 0.;
  if (ph0 * phm < 0.) jm = p.nondi * (-icurvature(p, -1, ph0, phm, c0, cm));
  if (ph0 * php < 0.) {
    jp = p.nondi * (-icurvature(p, 1, ph0, php, c0, cpp));
    pface = jp;
  }
  return (jm + 0.) + jp;
}

// gfm4p jump shell of drop l (gfm.f90:95-238); first=1 assigns (l=1)
__global__ void __launch_bounds__(NT) k_jumps(Params p, Box3 r, const double* __restrict__ phi,
                                              const double* __restrict__ cv, int first,
                                              double* __restrict__ pjump, double* __restrict__ px,
                                              double* __restrict__ py, double* __restrict__ pz) {
  int i, j, k;
  if (!cell3(r.c0, r.c1, i, j, k)) return;
  if (i < 1 || i > p.imax || j < 1 || j > p.jmax || k < 1 || k > p.kmax) return;
  const long long cl = idxL(p, i, j, k);
  const double lv = phi[cl];
  if (!(fabs(lv) <= 2. * p.dz)) return;
  const long long cc = idxC(p, i, j, k);
  double fx, fy, fz;
  const double jump_x = axis_jump(p, phi, cv, cl, 1, cc, 1, fx);
  const double jump_y = axis_jump(p, phi, cv, cl, p.nLx, cc, p.nCx, fy);
  const double jump_z = axis_jump(p, phi, cv, cl, (long long)p.nLx * p.nLy, cc, (long long)p.nCx * p.nCy, fz);
  double pj;
  if (lv > 0.) {
    pj = (div2(p, jump_x, p.dx, p.rdx) + div2(p, jump_y, p.dy, p.rdy)) + div2(p, jump_z, p.dz, p.rdz);
  } else if (lv < 0.) {
    pj = -((div2(p, jump_x, p.dx, p.rdx) + div2(p, jump_y, p.dy, p.rdy)) + div2(p, jump_z, p.dz, p.rdz));
    fx = -fx; fy = -fy; fz = -fz;
  } else {
    pj = 0.; fx = 0.; fy = 0.; fz = 0.;
  }
  if (first) {
    pjump[cc] = pj; px[cc] = fx; py[cc] = fy; pz[cc] = fz;
  } else {
    pjump[cc] = pjump[cc] + pj; px[cc] = px[cc] + fx; py[cc] = py[cc] + fy; pz[cc] = pz[cc] + fz;
  }
}

// ipot: dtemp(m,n) = minval(where(|phi_m|<dz and phi_n<cutoff) phi_m+phi_n, 1e3)
__device__ __forceinline__ unsigned long long ord_bits(double x) {
  unsigned long long b = (unsigned long long)__double_as_longlong(x);
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}
__global__ void __launch_bounds__(NT) k_ipot_pair(Params p, Box3 r, const double* __restrict__ pm,
                                                  const double* __restrict__ pn,
                                                  unsigned long long* __restrict__ out) {
  int i, j, k;
  double s = 1e3;
  if (cell3(r.w0, r.w1, i, j, k)) {
    const long long n = idxL(p, i, j, k);
    const double a = pm[n], b = pn[n];
    if (a > -1. * p.dz && a < 1. * p.dz && b < p.NB) s = a + b;
  }
  // block min through the ordered bit pattern
  unsigned long long bits = ord_bits(s);
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long t = __shfl_down_sync(0xffffffffu, bits, o);
    bits = t < bits ? t : bits;
  }
  __shared__ unsigned long long red[NT / 32];
  if ((flat_tid() & 31) == 0) red[flat_tid() >> 5] = bits;
  __syncthreads();
  if (flat_tid() == 0) {
    unsigned long long m = red[0];
    for (int w = 1; w < NT / 32; ++w) m = red[w] < m ? red[w] : m;
    atomicMin(out, m);
  }
}

}  // namespace

void set_pseudo_inverse(const double* P270, cudaStream_t s) {
  cudaMemcpyToSymbolAsync(cP, P270, 270 * sizeof(double), 0, cudaMemcpyHostToDevice, s);
}

void launch_curvature(Ctx& c, const Box3& b, const double* phi, double* curv_out, double* nrm_m_out) {
  Scope sc_(c.prof, c.s, "curvature", 1);
  const Box3 r = c_region(c.P, b, 1);
  k_curvature<<<grid_of(r.w0, r.w1), dim3(BX, BY, 1), 0, c.s>>>(c.P, r, phi, curv_out, nrm_m_out);
}
void launch_recurvature(Ctx& c, const Box3& b, const double* phi, const double* curv_in, double* out) {
  Scope sc_(c.prof, c.s, "recurvature", 1);
  const Box3 r = c_region(c.P, b, 1);
  k_recurvature<<<grid_of(r.w0, r.w1), dim3(BX, BY, 1), 0, c.s>>>(c.P, r, phi, curv_in, out);
}
void launch_jumps(Ctx& c, const Box3& b, const double* phi, const double* cv, int first) {
  Scope sc_(c.prof, c.s, "jumps", 1);
  const Box3 r = c_region(c.P, b, 0);
  k_jumps<<<grid_of(r.c0, r.c1), dim3(BX, BY, 1), 0, c.s>>>(c.P, r, phi, cv, first, c.pjump, c.px, c.py, c.pz);
}
// dmin_dev: L*L unsigned long long ordered bits, filled here
// only the overlap of the two drops' write regions can hold cells with
// |phi_m| < dz and phi_n < 6dz: elsewhere one of them is in its far field
void launch_ipot(Ctx& c, double* dmin_dev) {
  unsigned long long* o = reinterpret_cast<unsigned long long*>(dmin_dev);
  for (int m = 0; m < c.P.L; ++m)
    for (int n = 0; n < c.P.L; ++n) {
      if (m == n) continue;
      const Box3& a = c.win[m].valid;
      const Box3& b = c.win[n].valid;
      Box3 r;
      bool empty = false;
      for (int ax = 0; ax < 3; ++ax) {
        r.w0[ax] = r.c0[ax] = std::max(a.w0[ax], b.w0[ax]);
        r.w1[ax] = r.c1[ax] = std::min(a.w1[ax], b.w1[ax]);
        if (r.w0[ax] > r.w1[ax]) empty = true;
      }
      if (empty) continue;
      Scope sc_(c.prof, c.s, "ipot", 1);
      k_ipot_pair<<<grid_of(r.w0, r.w1), dim3(BX, BY, 1), 0, c.s>>>(c.P, r, c.lv[m], c.lv[n],
                                                                    o + m + (long long)c.P.L * n);
    }
}

}  // namespace icls
