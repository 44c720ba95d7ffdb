// k_navier.cu — momentum, projection and check kernels (FP64, -fmad=false).
//
//   mom_main       mom.f90:13-62 (CNTR2_conv 67-130, delta_diff 134-273,
//                  NS_grav 277-301)
//   ab2            ab2.f90:21-138 with momxp/yp/zp mom.f90:779-851
//   fillps         fillps.f90:13-57
//   correc         correc.f90:15-44
//   bounduvw/boundp bound.f90:15-287
//   pressure update main.f90:164-185
//   averages       misc.f90:587-655;  chkdiv chkdiv.f90:10-90;
//   chkdt          chkdt.f90:11-105
//
// Boundary rows and periodic halos are produced in the kernel that computes
// the field: a halo or wall cell evaluates the interior value(s) it copies
// or extrapolates from (bound.f90:36-75), so no separate boundary pass runs.
#include "ctx.h"

namespace icls {

namespace {

constexpr int NT = 256;
inline unsigned nblocks(long long n, int nt = NT) { return (unsigned)((n + nt - 1) / nt); }

__device__ __forceinline__ void decodeI(const Params& p, int q, int& i, int& j, int& k) {
  i = q % p.imax + 1;
  const int r = q / p.imax;
  j = r % p.jmax + 1;
  k = r / p.jmax + 1;
}

__constant__ int kC0[3] = {0, 0, 0};
__constant__ int kI0[3] = {1, 1, 1};
struct I3 {
  int v[3];
};
__device__ __forceinline__ I3 cC1(const Params& p) { return I3{{p.i1, p.j1, p.k1}}; }
__device__ __forceinline__ I3 cI1(const Params& p) { return I3{{p.imax, p.jmax, p.kmax}}; }
const dim3 kBlock(BX, BY, 1);
inline dim3 gridC(const Params& p) {
  return dim3((unsigned)((p.nCx + BX - 1) / BX), (unsigned)((p.nCy + BY - 1) / BY), (unsigned)p.nCz);
}
inline dim3 gridI(const Params& p) {
  return dim3((unsigned)((p.imax + BX - 1) / BX), (unsigned)((p.jmax + BY - 1) / BY), (unsigned)p.kmax);
}

struct MomArgs {
  const double *u, *v, *w, *miu, *rho_u, *rho_v, *rho_w;
  const double *duold, *dvold, *dwold;
  const double *pnew, *pold, *px, *py, *pz, *pxold, *pyold, *pzold;
  const double* rho_avr;
};

// ---- RHS of mom_main for one component at interior (i,j,k) -------------
__device__ __forceinline__ double rhs_u(const Params& p, const MomArgs& a, int i, int j, int k, double rho_avr) {
  const double *u = a.u, *v = a.v, *w = a.w, *miu = a.miu;
  const long long c = idxC(p, i, j, k);
  const long long sx = 1, sy = p.nCx, sz = (long long)p.nCx * p.nCy;
  double RCu = 0.;
  if (!p.TwoD) {
    double uuip = 0.25 * (u[c + sx] + u[c]) * (u[c + sx] + u[c]);
    double uuim = 0.25 * (u[c - sx] + u[c]) * (u[c - sx] + u[c]);
    double uvjp = 0.25 * (u[c + sy] + u[c]) * (v[c + sx] + v[c]);
    double uvjm = 0.25 * (u[c - sy] + u[c]) * (v[c + sx - sy] + v[c - sy]);
    double uwkp = 0.25 * (u[c + sz] + u[c]) * (w[c + sx] + w[c]);
    double uwkm = 0.25 * (u[c - sz] + u[c]) * (w[c + sx - sz] + w[c - sz]);
    RCu = (divx(p, (-uuip + uuim)) + divy(p, (-uvjp + uvjm))) + divz(p, (-uwkp + uwkm));
  }
  double RDu = 0.;
  if (!p.TwoD) {
    double dudxp = divx(p, (u[c + sx] - u[c]));
    double dudxm = divx(p, (u[c] - u[c - sx]));
    double dudyp = divy(p, (u[c + sy] - u[c]));
    double dudym = divy(p, (u[c] - u[c - sy]));
    double dvdxp = divx(p, (v[c + sx] - v[c]));
    double dvdxm = divx(p, (v[c + sx - sy] - v[c - sy]));
    double dudzp = divz(p, (u[c + sz] - u[c]));
    double dudzm = divz(p, (u[c] - u[c - sz]));
    double dwdxp = divx(p, (w[c + sx] - w[c]));
    double dwdxm = divx(p, (w[c + sx - sz] - w[c - sz]));
    double ma1 = 0.25 * (((miu[c] + miu[c - sy]) + miu[c + sx - sy]) + miu[c + sx]);
    double ma2 = 0.25 * (((miu[c] + miu[c + sy]) + miu[c + sx + sy]) + miu[c + sx]);
    double ma3 = 0.25 * (((miu[c] + miu[c - sz]) + miu[c + sx - sz]) + miu[c + sx]);
    double ma4 = 0.25 * (((miu[c] + miu[c + sz]) + miu[c + sx + sz]) + miu[c + sx]);
    double RD1 = divx(p, 2. * (dudxp * miu[c + sx] - dudxm * miu[c]));
    double RD2 = divy(p, (dudyp * ma2 - dudym * ma1));
    double RD3 = divy(p, (dvdxp * ma2 - dvdxm * ma1));
    double RD4 = divz(p, (dudzp * ma4 - dudzm * ma3));
    double RD5 = divz(p, (dwdxp * ma4 - dwdxm * ma3));
    RDu = ((((RD1 + RD2) + RD3) + RD4) + RD5) / a.rho_u[idxI(p, i, j, k)];
  }
  double RGu = p.TwoD ? 0. : p.iFr * (1. - rho_avr / a.rho_u[idxI(p, i, j, k)]) * p.g1;
  return (RCu + RDu * p.visc) + RGu;
}

__device__ __forceinline__ double rhs_v(const Params& p, const MomArgs& a, int i, int j, int k, double rho_avr) {
  const double *u = a.u, *v = a.v, *w = a.w, *miu = a.miu;
  const long long c = idxC(p, i, j, k);
  const long long sx = 1, sy = p.nCx, sz = (long long)p.nCx * p.nCy;
  double uvip = 0.25 * (u[c] + u[c + sy]) * (v[c] + v[c + sx]);
  double uvim = 0.25 * (u[c - sx] + u[c - sx + sy]) * (v[c] + v[c - sx]);
  double vvjp = 0.25 * (v[c] + v[c + sy]) * (v[c] + v[c + sy]);
  double vvjm = 0.25 * (v[c] + v[c - sy]) * (v[c] + v[c - sy]);
  double wvkp = 0.25 * (w[c] + w[c + sy]) * (v[c + sz] + v[c]);
  double wvkm = 0.25 * (w[c - sz] + w[c + sy - sz]) * (v[c - sz] + v[c]);
  double RCv = (divx(p, (-uvip + uvim)) + divy(p, (-vvjp + vvjm))) + divz(p, (-wvkp + wvkm));
  double dvdxp = divx(p, (v[c + sx] - v[c]));
  double dvdxm = divx(p, (v[c] - v[c - sx]));
  double dudyp = divy(p, (u[c + sy] - u[c]));
  double dudym = divy(p, (u[c - sx + sy] - u[c - sx]));
  double dvdyp = divy(p, (v[c + sy] - v[c]));
  double dvdym = divy(p, (v[c] - v[c - sy]));
  double dvdzp = divz(p, (v[c + sz] - v[c]));
  double dvdzm = divz(p, (v[c] - v[c - sz]));
  double dwdyp = divy(p, (w[c + sy] - w[c]));
  double dwdym = divy(p, (w[c + sy - sz] - w[c - sz]));
  double ma2 = 0.25 * (((miu[c] + miu[c + sy]) + miu[c + sx + sy]) + miu[c + sx]);
  double ma5 = 0.25 * (((miu[c] + miu[c + sy]) + miu[c - sx + sy]) + miu[c - sx]);
  double ma6 = 0.25 * (((miu[c] + miu[c - sz]) + miu[c + sy - sz]) + miu[c + sy]);
  double ma7 = 0.25 * (((miu[c] + miu[c + sz]) + miu[c + sy + sz]) + miu[c + sy]);
  double RD1 = divx(p, (dvdxp * ma2 - dvdxm * ma5));
  double RD2 = divx(p, (dudyp * ma2 - dudym * ma5));
  double RD3 = divy(p, 2. * (dvdyp * miu[c + sy] - dvdym * miu[c]));
  double RD4 = divz(p, (dvdzp * ma7 - dvdzm * ma6));
  double RD5 = divz(p, (dwdyp * ma7 - dwdym * ma6));
  const double rv = a.rho_v[idxI(p, i, j, k)];
  double RDv = ((((RD1 + RD2) + RD3) + RD4) + RD5) / rv;
  double RGv = p.iFr * (1. - rho_avr / rv) * p.g2;
  return (RCv + RDv * p.visc) + RGv;
}

__device__ __forceinline__ double rhs_w(const Params& p, const MomArgs& a, int i, int j, int k, double rho_avr) {
  const double *u = a.u, *v = a.v, *w = a.w, *miu = a.miu;
  const long long c = idxC(p, i, j, k);
  const long long sx = 1, sy = p.nCx, sz = (long long)p.nCx * p.nCy;
  double uwip = 0.25 * (w[c] + w[c + sx]) * (u[c] + u[c + sz]);
  double uwim = 0.25 * (w[c] + w[c - sx]) * (u[c - sx] + u[c - sx + sz]);
  double vwjp = 0.25 * (w[c] + w[c + sy]) * (v[c] + v[c + sz]);
  double vwjm = 0.25 * (w[c] + w[c - sy]) * (v[c - sy] + v[c - sy + sz]);
  double wwkp = 0.25 * (w[c] + w[c + sz]) * (w[c] + w[c + sz]);
  double wwkm = 0.25 * (w[c] + w[c - sz]) * (w[c] + w[c - sz]);
  double RCw = (divx(p, (-uwip + uwim)) + divy(p, (-vwjp + vwjm))) + divz(p, (-wwkp + wwkm));
  double dwdxp = divx(p, (w[c + sx] - w[c]));
  double dwdxm = divx(p, (w[c] - w[c - sx]));
  double dudzp = divz(p, (u[c + sz] - u[c]));
  double dudzm = divz(p, (u[c - sx + sz] - u[c - sx]));
  double dwdyp = divy(p, (w[c + sy] - w[c]));
  double dwdym = divy(p, (w[c] - w[c - sy]));
  double dvdzp = divz(p, (v[c + sz] - v[c]));
  double dvdzm = divz(p, (v[c - sy + sz] - v[c - sy]));
  double dwdzp = divz(p, (w[c + sz] - w[c]));
  double dwdzm = divz(p, (w[c] - w[c - sz]));
  double ma4 = 0.25 * (((miu[c] + miu[c + sz]) + miu[c + sx + sz]) + miu[c + sx]);
  double ma8 = 0.25 * (((miu[c] + miu[c + sz]) + miu[c - sx + sz]) + miu[c - sx]);
  double ma7 = 0.25 * (((miu[c] + miu[c + sz]) + miu[c + sy + sz]) + miu[c + sy]);
  double ma9 = 0.25 * (((miu[c] + miu[c + sz]) + miu[c - sy + sz]) + miu[c - sy]);
  double RD1 = divx(p, (dwdxp * ma4 - dwdxm * ma8));
  double RD2 = divx(p, (dudzp * ma4 - dudzm * ma8));
  double RD3 = divy(p, (dwdyp * ma7 - dwdym * ma9));
  double RD4 = divy(p, (dvdzp * ma7 - dvdzm * ma9));
  double RD5 = divz(p, 2. * (dwdzp * miu[c + sz] - dwdzm * miu[c]));
  const double rw = a.rho_w[idxI(p, i, j, k)];
  double RDw = ((((RD1 + RD2) + RD3) + RD4) + RD5) / rw;
  double RGw = p.iFr * (1. - rho_avr / rw) * p.g3;
  return (RCw + RDw * p.visc) + RGw;
}

// ---- ab2 predictor of one component (ab2.f90:51-61, 79-129) -------------
// R is the mom_main RHS stored as the next AB2 history.
__device__ __forceinline__ double ab2_u(const Params& p, const MomArgs& a, int i, int j, int k, double rho_avr,
                                        double& R) {
  R = rhs_u(p, a, i, j, k, rho_avr);
  const long long c = idxC(p, i, j, k), q = idxI(p, i, j, k);
  double d = a.u[c] + p.dt * (1.5 * R - 0.5 * a.duold[q]);
  const double ph_p = 2. * a.pnew[c + 1] - a.pold[c + 1];
  const double ph_0 = 2. * a.pnew[c] - a.pold[c];
  const double pj = 2. * a.px[c] - a.pxold[c];
  const double dun = -((1. / a.rho_u[q] - 1. / p.rho0) * p.dxi * ((ph_p - pj) - ph_0));
  return d + p.dt * dun;
}
__device__ __forceinline__ double ab2_v(const Params& p, const MomArgs& a, int i, int j, int k, double rho_avr,
                                        double& R) {
  R = rhs_v(p, a, i, j, k, rho_avr);
  const long long c = idxC(p, i, j, k), q = idxI(p, i, j, k);
  double d = a.v[c] + p.dt * (1.5 * R - 0.5 * a.dvold[q]);
  const long long sy = p.nCx;
  const double ph_p = 2. * a.pnew[c + sy] - a.pold[c + sy];
  const double ph_0 = 2. * a.pnew[c] - a.pold[c];
  const double pj = 2. * a.py[c] - a.pyold[c];
  const double dvn = -((1. / a.rho_v[q] - 1. / p.rho0) * p.dyi * ((ph_p - pj) - ph_0));
  return (d + p.dt * dvn) - p.forceytot * p.dt / a.rho_v[q];
}
__device__ __forceinline__ double ab2_w(const Params& p, const MomArgs& a, int i, int j, int k, double rho_avr,
                                        double& R) {
  R = rhs_w(p, a, i, j, k, rho_avr);
  const long long c = idxC(p, i, j, k), q = idxI(p, i, j, k);
  double d = a.w[c] + p.dt * (1.5 * R - 0.5 * a.dwold[q]);
  const long long sz = (long long)p.nCx * p.nCy;
  const double ph_p = 2. * a.pnew[c + sz] - a.pold[c + sz];
  const double ph_0 = 2. * a.pnew[c] - a.pold[c];
  const double pj = 2. * a.pz[c] - a.pzold[c];
  const double dwn = -((1. / a.rho_w[q] - 1. / p.rho0) * p.dzi * ((ph_p - pj) - ph_0));
  return d + p.dt * dwn;
}

// ab2 over shape C with bounduvw(dudt,dvdt,dwdt) (bound.f90:36-75) in-kernel
__global__ void __launch_bounds__(NT) k_ab2(Params p, MomArgs a, double* __restrict__ dudt,
                                            double* __restrict__ dvdt, double* __restrict__ dwdt,
                                            double* __restrict__ duold_out, double* __restrict__ dvold_out,
                                            double* __restrict__ dwold_out) {
  int i, j, k;
  if (!cell3(kC0, cC1(p).v, i, j, k)) return;
  const long long n = idxC(p, i, j, k);
  const int I = wrapx(p, i), J = wrapy(p, j);
  const double rho_avr = *a.rho_avr;
  double Ru, Rv, Rw, du, dv, dw;
  if (k >= 1 && k <= p.kmax) {
    du = ab2_u(p, a, I, J, k, rho_avr, Ru);
    dv = ab2_v(p, a, I, J, k, rho_avr, Rv);
    dw = ab2_w(p, a, I, J, k, rho_avr, Rw);
    if (k == p.kmax) dw = 0.;
    if (I == i && J == j) {
      const long long q = idxI(p, i, j, k);
      duold_out[q] = Ru;
      dvold_out[q] = Rv;
      dwold_out[q] = Rw;
    }
  } else if (k == 0) {
    du = -ab2_u(p, a, I, J, 1, rho_avr, Ru);
    dv = 2. * p.v_lower - ab2_v(p, a, I, J, 1, rho_avr, Rv);
    dw = 0.;
  } else {
    du = -ab2_u(p, a, I, J, p.kmax, rho_avr, Ru);
    dv = 2. * p.v_upper - ab2_v(p, a, I, J, p.kmax, rho_avr, Rv);
    dw = ab2_w(p, a, I, J, p.kmax - 1, rho_avr, Rw);
  }
  dudt[n] = du;
  dvdt[n] = dv;
  dwdt[n] = dw;
}

// mom_main alone (init.f90:90): RHS into shape-I arrays
__global__ void __launch_bounds__(NT) k_mom_main(Params p, MomArgs a, double* __restrict__ ru,
                                                 double* __restrict__ rv, double* __restrict__ rw) {
  int i, j, k;
  if (!cell3(kI0, cI1(p).v, i, j, k)) return;
  const long long q = idxI(p, i, j, k);
  const double rho_avr = *a.rho_avr;
  ru[q] = rhs_u(p, a, i, j, k, rho_avr);
  rv[q] = rhs_v(p, a, i, j, k, rho_avr);
  rw[q] = rhs_w(p, a, i, j, k, rho_avr);
}

// fillps (fillps.f90:36-53), optionally followed by p = p + p_jump
__global__ void __launch_bounds__(NT) k_fillps(Params p, const double* __restrict__ dudt,
                                               const double* __restrict__ dvdt, const double* __restrict__ dwdt,
                                               const double* __restrict__ pjump, int add, double* __restrict__ out) {
  int i, j, k;
  if (!cell3(kI0, cI1(p).v, i, j, k)) return;
  const long long q = idxI(p, i, j, k);
  const long long c = idxC(p, i, j, k);
  const double coef = p.rho0 / p.dt;
  const double vel_x = (dudt[c] - dudt[c - 1]) * p.dxi;
  const double vel_y = (dvdt[c] - dvdt[c - p.nCx]) * p.dyi;
  const double vel_z = (dwdt[c] - dwdt[c - (long long)p.nCx * p.nCy]) * p.dzi;
  double v = coef * ((vel_x + vel_y) + vel_z);
  if (add) v = v + pjump[c];
  out[c] = v;
}

__global__ void __launch_bounds__(NT) k_add(Params p, double* __restrict__ a, const double* __restrict__ b) {
  const long long n = blockIdx.x * (long long)NT + threadIdx.x;
  if (n < p.nC) a[n] = a[n] + b[n];
}

// correc of one component (correc.f90:27-39)
__device__ __forceinline__ double corr_u(const Params& p, const double* dudt, const double* pp, const double* px,
                                         int i, int j, int k) {
  const long long c = idxC(p, i, j, k);
  return dudt[c] - p.dt * p.dxi * ((pp[c + 1] - pp[c]) - px[c]) / p.rho0;
}
__device__ __forceinline__ double corr_v(const Params& p, const double* dvdt, const double* pp, const double* py,
                                         int i, int j, int k) {
  const long long c = idxC(p, i, j, k);
  return dvdt[c] - p.dt * p.dyi * ((pp[c + p.nCx] - pp[c]) - py[c]) / p.rho0;
}
__device__ __forceinline__ double corr_w(const Params& p, const double* dwdt, const double* pp, const double* pz,
                                         int i, int j, int k) {
  const long long c = idxC(p, i, j, k);
  return dwdt[c] - p.dt * p.dzi * ((pp[c + (long long)p.nCx * p.nCy] - pp[c]) - pz[c]) / p.rho0;
}

struct CorrArgs {
  const double *dudt, *dvdt, *dwdt, *p, *px, *py, *pz;
  double *u, *v, *w, *ucc, *vcc, *wcc;
  DevScalars* dsc;
};

// correc over the interior only (the separate reference call)
__global__ void __launch_bounds__(NT) k_correc_interior(Params p, CorrArgs a) {
  int i, j, k;
  if (!cell3(kI0, cI1(p).v, i, j, k)) return;
  const long long q = idxI(p, i, j, k);
  const long long c = idxC(p, i, j, k);
  a.u[c] = corr_u(p, a.dudt, a.p, a.px, i, j, k);
  a.v[c] = corr_v(p, a.dvdt, a.p, a.py, i, j, k);
  a.w[c] = corr_w(p, a.dwdt, a.p, a.pz, i, j, k);
}

// correc + bounduvw(unew,vnew,wnew) + average_vel_at_center + NaN probe
// (main.f90:159-160,190,207) over shape C
__global__ void __launch_bounds__(NT) k_correc_fused(Params p, CorrArgs a) {
  int i, j, k;
  if (!cell3(kC0, cC1(p).v, i, j, k)) return;
  const long long n = idxC(p, i, j, k);
  const int I = wrapx(p, i), J = wrapy(p, j);
  double uu, vv, ww;
  if (k >= 1 && k <= p.kmax) {
    uu = corr_u(p, a.dudt, a.p, a.px, I, J, k);
    vv = corr_v(p, a.dvdt, a.p, a.py, I, J, k);
    ww = (k == p.kmax) ? 0. : corr_w(p, a.dwdt, a.p, a.pz, I, J, k);
  } else if (k == 0) {
    uu = -corr_u(p, a.dudt, a.p, a.px, I, J, 1);
    vv = 2. * p.v_lower - corr_v(p, a.dvdt, a.p, a.py, I, J, 1);
    ww = 0.;
  } else {
    uu = -corr_u(p, a.dudt, a.p, a.px, I, J, p.kmax);
    vv = 2. * p.v_upper - corr_v(p, a.dvdt, a.p, a.py, I, J, p.kmax);
    ww = corr_w(p, a.dwdt, a.p, a.pz, I, J, p.kmax - 1);
  }
  a.u[n] = uu;
  a.v[n] = vv;
  a.w[n] = ww;
  if (i == I && j == J && k >= 1 && k <= p.kmax) {
    const long long q = idxI(p, i, j, k);
    const double um = corr_u(p, a.dudt, a.p, a.px, wrapx(p, i - 1), j, k);
    const double vm = corr_v(p, a.dvdt, a.p, a.py, i, wrapy(p, j - 1), k);
    const double wm = (k == 1) ? 0. : corr_w(p, a.dwdt, a.p, a.pz, i, j, k - 1);
    a.ucc[q] = (um + uu) / 2.;
    a.vcc[q] = (vm + vv) / 2.;
    a.wcc[q] = (wm + ww) / 2.;
    if (i == 1 && j == 1 && k == 1 && isnan(vv)) a.dsc->nan_flag = 1;
  }
}

// bounduvw (bound.f90:15-177, Dirichl z, periodic x,y) on an existing triple
__global__ void __launch_bounds__(NT) k_bounduvw(Params p, double* __restrict__ u, double* __restrict__ v,
                                                 double* __restrict__ w) {
  int i, j, k;
  if (!cell3(kC0, cC1(p).v, i, j, k)) return;
  const long long n = idxC(p, i, j, k);
  const int I = wrapx(p, i), J = wrapy(p, j);
  const bool col = (I == i && J == j);
  if (k >= 1 && k <= p.kmax) {
    if (!col) {
      u[n] = u[idxC(p, I, J, k)];
      v[n] = v[idxC(p, I, J, k)];
    }
    if (k == p.kmax) w[n] = 0.;
    else if (!col) w[n] = w[idxC(p, I, J, k)];
  } else if (k == 0) {
    u[n] = -u[idxC(p, I, J, 1)];
    v[n] = 2. * p.v_lower - v[idxC(p, I, J, 1)];
    w[n] = 0.;
  } else {
    u[n] = -u[idxC(p, I, J, p.kmax)];
    v[n] = 2. * p.v_upper - v[idxC(p, I, J, p.kmax)];
    w[n] = w[idxC(p, I, J, p.kmax - 1)];
  }
}

// boundp (bound.f90:182-287, BC_in_y='Periodic')
__global__ void __launch_bounds__(NT) k_boundp(Params p, double* __restrict__ a) {
  int i, j, k;
  if (!cell3(kC0, cC1(p).v, i, j, k)) return;
  const long long n = idxC(p, i, j, k);
  const int I = wrapx(p, i), J = wrapy(p, j);
  const int K = k == 0 ? 1 : (k == p.k1 ? p.kmax : k);
  if (I == i && J == j && K == k) return;
  a[n] = a[idxC(p, I, J, K)];
}

// average_vel_at_center (misc.f90:587-604)
__global__ void __launch_bounds__(NT) k_average_vel(Params p, const double* __restrict__ u,
                                                    const double* __restrict__ v, const double* __restrict__ w,
                                                    double* __restrict__ ucc, double* __restrict__ vcc,
                                                    double* __restrict__ wcc) {
  int i, j, k;
  if (!cell3(kI0, cI1(p).v, i, j, k)) return;
  const long long q = idxI(p, i, j, k);
  const long long c = idxC(p, i, j, k);
  ucc[q] = (u[c - 1] + u[c]) / 2.;
  vcc[q] = (v[c - p.nCx] + v[c]) / 2.;
  wcc[q] = (w[c - (long long)p.nCx * p.nCy] + w[c]) / 2.;
}

// ---- pressure update (main.f90:164-185) ----------------------------------
// norm = sum(sum(pnew(:,:,1),2),1) in the Fortran order: for each i the
// sum over j, then the sum of those over i.
__global__ void k_plane_norm(Params p, const double* __restrict__ pp, double* __restrict__ colsum,
                             DevScalars* __restrict__ dsc) {
  for (int i = threadIdx.x; i <= p.i1; i += blockDim.x) {
    double s = 0.;
    for (int j = 0; j <= p.j1; ++j) s += pp[idxC(p, i, j, 1)];
    colsum[i] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.;
    for (int i = 0; i <= p.i1; ++i) s += colsum[i];
    dsc->norm_old = dsc->norm;
    dsc->norm = s / (1. * (p.imax) * p.jmax);
  }
}
__global__ void __launch_bounds__(NT) k_pupdate(Params p, const double* __restrict__ pp,
                                                double* __restrict__ pnew, double* __restrict__ pold, int first,
                                                const DevScalars* __restrict__ dsc) {
  const long long n = blockIdx.x * (long long)NT + threadIdx.x;
  if (n >= p.nC) return;
  const double norm = dsc->norm;
  const double po = pnew[n];
  pold[n] = first ? po - norm : (po + dsc->norm_old) - norm;
  pnew[n] = pp[n] - norm;
}

// ---- reductions ------------------------------------------------------------
__global__ void __launch_bounds__(kRedThreads) k_sum_interior(Params p, const double* __restrict__ a,
                                                              double* __restrict__ partial) {
  double s = 0.;
  for (int q = blockIdx.x * kRedThreads + threadIdx.x; q < (int)p.nI; q += gridDim.x * kRedThreads) {
    int i, j, k;
    decodeI(p, q, i, j, k);
    s += a[idxC(p, i, j, k)];
  }
  double b = block_sum<double, kRedThreads>(s);
  if (threadIdx.x == 0) partial[blockIdx.x] = b;
}
__global__ void k_stream_final(Params p, const double* __restrict__ partial, int nblk,
                               DevScalars* __restrict__ dsc) {
  if (threadIdx.x) return;
  double s = 0.;
  for (int b = 0; b < nblk; ++b) s += partial[b];
  dsc->v_bulk = s / (double)((long long)p.imax * p.jmax * p.kmax);
}

// chkdiv: sum of div and max|div| with its first column-major location
__global__ void __launch_bounds__(kRedThreads) k_chkdiv(Params p, const double* __restrict__ u,
                                                        const double* __restrict__ v, const double* __restrict__ w,
                                                        double* __restrict__ part_sum, double* __restrict__ part_max,
                                                        long long* __restrict__ part_loc) {
  double s = 0., m = 0.;
  long long loc = -1;
  for (int q = blockIdx.x * kRedThreads + threadIdx.x; q < (int)p.nI; q += gridDim.x * kRedThreads) {
    int i, j, k;
    decodeI(p, q, i, j, k);
    const long long c = idxC(p, i, j, k);
    double div = ((w[c] - w[c - (long long)p.nCx * p.nCy]) * p.dzi + (v[c] - v[c - p.nCx]) * p.dyi) +
                 (u[c] - u[c - 1]) * p.dxi;
    s += div;
    div = fabs(div);
    if (div > m) { m = div; loc = (long long)q; }
  }
  __shared__ double sm[kRedThreads];
  __shared__ long long sl[kRedThreads];
  double b = block_sum<double, kRedThreads>(s);
  sm[threadIdx.x] = m;
  sl[threadIdx.x] = loc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double bm = 0.;
    long long bl = -1;
    for (int t = 0; t < kRedThreads; ++t) {
      if (sm[t] > bm || (sm[t] == bm && sm[t] > 0. && sl[t] < bl)) { bm = sm[t]; bl = sl[t]; }
    }
    part_sum[blockIdx.x] = b;
    part_max[blockIdx.x] = bm;
    part_loc[blockIdx.x] = bl;
  }
}
__global__ void k_chkdiv_final(const double* __restrict__ part_sum, const double* __restrict__ part_max,
                               const long long* __restrict__ part_loc, int nblk, DevScalars* __restrict__ dsc) {
  if (threadIdx.x) return;
  double s = 0., m = 0.;
  long long l = -1;
  for (int b = 0; b < nblk; ++b) {
    s += part_sum[b];
    if (part_max[b] > m || (part_max[b] == m && part_max[b] > 0. && part_loc[b] < l)) { m = part_max[b]; l = part_loc[b]; }
  }
  dsc->divtot = s;
  dsc->divmax = m;
  dsc->divloc = l;
}

// chkdt maxima (chkdt.f90:31-52) and max_vel_at_center (misc.f90:619-633)
__global__ void __launch_bounds__(NT) k_chkdt(Params p, const double* __restrict__ u, const double* __restrict__ v,
                                              const double* __restrict__ w, DevScalars* __restrict__ dsc) {
  double a = 0., b = 0., c = 0.;
  int i, j, k;
  const I3 hi = cC1(p);
  if (cell3(kI0, hi.v, i, j, k)) {
    const long long cc = idxC(p, i, j, k);
    a = fabs((u[cc] + u[cc - 1]) / 2.);
    b = fabs((v[cc] + v[cc - p.nCx]) / 2.);
    c = fabs((w[cc] + w[cc - (long long)p.nCx * p.nCy]) / 2.);
  }
  a = block_max<double, NT>(a);
  b = block_max<double, NT>(b);
  c = block_max<double, NT>(c);
  if (flat_tid() == 0) {
    atomic_max_nonneg(&dsc->umax, a);
    atomic_max_nonneg(&dsc->vmax, b);
    atomic_max_nonneg(&dsc->wmax, c);
  }
}
__global__ void __launch_bounds__(NT) k_maxvel(Params p, const double* __restrict__ ucc,
                                               const double* __restrict__ vcc, const double* __restrict__ wcc,
                                               DevScalars* __restrict__ dsc) {
  const long long q = blockIdx.x * (long long)NT + threadIdx.x;
  double m = 0.;
  if (q < p.nI) m = sqrt((ucc[q] * ucc[q] + vcc[q] * vcc[q]) + wcc[q] * wcc[q]);
  m = block_max<double, NT>(m);
  if (threadIdx.x == 0) atomic_max_nonneg(&dsc->velmax, m);
}

MomArgs mom_args(Ctx& c) {
  MomArgs a;
  a.u = c.u; a.v = c.v; a.w = c.w; a.miu = c.miu;
  a.rho_u = c.rho_u; a.rho_v = c.rho_v; a.rho_w = c.rho_w;
  a.duold = c.duold[c.hist]; a.dvold = c.dvold[c.hist]; a.dwold = c.dwold[c.hist];
  a.pnew = c.pnew; a.pold = c.pold;
  a.px = c.px; a.py = c.py; a.pz = c.pz; a.pxold = c.pxold; a.pyold = c.pyold; a.pzold = c.pzold;
  a.rho_avr = &c.dsc->rho_avr;
  return a;
}
CorrArgs corr_args(Ctx& c) {
  CorrArgs a;
  a.dudt = c.dudt; a.dvdt = c.dvdt; a.dwdt = c.dwdt; a.p = c.p; a.px = c.px; a.py = c.py; a.pz = c.pz;
  a.u = c.u; a.v = c.v; a.w = c.w; a.ucc = c.ucc; a.vcc = c.vcc; a.wcc = c.wcc; a.dsc = c.dsc;
  return a;
}

}  // namespace

// ================================================================ launchers
void launch_ab2(Ctx& c) {
  Scope sc_(c.prof, c.s, "ab2", 1);
  MomArgs a = mom_args(c);
  const int o = c.hist ^ 1;
  k_ab2<<<gridC(c.P), kBlock, 0, c.s>>>(c.P, a, c.dudt, c.dvdt, c.dwdt, c.duold[o], c.dvold[o], c.dwold[o]);
  c.hist = o;
}
void launch_mom_main(Ctx& c, double* du, double* dv, double* dw) {
  Scope sc_(c.prof, c.s, "mom_main", 1);
  MomArgs a = mom_args(c);
  k_mom_main<<<gridI(c.P), kBlock, 0, c.s>>>(c.P, a, du, dv, dw);
}
void launch_fillps(Ctx& c, int add_pjump) {
  Scope sc_(c.prof, c.s, "fillps", 1);
  k_fillps<<<gridI(c.P), kBlock, 0, c.s>>>(c.P, c.dudt, c.dvdt, c.dwdt, c.pjump, add_pjump, c.p);
}
void launch_add_pjump(Ctx& c) {
  Scope sc_(c.prof, c.s, "add_pjump", 1); k_add<<<nblocks(c.P.nC), NT, 0, c.s>>>(c.P, c.p, c.pjump); }
void launch_correc(Ctx& c, int fused_bc) {
  Scope sc_(c.prof, c.s, "correc", 1);
  CorrArgs a = corr_args(c);
  if (fused_bc) k_correc_fused<<<gridC(c.P), kBlock, 0, c.s>>>(c.P, a);
  else k_correc_interior<<<gridI(c.P), kBlock, 0, c.s>>>(c.P, a);
}
void launch_bounduvw(Ctx& c, double* u, double* v, double* w) {
  Scope sc_(c.prof, c.s, "bounduvw", 1);
  k_bounduvw<<<gridC(c.P), kBlock, 0, c.s>>>(c.P, u, v, w);
}
void launch_boundp(Ctx& c, double* pp) {
  Scope sc_(c.prof, c.s, "boundp", 1); k_boundp<<<gridC(c.P), kBlock, 0, c.s>>>(c.P, pp); }
void launch_average_vel(Ctx& c) {
  Scope sc_(c.prof, c.s, "average_vel", 1);
  k_average_vel<<<gridI(c.P), kBlock, 0, c.s>>>(c.P, c.u, c.v, c.w, c.ucc, c.vcc, c.wcc);
}
void launch_pressure_update(Ctx& c, int first) {
  Scope sc_(c.prof, c.s, "pressure_update", 2);
  k_plane_norm<<<1, 512, 0, c.s>>>(c.P, c.p, c.partials, c.dsc);
  k_pupdate<<<nblocks(c.P.nC), NT, 0, c.s>>>(c.P, c.p, c.pnew, c.pold, first, c.dsc);
}
void launch_stream_vel(Ctx& c) {
  Scope sc_(c.prof, c.s, "stream_vel", 2);
  k_sum_interior<<<kRedBlocks, kRedThreads, 0, c.s>>>(c.P, c.v, c.partials);
  k_stream_final<<<1, 32, 0, c.s>>>(c.P, c.partials, kRedBlocks, c.dsc);
}
void launch_chkdiv(Ctx& c) {
  Scope sc_(c.prof, c.s, "chkdiv", 2);
  double* ps = c.partials;
  double* pm = c.partials + kRedBlocks;
  k_chkdiv<<<kRedBlocks, kRedThreads, 0, c.s>>>(c.P, c.u, c.v, c.w, ps, pm, c.lpartials);
  k_chkdiv_final<<<1, 32, 0, c.s>>>(ps, pm, c.lpartials, kRedBlocks, c.dsc);
}
void launch_chkdt(Ctx& c) {
  Scope sc_(c.prof, c.s, "chkdt", 1);
  cudaMemsetAsync(&c.dsc->umax, 0, 3 * sizeof(double), c.s);
  k_chkdt<<<gridC(c.P), kBlock, 0, c.s>>>(c.P, c.u, c.v, c.w, c.dsc);
}
void launch_maxvel(Ctx& c) {
  Scope sc_(c.prof, c.s, "maxvel", 1);
  cudaMemsetAsync(&c.dsc->velmax, 0, sizeof(double), c.s);
  k_maxvel<<<nblocks(c.P.nI), NT, 0, c.s>>>(c.P, c.ucc, c.vcc, c.wcc, c.dsc);
}

}  // namespace icls
