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
#include <algorithm>

#include "ab2.cuh"
#include "batch.cuh"

namespace icls {

namespace {

constexpr int NT = 256;
// T is the form's field type (double, or float in the precision form);
// TC(x) is the constant x in T
#define TC(x) static_cast<T>(x)
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


// mom_main alone (init.f90:90): RHS into shape-I arrays
template <typename T>
__global__ void __launch_bounds__(NT) k_mom_main(Params p, MomArgs a, T* __restrict__ ru, T* __restrict__ rv,
                                                 T* __restrict__ rw) {
  int i, j, k;
  if (!cell3(kI0, cI1(p).v, i, j, k)) return;
  const long long q = idxI(p, i, j, k);
  const long long c = idxC(p, i, j, k);
  const long long sy = p.nCx, sz = (long long)p.nCx * p.nCy;
  const T rho_avr = TC(*a.rho_avr);
  const T *u = cT<T>(a.u), *v = cT<T>(a.v), *w = cT<T>(a.w), *miu = cT<T>(a.miu);
  auto U = [&](int di, int dj, int dk) { return u[c + di + dj * sy + dk * sz]; };
  auto V = [&](int di, int dj, int dk) { return v[c + di + dj * sy + dk * sz]; };
  auto W = [&](int di, int dj, int dk) { return w[c + di + dj * sy + dk * sz]; };
  auto M = [&](int di, int dj, int dk) { return miu[c + di + dj * sy + dk * sz]; };
  ru[q] = rhs_u<T>(p, U, V, W, M, cT<T>(a.rho_u)[q], rho_avr);
  rv[q] = rhs_v<T>(p, U, V, W, M, cT<T>(a.rho_v)[q], rho_avr);
  rw[q] = rhs_w<T>(p, U, V, W, M, cT<T>(a.rho_w)[q], rho_avr);
}

// fillps (fillps.f90:36-53), optionally followed by p = p + p_jump
template <typename T>
__global__ void __launch_bounds__(NT) k_fillps(Params p, const T* __restrict__ dudt, const T* __restrict__ dvdt,
                                               const T* __restrict__ dwdt, const double* __restrict__ pjump, int add,
                                               double* __restrict__ out) {
  int i, j, k;
  if (!cell3(kI0, cI1(p).v, i, j, k)) return;
  const long long q = idxI(p, i, j, k);
  const long long c = idxC(p, i, j, k);
  const double coef = p.rho0 / p.dt;
  const double vel_x = ((double)dudt[c] - (double)dudt[c - 1]) * p.dxi;
  const double vel_y = ((double)dvdt[c] - (double)dvdt[c - p.nCx]) * p.dyi;
  const double vel_z = ((double)dwdt[c] - (double)dwdt[c - (long long)p.nCx * p.nCy]) * p.dzi;
  double v = coef * ((vel_x + vel_y) + vel_z);
  if (add) v = v + pjump[c];
  out[c] = v;
}

__global__ void __launch_bounds__(NT) k_add(Params p, double* __restrict__ a, const double* __restrict__ b) {
  const long long n = blockIdx.x * (long long)NT + threadIdx.x;
  if (n < p.nC) a[n] = a[n] + b[n];
}

// correc of one component (correc.f90:27-39)
// (the pressure gradient in FP64, the result in the form's type T)
template <typename T>
__device__ __forceinline__ T corr_u(const Params& p, const T* dudt, const double* pp, const T* px, int i, int j,
                                    int k) {
  const long long c = idxC(p, i, j, k);
  if (sizeof(T) == sizeof(double)) return (T)(dudt[c] - div_rho0(p, p.dt * p.dxi * ((pp[c + 1] - pp[c]) - (double)px[c])));
  return dudt[c] - (T)(div_rho0(p, p.dt * p.dxi * ((pp[c + 1] - pp[c]) - (double)px[c])));
}
template <typename T>
__device__ __forceinline__ T corr_v(const Params& p, const T* dvdt, const double* pp, const T* py, int i, int j,
                                    int k) {
  const long long c = idxC(p, i, j, k);
  if (sizeof(T) == sizeof(double)) return (T)(dvdt[c] - div_rho0(p, p.dt * p.dyi * ((pp[c + p.nCx] - pp[c]) - (double)py[c])));
  return dvdt[c] - (T)(div_rho0(p, p.dt * p.dyi * ((pp[c + p.nCx] - pp[c]) - (double)py[c])));
}
template <typename T>
__device__ __forceinline__ T corr_w(const Params& p, const T* dwdt, const double* pp, const T* pz, int i, int j,
                                    int k) {
  const long long c = idxC(p, i, j, k);
  const long long sz = (long long)p.nCx * p.nCy;
  if (sizeof(T) == sizeof(double)) return (T)(dwdt[c] - div_rho0(p, p.dt * p.dzi * ((pp[c + sz] - pp[c]) - (double)pz[c])));
  return dwdt[c] - (T)(div_rho0(p, p.dt * p.dzi * ((pp[c + sz] - pp[c]) - (double)pz[c])));
}

struct CorrArgs {
  const double *dudt, *dvdt, *dwdt, *p, *px, *py, *pz;
  double *u, *v, *w, *ucc, *vcc, *wcc;
  DevScalars* dsc;
};

// correc over the interior only (the separate reference call)
template <typename T>
__global__ void __launch_bounds__(NT) k_correc_interior(Params p, CorrArgs a) {
  int i, j, k;
  if (!cell3(kI0, cI1(p).v, i, j, k)) return;
  const long long c = idxC(p, i, j, k);
  mT<T>(a.u)[c] = corr_u(p, cT<T>(a.dudt), a.p, cT<T>(a.px), i, j, k);
  mT<T>(a.v)[c] = corr_v(p, cT<T>(a.dvdt), a.p, cT<T>(a.py), i, j, k);
  mT<T>(a.w)[c] = corr_w(p, cT<T>(a.dwdt), a.p, cT<T>(a.pz), i, j, k);
}

// correc + bounduvw(unew,vnew,wnew) + average_vel_at_center + NaN probe
// (main.f90:159-160,190,207) over shape C
template <typename T>
__global__ void __launch_bounds__(NT) k_correc_fused(Params p, CorrArgs a) {
  int i, j, k;
  if (!cell3(kC0, cC1(p).v, i, j, k)) return;
  const long long n = idxC(p, i, j, k);
  const int I = wrapx(p, i), J = wrapy(p, j);
  const T *du = cT<T>(a.dudt), *dv = cT<T>(a.dvdt), *dw = cT<T>(a.dwdt);
  T uu, vv, ww;
  if (k >= 1 && k <= p.kmax) {
    uu = corr_u(p, du, a.p, cT<T>(a.px), I, J, k);
    vv = corr_v(p, dv, a.p, cT<T>(a.py), I, J, k);
    ww = (k == p.kmax) ? TC(0.) : corr_w(p, dw, a.p, cT<T>(a.pz), I, J, k);
  } else if (k == 0) {
    uu = -corr_u(p, du, a.p, cT<T>(a.px), I, J, 1);
    vv = TC(2. * p.v_lower) - corr_v(p, dv, a.p, cT<T>(a.py), I, J, 1);
    ww = TC(0.);
  } else {
    uu = -corr_u(p, du, a.p, cT<T>(a.px), I, J, p.kmax);
    vv = TC(2. * p.v_upper) - corr_v(p, dv, a.p, cT<T>(a.py), I, J, p.kmax);
    ww = corr_w(p, dw, a.p, cT<T>(a.pz), I, J, p.kmax - 1);
  }
  mT<T>(a.u)[n] = uu;
  mT<T>(a.v)[n] = vv;
  mT<T>(a.w)[n] = ww;
  if (i == I && j == J && k >= 1 && k <= p.kmax) {
    const long long q = idxI(p, i, j, k);
    const T um = corr_u(p, du, a.p, cT<T>(a.px), wrapx(p, i - 1), j, k);
    const T vm = corr_v(p, dv, a.p, cT<T>(a.py), i, wrapy(p, j - 1), k);
    const T wm = (k == 1) ? TC(0.) : corr_w(p, dw, a.p, cT<T>(a.pz), i, j, k - 1);
    mT<T>(a.ucc)[q] = (um + uu) / TC(2.);
    mT<T>(a.vcc)[q] = (vm + vv) / TC(2.);
    mT<T>(a.wcc)[q] = (wm + ww) / TC(2.);
    if (i == 1 && j == 1 && k == 1 && isnan(vv)) a.dsc->nan_flag = 1;
  }
}

// One correc value (correc.f90:27-39) at shape-C index c: d - dt dhi
// ((p(c+off) - p(c)) - jump) / rho0, the expression of corr_u/v/w, with
// the division by rho0 chosen at compile time (RP 1: rho0 a power of two,
// the product by its exact reciprocal)
template <typename T, int RP>
__device__ __forceinline__ T corr_at(const Params& p, const T* __restrict__ d, const double* __restrict__ pp,
                                     const T* __restrict__ jump, long long c, long long off, double dhi) {
  const double a = p.dt * dhi * ((pp[c + off] - pp[c]) - (double)jump[c]);
  const double g = RP == 1 ? a * p.rrho0 : a / p.rho0;
  if (sizeof(T) == sizeof(double)) return (T)((double)d[c] - g);
  return d[c] - (T)g;
}

// k_correc_fused's fields with one thread per interior cell: the thread
// writes its cell's u, v, w with their periodic images (putC), at k = 1 and
// k = kmax the wall rows k = 0 and k1 with theirs, and the cell-centre
// velocities.  The halo and wall cells are the images k_correc_fused
// computes from the same source cells, so the fields are the same bits;
// every warp is a full row segment and no thread recomputes a source
// column's corrections for a halo cell.
template <typename T, int RP>
__global__ void __launch_bounds__(NT, (sizeof(T) == 4 ? 8 : 5)) k_correc_own(Params p, CorrArgs a) {
  int i, j, k;
  if (!cell3(kI0, cI1(p).v, i, j, k)) return;
  const long long sy = p.nCx, sz = (long long)p.nCx * p.nCy;
  const long long c = idxC(p, i, j, k);
  const T* __restrict__ du = cT<T>(a.dudt);
  const T* __restrict__ dv = cT<T>(a.dvdt);
  const T* __restrict__ dw = cT<T>(a.dwdt);
  const T* __restrict__ px = cT<T>(a.px);
  const T* __restrict__ py = cT<T>(a.py);
  const T* __restrict__ pz = cT<T>(a.pz);
  const double* __restrict__ pp = a.p;
  const T uu = corr_at<T, RP>(p, du, pp, px, c, 1, p.dxi);
  const T vv = corr_at<T, RP>(p, dv, pp, py, c, sy, p.dyi);
  const T ww = (k == p.kmax) ? TC(0.) : corr_at<T, RP>(p, dw, pp, pz, c, sz, p.dzi);
  // the cell-centre average's (i-1), (j-1) and (k-1) corrections
  const T um = corr_at<T, RP>(p, du, pp, px, idxC(p, wrapx(p, i - 1), j, k), 1, p.dxi);
  const T vm = corr_at<T, RP>(p, dv, pp, py, idxC(p, i, wrapy(p, j - 1), k), sy, p.dyi);
  const T wm = (k == 1) ? TC(0.) : corr_at<T, RP>(p, dw, pp, pz, c - sz, sz, p.dzi);
  T* u = mT<T>(a.u);
  T* v = mT<T>(a.v);
  T* w = mT<T>(a.w);
  putC(p, u, i, j, k, uu);
  putC(p, v, i, j, k, vv);
  putC(p, w, i, j, k, ww);
  if (k == 1) {
    putC(p, u, i, j, 0, -uu);
    putC(p, v, i, j, 0, TC(2. * p.v_lower) - vv);
    putC(p, w, i, j, 0, TC(0.));
  }
  if (k == p.kmax) {
    putC(p, u, i, j, p.k1, -uu);
    putC(p, v, i, j, p.k1, TC(2. * p.v_upper) - vv);
    putC(p, w, i, j, p.k1, corr_at<T, RP>(p, dw, pp, pz, c - sz, sz, p.dzi));
  }
  const long long q = idxI(p, i, j, k);
  mT<T>(a.ucc)[q] = (um + uu) / TC(2.);
  mT<T>(a.vcc)[q] = (vm + vv) / TC(2.);
  mT<T>(a.wcc)[q] = (wm + ww) / TC(2.);
  if (i == 1 && j == 1 && k == 1 && isnan(vv)) a.dsc->nan_flag = 1;
}

// bounduvw (bound.f90:15-177, Dirichl z, periodic x,y) on an existing triple
template <typename T>
__global__ void __launch_bounds__(NT) k_bounduvw(Params p, T* __restrict__ u, T* __restrict__ v, T* __restrict__ w) {
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
    if (k == p.kmax) w[n] = TC(0.);
    else if (!col) w[n] = w[idxC(p, I, J, k)];
  } else if (k == 0) {
    u[n] = -u[idxC(p, I, J, 1)];
    v[n] = TC(2. * p.v_lower) - v[idxC(p, I, J, 1)];
    w[n] = TC(0.);
  } else {
    u[n] = -u[idxC(p, I, J, p.kmax)];
    v[n] = TC(2. * p.v_upper) - v[idxC(p, I, J, p.kmax)];
    w[n] = w[idxC(p, I, J, p.kmax - 1)];
  }
}

// boundp (bound.f90:182-287, BC_in_y='Periodic')
template <typename T>
__global__ void __launch_bounds__(NT) k_boundp(Params p, T* __restrict__ a) {
  int i, j, k;
  if (!cell3(kC0, cC1(p).v, i, j, k)) return;
  const long long n = idxC(p, i, j, k);
  const int I = wrapx(p, i), J = wrapy(p, j);
  const int K = k == 0 ? 1 : (k == p.k1 ? p.kmax : k);
  if (I == i && J == j && K == k) return;
  a[n] = a[idxC(p, I, J, K)];
}

// the y boundaries of bounduvw for BC_in_y = Walls, InOut, OutOut
// (bound.f90:81-172), over i = 1..imax, k = 1..kmax once the periodic halos
// are in place: a thread does its (i,k) front row, then its back row
template <typename T>
__global__ void __launch_bounds__(NT) k_ywalls_uvw(Params p, T* __restrict__ u, T* __restrict__ v,
                                                   T* __restrict__ w, const double* __restrict__ vin) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, k = blockIdx.y + 1;
  if (i > p.imax) return;
  const long long f0 = idxC(p, i, 0, k), f1 = idxC(p, i, 1, k);
  if (p.bcy == ICLS_BCY_WALLS || p.bcy == ICLS_BCY_INOUT) {
    u[f0] = -u[f1];
    w[f0] = -w[f1];
    v[f0] = p.bcy == ICLS_BCY_WALLS ? TC(0.) : TC(vin[i + (long long)(p.i1 + 1) * k]);
  } else {
    u[f0] = u[f1];
    w[f0] = w[f1];
    v[f0] = v[f1] + TC(p.dy / p.dz) * (w[f1] - w[idxC(p, i, 1, k - 1)]);
  }
  const long long bj = idxC(p, i, p.jmax, k), b1 = idxC(p, i, p.j1, k);
  if (p.bcy == ICLS_BCY_WALLS) {
    u[b1] = -u[bj];
    v[bj] = TC(0.);
    v[b1] = v[bj];
    w[b1] = -w[bj];
  } else {
    u[b1] = u[bj];
    v[b1] = TC(2.) * v[bj] - v[idxC(p, i, p.jmax - 1, k)];
    w[b1] = w[bj];
  }
}
// the y boundaries of boundp (bound.f90:207-282): zero Neumann, or zero
// Dirichlet at an outflow end
template <typename T>
__global__ void __launch_bounds__(NT) k_ywalls_p(Params p, T* __restrict__ a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, k = blockIdx.y + 1;
  if (i > p.imax) return;
  const T f = a[idxC(p, i, 1, k)], b = a[idxC(p, i, p.jmax, k)];
  a[idxC(p, i, 0, k)] = p.bcy == ICLS_BCY_OUTOUT ? -f : f;
  a[idxC(p, i, p.j1, k)] = p.bcy == ICLS_BCY_WALLS ? b : -b;
}
// isnan(vnew(1,1,1)) (main.f90:207)
template <typename T>
__global__ void k_nan_probe(Params p, const T* __restrict__ v, DevScalars* __restrict__ dsc) {
  if (isnan(v[idxC(p, 1, 1, 1)])) dsc->nan_flag = 1;
}

// the plane i = const of an array with extents nx x ny x nz: dst(j,k) =
// src(ioff + nx j + nx ny k), j < n1, k < n2, converted to FP64
template <typename T>
__global__ void __launch_bounds__(NT) k_gather_plane_x(const T* __restrict__ src, long long nx, long long nxy, long long ioff,
                                                       int n1, int n2, double* __restrict__ dst) {
  const long long q = blockIdx.x * (long long)NT + threadIdx.x;
  if (q >= (long long)n1 * n2) return;
  const long long j = q % n1, k = q / n1;
  dst[q] = (double)src[ioff + nx * j + nxy * k];
}

// average_vel_at_center (misc.f90:587-604)
template <typename T>
__global__ void __launch_bounds__(NT) k_average_vel(Params p, const T* __restrict__ u, const T* __restrict__ v,
                                                    const T* __restrict__ w, T* __restrict__ ucc, T* __restrict__ vcc,
                                                    T* __restrict__ wcc) {
  int i, j, k;
  if (!cell3(kI0, cI1(p).v, i, j, k)) return;
  const long long q = idxI(p, i, j, k);
  const long long c = idxC(p, i, j, k);
  ucc[q] = (u[c - 1] + u[c]) / TC(2.);
  vcc[q] = (v[c - p.nCx] + v[c]) / TC(2.);
  wcc[q] = (w[c - (long long)p.nCx * p.nCy] + w[c]) / TC(2.);
}

// ---- pressure update (main.f90:164-185) ----------------------------------
// norm = sum(sum(pnew(:,:,1),2),1) in the Fortran order: for each i the
// sum over j, then the sum of those over i.
// the mean of p over the k = 1 plane, halo included (main.f90:173-175), by
// one block: the plane's (i, j) cells in a fixed strided order per thread,
// then a fixed tree
constexpr int kNormThreads = 1024;
__global__ void __launch_bounds__(kNormThreads) k_plane_norm(Params p, const double* __restrict__ pp,
                                                             DevScalars* __restrict__ dsc) {
  const long long n = (long long)p.nCx * p.nCy, base = idxC(p, 0, 0, 1);
  double s = 0.;
  for (long long e = threadIdx.x; e < n; e += kNormThreads) s += pp[base + e];
  s = block_sum<double, kNormThreads>(s);
  if (threadIdx.x == 0) {
    dsc->norm_old = dsc->norm;
    dsc->norm = s / (1. * (p.imax) * p.jmax);
  }
}
// pnew and pold in the form's field type T (the arithmetic in FP64), two
// consecutive cells per thread through vector loads and stores (the
// buffers are 256-byte aligned and n is even); the same expressions per cell
template <typename T>
struct Vec2;
template <>
struct Vec2<float> {
  typedef float2 type;
};
template <>
struct Vec2<double> {
  typedef double2 type;
};
template <typename T>
__device__ __forceinline__ void pupdate_pair(double p0, double p1, T o0, T o1, T& n0, T& n1, T& d0, T& d1,
                                             int first, int normalise, double norm, double norm_old) {
  if (!normalise) {
    d0 = o0; d1 = o1;
    n0 = TC(p0); n1 = TC(p1);
    return;
  }
  const double a = (double)o0, b = (double)o1;
  d0 = TC(first ? a - norm : (a + norm_old) - norm);
  d1 = TC(first ? b - norm : (b + norm_old) - norm);
  n0 = TC(p0 - norm);
  n1 = TC(p1 - norm);
}
template <typename T>
__global__ void __launch_bounds__(NT) k_pupdate(Params p, const double* __restrict__ pp,
                                                T* __restrict__ pnew, T* __restrict__ pold, int first,
                                                int normalise, const DevScalars* __restrict__ dsc) {
  typedef typename Vec2<T>::type T2;
  const long long n = 2 * (blockIdx.x * (long long)NT + threadIdx.x);
  if (n >= p.nC) return;
  const double norm = normalise ? dsc->norm : 0., norm_old = normalise ? dsc->norm_old : 0.;
  if (n + 1 < p.nC) {
    const double2 pv = *reinterpret_cast<const double2*>(pp + n);
    const T2 ov = *reinterpret_cast<const T2*>(pnew + n);
    T2 nv, dv;
    pupdate_pair<T>(pv.x, pv.y, ov.x, ov.y, nv.x, nv.y, dv.x, dv.y, first, normalise, norm, norm_old);
    *reinterpret_cast<T2*>(pold + n) = dv;
    *reinterpret_cast<T2*>(pnew + n) = nv;
  } else {  // an odd last cell
    T n0, n1, d0, d1;
    pupdate_pair<T>(pp[n], 0., pnew[n], TC(0.), n0, n1, d0, d1, first, normalise, norm, norm_old);
    pold[n] = d0;
    pnew[n] = n0;
  }
}

// ---- reductions ------------------------------------------------------------
// sum over the interior: warp w of the grid takes rows (j,k) w, w + W, ...
// (W warps), its lanes the i of a row, eight loads in flight per lane
// before the adds (fixed grid, fixed order)
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_sum_interior(Params p, const T* __restrict__ a,
                                                              double* __restrict__ partial) {
  const int rows = p.jmax * p.kmax;
  const int W = (int)((gridDim.x * kRedThreads) >> 5);
  const int lane = threadIdx.x & 31;
  double acc[8] = {0., 0., 0., 0., 0., 0., 0., 0.};
  for (int r = (int)((blockIdx.x * kRedThreads + threadIdx.x) >> 5); r < rows; r += W) {
    const T* __restrict__ row = a + idxC(p, 1, 1 + r % p.jmax, 1 + r / p.jmax);
    for (int i0 = lane; i0 < p.imax; i0 += 256) {
      double v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) v[u] = (i0 + 32 * u < p.imax) ? (double)row[i0 + 32 * u] : 0.;
#pragma unroll
      for (int u = 0; u < 8; ++u) acc[u] += v[u];
    }
  }
  const double s = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
  double b = block_sum<double, kRedThreads>(s);
  if (threadIdx.x == 0) partial[blockIdx.x] = b;
}
__global__ void __launch_bounds__(kRedThreads) k_stream_final(Params p, const double* __restrict__ partial, int nblk,
                                                              DevScalars* __restrict__ dsc) {
  double s = 0.;
  for (int b = threadIdx.x; b < nblk; b += kRedThreads) s += partial[b];
  s = block_sum<double, kRedThreads>(s);
  if (threadIdx.x == 0) dsc->v_bulk = s / (double)((long long)p.imax * p.jmax * p.kmax);
}

// chkdiv: sum of div and max|div| with its first column-major location
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_chkdiv(Params p, const T* __restrict__ u, const T* __restrict__ v,
                                                        const T* __restrict__ w,
                                                        double* __restrict__ part_sum, double* __restrict__ part_max,
                                                        long long* __restrict__ part_loc) {
  double s = 0., m = 0.;
  long long loc = -1;
  for (int q = blockIdx.x * kRedThreads + threadIdx.x; q < (int)p.nI; q += gridDim.x * kRedThreads) {
    int i, j, k;
    decodeI(p, q, i, j, k);
    const long long c = idxC(p, i, j, k);
    const double wc = w[c], wm = w[c - (long long)p.nCx * p.nCy], vc = v[c], vm = v[c - p.nCx];
    const double uc = u[c], um = u[c - 1];
    double div = ((wc - wm) * p.dzi + (vc - vm) * p.dyi) + (uc - um) * p.dxi;
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
template <typename T>
__global__ void __launch_bounds__(NT) k_chkdt(Params p, const T* __restrict__ u, const T* __restrict__ v,
                                              const T* __restrict__ w, DevScalars* __restrict__ dsc) {
  double a = 0., b = 0., c = 0.;
  int i, j, k;
  const I3 hi = cC1(p);
  if (cell3(kI0, hi.v, i, j, k)) {
    const long long cc = idxC(p, i, j, k);
    a = fabs(((double)u[cc] + (double)u[cc - 1]) / 2.);
    b = fabs(((double)v[cc] + (double)v[cc - p.nCx]) / 2.);
    c = fabs(((double)w[cc] + (double)w[cc - (long long)p.nCx * p.nCy]) / 2.);
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
template <typename T>
__global__ void __launch_bounds__(NT) k_maxvel(Params p, const T* __restrict__ ucc, const T* __restrict__ vcc,
                                               const T* __restrict__ wcc, DevScalars* __restrict__ dsc) {
  const long long q = blockIdx.x * (long long)NT + threadIdx.x;
  double m = 0.;
  if (q < p.nI) {
    const double a = ucc[q], b = vcc[q], cc = wcc[q];
    m = sqrt((a * a + b * b) + cc * cc);
  }
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

#undef TC
}  // namespace

// ================================================================ launchers
template <typename T>
T* fp(double* q) { return reinterpret_cast<T*>(q); }

void launch_ab2(Ctx& c) {
  Scope sc_(c.prof, c.s, "ab2", 1);
  MomArgs a = mom_args(c);
  const int o = c.hist ^ 1;
  if (c.P.f32) ab2_launch_f32(c, a, o);     // k_ab2_f32.cu
  else if (!ab2_tma_launch(c, a, o)) ab2_launch<double>(c, a, o);  // k_ab2_tma.cu when chosen, else the ring
  launch_ywalls_uvw(c, c.dudt, c.dvdt, c.dwdt);  // the y walls of bounduvw(dudt,dvdt,dwdt)
  c.hist = o;
}
void launch_mom_main(Ctx& c, double* du, double* dv, double* dw) {
  Scope sc_(c.prof, c.s, "mom_main", 1);
  MomArgs a = mom_args(c);
  if (c.P.f32)
    k_mom_main<float><<<gridI(c.P), kBlock, 0, c.s>>>(c.P, a, fp<float>(du), fp<float>(dv), fp<float>(dw));
  else
    k_mom_main<double><<<gridI(c.P), kBlock, 0, c.s>>>(c.P, a, du, dv, dw);
}
void launch_fillps(Ctx& c, int add_pjump) {
  Scope sc_(c.prof, c.s, "fillps", 1);
  if (c.P.f32)
    k_fillps<float><<<gridI(c.P), kBlock, 0, c.s>>>(c.P, fp<float>(c.dudt), fp<float>(c.dvdt), fp<float>(c.dwdt),
                                                     c.pjump, add_pjump, c.p);
  else
    k_fillps<double><<<gridI(c.P), kBlock, 0, c.s>>>(c.P, c.dudt, c.dvdt, c.dwdt, c.pjump, add_pjump, c.p);
}
void launch_add_pjump(Ctx& c) {
  Scope sc_(c.prof, c.s, "add_pjump", 1); k_add<<<nblocks(c.P.nC), NT, 0, c.s>>>(c.P, c.p, c.pjump); }
void launch_correc(Ctx& c, int fused_bc) {
  Scope sc_(c.prof, c.s, "correc", 1);
  CorrArgs a = corr_args(c);
  // the fused form: one thread per interior cell writing the halo and wall
  // images (ICLS_CORREC=shapec: one thread per shape-C cell)
  if (fused_bc && !c.correc_shapec) {
    const bool rp = c.P.rho0_pow2 != 0;
    if (c.P.f32) {
      if (rp) k_correc_own<float, 1><<<gridI(c.P), kBlock, 0, c.s>>>(c.P, a);
      else k_correc_own<float, 0><<<gridI(c.P), kBlock, 0, c.s>>>(c.P, a);
    } else {
      if (rp) k_correc_own<double, 1><<<gridI(c.P), kBlock, 0, c.s>>>(c.P, a);
      else k_correc_own<double, 0><<<gridI(c.P), kBlock, 0, c.s>>>(c.P, a);
    }
    return;
  }
  if (c.P.f32) {
    if (fused_bc) k_correc_fused<float><<<gridC(c.P), kBlock, 0, c.s>>>(c.P, a);
    else k_correc_interior<float><<<gridI(c.P), kBlock, 0, c.s>>>(c.P, a);
  } else {
    if (fused_bc) k_correc_fused<double><<<gridC(c.P), kBlock, 0, c.s>>>(c.P, a);
    else k_correc_interior<double><<<gridI(c.P), kBlock, 0, c.s>>>(c.P, a);
  }
}
void launch_bounduvw(Ctx& c, double* u, double* v, double* w) {
  Scope sc_(c.prof, c.s, "bounduvw", 1);
  if (c.P.f32) k_bounduvw<float><<<gridC(c.P), kBlock, 0, c.s>>>(c.P, fp<float>(u), fp<float>(v), fp<float>(w));
  else k_bounduvw<double><<<gridC(c.P), kBlock, 0, c.s>>>(c.P, u, v, w);
  launch_ywalls_uvw(c, u, v, w);
}
inline dim3 grid_ik(const Params& p) { return dim3((unsigned)((p.imax + NT - 1) / NT), (unsigned)p.kmax, 1); }
void launch_boundp(Ctx& c, double* pp, bool tfield) {
  Scope sc_(c.prof, c.s, "boundp", 1);
  if (tfield && c.P.f32) {
    k_boundp<float><<<gridC(c.P), kBlock, 0, c.s>>>(c.P, fp<float>(pp));
    if (c.P.bcy != ICLS_BCY_PERIODIC) k_ywalls_p<float><<<grid_ik(c.P), NT, 0, c.s>>>(c.P, fp<float>(pp));
    return;
  }
  k_boundp<double><<<gridC(c.P), kBlock, 0, c.s>>>(c.P, pp);
  launch_ywalls_p(c, pp);
}
void launch_ywalls_uvw(Ctx& c, double* u, double* v, double* w) {
  if (c.P.bcy == ICLS_BCY_PERIODIC) return;
  if (c.P.f32)
    k_ywalls_uvw<float><<<grid_ik(c.P), NT, 0, c.s>>>(c.P, fp<float>(u), fp<float>(v), fp<float>(w), c.vin);
  else
    k_ywalls_uvw<double><<<grid_ik(c.P), NT, 0, c.s>>>(c.P, u, v, w, c.vin);
}
void launch_ywalls_p(Ctx& c, double* pp) {
  if (c.P.bcy == ICLS_BCY_PERIODIC) return;
  k_ywalls_p<double><<<grid_ik(c.P), NT, 0, c.s>>>(c.P, pp);
}
void launch_gather_plane_x(Ctx& c, const double* d, bool f32, long long nx, long long ny, long long ioff, int n1,
                           int n2, double* dst) {
  const unsigned g = nblocks((long long)n1 * n2);
  if (f32) k_gather_plane_x<float><<<g, NT, 0, c.s>>>(reinterpret_cast<const float*>(d), nx, nx * ny, ioff, n1, n2, dst);
  else k_gather_plane_x<double><<<g, NT, 0, c.s>>>(d, nx, nx * ny, ioff, n1, n2, dst);
}
void launch_nan_probe(Ctx& c) {
  if (c.P.f32) k_nan_probe<float><<<1, 1, 0, c.s>>>(c.P, fp<float>(c.v), c.dsc);
  else k_nan_probe<double><<<1, 1, 0, c.s>>>(c.P, c.v, c.dsc);
}
void launch_average_vel(Ctx& c) {
  Scope sc_(c.prof, c.s, "average_vel", 1);
  if (c.P.f32)
    k_average_vel<float><<<gridI(c.P), kBlock, 0, c.s>>>(c.P, fp<float>(c.u), fp<float>(c.v), fp<float>(c.w),
                                                          fp<float>(c.ucc), fp<float>(c.vcc), fp<float>(c.wcc));
  else
    k_average_vel<double><<<gridI(c.P), kBlock, 0, c.s>>>(c.P, c.u, c.v, c.w, c.ucc, c.vcc, c.wcc);
}
void launch_pressure_update(Ctx& c, int first) {
  Scope sc_(c.prof, c.s, "pressure_update", 2);
  // the plane-1 normalisation runs for BC_in_y Periodic and Walls only
  // (main.f90:169-185); otherwise pold = pnew, pnew = p
  const int norm = c.P.bcy == ICLS_BCY_PERIODIC || c.P.bcy == ICLS_BCY_WALLS;
  if (norm) k_plane_norm<<<1, kNormThreads, 0, c.s>>>(c.P, c.p, c.dsc);
  if (c.P.f32)
    k_pupdate<float><<<nblocks((c.P.nC + 1) / 2), NT, 0, c.s>>>(c.P, c.p, fp<float>(c.pnew), fp<float>(c.pold), first, norm,
                                                       c.dsc);
  else
    k_pupdate<double><<<nblocks((c.P.nC + 1) / 2), NT, 0, c.s>>>(c.P, c.p, c.pnew, c.pold, first, norm, c.dsc);
}
void launch_stream_vel(Ctx& c) {
  Scope sc_(c.prof, c.s, "stream_vel", 2);
  if (c.P.f32) k_sum_interior<float><<<kRedBlocks, kRedThreads, 0, c.s>>>(c.P, fp<float>(c.v), c.partials);
  else k_sum_interior<double><<<kRedBlocks, kRedThreads, 0, c.s>>>(c.P, c.v, c.partials);
  k_stream_final<<<1, kRedThreads, 0, c.s>>>(c.P, c.partials, kRedBlocks, c.dsc);
}
void launch_chkdiv(Ctx& c) {
  Scope sc_(c.prof, c.s, "chkdiv", 2);
  double* ps = c.partials;
  double* pm = c.partials + kRedBlocks;
  if (c.P.f32)
    k_chkdiv<float><<<kRedBlocks, kRedThreads, 0, c.s>>>(c.P, fp<float>(c.u), fp<float>(c.v), fp<float>(c.w), ps, pm,
                                                          c.lpartials);
  else
    k_chkdiv<double><<<kRedBlocks, kRedThreads, 0, c.s>>>(c.P, c.u, c.v, c.w, ps, pm, c.lpartials);
  k_chkdiv_final<<<1, 32, 0, c.s>>>(ps, pm, c.lpartials, kRedBlocks, c.dsc);
}
void launch_chkdt(Ctx& c) {
  Scope sc_(c.prof, c.s, "chkdt", 1);
  cudaMemsetAsync(&c.dsc->umax, 0, 3 * sizeof(double), c.s);
  if (c.P.f32) k_chkdt<float><<<gridC(c.P), kBlock, 0, c.s>>>(c.P, fp<float>(c.u), fp<float>(c.v), fp<float>(c.w), c.dsc);
  else k_chkdt<double><<<gridC(c.P), kBlock, 0, c.s>>>(c.P, c.u, c.v, c.w, c.dsc);
}
void launch_maxvel(Ctx& c) {
  Scope sc_(c.prof, c.s, "maxvel", 1);
  cudaMemsetAsync(&c.dsc->velmax, 0, sizeof(double), c.s);
  if (c.P.f32)
    k_maxvel<float><<<nblocks(c.P.nI), NT, 0, c.s>>>(c.P, fp<float>(c.ucc), fp<float>(c.vcc), fp<float>(c.wcc), c.dsc);
  else
    k_maxvel<double><<<nblocks(c.P.nI), NT, 0, c.s>>>(c.P, c.ucc, c.vcc, c.wcc, c.dsc);
}

}  // namespace icls
