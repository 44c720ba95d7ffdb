// ab2.cuh — the AB2 predictor (ab2.f90:21-138 with mom_main's RHS,
// mom.f90:13-301) as a kernel template.  k_navier.cu instantiates it for the
// plain FP64 path, compiled with -fmad=false so every expression keeps the
// reference's evaluation order; k_ab2_f32.cu instantiates the FP32 form,
// compiled with multiply-add contraction (that form is held to tolerances,
// not to the reference's rounding).  The device code sits in each file's
// own anonymous namespace.
#pragma once

#include <type_traits>

#include "batch.cuh"

namespace icls {

// the fields of the predictor, type-erased: all but rho_avr hold the form's
// field type (FP64, or FP32 in the precision form)
struct MomArgs {
  const double *u, *v, *w, *miu, *rho_u, *rho_v, *rho_w;
  const double *duold, *dvold, *dwold;
  const double *pnew, *pold, *px, *py, *pz, *pxold, *pyold, *pzold;
  const double* rho_avr;
};

namespace {

// T is the form's field type (double, or float in the precision form);
// TC(x) is the constant x in T
#define TC(x) static_cast<T>(x)

// ---- RHS of mom_main for one component ----------------------------------
// U(di,dj,dk) returns u at (i+di, j+dj, k+dk), likewise V, W and M (miu):
// the same expressions serve the shared-memory march of k_ab2 and the
// global-memory k_mom_main.  T is the form's field type; TC(x) the
// constant x in T.
template <typename T, int PW = -1, class FU, class FV, class FW, class FM>
__device__ __forceinline__ T rhs_u(const Params& p, const FU& U, const FV& V, const FW& W, const FM& M,
                                        T rho_u, T rho_avr) {
  T RCu = TC(0.);
  if (!p.TwoD) {
    T uuip = TC(0.25) * (U(1, 0, 0) + U(0, 0, 0)) * (U(1, 0, 0) + U(0, 0, 0));
    T uuim = TC(0.25) * (U(-1, 0, 0) + U(0, 0, 0)) * (U(-1, 0, 0) + U(0, 0, 0));
    T uvjp = TC(0.25) * (U(0, 1, 0) + U(0, 0, 0)) * (V(1, 0, 0) + V(0, 0, 0));
    T uvjm = TC(0.25) * (U(0, -1, 0) + U(0, 0, 0)) * (V(1, -1, 0) + V(0, -1, 0));
    T uwkp = TC(0.25) * (U(0, 0, 1) + U(0, 0, 0)) * (W(1, 0, 0) + W(0, 0, 0));
    T uwkm = TC(0.25) * (U(0, 0, -1) + U(0, 0, 0)) * (W(1, 0, -1) + W(0, 0, -1));
    RCu = (divx<PW>(p, (-uuip + uuim)) + divy<PW>(p, (-uvjp + uvjm))) + divz<PW>(p, (-uwkp + uwkm));
  }
  T RDu = TC(0.);
  if (!p.TwoD) {
    T dudxp = divx<PW>(p, (U(1, 0, 0) - U(0, 0, 0)));
    T dudxm = divx<PW>(p, (U(0, 0, 0) - U(-1, 0, 0)));
    T dudyp = divy<PW>(p, (U(0, 1, 0) - U(0, 0, 0)));
    T dudym = divy<PW>(p, (U(0, 0, 0) - U(0, -1, 0)));
    T dvdxp = divx<PW>(p, (V(1, 0, 0) - V(0, 0, 0)));
    T dvdxm = divx<PW>(p, (V(1, -1, 0) - V(0, -1, 0)));
    T dudzp = divz<PW>(p, (U(0, 0, 1) - U(0, 0, 0)));
    T dudzm = divz<PW>(p, (U(0, 0, 0) - U(0, 0, -1)));
    T dwdxp = divx<PW>(p, (W(1, 0, 0) - W(0, 0, 0)));
    T dwdxm = divx<PW>(p, (W(1, 0, -1) - W(0, 0, -1)));
    T ma1 = TC(0.25) * (((M(0, 0, 0) + M(0, -1, 0)) + M(1, -1, 0)) + M(1, 0, 0));
    T ma2 = TC(0.25) * (((M(0, 0, 0) + M(0, 1, 0)) + M(1, 1, 0)) + M(1, 0, 0));
    T ma3 = TC(0.25) * (((M(0, 0, 0) + M(0, 0, -1)) + M(1, 0, -1)) + M(1, 0, 0));
    T ma4 = TC(0.25) * (((M(0, 0, 0) + M(0, 0, 1)) + M(1, 0, 1)) + M(1, 0, 0));
    T RD1 = divx<PW>(p, TC(2.) * (dudxp * M(1, 0, 0) - dudxm * M(0, 0, 0)));
    T RD2 = divy<PW>(p, (dudyp * ma2 - dudym * ma1));
    T RD3 = divy<PW>(p, (dvdxp * ma2 - dvdxm * ma1));
    T RD4 = divz<PW>(p, (dudzp * ma4 - dudzm * ma3));
    T RD5 = divz<PW>(p, (dwdxp * ma4 - dwdxm * ma3));
    RDu = ((((RD1 + RD2) + RD3) + RD4) + RD5) / rho_u;
  }
  // buoyancy iFr (1 - rho_avr/rho) g: skipped (with its divide) where iFr or
  // this component of g is zero; the term is then an exact +-0, which
  // changes the sum at most in the sign of an exactly zero result
  if (p.TwoD || p.iFr == 0. || p.g1 == 0.) return RCu + RDu * TC(p.visc);
  T RGu = TC(p.iFr) * (TC(1.) - rho_avr / rho_u) * TC(p.g1);
  return (RCu + RDu * TC(p.visc)) + RGu;
}

template <typename T, int PW = -1, class FU, class FV, class FW, class FM>
__device__ __forceinline__ T rhs_v(const Params& p, const FU& U, const FV& V, const FW& W, const FM& M,
                                        T rv, T rho_avr) {
  T uvip = TC(0.25) * (U(0, 0, 0) + U(0, 1, 0)) * (V(0, 0, 0) + V(1, 0, 0));
  T uvim = TC(0.25) * (U(-1, 0, 0) + U(-1, 1, 0)) * (V(0, 0, 0) + V(-1, 0, 0));
  T vvjp = TC(0.25) * (V(0, 0, 0) + V(0, 1, 0)) * (V(0, 0, 0) + V(0, 1, 0));
  T vvjm = TC(0.25) * (V(0, 0, 0) + V(0, -1, 0)) * (V(0, 0, 0) + V(0, -1, 0));
  T wvkp = TC(0.25) * (W(0, 0, 0) + W(0, 1, 0)) * (V(0, 0, 1) + V(0, 0, 0));
  T wvkm = TC(0.25) * (W(0, 0, -1) + W(0, 1, -1)) * (V(0, 0, -1) + V(0, 0, 0));
  T RCv = (divx<PW>(p, (-uvip + uvim)) + divy<PW>(p, (-vvjp + vvjm))) + divz<PW>(p, (-wvkp + wvkm));
  T dvdxp = divx<PW>(p, (V(1, 0, 0) - V(0, 0, 0)));
  T dvdxm = divx<PW>(p, (V(0, 0, 0) - V(-1, 0, 0)));
  T dudyp = divy<PW>(p, (U(0, 1, 0) - U(0, 0, 0)));
  T dudym = divy<PW>(p, (U(-1, 1, 0) - U(-1, 0, 0)));
  T dvdyp = divy<PW>(p, (V(0, 1, 0) - V(0, 0, 0)));
  T dvdym = divy<PW>(p, (V(0, 0, 0) - V(0, -1, 0)));
  T dvdzp = divz<PW>(p, (V(0, 0, 1) - V(0, 0, 0)));
  T dvdzm = divz<PW>(p, (V(0, 0, 0) - V(0, 0, -1)));
  T dwdyp = divy<PW>(p, (W(0, 1, 0) - W(0, 0, 0)));
  T dwdym = divy<PW>(p, (W(0, 1, -1) - W(0, 0, -1)));
  T ma2 = TC(0.25) * (((M(0, 0, 0) + M(0, 1, 0)) + M(1, 1, 0)) + M(1, 0, 0));
  T ma5 = TC(0.25) * (((M(0, 0, 0) + M(0, 1, 0)) + M(-1, 1, 0)) + M(-1, 0, 0));
  T ma6 = TC(0.25) * (((M(0, 0, 0) + M(0, 0, -1)) + M(0, 1, -1)) + M(0, 1, 0));
  T ma7 = TC(0.25) * (((M(0, 0, 0) + M(0, 0, 1)) + M(0, 1, 1)) + M(0, 1, 0));
  T RD1 = divx<PW>(p, (dvdxp * ma2 - dvdxm * ma5));
  T RD2 = divx<PW>(p, (dudyp * ma2 - dudym * ma5));
  T RD3 = divy<PW>(p, TC(2.) * (dvdyp * M(0, 1, 0) - dvdym * M(0, 0, 0)));
  T RD4 = divz<PW>(p, (dvdzp * ma7 - dvdzm * ma6));
  T RD5 = divz<PW>(p, (dwdyp * ma7 - dwdym * ma6));
  T RDv = ((((RD1 + RD2) + RD3) + RD4) + RD5) / rv;
  if (p.iFr == 0. || p.g2 == 0.) return RCv + RDv * TC(p.visc);  // buoyancy as in rhs_u
  T RGv = TC(p.iFr) * (TC(1.) - rho_avr / rv) * TC(p.g2);
  return (RCv + RDv * TC(p.visc)) + RGv;
}

template <typename T, int PW = -1, class FU, class FV, class FW, class FM>
__device__ __forceinline__ T rhs_w(const Params& p, const FU& U, const FV& V, const FW& W, const FM& M,
                                        T rw, T rho_avr) {
  T uwip = TC(0.25) * (W(0, 0, 0) + W(1, 0, 0)) * (U(0, 0, 0) + U(0, 0, 1));
  T uwim = TC(0.25) * (W(0, 0, 0) + W(-1, 0, 0)) * (U(-1, 0, 0) + U(-1, 0, 1));
  T vwjp = TC(0.25) * (W(0, 0, 0) + W(0, 1, 0)) * (V(0, 0, 0) + V(0, 0, 1));
  T vwjm = TC(0.25) * (W(0, 0, 0) + W(0, -1, 0)) * (V(0, -1, 0) + V(0, -1, 1));
  T wwkp = TC(0.25) * (W(0, 0, 0) + W(0, 0, 1)) * (W(0, 0, 0) + W(0, 0, 1));
  T wwkm = TC(0.25) * (W(0, 0, 0) + W(0, 0, -1)) * (W(0, 0, 0) + W(0, 0, -1));
  T RCw = (divx<PW>(p, (-uwip + uwim)) + divy<PW>(p, (-vwjp + vwjm))) + divz<PW>(p, (-wwkp + wwkm));
  T dwdxp = divx<PW>(p, (W(1, 0, 0) - W(0, 0, 0)));
  T dwdxm = divx<PW>(p, (W(0, 0, 0) - W(-1, 0, 0)));
  T dudzp = divz<PW>(p, (U(0, 0, 1) - U(0, 0, 0)));
  T dudzm = divz<PW>(p, (U(-1, 0, 1) - U(-1, 0, 0)));
  T dwdyp = divy<PW>(p, (W(0, 1, 0) - W(0, 0, 0)));
  T dwdym = divy<PW>(p, (W(0, 0, 0) - W(0, -1, 0)));
  T dvdzp = divz<PW>(p, (V(0, 0, 1) - V(0, 0, 0)));
  T dvdzm = divz<PW>(p, (V(0, -1, 1) - V(0, -1, 0)));
  T dwdzp = divz<PW>(p, (W(0, 0, 1) - W(0, 0, 0)));
  T dwdzm = divz<PW>(p, (W(0, 0, 0) - W(0, 0, -1)));
  T ma4 = TC(0.25) * (((M(0, 0, 0) + M(0, 0, 1)) + M(1, 0, 1)) + M(1, 0, 0));
  T ma8 = TC(0.25) * (((M(0, 0, 0) + M(0, 0, 1)) + M(-1, 0, 1)) + M(-1, 0, 0));
  T ma7 = TC(0.25) * (((M(0, 0, 0) + M(0, 0, 1)) + M(0, 1, 1)) + M(0, 1, 0));
  T ma9 = TC(0.25) * (((M(0, 0, 0) + M(0, 0, 1)) + M(0, -1, 1)) + M(0, -1, 0));
  T RD1 = divx<PW>(p, (dwdxp * ma4 - dwdxm * ma8));
  T RD2 = divx<PW>(p, (dudzp * ma4 - dudzm * ma8));
  T RD3 = divy<PW>(p, (dwdyp * ma7 - dwdym * ma9));
  T RD4 = divy<PW>(p, (dvdzp * ma7 - dvdzm * ma9));
  T RD5 = divz<PW>(p, TC(2.) * (dwdzp * M(0, 0, 1) - dwdzm * M(0, 0, 0)));
  T RDw = ((((RD1 + RD2) + RD3) + RD4) + RD5) / rw;
  if (p.iFr == 0. || p.g3 == 0.) return RCw + RDw * TC(p.visc);  // buoyancy as in rhs_u
  T RGw = TC(p.iFr) * (TC(1.) - rho_avr / rw) * TC(p.g3);
  return (RCw + RDw * TC(p.visc)) + RGw;
}

// ---- the ab2 update of one component (ab2.f90:51-61, 79-129) -------------
// u0 = u at the cell, R = its mom_main RHS, rold the previous RHS, rf its
// face density, dhi the 1/dx of the component's axis; the pressure-split
// term is formed in FP64 (the pressures are FP64 fields) from: ph_p / ph_0 the
// extrapolated pressures 2 pnew - pold at the + neighbour and the cell,
// pjh the extrapolated pressure gradient 2 p_x - p_x,old
// PT is the pressure term's arithmetic: FP64 in the plain path; in the FP32
// form, whose pressures are stored in FP32, the term is formed in FP32 too
// (it is part of the momentum predictor, which that form computes in FP32)
template <typename T, typename PT>
__device__ __forceinline__ T ab2_update_v(const Params& p, T u0, T R, T rold, T rf, PT ph_p, PT ph_0, PT pjh,
                                          double dhi) {
  T d = u0 + TC(p.dt) * (TC(1.5) * R - TC(0.5) * rold);
  const PT dn = -((PT(1.) / (PT)rf - (PT)p.rrho0) * (PT)dhi * ((ph_p - pjh) - ph_0));
  return d + TC((PT)p.dt * dn);
}

// element copies global -> shared that complete asynchronously (waited for
// with cp_async_wait_all before the block's barrier)
template <typename T>
__device__ __forceinline__ void cp_async_el(T* dst, const T* src) {
  const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
  if (sizeof(T) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
// two consecutive elements (8 bytes in FP32, 16 in FP64); both addresses
// aligned to the pair's size
template <typename T>
__device__ __forceinline__ void cp_async_pair(T* dst, const T* src) {
  const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
  if (sizeof(T) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// ab2 over shape C with bounduvw(dudt,dvdt,dwdt) (bound.f90:36-75) in-kernel.
// A block is a 32 x 8 column tile marching up a chunk of interior rows.
// u, v, w, miu (tile plus one halo column each side) and pnew, pold (tile
// plus the + neighbours in x and y) pass through a four-plane shared-memory
// ring filled by asynchronous copies: at row k the block issues row k+1's
// planes and this cell's own operands together, then waits once, so one
// memory latency is exposed per row and the ring needs one barrier per row
// (the slot a row's copies fill is not one any thread can still be reading).
// A thread writes its column's periodic halo images and, at k = 1 and
// k = kmax, the wall rows k = 0 and k = k1.  Every plane row starts at
// column i0 - 1 (even).
constexpr int MX = 32, MY = 8, MSX = MX + 2, MSY = MY + 2, MPY = MY + 1, MRING = 4;
template <typename T>
constexpr int ab2_smem() {
  return (int)(4 * MRING * MSY * MSX * sizeof(T) + 2 * MRING * MPY * MSX * sizeof(T));
}
template <typename T, int PW, int MB>
__global__ void __launch_bounds__(MX * MY, MB)
    k_ab2(Params p, MomArgs a, T* __restrict__ dudt, T* __restrict__ dvdt, T* __restrict__ dwdt,
          T* __restrict__ duold_out, T* __restrict__ dvold_out, T* __restrict__ dwold_out, int kc, int nch) {
  extern __shared__ __align__(16) unsigned char ab2_dyn[];
  typedef T Plane[MSY][MSX];
  typedef T PPlane[MPY][MSX];  // pnew, pold (columns i0-1.., rows j0..) in the form's field type
  Plane* ring = reinterpret_cast<Plane*>(ab2_dyn);  // [field * MRING + slot]
  PPlane* pring = reinterpret_cast<PPlane*>(ab2_dyn + 4 * MRING * sizeof(Plane));
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + MX * ty;
  const int i0 = 1 + MX * (int)blockIdx.x, j0 = 1 + MY * (int)blockIdx.y;
  const int ch = blockIdx.z;
  const int ka = 1 + ch * kc, kb = (ch == nch - 1) ? p.kmax : ka + kc - 1;
  const int i = i0 + tx, j = j0 + ty;
  const bool ok = i <= p.imax && j <= p.jmax;
  const T* __restrict__ F[4] = {cT<T>(a.u), cT<T>(a.v), cT<T>(a.w), cT<T>(a.miu)};
  const T* __restrict__ rhu = cT<T>(a.rho_u);
  const T* __restrict__ rhv = cT<T>(a.rho_v);
  const T* __restrict__ rhw = cT<T>(a.rho_w);
  const T* __restrict__ hu = cT<T>(a.duold);
  const T* __restrict__ hv = cT<T>(a.dvold);
  const T* __restrict__ hw = cT<T>(a.dwold);
  // FP64: imax is even (every FFT length validate() admits is), so the rows
  // of shape C have an even length and each plane row's first element
  // (column i0-1, even) sits at an even index: 16-byte pair copies are
  // aligned, and halve the copy instructions (1.37 -> 1.30 ms at 256^3).
  // FP32 keeps one 4-byte copy per element: at its 64-register budget the
  // pair loop spilled and measured slower (0.77 -> 0.84 ms).
  // This thread's copy slots, the same for every row: slot r is element
  // tid + r MX MY of a plane (a pair of elements in FP64), at plane offset
  // gi + nCx gj of storage row 0 (row kk is kk nCx nCy further), -1 where
  // the element lies outside the grid.  NS slots cover a plane.
  constexpr int EPC = sizeof(T) == 8 ? 2 : 1;  // elements per copy
  constexpr int RW = MSX / EPC;                // copies per plane row
  constexpr int NS = (RW * MSY + MX * MY - 1) / (MX * MY);
  int ro[NS], po[NS];
#pragma unroll
  for (int r = 0; r < NS; ++r) {
    const int e = tid + r * MX * MY;
    const int sy = e / RW, sx = EPC * (e - sy * RW);
    const int gi = i0 - 1 + sx;
    // gi even in FP64: gi + 1 <= imax + 1
    const bool xin = sizeof(T) == 8 ? gi <= p.imax : gi <= p.imax + 1;
    ro[r] = (e < RW * MSY && xin && j0 - 1 + sy <= p.jmax + 1) ? gi + p.nCx * (j0 - 1 + sy) : -1;
    // pnew, pold rows start at j0; their column i0-1 is not read (FP32
    // skips it, FP64 copies it with its pair)
    po[r] = (e < RW * MPY && xin && j0 + sy <= p.jmax + 1 && (sizeof(T) == 8 || sx > 0)) ? gi + p.nCx * (j0 + sy)
                                                                                        : -1;
  }
  const long long psz = (long long)p.nCx * p.nCy;
  auto issue_plane = [&](int kk) {
    const int s = kk & (MRING - 1);
    const long long kb = (long long)kk * psz;
#pragma unroll
    for (int r = 0; r < NS; ++r) {
      const int e = EPC * (tid + r * MX * MY);  // element offset in the plane
      if (ro[r] >= 0) {
        const long long g = kb + ro[r];
#pragma unroll
        for (int f = 0; f < 4; ++f) {
          T* dst = &ring[f * MRING + s][0][0] + e;
          if constexpr (sizeof(T) == 8) cp_async_pair(dst, F[f] + g);
          else cp_async_el(dst, F[f] + g);
        }
      }
      if (po[r] >= 0) {
        const long long g = kb + po[r];
        T* d0 = &pring[s][0][0] + e;
        T* d1 = &pring[MRING + s][0][0] + e;
        if constexpr (sizeof(T) == 8) {
          cp_async_pair(d0, cT<T>(a.pnew) + g);
          cp_async_pair(d1, cT<T>(a.pold) + g);
        } else {
          cp_async_el(d0, cT<T>(a.pnew) + g);
          cp_async_el(d1, cT<T>(a.pold) + g);
        }
      }
    }
  };
  issue_plane(ka - 1);
  issue_plane(ka);
  const T rho_avr = TC(*a.rho_avr);
  T dw_km1 = TC(0.);
  for (int k = ka; k <= kb; ++k) {
    // this cell's own operands, in flight together with row k+1's planes
    T ru = TC(1.), rv = TC(1.), rw = TC(1.), ou = TC(0.), ov = TC(0.), ow = TC(0.);
    typedef typename std::conditional<sizeof(T) == 8, double, float>::type PT;
    PT qx = 0., qxo = 0., qy = 0., qyo = 0., qz = 0., qzo = 0.;
    const long long c = idxC(p, i, j, k), q = idxI(p, i, j, k);
    if (ok) {
      ru = rhu[q]; rv = rhv[q]; rw = rhw[q];
      ou = hu[q]; ov = hv[q]; ow = hw[q];
      qx = (PT)cT<T>(a.px)[c]; qxo = (PT)cT<T>(a.pxold)[c];
      qy = (PT)cT<T>(a.py)[c]; qyo = (PT)cT<T>(a.pyold)[c];
      qz = (PT)cT<T>(a.pz)[c]; qzo = (PT)cT<T>(a.pzold)[c];
    }
    issue_plane(k + 1);
    cp_async_wait_all();
    __syncthreads();
    if (ok) {
      const int s_m = (k - 1) & (MRING - 1), s_0 = k & (MRING - 1), s_p = (k + 1) & (MRING - 1);
      auto sl = [&](int dk) { return dk < 0 ? s_m : (dk > 0 ? s_p : s_0); };
      auto U = [&](int di, int dj, int dk) { return ring[0 * MRING + sl(dk)][ty + 1 + dj][tx + 1 + di]; };
      auto V = [&](int di, int dj, int dk) { return ring[1 * MRING + sl(dk)][ty + 1 + dj][tx + 1 + di]; };
      auto W = [&](int di, int dj, int dk) { return ring[2 * MRING + sl(dk)][ty + 1 + dj][tx + 1 + di]; };
      auto M = [&](int di, int dj, int dk) { return ring[3 * MRING + sl(dk)][ty + 1 + dj][tx + 1 + di]; };
      auto PH = [&](int di, int dj, int dk) {
        return PT(2.) * (PT)pring[sl(dk)][ty + dj][tx + 1 + di] - (PT)pring[MRING + sl(dk)][ty + dj][tx + 1 + di];
      };
      const PT ph0 = PH(0, 0, 0);
      const T Ru = rhs_u<T, PW>(p, U, V, W, M, ru, rho_avr);
      const T Rv = rhs_v<T, PW>(p, U, V, W, M, rv, rho_avr);
      const T Rw = rhs_w<T, PW>(p, U, V, W, M, rw, rho_avr);
      const T du = ab2_update_v<T, PT>(p, U(0, 0, 0), Ru, ou, ru, PH(1, 0, 0), ph0, PT(2.) * qx - qxo, p.dxi);
      T dv = ab2_update_v<T, PT>(p, V(0, 0, 0), Rv, ov, rv, PH(0, 1, 0), ph0, PT(2.) * qy - qyo, p.dyi);
      if (p.forceytot != 0.) dv = dv - TC(p.forceytot * p.dt) / rv;  // constPoi driving (exact zero otherwise)
      T dw = ab2_update_v<T, PT>(p, W(0, 0, 0), Rw, ow, rw, PH(0, 0, 1), ph0, PT(2.) * qz - qzo, p.dzi);
      duold_out[q] = Ru;
      dvold_out[q] = Rv;
      dwold_out[q] = Rw;
      if (k == p.kmax - 1) dw_km1 = dw;
      if (k == p.kmax) dw = TC(0.);
      putC(p, dudt, i, j, k, du);
      putC(p, dvdt, i, j, k, dv);
      putC(p, dwdt, i, j, k, dw);
      if (k == 1) {
        putC(p, dudt, i, j, 0, -du);
        putC(p, dvdt, i, j, 0, TC(2. * p.v_lower) - dv);
        putC(p, dwdt, i, j, 0, TC(0.));
      }
      if (k == p.kmax) {
        putC(p, dudt, i, j, p.k1, -du);
        putC(p, dvdt, i, j, p.k1, TC(2. * p.v_upper) - dv);
        putC(p, dwdt, i, j, p.k1, dw_km1);
      }
    }
  }
}

template <typename T>
T* ab2_ptr(double* q) { return reinterpret_cast<T*>(q); }

template <typename T, int PW, int MB>
void ab2_launch_pw(Ctx& c, const MomArgs& a, int o) {
  // rows per block: 32 for the FP32 form (four blocks per SM, shorter
  // ring prologues), 16 for FP64 (three blocks per SM, more blocks per wave)
  const int kc = sizeof(T) == 8 ? 16 : 32, nch = std::max(1, c.P.kmax / kc);
  const dim3 grid((unsigned)((c.P.imax + MX - 1) / MX), (unsigned)((c.P.jmax + MY - 1) / MY), (unsigned)nch);
  static unsigned attr = 0;  // devices this instance's shared-memory limit is raised on
  int dev = 0;
  cudaGetDevice(&dev);
  if (!(attr & (1u << (dev & 31)))) {
    cudaFuncSetAttribute(k_ab2<T, PW, MB>, cudaFuncAttributeMaxDynamicSharedMemorySize, ab2_smem<T>());
    attr |= 1u << (dev & 31);
  }
  k_ab2<T, PW, MB><<<grid, dim3(MX, MY, 1), ab2_smem<T>(), c.s>>>(
      c.P, a, ab2_ptr<T>(c.dudt), ab2_ptr<T>(c.dvdt), ab2_ptr<T>(c.dwdt), ab2_ptr<T>(c.duold[o]),
      ab2_ptr<T>(c.dvold[o]), ab2_ptr<T>(c.dwold[o]), nch == 1 ? c.P.kmax : kc, nch);
}
// one instance per spacing case: with power-of-two spacings every a/dx is
// the product, so neither the test nor the division is in the kernel.  The
// FP32 form, held to tolerances rather than to the reference's rounding,
// always takes the product by the reciprocal (within an ulp of the quotient).
// MB: blocks per SM the registers are budgeted for.  FP64 three (80
// registers, a few spilled: 0.895 -> 0.840 ms at 256^3 against two blocks
// at 120 registers); FP32 four (64 registers).
template <typename T>
void ab2_launch(Ctx& c, const MomArgs& a, int o) {
  if constexpr (sizeof(T) == 8) {
    if (c.P.pow2) ab2_launch_pw<T, 1, 3>(c, a, o);
    else ab2_launch_pw<T, 0, 3>(c, a, o);
  } else {
    ab2_launch_pw<T, 1, 4>(c, a, o);
  }
}

#undef TC
}  // namespace

// the FP32 form's instance (k_ab2_f32.cu)
void ab2_launch_f32(Ctx& c, const MomArgs& a, int o);
// the TMA-fed FP64 predictor (k_ab2_tma.cu); false when it does not apply
bool ab2_tma_launch(Ctx& c, const MomArgs& a, int o);

}  // namespace icls
