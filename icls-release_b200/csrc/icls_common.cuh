// icls_common.cuh — device-side parameters, index maps and the numerical
// building blocks shared by all kernels of the ICLS hot path.
//
// Arrays keep the reference's Fortran index space (src/common.f90:7-71):
//   shape C (0:i1,0:j1,0:k1), shape I (1:imax,..), shape L (-2:i1+2,..),
// column-major, i fastest.  The FP64 kernels are compiled with -fmad=false
// and evaluate every expression in the reference's left-to-right order, so
// the arithmetic matches the Fortran bit for bit wherever no
// transcendental function or reordered reduction is involved.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace icls {

struct Params {
  int imax, jmax, kmax;      // one domain: imax=itot, ...
  int i1, j1, k1;
  int L;                     // number of level sets
  // extents of the three array shapes
  int nCx, nCy, nCz;         // C: imax+2, ...
  int nLx, nLy, nLz;         // L: imax+6, ...
  long long nC, nI, nL;      // element counts
  double lx, ly, lz;
  double dxi, dyi, dzi, dx, dy, dz;
  // 1/dx, 1/dy, 1/dz; when all three spacings are powers of two these are
  // exact and a/dx == a*rdx for every a, so divisions become products
  double rdx, rdy, rdz;
  int pow2;
  double NB;                 // NarrowBand_2 = 6dz (param.f90:41)
  double pi;
  double dt;
  double rho1, rho2, miu1, miu2, rho0, visc, iFr, nondi;
  double rrho0;              // 1./rho0, the IEEE quotient the reference evaluates per cell
  int rho0_pow2;             // rho0 is a power of two: x / rho0 == x * rrho0 exactly
  double g1, g2, g3;
  double v_lower, v_upper;
  double forceytot;
  int bcy;                   // BC_in_y: ICLS_BCY_* (param.f90:115)
  int TwoD;
  int ls_adv_space, i_space, ispeed_curv;
  int f32;                   // precision form: bulk fields stored and computed in FP32
};

// ---------------------------------------------------------------- indexing
__host__ __device__ __forceinline__ long long idxC(const Params& p, int i, int j, int k) {
  return (long long)i + (long long)p.nCx * ((long long)j + (long long)p.nCy * (long long)k);
}
__host__ __device__ __forceinline__ long long idxI(const Params& p, int i, int j, int k) {
  return (long long)(i - 1) + (long long)p.imax * ((long long)(j - 1) + (long long)p.jmax * (long long)(k - 1));
}
__host__ __device__ __forceinline__ long long idxL(const Params& p, int i, int j, int k) {
  return (long long)(i + 2) + (long long)p.nLx * ((long long)(j + 2) + (long long)p.nLy * (long long)(k + 2));
}
// periodic source index of a halo coordinate (x: 1..imax, y: 1..jmax)
__host__ __device__ __forceinline__ int wrapx(const Params& p, int i) {
  return i < 1 ? i + p.imax : (i > p.imax ? i - p.imax : i);
}
__host__ __device__ __forceinline__ int wrapy(const Params& p, int j) {
  return j < 1 ? j + p.jmax : (j > p.jmax ? j - p.jmax : j);
}

template <typename T>
__device__ __forceinline__ T sq(T x) { return x * x; }

// a/dx, a/dy, a/dz exactly as the reference divides (a product when the
// spacing is a power of two, which is then bit-identical).  PW fixes the
// choice at compile time for a kernel instantiated per case (1: the
// spacings are powers of two, 0: they are not); -1 reads p.pow2.
template <int PW = -1, typename T>
__device__ __forceinline__ T divx(const Params& p, T a) {
  if constexpr (PW == 1) return a * (T)p.rdx;
  else if constexpr (PW == 0) return a / (T)p.dx;
  else return p.pow2 ? a * (T)p.rdx : a / (T)p.dx;
}
template <int PW = -1, typename T>
__device__ __forceinline__ T divy(const Params& p, T a) {
  if constexpr (PW == 1) return a * (T)p.rdy;
  else if constexpr (PW == 0) return a / (T)p.dy;
  else return p.pow2 ? a * (T)p.rdy : a / (T)p.dy;
}
template <int PW = -1, typename T>
__device__ __forceinline__ T divz(const Params& p, T a) {
  if constexpr (PW == 1) return a * (T)p.rdz;
  else if constexpr (PW == 0) return a / (T)p.dz;
  else return p.pow2 ? a * (T)p.rdz : a / (T)p.dz;
}
// a / rho0: a product by the exact reciprocal when rho0 is a power of two
__device__ __forceinline__ double div_rho0(const Params& p, double a) { return p.rho0_pow2 ? a * p.rrho0 : a / p.rho0; }

// -------------------------------------------------------------- regions
// A per-drop sweep region.  x and y are periodic: the region holds the
// interior columns xa, xa+1, ..., xa+xn-1 (mod imax) and likewise in y,
// and a kernel that writes a column also writes its periodic halo images,
// so the stored halos always equal their source columns.  z is walled: a
// plain range of the storage index (ghost rows -2,-1 and k1+1,k1+2
// included).  The computed part is given by offsets into the written
// spans; written cells outside it form the apron and receive the far-field
// value.  A full axis has xa = 1, xn = imax and no apron.
struct Region {
  int xa, xn, ya, yn;      // written columns
  int cx0, cx1, cy0, cy1;  // computed part, offsets into the written spans
  int z0, z1, cz0, cz1;    // written and computed storage rows
};
// column col (1..n) lies in the periodic span a..a+len-1
__host__ __device__ __forceinline__ bool span_has(int a, int len, int n, int col) {
  int d = col - a;
  if (d < 0) d += n;
  return d < len;
}

// 3-D launch over a region: 32 x 8 threads per block in (i,j), one k per
// block layer.  The thread's cell is (r0 + ...), valid while <= r1.
constexpr int BX = 32, BY = 8;
__device__ __forceinline__ bool cell3(const int* r0, const int* r1, int& i, int& j, int& k) {
  i = r0[0] + (int)(blockIdx.x * BX + threadIdx.x);
  j = r0[1] + (int)(blockIdx.y * BY + threadIdx.y);
  k = r0[2] + (int)blockIdx.z;
  return i <= r1[0] && j <= r1[1] && k <= r1[2];
}
__device__ __forceinline__ int flat_tid() { return threadIdx.x + blockDim.x * threadIdx.y; }

// ------------------------------------------------------------ WENO5, HOUC5
// One WENO5 upwind-biased derivative from the five differences v1..v5
// (hyperPDE.f90:545-576, repeated at 579-611, 622-687, 698-763, 2972-3180).
template <typename T>
__device__ __forceinline__ T weno5(T v1, T v2, T v3, T v4, T v5) {
  const T eps_weno = (T)1.e-6;
  const T sigma_1 = (T)0.1, sigma_2 = (T)0.6, sigma_3 = (T)0.3;
  const T c1312 = (T)(13. / 12.), c14 = (T)(1. / 4.);
  T S1 = c1312 * sq((v1 - (T)2. * v2) + v3) + c14 * sq((v1 - (T)4. * v2) + (T)3. * v3);
  T S2 = c1312 * sq((v2 - (T)2. * v3) + v4) + c14 * sq(v2 - v4);
  T S3 = c1312 * sq((v3 - (T)2. * v4) + v5) + c14 * sq(((T)3. * v3 - (T)4. * v4) + v5);
  T a1 = sigma_1 / sq(eps_weno + S1);
  T a2 = sigma_2 / sq(eps_weno + S2);
  T a3 = sigma_3 / sq(eps_weno + S3);
  T s = (a1 + a2) + a3;
  T w1 = a1 / s, w2 = a2 / s, w3 = a3 / s;
  const T c13 = (T)(1. / 3.), c76 = (T)(7. / 6.), c116 = (T)(11. / 6.), cm16 = (T)(-1. / 6.),
          c56 = (T)(5. / 6.), c16 = (T)(1. / 6.);
  return (w1 * ((c13 * v1 - c76 * v2) + c116 * v3) + w2 * ((cm16 * v2 + c56 * v3) + c13 * v4)) +
         w3 * ((c13 * v3 + c56 * v4) - c16 * v5);
}

// HOUC5 6-point numerators (hyperPDE.f90:428-432)
template <typename T>
__device__ __forceinline__ T houc5_pos(T m3, T m2, T m1, T c0, T p1, T p2) {
  return (T)(1. / 60.) * (((((-((T)2. * m3) + (T)15. * m2) - (T)60. * m1) + (T)20. * c0) + (T)30. * p1) - (T)3. * p2);
}
template <typename T>
__device__ __forceinline__ T houc5_neg(T p3, T p2, T p1, T c0, T m1, T m2) {
  return (T)(1. / 60.) * ((((((T)2. * p3 - (T)15. * p2) + (T)60. * p1) - (T)20. * c0) - (T)30. * m1) + (T)3. * m2);
}

// ------------------------------------------------------------- reductions
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
template <typename T>
__device__ __forceinline__ T warp_max(T v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}
// Block-wide sum in a fixed tree order (result valid in thread 0).
template <typename T, int NT>
__device__ __forceinline__ T block_sum(T v) {
  __shared__ T red[NT / 32];
  v = warp_sum(v);
  const int t = flat_tid();
  const int w = t >> 5, ln = t & 31;
  if (ln == 0) red[w] = v;
  __syncthreads();
  T r = (T)0;
  if (w == 0) {
    r = (ln < NT / 32) ? red[ln] : (T)0;
    r = warp_sum(r);
  }
  __syncthreads();
  return r;
}
template <typename T, int NT>
__device__ __forceinline__ T block_max(T v) {
  __shared__ T red[NT / 32];
  v = warp_max(v);
  const int t = flat_tid();
  const int w = t >> 5, ln = t & 31;
  if (ln == 0) red[w] = v;
  __syncthreads();
  T r = (T)0;
  if (w == 0) {
    r = (ln < NT / 32) ? red[ln] : (T)(-1e300);
    r = warp_max(r);
  }
  __syncthreads();
  return r;
}
// ------------------------------------------------------- exact sums of H
// The drop volume is volume = 1 - sum(H)/N (misc.f90:127-139,
// levelset.f90:505-506): a sum of N ~ 1e7 values near 1 whose complement
// ~1e-4 is kept, so a floating-point sum's rounding, which depends on its
// order, is magnified 1e4-fold in the volume and again, by the correction's
// gain, in the mass-correction step that follows it.  (The reference's own
// result depends on its MPI rank count through that order.)  These sums are
// therefore accumulated exactly: each element is truncated toward zero to a
// multiple of 2^-144 and added as an integer, held in four signed 64-bit
// limbs of 48 bits (value = sum_q L[q] 2^(48q - 144)); the integer does
// not depend on the order of the additions, and it is rounded once to the
// nearest double (ties to even).  Elements must satisfy |x| < 32.
struct XSum {
  long long L[4];
};
constexpr long long kXMask = (1LL << 48) - 1;
__device__ __forceinline__ void xs_zero(XSum& a) { a.L[0] = a.L[1] = a.L[2] = a.L[3] = 0; }
// carry limbs 0..2 into [0, 2^48); limb 3 keeps the sign
__device__ __forceinline__ void xs_norm(XSum& a) {
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const long long c = a.L[q] >> 48;  // arithmetic shift: floor(L / 2^48)
    a.L[q] -= c * (1LL << 48);
    a.L[q + 1] += c;
  }
}
__device__ __forceinline__ void xs_add(XSum& a, double x) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(x);
  int e = (int)((b >> 52) & 0x7FF);
  unsigned long long m = b & ((1ULL << 52) - 1);
  if (e == 0) e = 1;
  else m |= 1ULL << 52;
  if (m == 0) return;
  // |x| = m 2^(e-1075) = m 2^(e-931) units of 2^-144
  int s = e - 931;
  if (s < 0) {
    if (s <= -53) return;
    m >>= -s;
    s = 0;
  }
  // bits s .. s+52 of the integer: limb q = s/48 and the two above it
  const int q = s / 48, o = s - 48 * q;
  const long long sg = (b >> 63) ? -1LL : 1LL;
  const long long lo = sg * (long long)((m << o) & (unsigned long long)kXMask);
  const long long mid = sg * (long long)((m >> (48 - o)) & (unsigned long long)kXMask);
  const long long hi = (96 - o < 64) ? sg * (long long)(m >> (96 - o)) : 0LL;
  if (q == 0) {
    a.L[0] += lo; a.L[1] += mid; a.L[2] += hi;
  } else if (q == 1) {
    a.L[1] += lo; a.L[2] += mid; a.L[3] += hi;
  } else {  // 16 <= |x| < 32: s = 96, nothing above limb 3
    a.L[2] += lo; a.L[3] += mid;
  }
  xs_norm(a);
}
// n elements equal to exactly 1 (the far field of H)
__device__ __forceinline__ void xs_add_count(XSum& a, long long n) { a.L[3] += n; }
__device__ __forceinline__ void xs_merge(XSum& a, const XSum& b) {
#pragma unroll
  for (int q = 0; q < 4; ++q) a.L[q] += b.L[q];
  xs_norm(a);
}
// the sum rounded to the nearest double, ties to even
__device__ __forceinline__ double xs_value(XSum a) {
  xs_norm(a);
  bool neg = false;
  if (a.L[3] < 0) {
    neg = true;
#pragma unroll
    for (int q = 0; q < 4; ++q) a.L[q] = -a.L[q];
    xs_norm(a);
  }
  unsigned long long w[3];
  w[0] = (unsigned long long)a.L[0] | ((unsigned long long)a.L[1] << 48);
  w[1] = ((unsigned long long)a.L[1] >> 16) | ((unsigned long long)a.L[2] << 32);
  w[2] = ((unsigned long long)a.L[2] >> 32) | ((unsigned long long)a.L[3] << 16);
  int top = -1;
  for (int q = 2; q >= 0 && top < 0; --q)
    if (w[q]) top = 64 * q + 63 - __clzll((long long)w[q]);
  if (top < 0) return 0.;
  double r;
  if (top <= 52) {
    r = ldexp((double)w[0], -144);
  } else {
    const int sh = top - 52;
    auto bits = [&](int pos) {  // 64 bits of the integer from bit pos up
      const int wd = pos >> 6, of = pos & 63;
      unsigned long long v = wd < 3 ? w[wd] >> of : 0ULL;
      if (of && wd + 1 < 3) v |= w[wd + 1] << (64 - of);
      return v;
    };
    unsigned long long mant = bits(sh) & ((1ULL << 53) - 1);
    const bool half = (bits(sh - 1) & 1ULL) != 0;
    bool sticky = false;
    for (int pos = 0; pos < sh - 1 && !sticky; pos += 64) {
      const int n = min(64, sh - 1 - pos);
      const unsigned long long v = bits(pos);
      sticky = (n == 64 ? v : (v & ((1ULL << n) - 1))) != 0ULL;
    }
    int ex = sh;
    if (half && (sticky || (mant & 1ULL))) {
      ++mant;
      if (mant == (1ULL << 53)) {
        mant >>= 1;
        ++ex;
      }
    }
    r = ldexp((double)mant, ex - 144);
  }
  return neg ? -r : r;
}
// block-wide exact sum (valid in thread 0): limbs in [0, 2^48) after the
// threads' own normalisation, so a block of up to 2^14 threads cannot
// overflow a limb
template <int NT>
__device__ __forceinline__ XSum block_xsum(XSum a) {
  xs_norm(a);
  XSum r;
#pragma unroll
  for (int q = 0; q < 4; ++q) r.L[q] = block_sum<long long, NT>(a.L[q]);
  return r;
}

// atomic max of a non-negative double through its ordered bit pattern
__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v) {
  atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

// Device scalars kept in HBM between kernels (no host round trip).
struct DevScalars {
  double rho_avr;         // misc.f90:173
  double v_bulk;          // misc.f90:642-655
  double norm;            // main.f90:173-175
  double norm_old;        // main.f90:183
  double residual;        // levelset.f90:831
  double area;            // levelset.f90:499-501
  double heav_sum;        // levelset.f90:505
  double inflate_temp;    // levelset.f90:514
  double inflate_gain;    // blend factor of the last gain-one inflation
  double maxchk;          // levelset.f90:521
  double divtot, divmax;  // chkdiv.f90
  double umax, vmax, wmax;// chkdt.f90:42-44
  double velmax;          // misc.f90:632
  long long divloc;       // linear interior index of max|div|
  int reinit_done;        // residual < dz**5 reached (levelset.f90:833)
  int reinit_iters;
  int nan_flag;           // main.f90:207
  int wait_err;           // a kernel's bounded mbarrier wait gave up
};

}  // namespace icls
