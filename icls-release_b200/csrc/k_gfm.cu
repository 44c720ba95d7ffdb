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
// cache broadcasts.  Curvature runs in the form's field type T (FP64 or the
// precision form's FP32); the jump assembly reads T fields and runs in FP64.
#include <algorithm>

#include "batch.cuh"

namespace icls {

__constant__ double cP[270];
__constant__ float cPf[270];  // the same coefficients rounded to FP32

namespace {

constexpr int NT = 256;
#define TC(x) static_cast<T>(x)

// acc + a b: one fused multiply-add in the FP32 form (held to tolerances;
// this file is compiled without contraction), separately rounded in FP64
// as the reference evaluates it
__device__ __forceinline__ float mac(float acc, float a, float b) { return __fmaf_rn(a, b, acc); }
__device__ __forceinline__ double mac(double acc, double a, double b) { return acc + a * b; }

template <typename T>
__device__ __forceinline__ T coef(int q);
template <>
__device__ __forceinline__ double coef<double>(int q) { return cP[q]; }
template <>
__device__ __forceinline__ float coef<float>(int q) { return cPf[q]; }

// curvature at an interior cell (interface.f90:57-111); m = |grad phi| or 1
template <typename T>
__device__ __forceinline__ T curvature_at(const Params& p, const T* __restrict__ phi, int i, int j, int k, T& m) {
  const long long c = idxL(p, i, j, k);
  m = TC(1.);
  if (!(fabs(phi[c]) <= TC(p.NB - 1. * p.dz))) return TC(0.);
  // x[r] = sum over the 27 stencil values in order q = 0..26 of P(r,q)*phi_q,
  // accumulated while the stencil is read
  T x[10];
#pragma unroll
  for (int r = 1; r < 10; ++r) x[r] = TC(0.);
  const long long sy = p.nLx, sz = (long long)p.nLx * p.nLy;
  if constexpr (sizeof(T) == 4) {
    // FP32: the 27 values first, then each x[r] as one chain over q in the
    // same order, every coefficient index a compile-time constant (an
    // operand of the product, no separate load)
    T v[27];
#pragma unroll
    for (int q = 0; q < 27; ++q) v[q] = phi[c + (q % 3 - 1) + (q / 3 % 3 - 1) * sy + (q / 9 - 1) * sz];
#pragma unroll
    for (int r = 1; r < 10; ++r)
#pragma unroll
      for (int q = 0; q < 27; ++q) x[r] = mac(x[r], coef<T>(r * 27 + q), v[q]);
  } else {
    int n = 0;
#pragma unroll 1
    for (int dk = -1; dk <= 1; ++dk)
#pragma unroll
      for (int dj = -1; dj <= 1; ++dj)
#pragma unroll
        for (int di = -1; di <= 1; ++di) {
          const T v = phi[c + di + dj * sy + dk * sz];
#pragma unroll
          for (int r = 1; r < 10; ++r) x[r] = x[r] + coef<T>(r * 27 + n) * v;
          ++n;
        }
  }
  const T dphidx = x[1], dphidy = x[2], dphidz = x[3];
  const T d2phidx = x[4], d2phidy = x[5], d2phidz = x[6];
  const T d2phidxdy = x[7], d2phidxdz = x[8], d2phidydz = x[9];
  const T norm_val = sqrt((dphidx * dphidx + dphidy * dphidy) + dphidz * dphidz);
  m = norm_val;
  T cv;
  if (norm_val < TC(0.9)) {
    cv = TC(0.);
  } else {
    const T n3 = norm_val * norm_val * norm_val;
    const T term1 = ((d2phidx + d2phidy) + d2phidz) / norm_val;
    T term2 = (dphidx * dphidx * d2phidx + dphidy * dphidy * d2phidy) + dphidz * dphidz * d2phidz;
    term2 = term2 / n3;
    T term3 = (dphidx * dphidy * d2phidxdy + dphidx * dphidz * d2phidxdz) + dphidy * dphidz * d2phidydz;
    term3 = TC(2.) * term3 / n3;
    cv = -((term1 - term2) - term3);
  }
  const T max_kappa = TC(1. / p.dz);
  if (cv < -max_kappa) cv = -max_kappa;
  else if (cv > max_kappa) cv = max_kappa;
  else if (fabs(cv) < TC(1e-9)) cv = TC(0.);
  return cv;
}

// get_curvature + boundc over the tasks' shape-C regions (phi0 = the
// drop's level set, out = its curvature): wall rows stay 0, halos are the
// periodic copies (bound.f90:292-305), the apron (far field, |phi| > 5dz)
// is 0.
template <typename T>
__global__ void __launch_bounds__(NT, 4) k_curvature(Params p, const __grid_constant__ LsBatch B, T* __restrict__ nrm_m,
                                                  MlpCell* __restrict__ rec, int* __restrict__ count, int cap) {
  const int ti = task_of(B);
  const LsTask& t = B.t[ti];
  const Col c = col_of(p, t, (int)blockIdx.x - B.start[ti]);
  const T* phi = cT<T>(t.phi0);
  T* out = mT<T>(t.out);
  const T lim = TC(4. * p.dz);
  const unsigned lane = threadIdx.x & 31u;
  // every lane of the warp walks the same rows, so the ballots line up
  for (int k = c.ka; k <= c.kb; ++k) {
    if (c.ok) {
      T v = TC(0.);
      if (k != 0 && k != p.k1 && computed(c, t.r, k)) {
        T m;
        v = curvature_at(p, phi, c.i, c.j, k, m);
        if (nrm_m) nrm_m[idxI(p, c.i, c.j, k)] = m;
      }
      putC(p, out, c.i, c.j, k, v);
    }
    if (rec) {  // the network's cells: slots by a warp-aggregated counter
      const bool take = c.ok && k >= 1 && k <= p.kmax && computed(c, t.r, k) &&
                        fabs(phi[idxL(p, c.i, c.j, k)]) <= lim;
      const unsigned msk = __ballot_sync(0xffffffffu, take);
      if (msk) {
        int base = 0;
        if (lane == (unsigned)(__ffs(msk) - 1)) base = atomicAdd(count, __popc(msk));
        base = __shfl_sync(0xffffffffu, base, __ffs(msk) - 1);
        const int slot = base + __popc(msk & ((1u << lane) - 1u));
        if (take && slot < cap) rec[slot] = MlpCell{ti, c.i, c.j, k};
      }
    }
  }
}

// re_curvature + boundc (interface.f90:186-218) over the tasks' regions:
// phis (get_curvature) -> out
template <typename T>
__global__ void __launch_bounds__(NT, (sizeof(T) == 4 ? 6 : 5)) k_recurvature(Params p, const __grid_constant__ LsBatch B) {
  const int ti = task_of(B);
  const LsTask& t = B.t[ti];
  const T* __restrict__ cin = cT<T>(t.phis);
  const T* __restrict__ phi = cT<T>(t.phi0);
  T* out = mT<T>(t.out);
  const Col c = col_of(p, t, (int)blockIdx.x - B.start[ti]);
  if (!c.ok) return;
  const long long sy = p.nCx, sz = (long long)p.nCx * p.nCy;
  for (int k = c.ka; k <= c.kb; ++k) {
    T acc = TC(0.);
    if (k != 0 && k != p.k1 && computed(c, t.r, k) && fabs(phi[idxL(p, c.i, c.j, k)]) < TC(2. * p.dz)) {
      const long long cc = idxC(p, c.i, c.j, k);
      int q = 0;
#pragma unroll
      for (int dk = -1; dk <= 1; ++dk)
#pragma unroll
        for (int dj = -1; dj <= 1; ++dj)
#pragma unroll
          for (int di = -1; di <= 1; ++di) acc = mac(acc, coef<T>(q++), cin[cc + di + dj * sy + dk * sz]);
    }
    putC(p, out, c.i, c.j, k, acc);
  }
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
template <typename T>
__device__ __forceinline__ double axis_jump(const Params& p, const T* __restrict__ phi, const T* __restrict__ cv,
                                            long long cl, long long sl, long long cc, long long sc, double& pface) {
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

// gfm4p jump shell of the tasks' drops (gfm.f90:95-238; phis = the drop's
// re_curvature), added to the jump fields that gfm4p zeroed (gfm.f90:75-79).
// The additions are atomic: where at most two drops reach a cell the sum is
// the reference's exactly (0+a+b is exact in either order); a cell in the
// shells of three or more drops may differ in the last bit.
template <typename T>
__global__ void __launch_bounds__(NT, (sizeof(T) == 4 ? 5 : 4)) k_jumps(Params p, const __grid_constant__ LsBatch B,
                                              double* __restrict__ pjump, T* __restrict__ px,
                                              T* __restrict__ py, T* __restrict__ pz) {
  const int ti = task_of(B);
  const LsTask& t = B.t[ti];
  const T* __restrict__ cv = cT<T>(t.phis);
  const Col c = col_of(p, t, (int)blockIdx.x - B.start[ti]);
  if (!c.ok || !c.cxy) return;
  const T* __restrict__ phi = cT<T>(t.phi0);
  const int i = c.i, j = c.j;
  for (int k = max(c.ka, max(t.r.cz0, 1)); k <= min(c.kb, min(t.r.cz1, p.kmax)); ++k) {
    const long long cl = idxL(p, i, j, k);
    const double lv = phi[cl];
    if (!(fabs(lv) <= 2. * p.dz)) continue;
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
    atomicAdd(pjump + cc, pj);
    atomicAdd(px + cc, (T)fx);  // assembled in FP64, stored in the field type
    atomicAdd(py + cc, (T)fy);
    atomicAdd(pz + cc, (T)fz);
  }
}

// ipot: dtemp(m,n) = minval(where(|phi_m|<dz and phi_n<cutoff) phi_m+phi_n, 1e3)
__device__ __forceinline__ unsigned long long ord_bits(double x) {
  unsigned long long b = (unsigned long long)__double_as_longlong(x);
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}
// one pair (m, n): sweeps m's written cells (task 0, phi0 = phi_m); phi_n
// is read where n's region wrote it and is its far field bgn elsewhere
template <typename T>
__global__ void __launch_bounds__(NT) k_ipot_pair(Params p, const __grid_constant__ LsBatch B, const T* __restrict__ pn,
                                                  Region rn, double bgn, double bggn,
                                                  unsigned long long* __restrict__ out) {
  const LsTask& t = B.t[0];
  const T* pm = cT<T>(t.phi0);
  const Col c = col_of(p, t, (int)blockIdx.x);
  double s = 1e3;
  if (c.ok) {
    for (int k = c.ka; k <= c.kb; ++k) {
      const long long n = idxL(p, c.i, c.j, k);
      const double a = pm[n];
      const double b = in_written(p, rn, c.i, c.j, k) ? (double)pn[n] : ((k < 0 || k > p.k1) ? bggn : bgn);
      if (a > -1. * p.dz && a < 1. * p.dz && b < p.NB) s = fmin(s, a + b);
    }
  }
  // block min through the ordered bit pattern
  unsigned long long bits = ord_bits(s);
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long q = __shfl_down_sync(0xffffffffu, bits, o);
    bits = q < bits ? q : bits;
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

#undef TC
}  // namespace

void set_pseudo_inverse(const double* P270, cudaStream_t s) {
  static float f[270];
  for (int q = 0; q < 270; ++q) f[q] = (float)P270[q];
  cudaMemcpyToSymbolAsync(cP, P270, 270 * sizeof(double), 0, cudaMemcpyHostToDevice, s);
  cudaMemcpyToSymbolAsync(cPf, f, 270 * sizeof(float), 0, cudaMemcpyHostToDevice, s);
  cudaStreamSynchronize(s);
}

const dim3 kTile(TBX, TBY, 1);

void launch_curvature(Ctx& c, const LsBatch& b, double* nrm_m_out, bool collect) {
  if (b.n == 0) return;
  Scope sc_(c.prof, c.s, "curvature", 1);
  MlpCell* rec = collect ? reinterpret_cast<MlpCell*>(c.mlp_rec) : nullptr;
  if (collect) cudaMemsetAsync(c.mlp_count, 0, sizeof(int), c.s);
  if (c.P.f32)
    k_curvature<float><<<b.start[b.n], kTile, 0, c.s>>>(c.P, b, reinterpret_cast<float*>(nrm_m_out), rec, c.mlp_count,
                                                        c.mlp_cap);
  else
    k_curvature<double><<<b.start[b.n], kTile, 0, c.s>>>(c.P, b, nrm_m_out, rec, c.mlp_count, c.mlp_cap);
}
void launch_recurvature(Ctx& c, const LsBatch& b) {
  if (b.n == 0) return;
  Scope sc_(c.prof, c.s, "recurvature", 1);
  if (c.P.f32)
    k_recurvature<float><<<b.start[b.n], kTile, 0, c.s>>>(c.P, b);
  else
    k_recurvature<double><<<b.start[b.n], kTile, 0, c.s>>>(c.P, b);
}
void launch_jumps(Ctx& c, const LsBatch& b) {
  if (b.n == 0) return;
  Scope sc_(c.prof, c.s, "jumps", 1);
  if (c.P.f32)
    k_jumps<float><<<b.start[b.n], kTile, 0, c.s>>>(c.P, b, c.pjump, reinterpret_cast<float*>(c.px),
                                                     reinterpret_cast<float*>(c.py), reinterpret_cast<float*>(c.pz));
  else
    k_jumps<double><<<b.start[b.n], kTile, 0, c.s>>>(c.P, b, c.pjump, c.px, c.py, c.pz);
}
// the periodic column spans a..a+la-1 and b..b+lb-1 of n columns share a
// column (two arcs meet iff one starts inside the other)
bool spans_meet(int a, int la, int b, int lb, int n) {
  if (la >= n || lb >= n) return la > 0 && lb > 0;
  if (la <= 0 || lb <= 0) return false;
  const int d1 = ((b - a) % n + n) % n, d2 = ((a - b) % n + n) % n;
  return d1 < la || d2 < lb;
}
// dmin_dev: L*L unsigned long long ordered bits, filled here; only cells
// written by both drops' regions can hold |phi_m| < dz and phi_n < 6dz
// unless a far field is below 6dz, so each pair sweeps m's written cells.
// A pair whose written regions are disjoint, with n's far fields at or
// above 6dz, has no such cell: the reference's minimum stays at its initial
// 1e3 (interface.f90:250-260), which the buffer's preset bits already hold
// for every pair not launched (ordered bits of 1e3), so it is not swept.
void launch_ipot(Ctx& c, double* dmin_dev) {
  unsigned long long* o = reinterpret_cast<unsigned long long*>(dmin_dev);
  LsBatch b;
  b.n = 1;
  for (int m = 0; m < c.P.L; ++m)
    for (int n = 0; n < c.P.L; ++n) {
      if (m == n) continue;
      const Region& rm = c.win[m].valid;
      const Region& rn = c.win[n].valid;
      const bool meet = spans_meet(rm.xa, rm.xn, rn.xa, rn.xn, c.P.imax) &&
                        spans_meet(rm.ya, rm.yn, rn.ya, rn.yn, c.P.jmax) && rm.z0 <= rn.z1 && rn.z0 <= rm.z1;
      if (!meet && c.win[n].bg >= c.P.NB && c.win[n].bg_ghost >= c.P.NB) continue;
      LsTask& t = b.t[0];
      t = LsTask();
      t.r = c.win[m].valid;
      t.r.cx0 = 0; t.r.cx1 = t.r.xn - 1; t.r.cy0 = 0; t.r.cy1 = t.r.yn - 1;
      t.r.cz0 = t.r.z0; t.r.cz1 = t.r.z1;
      t.l = m;
      t.phi0 = c.lv[m];
      set_tiles(b, 8);
      Scope sc_(c.prof, c.s, "ipot", 1);
      if (c.P.f32)
        k_ipot_pair<float><<<b.start[1], kTile, 0, c.s>>>(c.P, b, reinterpret_cast<const float*>(c.lv[n]),
                                                          c.win[n].valid, c.win[n].bg, c.win[n].bg_ghost,
                                                          o + m + (long long)c.P.L * n);
      else
        k_ipot_pair<double><<<b.start[1], kTile, 0, c.s>>>(c.P, b, c.lv[n], c.win[n].valid, c.win[n].bg,
                                                           c.win[n].bg_ghost, o + m + (long long)c.P.L * n);
    }
}

}  // namespace icls
