// k_poisson.cu — the pressure Poisson solve of solver2d (solver.f90:68-196),
// FP64, with multiply-add contraction (the transforms and the elimination
// are held to a tolerance against the oracle, not to its rounding).
//
// Forward: real FFT along x of every (j,k) line, then along y of every
// (i,k) column of those coefficients, with VFFTPACK's contract (fft.f:
// 1123-1142): half-complex layout r0, Re1, Im1, ..., r_{N/2} and sqrt(1/N)
// scaling.  Thomas elimination in z per (i,j) with diagonal b(k)+xyrt(i,j)
// (solver.f90:119-160), the exactly-zero last pivot of mode (0,0) giving
// p=0.  Inverse: y then x, the exact inverse of the forward transform
// (fft.f:403-452).  The 2decomp transposes of the reference
// (transpose_*.f90) are replaced by the access pattern of each kernel: the
// x pass streams contiguous lines, the y pass loads 16-wide column tiles,
// the z pass walks k with one thread per (i,j).  In the fused time step the
// forward x pass forms fillps' right-hand side itself from the predicted
// velocities (and p_jump), so p is not written and read back in between.
//
// Two real lines share one complex FFT (z = a + i b).  Lines of 64, 128 or
// 256 points, and of 48, 96, 192 or 384 (a radix-3 factor), take the
// two-level transform (k_fft2): N = R1 x R2 with R1 = 16, a radix-16 DFT of
// every R2-strided subsequence in registers (each thread has its 32 loads in
// flight), the N-point twiddles, one padded shared-memory exchange, and a
// radix-R2 DFT in registers; other powers of two take radix-2 passes in
// shared memory (k_fft_x, k_fft_y).
#include <cmath>
#include <type_traits>
#include <vector>

#include "ctx.h"

namespace icls {

namespace {

constexpr int FT = 256;  // threads per FFT CTA

__device__ __forceinline__ int bitrev(int x, int logn) { return (int)(__brev((unsigned)x) >> (32 - logn)); }

// in-place radix-2 DIT over nl lines of length N = 2^logN stored at
// buf[l*ld + n], input in bit-reversed order.  inv: e^{+i} twiddles.
// Two consecutive stages run fused on four values held in registers: the
// same butterflies in the same order as stage-by-stage passes, with half
// the shared-memory round trips and barriers.
__device__ __forceinline__ void bfly(double2& x0, double2& x1, double2 w) {
  const double2 t1 = make_double2(x1.x * w.x - x1.y * w.y, x1.x * w.y + x1.y * w.x);
  x1 = make_double2(x0.x - t1.x, x0.y - t1.y);
  x0 = make_double2(x0.x + t1.x, x0.y + t1.y);
}
__device__ __forceinline__ double2 twid(const double2* __restrict__ tw, int idx, int inv) {
  double2 w = __ldg(&tw[idx]);
  if (inv) w.y = -w.y;
  return w;
}
__device__ __forceinline__ void smem_fft(double2* buf, int nl, int N, int logN, int ld,
                                         const double2* __restrict__ tw, int inv) {
  int s = 1;
  if (logN >= 2) {
    const int q4 = N >> 2, lq4 = logN - 2;
    for (; s + 1 <= logN; s += 2) {
      const int lh = s - 1, h = 1 << lh;
      for (int t = threadIdx.x; t < nl * q4; t += blockDim.x) {
        const int line = t >> lq4, b = t & (q4 - 1);
        const int grp = b >> lh, j = b & (h - 1);
        double2* L = buf + line * ld + (grp << (lh + 2)) + j;
        double2 x0 = L[0], x1 = L[h], x2 = L[2 * h], x3 = L[3 * h];
        const double2 w1 = twid(tw, j << (logN - s), inv);
        bfly(x0, x1, w1);
        bfly(x2, x3, w1);
        bfly(x0, x2, twid(tw, j << (logN - s - 1), inv));
        bfly(x1, x3, twid(tw, (j + h) << (logN - s - 1), inv));
        L[0] = x0; L[h] = x1; L[2 * h] = x2; L[3 * h] = x3;
      }
      __syncthreads();
    }
  }
  if (s == logN) {  // an odd stage count leaves the last stage
    const int lh = s - 1, h = 1 << lh, halfN = N >> 1, lhalf = logN - 1;
    for (int t = threadIdx.x; t < nl * halfN; t += blockDim.x) {
      const int line = t >> lhalf, b = t & (halfN - 1);
      const int grp = b >> lh, j = b & (h - 1);
      double2* L = buf + line * ld + (grp << (lh + 1)) + j;
      double2 x0 = L[0], x1 = L[h];
      bfly(x0, x1, twid(tw, j << (logN - s), inv));
      L[0] = x0; L[h] = x1;
    }
    __syncthreads();
  }
}

// split Z (FFT of a+ib) into the scaled half-complex spectra of a and b
__device__ __forceinline__ void unpack_hc(const double2* Z, int N, int n, double s, double& ha, double& hb) {
  // position n of the half-complex output
  if (n == 0) { ha = s * Z[0].x; hb = s * Z[0].y; return; }
  if (n == N - 1) { ha = s * Z[N / 2].x; hb = s * Z[N / 2].y; return; }
  const int k = (n + 1) >> 1;
  const double2 zk = Z[k], zn = Z[N - k];
  // A_k = (Z_k + conj Z_{N-k})/2 ; B_k = (Z_k - conj Z_{N-k})/(2i)
  if (n & 1) {  // real parts
    ha = s * (0.5 * (zk.x + zn.x));
    hb = s * (0.5 * (zk.y + zn.y));
  } else {      // imaginary parts
    ha = s * (0.5 * (zk.y - zn.y));
    hb = s * (-0.5 * (zk.x - zn.x));
  }
}

// Z_k of the Hermitian pair built from two half-complex lines a, b
__device__ __forceinline__ double2 pack_hc(const double* a, const double* b, int N, int k, long long st) {
  if (k == 0) return make_double2(a[0], b[0]);
  if (k == N / 2) return make_double2(a[(N - 1) * st], b[(N - 1) * st]);
  if (k < N / 2) {
    const double ar = a[(2 * k - 1) * st], ai = a[(2 * k) * st];
    const double br = b[(2 * k - 1) * st], bi = b[(2 * k) * st];
    return make_double2(ar - bi, ai + br);
  }
  const int m = N - k;
  const double ar = a[(2 * m - 1) * st], ai = a[(2 * m) * st];
  const double br = b[(2 * m - 1) * st], bi = b[(2 * m) * st];
  return make_double2(ar + bi, -ai + br);
}

// ---- x pass: lines (j,k) of length imax; CL complex lines per CTA --------
// dir 0: p (shape C interior) -> spec ; dir 1: spec -> p (+ boundp halos)
__global__ void __launch_bounds__(FT) k_fft_x(Params p, int dir, int CL, int logN, const double2* __restrict__ tw,
                                              double* __restrict__ pp, double* __restrict__ spec, int halos) {
  extern __shared__ double2 sm[];
  const int N = p.imax;
  const int ld = N + 1;
  const long long nlines = (long long)p.jmax * p.kmax;
  const long long l0 = (long long)blockIdx.x * (2 * CL);
  const double s = sqrt(1.0 / N);
  // load
  for (int t = threadIdx.x; t < CL * N; t += blockDim.x) {
    const int cl = t >> logN, n = t & (N - 1);
    const long long la = l0 + 2 * cl, lb = la + 1;
    double2 z = make_double2(0., 0.);
    if (lb < nlines) {
      if (dir == 0) {
        const int ja = (int)(la % p.jmax) + 1, ka = (int)(la / p.jmax) + 1;
        const int jb = (int)(lb % p.jmax) + 1, kb = (int)(lb / p.jmax) + 1;
        z = make_double2(pp[idxC(p, n + 1, ja, ka)], pp[idxC(p, n + 1, jb, kb)]);
        sm[cl * ld + bitrev(n, logN)] = z;
      } else {
        const double* a = spec + la * N;
        const double* b = spec + lb * N;
        sm[cl * ld + bitrev(n, logN)] = pack_hc(a, b, N, n, 1);
      }
    }
  }
  __syncthreads();
  smem_fft(sm, CL, N, logN, ld, tw, dir);
  for (int t = threadIdx.x; t < CL * N; t += blockDim.x) {
    const int cl = t >> logN, n = t & (N - 1);
    const long long la = l0 + 2 * cl, lb = la + 1;
    if (lb >= nlines) continue;
    if (dir == 0) {
      double ha, hb;
      unpack_hc(sm + cl * ld, N, n, s, ha, hb);
      spec[la * N + n] = ha;
      spec[lb * N + n] = hb;
    } else {
      const double2 z = sm[cl * ld + n];
      const double va = s * z.x, vb = s * z.y;
      for (int h = 0; h < 2; ++h) {
        const long long ll = h ? lb : la;
        const double v = h ? vb : va;
        const int j = (int)(ll % p.jmax) + 1, k = (int)(ll / p.jmax) + 1;
        const int i = n + 1;
        if (!halos) {
          pp[idxC(p, i, j, k)] = v;
          continue;
        }
        // boundp (bound.f90:182-287): every image of (i,j,k)
        const int nj = (j == 1) ? 2 : ((j == p.jmax) ? 2 : 1);
        const int nk = (k == 1) ? 2 : ((k == p.kmax) ? 2 : 1);
        const int ni = (i == 1) ? 2 : ((i == p.imax) ? 2 : 1);
        for (int a = 0; a < ni; ++a) {
          const int ii = a == 0 ? i : (i == 1 ? p.i1 : 0);
          for (int b = 0; b < nj; ++b) {
            const int jj = b == 0 ? j : (j == 1 ? p.j1 : 0);
            for (int cidx = 0; cidx < nk; ++cidx) {
              const int kk = cidx == 0 ? k : (k == 1 ? 0 : p.k1);
              pp[idxC(p, ii, jj, kk)] = v;
            }
          }
        }
      }
    }
  }
}

// ---- y pass: columns (i,k) of length jmax, TI real columns per CTA -------
__global__ void __launch_bounds__(FT) k_fft_y(Params p, int dir, int TI, int logN, const double2* __restrict__ tw,
                                              double* __restrict__ spec) {
  extern __shared__ double2 sm[];
  const int N = p.jmax;
  const int CL = TI / 2;
  const int ld = N + 1;
  const int tiles_i = p.imax / TI;
  const int k = blockIdx.x / tiles_i + 1;
  const int i0 = (blockIdx.x % tiles_i) * TI + 1;
  const int lt = __ffs(TI) - 1;  // TI is a power of two
  const long long sj = p.imax;
  double* base = spec + (long long)(i0 - 1) + (long long)p.imax * (long long)p.jmax * (k - 1);
  const double s = sqrt(1.0 / N);
  // load: consecutive threads read consecutive i
  for (int t = threadIdx.x; t < TI * N; t += blockDim.x) {
    const int ti = t & (TI - 1), n = t >> lt;
    const double v = base[ti + n * sj];
    double* slot = reinterpret_cast<double*>(&sm[(ti >> 1) * ld]);
    if (dir == 0) {
      slot[2 * bitrev(n, logN) + (ti & 1)] = v;
    } else {
      slot[2 * n + (ti & 1)] = v;  // raw half-complex, packed below
    }
  }
  __syncthreads();
  if (dir == 1) {
    // build Z in a second buffer region then copy back in bit-reversed order
    double2* tmp = sm + CL * ld;
    for (int t = threadIdx.x; t < CL * N; t += blockDim.x) {
      const int cl = t >> logN, kk = t & (N - 1);
      const double* raw = reinterpret_cast<const double*>(&sm[cl * ld]);
      // raw[2n] = a_n, raw[2n+1] = b_n
      tmp[cl * ld + bitrev(kk, logN)] = pack_hc(raw, raw + 1, N, kk, 2);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < CL * ld; t += blockDim.x) sm[t] = tmp[t];
    __syncthreads();
  }
  smem_fft(sm, CL, N, logN, ld, tw, dir);
  for (int t = threadIdx.x; t < TI * N; t += blockDim.x) {
    const int ti = t & (TI - 1), n = t >> lt;
    const int cl = ti >> 1;
    double v;
    if (dir == 0) {
      double ha, hb;
      unpack_hc(sm + cl * ld, N, n, s, ha, hb);
      v = (ti & 1) ? hb : ha;
    } else {
      const double2 z = sm[cl * ld + n];
      v = (ti & 1) ? s * z.y : s * z.x;
    }
    base[ti + n * sj] = v;
  }
}

// ---- two-level transform for N = R1 x R2 -----------------------------------
// The DFT of z[n], n = R2 n1 + n2, at k = k1 + R1 k2:
//   Z[k] = sum_n2 W_N^(n2 k1) [sum_n1 z[R2 n1 + n2] W_R1^(n1 k1)] W_R2^(n2 k2),
// W = e^{-2 pi i / N} (e^{+} for the inverse).  Register DFTs are radix-2
// decimation in time with the bit reversal done by register renaming.
constexpr int bitrev_c(int x, int bits) {
  int r = 0;
  for (int b = 0; b < bits; ++b) r |= ((x >> b) & 1) << (bits - 1 - b);
  return r;
}
constexpr int ilog2_c(int n) { return n <= 1 ? 0 : 1 + ilog2_c(n >> 1); }

// W_N^m, 0 <= m < N (N even), from the half table tw[m] = W_N^m, m < N/2
// (W_N^(m+N/2) = -W_N^m)
__device__ __forceinline__ double2 twid_full(const double2* __restrict__ tw, int m, int N, int inv) {
  double2 w;
  if (m >= N / 2) {
    w = __ldg(&tw[m - N / 2]);
    w = make_double2(-w.x, -w.y);
  } else {
    w = __ldg(&tw[m]);
  }
  if (inv) w.y = -w.y;
  return w;
}
__device__ __forceinline__ double2 cmul(double2 a, double2 w) {
  return make_double2(a.x * w.x - a.y * w.y, a.x * w.y + a.y * w.x);
}

// in-register DFT of R points, natural order in and out; tw is the N-point
// half table, W_R^m = W_N^(m N/R)
template <int R>
__device__ __forceinline__ void reg_dft(double2 (&x)[R], const double2* __restrict__ tw, int N, int inv);

// R = 3 Q (Q a power of two): n = Q n1 + n2, k = k1 + 3 k2; a 3-point DFT
// over n1 for every n2, the R-point twiddles W_R^(n2 k1), then a Q-point DFT
// over n2 for every k1
template <int R>
__device__ __forceinline__ void reg_dft3(double2 (&x)[R], const double2* __restrict__ tw, int N, int inv) {
  constexpr int Q = R / 3;
  const double2 w1 = twid_full(tw, N / 3, N, inv), w2 = twid_full(tw, 2 * (N / 3), N, inv);
  double2 y[3][Q];
#pragma unroll
  for (int n2 = 0; n2 < Q; ++n2) {
    const double2 a = x[n2], b = x[Q + n2], c = x[2 * Q + n2];
    const double2 b1 = cmul(b, w1), c2 = cmul(c, w2), b2 = cmul(b, w2), c1 = cmul(c, w1);
    y[0][n2] = make_double2((a.x + b.x) + c.x, (a.y + b.y) + c.y);
    y[1][n2] = make_double2((a.x + b1.x) + c2.x, (a.y + b1.y) + c2.y);
    y[2][n2] = make_double2((a.x + b2.x) + c1.x, (a.y + b2.y) + c1.y);
    if (n2 > 0) {
      y[1][n2] = cmul(y[1][n2], twid_full(tw, n2 * (N / R), N, inv));
      y[2][n2] = cmul(y[2][n2], twid_full(tw, 2 * n2 * (N / R), N, inv));
    }
  }
#pragma unroll
  for (int k1 = 0; k1 < 3; ++k1) {
    reg_dft<Q>(y[k1], tw, N, inv);
#pragma unroll
    for (int k2 = 0; k2 < Q; ++k2) x[k1 + 3 * k2] = y[k1][k2];
  }
}

template <int R>
__device__ __forceinline__ void reg_dft(double2 (&x)[R], const double2* __restrict__ tw, int N, int inv) {
  if constexpr (R % 3 == 0) {
    reg_dft3<R>(x, tw, N, inv);
    return;
  }
  constexpr int LR = ilog2_c(R);
  double2 y[R];
#pragma unroll
  for (int n = 0; n < R; ++n) y[bitrev_c(n, LR)] = x[n];
#pragma unroll
  for (int h = 1; h < R; h <<= 1) {
#pragma unroll
    for (int g = 0; g < R; g += 2 * h) {
#pragma unroll
      for (int j = 0; j < h; ++j) {
        if (j == 0) {  // W^0 = 1: the product is exact, skip it
          const double2 a = y[g], b = y[g + h];
          y[g] = make_double2(a.x + b.x, a.y + b.y);
          y[g + h] = make_double2(a.x - b.x, a.y - b.y);
        } else {
          bfly(y[g + j], y[g + j + h], twid(tw, j * (R / (2 * h)) * (N / R), inv));
        }
      }
    }
  }
#pragma unroll
  for (int n = 0; n < R; ++n) x[n] = y[n];
}

// The Poisson right-hand side of fillps (fillps.f90:36-53), plus p_jump when
// add is set, at shape-C index c from the predicted velocities of type T
// (float in the FP32 form): the expression of k_fillps, so the same bits.
struct RhsArgs {
  const void *du, *dv, *dw;
  const double* pj;
  int add;
};
template <typename T>
__device__ __forceinline__ double rhs_at(const Params& p, const RhsArgs& r, long long c) {
  const T* __restrict__ du = static_cast<const T*>(r.du);
  const T* __restrict__ dv = static_cast<const T*>(r.dv);
  const T* __restrict__ dw = static_cast<const T*>(r.dw);
  // explicitly rounded operations: this file allows multiply-add
  // contraction, k_fillps (k_navier.cu) does not
  const double coef = p.rho0 / p.dt;
  const double vel_x = __dmul_rn(__dsub_rn((double)du[c], (double)du[c - 1]), p.dxi);
  const double vel_y = __dmul_rn(__dsub_rn((double)dv[c], (double)dv[c - p.nCx]), p.dyi);
  const double vel_z = __dmul_rn(__dsub_rn((double)dw[c], (double)dw[c - (long long)p.nCx * p.nCy]), p.dzi);
  double v = __dmul_rn(coef, __dadd_rn(__dadd_rn(vel_x, vel_y), vel_z));
  if (r.add) v = __dadd_rn(v, r.pj[c]);
  return v;
}

// One CTA transforms LPC complex lines (2 LPC real lines).  YPASS false:
// x lines (j,k), contiguous; the R lanes of a line are adjacent threads.
// YPASS true: columns (i,k), columns adjacent in memory; the lines of a CTA
// are adjacent threads.  dir 0: p (x) or spec (y) -> half-complex spec;
// dir 1: the inverse, into spec (y) or p (x, with the boundp images when
// halos is set).  RHS (forward x pass only): 0 reads p; 4 or 8 forms
// fillps' right-hand side from float or double velocities instead (rhs_at),
// so p is neither written by fillps nor read here.
// LPC complex lines per CTA of 256 threads, TPL = max(R1, R2) threads per
// line; LPC * TPL <= 256 (the other threads idle)
template <int R1, int R2, bool YPASS, int LPC, int RHS = 0>
__global__ void __launch_bounds__(256, (R1 > 16 || R2 > 16) ? 1 : 2)
    k_fft2(Params p, int dir, const double2* __restrict__ tw, double* __restrict__ pp, double* __restrict__ spec,
           int halos, RhsArgs ra) {
  static_assert(RHS == 0 || !YPASS, "the right-hand side is formed in the forward x pass");
  constexpr int N = R1 * R2;
  constexpr int TPL = R1 > R2 ? R1 : R2;
  static_assert(LPC * TPL <= 256, "a CTA holds LPC lines of TPL threads");
  constexpr int SLD = R1 + 1;             // exchange row (padded)
  constexpr int LS = R2 * SLD + 1;        // exchange line stride (padded)
  constexpr int ZLD = N + 1;              // natural-order line stride
  extern __shared__ double2 sm[];
  const int lt = YPASS ? (int)threadIdx.x % LPC : (int)threadIdx.x / TPL;
  const int lane = YPASS ? (int)threadIdx.x / LPC : (int)threadIdx.x % TPL;
  const bool used = (int)threadIdx.x < LPC * TPL;  // the threads beyond LPC lines idle
  const double s = sqrt(1.0 / N);
  // the two real lines: element n of line a at A[n * st], of line b at B[n * st]
  const double* A;
  const double* B;
  long long st;
  bool live;
  int ja = 0, ka = 0, jb = 0, kb = 0;  // x pass: the (j,k) of lines a and b
  double* colbase = nullptr;            // y pass: the first column of the pair
  if (!YPASS) {
    const long long nlines = (long long)p.jmax * p.kmax;
    const long long la = 2 * ((long long)blockIdx.x * LPC + lt), lb = la + 1;
    live = used && lb < nlines;
    ja = (int)(la % p.jmax) + 1; ka = (int)(la / p.jmax) + 1;
    jb = (int)(lb % p.jmax) + 1; kb = (int)(lb / p.jmax) + 1;
    st = 1;
    if (dir == 0) {
      A = pp + idxC(p, 1, ja, ka);
      B = pp + idxC(p, 1, jb, kb);
    } else {
      A = spec + la * N;
      B = spec + lb * N;
    }
  } else {
    const int tiles_i = p.imax / (2 * LPC);
    const int k = (int)blockIdx.x / tiles_i + 1;
    const int i0 = ((int)blockIdx.x % tiles_i) * (2 * LPC) + 2 * lt;  // 0-based column
    live = used;
    colbase = spec + (long long)i0 + (long long)p.imax * p.jmax * (k - 1);
    st = p.imax;
    A = colbase;
    B = colbase + 1;
  }
  double2* S = sm + lt * LS;
  // step 1: lane n2 < R2 transforms z[R2 n1 + n2] over n1
  if (lane < R2 && live) {
    double2 x[R1];
#pragma unroll
    for (int n1 = 0; n1 < R1; ++n1) {
      const int n = R2 * n1 + lane;
      if constexpr (RHS != 0) {  // dir 0: lines a and b start at columns 1 of (ja,ka), (jb,kb)
        using T = typename std::conditional<RHS == 4, float, double>::type;
        x[n1] = make_double2(rhs_at<T>(p, ra, idxC(p, 1, ja, ka) + n), rhs_at<T>(p, ra, idxC(p, 1, jb, kb) + n));
      } else {
        x[n1] = dir == 0 ? make_double2(A[n * st], B[n * st]) : pack_hc(A, B, N, n, st);
      }
    }
    reg_dft<R1>(x, tw, N, dir);
#pragma unroll
    for (int k1 = 1; k1 < R1; ++k1) {
      if (lane == 0) continue;
      const double2 w = twid_full(tw, lane * k1, N, dir);
      const double2 v = x[k1];
      x[k1] = make_double2(v.x * w.x - v.y * w.y, v.x * w.y + v.y * w.x);
    }
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) S[lane * SLD + k1] = x[k1];
  }
  __syncthreads();
  // step 2: lane k1 < R1 transforms over n2 -> Z[k1 + R1 k2]
  double2 X[R2];
  if (lane < R1 && live) {
#pragma unroll
    for (int n2 = 0; n2 < R2; ++n2) X[n2] = S[n2 * SLD + lane];
    reg_dft<R2>(X, tw, N, dir);
  }
  if (dir == 1) {
    if (lane < R1 && live) {
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) {
        const int n = lane + R1 * k2;
        const double va = s * X[k2].x, vb = s * X[k2].y;
        if (YPASS) {
          colbase[(long long)n * st] = va;
          colbase[(long long)n * st + 1] = vb;
        } else {
        for (int h = 0; h < 2; ++h) {
          const int j = h ? jb : ja, k = h ? kb : ka;
          const double v = h ? vb : va;
          const int i = n + 1;
          if (!halos) {
            pp[idxC(p, i, j, k)] = v;
            continue;
          }
          // boundp (bound.f90:182-287): every image of (i,j,k)
          const int nj = (j == 1 || j == p.jmax) ? 2 : 1;
          const int nk = (k == 1 || k == p.kmax) ? 2 : 1;
          const int ni = (i == 1 || i == p.imax) ? 2 : 1;
          for (int a = 0; a < ni; ++a) {
            const int ii = a == 0 ? i : (i == 1 ? p.i1 : 0);
            for (int b = 0; b < nj; ++b) {
              const int jj = b == 0 ? j : (j == 1 ? p.j1 : 0);
              for (int cidx = 0; cidx < nk; ++cidx) {
                const int kk = cidx == 0 ? k : (k == 1 ? 0 : p.k1);
                pp[idxC(p, ii, jj, kk)] = v;
              }
            }
          }
        }
        }
      }
    }
    return;
  }
  // forward: natural order through shared memory for the half-complex split
  __syncthreads();  // every read of S is done
  double2* Z = sm + lt * ZLD;
  if (lane < R1 && live) {
#pragma unroll
    for (int k2 = 0; k2 < R2; ++k2) Z[lane + R1 * k2] = X[k2];
  }
  __syncthreads();
  if (!live) return;
  for (int n = lane; n < N; n += TPL) {
    double ha, hb;
    unpack_hc(Z, N, n, s, ha, hb);
    if (YPASS) {
      colbase[(long long)n * st] = ha;
      colbase[(long long)n * st + 1] = hb;
    } else {
      const long long la = 2 * ((long long)blockIdx.x * LPC + lt);
      spec[la * N + n] = ha;
      spec[(la + 1) * N + n] = hb;
    }
  }
}
template <int R1, int R2, int LPC>
constexpr size_t fft2_smem() {
  constexpr int ex = LPC * (R2 * (R1 + 1) + 1), nat = LPC * (R1 * R2 + 1);
  return (size_t)(ex > nat ? ex : nat) * sizeof(double2);
}

// ---- Thomas elimination in z (solver.f90:119-160) -------------------------
// zpiv(d,k) = 1/(b(k)+xy - a(k) d(k-1)) for k<kmax (z of the reference)
// and the raw last divisor at k=kmax.  The pivots depend on (i,j) only
// through xy = xrt(i) + yrt(j), and xrt(2m) = xrt(2m+1), yrt likewise, so
// one column per distinct pair d = (i/2) + (imax/2+1) (j/2) serves every
// (i,j) that shares it: (imax/2+1)(jmax/2+1) columns, L2-resident at 256^2.
__host__ __device__ __forceinline__ long long pivot_columns(const Params& p) {
  return (long long)(p.imax / 2 + 1) * (p.jmax / 2 + 1);
}
// 1/pivots of the Thomas elimination (solver.f90:119-160, 245-283) of each
// distinct eigenvalue column q < nd: zpiv[q + (r-1) nd], r = 1..K-1, and the
// last pivot itself at r = K
__global__ void k_thomas_setup(const double* __restrict__ eig, long long nd, int K, const double* __restrict__ a,
                               const double* __restrict__ b, const double* __restrict__ c,
                               double* __restrict__ zpiv) {
  const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (q >= nd) return;
  const double xy = eig[q];
  double z = 1. / (b[1] + xy);
  double d = c[1] * z;
  zpiv[q] = z;
  for (int k = 2; k <= K - 1; ++k) {
    const double bb = b[k] + xy;
    z = 1. / (bb - a[k] * d);
    d = c[k] * z;
    zpiv[q + (k - 1) * nd] = z;
  }
  const double bb = b[K] + xy;
  zpiv[q + (K - 1) * nd] = bb - a[K] * d;
}

// The sweeps read 8 rows ahead of the dependency chain (same operations,
// in the same order, as a row-by-row loop).
constexpr int TU = 8;
// one line of K values at col[0], col[st], ...: forward elimination with the
// stored 1/pivots zc[0], zc[nd], ..., the zero-pivot rule of the last row
// (p = 0, the singular mode), back substitution with d = c z
__device__ __forceinline__ void thomas_line(double* __restrict__ col, long long st, int K,
                                            const double* __restrict__ zc, long long nd,
                                            const double* __restrict__ a, const double* __restrict__ c) {
  double prev = col[0] * zc[0];
  col[0] = prev;
  for (int k0 = 2; k0 <= K - 1; k0 += TU) {
    double cv[TU], zv[TU];
#pragma unroll
    for (int u = 0; u < TU; ++u)
      if (k0 + u <= K - 1) {
        cv[u] = col[(k0 + u - 1) * st];
        zv[u] = zc[(k0 + u - 1) * nd];
      }
#pragma unroll
    for (int u = 0; u < TU; ++u)
      if (k0 + u <= K - 1) {
        const double v = (cv[u] - a[k0 + u] * prev) * zv[u];
        col[(k0 + u - 1) * st] = v;
        prev = v;
      }
  }
  const double zz = zc[(K - 1) * nd];
  double nxt;
  if (zz != 0.) nxt = (col[(K - 1) * st] - a[K] * prev) / zz;
  else nxt = 0.;
  col[(K - 1) * st] = nxt;
  for (int k0 = K - 1; k0 >= 1; k0 -= TU) {
    double cv[TU], zv[TU];
#pragma unroll
    for (int u = 0; u < TU; ++u)
      if (k0 - u >= 1) {
        cv[u] = col[(k0 - u - 1) * st];
        zv[u] = zc[(k0 - u - 1) * nd];
      }
#pragma unroll
    for (int u = 0; u < TU; ++u)
      if (k0 - u >= 1) {
        const double d = c[k0 - u] * zv[u];
        const double v = cv[u] - d * nxt;
        col[(k0 - u - 1) * st] = v;
        nxt = v;
      }
  }
}
// solver2d: lines along z, one thread per (i,j)
__global__ void __launch_bounds__(128) k_thomas(Params p, const double* __restrict__ a, const double* __restrict__ c,
                                                const double* __restrict__ zpiv, double* __restrict__ spec) {
  const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long nxy = (long long)p.imax * p.jmax, nd = pivot_columns(p);
  if (q >= nxy) return;
  const int i = (int)(q % p.imax) + 1, j = (int)(q / p.imax) + 1;
  thomas_line(spec + q, nxy, p.kmax, zpiv + (i >> 1) + (long long)(p.imax / 2 + 1) * (j >> 1), nd, a, c);
}
// solver2d_cos (solver.f90:245-283): lines along y, one thread per (i,k),
// diagonal b(j) + xzrt(i,k); the distinct columns are (i>>1, k)
__global__ void __launch_bounds__(128) k_thomas_y(Params p, const double* __restrict__ a, const double* __restrict__ c,
                                                  const double* __restrict__ zpiv, double* __restrict__ spec) {
  const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long nxz = (long long)p.imax * p.kmax, nd = (long long)(p.imax / 2 + 1) * p.kmax;
  if (q >= nxz) return;
  const int i = (int)(q % p.imax) + 1, k = (int)(q / p.imax) + 1;
  thomas_line(spec + (i - 1) + (long long)p.imax * p.jmax * (k - 1), p.imax, p.jmax,
              zpiv + (i >> 1) + (long long)(p.imax / 2 + 1) * (k - 1), nd, a, c);
}

// VCOSQB (dir 0) / VCOSQF (dir 1) along z of every (i,j) line of spec, as
// the matrix product out[m] = sum_k T[m][k] x[k] with the kmax x kmax table
// T of the transform's definition (fft.f:120-124, 270-274).  A CTA holds 32
// consecutive i of one j (all k) in shared memory; warp w forms rows
// m = 4w.., 4 at a time, each lane one i, summing in k order with fused
// multiply-adds.
constexpr int CZ_TI = 32, CZ_ROWS = 4;
constexpr int kCosqFftMaxN = 512;  // CZ_LINES x (N+1) complex values in shared memory
__global__ void __launch_bounds__(256) k_cosq_z(Params p, const double* __restrict__ T, double* __restrict__ spec) {
  extern __shared__ double czx[];  // [kmax][CZ_TI]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int i0 = 1 + CZ_TI * (int)blockIdx.x, j = 1 + (int)blockIdx.y;
  const int K = p.kmax;
  const long long plane = (long long)p.imax * p.jmax;
  double* __restrict__ base = spec + (i0 - 1) + (long long)p.imax * (j - 1);
  const int ni = min(CZ_TI, p.imax - i0 + 1);
  for (int t = threadIdx.x; t < K * CZ_TI; t += blockDim.x) {
    const int k = t / CZ_TI, l = t - k * CZ_TI;
    czx[t] = l < ni ? base[l + plane * k] : 0.;
  }
  __syncthreads();
  if (lane >= ni) return;
  for (int m0 = CZ_ROWS * warp; m0 < K; m0 += CZ_ROWS * 8) {
    double acc[CZ_ROWS];
    const double* __restrict__ tr[CZ_ROWS];
#pragma unroll
    for (int r = 0; r < CZ_ROWS; ++r) {
      acc[r] = 0.;
      tr[r] = T + (long long)min(m0 + r, K - 1) * K;
    }
    for (int k = 0; k < K; ++k) {
      const double xv = czx[k * CZ_TI + lane];
#pragma unroll
      for (int r = 0; r < CZ_ROWS; ++r) acc[r] = __fma_rn(__ldg(tr[r] + k), xv, acc[r]);
    }
#pragma unroll
    for (int r = 0; r < CZ_ROWS; ++r)
      if (m0 + r < K) base[lane + plane * (m0 + r)] = acc[r];
  }
}

// The same transforms for a power-of-two kmax up to kCosqFftMaxN through one
// N-point complex FFT per two lines (Makhoul's reordering; J. Makhoul, "A
// fast cosine transform in one and two dimensions", IEEE Trans. ASSP 28,
// 1980): with W_k = e^{i pi k/(2N)},
//   VCOSQB: v = (x0, x2, ..., x3, x1), V = FFT(v), out_k = (2/sqrt N) Re(conj(W_k) V_k);
//   VCOSQF: V_k = W_k (y_k - i y_{N-k})/2 (y_N = 0), z = sum_k V_k e^{+2 pi i kn/N},
//           out_{2n} = z_n/sqrt N, out_{2n+1} = z_{N-1-n}/sqrt N.
// Columns 2c and 2c+1 of the CTA's 32 i travel as the real and imaginary
// parts of complex line c (16 lines, 66 KB of shared memory per CTA for
// N = 256; 16 columns per CTA measured no faster); the transform is
// smem_fft (bit-reversed input).
constexpr int CZF_TI = 32, CZ_LINES = CZF_TI / 2;  // columns and complex lines per CTA
__device__ __forceinline__ int makhoul_pos(int k, int N) { return (k & 1) ? N - 1 - (k >> 1) : (k >> 1); }
__global__ void __launch_bounds__(256) k_cosq_fft_z(Params p, int dir, int logN, const double2* __restrict__ tw,
                                                    const double2* __restrict__ cw, double* __restrict__ spec) {
  extern __shared__ double2 czb[];  // [CZ_LINES][N+1]
  const int N = p.kmax, ld = N + 1;
  const int i0 = 1 + CZF_TI * (int)blockIdx.x, j = 1 + (int)blockIdx.y;
  const long long plane = (long long)p.imax * p.jmax;
  double* __restrict__ base = spec + (i0 - 1) + (long long)p.imax * (j - 1);
  const int ni = min(CZF_TI, p.imax - i0 + 1);
  const double rs = 1. / sqrt((double)N);
  if (dir == 0) {
    for (int t = threadIdx.x; t < N * CZF_TI; t += blockDim.x) {
      const int k = t / CZF_TI, l = t - k * CZF_TI;
      double* slot = reinterpret_cast<double*>(&czb[(l >> 1) * ld + bitrev(makhoul_pos(k, N), logN)]) + (l & 1);
      *slot = l < ni ? base[l + plane * k] : 0.;
    }
  } else {
    for (int t = threadIdx.x; t < N * CZ_LINES; t += blockDim.x) {
      const int k = t / CZ_LINES, c = t - k * CZ_LINES, la = 2 * c, lb = la + 1;
      const double ya = la < ni ? base[la + plane * k] : 0., yb = lb < ni ? base[lb + plane * k] : 0.;
      const double yan = (k && la < ni) ? base[la + plane * (N - k)] : 0.;
      const double ybn = (k && lb < ni) ? base[lb + plane * (N - k)] : 0.;
      const double2 w = cw[k];
      const double2 va = make_double2(0.5 * (w.x * ya + w.y * yan), 0.5 * (w.y * ya - w.x * yan));
      const double2 vb = make_double2(0.5 * (w.x * yb + w.y * ybn), 0.5 * (w.y * yb - w.x * ybn));
      czb[c * ld + bitrev(k, logN)] = make_double2(va.x - vb.y, va.y + vb.x);
    }
  }
  __syncthreads();
  smem_fft(czb, CZ_LINES, N, logN, ld, tw, dir);
  for (int t = threadIdx.x; t < N * CZF_TI; t += blockDim.x) {
    const int k = t / CZF_TI, l = t - k * CZF_TI;
    if (l >= ni) continue;
    const double2* L = czb + (l >> 1) * ld;
    double out;
    if (dir == 0) {
      const double2 zk = L[k], zn = L[(N - k) & (N - 1)];
      double vr, vi;
      if (l & 1) { vr = 0.5 * (zk.y + zn.y); vi = -0.5 * (zk.x - zn.x); }
      else { vr = 0.5 * (zk.x + zn.x); vi = 0.5 * (zk.y - zn.y); }
      const double2 w = cw[k];
      out = (2. * rs) * (w.x * vr + w.y * vi);
    } else {
      const double2 z = L[makhoul_pos(k, N)];
      out = ((l & 1) ? z.y : z.x) * rs;
    }
    base[l + plane * k] = out;
  }
}

int ilog2(int n) {
  int l = 0;
  while ((1 << l) < n) ++l;
  return l;
}

void make_twiddles(int N, std::vector<double2>& t) {
  t.resize(N / 2 > 0 ? N / 2 : 1);
  const long double pi = 3.141592653589793238462643383279502884L;
  for (int m = 0; m < N / 2; ++m) {
    long double a = -2.0L * pi * (long double)m / (long double)N;
    t[m] = make_double2((double)cosl(a), (double)sinl(a));
  }
}

}  // namespace

// tables of initsolver (initsolver.f90:20-82) and the twiddles
void poisson_setup_cos(Ctx& c);
void poisson_setup(Ctx& c) {
  if (c.P.bcy != ICLS_BCY_PERIODIC) {
    poisson_setup_cos(c);
    return;
  }
  const Params& P = c.P;
  const int itot = P.imax, jtot = P.jmax, kmax = P.kmax;
  std::vector<double> a(kmax + 1, 0.), b(kmax + 1, 0.), cc(kmax + 1, 0.);
  for (int k = 1; k <= kmax; ++k) { a[k] = P.dzi * P.dzi; cc[k] = P.dzi * P.dzi; b[k] = -(a[k] + cc[k]); }
  b[1] = b[1] + a[1];
  b[kmax] = b[kmax] + cc[kmax];
  a[1] = 0.; cc[kmax] = 0.;
  std::vector<double> xrt(itot + 1, 0.), yrt(jtot + 1, 0.);
  const double pi = P.pi;
  for (int i = 3; i <= itot; i += 2) {
    double s = std::sin((double)(i - 1) * pi / (2. * itot));
    xrt[i - 1] = -4. * P.dxi * P.dxi * (s * s);
    xrt[i] = xrt[i - 1];
  }
  xrt[1] = 0.; xrt[itot] = -4. * P.dxi * P.dxi;
  for (int j = 3; j <= jtot; j += 2) {
    double s = std::sin((double)(j - 1) * pi / (2. * jtot));
    yrt[j - 1] = -4. * P.dyi * P.dyi * (s * s);
    yrt[j] = yrt[j - 1];
  }
  yrt[1] = 0.; yrt[jtot] = -4. * P.dyi * P.dyi;
  // one entry per distinct (xrt, yrt) pair: column d = ix + (itot/2+1) iy
  // stands for i = 1 (ix = 0) or i = 2 ix, j likewise
  const int nxd = itot / 2 + 1, nyd = jtot / 2 + 1;
  std::vector<double> xy((size_t)nxd * nyd);
  for (int iy = 0; iy < nyd; ++iy)
    for (int ix = 0; ix < nxd; ++ix) {
      const int i = ix == 0 ? 1 : 2 * ix, j = iy == 0 ? 1 : 2 * iy;
      xy[ix + (size_t)nxd * iy] = xrt[i] + yrt[j];
    }
  cudaMemcpyAsync(c.xyrt, xy.data(), xy.size() * sizeof(double), cudaMemcpyHostToDevice, c.s);
  cudaMemcpyAsync(c.tri_a, a.data(), a.size() * sizeof(double), cudaMemcpyHostToDevice, c.s);
  cudaMemcpyAsync(c.tri_b, b.data(), b.size() * sizeof(double), cudaMemcpyHostToDevice, c.s);
  cudaMemcpyAsync(c.tri_c, cc.data(), cc.size() * sizeof(double), cudaMemcpyHostToDevice, c.s);
  std::vector<double2> tx, ty;
  make_twiddles(itot, tx);
  make_twiddles(jtot, ty);
  cudaMemcpyAsync(c.twx, tx.data(), tx.size() * sizeof(double2), cudaMemcpyHostToDevice, c.s);
  cudaMemcpyAsync(c.twy, ty.data(), ty.size() * sizeof(double2), cudaMemcpyHostToDevice, c.s);
  const long long nd = pivot_columns(P);
  k_thomas_setup<<<(unsigned)((nd + 127) / 128), 128, 0, c.s>>>(c.xyrt, nd, P.kmax, c.tri_a, c.tri_b, c.tri_c,
                                                                 c.zpiv);
  cudaStreamSynchronize(c.s);  // host vectors above go out of scope
}

namespace {
// cos(m pi / (2n)) with m reduced mod 4n, in long double
double cos_quarter(long long m, int n) {
  const long long q = 4LL * n;
  m %= q;
  const long double pi = 3.141592653589793238462643383279502884L;
  return (double)cosl((long double)m * pi / (2.0L * n));
}
}  // namespace

// initsolver for BC_in_y = Walls, InOut, OutOut (initsolver.f90:85-156):
// a(j), b(j), c(j) with the end rows of the y boundary, xzrt = xrt(i) +
// zrt(k) per distinct column (i>>1, k), their Thomas pivots, the x twiddles
// and the VCOSQB / VCOSQF matrices (fft.f:120-124, 270-274)
void poisson_setup_cos(Ctx& c) {
  const Params& P = c.P;
  const int itot = P.imax, jtot = P.jmax, kmax = P.kmax;
  std::vector<double> a(jtot + 1, 0.), b(jtot + 1, 0.), cc(jtot + 1, 0.);
  for (int j = 1; j <= jtot; ++j) { a[j] = P.dyi * P.dyi; cc[j] = P.dyi * P.dyi; b[j] = -(a[j] + cc[j]); }
  if (P.bcy == ICLS_BCY_WALLS) {
    b[1] = b[1] + a[1];
    b[jtot] = b[jtot] + cc[jtot];
  } else if (P.bcy == ICLS_BCY_INOUT) {
    b[1] = b[1] + a[1];
    b[jtot] = b[jtot] - cc[jtot];
  } else {
    b[1] = b[1] - a[1];
    b[jtot] = b[jtot] - cc[jtot];
  }
  a[1] = 0.; cc[jtot] = 0.;
  std::vector<double> xrt(itot + 1, 0.), zrt(kmax + 1, 0.);
  const double pi = P.pi;
  for (int i = 3; i <= itot; i += 2) {
    double s = std::sin((double)(i - 1) * pi / (2. * itot));
    xrt[i - 1] = -4. * P.dxi * P.dxi * (s * s);
    xrt[i] = xrt[i - 1];
  }
  xrt[1] = 0.; xrt[itot] = -4. * P.dxi * P.dxi;
  for (int k = 1; k <= kmax; ++k) zrt[k] = (P.dzi * P.dzi) * (-2. + 2. * std::cos((double)(k - 1) * pi / kmax));
  const int nxd = itot / 2 + 1;
  std::vector<double> xz((size_t)nxd * kmax);
  for (int k = 1; k <= kmax; ++k)
    for (int ix = 0; ix < nxd; ++ix) xz[ix + (size_t)nxd * (k - 1)] = xrt[ix == 0 ? 1 : 2 * ix] + zrt[k];
  std::vector<double> tb((size_t)kmax * kmax), tf((size_t)kmax * kmax);
  const double sb = 4. / std::sqrt(4. * kmax), sf = 1. / std::sqrt(4. * kmax);
  for (int m = 0; m < kmax; ++m)
    for (int k = 0; k < kmax; ++k) {
      tb[(size_t)m * kmax + k] = sb * cos_quarter((long long)(2 * k + 1) * m, kmax);
      tf[(size_t)m * kmax + k] = sf * (k == 0 ? 1. : 2. * cos_quarter((long long)(2 * m + 1) * k, kmax));
    }
  cudaMemcpyAsync(c.xyrt, xz.data(), xz.size() * sizeof(double), cudaMemcpyHostToDevice, c.s);
  cudaMemcpyAsync(c.tri_a, a.data(), a.size() * sizeof(double), cudaMemcpyHostToDevice, c.s);
  cudaMemcpyAsync(c.tri_b, b.data(), b.size() * sizeof(double), cudaMemcpyHostToDevice, c.s);
  cudaMemcpyAsync(c.tri_c, cc.data(), cc.size() * sizeof(double), cudaMemcpyHostToDevice, c.s);
  cudaMemcpyAsync(c.cosb, tb.data(), tb.size() * sizeof(double), cudaMemcpyHostToDevice, c.s);
  cudaMemcpyAsync(c.cosf, tf.data(), tf.size() * sizeof(double), cudaMemcpyHostToDevice, c.s);
  std::vector<double2> tx;
  make_twiddles(itot, tx);
  cudaMemcpyAsync(c.twx, tx.data(), tx.size() * sizeof(double2), cudaMemcpyHostToDevice, c.s);
  std::vector<double2> tz, wz(kmax);
  make_twiddles(kmax, tz);
  {
    const long double pi_l = 3.141592653589793238462643383279502884L;
    for (int k = 0; k < kmax; ++k) {
      const long double a = pi_l * (long double)k / (2.0L * kmax);
      wz[k] = make_double2((double)cosl(a), (double)sinl(a));
    }
  }
  cudaMemcpyAsync(c.twy, tz.data(), tz.size() * sizeof(double2), cudaMemcpyHostToDevice, c.s);
  cudaMemcpyAsync(c.czw, wz.data(), wz.size() * sizeof(double2), cudaMemcpyHostToDevice, c.s);
  const long long nd = (long long)nxd * kmax;
  k_thomas_setup<<<(unsigned)((nd + 127) / 128), 128, 0, c.s>>>(c.xyrt, nd, jtot, c.tri_a, c.tri_b, c.tri_c, c.zpiv);
  cudaStreamSynchronize(c.s);  // host vectors above go out of scope
}

static int x_lines_per_cta(int N) {
  int cl = 2048 / N;
  if (cl < 1) cl = 1;
  if (cl > 16) cl = 16;
  return cl;
}
static int y_tile(int imax) {
  int ti = 16;
  while (ti > 2 && imax % ti) ti >>= 1;
  return ti;
}

template <int R1, int R2, bool Y, int LPC, int RHS = 0>
void fft2_launch(Ctx& c, int dir, const double2* tw, int halos, const RhsArgs& ra) {
  const Params& P = c.P;
  static unsigned attr = 0;  // devices this instance's shared-memory limit is raised on
  int dev = 0;
  cudaGetDevice(&dev);
  if (!(attr & (1u << (dev & 31)))) {
    cudaFuncSetAttribute(k_fft2<R1, R2, Y, LPC, RHS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)fft2_smem<R1, R2, LPC>());
    attr |= 1u << (dev & 31);
  }
  const long long units = Y ? (long long)(P.imax / (2 * LPC)) * P.kmax
                            : ((long long)P.jmax * P.kmax + 2 * LPC - 1) / (2 * LPC);
  k_fft2<R1, R2, Y, LPC, RHS>
      <<<(unsigned)units, 256, fft2_smem<R1, R2, LPC>(), c.s>>>(P, dir, tw, c.p, c.spec, halos, ra);
}
// the lengths with a radix-3 factor: 16 lines per CTA where the columns tile
// by 32 (y pass) and the lines need at most 16 threads, else 8
template <int R2, bool Y, int RHS = 0>
void fft2_launch3(Ctx& c, int dir, const double2* tw, int halos, const RhsArgs& ra) {
  if (R2 <= 16 && (!Y || c.P.imax % 32 == 0)) fft2_launch<16, R2, Y, R2 <= 16 ? 16 : 8, RHS>(c, dir, tw, halos, ra);
  else fft2_launch<16, R2, Y, 8, RHS>(c, dir, tw, halos, ra);
}

// the two-level transform of one pass if its length has one (and, for the
// y pass, the columns tile the CTAs); false: the radix-2 kernels.  RHS (the
// forward x pass): fillps' right-hand side formed in the pass (k_fft2).
template <bool Y, int RHS = 0>
bool fft2_pass(Ctx& c, int dir, int halos, const RhsArgs& ra = RhsArgs{}) {
  const Params& P = c.P;
  const int N = Y ? P.jmax : P.imax;
  const double2* tw = Y ? c.twy : c.twx;
  auto fits = [&](int lpc) { return !Y || P.imax % (2 * lpc) == 0; };
  switch (N) {
    case 64: if (!fits(16)) return false; fft2_launch<16, 4, Y, 16, RHS>(c, dir, tw, halos, ra); return true;
    case 128: if (!fits(16)) return false; fft2_launch<16, 8, Y, 16, RHS>(c, dir, tw, halos, ra); return true;
    case 256: if (!fits(16)) return false; fft2_launch<16, 16, Y, 16, RHS>(c, dir, tw, halos, ra); return true;
    case 48: if (!fits(8)) return false; fft2_launch3<3, Y, RHS>(c, dir, tw, halos, ra); return true;
    case 96: if (!fits(8)) return false; fft2_launch3<6, Y, RHS>(c, dir, tw, halos, ra); return true;
    case 192: if (!fits(8)) return false; fft2_launch3<12, Y, RHS>(c, dir, tw, halos, ra); return true;
    case 384: if (!fits(8)) return false; fft2_launch3<24, Y, RHS>(c, dir, tw, halos, ra); return true;
    default: return false;
  }
}
// x line lengths the two-level transform takes
bool fft2_x_length(int n) {
  switch (n) {
    case 64: case 128: case 256: case 48: case 96: case 192: case 384: return true;
    default: return false;
  }
}

// a line length the solve supports along x (y_pass false) or y, for a grid
// with imax columns: powers of two from 8 (radix-2 passes where the
// two-level transform does not apply), and 48, 96, 192, 384 (two-level only;
// the y pass tiles at least 16 columns)
bool fft_length_ok(int n, bool y_pass, int imax) {
  if (n >= 8 && (n & (n - 1)) == 0) return true;
  switch (n) {
    case 48: case 96: case 192: case 384: return !y_pass || imax % 16 == 0;
    default: return false;
  }
}

void launch_solver2d_cos(Ctx& c, int write_halos);
void solver2d_periodic(Ctx& c, int write_halos, const RhsArgs* ra);
void launch_solver2d(Ctx& c, int write_halos) {
  if (c.P.bcy != ICLS_BCY_PERIODIC) {
    launch_solver2d_cos(c, write_halos);
    return;
  }
  solver2d_periodic(c, write_halos, nullptr);
}
// fillps (+ p_jump when add) and solver2d: the right-hand side formed in the
// forward x pass where that pass is the two-level transform, else fillps
// into p first
void launch_fillps_solver2d(Ctx& c, int write_halos, int add) {
  if (c.P.bcy != ICLS_BCY_PERIODIC || !fft2_x_length(c.P.imax)) {
    launch_fillps(c, add);
    launch_solver2d(c, write_halos);
    return;
  }
  RhsArgs ra{c.dudt, c.dvdt, c.dwdt, c.pjump, add};
  solver2d_periodic(c, write_halos, &ra);
}
void solver2d_periodic(Ctx& c, int write_halos, const RhsArgs* ra) {
  Scope sc_(c.prof, c.s, "solver2d", 5);
  const Params& P = c.P;
  const int lx = ilog2(P.imax), ly = ilog2(P.jmax);
  const int CL = x_lines_per_cta(P.imax);
  const long long nlines = (long long)P.jmax * P.kmax;
  const unsigned gx = (unsigned)((nlines + 2 * CL - 1) / (2 * CL));
  const size_t smx = (size_t)CL * (P.imax + 1) * sizeof(double2);
  const int TI = y_tile(P.imax);
  const unsigned gy = (unsigned)((P.imax / TI) * P.kmax);
  const size_t smy = (size_t)2 * (TI / 2) * (P.jmax + 1) * sizeof(double2);
  static unsigned attr = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  if (!(attr & (1u << (dev & 31)))) {
    cudaFuncSetAttribute(k_fft_x, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(k_fft_y, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr |= 1u << (dev & 31);
  }
  if (ra) {  // fft2_x_length(imax): the two-level x pass exists
    if (P.f32) fft2_pass<false, 4>(c, 0, 0, *ra);
    else fft2_pass<false, 8>(c, 0, 0, *ra);
  } else if (!fft2_pass<false>(c, 0, 0)) {
    k_fft_x<<<gx, FT, smx, c.s>>>(P, 0, CL, lx, c.twx, c.p, c.spec, 0);
  }
  if (!fft2_pass<true>(c, 0, 0)) k_fft_y<<<gy, FT, smy, c.s>>>(P, 0, TI, ly, c.twy, c.spec);
  const long long nxy = (long long)P.imax * P.jmax;
  k_thomas<<<(unsigned)((nxy + 127) / 128), 128, 0, c.s>>>(P, c.tri_a, c.tri_c, c.zpiv, c.spec);
  if (!fft2_pass<true>(c, 1, 0)) k_fft_y<<<gy, FT, smy, c.s>>>(P, 1, TI, ly, c.twy, c.spec);
  if (!fft2_pass<false>(c, 1, write_halos)) k_fft_x<<<gx, FT, smx, c.s>>>(P, 1, CL, lx, c.twx, c.p, c.spec, write_halos);
}

// solver2d_cos (solver.f90:202-317): x FFT, VCOSQB in z, Thomas in y,
// VCOSQF in z, inverse x FFT (+ boundp halos and the y-wall rows)
void launch_solver2d_cos(Ctx& c, int write_halos) {
  Scope sc_(c.prof, c.s, "solver2d", 5);
  const Params& P = c.P;
  const int lx = ilog2(P.imax);
  const int CL = x_lines_per_cta(P.imax);
  const long long nlines = (long long)P.jmax * P.kmax;
  const unsigned gx = (unsigned)((nlines + 2 * CL - 1) / (2 * CL));
  const size_t smx = (size_t)CL * (P.imax + 1) * sizeof(double2);
  const size_t smz = (size_t)P.kmax * CZ_TI * sizeof(double);
  static unsigned attr = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  if (!(attr & (1u << (dev & 31)))) {
    cudaFuncSetAttribute(k_fft_x, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(k_cosq_z, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(kCosqMaxN * CZ_TI * sizeof(double)));
    cudaFuncSetAttribute(k_cosq_fft_z, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(CZ_LINES * (kCosqFftMaxN + 1) * sizeof(double2)));
    attr |= 1u << (dev & 31);
  }
  const dim3 gz((unsigned)((P.imax + CZ_TI - 1) / CZ_TI), (unsigned)P.jmax, 1);
  const bool fz = (P.kmax & (P.kmax - 1)) == 0 && P.kmax >= 8 && P.kmax <= kCosqFftMaxN;
  const int lz = ilog2(P.kmax);
  const size_t smf = (size_t)CZ_LINES * (P.kmax + 1) * sizeof(double2);
  const dim3 gzf((unsigned)((P.imax + CZF_TI - 1) / CZF_TI), (unsigned)P.jmax, 1);
  auto cosq = [&](int dir) {
    if (fz) k_cosq_fft_z<<<gzf, 256, smf, c.s>>>(P, dir, lz, c.twy, c.czw, c.spec);
    else k_cosq_z<<<gz, 256, smz, c.s>>>(P, dir ? c.cosf : c.cosb, c.spec);
  };
  if (!fft2_pass<false>(c, 0, 0)) k_fft_x<<<gx, FT, smx, c.s>>>(P, 0, CL, lx, c.twx, c.p, c.spec, 0);
  cosq(0);
  const long long nxz = (long long)P.imax * P.kmax;
  k_thomas_y<<<(unsigned)((nxz + 127) / 128), 128, 0, c.s>>>(P, c.tri_a, c.tri_c, c.zpiv, c.spec);
  cosq(1);
  if (!fft2_pass<false>(c, 1, write_halos)) k_fft_x<<<gx, FT, smx, c.s>>>(P, 1, CL, lx, c.twx, c.p, c.spec, write_halos);
  if (write_halos) launch_ywalls_p(c, c.p);
}

}  // namespace icls
