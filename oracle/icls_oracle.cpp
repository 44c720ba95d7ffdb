// icls_oracle.cpp — CPU restatement of the ICLS per-timestep hot path.
//
// TEST INFRASTRUCTURE ONLY: the checker that the CUDA path is compared to.
//
// Each routine below restates one Fortran routine of GeZhouyang/ICLS-release
// (cited as file:line) in FP64, single domain (one MPI rank: imax=itot,
// jmax=jtot, kmax=ktot), keeping the reference's array bounds, column-major
// layout, loop order for reductions, and left-to-right Fortran expression
// order.  Build with -ffp-contract=off so no multiply-add is fused, as in a
// baseline x86-64 gfortran -O3 build (src/Makefile:4).
//
// Parity status.  No Fortran compiler, MPI or LAPACK exists in this image,
// so the reference itself cannot be built or run here, and the reference
// ships no tests, fixtures or golden data.  This restatement is pinned to
// known answers that follow from the reference's own definitions (sphere
// curvature -2/R, the VFFTPACK transform contract checked against numpy,
// exact derivatives of polynomials for HOUC5/WENO5, the Poisson
// eigenvalues, divergence-free correction); it is NOT pinned to reference
// binary outputs: parity unpinned against the Fortran executable.
//
// Two deliberate differences from a literal transcription, both below the
// 1e-10 parity tolerance:
//  * the pseudo-inverse of init_matrix (init.f90:1587-1723) is formed by
//    Gauss-Jordan in long double instead of LAPACK dgetrf/dgetri
//    (misc.f90:549-581), which is unpinned third-party arithmetic;
//  * the real FFTs implement the VFFTPACK input/output contract
//    (fft.f:1123-1142, 403-452: half-complex layout, sqrt(1/N) both ways)
//    with a radix-2 complex FFT instead of FFTPACK's mixed-radix passes.
//
// One deliberate difference that the CUDA path shares: the sum of the
// Heaviside function in the drop volume (misc.f90:127-133) and in the
// inflation (levelset.f90:505-506) is exact (XSum below), not a running
// double sum.  volume = 1 - sum(H)/N keeps a 1e-4 complement of a sum near
// N, so a running sum's rounding, which depends on the order (the
// reference's depends on its MPI rank count through MPI_ALLREDUCE), shows
// up 1e4-fold in the volume and again, multiplied by the correction's gain,
// in the mass correction; with an exact sum every order gives one value.

#include "icls_oracle.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// Exact, order-independent sum of doubles: every element is truncated
// toward zero to a multiple of 2^-144, the integers are added exactly, and
// the total is rounded once to the nearest double (ties to even).  The
// magnitudes of the positive and of the negative elements are kept apart
// as base-2^32 digits (digit d weighs 2^(32d-144)), carried lazily.
struct XSum {
  static constexpr int ND = 8;  // 256 bits: |total| < 2^112
  uint64_t pos[ND] = {0, 0, 0, 0, 0, 0, 0, 0}, neg[ND] = {0, 0, 0, 0, 0, 0, 0, 0};
  int pending = 0;
  void add(double x) {
    if (x == 0.) return;
    uint64_t* a = x < 0. ? neg : pos;
    int E = 0;
    const double f = std::frexp(std::fabs(x), &E);  // |x| = f 2^E, f in [0.5, 1)
    uint64_t m = (uint64_t)std::ldexp(f, 53);        // exact: |x| = m 2^(E-53)
    int sh = E - 53 + 144;                            // |x| = m 2^sh units
    if (sh < 0) {
      if (sh <= -64) return;
      m >>= -sh;
      sh = 0;
    }
    unsigned __int128 t = (unsigned __int128)m << (sh % 32);
    for (int d = sh / 32; t != 0; ++d, t >>= 32) a[d] += (uint64_t)(t & 0xffffffffu);
    if (++pending == (1 << 20)) carry();
  }
  void carry() {
    for (uint64_t* a : {pos, neg})
      for (int d = 0; d + 1 < ND; ++d) {
        a[d + 1] += a[d] >> 32;
        a[d] &= 0xffffffffu;
      }
    pending = 0;
  }
  double value() {
    carry();
    int cmp = 0;
    for (int d = ND - 1; d >= 0 && !cmp; --d)
      if (pos[d] != neg[d]) cmp = pos[d] > neg[d] ? 1 : -1;
    if (!cmp) return 0.;
    const uint64_t* big = cmp > 0 ? pos : neg;
    const uint64_t* sml = cmp > 0 ? neg : pos;
    uint64_t dg[ND];
    int64_t borrow = 0;
    for (int d = 0; d < ND; ++d) {
      int64_t v = (int64_t)big[d] - (int64_t)sml[d] - borrow;
      borrow = v < 0;
      if (v < 0) v += (int64_t)1 << 32;
      dg[d] = (uint64_t)v;
    }
    auto bit = [&](int b) { return b < 0 ? 0 : (int)((dg[b / 32] >> (b % 32)) & 1u); };
    int top = 32 * ND - 1;
    while (!bit(top)) --top;
    const int sh = top > 52 ? top - 52 : 0;
    uint64_t mant = 0;
    for (int b = top; b >= sh; --b) mant = (mant << 1) | (uint64_t)bit(b);
    int ex = sh;
    if (sh > 0 && bit(sh - 1)) {
      bool sticky = false;
      for (int b = 0; b < sh - 1 && !sticky; ++b) sticky = bit(b);
      if (sticky || (mant & 1u)) {
        if (++mant == (1ULL << 53)) {
          mant >>= 1;
          ++ex;
        }
      }
    }
    const double r = std::ldexp((double)mant, ex - 144);
    return cmp > 0 ? r : -r;
  }
};

// Fortran-bounds 3-D array, column-major (i fastest).
struct F3 {
  int l0 = 0, l1 = 0, l2 = 0, n0 = 0, n1 = 0, n2 = 0;
  std::vector<double> v;
  void init(int lo0, int hi0, int lo1, int hi1, int lo2, int hi2, double val = 0.0) {
    l0 = lo0; l1 = lo1; l2 = lo2;
    n0 = hi0 - lo0 + 1; n1 = hi1 - lo1 + 1; n2 = hi2 - lo2 + 1;
    v.assign((size_t)n0 * n1 * n2, val);
  }
  inline double& operator()(int i, int j, int k) {
    return v[(size_t)(i - l0) + (size_t)n0 * ((size_t)(j - l1) + (size_t)n1 * (size_t)(k - l2))];
  }
  inline double operator()(int i, int j, int k) const {
    return v[(size_t)(i - l0) + (size_t)n0 * ((size_t)(j - l1) + (size_t)n1 * (size_t)(k - l2))];
  }
  void fill(double x) { std::fill(v.begin(), v.end(), x); }
  size_t size() const { return v.size(); }
};

inline double sq(double x) { return x * x; }

// One WENO5 upwind-biased derivative from the five differences v1..v5
// (hyperPDE.f90:545-576; identical blocks at 579-611, 622-687, 698-763,
// 2972-3180).
inline double weno5(double v1, double v2, double v3, double v4, double v5) {
  const double eps_weno = 1.e-6;
  const double sigma_1 = 0.1, sigma_2 = 0.6, sigma_3 = 0.3;
  const double c1312 = 13. / 12., c14 = 1. / 4.;
  double S1 = c1312 * sq((v1 - 2. * v2) + v3) + c14 * sq((v1 - 4. * v2) + 3. * v3);
  double S2 = c1312 * sq((v2 - 2. * v3) + v4) + c14 * sq(v2 - v4);
  double S3 = c1312 * sq((v3 - 2. * v4) + v5) + c14 * sq((3. * v3 - 4. * v4) + v5);
  double a1 = sigma_1 / sq(eps_weno + S1);
  double a2 = sigma_2 / sq(eps_weno + S2);
  double a3 = sigma_3 / sq(eps_weno + S3);
  double w1 = a1 / ((a1 + a2) + a3);
  double w2 = a2 / ((a1 + a2) + a3);
  double w3 = a3 / ((a1 + a2) + a3);
  const double c13 = 1. / 3., c76 = 7. / 6., c116 = 11. / 6., cm16 = -1. / 6., c56 = 5. / 6., c16 = 1. / 6.;
  return (w1 * ((c13 * v1 - c76 * v2) + c116 * v3) + w2 * ((cm16 * v2 + c56 * v3) + c13 * v4)) +
         w3 * ((c13 * v3 + c56 * v4) - c16 * v5);
}

// HOUC5 one-sided 6-point derivative numerators (hyperPDE.f90:428-432).
inline double houc5_pos(double m3, double m2, double m1, double c0, double p1, double p2) {
  return (1. / 60.) * (((((-(2. * m3) + 15. * m2) - 60. * m1) + 20. * c0) + 30. * p1) - 3. * p2);
}
inline double houc5_neg(double p3, double p2, double p1, double c0, double m1, double m2) {
  return (1. / 60.) * (((((2. * p3 - 15. * p2) + 60. * p1) - 20. * c0) - 30. * m1) + 3. * m2);
}

// ---------------------------------------------------------------- FFT ----
// Radix-2 complex FFT, e^{-i} for forward.  Power-of-two lengths only;
// other lengths use the O(N^2) DFT below.
void fft_pow2(std::vector<std::complex<double>>& a, bool inverse) {
  const size_t n = a.size();
  for (size_t i = 1, j = 0; i < n; ++i) {
    size_t bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(a[i], a[j]);
  }
  const double pi = std::acos(-1.0);
  for (size_t len = 2; len <= n; len <<= 1) {
    double ang = 2.0 * pi / (double)len * (inverse ? 1.0 : -1.0);
    for (size_t i = 0; i < n; i += len) {
      for (size_t j = 0; j < len / 2; ++j) {
        std::complex<double> w(std::cos(ang * (double)j), std::sin(ang * (double)j));
        std::complex<double> u = a[i + j], t = a[i + j + len / 2] * w;
        a[i + j] = u + t;
        a[i + j + len / 2] = u - t;
      }
    }
  }
}

void dft(std::vector<std::complex<double>>& a, bool inverse) {
  const size_t n = a.size();
  const double pi = std::acos(-1.0);
  std::vector<std::complex<double>> b(n);
  for (size_t k = 0; k < n; ++k) {
    std::complex<double> s = 0;
    for (size_t j = 0; j < n; ++j) {
      double ang = 2.0 * pi * (double)((j * k) % n) / (double)n * (inverse ? 1.0 : -1.0);
      s += a[j] * std::complex<double>(std::cos(ang), std::sin(ang));
    }
    b[k] = s;
  }
  a.swap(b);
}

void cfft(std::vector<std::complex<double>>& a, bool inverse) {
  size_t n = a.size();
  if ((n & (n - 1)) == 0) fft_pow2(a, inverse);
  else dft(a, inverse);
}

// VRFFTF contract (fft.f:1123-1142): r[0]=sqrt(1/N) sum x, r[2k-1]=Re F_k,
// r[2k]=Im F_k (k=1..), r[N-1]=F_{N/2} for even N; all scaled by sqrt(1/N).
void rfftf_line(int n, double* r) {
  std::vector<std::complex<double>> a(n);
  for (int j = 0; j < n; ++j) a[j] = r[j];
  cfft(a, false);
  double s = std::sqrt(1.0 / n);
  r[0] = s * a[0].real();
  for (int k = 1; k < (n + 1) / 2; ++k) {
    r[2 * k - 1] = s * a[k].real();
    r[2 * k] = s * a[k].imag();
  }
  if (n % 2 == 0) r[n - 1] = s * a[n / 2].real();
}

// VRFFTB contract (fft.f:403-452): exact inverse of rfftf_line.
void rfftb_line(int n, double* r) {
  std::vector<std::complex<double>> a(n);
  a[0] = r[0];
  for (int k = 1; k < (n + 1) / 2; ++k) {
    a[k] = std::complex<double>(r[2 * k - 1], r[2 * k]);
    a[n - k] = std::conj(a[k]);
  }
  if (n % 2 == 0) a[n / 2] = r[n - 1];
  cfft(a, true);
  double s = std::sqrt(1.0 / n);
  for (int j = 0; j < n; ++j) r[j] = s * a[j].real();
}

// VCOSQB / VCOSQF (fft.f:218-372 / 68-216) on one line, from their
// documented definitions (fft.f:120-124, 270-274), summed directly in long
// double: backward (the forward transform of solver2d_cos)
//   x(i) = sum_{k=1..n} 4 x(k) cos((2k-1)(i-1) pi/(2n)) / sqrt(4n),
// forward (its normalised inverse)
//   x(i) = (x(1) + sum_{k=2..n} 2 x(k) cos((2i-1)(k-1) pi/(2n))) / sqrt(4n).
// Angles are reduced exactly: cos(m pi/(2n)) with m taken mod 4n.
long double cos_q(long long m, int n) {
  const long long q = 4LL * n;
  m %= q;
  if (m < 0) m += q;
  return std::cos((long double)m * 3.14159265358979323846264338327950288L / (2.0L * n));
}
void cosqb_line(int n, double* x) {
  std::vector<long double> o(n, 0.0L);
  const long double s = 4.0L / std::sqrt(4.0L * n);
  for (int i = 0; i < n; ++i) {
    long double acc = 0.0L;
    for (int k = 0; k < n; ++k) acc += (long double)x[k] * cos_q((long long)(2 * k + 1) * i, n);
    o[i] = s * acc;
  }
  for (int i = 0; i < n; ++i) x[i] = (double)o[i];
}
void cosqf_line(int n, double* x) {
  std::vector<long double> o(n, 0.0L);
  const long double s = 1.0L / std::sqrt(4.0L * n);
  for (int i = 0; i < n; ++i) {
    long double acc = x[0];
    for (int k = 1; k < n; ++k) acc += 2.0L * (long double)x[k] * cos_q((long long)(2 * i + 1) * k, n);
    o[i] = s * acc;
  }
  for (int i = 0; i < n; ++i) x[i] = (double)o[i];
}

}  // namespace

// ======================================================================
struct ora_ctx {
  icls_config c;
  int itot, jtot, ktot, imax, jmax, kmax, i1, j1, k1, L;
  double lx, ly, lz, dxi, dyi, dzi, dx, dy, dz, NB, pi, rho0, visc, nondi;
  double time = 0, dt = 0;

  // mod_common (common.f90:7-71), one domain
  F3 unew, vnew, wnew, pnew, dudt, dvdt, dwdt;
  F3 jiemian, miu, rho, u_l, v_l, w_l, slset, curv_cmn;
  F3 p_x, p_y, p_z, p_xold, p_yold, p_zold;
  F3 uccnew, vccnew, wccnew, rho_u, rho_v, rho_w;
  F3 nrm_m, nrm_x, nrm_y, nrm_z;          // normal%m, %x, %y, %z
  std::vector<F3> lvset, hnew_mls;
  std::vector<uint8_t> mask;               // tube mask of the current drop (interior)
  std::vector<long long> nb_cnt;           // per drop
  std::vector<int> nb_i, nb_j, nb_k;       // index lists of the current drop
  std::vector<double> volume, init_volume, dmin;
  double P[10][27];                        // pseudo_inv_A
  double rho_avr = 0, v_bulk = 0, forceytot = 0, maxchk_glb = 0;
  double reinit_residual = 0; int reinit_iters = 0, last_inflated = 0;
  double last_gain = 0;  // blend factor of the last gain-one inflation
  // main.f90 locals
  F3 duold, dvold, dwold, pold, p_jump, p;
  double norm_old = 0;
  bool initialised = false;
  // solver (solver.f90:42-47)
  std::vector<double> xyrt, ta, tb, tc;
  // solver2d_cos (solver.f90:202-317): tridiagonal in y, eigenvalues
  // xzrt(i,k) = xrt(i) + zrt(k) (initsolver.f90:85-156)
  std::vector<double> xzrt;
  std::vector<double> v_inflow;            // v_inflow(0:i1,0:k1) (common.f90:36)
  int bcy = ICLS_BCY_PERIODIC;

  // ------------------------------------------------------------ shapes
  void shapeC(F3& a) { a.init(0, i1, 0, j1, 0, k1); }
  void shapeI(F3& a) { a.init(1, imax, 1, jmax, 1, kmax); }
  void shapeL(F3& a) { a.init(-2, i1 + 2, -2, j1 + 2, -2, k1 + 2); }

  int setup(const icls_config* cfg) {
    c = *cfg;
    itot = c.itot; jtot = c.jtot; ktot = c.ktot; L = c.lmax;
    if (itot < 4 || jtot < 4 || ktot < 6 || L < 1) return ICLS_E_CONFIG;
    if (itot % 2 || jtot % 2) return ICLS_E_CONFIG;
    // the CUDA path's limit: a level set with its halos below 2^30 elements
    if ((long long)(itot + 6) * (jtot + 6) * (ktot + 6) > (1LL << 30)) return ICLS_E_CONFIG;
    if (c.bc_y < ICLS_BCY_PERIODIC || c.bc_y > ICLS_BCY_OUTOUT) return ICLS_E_CONFIG;
    if (c.ns_conv == ICLS_NS_WENO5) return ICLS_E_UNSUPPORTED;  // boundfu stops (bound.f90:310-322)
    if (c.ns_conv != ICLS_NS_CNTR2) return ICLS_E_CONFIG;
    if (!(c.mass_threshold >= 0.)) return ICLS_E_CONFIG;
    if (c.mass_gain_one != 0 && c.mass_gain_one != 1) return ICLS_E_CONFIG;
    bcy = c.bc_y;
    imax = itot; jmax = jtot; kmax = ktot;
    i1 = imax + 1; j1 = jmax + 1; k1 = kmax + 1;
    lx = c.lx; ly = c.ly; lz = c.lz;
    // param.f90:37-38
    dxi = itot / lx; dyi = jtot / ly; dzi = ktot / lz;
    dx = 1. / dxi; dy = 1. / dyi; dz = 1. / dzi;
    NB = 6. * dz;                                  // param.f90:41
    pi = std::acos(-1.);                           // param.f90:50
    rho0 = std::min(c.rho1, c.rho2);               // param.f90:63
    visc = 1. / c.Re;                              // param.f90:73
    nondi = 1. / c.We;                             // gfm.f90:40
    F3* cs[] = {&unew, &vnew, &wnew, &pnew, &dudt, &dvdt, &dwdt, &jiemian, &miu, &rho, &u_l, &v_l,
                &w_l, &slset, &curv_cmn, &p_x, &p_y, &p_z, &p_xold, &p_yold, &p_zold, &pold, &p_jump, &p};
    for (F3* a : cs) shapeC(*a);
    F3* is[] = {&uccnew, &vccnew, &wccnew, &rho_u, &rho_v, &rho_w, &nrm_m, &nrm_x, &nrm_y, &nrm_z,
                &duold, &dvold, &dwold};
    for (F3* a : is) shapeI(*a);
    lvset.resize(L); hnew_mls.resize(L);
    for (int l = 0; l < L; ++l) { shapeL(lvset[l]); shapeC(hnew_mls[l]); }
    mask.assign((size_t)imax * jmax * kmax, 0);
    nb_cnt.assign(L, 0);
    volume.assign(L, 0.); init_volume.assign(L, 0.); dmin.assign((size_t)L * L, 0.);
    v_inflow.assign((size_t)(i1 + 1) * (k1 + 1), 0.);
    nrm_m.fill(1.);
    return ICLS_OK;
  }

  F3* field(int id, int l) {
    switch (id) {
      case ICLS_F_U: return &unew; case ICLS_F_V: return &vnew; case ICLS_F_W: return &wnew;
      case ICLS_F_PNEW: return &pnew; case ICLS_F_POLD: return &pold; case ICLS_F_P: return &p;
      case ICLS_F_DUDT: return &dudt; case ICLS_F_DVDT: return &dvdt; case ICLS_F_DWDT: return &dwdt;
      case ICLS_F_DUOLD: return &duold; case ICLS_F_DVOLD: return &dvold; case ICLS_F_DWOLD: return &dwold;
      case ICLS_F_PX: return &p_x; case ICLS_F_PY: return &p_y; case ICLS_F_PZ: return &p_z;
      case ICLS_F_PXOLD: return &p_xold; case ICLS_F_PYOLD: return &p_yold; case ICLS_F_PZOLD: return &p_zold;
      case ICLS_F_PJUMP: return &p_jump;
      case ICLS_F_MIU: return &miu; case ICLS_F_RHO: return &rho; case ICLS_F_JIEMIAN: return &jiemian;
      case ICLS_F_RHO_U: return &rho_u; case ICLS_F_RHO_V: return &rho_v; case ICLS_F_RHO_W: return &rho_w;
      case ICLS_F_UCC: return &uccnew; case ICLS_F_VCC: return &vccnew; case ICLS_F_WCC: return &wccnew;
      case ICLS_F_CURV: return &curv_cmn; case ICLS_F_NORMAL_M: return &nrm_m;
      case ICLS_F_LVSET: return (l >= 1 && l <= L) ? &lvset[l - 1] : nullptr;
    }
    return nullptr;
  }

  // ============================================================ bound.f90
  // updthalos (bound.f90:668-716) with the vector types of
  // initmpi.f90:144-147 on a periodic single-rank grid: x then y.
  void updthalos(F3& a) {
    for (int k = 0; k <= k1; ++k)
      for (int j = 0; j <= j1; ++j) { a(i1, j, k) = a(1, j, k); a(0, j, k) = a(imax, j, k); }
    for (int k = 0; k <= k1; ++k)
      for (int i = 0; i <= i1; ++i) { a(i, j1, k) = a(i, 1, k); a(i, 0, k) = a(i, jmax, k); }
  }
  // updthalos_ls (bound.f90:760-797), types initmpi.f90:157-160: 3 layers.
  void updthalos_ls(F3& a) {
    for (int k = -2; k <= k1 + 2; ++k)
      for (int j = -2; j <= j1 + 2; ++j)
        for (int s = 0; s < 3; ++s) { a(i1 + s, j, k) = a(1 + s, j, k); a(-2 + s, j, k) = a(imax - 2 + s, j, k); }
    for (int k = -2; k <= k1 + 2; ++k)
      for (int s = 0; s < 3; ++s)
        for (int i = -2; i <= i1 + 2; ++i) { a(i, j1 + s, k) = a(i, 1 + s, k); a(i, -2 + s, k) = a(i, jmax - 2 + s, k); }
  }
  // bounduvw, BC_in_z='Dirichl', BC_in_y='Periodic' (bound.f90:15-177)
  void bounduvw(F3& u, F3& v, F3& w) {
    const double v_lower = c.v_wall_lower, v_upper = c.v_wall_upper;
    for (int j = 0; j <= j1; ++j)
      for (int i = 0; i <= i1; ++i) {
        u(i, j, 0) = -u(i, j, 1);
        u(i, j, k1) = -u(i, j, kmax);
        v(i, j, 0) = 2. * v_lower - v(i, j, 1);
        v(i, j, k1) = 2. * v_upper - v(i, j, kmax);
        w(i, j, 0) = 0.;
        w(i, j, kmax) = 0.;
        w(i, j, k1) = w(i, j, kmax - 1);
      }
    updthalos(u); updthalos(v); updthalos(w);
    if (bcy != ICLS_BCY_PERIODIC) ywalls_uvw(u, v, w);
  }
  // the y boundaries of bounduvw for BC_in_y = Walls, InOut, OutOut
  // (bound.f90:81-172), over i = 1..imax, k = 1..kmax, after the halos
  void ywalls_uvw(F3& u, F3& v, F3& w) {
    for (int k = 1; k <= kmax; ++k)
      for (int i = 1; i <= imax; ++i) {
        if (bcy == ICLS_BCY_WALLS) {
          u(i, 0, k) = -u(i, 1, k);
          w(i, 0, k) = -w(i, 1, k);
          v(i, 0, k) = 0.;
        } else if (bcy == ICLS_BCY_INOUT) {
          u(i, 0, k) = -u(i, 1, k);
          w(i, 0, k) = -w(i, 1, k);
          v(i, 0, k) = v_inflow[(size_t)i + (size_t)(i1 + 1) * k];
        } else {
          u(i, 0, k) = u(i, 1, k);
          w(i, 0, k) = w(i, 1, k);
          v(i, 0, k) = v(i, 1, k) + dy / dz * (w(i, 1, k) - w(i, 1, k - 1));
        }
      }
    for (int k = 1; k <= kmax; ++k)
      for (int i = 1; i <= imax; ++i) {
        if (bcy == ICLS_BCY_WALLS) {
          u(i, j1, k) = -u(i, jmax, k);
          v(i, jmax, k) = 0.;
          v(i, j1, k) = v(i, jmax, k);
          w(i, j1, k) = -w(i, jmax, k);
        } else {
          u(i, j1, k) = u(i, jmax, k);
          v(i, j1, k) = 2. * v(i, jmax, k) - v(i, jmax - 1, k);
          w(i, j1, k) = w(i, jmax, k);
        }
      }
  }
  // boundp, BC_in_y='Periodic' (bound.f90:182-287)
  void boundp(F3& a) {
    for (int j = 0; j <= j1; ++j)
      for (int i = 0; i <= i1; ++i) { a(i, j, 0) = a(i, j, 1); a(i, j, k1) = a(i, j, kmax); }
    updthalos(a);
    if (bcy == ICLS_BCY_PERIODIC) return;
    // y boundaries (bound.f90:207-282): zero Neumann, or zero Dirichlet at
    // an outflow end
    for (int k = 1; k <= kmax; ++k)
      for (int i = 1; i <= imax; ++i) a(i, 0, k) = bcy == ICLS_BCY_OUTOUT ? -a(i, 1, k) : a(i, 1, k);
    for (int k = 1; k <= kmax; ++k)
      for (int i = 1; i <= imax; ++i) a(i, j1, k) = bcy == ICLS_BCY_WALLS ? a(i, jmax, k) : -a(i, jmax, k);
  }
  // boundc (bound.f90:292-305)
  void boundc(F3& a) { updthalos(a); }
  // boundsls, extrap='line', open_end_in_y=.false. (bound.f90:386-483)
  void boundsls(F3& y) {
    for (int j = -2; j <= j1 + 2; ++j)
      for (int i = -2; i <= i1 + 2; ++i) {
        y(i, j, 0) = 2. * y(i, j, 1) - y(i, j, 2);
        y(i, j, k1) = 2. * y(i, j, kmax) - y(i, j, kmax - 1);
      }
    updthalos_ls(y);
  }
  // boundmls, extrap='line' (bound.f90:518-~657)
  void boundmls() {
    for (int l = 0; l < L; ++l) {
      F3& y = lvset[l];
      for (int j = -2; j <= j1 + 2; ++j)
        for (int i = -2; i <= i1 + 2; ++i) {
          y(i, j, 0) = 2. * y(i, j, 1) - y(i, j, 2);
          y(i, j, -1) = 2. * y(i, j, 0) - y(i, j, 1);
          y(i, j, -2) = 2. * y(i, j, -1) - y(i, j, 0);
          y(i, j, k1) = 2. * y(i, j, kmax) - y(i, j, kmax - 1);
          y(i, j, k1 + 1) = 2. * y(i, j, k1) - y(i, j, kmax);
          y(i, j, k1 + 2) = 2. * y(i, j, k1 + 1) - y(i, j, k1);
        }
    }
    for (int l = 0; l < L; ++l) updthalos_ls(lvset[l]);
  }

  // ===================================================== init.f90 pieces
  // init_matrix (init.f90:1587-1723): pseudo_inv_A = (A^T A)^-1 A^T.
  void init_matrix() {
    long double A[27][10];
    int counter = 0;
    for (int dzs = -1; dzs <= 1; ++dzs)
      for (int dys = -1; dys <= 1; ++dys)
        for (int dxs = -1; dxs <= 1; ++dxs) {
          long double a2 = (long double)(dx * dxs), a3 = (long double)(dy * dys), a4 = (long double)(dz * dzs);
          A[counter][0] = 1; A[counter][1] = a2; A[counter][2] = a3; A[counter][3] = a4;
          A[counter][4] = 0.5L * a2 * a2; A[counter][5] = 0.5L * a3 * a3; A[counter][6] = 0.5L * a4 * a4;
          A[counter][7] = a2 * a3; A[counter][8] = a2 * a4; A[counter][9] = a3 * a4;
          ++counter;
        }
    long double M[10][20];
    for (int r = 0; r < 10; ++r)
      for (int q = 0; q < 10; ++q) {
        long double s = 0;
        for (int n = 0; n < 27; ++n) s += A[n][r] * A[n][q];
        M[r][q] = s;
        M[r][10 + q] = (r == q) ? 1 : 0;
      }
    for (int col = 0; col < 10; ++col) {  // Gauss-Jordan with partial pivoting
      int piv = col;
      for (int r = col + 1; r < 10; ++r) if (fabsl(M[r][col]) > fabsl(M[piv][col])) piv = r;
      if (piv != col) for (int q = 0; q < 20; ++q) std::swap(M[col][q], M[piv][q]);
      long double d = M[col][col];
      for (int q = 0; q < 20; ++q) M[col][q] /= d;
      for (int r = 0; r < 10; ++r) {
        if (r == col) continue;
        long double f = M[r][col];
        if (f != 0) for (int q = 0; q < 20; ++q) M[r][q] -= f * M[col][q];
      }
    }
    for (int r = 0; r < 10; ++r)
      for (int n = 0; n < 27; ++n) {
        long double s = 0;
        for (int q = 0; q < 10; ++q) s += M[r][10 + q] * A[n][q];
        P[r][n] = (double)s;
      }
  }

  // initsolver, BC_in_y='Walls','InOut','OutOut' (initsolver.f90:85-156):
  // tridiagonal in y, cosine eigenvalues in z
  void initsolver_cos() {
    ta.assign(jtot + 1, 0); tb.assign(jtot + 1, 0); tc.assign(jtot + 1, 0);
    for (int j = 1; j <= jtot; ++j) { ta[j] = dyi * dyi; tc[j] = dyi * dyi; tb[j] = -(ta[j] + tc[j]); }
    if (bcy == ICLS_BCY_WALLS) {
      tb[1] = tb[1] + ta[1];
      tb[jtot] = tb[jtot] + tc[jtot];
    } else if (bcy == ICLS_BCY_INOUT) {
      tb[1] = tb[1] + ta[1];
      tb[jtot] = tb[jtot] - tc[jtot];
    } else {
      tb[1] = tb[1] - ta[1];
      tb[jtot] = tb[jtot] - tc[jtot];
    }
    ta[1] = 0.; tc[jtot] = 0.;
    std::vector<double> xrt(itot + 1), zrt(kmax + 1);
    for (int i = 3; i <= itot; i += 2) {
      xrt[i - 1] = -4. * dxi * dxi * sq(std::sin((double)(i - 1) * pi / (2. * itot)));
      xrt[i] = xrt[i - 1];
    }
    xrt[1] = 0.; xrt[itot] = -4. * dxi * dxi;
    for (int k = 1; k <= kmax; ++k) zrt[k] = (dzi * dzi) * (-2. + 2. * std::cos((double)(k - 1) * pi / kmax));
    xzrt.assign((size_t)imax * kmax, 0);
    for (int k = 1; k <= kmax; ++k)
      for (int i = 1; i <= imax; ++i) xzrt[(i - 1) + (size_t)imax * (k - 1)] = xrt[i] + zrt[k];
  }
  // initsolver, BC_in_y='Periodic' (initsolver.f90:20-82)
  void initsolver() {
    if (bcy != ICLS_BCY_PERIODIC) { initsolver_cos(); return; }
    ta.assign(kmax + 1, 0); tb.assign(kmax + 1, 0); tc.assign(kmax + 1, 0);
    for (int k = 1; k <= kmax; ++k) { ta[k] = dzi * dzi; tc[k] = dzi * dzi; tb[k] = -(ta[k] + tc[k]); }
    tb[1] = tb[1] + ta[1];
    tb[kmax] = tb[kmax] + tc[kmax];
    ta[1] = 0.; tc[kmax] = 0.;
    std::vector<double> xrt(itot + 1), yrt(jtot + 1);
    for (int i = 3; i <= itot; i += 2) {
      xrt[i - 1] = -4. * dxi * dxi * sq(std::sin((double)(i - 1) * pi / (2. * itot)));
      xrt[i] = xrt[i - 1];
    }
    xrt[1] = 0.; xrt[itot] = -4. * dxi * dxi;
    for (int j = 3; j <= jtot; j += 2) {
      yrt[j - 1] = -4. * dyi * dyi * sq(std::sin((double)(j - 1) * pi / (2. * jtot)));
      yrt[j] = yrt[j - 1];
    }
    yrt[1] = 0.; yrt[jtot] = -4. * dyi * dyi;
    xyrt.assign((size_t)imax * jmax, 0);
    for (int j = 1; j <= jmax; ++j)
      for (int i = 1; i <= imax; ++i) xyrt[(i - 1) + (size_t)imax * (j - 1)] = xrt[i] + yrt[j];
  }

  // ======================================================= misc.f90
  // Heaviside(var='0', shape='trig', l, eps) (misc.f90:297-464)
  void heaviside_c(int l, double eps, F3& H) {
    const F3& ls = lvset[l];
#pragma omp parallel for
    for (int k = 0; k <= k1; ++k)
      for (int j = 0; j <= j1; ++j)
        for (int i = 0; i <= i1; ++i) {
          double phi = ls(i, j, k);
          double h;
          if (phi < -eps) h = 0.;
          else if (phi < eps) h = (.5 + .5 * phi / eps) + .5 / pi * std::sin(pi * phi / eps);
          else h = 1.;
          H(i, j, k) = h;
        }
  }
  // Dirac(flag='trig', l, eps) (misc.f90:470-543)
  void dirac_trig(int l, double eps, F3& del) {
    const F3& ls = lvset[l];
#pragma omp parallel for
    for (int k = 1; k <= kmax; ++k)
      for (int j = 1; j <= jmax; ++j)
        for (int i = 1; i <= imax; ++i) {
          double phi = ls(i, j, k), d;
          if (phi < -eps) d = 0.;
          else if (phi < eps) d = .5 / eps + .5 / eps * std::cos(pi * phi / eps);
          else d = 0.;
          del(i, j, k) = d;
        }
  }
  // sum(a(1:imax,1:jmax,1:kmax)) of the volume integral, exactly (XSum)
  double exact_sum_interior(const F3& a) {
    XSum s;
    for (int k = 1; k <= kmax; ++k)
      for (int j = 1; j <= jmax; ++j)
        for (int i = 1; i <= imax; ++i) s.add(a(i, j, k));
    return s.value();
  }
  double sum_interior(const F3& a) {  // sum(a(1:imax,1:jmax,1:kmax)), column order
    double s = 0.;
    for (int k = 1; k <= kmax; ++k)
      for (int j = 1; j <= jmax; ++j)
        for (int i = 1; i <= imax; ++i) s += a(i, j, k);
    return s;
  }

  // update_materials, average_method=0 (misc.f90:79-290)
  void update_materials() {
    for (int k = 0; k <= k1; ++k)
      for (int j = 0; j <= j1; ++j)
        for (int i = 0; i <= i1; ++i) {
          double s = lvset[0](i, j, k);
          if (L > 1) for (int l = 0; l < L; ++l) s = std::min(s, lvset[l](i, j, k));
          slset(i, j, k) = s;
        }
    for (int l = 0; l < L; ++l) heaviside_c(l, 1.5 * dz, hnew_mls[l]);
    jiemian.v = hnew_mls[0].v;
    if (L > 1)
      for (int l = 0; l < L; ++l)
        for (size_t n = 0; n < jiemian.size(); ++n) jiemian.v[n] = std::min(jiemian.v[n], hnew_mls[l].v[n]);
    for (size_t n = 0; n < miu.size(); ++n) miu.v[n] = c.miu1 * jiemian.v[n] + c.miu2 * (1. - jiemian.v[n]);
    F3 h_rho; shapeC(h_rho);
    F3 h_temp; shapeC(h_temp);
    for (int l = 0; l < L; ++l) {
      heaviside_c(l, 1.5 * dz, h_temp);
      double vol = exact_sum_interior(h_temp);  // misc.f90:127-133, order-free
      volume[l] = 1. - vol / ((1. * itot * jtot) * ktot);
      if (l == 0) h_rho.v = h_temp.v;
      else for (size_t n = 0; n < h_rho.size(); ++n) h_rho.v[n] = std::min(h_rho.v[n], h_temp.v[n]);
    }
    for (size_t n = 0; n < rho.size(); ++n) rho.v[n] = c.rho1 * h_rho.v[n] + c.rho2 * (1. - h_rho.v[n]);
    double sv = 0.;
    for (int l = 0; l < L; ++l) sv += volume[l];
    rho_avr = c.rho1 * (1. - sv) + c.rho2 * sv;
    if (c.rho1 == c.rho2) {
      rho_u.fill(c.rho1); rho_v.fill(c.rho1); rho_w.fill(c.rho1);
    } else {
#pragma omp parallel for
      for (int k = 1; k <= kmax; ++k)
        for (int j = 1; j <= jmax; ++j)
          for (int i = 1; i <= imax; ++i) {
            rho_u(i, j, k) = (rho(i, j, k) + rho(i + 1, j, k)) / 2.;
            rho_v(i, j, k) = (rho(i, j, k) + rho(i, j + 1, k)) / 2.;
            rho_w(i, j, k) = (rho(i, j, k) + rho(i, j, k + 1)) / 2.;
          }
    }
  }

  // average_vel_at_center (misc.f90:587-604)
  void average_vel_at_center() {
#pragma omp parallel for
    for (int k = 1; k <= kmax; ++k)
      for (int j = 1; j <= jmax; ++j)
        for (int i = 1; i <= imax; ++i) {
          uccnew(i, j, k) = (unew(i - 1, j, k) + unew(i, j, k)) / 2.;
          vccnew(i, j, k) = (vnew(i, j - 1, k) + vnew(i, j, k)) / 2.;
          wccnew(i, j, k) = (wnew(i, j, k - 1) + wnew(i, j, k)) / 2.;
        }
  }
  // disp_cg and disp_speed (write_vtk.f90:438-566) of drop l (0-based), one
  // rank: the centroid of the cells with lvset <= 1.5dz and their velocity
  // integral ucc dx dy dz (1 - hnew_mls) over lx ly lz init_volume(l)
  void disp(int l, double* cg, double* vel) {
    double counter = 0., xd = 0., yd = 0., zd = 0., ud = 0., vd = 0., wd = 0.;
    for (int k = 1; k <= kmax; ++k) {
      const double coorz = (k - 0.5) / dzi;
      for (int j = 1; j <= jmax; ++j) {
        const double coory = 0. + (j - 0.5) / dyi;
        for (int i = 1; i <= imax; ++i) {
          const double coorx = 0. + (i - 0.5) / dxi;
          if (lvset[l](i, j, k) <= 1.5 * dz) {
            counter = counter + 1.;
            xd = xd + coorx;
            yd = yd + coory;
            zd = zd + coorz;
            const double g = 1. - hnew_mls[l](i, j, k);
            ud = ud + uccnew(i, j, k) * dx * dy * dz * g;
            vd = vd + vccnew(i, j, k) * dx * dy * dz * g;
            wd = wd + wccnew(i, j, k) * dx * dy * dz * g;
          }
        }
      }
    }
    cg[0] = xd / counter;
    cg[1] = yd / counter;
    cg[2] = zd / counter;
    const double v0 = lx * ly * lz * init_volume[l];
    vel[0] = ud / v0;
    vel[1] = vd / v0;
    vel[2] = wd / v0;
  }

  // max_vel_at_center (misc.f90:610-636)
  double max_vel_at_center() {
    double m = 0; bool first = true;
    for (int k = 1; k <= kmax; ++k)
      for (int j = 1; j <= jmax; ++j)
        for (int i = 1; i <= imax; ++i) {
          double vm = std::sqrt((sq(uccnew(i, j, k)) + sq(vccnew(i, j, k))) + sq(wccnew(i, j, k)));
          if (first || vm > m) { m = vm; first = false; }
        }
    return m;
  }
  // average_stream_vel (misc.f90:642-655)
  double average_stream_vel() {
    double s = sum_interior(vnew);
    return s / (double)((long long)itot * jtot * kmax);
  }

  // ================================================== interface.f90
  // get_curvature (interface.f90:20-119)
  void get_curvature(const F3& phi, F3& curvature) {
    nrm_m.fill(1.); nrm_x.fill(0.); nrm_y.fill(0.); nrm_z.fill(0.);
    curvature.fill(0.);
    const double max_kappa = 1. / dz;
    const double lim = NB - 1. * dz;
#pragma omp parallel for
    for (int k = 1; k <= kmax; ++k)
      for (int j = 1; j <= jmax; ++j)
        for (int i = 1; i <= imax; ++i) {
          if (!(std::fabs(phi(i, j, k)) <= lim)) continue;
          double s27[27];
          int n = 0;
          for (int dk = -1; dk <= 1; ++dk)
            for (int dj = -1; dj <= 1; ++dj)
              for (int di = -1; di <= 1; ++di) s27[n++] = phi(i + di, j + dj, k + dk);
          double x[10];
          for (int r = 0; r < 10; ++r) {
            double s = 0.;
            for (int m = 0; m < 27; ++m) s = s + P[r][m] * s27[m];
            x[r] = s;
          }
          double dphidx = x[1], dphidy = x[2], dphidz = x[3];
          double d2phidx = x[4], d2phidy = x[5], d2phidz = x[6];
          double d2phidxdy = x[7], d2phidxdz = x[8], d2phidydz = x[9];
          double norm_val = std::sqrt((sq(dphidx) + sq(dphidy)) + sq(dphidz));
          nrm_m(i, j, k) = norm_val;
          nrm_x(i, j, k) = dphidx / norm_val;
          nrm_y(i, j, k) = dphidy / norm_val;
          nrm_z(i, j, k) = dphidz / norm_val;
          double cv;
          if (norm_val < 0.9) {
            cv = 0.;
          } else {
            double n3 = norm_val * norm_val * norm_val;
            double term1 = ((d2phidx + d2phidy) + d2phidz) / norm_val;
            double term2 = (dphidx * dphidx * d2phidx + dphidy * dphidy * d2phidy) + dphidz * dphidz * d2phidz;
            term2 = term2 / n3;
            double term3 = (dphidx * dphidy * d2phidxdy + dphidx * dphidz * d2phidxdz) + dphidy * dphidz * d2phidydz;
            term3 = 2. * term3 / n3;
            cv = -((term1 - term2) - term3);
          }
          if (cv < -max_kappa) cv = -max_kappa;
          else if (cv > max_kappa) cv = max_kappa;
          else if (std::fabs(cv) < 1e-9) cv = 0.;
          curvature(i, j, k) = cv;
        }
  }
  // re_curvature (interface.f90:186-218)
  void re_curvature(const F3& phi, const F3& curv, F3& re_curv) {
    re_curv.fill(0.);
#pragma omp parallel for
    for (int k = 1; k <= kmax; ++k)
      for (int j = 1; j <= jmax; ++j)
        for (int i = 1; i <= imax; ++i) {
          if (!(std::fabs(phi(i, j, k)) < 2. * dz)) continue;
          double s = 0.;
          int n = 0;
          for (int dk = -1; dk <= 1; ++dk)
            for (int dj = -1; dj <= 1; ++dj)
              for (int di = -1; di <= 1; ++di) s = s + P[0][n++] * curv(i + di, j + dj, k + dk);
          re_curv(i, j, k) = s;
        }
  }
  // icurvature, 3-D branch (interface.f90:126-179)
  double icurvature(int nb, const double ph[3], const double cv[3]) {
    double sp = 0.;
    if (cv[1] < 0.) sp = -1.;
    if (cv[1] > 0.) sp = 1.;
    double eps_0 = sp * ph[1];
    double eps_nb = sp * ph[1 + nb];
    if (c.TwoD) {
      if (cv[1] * cv[1 + nb] > 0.) {
        double r_0 = -1. / cv[1] + eps_0;
        double r_nb = -1. / cv[1 + nb] + eps_nb;
        double r_i = (r_0 + r_nb) / 2.;
        return -1. / r_i;
      }
      return 0.;
    }
    if (cv[1] * cv[1 + nb] > 0.) {
      double a1 = eps_nb * cv[1];
      double a2 = eps_0 * cv[1 + nb];
      return (a1 - a2) / (eps_nb - eps_0);
    }
    return 0.;
  }
  // ipot (interface.f90:225-277)
  void ipot() {
    std::vector<double> dtemp((size_t)L * L, 0.);
    std::fill(dmin.begin(), dmin.end(), 0.);
    const double cutoff = NB;
    for (int m = 0; m < L; ++m)
      for (int n = 0; n < L; ++n) {
        if (n == m) continue;
        double d1 = 1e3;
        const F3& pm = lvset[m]; const F3& pn = lvset[n];
        for (size_t q = 0; q < pm.size(); ++q) {
          double s = 1e3;
          if (pm.v[q] > -1. * dz && pm.v[q] < 1. * dz && pn.v[q] < cutoff) s = pm.v[q] + pn.v[q];
          if (s < d1) d1 = s;
        }
        dtemp[m + (size_t)L * n] = d1;
      }
    for (int m = 0; m < L - 1; ++m)
      for (int n = m + 1; n < L; ++n) dmin[m + (size_t)L * n] = 0.5 * (dtemp[m + (size_t)L * n] + dtemp[n + (size_t)L * m]);
  }

  // ================================================== hyperPDE.f90
  // HOUC5_nb (hyperPDE.f90:397-495) and WENO5_nb (503-800) over the band.
  void adv_rhs(int scheme, const F3& vu, const F3& vv, const F3& vw, const F3& phi, F3& dfdt) {
    dfdt.fill(0.);
    const int cnt = (int)nb_i.size();
#pragma omp parallel for
    for (int q = 0; q < cnt; ++q) {
      const int i = nb_i[q], j = nb_j[q], k = nb_k[q];
      double udfdx, vdfdy, wdfdz, dfx, dfy, dfz;
      if (scheme == ICLS_HOUC5) {
        if (c.TwoD) {
          udfdx = 0.;
        } else {
          if (vu(i, j, k) >= 0.)
            dfx = houc5_pos(phi(i - 3, j, k), phi(i - 2, j, k), phi(i - 1, j, k), phi(i, j, k), phi(i + 1, j, k), phi(i + 2, j, k));
          else
            dfx = houc5_neg(phi(i + 3, j, k), phi(i + 2, j, k), phi(i + 1, j, k), phi(i, j, k), phi(i - 1, j, k), phi(i - 2, j, k));
          udfdx = -(vu(i, j, k) * dfx / dx);
        }
        if (vv(i, j, k) >= 0.)
          dfy = houc5_pos(phi(i, j - 3, k), phi(i, j - 2, k), phi(i, j - 1, k), phi(i, j, k), phi(i, j + 1, k), phi(i, j + 2, k));
        else
          dfy = houc5_neg(phi(i, j + 3, k), phi(i, j + 2, k), phi(i, j + 1, k), phi(i, j, k), phi(i, j - 1, k), phi(i, j - 2, k));
        vdfdy = -(vv(i, j, k) * dfy / dy);
      } else {
        if (c.TwoD) {
          udfdx = 0.;
        } else {
          if (vu(i, j, k) >= 0.)
            dfx = weno5((phi(i - 2, j, k) - phi(i - 3, j, k)) / dx, (phi(i - 1, j, k) - phi(i - 2, j, k)) / dx,
                        (phi(i, j, k) - phi(i - 1, j, k)) / dx, (phi(i + 1, j, k) - phi(i, j, k)) / dx,
                        (phi(i + 2, j, k) - phi(i + 1, j, k)) / dx);
          else
            dfx = weno5((phi(i + 3, j, k) - phi(i + 2, j, k)) / dx, (phi(i + 2, j, k) - phi(i + 1, j, k)) / dx,
                        (phi(i + 1, j, k) - phi(i, j, k)) / dx, (phi(i, j, k) - phi(i - 1, j, k)) / dx,
                        (phi(i - 1, j, k) - phi(i - 2, j, k)) / dx);
          udfdx = -(vu(i, j, k) * dfx);
        }
        // y uses dx as in the reference (hyperPDE.f90:622-626)
        if (vv(i, j, k) >= 0.)
          dfy = weno5((phi(i, j - 2, k) - phi(i, j - 3, k)) / dx, (phi(i, j - 1, k) - phi(i, j - 2, k)) / dx,
                      (phi(i, j, k) - phi(i, j - 1, k)) / dx, (phi(i, j + 1, k) - phi(i, j, k)) / dx,
                      (phi(i, j + 2, k) - phi(i, j + 1, k)) / dx);
        else
          dfy = weno5((phi(i, j + 3, k) - phi(i, j + 2, k)) / dx, (phi(i, j + 2, k) - phi(i, j + 1, k)) / dx,
                      (phi(i, j + 1, k) - phi(i, j, k)) / dx, (phi(i, j, k) - phi(i, j - 1, k)) / dx,
                      (phi(i, j - 1, k) - phi(i, j - 2, k)) / dx);
        vdfdy = -(vv(i, j, k) * dfy);
      }
      // z: 5th order inside, HOUC3 at k=2,kmax-1, first order at walls
      if (k > 2 && k < kmax - 1) {
        if (scheme == ICLS_HOUC5) {
          if (vw(i, j, k) >= 0.)
            dfz = houc5_pos(phi(i, j, k - 3), phi(i, j, k - 2), phi(i, j, k - 1), phi(i, j, k), phi(i, j, k + 1), phi(i, j, k + 2));
          else
            dfz = houc5_neg(phi(i, j, k + 3), phi(i, j, k + 2), phi(i, j, k + 1), phi(i, j, k), phi(i, j, k - 1), phi(i, j, k - 2));
          wdfdz = -(vw(i, j, k) * dfz / dz);
        } else {
          if (vw(i, j, k) >= 0.)
            dfz = weno5((phi(i, j, k - 2) - phi(i, j, k - 3)) / dz, (phi(i, j, k - 1) - phi(i, j, k - 2)) / dz,
                        (phi(i, j, k) - phi(i, j, k - 1)) / dz, (phi(i, j, k + 1) - phi(i, j, k)) / dz,
                        (phi(i, j, k + 2) - phi(i, j, k + 1)) / dz);
          else
            dfz = weno5((phi(i, j, k + 3) - phi(i, j, k + 2)) / dz, (phi(i, j, k + 2) - phi(i, j, k + 1)) / dz,
                        (phi(i, j, k + 1) - phi(i, j, k)) / dz, (phi(i, j, k) - phi(i, j, k - 1)) / dz,
                        (phi(i, j, k - 1) - phi(i, j, k - 2)) / dz);
          wdfdz = -(vw(i, j, k) * dfz);
        }
      } else if (k == 2 || k == kmax - 1) {
        if (vw(i, j, k) >= 0.)
          dfz = (((1. / 6.) * phi(i, j, k - 2) - phi(i, j, k - 1)) + (1. / 2.) * phi(i, j, k)) + (1. / 3.) * phi(i, j, k + 1);
        else
          dfz = ((-((1. / 6.) * phi(i, j, k + 2)) + phi(i, j, k + 1)) - (1. / 2.) * phi(i, j, k)) - (1. / 3.) * phi(i, j, k - 1);
        wdfdz = -(vw(i, j, k) * dfz / dz);
      } else {
        if (vw(i, j, k) >= 0.) dfz = phi(i, j, k) - phi(i, j, k - 1);
        else dfz = phi(i, j, k + 1) - phi(i, j, k);
        wdfdz = -(vw(i, j, k) * dfz / dz);
      }
      dfdt(i, j, k) = (udfdx + vdfdy) + wdfdz;
    }
  }

  // RK_nb (levelset.f90:342-367): out = in everywhere, band += factor*dt*dfdt
  void rk_nb(F3& out, const F3& in, double factor, const F3& dfdt) {
    out.v = in.v;
    const int cnt = (int)nb_i.size();
    const double fdt = factor * dt;
    for (int q = 0; q < cnt; ++q) {
      const int i = nb_i[q], j = nb_j[q], k = nb_k[q];
      out(i, j, k) = in(i, j, k) + fdt * dfdt(i, j, k);
    }
    boundsls(out);
  }
  static void lincomb(F3& out, double a, const F3& x, double b, const F3& y) {
    for (size_t n = 0; n < out.size(); ++n) out.v[n] = a * x.v[n] + b * y.v[n];
  }
  // SSP-RK3 of ls_advection / inflation (levelset.f90:235-243, 558-565)
  void rk3_advect(int scheme, const F3& vu, const F3& vv, const F3& vw, const F3& phi0, F3& phi3) {
    F3 dfdt; shapeI(dfdt);
    F3 phi1, phi2, tmp; shapeL(phi1); shapeL(phi2); shapeL(tmp);
    adv_rhs(scheme, vu, vv, vw, phi0, dfdt);
    rk_nb(phi1, phi0, 1., dfdt);
    adv_rhs(scheme, vu, vv, vw, phi1, dfdt);
    lincomb(tmp, 3. / 4., phi0, 1. / 4., phi1);
    rk_nb(phi2, tmp, 1. / 4., dfdt);
    adv_rhs(scheme, vu, vv, vw, phi2, dfdt);
    lincomb(tmp, 1. / 3., phi0, 2. / 3., phi2);
    rk_nb(phi3, tmp, 2. / 3., dfdt);
  }

  // WENO5_deri (hyperPDE.f90:2932-3197) + WENO5_reinit (2646-2746)
  void weno5_reinit(const F3& sgn, const F3& phi, F3& RHS) {
    RHS.fill(0.);
    const double lim = NB + dz;
#pragma omp parallel for
    for (int k = 1; k <= kmax; ++k)
      for (int j = 1; j <= jmax; ++j)
        for (int i = 1; i <= imax; ++i) {
          if (!(std::fabs(phi(i, j, k)) < lim)) continue;
          double A = 0., B = 0., C, D, E, F;
          if (!c.TwoD) {
            A = weno5((phi(i - 2, j, k) - phi(i - 3, j, k)) / dx, (phi(i - 1, j, k) - phi(i - 2, j, k)) / dx,
                      (phi(i, j, k) - phi(i - 1, j, k)) / dx, (phi(i + 1, j, k) - phi(i, j, k)) / dx,
                      (phi(i + 2, j, k) - phi(i + 1, j, k)) / dx);
            B = weno5((phi(i + 3, j, k) - phi(i + 2, j, k)) / dx, (phi(i + 2, j, k) - phi(i + 1, j, k)) / dx,
                      (phi(i + 1, j, k) - phi(i, j, k)) / dx, (phi(i, j, k) - phi(i - 1, j, k)) / dx,
                      (phi(i - 1, j, k) - phi(i - 2, j, k)) / dx);
          }
          C = weno5((phi(i, j - 2, k) - phi(i, j - 3, k)) / dx, (phi(i, j - 1, k) - phi(i, j - 2, k)) / dx,
                    (phi(i, j, k) - phi(i, j - 1, k)) / dx, (phi(i, j + 1, k) - phi(i, j, k)) / dx,
                    (phi(i, j + 2, k) - phi(i, j + 1, k)) / dx);
          D = weno5((phi(i, j + 3, k) - phi(i, j + 2, k)) / dx, (phi(i, j + 2, k) - phi(i, j + 1, k)) / dx,
                    (phi(i, j + 1, k) - phi(i, j, k)) / dx, (phi(i, j, k) - phi(i, j - 1, k)) / dx,
                    (phi(i, j - 1, k) - phi(i, j - 2, k)) / dx);
          if (k >= 3 && k <= kmax - 2) {
            E = weno5((phi(i, j, k - 2) - phi(i, j, k - 3)) / dz, (phi(i, j, k - 1) - phi(i, j, k - 2)) / dz,
                      (phi(i, j, k) - phi(i, j, k - 1)) / dz, (phi(i, j, k + 1) - phi(i, j, k)) / dz,
                      (phi(i, j, k + 2) - phi(i, j, k + 1)) / dz);
            F = weno5((phi(i, j, k + 3) - phi(i, j, k + 2)) / dz, (phi(i, j, k + 2) - phi(i, j, k + 1)) / dz,
                      (phi(i, j, k + 1) - phi(i, j, k)) / dz, (phi(i, j, k) - phi(i, j, k - 1)) / dz,
                      (phi(i, j, k - 1) - phi(i, j, k - 2)) / dz);
          } else {
            E = (phi(i, j, k) - phi(i, j, k - 1)) / dz;
            F = (phi(i, j, k + 1) - phi(i, j, k)) / dz;
          }
          const double s = sgn(i, j, k);
          double dydx, dydy, dydz;
          if (c.TwoD) {
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
          RHS(i, j, k) = s * (1. - std::sqrt((sq(dydx) + sq(dydy)) + sq(dydz)));
        }
  }

  // ================================================== levelset.f90
  // tube_construction (levelset.f90:87-197)
  void tube_construction(int l) {
    F3& phi = lvset[l];
    for (size_t n = 0; n < phi.size(); ++n) {
      if (phi.v[n] > NB) phi.v[n] = NB;
      else if (phi.v[n] < -NB) phi.v[n] = -NB;
    }
    long long cnt = 0;
    for (int k = 1; k <= kmax; ++k)
      for (int j = 1; j <= jmax; ++j)
        for (int i = 1; i <= imax; ++i) {
          uint8_t m;
          if (std::fabs(phi(i, j, k)) < NB) {
            m = 1;
          } else {
            double xsum = 0., ysum = 0., zsum = 0.;
            for (int d = -2; d <= 2; ++d) xsum += std::fabs(phi(i + d, j, k)) - NB;
            for (int d = -2; d <= 2; ++d) ysum += std::fabs(phi(i, j + d, k)) - NB;
            for (int d = -2; d <= 2; ++d) zsum += std::fabs(phi(i, j, k + d)) - NB;
            m = (xsum == 0. && ysum == 0. && zsum == 0.) ? 0 : 1;
          }
          mask[(i - 1) + (size_t)imax * ((j - 1) + (size_t)jmax * (k - 1))] = m;
          cnt += m;
        }
    nb_cnt[l] = cnt;
    nb_i.clear(); nb_j.clear(); nb_k.clear();
    nb_i.reserve(cnt); nb_j.reserve(cnt); nb_k.reserve(cnt);
    for (int k = 1; k <= kmax; ++k)
      for (int j = 1; j <= jmax; ++j)
        for (int i = 1; i <= imax; ++i)
          if (mask[(i - 1) + (size_t)imax * ((j - 1) + (size_t)jmax * (k - 1))]) {
            nb_i.push_back(i); nb_j.push_back(j); nb_k.push_back(k);
          }
    boundsls(phi);
  }

  // ls_advection, RK3 branch (levelset.f90:208-335)
  void ls_advection(int l) {
    F3 phi3; shapeL(phi3);
    rk3_advect(c.ls_adv_space, uccnew, vccnew, wccnew, lvset[l], phi3);
    lvset[l].v.swap(phi3.v);
  }

  // inflation (levelset.f90:407-582)
  void inflation(int l) {
    const double s1 = 1.5 * dz;
    F3 delta, u_lc, v_lc, w_lc; shapeI(delta); shapeI(u_lc); shapeI(v_lc); shapeI(w_lc);
    F3 dheav, kappa; shapeC(dheav); shapeC(kappa);
    dheav.fill(1.);
    F3& phi = lvset[l];
    get_curvature(phi, kappa);
    boundc(kappa);
    dirac_trig(l, s1, delta);
    heaviside_c(l, s1, dheav);
    double temp, area;
    if (c.ispeed_dependence == ICLS_SPEED_UNFM) {
      double s = 0.;
      for (int k = 1; k <= kmax; ++k)
        for (int j = 1; j <= jmax; ++j)
          for (int i = 1; i <= imax; ++i) s += delta(i, j, k) * nrm_m(i, j, k);
      temp = s * dx * dy * dz;
    } else {
      double s = 0.;
      for (int k = 1; k <= kmax; ++k)
        for (int j = 1; j <= jmax; ++j)
          for (int i = 1; i <= imax; ++i) s += delta(i, j, k) * kappa(i, j, k) * nrm_m(i, j, k);
      temp = s * dx * dy * dz;
    }
    area = temp;
    if (c.TwoD) area = area / lx;
    temp = exact_sum_interior(dheav);  // levelset.f90:505-506, order-free
    volume[l] = 1. - temp / ((1. * itot * jtot) * ktot);
    double loss_rate = lx * ly * lz * (volume[l] - init_volume[l]) / ((double)c.inflate_step * dt);
    if (c.TwoD) loss_rate = loss_rate / lx;
    temp = loss_rate / area;
    maxchk_glb = temp / s1;
    boundp(dheav);
#pragma omp parallel for
    for (int k = 1; k <= kmax; ++k)
      for (int j = 1; j <= jmax; ++j)
        for (int i = 1; i <= imax; ++i) {
          u_l(i, j, k) = -(temp * (dheav(i + 1, j, k) - dheav(i, j, k)) / dx);
          v_l(i, j, k) = -(temp * (dheav(i, j + 1, k) - dheav(i, j, k)) / dy);
          w_l(i, j, k) = -(temp * (dheav(i, j, k + 1) - dheav(i, j, k)) / dz);
        }
    bounduvw(u_l, v_l, w_l);
    const bool curv = (c.ispeed_dependence == ICLS_SPEED_CURV);
#pragma omp parallel for
    for (int k = 1; k <= kmax; ++k)
      for (int j = 1; j <= jmax; ++j)
        for (int i = 1; i <= imax; ++i) {
          double a = (u_l(i - 1, j, k) + u_l(i, j, k)) / 2.;
          double b = (v_l(i, j - 1, k) + v_l(i, j, k)) / 2.;
          double cc = (w_l(i, j, k - 1) + w_l(i, j, k)) / 2.;
          if (curv) { a = a * kappa(i, j, k); b = b * kappa(i, j, k); cc = cc * kappa(i, j, k); }
          u_lc(i, j, k) = a; v_lc(i, j, k) = b; w_lc(i, j, k) = cc;
        }
    F3 phi3; shapeL(phi3);
    rk3_advect(c.i_space, u_lc, v_lc, w_lc, phi, phi3);
    if (c.mass_gain_one) gain_one(l, phi, phi3);
    phi.v.swap(phi3.v);
  }

  // icls_config.mass_gain_one (no counterpart in the reference): the
  // inflation moves the interface by about K/inflate_step times the volume
  // error it measured (K ~ 0.66/s1 in grid units), so with the option the
  // inflated level set phi1 is blended with the one before it,
  // phi = phi0 + g (phi1 - phi0), g = (V0 - V)/(V1 - V), V and V1 the exact
  // volumes before and after the inflation: the blend removes the measured
  // error V - V0 to first order in the (small) displacement
  void gain_one(int l, const F3& phi0, F3& phi1) {
    const double s1 = 1.5 * dz;
    lvset[l].v.swap(phi1.v);  // heaviside_c reads lvset[l]
    F3 h1; shapeC(h1);
    heaviside_c(l, s1, h1);
    lvset[l].v.swap(phi1.v);
    const double v1 = 1. - exact_sum_interior(h1) / ((1. * itot * jtot) * ktot);
    const double d = v1 - volume[l];
    const double g = d != 0. ? (init_volume[l] - volume[l]) / d : 0.;
    for (size_t n = 0; n < phi1.size(); ++n) phi1.v[n] = phi0.v[n] + g * (phi1.v[n] - phi0.v[n]);
    last_gain = g;
  }

  // ls_mass_correction (levelset.f90:377-400)
  void ls_mass_correction(int istep, int l) {
    maxchk_glb = 0.;
    if (istep % c.inflate_step == 0) {
      // the gain-one correction tests the drop's volume as it is now (after
      // this step's advection and reinitialisation); the reference, the
      // volume of the last update_materials
      double v = volume[l];
      if (c.mass_gain_one) {
        F3 h; shapeC(h);
        heaviside_c(l, 1.5 * dz, h);
        v = 1. - exact_sum_interior(h) / ((1. * itot * jtot) * ktot);
      }
      double massloss = (v - init_volume[l]) / init_volume[l];
      const double eps = c.mass_threshold > 0. ? c.mass_threshold : 1e-5;
      if (std::fabs(massloss) > eps) { inflation(l); ++last_inflated; }
    }
  }

  // ls_reinit, WENO5/RK3 branch (levelset.f90:619-882)
  void ls_reinit(int l, int maxiter, int& iter, double& residual) {
    F3 phi_0 = lvset[l];
    F3 phi_new = phi_0;
    F3 sgn; shapeI(sgn);
    for (int k = 1; k <= kmax; ++k)
      for (int j = 1; j <= jmax; ++j)
        for (int i = 1; i <= imax; ++i) {
          double p0 = phi_0(i, j, k);
          if (p0 < -dz) sgn(i, j, k) = -1.;
          else if (p0 > dz) sgn(i, j, k) = 1.;
          else sgn(i, j, k) = p0 / std::sqrt(p0 * p0 + dz * dz);
        }
    const double dtau = 0.5 * dz;
    F3 RHS, phi_n1, phi_n2; shapeL(RHS); shapeL(phi_n1); shapeL(phi_n2);
    iter = maxiter; residual = 0.;
    const double thr = dz * dz * dz * dz * dz;
    for (int it = 1; it <= maxiter; ++it) {
      weno5_reinit(sgn, phi_0, RHS);
      for (size_t n = 0; n < RHS.size(); ++n) phi_n1.v[n] = phi_0.v[n] + dtau * RHS.v[n];
      boundsls(phi_n1);
      weno5_reinit(sgn, phi_n1, RHS);
      for (size_t n = 0; n < RHS.size(); ++n)
        phi_n2.v[n] = 3. / 4. * phi_0.v[n] + 1. / 4. * (phi_n1.v[n] + dtau * RHS.v[n]);
      boundsls(phi_n2);
      weno5_reinit(sgn, phi_n2, RHS);
      for (size_t n = 0; n < RHS.size(); ++n)
        phi_new.v[n] = 1. / 3. * phi_0.v[n] + 2. / 3. * (phi_n2.v[n] + dtau * RHS.v[n]);
      boundsls(phi_new);
      double r = 0.;
      for (size_t n = 0; n < RHS.size(); ++n) r = std::max(r, std::fabs(phi_new.v[n] - phi_0.v[n]));
      residual = r;
      if (residual < thr) { iter = it; break; }
      iter = maxiter;
      phi_0.v = phi_new.v;
    }
    lvset[l].v = phi_new.v;
  }
  void ls_reinit_main(int istep, int l) {
    if (istep % c.reinit_step == 0) {
      ls_reinit(l, c.reinit_iter_max, reinit_iters, reinit_residual);
      boundsls(lvset[l]);
    }
  }
  // ls_main (levelset.f90:28-76)
  void ls_main(int istep) {
    last_inflated = 0;
    for (int l = 0; l < L; ++l) {
      tube_construction(l);
      ls_advection(l);
      // with the gain-one correction (no counterpart in the reference) the
      // correction follows the reinitialisation, so it also removes the
      // reinitialisation's volume change in the same step
      if (c.mass_gain_one && c.re_initialization) ls_reinit_main(istep, l);
      if (c.mass_correction) ls_mass_correction(istep, l);
      if (!c.mass_gain_one && c.re_initialization) ls_reinit_main(istep, l);
    }
    update_materials();
  }

  // ================================================== mom.f90, ab2.f90
  // CNTR2_conv + delta_diff + NS_grav -> mom_main (mom.f90:13-301)
  void mom_main(F3& RHSu, F3& RHSv, F3& RHSw) {
    const F3 &u = unew, &v = vnew, &w = wnew;
#pragma omp parallel for
    for (int k = 1; k <= kmax; ++k)
      for (int j = 1; j <= jmax; ++j)
        for (int i = 1; i <= imax; ++i) {
          const int ip = i + 1, jp = j + 1, kp = k + 1, im = i - 1, jm = j - 1, km = k - 1;
          // CNTR2_conv (mom.f90:67-130)
          double uuip = 0.25 * (u(ip, j, k) + u(i, j, k)) * (u(ip, j, k) + u(i, j, k));
          double uuim = 0.25 * (u(im, j, k) + u(i, j, k)) * (u(im, j, k) + u(i, j, k));
          double uvjp = 0.25 * (u(i, jp, k) + u(i, j, k)) * (v(ip, j, k) + v(i, j, k));
          double uvjm = 0.25 * (u(i, jm, k) + u(i, j, k)) * (v(ip, jm, k) + v(i, jm, k));
          double uwkp = 0.25 * (u(i, j, kp) + u(i, j, k)) * (w(ip, j, k) + w(i, j, k));
          double uwkm = 0.25 * (u(i, j, km) + u(i, j, k)) * (w(ip, j, km) + w(i, j, km));
          double RCu = ((-uuip + uuim) / dx + (-uvjp + uvjm) / dy) + (-uwkp + uwkm) / dz;
          double uvip = 0.25 * (u(i, j, k) + u(i, jp, k)) * (v(i, j, k) + v(ip, j, k));
          double uvim = 0.25 * (u(im, j, k) + u(im, jp, k)) * (v(i, j, k) + v(im, j, k));
          double vvjp = 0.25 * (v(i, j, k) + v(i, jp, k)) * (v(i, j, k) + v(i, jp, k));
          double vvjm = 0.25 * (v(i, j, k) + v(i, jm, k)) * (v(i, j, k) + v(i, jm, k));
          double wvkp = 0.25 * (w(i, j, k) + w(i, jp, k)) * (v(i, j, kp) + v(i, j, k));
          double wvkm = 0.25 * (w(i, j, km) + w(i, jp, km)) * (v(i, j, km) + v(i, j, k));
          double RCv = ((-uvip + uvim) / dx + (-vvjp + vvjm) / dy) + (-wvkp + wvkm) / dz;
          double uwip = 0.25 * (w(i, j, k) + w(ip, j, k)) * (u(i, j, k) + u(i, j, kp));
          double uwim = 0.25 * (w(i, j, k) + w(im, j, k)) * (u(im, j, k) + u(im, j, kp));
          double vwjp = 0.25 * (w(i, j, k) + w(i, jp, k)) * (v(i, j, k) + v(i, j, kp));
          double vwjm = 0.25 * (w(i, j, k) + w(i, jm, k)) * (v(i, jm, k) + v(i, jm, kp));
          double wwkp = 0.25 * (w(i, j, k) + w(i, j, kp)) * (w(i, j, k) + w(i, j, kp));
          double wwkm = 0.25 * (w(i, j, k) + w(i, j, km)) * (w(i, j, k) + w(i, j, km));
          double RCw = ((-uwip + uwim) / dx + (-vwjp + vwjm) / dy) + (-wwkp + wwkm) / dz;
          if (c.TwoD) RCu = 0.;
          // delta_diff (mom.f90:134-273)
          double dudxp, dudxm, dudyp, dudym, dudzp, dudzm, dvdxp, dvdxm, dvdyp, dvdym, dvdzp, dvdzm;
          double dwdxp, dwdxm, dwdyp, dwdym, dwdzp, dwdzm, ma1, ma2, ma3, ma4, ma5, ma6, ma7, ma8, ma9;
          double RD1, RD2, RD3, RD4, RD5;
          dudxp = (u(ip, j, k) - u(i, j, k)) / dx;
          dudxm = (u(i, j, k) - u(im, j, k)) / dx;
          dudyp = (u(i, jp, k) - u(i, j, k)) / dy;
          dudym = (u(i, j, k) - u(i, jm, k)) / dy;
          dvdxp = (v(ip, j, k) - v(i, j, k)) / dx;
          dvdxm = (v(ip, jm, k) - v(i, jm, k)) / dx;
          dudzp = (u(i, j, kp) - u(i, j, k)) / dz;
          dudzm = (u(i, j, k) - u(i, j, km)) / dz;
          dwdxp = (w(ip, j, k) - w(i, j, k)) / dx;
          dwdxm = (w(ip, j, km) - w(i, j, km)) / dx;
          ma1 = 0.25 * (((miu(i, j, k) + miu(i, jm, k)) + miu(ip, jm, k)) + miu(ip, j, k));
          ma2 = 0.25 * (((miu(i, j, k) + miu(i, jp, k)) + miu(ip, jp, k)) + miu(ip, j, k));
          ma3 = 0.25 * (((miu(i, j, k) + miu(i, j, km)) + miu(ip, j, km)) + miu(ip, j, k));
          ma4 = 0.25 * (((miu(i, j, k) + miu(i, j, kp)) + miu(ip, j, kp)) + miu(ip, j, k));
          RD1 = 2. * (dudxp * miu(ip, j, k) - dudxm * miu(i, j, k)) / dx;
          RD2 = (dudyp * ma2 - dudym * ma1) / dy;
          RD3 = (dvdxp * ma2 - dvdxm * ma1) / dy;
          RD4 = (dudzp * ma4 - dudzm * ma3) / dz;
          RD5 = (dwdxp * ma4 - dwdxm * ma3) / dz;
          double RDu = ((((RD1 + RD2) + RD3) + RD4) + RD5) / rho_u(i, j, k);
          dvdxp = (v(ip, j, k) - v(i, j, k)) / dx;
          dvdxm = (v(i, j, k) - v(im, j, k)) / dx;
          dudyp = (u(i, jp, k) - u(i, j, k)) / dy;
          dudym = (u(im, jp, k) - u(im, j, k)) / dy;
          dvdyp = (v(i, jp, k) - v(i, j, k)) / dy;
          dvdym = (v(i, j, k) - v(i, jm, k)) / dy;
          dvdzp = (v(i, j, kp) - v(i, j, k)) / dz;
          dvdzm = (v(i, j, k) - v(i, j, km)) / dz;
          dwdyp = (w(i, jp, k) - w(i, j, k)) / dy;
          dwdym = (w(i, jp, km) - w(i, j, km)) / dy;
          ma2 = 0.25 * (((miu(i, j, k) + miu(i, jp, k)) + miu(ip, jp, k)) + miu(ip, j, k));
          ma5 = 0.25 * (((miu(i, j, k) + miu(i, jp, k)) + miu(im, jp, k)) + miu(im, j, k));
          ma6 = 0.25 * (((miu(i, j, k) + miu(i, j, km)) + miu(i, jp, km)) + miu(i, jp, k));
          ma7 = 0.25 * (((miu(i, j, k) + miu(i, j, kp)) + miu(i, jp, kp)) + miu(i, jp, k));
          RD1 = (dvdxp * ma2 - dvdxm * ma5) / dx;
          RD2 = (dudyp * ma2 - dudym * ma5) / dx;
          RD3 = 2. * (dvdyp * miu(i, jp, k) - dvdym * miu(i, j, k)) / dy;
          RD4 = (dvdzp * ma7 - dvdzm * ma6) / dz;
          RD5 = (dwdyp * ma7 - dwdym * ma6) / dz;
          double RDv = ((((RD1 + RD2) + RD3) + RD4) + RD5) / rho_v(i, j, k);
          dwdxp = (w(ip, j, k) - w(i, j, k)) / dx;
          dwdxm = (w(i, j, k) - w(im, j, k)) / dx;
          dudzp = (u(i, j, kp) - u(i, j, k)) / dz;
          dudzm = (u(im, j, kp) - u(im, j, k)) / dz;
          dwdyp = (w(i, jp, k) - w(i, j, k)) / dy;
          dwdym = (w(i, j, k) - w(i, jm, k)) / dy;
          dvdzp = (v(i, j, kp) - v(i, j, k)) / dz;
          dvdzm = (v(i, jm, kp) - v(i, jm, k)) / dz;
          dwdzp = (w(i, j, kp) - w(i, j, k)) / dz;
          dwdzm = (w(i, j, k) - w(i, j, km)) / dz;
          ma4 = 0.25 * (((miu(i, j, k) + miu(i, j, kp)) + miu(ip, j, kp)) + miu(ip, j, k));
          ma8 = 0.25 * (((miu(i, j, k) + miu(i, j, kp)) + miu(im, j, kp)) + miu(im, j, k));
          ma7 = 0.25 * (((miu(i, j, k) + miu(i, j, kp)) + miu(i, jp, kp)) + miu(i, jp, k));
          ma9 = 0.25 * (((miu(i, j, k) + miu(i, j, kp)) + miu(i, jm, kp)) + miu(i, jm, k));
          RD1 = (dwdxp * ma4 - dwdxm * ma8) / dx;
          RD2 = (dudzp * ma4 - dudzm * ma8) / dx;
          RD3 = (dwdyp * ma7 - dwdym * ma9) / dy;
          RD4 = (dvdzp * ma7 - dvdzm * ma9) / dy;
          RD5 = 2. * (dwdzp * miu(i, j, kp) - dwdzm * miu(i, j, k)) / dz;
          double RDw = ((((RD1 + RD2) + RD3) + RD4) + RD5) / rho_w(i, j, k);
          if (c.TwoD) RDu = 0.;
          // NS_grav (mom.f90:277-301)
          double RGu = c.iFr * (1. - rho_avr / rho_u(i, j, k)) * c.g_unit[0];
          double RGv = c.iFr * (1. - rho_avr / rho_v(i, j, k)) * c.g_unit[1];
          double RGw = c.iFr * (1. - rho_avr / rho_w(i, j, k)) * c.g_unit[2];
          if (c.TwoD) RGu = 0.;
          RHSu(i, j, k) = (RCu + RDu * visc) + RGu;
          RHSv(i, j, k) = (RCv + RDv * visc) + RGv;
          RHSw(i, j, k) = (RCw + RDw * visc) + RGw;
        }
  }

  // ab2, GFM branch (ab2.f90:21-138) with momxp/yp/zp (mom.f90:779-851)
  void ab2() {
    F3 dunew, dvnew, dwnew; shapeI(dunew); shapeI(dvnew); shapeI(dwnew);
    mom_main(dunew, dvnew, dwnew);
#pragma omp parallel for
    for (int k = 1; k <= kmax; ++k)
      for (int j = 1; j <= jmax; ++j)
        for (int i = 1; i <= imax; ++i) {
          dudt(i, j, k) = unew(i, j, k) + dt * (1.5 * dunew(i, j, k) - 0.5 * duold(i, j, k));
          dvdt(i, j, k) = vnew(i, j, k) + dt * (1.5 * dvnew(i, j, k) - 0.5 * dvold(i, j, k));
          dwdt(i, j, k) = wnew(i, j, k) + dt * (1.5 * dwnew(i, j, k) - 0.5 * dwold(i, j, k));
        }
    duold.v = dunew.v; dvold.v = dvnew.v; dwold.v = dwnew.v;
    F3 phat, pjx, pjy, pjz; shapeC(phat); shapeC(pjx); shapeC(pjy); shapeC(pjz);
    for (size_t n = 0; n < phat.size(); ++n) {
      pjx.v[n] = 2. * p_x.v[n] - p_xold.v[n];
      pjy.v[n] = 2. * p_y.v[n] - p_yold.v[n];
      pjz.v[n] = 2. * p_z.v[n] - p_zold.v[n];
      phat.v[n] = 2. * pnew.v[n] - pold.v[n];
    }
#pragma omp parallel for
    for (int k = 1; k <= kmax; ++k)
      for (int j = 1; j <= jmax; ++j)
        for (int i = 1; i <= imax; ++i) {
          dunew(i, j, k) = -((1. / rho_u(i, j, k) - 1. / rho0) * dxi * ((phat(i + 1, j, k) - pjx(i, j, k)) - phat(i, j, k)));
          dvnew(i, j, k) = -((1. / rho_v(i, j, k) - 1. / rho0) * dyi * ((phat(i, j + 1, k) - pjy(i, j, k)) - phat(i, j, k)));
          dwnew(i, j, k) = -((1. / rho_w(i, j, k) - 1. / rho0) * dzi * ((phat(i, j, k + 1) - pjz(i, j, k)) - phat(i, j, k)));
        }
    forceytot = (bcy == ICLS_BCY_PERIODIC && c.constPoi) ? -12. * visc / (lz * lz) : 0.;  // ab2.f90:103-118
#pragma omp parallel for
    for (int k = 1; k <= kmax; ++k)
      for (int j = 1; j <= jmax; ++j)
        for (int i = 1; i <= imax; ++i) {
          dudt(i, j, k) = dudt(i, j, k) + dt * dunew(i, j, k);
          dvdt(i, j, k) = (dvdt(i, j, k) + dt * dvnew(i, j, k)) - forceytot * dt / rho_v(i, j, k);
          dwdt(i, j, k) = dwdt(i, j, k) + dt * dwnew(i, j, k);
        }
    bounduvw(dudt, dvdt, dwdt);
  }

  // fillps (fillps.f90:13-57) into p
  void fillps() {
    const double coef = rho0 / dt;
#pragma omp parallel for
    for (int k = 1; k <= kmax; ++k)
      for (int j = 1; j <= jmax; ++j)
        for (int i = 1; i <= imax; ++i) {
          double vel_x = (dudt(i, j, k) - dudt(i - 1, j, k)) * dxi;
          double vel_y = (dvdt(i, j, k) - dvdt(i, j - 1, k)) * dyi;
          double vel_z = (dwdt(i, j, k) - dwdt(i, j, k - 1)) * dzi;
          p(i, j, k) = coef * ((vel_x + vel_y) + vel_z);
        }
  }

  // gfm4p, surface_tension_method='GFM', NS_diff='del' (gfm.f90:17-267)
  void gfm4p() {
    // ipot (gfm.f90:57) only feeds the dmin diagnostic (main.f90:240); it is
    // evaluated on demand by ora_ipot, which changes no state.
    p_xold.v = p_x.v; p_yold.v = p_y.v; p_zold.v = p_z.v;
    p_jump.fill(0.); p_x.fill(0.); p_y.fill(0.); p_z.fill(0.);
    F3 re_curv; shapeC(re_curv);
    for (int l = 0; l < L; ++l) {
      const F3& ls = lvset[l];
      get_curvature(ls, curv_cmn);
      boundc(curv_cmn);
      if (!c.TwoD) {
        re_curvature(ls, curv_cmn, re_curv);
        curv_cmn.v = re_curv.v;
        boundc(curv_cmn);
      }
#pragma omp parallel for
      for (int k = 1; k <= kmax; ++k)
        for (int j = 1; j <= jmax; ++j)
          for (int i = 1; i <= imax; ++i) {
            if (!(std::fabs(ls(i, j, k)) <= 2. * dz)) continue;
            double jp_x[3] = {0., 0., 0.}, jp_y[3] = {0., 0., 0.}, jp_z[3] = {0., 0., 0.};
            double px = 0., py = 0., pz = 0.;
            double ph[3], cv[3];
            for (int nx = -1; nx <= 1; nx += 2) {
              for (int d = -1; d <= 1; ++d) { ph[d + 1] = ls(i + d, j, k); cv[d + 1] = curv_cmn(i + d, j, k); }
              if (ph[1] * ph[1 + nx] < 0.) {
                double icurv = icurvature(nx, ph, cv);
                jp_x[nx + 1] = nondi * (-icurv);
                if (nx == 1) px = jp_x[nx + 1];
              }
            }
            double jump_x = (jp_x[0] + jp_x[1]) + jp_x[2];
            for (int ny = -1; ny <= 1; ny += 2) {
              for (int d = -1; d <= 1; ++d) { ph[d + 1] = ls(i, j + d, k); cv[d + 1] = curv_cmn(i, j + d, k); }
              if (ph[1] * ph[1 + ny] < 0.) {
                double icurv = icurvature(ny, ph, cv);
                jp_y[ny + 1] = nondi * (-icurv);
                if (ny == 1) py = jp_y[ny + 1];
              }
            }
            double jump_y = (jp_y[0] + jp_y[1]) + jp_y[2];
            for (int nz = -1; nz <= 1; nz += 2) {
              for (int d = -1; d <= 1; ++d) { ph[d + 1] = ls(i, j, k + d); cv[d + 1] = curv_cmn(i, j, k + d); }
              if (ph[1] * ph[1 + nz] < 0.) {
                double icurv = icurvature(nz, ph, cv);
                jp_z[nz + 1] = nondi * (-icurv);
                if (nz == 1) pz = jp_z[nz + 1];
              }
            }
            double jump_z = (jp_z[0] + jp_z[1]) + jp_z[2];
            double pj;
            const double lv = ls(i, j, k);
            if (lv > 0.) {
              pj = (jump_x / (dx * dx) + jump_y / (dy * dy)) + jump_z / (dz * dz);
            } else if (lv < 0.) {
              pj = -((jump_x / (dx * dx) + jump_y / (dy * dy)) + jump_z / (dz * dz));
              px = -px; py = -py; pz = -pz;
            } else {
              pj = 0.; px = 0.; py = 0.; pz = 0.;
            }
            if (l == 0) {
              p_jump(i, j, k) = pj; p_x(i, j, k) = px; p_y(i, j, k) = py; p_z(i, j, k) = pz;
            } else {
              p_jump(i, j, k) = p_jump(i, j, k) + pj;
              p_x(i, j, k) = p_x(i, j, k) + px;
              p_y(i, j, k) = p_y(i, j, k) + py;
              p_z(i, j, k) = p_z(i, j, k) + pz;
            }
          }
    }
  }

  void add_pjump() { for (size_t n = 0; n < p.size(); ++n) p.v[n] = p.v[n] + p_jump.v[n]; }

  // solver2d (solver.f90:68-196) on p(1:imax,1:jmax,1:kmax)
  void solver2d() {
    // forward x
#pragma omp parallel for
    for (int k = 1; k <= kmax; ++k) {
      std::vector<double> line(imax);
      for (int j = 1; j <= jmax; ++j) {
        for (int i = 1; i <= imax; ++i) line[i - 1] = p(i, j, k);
        rfftf_line(imax, line.data());
        for (int i = 1; i <= imax; ++i) p(i, j, k) = line[i - 1];
      }
    }
    // forward y
#pragma omp parallel for
    for (int k = 1; k <= kmax; ++k) {
      std::vector<double> line(jmax);
      for (int i = 1; i <= imax; ++i) {
        for (int j = 1; j <= jmax; ++j) line[j - 1] = p(i, j, k);
        rfftf_line(jmax, line.data());
        for (int j = 1; j <= jmax; ++j) p(i, j, k) = line[j - 1];
      }
    }
    // Gauss elimination in z (solver.f90:119-160)
#pragma omp parallel for
    for (int j = 1; j <= jmax; ++j) {
      std::vector<double> d(kmax + 1);
      for (int i = 1; i <= imax; ++i) {
        const double xy = xyrt[(i - 1) + (size_t)imax * (j - 1)];
        double z = 1. / (tb[1] + xy);
        d[1] = tc[1] * z;
        p(i, j, 1) = p(i, j, 1) * z;
        for (int k = 2; k <= kmax - 1; ++k) {
          double bb = tb[k] + xy;
          z = 1. / (bb - ta[k] * d[k - 1]);
          d[k] = tc[k] * z;
          p(i, j, k) = (p(i, j, k) - ta[k] * p(i, j, k - 1)) * z;
        }
        double bb = tb[kmax] + xy;
        z = bb - ta[kmax] * d[kmax - 1];
        if (z != 0.) p(i, j, kmax) = (p(i, j, kmax) - ta[kmax] * p(i, j, kmax - 1)) / z;
        else p(i, j, kmax) = 0.;
        for (int k = kmax - 1; k >= 1; --k) p(i, j, k) = p(i, j, k) - d[k] * p(i, j, k + 1);
      }
    }
    // backward y
#pragma omp parallel for
    for (int k = 1; k <= kmax; ++k) {
      std::vector<double> line(jmax);
      for (int i = 1; i <= imax; ++i) {
        for (int j = 1; j <= jmax; ++j) line[j - 1] = p(i, j, k);
        rfftb_line(jmax, line.data());
        for (int j = 1; j <= jmax; ++j) p(i, j, k) = line[j - 1];
      }
    }
    // backward x
#pragma omp parallel for
    for (int k = 1; k <= kmax; ++k) {
      std::vector<double> line(imax);
      for (int j = 1; j <= jmax; ++j) {
        for (int i = 1; i <= imax; ++i) line[i - 1] = p(i, j, k);
        rfftb_line(imax, line.data());
        for (int i = 1; i <= imax; ++i) p(i, j, k) = line[i - 1];
      }
    }
  }

  // solver2d_cos (solver.f90:202-317) on p(1:imax,1:jmax,1:kmax): real FFT
  // in x, VCOSQB in z, Gauss elimination in y with diagonal b(j)+xzrt(i,k),
  // VCOSQF in z, inverse FFT in x
  void solver2d_cos() {
#pragma omp parallel for
    for (int k = 1; k <= kmax; ++k) {
      std::vector<double> line(imax);
      for (int j = 1; j <= jmax; ++j) {
        for (int i = 1; i <= imax; ++i) line[i - 1] = p(i, j, k);
        rfftf_line(imax, line.data());
        for (int i = 1; i <= imax; ++i) p(i, j, k) = line[i - 1];
      }
    }
#pragma omp parallel for
    for (int j = 1; j <= jmax; ++j) {
      std::vector<double> line(kmax);
      for (int i = 1; i <= imax; ++i) {
        for (int k = 1; k <= kmax; ++k) line[k - 1] = p(i, j, k);
        cosqb_line(kmax, line.data());
        for (int k = 1; k <= kmax; ++k) p(i, j, k) = line[k - 1];
      }
    }
    // Gauss elimination in y (solver.f90:245-283)
#pragma omp parallel for
    for (int k = 1; k <= kmax; ++k) {
      std::vector<double> d(jtot + 1);
      for (int i = 1; i <= imax; ++i) {
        const double xz = xzrt[(i - 1) + (size_t)imax * (k - 1)];
        double z = 1. / (tb[1] + xz);
        d[1] = tc[1] * z;
        p(i, 1, k) = p(i, 1, k) * z;
        for (int j = 2; j <= jtot - 1; ++j) {
          double bb = tb[j] + xz;
          z = 1. / (bb - ta[j] * d[j - 1]);
          d[j] = tc[j] * z;
          p(i, j, k) = (p(i, j, k) - ta[j] * p(i, j - 1, k)) * z;
        }
        double bb = tb[jtot] + xz;
        z = bb - ta[jtot] * d[jtot - 1];
        if (z != 0.) p(i, jtot, k) = (p(i, jtot, k) - ta[jtot] * p(i, jtot - 1, k)) / z;
        else p(i, jtot, k) = 0.;
        for (int j = jtot - 1; j >= 1; --j) p(i, j, k) = p(i, j, k) - d[j] * p(i, j + 1, k);
      }
    }
#pragma omp parallel for
    for (int j = 1; j <= jmax; ++j) {
      std::vector<double> line(kmax);
      for (int i = 1; i <= imax; ++i) {
        for (int k = 1; k <= kmax; ++k) line[k - 1] = p(i, j, k);
        cosqf_line(kmax, line.data());
        for (int k = 1; k <= kmax; ++k) p(i, j, k) = line[k - 1];
      }
    }
#pragma omp parallel for
    for (int k = 1; k <= kmax; ++k) {
      std::vector<double> line(imax);
      for (int j = 1; j <= jmax; ++j) {
        for (int i = 1; i <= imax; ++i) line[i - 1] = p(i, j, k);
        rfftb_line(imax, line.data());
        for (int i = 1; i <= imax; ++i) p(i, j, k) = line[i - 1];
      }
    }
  }
  // the pressure solve main.f90 selects by BC_in_y (main.f90:147-153)
  void pressure_solve() {
    if (bcy == ICLS_BCY_PERIODIC) solver2d();
    else solver2d_cos();
  }

  // correc (correc.f90:15-44)
  void correc() {
#pragma omp parallel for
    for (int k = 1; k <= kmax; ++k)
      for (int j = 1; j <= jmax; ++j)
        for (int i = 1; i <= imax; ++i) {
          unew(i, j, k) = dudt(i, j, k) - dt * dxi * ((p(i + 1, j, k) - p(i, j, k)) - p_x(i, j, k)) / rho0;
          vnew(i, j, k) = dvdt(i, j, k) - dt * dyi * ((p(i, j + 1, k) - p(i, j, k)) - p_y(i, j, k)) / rho0;
          wnew(i, j, k) = dwdt(i, j, k) - dt * dzi * ((p(i, j, k + 1) - p(i, j, k)) - p_z(i, j, k)) / rho0;
        }
  }

  // pressure update and normalisation, BC_in_y='Periodic' (main.f90:164-185)
  void pressure_update(int istep, int begin) {
    pold.v = pnew.v;
    pnew.v = p.v;
    boundp(pnew);
    if (bcy != ICLS_BCY_PERIODIC && bcy != ICLS_BCY_WALLS) return;  // main.f90:169-185
    const int k = 1;
    double norm = 0.;
    for (int i = 0; i <= i1; ++i) {
      double s = 0.;
      for (int j = 0; j <= j1; ++j) s += pnew(i, j, k);
      norm += s;
    }
    norm = norm / (1. * itot * jtot);
    for (size_t n = 0; n < pnew.size(); ++n) pnew.v[n] = pnew.v[n] - norm;
    if (istep == begin + 1) {
      for (size_t n = 0; n < pold.size(); ++n) pold.v[n] = pold.v[n] - norm;
    } else {
      for (size_t n = 0; n < pold.size(); ++n) pold.v[n] = (pold.v[n] + norm_old) - norm;
    }
    norm_old = norm;
  }

  // chkdiv (chkdiv.f90:10-90)
  int chkdiv(int istep, double* divtot_out, double* divmax_out, int* ijk) {
    double divmax = 0., divtot = 0.;
    int im = 0, jm = 0, km = 0;
    for (int k = 1; k <= kmax; ++k)
      for (int j = 1; j <= jmax; ++j)
        for (int i = 1; i <= imax; ++i) {
          double div = ((wnew(i, j, k) - wnew(i, j, k - 1)) * dzi + (vnew(i, j, k) - vnew(i, j - 1, k)) * dyi) +
                       (unew(i, j, k) - unew(i - 1, j, k)) * dxi;
          divtot = divtot + div;
          div = std::fabs(div);
          if (div > divmax) { divmax = div; im = i; jm = j; km = k; }
        }
    if (divtot_out) *divtot_out = divtot;
    if (divmax_out) *divmax_out = divmax;
    if (ijk) { ijk[0] = im; ijk[1] = jm; ijk[2] = km; }
    if (divmax > 1e-12 && istep != 0) return ICLS_E_DIVERGENCE;
    return ICLS_OK;
  }

  // chkdt (chkdt.f90:11-105)
  double chkdt() {
    double u_max = 0., v_max = 0., w_max = 0.;
    for (int k = 1; k <= k1; ++k)
      for (int j = 1; j <= j1; ++j)
        for (int i = 1; i <= i1; ++i) {
          u_max = std::max(u_max, std::fabs((unew(i, j, k) + unew(i - 1, j, k)) / 2.));
          v_max = std::max(v_max, std::fabs((vnew(i, j, k) + vnew(i, j - 1, k)) / 2.));
          w_max = std::max(w_max, std::fabs((wnew(i, j, k) + wnew(i, j, k - 1)) / 2.));
        }
    double speed_conv = (u_max / dx + v_max / dy) + w_max / dz;
    const double* g = c.g_unit;
    double g1 = std::fabs(c.iFr * (1. - rho_avr / c.rho1) * g[0]);
    double g2 = std::fabs(c.iFr * (1. - rho_avr / c.rho2) * g[0]);
    double g3 = std::fabs(c.iFr * (1. - rho_avr / c.rho1) * g[1]);
    double g4 = std::fabs(c.iFr * (1. - rho_avr / c.rho2) * g[1]);
    double g5 = std::fabs(c.iFr * (1. - rho_avr / c.rho1) * g[2]);
    double g6 = std::fabs(c.iFr * (1. - rho_avr / c.rho2) * g[2]);
    double g_max = std::max(std::max(std::max(g1, g2), std::max(g3, g4)), std::max(g5, g6));
    double h_min = std::min(std::min(dx, dy), dz);
    double speed_grav = std::sqrt(g_max / h_min);
    double v1 = std::max(c.miu1 / c.rho1, c.miu2 / c.rho2) * visc;
    double v2 = (2. / (dx * dx) + 2. / (dy * dy)) + 2. / (dz * dz);
    double speed_visc = v1 * v2;
    double curv_max = c.TwoD ? 1. / h_min : 2. / h_min;
    double speed_surf = std::sqrt(curv_max / (c.We * rho0 * (h_min * h_min)));
    double s1 = speed_conv + speed_visc;
    double speed = (s1 + std::sqrt((s1 * s1 + 4. * (speed_grav * speed_grav)) + 4. * (speed_surf * speed_surf))) / 2.;
    return 0.5 / speed;
  }

  // init_program, begin=0, GFM (init.f90:22-117)
  int init_program() {
    init_matrix();
    initsolver();
    dt = c.timestep;
    time = 0.;
    bounduvw(unew, vnew, wnew);
    bounduvw(dudt, dvdt, dwdt);
    boundmls();
    boundp(pnew);
    average_vel_at_center();
    update_materials();
    init_volume = volume;
    mom_main(duold, dvold, dwold);
    pold.v = pnew.v;
    p_xold.v = p_x.v; p_yold.v = p_y.v; p_zold.v = p_z.v;
    initialised = true;
    return ICLS_OK;
  }

  // one main-loop iteration (main.f90:103-210)
  int step(int istep, int begin) {
    time = time + dt;
    if (c.solveLS) ls_main(istep);
    v_bulk = average_stream_vel();
    ab2();
    fillps();
    if (c.solveLS) { gfm4p(); add_pjump(); }
    pressure_solve();
    boundp(p);
    correc();
    bounduvw(unew, vnew, wnew);
    pressure_update(istep, begin);
    average_vel_at_center();
    if (std::isnan(vnew(1, 1, 1))) return ICLS_E_NAN;
    if (c.ioutchk > 0 && istep % c.ioutchk == 0) {
      int rc = chkdiv(istep, nullptr, nullptr, nullptr);
      if (rc) return rc;
      dt = c.timestep;
    }
    return ICLS_OK;
  }
};

// ============================================================= C API ====
extern "C" {

int ora_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

int ora_create(const icls_config* cfg, ora_ctx** out) {
  if (!cfg || !out) return ICLS_E_ARG;
  ora_ctx* o = new ora_ctx();
  int rc = o->setup(cfg);
  if (rc) { delete o; return rc; }
  *out = o;
  return ICLS_OK;
}
int ora_destroy(ora_ctx* o) { delete o; return ICLS_OK; }

int ora_field_bounds(const ora_ctx* o, int id, int lo[3], int hi[3]) {
  F3* f = const_cast<ora_ctx*>(o)->field(id, 1);
  if (!f) return ICLS_E_ARG;
  lo[0] = f->l0; lo[1] = f->l1; lo[2] = f->l2;
  hi[0] = f->l0 + f->n0 - 1; hi[1] = f->l1 + f->n1 - 1; hi[2] = f->l2 + f->n2 - 1;
  return ICLS_OK;
}
int ora_upload_field(ora_ctx* o, int id, int l, const double* h) {
  F3* f = o->field(id, l);
  if (!f || !h) return ICLS_E_ARG;
  std::memcpy(f->v.data(), h, f->size() * sizeof(double));
  return ICLS_OK;
}
int ora_download_field(ora_ctx* o, int id, int l, double* h) {
  F3* f = o->field(id, l);
  if (!f || !h) return ICLS_E_ARG;
  std::memcpy(h, f->v.data(), f->size() * sizeof(double));
  return ICLS_OK;
}
int ora_get_scalars(ora_ctx* o, icls_scalars* s) {
  s->time = o->time; s->dt = o->dt; s->rho_avr = o->rho_avr; s->v_bulk = o->v_bulk;
  s->norm_old = o->norm_old; s->maxchk_glb = o->maxchk_glb;
  s->reinit_residual = o->reinit_residual; s->reinit_iters = o->reinit_iters;
  s->last_inflated = o->last_inflated;
  return ICLS_OK;
}
int ora_set_dt(ora_ctx* o, double dt) { o->dt = dt; return ICLS_OK; }
// the exact sum of n doubles (XSum), for the tests of its contract
double ora_exact_sum(const double* x, long long n) {
  XSum s;
  for (long long q = 0; q < n; ++q) s.add(x[q]);
  return s.value();
}

int ora_get_volumes(ora_ctx* o, double* v, double* v0) {
  for (int l = 0; l < o->L; ++l) { if (v) v[l] = o->volume[l]; if (v0) v0[l] = o->init_volume[l]; }
  return ICLS_OK;
}
int ora_get_pseudo_inv(ora_ctx* o, double* P) {
  o->init_matrix();
  for (int r = 0; r < 10; ++r) for (int n = 0; n < 27; ++n) P[r * 27 + n] = o->P[r][n];
  return ICLS_OK;
}

int ora_init_program(ora_ctx* o) { return o->init_program(); }
#define NEED_INIT if (!o->initialised) return ICLS_E_STATE
#define LCHK if (l < 1 || l > o->L) return ICLS_E_ARG
int ora_ls_main(ora_ctx* o, int istep) { NEED_INIT; o->ls_main(istep); return ICLS_OK; }
int ora_average_stream_vel(ora_ctx* o, double* vb) { NEED_INIT; o->v_bulk = o->average_stream_vel(); if (vb) *vb = o->v_bulk; return ICLS_OK; }
int ora_ab2(ora_ctx* o) { NEED_INIT; o->ab2(); return ICLS_OK; }
int ora_fillps(ora_ctx* o) { NEED_INIT; o->fillps(); return ICLS_OK; }
int ora_gfm4p(ora_ctx* o) { NEED_INIT; o->gfm4p(); return ICLS_OK; }
int ora_add_pjump(ora_ctx* o) { NEED_INIT; o->add_pjump(); return ICLS_OK; }
int ora_solver2d(ora_ctx* o) { NEED_INIT; o->pressure_solve(); return ICLS_OK; }
int ora_set_inflow(ora_ctx* o, const double* v) {
  if (!o || !v) return ICLS_E_ARG;
  std::memcpy(o->v_inflow.data(), v, o->v_inflow.size() * sizeof(double));
  return ICLS_OK;
}
int ora_boundp(ora_ctx* o, int id) {
  F3* f = o->field(id, 1);
  if (!f || f->l0 != 0) return ICLS_E_ARG;
  o->boundp(*f);
  return ICLS_OK;
}
int ora_correc(ora_ctx* o) { NEED_INIT; o->correc(); return ICLS_OK; }
int ora_bounduvw(ora_ctx* o, int id) {
  if (id == ICLS_F_U) o->bounduvw(o->unew, o->vnew, o->wnew);
  else if (id == ICLS_F_DUDT) o->bounduvw(o->dudt, o->dvdt, o->dwdt);
  else return ICLS_E_ARG;
  return ICLS_OK;
}
int ora_pressure_update(ora_ctx* o, int istep, int begin) { NEED_INIT; o->pressure_update(istep, begin); return ICLS_OK; }
int ora_average_vel_at_center(ora_ctx* o) { o->average_vel_at_center(); return ICLS_OK; }
int ora_max_vel_at_center(ora_ctx* o, double* vm) { *vm = o->max_vel_at_center(); return ICLS_OK; }
int ora_disp(ora_ctx* o, int l, double* cg, double* vel) {
  if (!o || !cg || !vel || l < 1 || l > o->L) return ICLS_E_ARG;
  o->disp(l - 1, cg, vel);
  return ICLS_OK;
}
int ora_chkdiv(ora_ctx* o, int istep, double* dt_, double* dm, int ijk[3]) { return o->chkdiv(istep, dt_, dm, ijk); }
int ora_chkdt(ora_ctx* o, double* dtmax) { *dtmax = o->chkdt(); return ICLS_OK; }
int ora_ipot(ora_ctx* o, double* dmin) {
  o->ipot();
  if (dmin) for (size_t q = 0; q < o->dmin.size(); ++q) dmin[q] = o->dmin[q];
  return ICLS_OK;
}
int ora_step(ora_ctx* o, int istep, int begin) { NEED_INIT; return o->step(istep, begin); }
// the plane i = const of a field: out(j,k), j fastest
int ora_download_plane_x(ora_ctx* o, int id, int l, int i, double* out) {
  F3* f = o->field(id, l);
  if (!f || !out) return ICLS_E_ARG;
  if (i < f->l0 || i > f->l0 + f->n0 - 1) return ICLS_E_ARG;
  size_t q = 0;
  for (int k = f->l2; k < f->l2 + f->n2; ++k)
    for (int j = f->l1; j < f->l1 + f->n1; ++j) out[q++] = (*f)(i, j, k);
  return ICLS_OK;
}
// timestep.txt record (main.f90:243-256)
int ora_timestep_record(ora_ctx* o, int istep, double rec[6]) {
  double massloss = 0.;
  for (int l = 0; l < o->L; ++l) massloss = massloss + (1. - o->volume[l] / o->init_volume[l]);
  double quck = 0.;
  if (o->L >= 2) {
    o->ipot();
    quck = o->dmin[0 + (size_t)o->L * 1] / o->dz;
  }
  rec[0] = 1. * istep; rec[1] = o->time; rec[2] = o->dt;
  rec[3] = massloss; rec[4] = quck; rec[5] = o->maxchk_glb;
  return ICLS_OK;
}
int ora_tube_construction(ora_ctx* o, int l) { LCHK; o->tube_construction(l - 1); return ICLS_OK; }
int ora_ls_advection(ora_ctx* o, int l) { NEED_INIT; LCHK; o->ls_advection(l - 1); return ICLS_OK; }
int ora_ls_mass_correction(ora_ctx* o, int istep, int l) { NEED_INIT; LCHK; o->ls_mass_correction(istep, l - 1); return ICLS_OK; }
int ora_ls_reinit_main(ora_ctx* o, int istep, int l) { NEED_INIT; LCHK; o->ls_reinit_main(istep, l - 1); return ICLS_OK; }
int ora_update_materials(ora_ctx* o) { o->update_materials(); return ICLS_OK; }
int ora_get_curvature(ora_ctx* o, int l) {
  NEED_INIT; LCHK;
  o->get_curvature(o->lvset[l - 1], o->curv_cmn);
  o->boundc(o->curv_cmn);
  return ICLS_OK;
}
int ora_band_count(ora_ctx* o, int l, long long* n) { LCHK; *n = o->nb_cnt[l - 1]; return ICLS_OK; }

int ora_vrfftf(int m, int n, double* r) {
  for (int s = 0; s < m; ++s) rfftf_line(n, r + (size_t)s * n);
  return ICLS_OK;
}
int ora_vrfftb(int m, int n, double* r) {
  for (int s = 0; s < m; ++s) rfftb_line(n, r + (size_t)s * n);
  return ICLS_OK;
}
int ora_vcosqf(int m, int n, double* r) {
  for (int l = 0; l < m; ++l) cosqf_line(n, r + (size_t)l * n);
  return ICLS_OK;
}
int ora_vcosqb(int m, int n, double* r) {
  for (int l = 0; l < m; ++l) cosqb_line(n, r + (size_t)l * n);
  return ICLS_OK;
}

// 'drp' / 'mdp' initial level sets (init.f90:717-753, 901-984): signed
// distance to the sphere, with the periodic images in y then x taken on
// the positive side.
int ora_init_drops(const icls_config* cfg, int ndrop, const double* xc, const double* yc,
                   const double* zc, const double* radius, double* out) {
  const int i1 = cfg->itot + 1, j1 = cfg->jtot + 1, k1 = cfg->ktot + 1;
  const double dxi = cfg->itot / cfg->lx, dyi = cfg->jtot / cfg->ly, dzi = cfg->ktot / cfg->lz;
  const size_t n0 = i1 + 5, n1 = j1 + 5, n2 = k1 + 5;
  for (int l = 0; l < ndrop; ++l) {
    double* o = out + (size_t)l * n0 * n1 * n2;
    for (int k = -2; k <= k1 + 2; ++k) {
      double coorz = (k - 0.5) / dzi;
      for (int j = -2; j <= j1 + 2; ++j) {
        double coory = (j - 0.5) / dyi;
        for (int i = -2; i <= i1 + 2; ++i) {
          double coorx = (i - 0.5) / dxi;
          double ph = std::sqrt((sq(coorx - xc[l]) + sq(coory - yc[l])) + sq(coorz - zc[l])) - radius[l];
          double p1 = std::sqrt((sq(coorx - xc[l]) + sq(coory - yc[l] - cfg->ly)) + sq(coorz - zc[l])) - radius[l];
          if (ph > 0.) ph = std::min(ph, p1);
          double p2 = std::sqrt((sq(coorx - xc[l] - cfg->lx) + sq(coory - yc[l])) + sq(coorz - zc[l])) - radius[l];
          if (ph > 0.) ph = std::min(ph, p2);
          o[(size_t)(i + 2) + n0 * ((size_t)(j + 2) + n1 * (size_t)(k + 2))] = ph;
        }
      }
    }
  }
  return ICLS_OK;
}

}  // extern "C"

// ---------------------------------------------------- checkpoint / restart
// loadflds (loadd.f90:28-103): u, v, w, pnew, lvset(1..L), jiemian over the
// interior, FP64, i fastest, then (time, nr, dt); path.hist: the AB2 and
// pressure history, the normalisation mean and the initial volumes (the
// same layout as the CUDA library writes)
namespace {
// whole arrays: the AB2 and pressure history, then the level sets with the
// ghost layers boundsls leaves untouched (k = -2, -1, k1+1, k1+2)
std::vector<std::pair<int, int>> ora_hist_fields(int L) {
  std::vector<std::pair<int, int>> f;
  for (int id : {ICLS_F_DUOLD, ICLS_F_DVOLD, ICLS_F_DWOLD, ICLS_F_POLD, ICLS_F_PX, ICLS_F_PY, ICLS_F_PZ,
                 ICLS_F_PXOLD, ICLS_F_PYOLD, ICLS_F_PZOLD})
    f.push_back({id, 1});
  for (int l = 1; l <= L; ++l) f.push_back({ICLS_F_LVSET, l});
  return f;
}
struct OraShape {
  int lo[3], hi[3];
  size_t n() const { return (size_t)(hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1); }
  size_t at(int i, int j, int k) const {
    return (size_t)(i - lo[0]) + (size_t)(hi[0] - lo[0] + 1) * ((size_t)(j - lo[1]) + (size_t)(hi[1] - lo[1] + 1) * (k - lo[2]));
  }
};
std::vector<std::pair<int, int>> ora_ck_fields(int L) {
  std::vector<std::pair<int, int>> f = {{ICLS_F_U, 1}, {ICLS_F_V, 1}, {ICLS_F_W, 1}, {ICLS_F_PNEW, 1}};
  for (int l = 1; l <= L; ++l) f.push_back({ICLS_F_LVSET, l});
  f.push_back({ICLS_F_JIEMIAN, 1});
  return f;
}
}  // namespace

int ora_write_checkpoint(ora_ctx* o, const char* path, int nr, int history) {
  if (!o || !path) return ICLS_E_ARG;
  const int I = o->imax, J = o->jmax, K = o->kmax;
  std::vector<double> full, in((size_t)I * J * K);
  FILE* f = std::fopen(path, "wb");
  if (!f) return ICLS_E_IO;
  bool ok = true;
  for (const auto& fl : ora_ck_fields(o->L)) {
    OraShape sh;
    ora_field_bounds(o, fl.first, sh.lo, sh.hi);
    full.assign(sh.n(), 0.);
    ora_download_field(o, fl.first, fl.second, full.data());
    size_t q = 0;
    for (int k = 1; k <= K; ++k)
      for (int j = 1; j <= J; ++j)
        for (int i = 1; i <= I; ++i) in[q++] = full[sh.at(i, j, k)];
    ok = ok && std::fwrite(in.data(), sizeof(double), in.size(), f) == in.size();
  }
  const double info[3] = {o->time, 1. * nr, o->dt};
  ok = ok && std::fwrite(info, sizeof(double), 3, f) == 3;
  if (std::fclose(f) != 0) ok = false;
  if (!ok) return ICLS_E_IO;
  if (!history) return ICLS_OK;
  f = std::fopen((std::string(path) + ".hist").c_str(), "wb");
  if (!f) return ICLS_E_IO;
  const char magic[8] = {'I', 'C', 'L', 'S', 'H', 'S', 'T', '1'};
  const int dims[4] = {I, J, K, o->L};
  ok = std::fwrite(magic, 1, 8, f) == 8 && std::fwrite(dims, sizeof(int), 4, f) == 4;
  for (const auto& fl : ora_hist_fields(o->L)) {
    OraShape sh;
    ora_field_bounds(o, fl.first, sh.lo, sh.hi);
    full.assign(sh.n(), 0.);
    ora_download_field(o, fl.first, fl.second, full.data());
    ok = ok && std::fwrite(full.data(), sizeof(double), full.size(), f) == full.size();
  }
  ok = ok && std::fwrite(&o->norm_old, sizeof(double), 1, f) == 1 &&
       std::fwrite(o->init_volume.data(), sizeof(double), (size_t)o->L, f) == (size_t)o->L;
  if (std::fclose(f) != 0) ok = false;
  return ok ? ICLS_OK : ICLS_E_IO;
}

int ora_read_checkpoint(ora_ctx* o, const char* path, int* nr) {
  if (!o || !path) return ICLS_E_ARG;
  const int I = o->imax, J = o->jmax, K = o->kmax;
  std::vector<double> full, in((size_t)I * J * K);
  FILE* f = std::fopen(path, "rb");
  if (!f) return ICLS_E_IO;
  bool ok = true;
  for (const auto& fl : ora_ck_fields(o->L)) {
    ok = ok && std::fread(in.data(), sizeof(double), in.size(), f) == in.size();
    if (!ok) break;
    OraShape sh;
    ora_field_bounds(o, fl.first, sh.lo, sh.hi);
    full.assign(sh.n(), 0.);
    size_t q = 0;
    for (int k = 1; k <= K; ++k)
      for (int j = 1; j <= J; ++j)
        for (int i = 1; i <= I; ++i) full[sh.at(i, j, k)] = in[q++];
    ora_upload_field(o, fl.first, fl.second, full.data());
  }
  double info[3] = {0., 0., 0.};
  ok = ok && std::fread(info, sizeof(double), 3, f) == 3;
  std::fclose(f);
  if (!ok) return ICLS_E_IO;
  int rc = ora_init_program(o);
  if (rc) return rc;
  o->time = info[0];
  o->dt = info[2];
  if (nr) *nr = (int)info[1];
  f = std::fopen((std::string(path) + ".hist").c_str(), "rb");
  if (!f) return ICLS_OK;
  char magic[8];
  int dims[4];
  ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "ICLSHST1", 8) == 0 &&
       std::fread(dims, sizeof(int), 4, f) == 4 && dims[0] == I && dims[1] == J && dims[2] == K && dims[3] == o->L;
  for (const auto& fl : ora_hist_fields(o->L)) {
    if (!ok) break;
    OraShape sh;
    ora_field_bounds(o, fl.first, sh.lo, sh.hi);
    full.assign(sh.n(), 0.);
    ok = std::fread(full.data(), sizeof(double), full.size(), f) == full.size();
    if (ok) ora_upload_field(o, fl.first, fl.second, full.data());
  }
  std::vector<double> v0((size_t)o->L);
  double norm = 0.;
  ok = ok && std::fread(&norm, sizeof(double), 1, f) == 1 && std::fread(v0.data(), sizeof(double), v0.size(), f) == v0.size();
  std::fclose(f);
  if (!ok) return ICLS_E_IO;
  o->norm_old = norm;
  o->init_volume = v0;
  return ICLS_OK;
}
