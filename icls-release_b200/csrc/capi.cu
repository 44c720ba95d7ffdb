// capi.cu — the extern "C" entry points of include/icls_gpu.h and the host
// orchestration of the ICLS time step on one B200.
//
// Each entry point replaces one subroutine of GeZhouyang/ICLS-release that
// src/main.f90 calls (cited at the function), enqueuing its kernels on the
// context's stream.  Host-side decisions that the reference takes on
// globally reduced scalars (the mass-correction trigger, the divergence
// abort, the NaN stop) read those scalars back; the reinitialisation early
// exit is decided on the device.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "ctx.h"

using namespace icls;

namespace icls {
// init_matrix (init.f90:1587-1723): pseudo_inv_A = (A^T A)^-1 A^T of the
// quadratic least-squares fit on the 27-point stencil; inverted by
// Gauss-Jordan in long double.
// the 10x27 least-squares pseudo-inverse of init.f90:1587-1723 for spacings
// (dx, dy, dz), into out[r*27 + n]
void pseudo_inverse(double dx, double dy, double dz, double* out) {
  long double A[27][10];
  int row = 0;
  for (int dzs = -1; dzs <= 1; ++dzs)
    for (int dys = -1; dys <= 1; ++dys)
      for (int dxs = -1; dxs <= 1; ++dxs) {
        long double a2 = (long double)(dx * dxs), a3 = (long double)(dy * dys), a4 = (long double)(dz * dzs);
        long double* r = A[row++];
        r[0] = 1; r[1] = a2; r[2] = a3; r[3] = a4;
        r[4] = 0.5L * a2 * a2; r[5] = 0.5L * a3 * a3; r[6] = 0.5L * a4 * a4;
        r[7] = a2 * a3; r[8] = a2 * a4; r[9] = a3 * a4;
      }
  long double M[10][20];
  for (int r = 0; r < 10; ++r)
    for (int q = 0; q < 10; ++q) {
      long double s = 0;
      for (int n = 0; n < 27; ++n) s += A[n][r] * A[n][q];
      M[r][q] = s;
      M[r][10 + q] = (r == q) ? 1 : 0;
    }
  for (int col = 0; col < 10; ++col) {
    int piv = col;
    for (int r = col + 1; r < 10; ++r)
      if (fabsl(M[r][col]) > fabsl(M[piv][col])) piv = r;
    if (piv != col)
      for (int q = 0; q < 20; ++q) std::swap(M[col][q], M[piv][q]);
    const long double d = M[col][col];
    for (int q = 0; q < 20; ++q) M[col][q] /= d;
    for (int r = 0; r < 10; ++r) {
      if (r == col) continue;
      const long double f = M[r][col];
      if (f != 0)
        for (int q = 0; q < 20; ++q) M[r][q] -= f * M[col][q];
    }
  }
  for (int r = 0; r < 10; ++r)
    for (int n = 0; n < 27; ++n) {
      long double s = 0;
      for (int q = 0; q < 10; ++q) s += M[r][10 + q] * A[n][q];
      out[r * 27 + n] = (double)s;
    }
}

}  // namespace icls

struct icls_ctx {
  Ctx c;
};

namespace {

#define CK(x)                                  \
  do {                                         \
    cudaError_t e_ = (x);                      \
    if (e_ != cudaSuccess) return ICLS_E_CUDA; \
  } while (0)


constexpr long long kMaxFieldElems = 1LL << 30;

int validate(const icls_config* c) {
  if (!c) return ICLS_E_ARG;
  if (c->bc_y < ICLS_BCY_PERIODIC || c->bc_y > ICLS_BCY_OUTOUT) return ICLS_E_CONFIG;
  if (c->ns_conv == ICLS_NS_WENO5) return ICLS_E_UNSUPPORTED;  // boundfu stops (bound.f90:310-322)
  if (c->ns_conv != ICLS_NS_CNTR2) return ICLS_E_CONFIG;
  if (!fft_length_ok(c->itot, false, c->itot)) return ICLS_E_CONFIG;  // FFT length in x
  if (c->bc_y == ICLS_BCY_PERIODIC && !fft_length_ok(c->jtot, true, c->itot)) return ICLS_E_CONFIG;
  if (c->bc_y != ICLS_BCY_PERIODIC && c->ktot > kCosqMaxN) return ICLS_E_CONFIG;  // z cosine lines
  if (c->itot > 4096 || c->jtot > 4096) return ICLS_E_CONFIG;
  if (c->itot < 8 || c->jtot < 8) return ICLS_E_CONFIG;  // periodic images of 3 halo layers
  if (c->itot % 2) return ICLS_E_CONFIG;  // (implied by the FFT lengths) the predictor copies column pairs
  if (c->ktot < 6 || c->lmax < 1) return ICLS_E_CONFIG;
  // grid-stride loops index cells with 32-bit integers: keep the largest
  // array (a level set with its 3 halo layers per side) below 2^30 elements
  // so that no index plus one grid stride can pass INT_MAX
  if ((long long)(c->itot + 6) * (c->jtot + 6) * (c->ktot + 6) > kMaxFieldElems) return ICLS_E_CONFIG;
  if (!(c->lx > 0 && c->ly > 0 && c->lz > 0 && c->timestep > 0)) return ICLS_E_CONFIG;
  if (c->reinit_step < 1 || c->inflate_step < 1 || c->reinit_iter_max < 1) return ICLS_E_CONFIG;
  if (!(c->mass_threshold >= 0.)) return ICLS_E_CONFIG;
  if (c->mass_gain_one != 0 && c->mass_gain_one != 1) return ICLS_E_CONFIG;
  if (c->ls_adv_space != ICLS_HOUC5 && c->ls_adv_space != ICLS_WENO5) return ICLS_E_CONFIG;
  if (c->i_space != ICLS_HOUC5 && c->i_space != ICLS_WENO5) return ICLS_E_CONFIG;
  if (c->precision != ICLS_FP64 && c->precision != ICLS_FP32) return ICLS_E_CONFIG;
  if (c->curvature_model != ICLS_CURV_STENCIL && c->curvature_model != ICLS_CURV_MLP) return ICLS_E_CONFIG;
  if (c->curvature_model == ICLS_CURV_MLP) {
    // the network reads the stencil in units of one isotropic spacing
    const double dx = c->lx / c->itot, dy = c->ly / c->jtot, dz = c->lz / c->ktot;
    if (dx != dy || dx != dz) return ICLS_E_UNSUPPORTED;
    if (!(c->mlp_fallback_tol > 0.)) return ICLS_E_CONFIG;
  }
  return ICLS_OK;
}

void fill_params(Ctx& c) {
  const icls_config& f = c.cfg;
  Params& P = c.P;
  P.imax = f.itot; P.jmax = f.jtot; P.kmax = f.ktot;
  P.i1 = P.imax + 1; P.j1 = P.jmax + 1; P.k1 = P.kmax + 1;
  P.L = f.lmax;
  P.nCx = P.imax + 2; P.nCy = P.jmax + 2; P.nCz = P.kmax + 2;
  P.nLx = P.imax + 6; P.nLy = P.jmax + 6; P.nLz = P.kmax + 6;
  P.nC = (long long)P.nCx * P.nCy * P.nCz;
  P.nI = (long long)P.imax * P.jmax * P.kmax;
  P.nL = (long long)P.nLx * P.nLy * P.nLz;
  P.lx = f.lx; P.ly = f.ly; P.lz = f.lz;
  // param.f90:37-41
  P.dxi = f.itot / f.lx; P.dyi = f.jtot / f.ly; P.dzi = f.ktot / f.lz;
  P.dx = 1. / P.dxi; P.dy = 1. / P.dyi; P.dz = 1. / P.dzi;
  P.rdx = 1. / P.dx; P.rdy = 1. / P.dy; P.rdz = 1. / P.dz;
  {
    int e;
    P.pow2 = (std::frexp(P.dx, &e) == 0.5 && std::frexp(P.dy, &e) == 0.5 && std::frexp(P.dz, &e) == 0.5) ? 1 : 0;
  }
  P.NB = 6. * P.dz;
  P.pi = std::acos(-1.);
  P.dt = f.timestep;
  P.rho1 = f.rho1; P.rho2 = f.rho2; P.miu1 = f.miu1; P.miu2 = f.miu2;
  P.rho0 = std::min(f.rho1, f.rho2);  // param.f90:63
  P.rrho0 = 1. / P.rho0;
  {
    int e2;
    P.rho0_pow2 = std::frexp(P.rho0, &e2) == 0.5 ? 1 : 0;
  }
  P.f32 = f.precision == ICLS_FP32 ? 1 : 0;
  P.visc = 1. / f.Re;                 // param.f90:73
  P.iFr = f.iFr;
  P.nondi = 1. / f.We;                // gfm.f90:40
  P.g1 = f.g_unit[0]; P.g2 = f.g_unit[1]; P.g3 = f.g_unit[2];
  P.v_lower = f.v_wall_lower; P.v_upper = f.v_wall_upper;
  P.bcy = f.bc_y;
  // ab2.f90:103-118: the driving gradient only with periodic y
  P.forceytot = (f.bc_y == ICLS_BCY_PERIODIC && f.constPoi) ? -12. * P.visc / (f.lz * f.lz) : 0.;
  P.TwoD = f.TwoD;
  P.ls_adv_space = f.ls_adv_space; P.i_space = f.i_space;
  P.ispeed_curv = (f.ispeed_dependence == ICLS_SPEED_CURV);
}

void init_matrix(Ctx& c) { pseudo_inverse(c.P.dx, c.P.dy, c.P.dz, c.P10x27); }

template <typename T>
int dalloc(T** p, size_t n) {
  if (cudaMalloc((void**)p, n * sizeof(T) + 16) != cudaSuccess) return ICLS_E_NOMEM;
  if (cudaMemset(*p, 0, n * sizeof(T) + 16) != cudaSuccess) return ICLS_E_CUDA;
  return ICLS_OK;
}

#define AL(ptr, n)                  \
  do {                              \
    int rc_ = dalloc(&(ptr), (n));  \
    if (rc_) return rc_;            \
  } while (0)

// doubles that hold n elements of the form's field type
size_t tn(const Params& P, long long n) { return P.f32 ? (size_t)(n + 1) / 2 : (size_t)n; }

int allocate(Ctx& c) {
  const Params& P = c.P;
  // FP64 in both forms: the Poisson work array and the Laplacian of the
  // jumps (the solve's right-hand side)
  for (double** f : {&c.p, &c.pjump}) AL(*f, (size_t)P.nC);
  // the form's field type, the pressures and face jumps included: the FP32
  // momentum and correction stencils read them (the jumps are assembled in
  // FP64 and stored in the field type)
  for (double** f : {&c.u, &c.v, &c.w, &c.dudt, &c.dvdt, &c.dwdt, &c.miu, &c.rho, &c.jiemian, &c.curv, &c.dheav,
                     &c.kappa, &c.pnew, &c.pold, &c.px, &c.py, &c.pz, &c.pxold, &c.pyold, &c.pzold})
    AL(*f, tn(P, P.nC));
  for (int h = 0; h < 2; ++h) {
    AL(c.duold[h], tn(P, P.nI)); AL(c.dvold[h], tn(P, P.nI)); AL(c.dwold[h], tn(P, P.nI));
  }
  for (double** f : {&c.rho_u, &c.rho_v, &c.rho_w, &c.ucc, &c.vcc, &c.wcc, &c.nrm_m, &c.ulc, &c.vlc, &c.wlc})
    AL(*f, tn(P, P.nI));
  c.lv.assign(P.L, nullptr);
  for (int l = 0; l < P.L; ++l) AL(c.lv[l], tn(P, P.nL));
  if (P.f32) AL(c.stage, (size_t)P.nL);
  AL(c.d_nbcnt, (size_t)P.L);
  AL(c.spec, (size_t)P.nI);
  AL(c.twx, (size_t)P.imax);
  AL(c.twy, (size_t)std::max(P.jmax, P.kmax));  // y twiddles, or z twiddles of solver2d_cos
  if (P.bcy == ICLS_BCY_PERIODIC) {
    AL(c.xyrt, (size_t)P.imax * P.jmax);
    AL(c.zpiv, (size_t)(P.imax / 2 + 1) * (P.jmax / 2 + 1) * P.kmax);  // pivots per distinct (xrt, yrt)
    AL(c.tri_a, (size_t)P.kmax + 1); AL(c.tri_b, (size_t)P.kmax + 1); AL(c.tri_c, (size_t)P.kmax + 1);
  } else {
    AL(c.xyrt, (size_t)(P.imax / 2 + 1) * P.kmax);                      // distinct xzrt
    AL(c.zpiv, (size_t)(P.imax / 2 + 1) * P.kmax * P.jmax);             // pivots per distinct (xrt, zrt)
    AL(c.tri_a, (size_t)P.jmax + 1); AL(c.tri_b, (size_t)P.jmax + 1); AL(c.tri_c, (size_t)P.jmax + 1);
    AL(c.cosb, (size_t)P.kmax * P.kmax); AL(c.cosf, (size_t)P.kmax * P.kmax);
    AL(c.czw, (size_t)P.kmax);
  }
  AL(c.vin, (size_t)(P.i1 + 1) * (P.k1 + 1));
  AL(c.partials, (size_t)kRedBlocks * std::max(P.L, 4) + (size_t)P.imax + 8);
  AL(c.diag, (size_t)7 * kRedBlocks + 8);
  AL(c.lpartials, (size_t)kRedBlocks);
  AL(c.dsc, 1);
  AL(c.dvol, (size_t)P.L); AL(c.dvol0, (size_t)P.L); AL(c.dmaxchk, (size_t)P.L);
  AL(c.dvolnow, (size_t)P.L);
  // band list of the advection stages: up to one entry per interior cell
  c.band_cap = P.nI;
  if (cudaMalloc(&c.band_list, (size_t)c.band_cap * 8) != cudaSuccess) return ICLS_E_NOMEM;
  if (cudaMalloc((void**)&c.band_count, sizeof(int)) != cudaSuccess) return ICLS_E_NOMEM;
  AL(c.drs, (size_t)P.L);
  c.red_cap = ((P.imax + TBX - 1) / TBX) * ((P.jmax + TBY - 1) / TBY);
  c.hcap = c.red_cap * ((P.kmax + 2 + kHeavRows - 1) / kHeavRows);
  // per-(tile, chunk) exact sums of H (4 words each) for every drop; the
  // inflation uses red_cap area sums and red_cap exact sums
  AL(c.hpart, std::max((size_t)4 * P.L * c.hcap, (size_t)5 * c.red_cap));
  CK(cudaMallocHost((void**)&c.h_vol, sizeof(double) * P.L));
  CK(cudaMallocHost((void**)&c.h_volnow, sizeof(double) * P.L));
  CK(cudaMallocHost((void**)&c.h_sc, sizeof(DevScalars)));
  CK(cudaEventCreateWithFlags(&c.ev_vol, cudaEventDisableTiming));
  // normal%m = 1 outside the curvature band (interface.f90:44)
  launch_fill(c, c.nrm_m, P.nI, 1.0, true);
  AL(c.d_bbox, (size_t)10 * P.L);
  CK(cudaMallocHost((void**)&c.h_bbox, sizeof(int) * 10 * P.L));
  CK(cudaEventCreateWithFlags(&c.ev_bbox, cudaEventDisableTiming));
  c.win.assign(P.L, DropWin());
  for (auto& w : c.win) w.box = w.valid = full_region(P);
  c.outside.assign(P.L, 0.);
  // ICLS_FULL_SWEEP=1 sweeps every drop's whole array (a check of the box
  // bookkeeping: both give bit-identical fields)
  const char* fs = std::getenv("ICLS_FULL_SWEEP");
  c.use_boxes = (P.L <= kMaxDropsParam) && !(fs && fs[0] == '1');
  // Alternative kernels of the same arithmetic (bit-identical fields), kept
  // for comparison:
  // ICLS_AB2=tma: the FP64 predictor on the TMA-fed kernel in place of the
  // cp.async-ring one (the ring kernel measured faster at 256^3, 1.37 vs
  // 1.68 ms);
  // ICLS_ADV=band: the advection stages after tube_construction as the
  // band-list split (measured no faster in FP64, slower in FP32, with the
  // list build included);
  // ICLS_CORREC=shapec: the fused correction one thread per shape-C cell
  // in place of one per interior cell writing the images;
  // ICLS_MATERIALS=rows1: the materials one row per thread, not two.
  const char* ab = std::getenv("ICLS_AB2");
  c.ab2_ring = !(ab && std::strcmp(ab, "tma") == 0);
  const char* cv = std::getenv("ICLS_CORREC");
  c.correc_shapec = cv && std::strcmp(cv, "shapec") == 0;
  const char* mv = std::getenv("ICLS_MATERIALS");
  c.materials_rows1 = mv && std::strcmp(mv, "rows1") == 0;
  const char* av = std::getenv("ICLS_ADV");
  c.adv_column = !(av && std::strcmp(av, "band") == 0);
  // working buffers of a group of drops: as many drops as half the free
  // HBM holds (ICLS_GROUP=n caps the group, e.g. to test the grouped path)
  {
    const size_t per = sizeof(double) * (3 * tn(P, P.nL) + 2 * tn(P, P.nC)) + (size_t)P.nI + 64;
    size_t freeb = 0, totalb = 0;
    CK(cudaMemGetInfo(&freeb, &totalb));
    long long G = (long long)((freeb / 2) / per);
    const char* gs = std::getenv("ICLS_GROUP");
    if (gs && std::atoi(gs) > 0) G = std::min<long long>(G, std::atoi(gs));
    G = std::max(1LL, std::min<long long>(G, P.L));
    c.mem.assign((size_t)G, Ctx::Member());
    for (Ctx::Member& m : c.mem) {
      AL(m.s1, tn(P, P.nL)); AL(m.s2, tn(P, P.nL)); AL(m.s3, tn(P, P.nL));
      AL(m.fit, tn(P, P.nC)); AL(m.cv, tn(P, P.nC));
      AL(m.mask, (size_t)P.nI);
    }
  }
  if (c.cfg.curvature_model == ICLS_CURV_MLP) {
    const int rc = mlp_buffers(c, (int)std::min<long long>(P.nI, 1LL << 21));
    if (rc) return rc;
  }
  c.inflated.assign(P.L, 0);
  c.vol_dirty.assign(P.L, 0);
  c.init_volume_h.assign(P.L, 0.);
  return ICLS_OK;
}

void release(Ctx& c) {
  for (double* f : {c.u, c.v, c.w, c.pnew, c.pold, c.p, c.dudt, c.dvdt, c.dwdt, c.px, c.py, c.pz, c.pxold,
                    c.pyold, c.pzold, c.pjump, c.miu, c.rho, c.jiemian, c.curv, c.dheav, c.kappa,
                    c.rho_u, c.rho_v, c.rho_w, c.ucc, c.vcc, c.wcc, c.nrm_m, c.ulc, c.vlc, c.wlc, c.spec,
                    c.xyrt, c.zpiv, c.tri_a, c.tri_b, c.tri_c, c.partials, c.diag, c.dvol, c.dvol0, c.dmaxchk, c.dvolnow,
                    c.hpart, c.cosb, c.cosf, c.vin})
    if (f) cudaFree(f);
  for (int h = 0; h < 2; ++h) {
    if (c.duold[h]) cudaFree(c.duold[h]);
    if (c.dvold[h]) cudaFree(c.dvold[h]);
    if (c.dwold[h]) cudaFree(c.dwold[h]);
  }
  for (double* f : c.lv) if (f) cudaFree(f);
  for (Ctx::Member& m : c.mem) {
    for (double* f : {m.s1, m.s2, m.s3, m.fit, m.cv}) if (f) cudaFree(f);
    if (m.mask) cudaFree(m.mask);
  }
  if (c.d_nbcnt) cudaFree(c.d_nbcnt);
  if (c.twx) cudaFree(c.twx);
  if (c.twy) cudaFree(c.twy);
  if (c.czw) cudaFree(c.czw);
  if (c.lpartials) cudaFree(c.lpartials);
  if (c.drs) cudaFree(c.drs);
  if (c.stage) cudaFree(c.stage);
  for (void* f : {(void*)c.mlp_X, c.mlp_rec, (void*)c.mlp_count, (void*)c.mlp_stats})
    if (f) cudaFree(f);
  if (c.dsc) cudaFree(c.dsc);
  if (c.h_vol) cudaFreeHost(c.h_vol);
  if (c.h_volnow) cudaFreeHost(c.h_volnow);
  if (c.band_list) cudaFree(c.band_list);
  if (c.band_count) cudaFree(c.band_count);
  if (c.h_sc) cudaFreeHost(c.h_sc);
  if (c.ev_vol) cudaEventDestroy(c.ev_vol);
  if (c.d_bbox) cudaFree(c.d_bbox);
  if (c.h_bbox) cudaFreeHost(c.h_bbox);
  if (c.ev_bbox) cudaEventDestroy(c.ev_bbox);
  c.prof.release();
  if (c.s) cudaStreamDestroy(c.s);
}

// field table: device pointer and element count
double* field_ptr(Ctx& c, int id, int l, long long* n) {
  const Params& P = c.P;
  *n = P.nC;
  switch (id) {
    case ICLS_F_U: return c.u; case ICLS_F_V: return c.v; case ICLS_F_W: return c.w;
    case ICLS_F_PNEW: return c.pnew; case ICLS_F_POLD: return c.pold; case ICLS_F_P: return c.p;
    case ICLS_F_DUDT: return c.dudt; case ICLS_F_DVDT: return c.dvdt; case ICLS_F_DWDT: return c.dwdt;
    case ICLS_F_PX: return c.px; case ICLS_F_PY: return c.py; case ICLS_F_PZ: return c.pz;
    case ICLS_F_PXOLD: return c.pxold; case ICLS_F_PYOLD: return c.pyold; case ICLS_F_PZOLD: return c.pzold;
    case ICLS_F_PJUMP: return c.pjump; case ICLS_F_MIU: return c.miu; case ICLS_F_RHO: return c.rho;
    case ICLS_F_JIEMIAN: return c.jiemian; case ICLS_F_CURV: return c.curv;
    default: break;
  }
  *n = P.nI;
  switch (id) {
    case ICLS_F_DUOLD: return c.duold[c.hist]; case ICLS_F_DVOLD: return c.dvold[c.hist];
    case ICLS_F_DWOLD: return c.dwold[c.hist];
    case ICLS_F_RHO_U: return c.rho_u; case ICLS_F_RHO_V: return c.rho_v; case ICLS_F_RHO_W: return c.rho_w;
    case ICLS_F_UCC: return c.ucc; case ICLS_F_VCC: return c.vcc; case ICLS_F_WCC: return c.wcc;
    case ICLS_F_NORMAL_M: return c.nrm_m;
    default: break;
  }
  *n = P.nL;
  if (id == ICLS_F_LVSET && l >= 1 && l <= P.L) return c.lv[l - 1];
  return nullptr;
}

// the field is stored in the form's field type (else FP64 in both forms)
bool tfield(int id) {
  switch (id) {
    case ICLS_F_P: case ICLS_F_PJUMP:
      return false;
    default:
      return true;
  }
}

int check_launch() {
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? ICLS_OK : ICLS_E_CUDA;
}

// ----------------------------------------------------------- level set
// Host replay of the far-field value: the same IEEE operations the kernels
// apply to a cell whose whole stencil is uniform (compiled without
// contraction, as the device code).
double clip_h(double x, double NB) { return x > NB ? NB : (x < -NB ? -NB : x); }
double reinit_sgn_h(const Params& p, double p0) {
  if (p0 < -p.dz) return -1.;
  if (p0 > p.dz) return 1.;
  return p0 / std::sqrt(p0 * p0 + p.dz * p.dz);
}
// WENO5_reinit RHS of a uniform neighbourhood: every one-sided derivative
// is exactly zero (hyperPDE.f90:2736)
double reinit_rhs_h(const Params& p, double phis, double orig) {
  if (!(std::fabs(phis) < p.NB + p.dz)) return 0.;
  const double s = reinit_sgn_h(p, orig);
  const double d = 0.5 * (0. + 0.);
  return s * (1. - std::sqrt((d * d + d * d) + d * d));
}

bool is_full(const Params& P, const Region& r) { return region_full(P, r); }

int wrap1(int v, int n) {
  v = (v - 1) % n;
  if (v < 0) v += n;
  return v + 1;
}

// interior cells of a drop outside the computed part of its region (their H is 1)
double outside_count(const Ctx& c, const Region& r) {
  const double nx = (double)(r.cx1 - r.cx0 + 1), ny = (double)(r.cy1 - r.cy0 + 1);
  const int z0 = std::max(1, r.cz0), z1 = std::min(c.P.kmax, r.cz1);
  const double nz = z1 >= z0 ? (double)(z1 - z0 + 1) : 0.;
  return (double)c.P.nI - nx * ny * nz;
}

// band extents measured by the last tube_construction sweep.  A periodic
// axis keeps the narrower of the spans seen from two frames half a period
// apart, so a band across the seam gives its true width.
// drop l's band box from the host copy of the device extents; false when
// the drop's array held nothing but far field
bool read_band(Ctx& c, int l) {
  const Params& P = c.P;
  DropWin& w = c.win[l];
  const int* lo = c.h_bbox + 5 * l;
  const int* hi = c.h_bbox + 5 * P.L + 5 * l;
  if (lo[4] > hi[4]) return false;
  auto span = [](const int* lo2, const int* hi2, int n, int& a, int& len) {
    const int nA = hi2[0] - lo2[0] + 1, nB = hi2[1] - lo2[1] + 1;
    if (nA <= nB) {
      a = lo2[0];
      len = nA;
    } else {
      a = wrap1(lo2[1] - n / 2, n);
      len = nB;
    }
  };
  span(lo, hi, P.imax, w.Dxa, w.Dxn);
  span(lo + 2, hi + 2, P.jmax, w.Dya, w.Dyn);
  w.Dz0 = lo[4];
  w.Dz1 = hi[4];
  return true;
}
int collect_bbox(Ctx& c) {
  if (!c.bbox_pending) return ICLS_OK;
  CK(cudaEventSynchronize(c.ev_bbox));
  c.bbox_pending = false;
  for (int l = 0; l < c.P.L; ++l) {
    DropWin& w = c.win[l];
    if (!read_band(c, l)) {
      w.have_D = false;  // nothing but far field: sweep everything next time
      continue;
    }
    w.grow = w.pending_grow;
    w.have_D = true;
  }
  return ICLS_OK;
}

// The region drop l sweeps in a step whose own spreading is g_now cells:
// the last measured band grown by what the field could have spread since
// (tube skin 2, 9 per reinitialisation iteration), plus a 3-cell apron.  A
// periodic axis becomes full when the span and its apron would cover the
// period; z becomes full when the box would reach the two rows next to a
// wall.
Region sweep_region(const Ctx& c, int l, int g_now) {
  const DropWin& w = c.win[l];
  const Params& P = c.P;
  if (!c.use_boxes || !w.have_D || !w.bg_valid) return full_region(P);
  // the band box is exact only if the clipped far field equals +6dz
  if (clip_h(w.bg, P.NB) != P.NB || clip_h(w.bg_ghost, P.NB) != P.NB) return full_region(P);
  const int g = w.grow + g_now;
  Region r = full_region(P);
  auto axis = [&](int Da, int Dn, int n, int& xa, int& xn, int& c0, int& c1) {
    const int len = Dn + 2 * g;
    if (len + 6 > n) return;  // stays full
    xa = wrap1(Da - g - 3, n);
    xn = len + 6;
    c0 = 3;
    c1 = 3 + len - 1;
  };
  axis(w.Dxa, w.Dxn, P.imax, r.xa, r.xn, r.cx0, r.cx1);
  axis(w.Dya, w.Dyn, P.jmax, r.ya, r.yn, r.cy0, r.cy1);
  const int lo = w.Dz0 - g, hi = w.Dz1 + g;
  if (lo >= 3 && hi <= P.kmax - 2) {
    r.cz0 = lo;
    r.cz1 = hi;
    r.z0 = lo - 3;
    r.z1 = hi + 3;
  }
  return r;
}

// batches of at most kTasks drops with region(l) as their regions
template <class RegionOf>
std::vector<LsBatch> make_batches(const std::vector<int>& drops, int kc, RegionOf region) {
  std::vector<LsBatch> out;
  for (size_t s = 0; s < drops.size(); s += kTasks) {
    out.emplace_back();
    LsBatch& b = out.back();
    b.n = (int)std::min<size_t>(kTasks, drops.size() - s);
    for (int q = 0; q < b.n; ++q) {
      b.t[q] = LsTask();
      b.t[q].l = drops[s + q];
      b.t[q].r = region(drops[s + q]);
    }
    set_tiles(b, kc);
  }
  return out;
}

constexpr int kStageRows = 8;  // z rows per block of the level-set stage kernels
// the chunk that starts at row -2 must reach row 2: a column's wall row 0 is
// written by the thread that holds rows 1 and 2 (measured: 8 rows beat 4
// and 16)
static_assert(kStageRows >= 5, "level-set chunks must span rows -2..2");

Ctx::Member& member(Ctx& c, int l) { return c.mem[l % (int)c.mem.size()]; }

// Make drop l's stored array valid everywhere and sweep it whole from now
// on (used before downloads and by the standalone routine calls).
void make_full(Ctx& c, int l) {
  collect_bbox(c);  // a pending measurement must not revive the old box
  DropWin& w = c.win[l];
  if (!is_full(c.P, w.valid)) launch_materialize(c, w.valid, w.bg, w.bg_ghost, c.lv[l]);
  w.box = w.valid = full_region(c.P);
  w.have_D = false;
}

void update_materials(Ctx& c) {
  const int L = c.P.L;
  launch_fill(c, c.jiemian, c.P.nC, 1.0, true);
  std::vector<int> all(L);
  for (int l = 0; l < L; ++l) all[l] = l;
  std::vector<int> ntiles(L, 0);  // partial sums per drop: column tiles x z chunks
  for (LsBatch& b : make_batches(all, kHeavRows, [&](int l) { return c_region(c.P, c.win[l].box, 0); })) {
    for (int q = 0; q < b.n; ++q) {
      b.t[q].phi0 = c.lv[b.t[q].l];
      ntiles[b.t[q].l] = b.t[q].tx * b.t[q].ty * b.t[q].nch;
    }
    launch_heaviside(c, b);
  }
  for (int l = 0; l < L; ++l) c.outside[l] = outside_count(c, c.win[l].box);
  launch_materials_final(c, c.outside.data(), ntiles.data());
  cudaMemcpyAsync(c.h_vol, c.dvol, sizeof(double) * L, cudaMemcpyDeviceToHost, c.s);
  cudaEventRecord(c.ev_vol, c.s);
  c.vol_pending = true;
  std::fill(c.vol_dirty.begin(), c.vol_dirty.end(), 0);
}

// tube_construction (levelset.f90:87-197) of the batches' drops into
// their members' s1 and band masks; every cell outside the measured band
// box is +6dz afterwards
void tube_batches(Ctx& c, std::vector<LsBatch>& bs) {
  for (LsBatch& b : bs) {
    for (int q = 0; q < b.n; ++q) {
      LsTask& t = b.t[q];
      const DropWin& w = c.win[t.l];
      t.phi0 = c.lv[t.l];
      t.vin = w.valid;
      t.bgin = w.bg;
      t.bggin = w.bg_ghost;
      t.out = member(c, t.l).s1;
      t.mask = member(c, t.l).mask;
    }
    launch_tube(c, b);
    for (int q = 0; q < b.n; ++q) {
      DropWin& w = c.win[b.t[q].l];
      w.valid = w.box;
      w.bg = c.P.NB;
      w.bg_ghost = c.P.NB;
      w.bg_valid = true;
    }
  }
}

// SSP-RK3 of ls_advection / inflation (levelset.f90:235-243, 558-565) on
// the batches' drops, with their members' buffers: from_tube, s1 -> s2 ->
// s3 -> the drop's own array; else the drop's array -> s1 -> s2 -> itself
// the band cells a batch's list can hold at most: its tasks' computed
// interior cells
long long band_bound(const Ctx& c, const LsBatch& b) {
  long long n = 0;
  for (int q = 0; q < b.n; ++q) {
    const Region& r = b.t[q].r;
    const long long z = std::max(0, std::min(r.cz1, c.P.kmax) - std::max(r.cz0, 1) + 1);
    n += (long long)(r.cx1 - r.cx0 + 1) * (r.cy1 - r.cy0 + 1) * z;
  }
  return n;
}

void rk3_batches(Ctx& c, std::vector<LsBatch>& bs, int scheme, bool from_tube, const double* vu, const double* vv,
                 const double* vw) {
  const double dt = c.dt;
  for (LsBatch& b : bs) {
    // after tube_construction the band flags are fresh: one band list serves
    // the three stages
    // (a list entry holds i and j in 12 bits each)
    const bool packs = c.P.imax <= 4096 && c.P.jmax <= 4096;
    const long long need = from_tube && !c.adv_column && packs ? band_bound(c, b) : -1;
    const bool split = need >= 0 && need <= c.band_cap;
    if (split) {
      for (int q = 0; q < b.n; ++q) b.t[q].mask = member(c, b.t[q].l).mask;
      launch_band_list(c, b);
    }
    double g[kTasks][4], h[kTasks][4];
    for (int q = 0; q < b.n; ++q) {
      const DropWin& w = c.win[b.t[q].l];
      g[q][0] = w.bg;
      h[q][0] = w.bg_ghost;
      g[q][1] = g[q][0];
      h[q][1] = h[q][0];
      g[q][2] = 3. / 4. * g[q][0] + 1. / 4. * g[q][1];
      h[q][2] = 3. / 4. * h[q][0] + 1. / 4. * h[q][1];
      g[q][3] = 1. / 3. * g[q][0] + 2. / 3. * g[q][2];
      h[q][3] = 1. / 3. * h[q][0] + 2. / 3. * h[q][2];
    }
    auto stage = [&](int st, double a, double bb, double fdt) {
      for (int q = 0; q < b.n; ++q) {
        LsTask& t = b.t[q];
        Ctx::Member& m = member(c, t.l);
        const double* src = from_tube ? m.s1 : c.lv[t.l];
        double* A = from_tube ? m.s2 : m.s1;
        double* B = from_tube ? m.s3 : m.s2;
        t.mask = m.mask;
        t.phi0 = src;
        t.phis = st == 1 ? src : (st == 2 ? A : B);
        t.out = st == 1 ? A : (st == 2 ? B : c.lv[t.l]);
        t.bg = g[q][st];
        t.bgg = h[q][st];
      }
      if (split) launch_adv_split(c, b, scheme, st == 1 ? 1 : 0, a, bb, fdt, vu, vv, vw, need);
      else launch_adv_stage(c, b, scheme, st == 1 ? 1 : 0, a, bb, fdt, vu, vv, vw);
    };
    stage(1, 1., 0., 1. * dt);
    stage(2, 3. / 4., 1. / 4., 1. / 4. * dt);
    stage(3, 1. / 3., 2. / 3., 2. / 3. * dt);
    for (int q = 0; q < b.n; ++q) {
      DropWin& w = c.win[b.t[q].l];
      w.bg = g[q][3];
      w.bg_ghost = h[q][3];
    }
  }
}

std::vector<LsBatch> single(const Ctx& c, int l, int kc, const Region& r) {
  std::vector<int> one{l};
  return make_batches(one, kc, [&](int) { return r; });
}

void ls_advection(Ctx& c, int l) {
  std::vector<LsBatch> bs = single(c, l, kStageRows, c.win[l].box);
  rk3_batches(c, bs, c.cfg.ls_adv_space, false, c.ucc, c.vcc, c.wcc);
}

// inflation (levelset.f90:407-582)
void inflation(Ctx& c, int l) {
  const Region b = c.win[l].box;
  const Region r1 = c_region(c.P, b, 1);
  std::vector<LsBatch> bc = single(c, l, kStageRows, r1);
  bc[0].t[0].phi0 = c.lv[l];
  bc[0].t[0].out = c.kappa;
  launch_curvature(c, bc[0], c.nrm_m);
  c.nrm_stale = true;
  std::vector<LsBatch> bsum = single(c, l, 0, r1);
  bsum[0].t[0].phi0 = c.lv[l];
  launch_inflate_sums(c, bsum[0], outside_count(c, b));
  std::vector<LsBatch> bvel = single(c, l, kStageRows, c_region(c.P, b, 0));
  launch_inflate_vel(c, bvel[0]);
  std::vector<LsBatch> bs = single(c, l, kStageRows, b);
  // gain one: keep phi0 on the written cells of the RK3 region (member s3
  // is free after the advection) and its far-field values
  DropWin& w = c.win[l];
  const double bg0 = w.bg, bgg0 = w.bg_ghost;
  if (c.cfg.mass_gain_one) {
    std::vector<LsBatch> bcp = single(c, l, kStageRows, b);
    bcp[0].t[0].phi0 = c.lv[l];
    bcp[0].t[0].out = member(c, l).s3;
    launch_region_copy(c, bcp[0]);
  }
  rk3_batches(c, bs, c.cfg.i_space, false, c.ulc, c.vlc, c.wlc);
  if (c.cfg.mass_gain_one) {
    std::vector<LsBatch> bv = single(c, l, 0, r1);
    bv[0].t[0].phi0 = c.lv[l];
    launch_gain(c, bv[0], outside_count(c, b));
    std::vector<LsBatch> bb = single(c, l, kStageRows, b);
    bb[0].t[0].phi0 = member(c, l).s3;
    bb[0].t[0].out = c.lv[l];
    launch_region_blend(c, bb[0]);
    // the far field (uniform, velocity zero there) keeps its value unless the
    // RK3 combinations rounded it; then it is blended like every cell
    if (w.bg != bg0 || w.bg_ghost != bgg0) {
      double gain = 0.;
      if (cudaMemcpyAsync(&gain, &c.dsc->inflate_gain, sizeof(double), cudaMemcpyDeviceToHost, c.s) ==
              cudaSuccess &&
          cudaStreamSynchronize(c.s) == cudaSuccess) {
        w.bg = bg0 + gain * (w.bg - bg0);
        w.bg_ghost = bgg0 + gain * (w.bg_ghost - bgg0);
      }
    }
  }
  c.inflated[l] = 1;
  c.vol_dirty[l] = 1;
  ++c.last_inflated;
}

int volume_of(Ctx& c, int l, double* v) {
  if (c.vol_dirty[l]) {
    CK(cudaMemcpyAsync(v, c.dvol + l, sizeof(double), cudaMemcpyDeviceToHost, c.s));
    CK(cudaStreamSynchronize(c.s));
    return ICLS_OK;
  }
  if (c.vol_pending) {
    CK(cudaEventSynchronize(c.ev_vol));
    c.vol_pending = false;
  }
  *v = c.h_vol[l];
  return ICLS_OK;
}

// each of the drops' volumes as they are now (the exact sum of H over the
// drop's box plus its far-field count), into h_volnow: one read-back
int measure_volumes_now(Ctx& c, const std::vector<int>& drops) {
  for (int l : drops) {
    const Region b = c.win[l].box;
    std::vector<LsBatch> bv = single(c, l, 0, c_region(c.P, b, 1));
    bv[0].t[0].phi0 = c.lv[l];
    launch_volume_now(c, bv[0], outside_count(c, b));
  }
  CK(cudaMemcpyAsync(c.h_volnow, c.dvolnow, sizeof(double) * c.P.L, cudaMemcpyDeviceToHost, c.s));
  CK(cudaStreamSynchronize(c.s));
  return ICLS_OK;
}

// ls_mass_correction (levelset.f90:377-400).  The reference tests the
// volume of the last update_materials; the gain-one correction tests the
// drop's volume as it is now (after this step's advection and
// reinitialisation, measured by measure_volumes_now into h_volnow)
int ls_mass_correction(Ctx& c, int istep, int l) {
  c.inflated[l] = 0;
  if (istep % c.cfg.inflate_step == 0) {
    double vol;
    int rc = ICLS_OK;
    if (c.cfg.mass_gain_one) vol = c.h_volnow[l];
    else rc = volume_of(c, l, &vol);
    if (rc) return rc;
    const double v0 = c.init_volume_h[l];
    const double massloss = (vol - v0) / v0;
    const double eps = c.cfg.mass_threshold > 0. ? c.cfg.mass_threshold : 1e-5;
    if (std::fabs(massloss) > eps) inflation(c, l);
  }
  return ICLS_OK;
}

// ls_reinit, WENO5/RK3 (levelset.f90:619-882) on the batches' drops; the
// early exit on residual < dz**5 is decided per drop on the device
// (k_reinit_check).  Far-field cells outside a drop's region change by
// |bg_new - bg_old| per iteration, which enters its residual as the
// reference's maxval over all cells does.  The original level set stays in
// the drop's own array until the last stage, which overwrites it in place.
void reinit_batches(Ctx& c, std::vector<LsBatch>& bs) {
  const Params& P = c.P;
  const int maxiter = c.cfg.reinit_iter_max;
  const double dz = P.dz;
  const double dtau = 0.5 * dz;
  const double thr = dz * dz * dz * dz * dz;
  for (LsBatch& b : bs) {
    double xg[kTasks], xh[kTasks], og[kTasks];
    bool partial[kTasks];
    for (int q = 0; q < b.n; ++q) {
      const DropWin& w = c.win[b.t[q].l];
      xg[q] = w.bg;
      xh[q] = w.bg_ghost;
      og[q] = w.bg;  // sgn source of the far field
      partial[q] = !is_full(P, w.box);
    }
    launch_reinit_reset(c, b, maxiter);
    for (int it = 1; it <= maxiter; ++it) {
      double ag[kTasks], ah[kTasks], bgv[kTasks], bh[kTasks], yg[kTasks], yh[kTasks];
      for (int q = 0; q < b.n; ++q) {
        ag[q] = xg[q] + dtau * reinit_rhs_h(P, xg[q], og[q]);
        ah[q] = xh[q] + dtau * 0.;
        bgv[q] = 3. / 4. * xg[q] + 1. / 4. * (ag[q] + dtau * reinit_rhs_h(P, ag[q], og[q]));
        bh[q] = 3. / 4. * xh[q] + 1. / 4. * (ah[q] + dtau * 0.);
        yg[q] = 1. / 3. * xg[q] + 2. / 3. * (bgv[q] + dtau * reinit_rhs_h(P, bgv[q], og[q]));
        yh[q] = 1. / 3. * xh[q] + 2. / 3. * (bh[q] + dtau * 0.);
      }
      auto stage = [&](int st) {
        for (int q = 0; q < b.n; ++q) {
          LsTask& t = b.t[q];
          double* own = c.lv[t.l];
          const Ctx::Member& m = member(c, t.l);
          double* S1 = m.s1;
          double* S2 = m.s2;
          double* S3 = m.s3;
          const double* X = it == 1 ? own : S3;
          t.phi0 = X;
          t.orig = own;
          t.phis = st == 1 ? X : (st == 2 ? S1 : S2);
          t.out = st == 1 ? S1 : (st == 2 ? S2 : (it == maxiter ? own : S3));
          t.bg = st == 1 ? ag[q] : (st == 2 ? bgv[q] : yg[q]);
          t.bgg = st == 1 ? ah[q] : (st == 2 ? bh[q] : yh[q]);
          t.far = partial[q] ? std::max(std::fabs(yg[q] - xg[q]), std::fabs(yh[q] - xh[q])) : 0.;
        }
        launch_reinit_stage(c, b, st, dtau);
      };
      stage(1);
      stage(2);
      stage(3);
      launch_reinit_check(c, b, it, maxiter, thr);
      for (int q = 0; q < b.n; ++q) {
        xg[q] = yg[q];
        xh[q] = yh[q];
      }
    }
    // with a far field the residual never drops below dz**5 (the far field
    // moves by ~dtau per iteration), so every iteration runs: the replayed
    // values are exact
    for (int q = 0; q < b.n; ++q) {
      DropWin& w = c.win[b.t[q].l];
      w.bg = xg[q];
      w.bg_ghost = xh[q];
    }
  }
}

void ls_reinit(Ctx& c, int l) {
  std::vector<LsBatch> bs = single(c, l, kStageRows, c.win[l].box);
  reinit_batches(c, bs);
}

// tube_construction of one drop over its whole array (standalone call)
void tube_construction(Ctx& c, int l) {
  std::vector<LsBatch> bs = single(c, l, kStageRows, c.win[l].box);
  cudaMemsetAsync(c.d_nbcnt + l, 0, sizeof(long long), c.s);
  tube_batches(c, bs);
  std::swap(c.lv[l], member(c, l).s1);
}

// the drops of group g: [g*G, min(L, (g+1)*G))
std::vector<int> group_drops(const Ctx& c, int g) {
  const int G = (int)c.mem.size();
  std::vector<int> d;
  for (int l = g * G; l < std::min(c.P.L, (g + 1) * G); ++l) d.push_back(l);
  return d;
}
int n_groups(const Ctx& c) { return (c.P.L + (int)c.mem.size() - 1) / (int)c.mem.size(); }

// The band box a tube_construction sweep of the whole array would measure
// now, for every drop whose stored array is valid everywhere (as after an
// upload).  The first sweep then needs only that box grown by the step's
// own spread: outside it the sweep would write +6dz, the value the box's far
// field stands for.  The stored arrays stay valid everywhere (a download
// still returns them as uploaded); a drop already swept by boxes keeps its
// state.
int measure_bands(Ctx& c) {
  if (!c.use_boxes) return ICLS_OK;
  const int L = c.P.L;
  collect_bbox(c);
  CK(cudaMemsetAsync(c.d_bbox, 0x7F, sizeof(int) * 5 * L, c.s));
  CK(cudaMemsetAsync(c.d_bbox + 5 * L, 0x80, sizeof(int) * 5 * L, c.s));
  for (int l = 0; l < L; ++l)
    if (is_full(c.P, c.win[l].valid)) launch_band_extents(c, l);
  CK(cudaMemcpyAsync(c.h_bbox, c.d_bbox, sizeof(int) * 10 * L, cudaMemcpyDeviceToHost, c.s));
  CK(cudaStreamSynchronize(c.s));
  for (int l = 0; l < L; ++l) {
    DropWin& w = c.win[l];
    if (!is_full(c.P, w.valid)) continue;
    if (!read_band(c, l)) {
      w.have_D = false;
      w.box = w.valid;
      continue;
    }
    w.grow = 0;
    w.have_D = true;
    w.bg = c.P.NB;
    w.bg_ghost = c.P.NB;
    w.bg_valid = true;
    w.box = sweep_region(c, l, 0);
  }
  return ICLS_OK;
}

// A drop without a measured band (the first step after its array was
// uploaded or swept whole) runs its tube construction over the whole array.
// That sweep leaves every cell outside the band box it measures at +6dz, so
// the rest of the step needs only that box grown by this step's own spread:
// read the extents now (one wait on the stream, on such steps only) and make
// that region the drop's sweep and valid region.
int narrow_after_tube(Ctx& c, const std::vector<int>& drops, int g_now) {
  CK(cudaMemcpyAsync(c.h_bbox, c.d_bbox, sizeof(int) * 10 * c.P.L, cudaMemcpyDeviceToHost, c.s));
  CK(cudaStreamSynchronize(c.s));
  for (int l : drops) {
    DropWin& w = c.win[l];
    if (w.have_D || !read_band(c, l)) continue;
    w.grow = 0;
    w.have_D = true;
    w.box = sweep_region(c, l, g_now);
    w.valid = w.box;
  }
  return ICLS_OK;
}

int ls_main(Ctx& c, int istep) {
  c.last_inflated = 0;
  int rc = collect_bbox(c);
  if (rc) return rc;
  const Params& P = c.P;
  const int L = P.L;
  const bool reinit_now = c.cfg.re_initialization && istep % c.cfg.reinit_step == 0;
  const int g_now = 2 + (reinit_now ? 9 * c.cfg.reinit_iter_max : 0);
  for (int l = 0; l < L; ++l) {
    c.win[l].box = sweep_region(c, l, g_now);
    c.win[l].pending_grow = g_now;
  }
  cudaMemsetAsync(c.d_nbcnt, 0, sizeof(long long) * L, c.s);
  cudaMemsetAsync(c.d_bbox, 0x7F, sizeof(int) * 5 * L, c.s);
  cudaMemsetAsync(c.d_bbox + 5 * L, 0x80, sizeof(int) * 5 * L, c.s);
  // per group: tube_construction, ls_advection, ls_mass_correction (which
  // still reads the drop's band mask) and ls_reinit, as the reference runs
  // them for each drop
  for (int g = 0; g < n_groups(c); ++g) {
    const std::vector<int> drops = group_drops(c, g);
    std::vector<LsBatch> bs = make_batches(drops, kStageRows, [&](int l) { return c.win[l].box; });
    bool unmeasured = false;
    for (int l : drops) unmeasured = unmeasured || (c.use_boxes && !c.win[l].have_D);
    tube_batches(c, bs);
    if (unmeasured) {
      rc = narrow_after_tube(c, drops, g_now);
      if (rc) return rc;
      bs = make_batches(drops, kStageRows, [&](int l) { return c.win[l].box; });
    }
    rk3_batches(c, bs, c.cfg.ls_adv_space, true, c.ucc, c.vcc, c.wcc);
    // the reference corrects the volume before reinitialising; with the
    // gain-one correction the order is swapped, so that one correction also
    // removes the volume change of the reinitialisation in the same step
    const bool correct_last = c.cfg.mass_gain_one != 0;
    if (reinit_now && correct_last) reinit_batches(c, bs);
    if (c.cfg.mass_correction && correct_last && istep % c.cfg.inflate_step == 0) {
      rc = measure_volumes_now(c, drops);
      if (rc) return rc;
    }
    if (c.cfg.mass_correction)
      for (int l : drops) {
        rc = ls_mass_correction(c, istep, l);
        if (rc) return rc;
      }
    if (reinit_now && !correct_last) reinit_batches(c, bs);
  }
  cudaMemcpyAsync(c.h_bbox, c.d_bbox, sizeof(int) * 10 * L, cudaMemcpyDeviceToHost, c.s);
  cudaEventRecord(c.ev_bbox, c.s);
  c.bbox_pending = true;
  update_materials(c);
  return check_launch();
}

// curv and normal%m as the reference leaves them after its last
// get_curvature/re_curvature call: the last drop's values, zero (one)
// elsewhere
void fix_curv(Ctx& c) {
  if (!c.curv_stale && !c.nrm_stale) return;
  const int l = c.P.L - 1;
  const size_t bytes = (c.P.f32 ? sizeof(float) : sizeof(double)) * (size_t)c.P.nC;
  launch_fill(c, c.nrm_m, c.P.nI, 1.0, true);
  cudaMemsetAsync(c.curv, 0, bytes, c.s);
  std::vector<LsBatch> b = single(c, l, kStageRows, c_region(c.P, c.win[l].box, 1));
  LsTask& t = b[0].t[0];
  t.phi0 = c.lv[l];
  const bool mlp = c.cfg.curvature_model == ICLS_CURV_MLP && c.net;
  if (c.cfg.TwoD) {
    t.out = c.curv;
    launch_curvature(c, b[0], c.nrm_m, mlp);
    if (mlp) launch_mlp_curvature(c, b[0]);
  } else {
    t.out = member(c, l).fit;
    launch_curvature(c, b[0], c.nrm_m, mlp);
    if (mlp) launch_mlp_curvature(c, b[0]);
    t.phis = member(c, l).fit;
    t.out = c.curv;
    launch_recurvature(c, b[0]);
  }
  c.curv_stale = c.nrm_stale = false;
}

// gfm4p, GFM/'del' (gfm.f90:17-267), one group of drops at a time, each
// drop with its member's curvature buffers; with the learned curvature the
// network replaces get_curvature's output near the interface.  ipot is
// evaluated by icls_ipot.
int gfm4p(Ctx& c) {
  if (c.cfg.curvature_model == ICLS_CURV_MLP && !c.net) return ICLS_E_STATE;
  std::swap(c.px, c.pxold);
  std::swap(c.py, c.pyold);
  std::swap(c.pz, c.pzold);
  const size_t bytes = sizeof(double) * (size_t)c.P.nC, tbytes = sizeof(double) * tn(c.P, c.P.nC);
  cudaMemsetAsync(c.px, 0, tbytes, c.s);
  cudaMemsetAsync(c.py, 0, tbytes, c.s);
  cudaMemsetAsync(c.pz, 0, tbytes, c.s);
  cudaMemsetAsync(c.pjump, 0, bytes, c.s);
  for (int g = 0; g < n_groups(c); ++g) {
    const std::vector<int> drops = group_drops(c, g);
    std::vector<LsBatch> b1 = make_batches(drops, kStageRows, [&](int l) { return c_region(c.P, c.win[l].box, 1); });
    std::vector<LsBatch> b0 = make_batches(drops, kStageRows, [&](int l) { return c_region(c.P, c.win[l].box, 0); });
    for (LsBatch& b : b1) {
      for (int q = 0; q < b.n; ++q) {
        LsTask& t = b.t[q];
        t.phi0 = c.lv[t.l];
        t.out = c.cfg.TwoD ? member(c, t.l).cv : member(c, t.l).fit;
      }
      const bool mlp = c.cfg.curvature_model == ICLS_CURV_MLP;
      launch_curvature(c, b, nullptr, mlp);
      if (mlp) launch_mlp_curvature(c, b);
    }
    if (!c.cfg.TwoD)
      for (LsBatch& b : b1) {
        for (int q = 0; q < b.n; ++q) {
          LsTask& t = b.t[q];
          t.phis = member(c, t.l).fit;
          t.out = member(c, t.l).cv;
        }
        launch_recurvature(c, b);
      }
    for (LsBatch& b : b0) {
      for (int q = 0; q < b.n; ++q) {
        LsTask& t = b.t[q];
        t.phi0 = c.lv[t.l];
        t.phis = member(c, t.l).cv;
      }
      launch_jumps(c, b);
    }
  }
  c.curv_stale = true;
  c.nrm_stale = true;
  return ICLS_OK;
}

int read_scalars(Ctx& c) {
  CK(cudaMemcpyAsync(c.h_sc, c.dsc, sizeof(DevScalars), cudaMemcpyDeviceToHost, c.s));
  CK(cudaStreamSynchronize(c.s));
  if (c.h_sc->wait_err) return ICLS_E_TIMEOUT;
  return ICLS_OK;
}

int chkdiv(Ctx& c, int istep, double* divtot, double* divmax, int* ijk) {
  launch_chkdiv(c);
  int rc = read_scalars(c);
  if (rc) return rc;
  if (divtot) *divtot = c.h_sc->divtot;
  if (divmax) *divmax = c.h_sc->divmax;
  if (ijk) {
    long long q = c.h_sc->divloc;
    if (q < 0) {
      ijk[0] = ijk[1] = ijk[2] = 0;
    } else {
      ijk[0] = (int)(q % c.P.imax) + 1;
      ijk[1] = (int)((q / c.P.imax) % c.P.jmax) + 1;
      ijk[2] = (int)(q / ((long long)c.P.imax * c.P.jmax)) + 1;
    }
  }
  // chkdiv.f90:60-87 stops above 1e-12; the precision form scales that bound
  // by the ratio of the FP32 and FP64 unit roundoffs, 2^-24 / 2^-53 = 2^29
  const double bound = c.P.f32 ? 1e-12 * 536870912.0 : 1e-12;
  if (c.h_sc->divmax > bound && istep != 0) return ICLS_E_DIVERGENCE;
  return ICLS_OK;
}

}  // namespace

// ======================================================================== C
extern "C" {

void icls_config_default(icls_config* c) {
  std::memset(c, 0, sizeof(*c));
  c->itot = c->jtot = c->ktot = 32;
  c->lmax = 1;
  c->lx = c->ly = c->lz = 1.0;
  c->timestep = 5e-4;
  c->rho1 = 1.0; c->rho2 = 10.0; c->miu1 = 1.0; c->miu2 = 0.1;
  c->Re = 10.0; c->We = 1.0; c->iFr = 0.0;
  c->TwoD = 0; c->constPoi = 0; c->solveLS = 1;
  c->ls_adv_space = ICLS_HOUC5;
  c->re_initialization = 1; c->reinit_step = 20; c->reinit_iter_max = 1;
  c->mass_correction = 1; c->inflate_step = 20;
  c->ispeed_dependence = ICLS_SPEED_CURV; c->i_space = ICLS_HOUC5;
  c->ioutchk = 20;
  c->precision = ICLS_FP64; c->curvature_model = ICLS_CURV_STENCIL;
  c->mlp_fallback_tol = 0.02;
  c->mass_threshold = 0.;
}

int icls_status_string(int code, char* buf, int n) {
  static const char* names[] = {"ok", "invalid or unsupported configuration", "CUDA error",
                                "NaN in vnew(1,1,1)", "max divergence above 1e-12", "bad argument",
                                "device allocation failed", "context not initialised",
                                "option not built into this library",
                                "grid larger than the no-allocation divergence check handles",
                                "checkpoint file could not be written or read",
                                "a kernel's bounded pipeline wait gave up"};
  const char* s = (code >= 0 && code <= 11) ? names[code] : "unknown status";
  if (buf && n > 0) {
    std::strncpy(buf, s, (size_t)n - 1);
    buf[n - 1] = 0;
  }
  return ICLS_OK;
}

int icls_create(const icls_config* cfg, icls_ctx** out) {
  if (!out) return ICLS_E_ARG;
  *out = nullptr;
  int rc = validate(cfg);
  if (rc) return rc;
  icls_ctx* h = new (std::nothrow) icls_ctx();
  if (!h) return ICLS_E_NOMEM;
  Ctx& c = h->c;
  c.cfg = *cfg;
  fill_params(c);
  if (cudaGetDevice(&c.device) != cudaSuccess || cudaStreamCreateWithFlags(&c.s, cudaStreamNonBlocking) != cudaSuccess) {
    delete h;
    return ICLS_E_CUDA;
  }
  rc = allocate(c);
  if (rc) {
    release(c);
    delete h;
    return rc;
  }
  c.dt = cfg->timestep;
  *out = h;
  return ICLS_OK;
}

int icls_destroy(icls_ctx* h) {
  if (!h) return ICLS_E_ARG;
  cudaStreamSynchronize(h->c.s);
  release(h->c);
  delete h;
  return ICLS_OK;
}

int icls_field_bounds(const icls_ctx* h, int id, int lo[3], int hi[3]) {
  if (!h || !lo || !hi) return ICLS_E_ARG;
  const Params& P = h->c.P;
  int kind;
  switch (id) {
    case ICLS_F_DUOLD: case ICLS_F_DVOLD: case ICLS_F_DWOLD: case ICLS_F_RHO_U: case ICLS_F_RHO_V:
    case ICLS_F_RHO_W: case ICLS_F_UCC: case ICLS_F_VCC: case ICLS_F_WCC: case ICLS_F_NORMAL_M:
      kind = 1; break;
    case ICLS_F_LVSET: kind = 2; break;
    default:
      if (id < 0 || id >= ICLS_F_COUNT) return ICLS_E_ARG;
      kind = 0;
  }
  const int l0 = kind == 0 ? 0 : (kind == 1 ? 1 : -2);
  const int pad = kind == 0 ? 1 : (kind == 1 ? 0 : 3);
  lo[0] = lo[1] = lo[2] = l0;
  hi[0] = P.imax + pad; hi[1] = P.jmax + pad; hi[2] = P.kmax + pad;
  return ICLS_OK;
}

int icls_upload_field(icls_ctx* h, int id, int l, const double* host) {
  if (!h || !host) return ICLS_E_ARG;
  Ctx& c = h->c;
  long long n;
  double* d = field_ptr(c, id, l, &n);
  if (!d) return ICLS_E_ARG;
  if (c.P.f32 && tfield(id)) {  // through the FP64 staging buffer
    CK(cudaMemcpyAsync(c.stage, host, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, c.s));
    launch_to_float(c, d, c.stage, n);
  } else {
    CK(cudaMemcpyAsync(d, host, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, c.s));
  }
  CK(cudaStreamSynchronize(c.s));
  if (id == ICLS_F_LVSET) {  // a new level set: sweep it whole until its band is measured
    collect_bbox(c);
    DropWin& w = c.win[l - 1];
    w.box = w.valid = full_region(c.P);
    w.have_D = false;
    w.bg_valid = false;
  }
  return ICLS_OK;
}

int icls_download_field(icls_ctx* h, int id, int l, double* host) {
  if (!h || !host) return ICLS_E_ARG;
  Ctx& c = h->c;
  long long n;
  double* d = field_ptr(c, id, l, &n);
  if (!d) return ICLS_E_ARG;
  if (id == ICLS_F_LVSET) {  // fill the far field outside the swept region
    const DropWin& w = c.win[l - 1];
    if (!is_full(c.P, w.valid)) launch_materialize(c, w.valid, w.bg, w.bg_ghost, d);
  }
  if (id == ICLS_F_CURV || id == ICLS_F_NORMAL_M) fix_curv(c);
  if (c.P.f32 && tfield(id)) {
    launch_to_double(c, c.stage, d, n);
    CK(cudaMemcpyAsync(host, c.stage, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, c.s));
  } else {
    CK(cudaMemcpyAsync(host, d, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, c.s));
  }
  CK(cudaStreamSynchronize(c.s));
  return ICLS_OK;
}

int icls_download_plane_x(icls_ctx* h, int id, int l, int i, double* host) {
  if (!h || !host) return ICLS_E_ARG;
  Ctx& c = h->c;
  int lo[3], hi[3];
  int rc = icls_field_bounds(h, id, lo, hi);
  if (rc) return rc;
  if (i < lo[0] || i > hi[0]) return ICLS_E_ARG;
  long long n;
  double* d = field_ptr(c, id, l, &n);
  if (!d) return ICLS_E_ARG;
  if (id == ICLS_F_LVSET) {  // fill the far field outside the swept region
    const DropWin& w = c.win[l - 1];
    if (!is_full(c.P, w.valid)) launch_materialize(c, w.valid, w.bg, w.bg_ghost, d);
  }
  if (id == ICLS_F_CURV || id == ICLS_F_NORMAL_M) fix_curv(c);
  const long long nx = hi[0] - lo[0] + 1, ny = hi[1] - lo[1] + 1;
  const int n1 = (int)ny, n2 = hi[2] - lo[2] + 1;
  double* dev = nullptr;
  CK(cudaMallocAsync((void**)&dev, sizeof(double) * (size_t)n1 * n2, c.s));
  launch_gather_plane_x(c, d, c.P.f32 && tfield(id), nx, ny, i - lo[0], n1, n2, dev);
  CK(cudaMemcpyAsync(host, dev, sizeof(double) * (size_t)n1 * n2, cudaMemcpyDeviceToHost, c.s));
  CK(cudaFreeAsync(dev, c.s));
  CK(cudaStreamSynchronize(c.s));
  return check_launch();
}

int icls_timestep_record(icls_ctx* h, int istep, double rec[6]) {
  if (!h || !rec) return ICLS_E_ARG;
  Ctx& c = h->c;
  const int L = c.P.L;
  icls_scalars sc;
  int rc = icls_get_scalars(h, &sc);
  if (rc) return rc;
  std::vector<double> vol(L), vol0(L);
  rc = icls_get_volumes(h, vol.data(), vol0.data());
  if (rc) return rc;
  double massloss = 0.;
  for (int l = 0; l < L; ++l) massloss = massloss + (1. - vol[l] / vol0[l]);
  double quck = 0.;
  if (L >= 2) {
    std::vector<double> dm((size_t)L * L);
    rc = icls_ipot(h, dm.data());
    if (rc) return rc;
    quck = dm[0 + (size_t)L * 1] / c.P.dz;  // dmin(1,2)/dz
  }
  rec[0] = 1. * istep; rec[1] = c.time; rec[2] = c.dt;
  rec[3] = massloss; rec[4] = quck; rec[5] = sc.maxchk_glb;
  return ICLS_OK;
}

int icls_get_scalars(icls_ctx* h, icls_scalars* out) {
  if (!h || !out) return ICLS_E_ARG;
  Ctx& c = h->c;
  int rc = read_scalars(c);
  if (rc) return rc;
  out->time = c.time;
  out->dt = c.dt;
  out->rho_avr = c.h_sc->rho_avr;
  out->v_bulk = c.h_sc->v_bulk;
  out->norm_old = c.h_sc->norm;
  out->reinit_residual = c.h_sc->residual;
  out->reinit_iters = c.h_sc->reinit_iters;
  out->last_inflated = c.last_inflated;
  out->maxchk_glb = 0.;
  if (c.cfg.mass_correction && c.inflated[c.P.L - 1]) {
    CK(cudaMemcpy(&out->maxchk_glb, c.dmaxchk + c.P.L - 1, sizeof(double), cudaMemcpyDeviceToHost));
  }
  return ICLS_OK;
}

int icls_get_volumes(icls_ctx* h, double* volume, double* init_volume) {
  if (!h) return ICLS_E_ARG;
  Ctx& c = h->c;
  if (volume) {
    CK(cudaMemcpyAsync(volume, c.dvol, sizeof(double) * c.P.L, cudaMemcpyDeviceToHost, c.s));
    CK(cudaStreamSynchronize(c.s));
  }
  if (init_volume)
    for (int l = 0; l < c.P.L; ++l) init_volume[l] = c.init_volume_h[l];
  return ICLS_OK;
}

int icls_synchronize(icls_ctx* h) {
  if (!h) return ICLS_E_ARG;
  CK(cudaStreamSynchronize(h->c.s));
  return check_launch();
}

// init_program, begin=0, GFM (init.f90:22-117)
int icls_init_program(icls_ctx* h) {
  if (!h) return ICLS_E_ARG;
  Ctx& c = h->c;
  init_matrix(c);
  set_pseudo_inverse(c.P10x27, c.s);
  poisson_setup(c);
  c.dt = c.cfg.timestep;
  c.time = 0.;
  CK(cudaMemsetAsync(c.dsc, 0, sizeof(DevScalars), c.s));
  launch_bounduvw(c, c.u, c.v, c.w);
  launch_bounduvw(c, c.dudt, c.dvdt, c.dwdt);
  for (int l = 0; l < c.P.L; ++l) launch_boundmls(c, c.lv[l]);
  int rc = measure_bands(c);
  if (rc) return rc;
  launch_boundp(c, c.pnew, true);
  launch_average_vel(c);
  update_materials(c);
  CK(cudaMemcpyAsync(c.dvol0, c.dvol, sizeof(double) * c.P.L, cudaMemcpyDeviceToDevice, c.s));
  CK(cudaStreamSynchronize(c.s));
  c.vol_pending = false;
  for (int l = 0; l < c.P.L; ++l) c.init_volume_h[l] = c.h_vol[l];
  c.hist = 0;
  launch_mom_main(c, c.duold[0], c.dvold[0], c.dwold[0]);
  const size_t bytes = sizeof(double) * tn(c.P, c.P.nC);  // the pressures are in the field type
  CK(cudaMemcpyAsync(c.pold, c.pnew, bytes, cudaMemcpyDeviceToDevice, c.s));
  CK(cudaMemcpyAsync(c.pxold, c.px, bytes, cudaMemcpyDeviceToDevice, c.s));
  CK(cudaMemcpyAsync(c.pyold, c.py, bytes, cudaMemcpyDeviceToDevice, c.s));
  CK(cudaMemcpyAsync(c.pzold, c.pz, bytes, cudaMemcpyDeviceToDevice, c.s));
  CK(cudaStreamSynchronize(c.s));
  c.initialised = true;
  return check_launch();
}

#define NEED(h)                                  \
  do {                                           \
    if (!(h)) return ICLS_E_ARG;                 \
    if (!(h)->c.initialised) return ICLS_E_STATE; \
  } while (0)
#define LARG(h, l) \
  if ((l) < 1 || (l) > (h)->c.P.L) return ICLS_E_ARG

int icls_ls_main(icls_ctx* h, int istep) {
  NEED(h);
  return ls_main(h->c, istep);
}

int icls_set_inflow(icls_ctx* h, const double* v_inflow) {
  if (!h || !v_inflow) return ICLS_E_ARG;
  Ctx& c = h->c;
  CK(cudaMemcpyAsync(c.vin, v_inflow, sizeof(double) * (size_t)(c.P.i1 + 1) * (c.P.k1 + 1),
                     cudaMemcpyHostToDevice, c.s));
  CK(cudaStreamSynchronize(c.s));
  return ICLS_OK;
}

int icls_average_stream_vel(icls_ctx* h, double* v_bulk) {
  NEED(h);
  launch_stream_vel(h->c);
  if (v_bulk) {
    int rc = read_scalars(h->c);
    if (rc) return rc;
    *v_bulk = h->c.h_sc->v_bulk;
  }
  return check_launch();
}

int icls_ab2(icls_ctx* h) {
  NEED(h);
  launch_ab2(h->c);
  return check_launch();
}

int icls_fillps(icls_ctx* h) {
  NEED(h);
  launch_fillps(h->c, 0);
  return check_launch();
}

int icls_gfm4p(icls_ctx* h) {
  NEED(h);
  const int rc = gfm4p(h->c);
  if (rc) return rc;
  return check_launch();
}

int icls_add_pjump(icls_ctx* h) {
  NEED(h);
  launch_add_pjump(h->c);
  return check_launch();
}

int icls_solver2d(icls_ctx* h) {
  NEED(h);
  launch_solver2d(h->c, 0);
  return check_launch();
}

int icls_boundp(icls_ctx* h, int id) {
  if (!h) return ICLS_E_ARG;
  long long n;
  double* d = field_ptr(h->c, id, 1, &n);
  if (!d || n != h->c.P.nC) return ICLS_E_ARG;
  launch_boundp(h->c, d, tfield(id));
  return check_launch();
}

int icls_correc(icls_ctx* h) {
  NEED(h);
  launch_correc(h->c, 0);
  return check_launch();
}

int icls_bounduvw(icls_ctx* h, int id) {
  if (!h) return ICLS_E_ARG;
  Ctx& c = h->c;
  if (id == ICLS_F_U) launch_bounduvw(c, c.u, c.v, c.w);
  else if (id == ICLS_F_DUDT) launch_bounduvw(c, c.dudt, c.dvdt, c.dwdt);
  else return ICLS_E_ARG;
  return check_launch();
}

int icls_pressure_update(icls_ctx* h, int istep, int begin) {
  NEED(h);
  launch_pressure_update(h->c, istep == begin + 1);
  return check_launch();
}

int icls_average_vel_at_center(icls_ctx* h) {
  if (!h) return ICLS_E_ARG;
  launch_average_vel(h->c);
  return check_launch();
}

int icls_max_vel_at_center(icls_ctx* h, double* vel_max) {
  if (!h || !vel_max) return ICLS_E_ARG;
  launch_maxvel(h->c);
  int rc = read_scalars(h->c);
  if (rc) return rc;
  *vel_max = h->c.h_sc->velmax;
  return ICLS_OK;
}

// ------------------------------------------------------------ checkpoints
namespace {
// the fields of loadflds (loadd.f90:66-103) in file order: (field id, drop)
std::vector<std::pair<int, int>> checkpoint_fields(const Ctx& c) {
  std::vector<std::pair<int, int>> f = {{ICLS_F_U, 1}, {ICLS_F_V, 1}, {ICLS_F_W, 1}, {ICLS_F_PNEW, 1}};
  for (int l = 1; l <= c.P.L; ++l) f.push_back({ICLS_F_LVSET, l});
  f.push_back({ICLS_F_JIEMIAN, 1});
  return f;
}
// the fields of path.hist, whole arrays (halos included): the AB2 and
// pressure history, then the level sets again, whose outer wall-normal
// ghost layers (k = -2, -1, k1+1, k1+2) are carried from step to step
// (boundsls refills only k = 0 and k1) and so are not implied by the interior
std::vector<std::pair<int, int>> hist_fields(const Ctx& c) {
  std::vector<std::pair<int, int>> f;
  for (int id : {ICLS_F_DUOLD, ICLS_F_DVOLD, ICLS_F_DWOLD, ICLS_F_POLD, ICLS_F_PX, ICLS_F_PY, ICLS_F_PZ,
                 ICLS_F_PXOLD, ICLS_F_PYOLD, ICLS_F_PZOLD})
    f.push_back({id, 1});
  for (int l = 1; l <= c.P.L; ++l) f.push_back({ICLS_F_LVSET, l});
  return f;
}
const char kHistMagic[8] = {'I', 'C', 'L', 'S', 'H', 'S', 'T', '1'};

struct Shape3 {
  int lo[3], hi[3];
  long long n() const { return (long long)(hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1); }
  long long at(int i, int j, int k) const {
    return (i - lo[0]) + (long long)(hi[0] - lo[0] + 1) * ((j - lo[1]) + (long long)(hi[1] - lo[1] + 1) * (k - lo[2]));
  }
};
Shape3 shape_of(const icls_ctx* h, int id) {
  Shape3 s;
  icls_field_bounds(h, id, s.lo, s.hi);
  return s;
}
}  // namespace

int icls_write_checkpoint(icls_ctx* h, const char* path, int nr, int history) {
  NEED(h);
  if (!path) return ICLS_E_ARG;
  Ctx& c = h->c;
  const int I = c.P.imax, J = c.P.jmax, K = c.P.kmax;
  std::vector<double> full, in((size_t)I * J * K);
  FILE* f = std::fopen(path, "wb");
  if (!f) return ICLS_E_IO;
  int rc = ICLS_OK;
  for (const auto& fl : checkpoint_fields(c)) {
    const Shape3 sh = shape_of(h, fl.first);
    full.assign((size_t)sh.n(), 0.);
    rc = icls_download_field(h, fl.first, fl.second, full.data());
    if (rc) break;
    size_t q = 0;
    for (int k = 1; k <= K; ++k)
      for (int j = 1; j <= J; ++j)
        for (int i = 1; i <= I; ++i) in[q++] = full[(size_t)sh.at(i, j, k)];
    if (std::fwrite(in.data(), sizeof(double), in.size(), f) != in.size()) { rc = ICLS_E_IO; break; }
  }
  const double info[3] = {c.time, 1. * nr, c.dt};
  if (!rc && std::fwrite(info, sizeof(double), 3, f) != 3) rc = ICLS_E_IO;
  if (std::fclose(f) != 0 && !rc) rc = ICLS_E_IO;
  if (rc || !history) return rc;
  const std::string hp = std::string(path) + ".hist";
  f = std::fopen(hp.c_str(), "wb");
  if (!f) return ICLS_E_IO;
  const int dims[4] = {I, J, K, c.P.L};
  bool ok = std::fwrite(kHistMagic, 1, 8, f) == 8 && std::fwrite(dims, sizeof(int), 4, f) == 4;
  for (const auto& fl : hist_fields(c)) {
    if (!ok) break;
    const Shape3 sh = shape_of(h, fl.first);
    full.assign((size_t)sh.n(), 0.);
    rc = icls_download_field(h, fl.first, fl.second, full.data());
    if (rc) break;
    ok = std::fwrite(full.data(), sizeof(double), full.size(), f) == full.size();
  }
  double norm = 0.;
  if (!rc && ok) {
    rc = read_scalars(c);
    norm = c.h_sc->norm;
  }
  if (!rc && ok) ok = std::fwrite(&norm, sizeof(double), 1, f) == 1 &&
                      std::fwrite(c.init_volume_h.data(), sizeof(double), (size_t)c.P.L, f) == (size_t)c.P.L;
  if (std::fclose(f) != 0) ok = false;
  if (rc) return rc;
  return ok ? ICLS_OK : ICLS_E_IO;
}

int icls_read_checkpoint(icls_ctx* h, const char* path, int* nr) {
  if (!h || !path) return ICLS_E_ARG;
  Ctx& c = h->c;
  const int I = c.P.imax, J = c.P.jmax, K = c.P.kmax;
  std::vector<double> full, in((size_t)I * J * K);
  FILE* f = std::fopen(path, "rb");
  if (!f) return ICLS_E_IO;
  int rc = ICLS_OK;
  for (const auto& fl : checkpoint_fields(c)) {
    if (std::fread(in.data(), sizeof(double), in.size(), f) != in.size()) { rc = ICLS_E_IO; break; }
    const Shape3 sh = shape_of(h, fl.first);
    full.assign((size_t)sh.n(), 0.);  // halos follow from init_program's boundary passes
    size_t q = 0;
    for (int k = 1; k <= K; ++k)
      for (int j = 1; j <= J; ++j)
        for (int i = 1; i <= I; ++i) full[(size_t)sh.at(i, j, k)] = in[q++];
    rc = icls_upload_field(h, fl.first, fl.second, full.data());
    if (rc) break;
  }
  double info[3] = {0., 0., 0.};
  if (!rc && std::fread(info, sizeof(double), 3, f) != 3) rc = ICLS_E_IO;
  std::fclose(f);
  if (rc) return rc;
  rc = icls_init_program(h);
  if (rc) return rc;
  c.time = info[0];
  c.dt = info[2];
  if (nr) *nr = (int)info[1];
  const std::string hp = std::string(path) + ".hist";
  f = std::fopen(hp.c_str(), "rb");
  if (!f) return ICLS_OK;  // the reference's restart: init_program's Euler start
  char magic[8];
  int dims[4];
  bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, kHistMagic, 8) == 0 &&
            std::fread(dims, sizeof(int), 4, f) == 4 && dims[0] == I && dims[1] == J && dims[2] == K &&
            dims[3] == c.P.L;
  for (const auto& fl : hist_fields(c)) {
    if (!ok) break;
    const Shape3 sh = shape_of(h, fl.first);
    full.assign((size_t)sh.n(), 0.);
    ok = std::fread(full.data(), sizeof(double), full.size(), f) == full.size();
    if (ok) rc = icls_upload_field(h, fl.first, fl.second, full.data());
    if (rc) break;
  }
  double norm = 0.;
  std::vector<double> v0((size_t)c.P.L);
  if (ok && !rc) ok = std::fread(&norm, sizeof(double), 1, f) == 1 &&
                      std::fread(v0.data(), sizeof(double), v0.size(), f) == v0.size();
  std::fclose(f);
  if (rc) return rc;
  if (!ok) return ICLS_E_IO;
  CK(cudaMemcpyAsync(&c.dsc->norm, &norm, sizeof(double), cudaMemcpyHostToDevice, c.s));
  CK(cudaMemcpyAsync(c.dvol0, v0.data(), sizeof(double) * v0.size(), cudaMemcpyHostToDevice, c.s));
  CK(cudaStreamSynchronize(c.s));
  c.init_volume_h = v0;
  return check_launch();
}

// disp_cg and disp_speed (write_vtk.f90:438-566) of drop l: sums on the
// device, the two quotients here
int icls_disp(icls_ctx* h, int l, double* cg, double* vel) {
  if (!h || !cg || !vel) return ICLS_E_ARG;
  LARG(h, l);
  Ctx& c = h->c;
  launch_disp(c, l - 1);
  double sm[7];
  CK(cudaMemcpyAsync(sm, c.diag + 7 * kRedBlocks, sizeof(sm), cudaMemcpyDeviceToHost, c.s));
  CK(cudaStreamSynchronize(c.s));
  for (int q = 0; q < 3; ++q) cg[q] = sm[1 + q] / sm[0];
  const double vol = ((c.cfg.lx * c.cfg.ly) * c.cfg.lz) * c.init_volume_h[l - 1];
  for (int q = 0; q < 3; ++q) vel[q] = sm[4 + q] / vol;
  return check_launch();
}

int icls_chkdiv(icls_ctx* h, int istep, double* divtot, double* divmax, int ijk[3]) {
  if (!h) return ICLS_E_ARG;
  return chkdiv(h->c, istep, divtot, divmax, ijk);
}

// chkdt (chkdt.f90:11-105): maxima on the device, the rest on the host
int icls_chkdt(icls_ctx* h, double* dtmax) {
  if (!h || !dtmax) return ICLS_E_ARG;
  Ctx& c = h->c;
  launch_chkdt(c);
  int rc = read_scalars(c);
  if (rc) return rc;
  const Params& P = c.P;
  const icls_config& f = c.cfg;
  const double rho_avr = c.h_sc->rho_avr;
  double speed_conv = (c.h_sc->umax / P.dx + c.h_sc->vmax / P.dy) + c.h_sc->wmax / P.dz;
  const double* g = f.g_unit;
  double gg[6] = {std::fabs(f.iFr * (1. - rho_avr / f.rho1) * g[0]), std::fabs(f.iFr * (1. - rho_avr / f.rho2) * g[0]),
                  std::fabs(f.iFr * (1. - rho_avr / f.rho1) * g[1]), std::fabs(f.iFr * (1. - rho_avr / f.rho2) * g[1]),
                  std::fabs(f.iFr * (1. - rho_avr / f.rho1) * g[2]), std::fabs(f.iFr * (1. - rho_avr / f.rho2) * g[2])};
  double g_max = gg[0];
  for (int q = 1; q < 6; ++q) g_max = std::max(g_max, gg[q]);
  const double h_min = std::min(std::min(P.dx, P.dy), P.dz);
  const double speed_grav = std::sqrt(g_max / h_min);
  const double v1 = std::max(f.miu1 / f.rho1, f.miu2 / f.rho2) * P.visc;
  const double v2 = (2. / (P.dx * P.dx) + 2. / (P.dy * P.dy)) + 2. / (P.dz * P.dz);
  const double speed_visc = v1 * v2;
  const double curv_max = f.TwoD ? 1. / h_min : 2. / h_min;
  const double speed_surf = std::sqrt(curv_max / (f.We * P.rho0 * (h_min * h_min)));
  const double s1 = speed_conv + speed_visc;
  const double speed =
      (s1 + std::sqrt((s1 * s1 + 4. * (speed_grav * speed_grav)) + 4. * (speed_surf * speed_surf))) / 2.;
  *dtmax = 0.5 / speed;
  return ICLS_OK;
}

int icls_ipot(icls_ctx* h, double* dmin) {
  NEED(h);
  Ctx& c = h->c;
  const int L = c.P.L;
  if (L < 2) {
    if (dmin) dmin[0] = 0.;
    return ICLS_OK;
  }
  double* dev = nullptr;
  CK(cudaMallocAsync((void**)&dev, sizeof(double) * L * L, c.s));
  // every pair starts at the ordered bits of 1e3, the reference's initial
  // super_phi (interface.f90:250): the value of a pair with no cell to sweep
  unsigned long long init = 0;
  const double big = 1e3;
  std::memcpy(&init, &big, sizeof(init));
  init |= 0x8000000000000000ull;
  const std::vector<unsigned long long> preset((size_t)L * L, init);
  CK(cudaMemcpyAsync(dev, preset.data(), sizeof(double) * L * L, cudaMemcpyHostToDevice, c.s));
  launch_ipot(c, dev);
  std::vector<unsigned long long> bits((size_t)L * L);
  CK(cudaMemcpyAsync(bits.data(), dev, sizeof(double) * L * L, cudaMemcpyDeviceToHost, c.s));
  CK(cudaFreeAsync(dev, c.s));
  CK(cudaStreamSynchronize(c.s));
  std::vector<double> dt((size_t)L * L, 0.);
  for (size_t q = 0; q < bits.size(); ++q) {
    unsigned long long b = bits[q];
    b = (b & 0x8000000000000000ull) ? (b & 0x7FFFFFFFFFFFFFFFull) : ~b;
    double v;
    std::memcpy(&v, &b, sizeof(v));
    dt[q] = v;
  }
  if (dmin) {
    for (size_t q = 0; q < (size_t)L * L; ++q) dmin[q] = 0.;
    for (int m = 0; m < L - 1; ++m)
      for (int n = m + 1; n < L; ++n) dmin[m + (size_t)L * n] = 0.5 * (dt[m + (size_t)L * n] + dt[n + (size_t)L * m]);
  }
  return ICLS_OK;
}

int icls_probe(icls_ctx* h, int id, int l, int i, int j, int k, double* value) {
  if (!h || !value) return ICLS_E_ARG;
  Ctx& c = h->c;
  int lo[3], hi[3];
  int rc = icls_field_bounds(h, id, lo, hi);
  if (rc) return rc;
  if (i < lo[0] || i > hi[0] || j < lo[1] || j > hi[1] || k < lo[2] || k > hi[2]) return ICLS_E_ARG;
  long long n;
  double* d = field_ptr(c, id, l, &n);
  if (!d) return ICLS_E_ARG;
  const long long nx = hi[0] - lo[0] + 1, ny = hi[1] - lo[1] + 1;
  const long long off = (i - lo[0]) + nx * ((j - lo[1]) + ny * (long long)(k - lo[2]));
  if (c.P.f32 && tfield(id)) {
    float f = 0.f;
    CK(cudaMemcpyAsync(&f, reinterpret_cast<float*>(d) + off, sizeof(float), cudaMemcpyDeviceToHost, c.s));
    CK(cudaStreamSynchronize(c.s));
    *value = f;
    return ICLS_OK;
  }
  CK(cudaMemcpyAsync(value, d + off, sizeof(double), cudaMemcpyDeviceToHost, c.s));
  CK(cudaStreamSynchronize(c.s));
  return ICLS_OK;
}

// one main-loop iteration (main.f90:107-258)
int icls_step(icls_ctx* h, int istep, int begin) {
  NEED(h);
  Ctx& c = h->c;
  c.time = c.time + c.dt;
  int rc;
  if (c.cfg.solveLS) {
    rc = ls_main(c, istep);
    if (rc) return rc;
  }
  launch_stream_vel(c);
  launch_ab2(c);
  int add_pjump = 0;
  if (c.cfg.solveLS) {
    rc = gfm4p(c);
    if (rc) return rc;
    add_pjump = 1;  // fillps, then p = p + p_jump (main.f90:139-142)
  }
  launch_fillps_solver2d(c, 1, add_pjump);  // fillps + solver2d + boundp(p)
  if (c.P.bcy == ICLS_BCY_PERIODIC) {
    launch_correc(c, 1);   // correc + bounduvw + average_vel_at_center + NaN probe
  } else {                 // the y walls change vnew before the cell-centre averages
    launch_correc(c, 0);
    launch_bounduvw(c, c.u, c.v, c.w);
    launch_average_vel(c);
    launch_nan_probe(c);
  }
  launch_pressure_update(c, istep == begin + 1);
  rc = check_launch();
  if (rc) return rc;
  rc = read_scalars(c);
  if (rc) return rc;
  if (c.h_sc->nan_flag) return ICLS_E_NAN;
  if (c.cfg.ioutchk > 0 && istep % c.cfg.ioutchk == 0) {
    rc = chkdiv(c, istep, nullptr, nullptr, nullptr);
    if (rc) return rc;
    c.dt = c.cfg.timestep;  // main.f90:216
  }
  return ICLS_OK;
}

int icls_tube_construction(icls_ctx* h, int l) {
  if (!h) return ICLS_E_ARG;
  LARG(h, l);
  make_full(h->c, l - 1);
  tube_construction(h->c, l - 1);
  return check_launch();
}

int icls_ls_advection(icls_ctx* h, int l) {
  NEED(h);
  LARG(h, l);
  make_full(h->c, l - 1);
  ls_advection(h->c, l - 1);
  return check_launch();
}

int icls_ls_mass_correction(icls_ctx* h, int istep, int l) {
  NEED(h);
  LARG(h, l);
  make_full(h->c, l - 1);
  int rc = ls_mass_correction(h->c, istep, l - 1);
  if (rc) return rc;
  return check_launch();
}

int icls_ls_reinit_main(icls_ctx* h, int istep, int l) {
  NEED(h);
  LARG(h, l);
  make_full(h->c, l - 1);
  if (istep % h->c.cfg.reinit_step == 0) ls_reinit(h->c, l - 1);
  return check_launch();
}

int icls_update_materials(icls_ctx* h) {
  if (!h) return ICLS_E_ARG;
  update_materials(h->c);
  return check_launch();
}

int icls_get_curvature(icls_ctx* h, int l) {
  NEED(h);
  LARG(h, l);
  Ctx& c = h->c;
  make_full(c, l - 1);
  std::vector<LsBatch> b = single(c, l - 1, kStageRows, c_region(c.P, c.win[l - 1].box, 1));
  b[0].t[0].phi0 = c.lv[l - 1];
  b[0].t[0].out = c.curv;
  // the learned form: the network's curvature near the interface, as gfm4p uses it
  const bool mlp = c.cfg.curvature_model == ICLS_CURV_MLP && c.net;
  launch_curvature(c, b[0], c.nrm_m, mlp);
  if (mlp) {
    const int rc = launch_mlp_curvature(c, b[0]);
    if (rc) return rc;
  }
  c.curv_stale = c.nrm_stale = false;
  return check_launch();
}

int icls_band_count(icls_ctx* h, int l, long long* nb_cnt) {
  if (!h || !nb_cnt) return ICLS_E_ARG;
  LARG(h, l);
  CK(cudaMemcpyAsync(nb_cnt, h->c.d_nbcnt + (l - 1), sizeof(long long), cudaMemcpyDeviceToHost, h->c.s));
  CK(cudaStreamSynchronize(h->c.s));
  return ICLS_OK;
}


int icls_profile_enable(icls_ctx* h, int on) {
  if (!h) return ICLS_E_ARG;
  CK(cudaStreamSynchronize(h->c.s));
  h->c.prof.collect();
  h->c.prof.on = on != 0;
  return ICLS_OK;
}

int icls_profile_reset(icls_ctx* h) {
  if (!h) return ICLS_E_ARG;
  CK(cudaStreamSynchronize(h->c.s));
  h->c.prof.collect();
  for (auto& e : h->c.prof.table) { e.total_ms = 0.; e.launches = 0; e.timed = 0; }
  h->c.prof.launches = 0;
  return ICLS_OK;
}

int icls_profile_count(icls_ctx* h, int* n) {
  if (!h || !n) return ICLS_E_ARG;
  CK(cudaStreamSynchronize(h->c.s));
  h->c.prof.collect();
  *n = (int)h->c.prof.table.size();
  return ICLS_OK;
}

int icls_profile_entry(icls_ctx* h, int idx, char* name, int name_len, double* total_ms, long long* launches,
                       long long* timed) {
  if (!h) return ICLS_E_ARG;
  Prof& pr = h->c.prof;
  if (idx < 0 || idx >= (int)pr.table.size()) return ICLS_E_ARG;
  const ProfEntry& e = pr.table[idx];
  if (name && name_len > 0) {
    std::strncpy(name, e.name.c_str(), (size_t)name_len - 1);
    name[name_len - 1] = 0;
  }
  if (total_ms) *total_ms = e.total_ms;
  if (launches) *launches = e.launches;
  if (timed) *timed = e.timed;
  return ICLS_OK;
}

int icls_launch_count(icls_ctx* h, long long* n) {
  if (!h || !n) return ICLS_E_ARG;
  *n = h->c.prof.launches;
  return ICLS_OK;
}

int icls_set_curvature_net(icls_ctx* h, icls_mlp* net) {
  if (!h) return ICLS_E_ARG;
  if (h->c.cfg.curvature_model != ICLS_CURV_MLP) return ICLS_E_CONFIG;
  h->c.net = net;
  return ICLS_OK;
}

int icls_curvature_stats(icls_ctx* h, long long* evaluated, long long* fallbacks, int reset) {
  if (!h) return ICLS_E_ARG;
  Ctx& c = h->c;
  unsigned long long st[2] = {0, 0};
  if (c.mlp_stats) {
    CK(cudaMemcpyAsync(st, c.mlp_stats, sizeof(st), cudaMemcpyDeviceToHost, c.s));
    CK(cudaStreamSynchronize(c.s));
    if (reset) CK(cudaMemsetAsync(c.mlp_stats, 0, sizeof(st), c.s));
  }
  if (evaluated) *evaluated = (long long)st[0];
  if (fallbacks) *fallbacks = (long long)st[1];
  return ICLS_OK;
}

int icls_get_stream(icls_ctx* h, void** stream) {
  if (!h || !stream) return ICLS_E_ARG;
  *stream = (void*)h->c.s;
  return ICLS_OK;
}

}  // extern "C"
