// ctx.h — host-side context of the B200 ICLS hot path and the launchers of
// its kernels.  The context owns every device array of the reference's
// mod_common (src/common.f90:7-71) plus the main-program locals of
// src/main.f90 (duold..dwold, pold, p, p_jump) and the solver tables of
// src/solver.f90:42-47.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "../../include/icls_gpu.h"
#include "icls_common.cuh"
#include "prof.h"

namespace icls {

constexpr int kRedBlocks = 1184;   // 8 x 148 SMs: fixed grid of the reduction kernels
constexpr int kRedThreads = 256;
constexpr int kMaxDropsParam = 256;  // drops whose far-field counts travel as a kernel parameter

// Sweep state of one drop's level set.  Outside valid's write region every
// cell holds the far-field value bg (the stored array there is stale);
// box is the region the current step sweeps.  D is the bounding box of the
// cells that differed from +6dz after the last tube_construction, grow the
// number of cells the non-uniform region can have spread since.
struct DropWin {
  Box3 box;
  Box3 valid;
  double bg = 0.0;        // far field of rows 0..k1
  double bg_ghost = 0.0;  // far field of the ghost rows k<0, k>k1
  bool bg_valid = false;  // bg/bg_ghost hold the far-field values
  bool have_D = false;
  int pending_grow = 0;
  int D[6] = {0, 0, 0, 0, 0, 0};
  int grow = 0;
};

struct Ctx {
  icls_config cfg;
  Params P;
  cudaStream_t s = nullptr;
  int device = 0;

  // shape C
  double *u = nullptr, *v = nullptr, *w = nullptr, *pnew = nullptr, *pold = nullptr, *p = nullptr;
  double *dudt = nullptr, *dvdt = nullptr, *dwdt = nullptr;
  double *px = nullptr, *py = nullptr, *pz = nullptr, *pxold = nullptr, *pyold = nullptr, *pzold = nullptr;
  double *pjump = nullptr, *miu = nullptr, *rho = nullptr, *jiemian = nullptr, *curv = nullptr, *recurv = nullptr;
  double *dheav = nullptr, *kappa = nullptr;
  // shape I
  double *duold[2] = {nullptr, nullptr}, *dvold[2] = {nullptr, nullptr}, *dwold[2] = {nullptr, nullptr};
  int hist = 0;  // which duold buffer holds the current history
  double *rho_u = nullptr, *rho_v = nullptr, *rho_w = nullptr;
  double *ucc = nullptr, *vcc = nullptr, *wcc = nullptr, *nrm_m = nullptr;
  double *ulc = nullptr, *vlc = nullptr, *wlc = nullptr;
  // level sets (shape L): one buffer per drop plus four scratch buffers
  std::vector<double*> lv;
  double* ls_scr[4] = {nullptr, nullptr, nullptr, nullptr};
  uint8_t* mask = nullptr;              // tube mask of the drop being advanced
  long long* d_nbcnt = nullptr;         // band counts per drop
  // Poisson
  double* spec = nullptr;               // compact (1:imax,1:jmax,1:kmax) spectral buffer
  double2* twx = nullptr;               // e^{-2 pi i m/N}, m < N/2, x and y
  double2* twy = nullptr;
  double* xyrt = nullptr;               // eigenvalues (initsolver.f90:76-82)
  double* zpiv = nullptr;               // 1/pivot of the Thomas sweep per (i,j,k)
  double* tri_a = nullptr, *tri_b = nullptr, *tri_c = nullptr;  // (kmax)
  // reductions and device scalars
  double* partials = nullptr;           // kRedBlocks * max(L,4)
  long long* lpartials = nullptr;
  DevScalars* dsc = nullptr;
  double* dvol = nullptr;               // volume(1:L)
  double* dvol0 = nullptr;              // init_volume(1:L)
  double* dmaxchk = nullptr;            // per drop maxchk of the last inflation
  // pinned host mirrors
  double* h_vol = nullptr;
  DevScalars* h_sc = nullptr;
  cudaEvent_t ev_vol = nullptr;
  std::vector<double> init_volume_h;
  std::vector<uint8_t> inflated;        // per drop, last ls_main
  std::vector<uint8_t> vol_dirty;       // volume(l) changed on the device since h_vol
  // host state
  double time = 0.0, dt = 0.0;
  bool initialised = false;
  bool vol_pending = false;
  int last_inflated = 0;
  double P10x27[270];
  Prof prof;
  // per-drop sweep boxes
  std::vector<DropWin> win;
  bool use_boxes = true;
  int* d_bbox = nullptr;                // 6 ints per drop, written by the tube kernel
  int* h_bbox = nullptr;                // pinned copy
  cudaEvent_t ev_bbox = nullptr;
  bool bbox_pending = false;
  std::vector<double> outside;          // interior cells outside each drop's box
};

// ---- kernel launchers (defined in the k_*.cu files) -----------------------
void set_pseudo_inverse(const double* P270, cudaStream_t s);

// level set (k_levelset.cu)
dim3 grid_of(const int* r0, const int* r1);
Box3 full_box(const Params& P);
Box3 c_region(const Params& P, const Box3& b, int apron);
void launch_tube(Ctx& c, const Box3& b, const Box3& vin, double bgin, double bgg, const double* in, double* out,
                 long long* cnt, int* bbox);
void launch_adv_stage(Ctx& c, const Box3& b, double bg_out, double bgg_out, int scheme, int stage1,
                      const double* phi0, const double* phis, double a, double bb, double fdt, const double* vu,
                      const double* vv, const double* vw, double* out);
void launch_reinit_stage(Ctx& c, const Box3& b, double bg_out, double bgg_out, int stage, const double* phi0,
                         const double* phis, const double* orig, double dtau, double* out);
void launch_reinit_check(Ctx& c, int it, int maxiter, double thr, double far);
void launch_reinit_reset(Ctx& c, int maxiter);
void launch_heaviside_drop(Ctx& c, const Box3& b, const double* phi, int l, int first);
void launch_fill(Ctx& c, double* a, long long n, double v);
void launch_materials_final(Ctx& c, const double* outside);
void launch_inflate_sums(Ctx& c, const Box3& b, const double* phi, int l, double outside);
void launch_inflate_vel(Ctx& c, const Box3& b);
void launch_copy(Ctx& c, double* dst, const double* src, long long n);
void launch_boundmls(Ctx& c, double* phi);
void launch_materialize(Ctx& c, const Box3& b, double bg, double bgg, double* phi);

// interface / GFM (k_gfm.cu)
void launch_curvature(Ctx& c, const Box3& b, const double* phi, double* curv_out, double* nrm_m_out);
void launch_recurvature(Ctx& c, const Box3& b, const double* phi, const double* curv_in, double* out);
void launch_jumps(Ctx& c, const Box3& b, const double* phi, const double* cv, int first);
void launch_ipot(Ctx& c, double* dmin_dev);

// Navier-Stokes (k_navier.cu)
void launch_ab2(Ctx& c);
void launch_mom_main(Ctx& c, double* du, double* dv, double* dw);
void launch_fillps(Ctx& c, int add_pjump);
void launch_add_pjump(Ctx& c);
void launch_correc(Ctx& c, int fused_bc);
void launch_bounduvw(Ctx& c, double* u, double* v, double* w);
void launch_boundp(Ctx& c, double* p);
void launch_average_vel(Ctx& c);
void launch_pressure_update(Ctx& c, int first);
void launch_stream_vel(Ctx& c);
void launch_chkdiv(Ctx& c);
void launch_chkdt(Ctx& c);
void launch_maxvel(Ctx& c);
void launch_nan_probe(Ctx& c);

// Poisson (k_poisson.cu)
void poisson_setup(Ctx& c);
void launch_solver2d(Ctx& c, int write_halos);

}  // namespace icls
