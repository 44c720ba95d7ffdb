// ctx.h — host-side context of the B200 ICLS hot path and the launchers of
// its kernels.  The context owns every device array of the reference's
// mod_common (src/common.f90:7-71) plus the main-program locals of
// src/main.f90 (duold..dwold, pold, p, p_jump) and the solver tables of
// src/solver.f90:42-47.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "../../include/icls_gpu.h"
#include "icls_common.cuh"
#include "prof.h"

namespace icls {

constexpr int kRedBlocks = 1184;   // 8 x 148 SMs: fixed grid of the reduction kernels
constexpr int kCosqMaxN = 768;     // longest z line of solver2d_cos (one shared-memory tile)
constexpr int kRedThreads = 256;
constexpr int kMaxDropsParam = 256;  // drops whose far-field counts travel as a kernel parameter

constexpr int kTasks = 64;          // drops per batched launch (tasks travel as a kernel parameter)
constexpr int TBX = 32, TBY = 8;    // column tile of a batched launch

// One drop's share of a batched launch.  A block of TBX x TBY threads
// sweeps one column tile of the region over one chunk of z rows, each
// thread walking its column upwards: chunk m covers rows z0 + m*kc ..
// z0 + (m+1)*kc - 1, the last chunk runs to z1.  Every chunk holds at least
// kc rows, so the rows a wall row extrapolates from lie in its chunk.
struct LsTask {
  Region r;
  int tx, ty, nch, kc;
  int l, flat;           // flat: a block takes 256 consecutive columns (else TBX x TBY tiles)
  double bg, bgg;        // far-field values of the apron: rows 0..k1 / ghost rows
  const double* phi0;    // RK base (read at the thread's own cell only)
  const double* phis;    // stage input (stencil reads)
  const double* orig;    // reinitialisation: sgn source
  double* out;
  uint8_t* mask;         // the drop's band mask (tube writes, advection reads)
  Region vin;            // tube: phi0 holds valid data on vin's written cells,
  double bgin, bggin;    //       these far-field values elsewhere
  double far;            // reinitialisation: change of the far field this iteration
};
struct LsBatch {
  int n;
  int start[kTasks + 1];  // first block of each task
  LsTask t[kTasks];
};

// per-drop state of the reinitialisation early exit (levelset.f90:827-835)
struct ReinitState {
  double residual;  // max |phi_new - phi_0| of the running iteration
  double last;      // residual of the last completed iteration
  int done;         // residual < dz**5 reached
  int iters;
};

// Sweep state of one drop's level set.  Outside valid's written cells every
// cell holds the far-field value bg (the stored array there is stale);
// box is the region the current step sweeps.  The band span (Dxa, Dxn),
// (Dya, Dyn), [Dz0, Dz1] covers the cells that differed from +6dz after the
// last tube_construction, grow the number of cells the non-uniform region
// can have spread since.
struct DropWin {
  Region box;
  Region valid;
  double bg = 0.0;        // far field of rows 0..k1
  double bg_ghost = 0.0;  // far field of the ghost rows k<0, k>k1
  bool bg_valid = false;  // bg/bg_ghost hold the far-field values
  bool have_D = false;
  int pending_grow = 0;
  int Dxa = 1, Dxn = 0, Dya = 1, Dyn = 0, Dz0 = 0, Dz1 = -1;
  int grow = 0;
};

// z rows per chunk of update_materials' Heaviside sweep (one exact partial
// sum per column tile and chunk)
constexpr int kHeavRows = 8;

struct Ctx {
  // tensor maps of the TMA predictor for up to four sets of its 18 input
  // pointers (the AB2 history and the p_x/p_xold pairs alternate between
  // buffers), keyed by the pointers themselves
  alignas(64) unsigned char ab2_maps[4][18 * 128];
  const void* ab2_keys[4][18] = {};
  int ab2_nmaps = 0, ab2_next = 0;
  bool ab2_tma_failed = false;  // a map could not be encoded: use the ring
  bool ab2_ring = true;  // FP64 predictor on the cp.async ring (else TMA: ICLS_AB2=tma)
  bool materials_rows1 = false;  // materials one row per thread (ICLS_MATERIALS=rows1)
  bool correc_shapec = false;  // fused correction one thread per shape-C cell (ICLS_CORREC=shapec)
  icls_config cfg;
  Params P;
  cudaStream_t s = nullptr;
  int device = 0;

  // shape C
  double *u = nullptr, *v = nullptr, *w = nullptr, *pnew = nullptr, *pold = nullptr, *p = nullptr;
  double *dudt = nullptr, *dvdt = nullptr, *dwdt = nullptr;
  double *px = nullptr, *py = nullptr, *pz = nullptr, *pxold = nullptr, *pyold = nullptr, *pzold = nullptr;
  double *pjump = nullptr, *miu = nullptr, *rho = nullptr, *jiemian = nullptr;
  double *curv = nullptr;      // curv_cmn: re_curvature of the last drop (get_curvature in TwoD)
  double *dheav = nullptr, *kappa = nullptr;
  // shape I
  double *duold[2] = {nullptr, nullptr}, *dvold[2] = {nullptr, nullptr}, *dwold[2] = {nullptr, nullptr};
  int hist = 0;  // which duold buffer holds the current history
  double *rho_u = nullptr, *rho_v = nullptr, *rho_w = nullptr;
  double *ucc = nullptr, *vcc = nullptr, *wcc = nullptr, *nrm_m = nullptr;
  double *ulc = nullptr, *vlc = nullptr, *wlc = nullptr;
  // level sets (shape L): one buffer per drop
  std::vector<double*> lv;
  // working buffers of the drops of one group (drop l uses member l % G):
  // three level-set stage buffers, the band mask, get_curvature and
  // re_curvature outputs.  G is sized to the free HBM at creation.
  struct Member {
    double *s1 = nullptr, *s2 = nullptr, *s3 = nullptr;  // shape L
    double *fit = nullptr, *cv = nullptr;                // shape C
    uint8_t* mask = nullptr;                             // shape I
  };
  std::vector<Member> mem;
  long long* d_nbcnt = nullptr;         // band counts per drop
  // Poisson
  double* spec = nullptr;               // compact (1:imax,1:jmax,1:kmax) spectral buffer
  double2* twx = nullptr;               // e^{-2 pi i m/N}, m < N/2, x and y
  double2* twy = nullptr;
  double* xyrt = nullptr;               // distinct eigenvalue sums (initsolver.f90:76-82)
  double* zpiv = nullptr;               // 1/pivot of the Thomas sweep per distinct (xrt, yrt) and k
  double* tri_a = nullptr, *tri_b = nullptr, *tri_c = nullptr;  // (kmax), or (jtot) for solver2d_cos
  // solver2d_cos: the VCOSQB and VCOSQF matrices (kmax x kmax, row m = output
  // m), and v_inflow(0:i1,0:k1) of the inflow boundary
  double* cosb = nullptr, *cosf = nullptr;
  double2* czw = nullptr;               // (cos, sin)(pi k/(2 kmax)), k < kmax
  double* vin = nullptr;
  // reductions and device scalars
  double* partials = nullptr;           // kRedBlocks * max(L,4)
  double* diag = nullptr;               // disp partials: 7 * kRedBlocks, then the 7 sums
  long long* lpartials = nullptr;
  DevScalars* dsc = nullptr;
  double* dvol = nullptr;               // volume(1:L)
  double* dvol0 = nullptr;              // init_volume(1:L)
  double* dvolnow = nullptr;            // gain-one trigger: each drop's volume after its reinitialisation
  // band-list advection: the band cells of a batch (8 bytes each) and their number
  void* band_list = nullptr;
  int* band_count = nullptr;
  long long band_cap = 0;
  bool adv_column = true;               // the one-kernel column stage (else the band-list split: ICLS_ADV=band)
  double* h_volnow = nullptr;           // pinned host copy
  double* dmaxchk = nullptr;            // per drop maxchk of the last inflation
  ReinitState* drs = nullptr;           // per drop
  double* stage = nullptr;              // precision form: FP64 staging of one field (upload/download)
  double* hpart = nullptr;              // per-tile exact sums of H (XSum), red_cap per drop
  int red_cap = 0;                      // column tiles of a whole x-y plane
  int hcap = 0;                         // Heaviside partials per drop: red_cap x the z chunks of shape C
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
  // 10 ints per drop, written by the tube kernel: minima then maxima of
  // {x, x shifted by imax/2, y, y shifted by jmax/2, z} over the band
  int* d_bbox = nullptr;
  int* h_bbox = nullptr;                // pinned copy
  // learned curvature (curvature_model = ICLS_CURV_MLP): the attached
  // network and the buffers of the gathered interface cells
  icls_mlp* net = nullptr;
  float* mlp_X = nullptr;
  void* mlp_rec = nullptr;
  int* mlp_count = nullptr;
  unsigned long long* mlp_stats = nullptr;  // cells evaluated, fallbacks to the stencil
  int mlp_cap = 0;
  bool curv_stale = false;              // curv / normal%m hold more than the last drop
  bool nrm_stale = false;
  cudaEvent_t ev_bbox = nullptr;
  bool bbox_pending = false;
  std::vector<double> outside;          // interior cells outside each drop's box
};

// the 10x27 least-squares pseudo-inverse for spacings (dx, dy, dz) (capi.cu)
void pseudo_inverse(double dx, double dy, double dz, double* out);

// ---- kernel launchers (defined in the k_*.cu files) -----------------------
void set_pseudo_inverse(const double* P270, cudaStream_t s);

// level set (k_levelset.cu)
Region full_region(const Params& P);
bool region_full(const Params& P, const Region& r);
Region c_region(const Params& P, const Region& r, int apron);
void set_tiles(LsBatch& b, int kc, bool flat = true);
void launch_tube(Ctx& c, const LsBatch& b);
void launch_adv_stage(Ctx& c, const LsBatch& b, int scheme, int stage1, double a, double bb, double fdt,
                      const double* vu, const double* vv, const double* vw);
void launch_reinit_stage(Ctx& c, const LsBatch& b, int stage, double dtau);
void launch_reinit_reset(Ctx& c, const LsBatch& b, int maxiter);
void launch_reinit_check(Ctx& c, const LsBatch& b, int it, int maxiter, double thr);
void launch_heaviside(Ctx& c, const LsBatch& b);
void launch_fill(Ctx& c, double* a, long long n, double v, bool tfield);
void launch_materials_final(Ctx& c, const double* outside, const int* ntiles);
void launch_inflate_sums(Ctx& c, const LsBatch& b, double outside);
void launch_inflate_vel(Ctx& c, const LsBatch& b);
void launch_region_copy(Ctx& c, const LsBatch& b);
void launch_gain(Ctx& c, const LsBatch& b, double outside);
void launch_region_blend(Ctx& c, const LsBatch& b);
void launch_band_list(Ctx& c, const LsBatch& b);
void launch_adv_split(Ctx& c, const LsBatch& b, int scheme, int stage1, double a, double bb, double fdt,
                      const double* vu, const double* vv, const double* vw, long long need);
void launch_volume_now(Ctx& c, const LsBatch& b, double outside);
void launch_copy(Ctx& c, double* dst, const double* src, long long n);
void launch_boundmls(Ctx& c, double* phi);
void launch_materialize(Ctx& c, const Region& r, double bg, double bgg, double* phi);
void launch_to_float(Ctx& c, double* dst_f32, const double* src, long long n);
void launch_to_double(Ctx& c, double* dst, const double* src_f32, long long n);

// interface / GFM (k_gfm.cu); the tasks carry shape-C regions
// curvature: phi0 -> out (+ normal%m); recurvature: phis -> out; jumps: phi0, phis
// A near-interface cell recorded for the learned curvature: task q of the
// batch, interior cell (i, j, k)
struct MlpCell {
  int q, i, j, k;
};
// get_curvature over the batch; with collect, also records the computed
// cells with |phi| <= 4dz for the network (count reset here)
void launch_curvature(Ctx& c, const LsBatch& b, double* nrm_m_out, bool collect = false);
bool fft_length_ok(int n, bool y_pass, int imax);
void launch_recurvature(Ctx& c, const LsBatch& b);
void launch_jumps(Ctx& c, const LsBatch& b);
void launch_ipot(Ctx& c, double* dmin_dev);

// learned curvature (k_mlp.cu)
int launch_mlp_curvature(Ctx& c, const LsBatch& b);
int mlp_buffers(Ctx& c, int cap);
int mlp_constants();

// Navier-Stokes (k_navier.cu)
void launch_ab2(Ctx& c);
void launch_mom_main(Ctx& c, double* du, double* dv, double* dw);
void launch_fillps(Ctx& c, int add_pjump);
void launch_add_pjump(Ctx& c);
// fused_bc: with bounduvw, the cell-centre velocities and the NaN probe
void launch_correc(Ctx& c, int fused_bc);
void launch_bounduvw(Ctx& c, double* u, double* v, double* w);
// tfield: the array holds the form's field type (FP32 in the precision form)
void launch_boundp(Ctx& c, double* p, bool tfield = false);
// the y-wall rows of bounduvw / boundp (bound.f90:81-282) for bc_y != periodic,
// applied after the periodic halos (i = 1..imax, k = 1..kmax)
void launch_ywalls_uvw(Ctx& c, double* u, double* v, double* w);
void launch_ywalls_p(Ctx& c, double* p);
void launch_nan_probe(Ctx& c);
// drop l's band box as a whole-array tube sweep would measure it, into d_bbox
void launch_band_extents(Ctx& c, int l);
// dst(j,k) = d(ioff + nx j + nx ny k) in FP64 (d holds float when f32)
void launch_gather_plane_x(Ctx& c, const double* d, bool f32, long long nx, long long ny, long long ioff, int n1,
                           int n2, double* dst);
void launch_average_vel(Ctx& c);
void launch_pressure_update(Ctx& c, int first);
void launch_stream_vel(Ctx& c);
void launch_chkdiv(Ctx& c);
void launch_chkdt(Ctx& c);
void launch_maxvel(Ctx& c);
void launch_nan_probe(Ctx& c);
// drop l's band box as a whole-array tube sweep would measure it, into d_bbox
void launch_band_extents(Ctx& c, int l);
// dst(j,k) = d(ioff + nx j + nx ny k) in FP64 (d holds float when f32)
void launch_gather_plane_x(Ctx& c, const double* d, bool f32, long long nx, long long ny, long long ioff, int n1,
                           int n2, double* dst);

// Poisson (k_poisson.cu)
void poisson_setup(Ctx& c);
void launch_solver2d(Ctx& c, int write_halos);
// fillps (+ p_jump when add) and solver2d, fillps folded into the solve's
// first pass where it can be
void launch_fillps_solver2d(Ctx& c, int write_halos, int add);
void launch_disp(Ctx& c, int l);

}  // namespace icls
