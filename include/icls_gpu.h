/*
 * icls_gpu.h — C ABI of the B200 (sm_100a) implementation of the ICLS
 * per-timestep hot path.
 *
 * Every entry point replaces one subroutine that the ICLS driver
 * (src/main.f90:103-291 of GeZhouyang/ICLS-release) calls, or one of the
 * routines those subroutines are built from.  The reference keeps its state
 * in Fortran module globals (src/common.f90:7-71); here an opaque context
 * owns the same arrays in HBM, one GPU holds the whole domain, and the
 * Fortran index space of every array is preserved:
 *
 *   element (i,j,k) of an array with Fortran bounds (lo0:hi0,lo1:hi1,lo2:hi2)
 *   sits at (i-lo0) + n0*((j-lo1) + n1*(k-lo2)),  n = hi-lo+1,
 *
 * so icls_upload_field / icls_download_field are plain copies of the
 * Fortran arrays.  All calls take plain pointers and sizes; no C++ or
 * torch types cross this boundary.  Every call returns an int status
 * (ICLS_OK = 0).  Calls on one context are stream-ordered on that
 * context's CUDA stream; calls that return host scalars synchronise.
 * A context is used by one host thread at a time.
 */
#ifndef ICLS_GPU_H
#define ICLS_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (the reference stops the program instead) ---------- */
enum {
  ICLS_OK = 0,
  ICLS_E_CONFIG = 1,      /* invalid or unsupported configuration          */
  ICLS_E_CUDA = 2,        /* a CUDA runtime call failed                    */
  ICLS_E_NAN = 3,         /* NaN in vnew(1,1,1)          (main.f90:207-210) */
  ICLS_E_DIVERGENCE = 4,  /* max|div| > 1e-12 after step 0 (chkdiv.f90:60) */
  ICLS_E_ARG = 5,         /* bad argument (field id, drop index, pointer)  */
  ICLS_E_NOMEM = 6,       /* device allocation failed                      */
  ICLS_E_STATE = 7,       /* call made before icls_init_program            */
  ICLS_E_UNSUPPORTED = 8, /* scheme/option not built into this library    */
  ICLS_E_SIZE = 9,        /* grid larger than icls_chkdiv_noalloc handles */
  ICLS_E_IO = 10,         /* checkpoint file could not be written or read  */
  ICLS_E_TIMEOUT = 11     /* a kernel's bounded wait on its own pipeline
                             gave up (the step's results are invalid)     */
};

/* ---- scheme selectors (param.f90 / mod_param_ls character parameters) */
enum { ICLS_HOUC5 = 0, ICLS_WENO5 = 1 };              /* ls_adv_space, i_space */
enum { ICLS_SPEED_UNFM = 0, ICLS_SPEED_CURV = 1 };    /* ispeed_dependence     */
enum { ICLS_FP64 = 0, ICLS_FP32 = 1 };                /* precision form        */
enum { ICLS_CURV_STENCIL = 0, ICLS_CURV_MLP = 1 };    /* curvature model       */
/* BC_in_y (param.f90:115): the y boundary of velocity and pressure, and
 * with it the pressure solver (main.f90:147-153): periodic -> solver2d;
 * walls, inflow/outflow, outflow/outflow -> solver2d_cos               */
enum { ICLS_BCY_PERIODIC = 0, ICLS_BCY_WALLS = 1, ICLS_BCY_INOUT = 2, ICLS_BCY_OUTOUT = 3 };
/* NS_conv (param.f90:135).  'WENO5' stops the reference in boundfu
 * (bound.f90:310-322: "WENO5 is not fully implemented yet"); icls_create
 * returns ICLS_E_UNSUPPORTED for it.                                    */
enum { ICLS_NS_CNTR2 = 0, ICLS_NS_WENO5 = 1 };

/*
 * Runtime configuration.  Restates the compile-time parameters of
 * src/param.f90 (grid 27-38, dt 47, materials 58-63, Re/We/iFr 69-77,
 * flags 93-172) and src/param.f90 module mod_param_ls (199-275).
 * BC_in_y and NS_conv are selectable (bc_y, ns_conv).  Fixed choices of
 * the reference defaults that this path implements: BC_in_z='Dirichl',
 * NS_diff_discretization='del', surface_tension_method='GFM',
 * ls_adv_time='RK3', ls_reinit_time='RK3', ls_reinit_space='WENO5',
 * attractive=.false., Riblet=.false., Contact_line=.false.
 */
typedef struct icls_config {
  int itot, jtot, ktot;          /* grid cells (param.f90:27)                */
  int lmax;                      /* number of level sets (param.f90:170)     */
  double lx, ly, lz;             /* domain lengths (param.f90:33-35)         */
  double timestep;               /* fixed dt (param.f90:47, main.f90:216)    */
  double rho1, rho2, miu1, miu2; /* param.f90:58-60                          */
  double Re, We, iFr;            /* param.f90:69-71                          */
  double g_unit[3];              /* param.f90:77                             */
  double v_wall_lower;           /* v at z=0 wall   (bound.f90:29-35)        */
  double v_wall_upper;           /* v at z=lz wall  (bound.f90:29-35)        */
  int TwoD;                      /* param.f90:94                             */
  int constPoi;                  /* param.f90:96 (driving gradient)          */
  int solveLS;                   /* param.f90:163                            */
  int ls_adv_space;              /* ICLS_HOUC5 / ICLS_WENO5 (param.f90:216)  */
  int re_initialization;         /* param.f90:164                            */
  int reinit_step;               /* param.f90:230                            */
  int reinit_iter_max;           /* param.f90:233                            */
  int mass_correction;           /* param.f90:165                            */
  int inflate_step;              /* param.f90:258                            */
  int ispeed_dependence;         /* ICLS_SPEED_* (param.f90:259)             */
  int i_space;                   /* ICLS_HOUC5 / ICLS_WENO5 (param.f90:266)  */
  int ioutchk;                   /* chkdiv/chkdt cadence (param.f90:85)      */
  int precision;                 /* ICLS_FP64 (plain) / ICLS_FP32 form       */
  int curvature_model;           /* ICLS_CURV_STENCIL / ICLS_CURV_MLP        */
  double mlp_fallback_tol;       /* |k_mlp-k_plain|*dx above which the plain
                                    stencil value is kept (MLP form only)   */
  int bc_y;                      /* ICLS_BCY_* (param.f90:115)               */
  int ns_conv;                   /* ICLS_NS_* (param.f90:135)                */
  double mass_threshold;         /* |V-V0|/V0 above which ls_mass_correction
                                    inflates a drop; 0 = the reference's
                                    fixed 1e-5 (levelset.f90:382); any
                                    value > 0 overrides it                  */
  int mass_gain_one;             /* 0: the reference's inflation
                                    (levelset.f90:407-582); 1: the same
                                    inflation blended with the level set
                                    before it so that it removes exactly the
                                    measured volume error (no counterpart in
                                    the reference)                          */
} icls_config;

/* Fill *cfg with the reference defaults of src/param.f90 for a 3-D run. */
void icls_config_default(icls_config* cfg);

/* ---- field identifiers and their Fortran bounds ------------------------
 *  shape C: (0:i1,0:j1,0:k1)          cell/face arrays with one halo layer
 *  shape I: (1:imax,1:jmax,1:kmax)    interior-only arrays
 *  shape L: (-2:i1+2,-2:j1+2,-2:k1+2) level set with three halo layers
 */
enum {
  ICLS_F_U = 0, ICLS_F_V, ICLS_F_W,            /* unew,vnew,wnew       C */
  ICLS_F_PNEW, ICLS_F_POLD, ICLS_F_P,          /* pnew, pold, p        C */
  ICLS_F_DUDT, ICLS_F_DVDT, ICLS_F_DWDT,       /* predicted velocity   C */
  ICLS_F_DUOLD, ICLS_F_DVOLD, ICLS_F_DWOLD,    /* AB2 history          I */
  ICLS_F_PX, ICLS_F_PY, ICLS_F_PZ,             /* GFM face jumps       C */
  ICLS_F_PXOLD, ICLS_F_PYOLD, ICLS_F_PZOLD,    /* previous jumps       C */
  ICLS_F_PJUMP,                                /* Laplacian of jump    C */
  ICLS_F_MIU, ICLS_F_RHO, ICLS_F_JIEMIAN,      /* materials            C */
  ICLS_F_RHO_U, ICLS_F_RHO_V, ICLS_F_RHO_W,    /* face densities       I */
  ICLS_F_UCC, ICLS_F_VCC, ICLS_F_WCC,          /* cell-centre velocity I */
  ICLS_F_CURV,                                 /* curv_cmn             C */
  ICLS_F_NORMAL_M,                             /* normal%m             I */
  ICLS_F_LVSET,                                /* lvset(:,:,:,l)       L */
  ICLS_F_COUNT
};

/* Scalars of the reference state (common.f90 / main.f90 locals). */
typedef struct icls_scalars {
  double time, dt;
  double rho_avr;        /* misc.f90:173                          */
  double v_bulk;         /* misc.f90:642-655                      */
  double norm_old;       /* main.f90:183                          */
  double maxchk_glb;     /* levelset.f90:384,521                  */
  double reinit_residual;/* last levelset.f90:831 residual        */
  int reinit_iters;      /* last levelset.f90:834-837 iteration   */
  int last_inflated;     /* number of drops inflated in last step */
} icls_scalars;

typedef struct icls_ctx icls_ctx;

/* ---- lifetime -------------------------------------------------------- */
int icls_create(const icls_config* cfg, icls_ctx** out);
int icls_destroy(icls_ctx* ctx);
int icls_field_bounds(const icls_ctx* ctx, int field_id, int lo[3], int hi[3]);
/* l is the 1-based level-set index for ICLS_F_LVSET, ignored otherwise. */
int icls_upload_field(icls_ctx* ctx, int field_id, int l, const double* host);
int icls_download_field(icls_ctx* ctx, int field_id, int l, double* host);
int icls_get_scalars(icls_ctx* ctx, icls_scalars* out);
/* volume(1:lmax) and init_volume(1:lmax) (common.f90:52). */
int icls_get_volumes(icls_ctx* ctx, double* volume, double* init_volume);
int icls_synchronize(icls_ctx* ctx);
int icls_status_string(int code, char* buf, int n);

/* ---- initialisation: init_program(begin=0,...) (init.f90:22-117) -------
 * After u,v,w,pnew and lvset(:,:,:,1:lmax) are uploaded: init_matrix,
 * initsolver, dt=timestep, bounduvw, boundmls, boundp, cell-centre
 * velocities, update_materials, init_volume=volume, mom_main -> duold,
 * pold=pnew, p_?old=p_? (=0).                                          */
int icls_init_program(icls_ctx* ctx);

/* ---- the subroutines main.f90 calls (main.f90:103-291) ---------------- */
int icls_ls_main(icls_ctx* ctx, int istep);                 /* levelset.f90:28-76   */
int icls_average_stream_vel(icls_ctx* ctx, double* v_bulk); /* misc.f90:642-655     */
/* v_inflow(0:i1,0:k1) (common.f90:36), i fastest, the inflow profile of
 * bc_y = ICLS_BCY_INOUT at the y = 0 boundary (bound.f90:118-130); the
 * reference fills it in inflow_profile (init.f90:418-455).  Zero until set. */
int icls_set_inflow(icls_ctx* ctx, const double* v_inflow);
/* The plane i = const of a field, for 2-D output (post2d, output.f90:179-432):
 * out(j,k) over the field's own j and k bounds, j fastest, FP64.          */
int icls_download_plane_x(icls_ctx* ctx, int id, int l, int i, double* out);
/* The timestep.txt record of main.f90:243-256: rec = (istep, time, dt,
 * massloss = sum_l (1 - volume(l)/init_volume(l)), dmin(1,2)/dz from ipot
 * (0 with one drop), maxchk_glb).  Runs ipot when lmax >= 2.            */
int icls_timestep_record(icls_ctx* ctx, int istep, double rec[6]);
int icls_ab2(icls_ctx* ctx);                                /* ab2.f90:21-138       */
int icls_fillps(icls_ctx* ctx);                             /* fillps.f90:13-57     */
int icls_gfm4p(icls_ctx* ctx);                              /* gfm.f90:17-267       */
int icls_add_pjump(icls_ctx* ctx);                          /* main.f90:142         */
int icls_solver2d(icls_ctx* ctx);                           /* solver.f90:68-196    */
int icls_boundp(icls_ctx* ctx, int field_id);               /* bound.f90:182-287    */
int icls_correc(icls_ctx* ctx);                             /* correc.f90:15-44     */
int icls_bounduvw(icls_ctx* ctx, int field_id_u);           /* bound.f90:15-177; U or DUDT triple */
int icls_pressure_update(icls_ctx* ctx, int istep, int begin); /* main.f90:164-185  */
int icls_average_vel_at_center(icls_ctx* ctx);              /* misc.f90:587-604     */
int icls_max_vel_at_center(icls_ctx* ctx, double* vel_max); /* misc.f90:610-636     */
/* disp_cg, disp_speed (write_vtk.f90:438-566): drop l's centroid of its cells with
 * phi <= 1.5dz, cg[3], and velocity sum ucc dV (1 - H_l) / (lx ly lz init_volume(l)), vel[3] */
int icls_disp(icls_ctx* ctx, int l, double cg[3], double vel[3]);

/* ---- checkpoint / restart -----------------------------------------------
 * loadflds(1, nr) (loadd.f90:66-103): the file `path` (the reference names it
 * datadir//'fld'//nr, 7 digits) holds u, v, w, pnew, lvset(1..lmax), jiemian,
 * each over the interior (itot x jtot x ktot FP64, i fastest, then j, then
 * k), then (time, nr, dt).  With history != 0 the file `path`.hist also
 * holds what the reference does not keep (it restarts with an Euler step,
 * init.f90:90): the AB2 history duold, dvold, dwold, pold, p_x, p_y, p_z
 * and their previous values, the whole level-set arrays (boundsls refills
 * only the first wall ghost layer, so the outer two carry over from step
 * to step), the pressure-normalisation mean and the initial drop volumes,
 * so that a restart continues the run exactly (call icls_step with
 * begin = 0).  Whole arrays are stored in the field's own layout.        */
int icls_write_checkpoint(icls_ctx* ctx, const char* path, int nr, int history);
/* loadflds(0, nr) (loadd.f90:28-64) into a created context, then
 * init_program; the history of `path`.hist is restored when that file
 * exists.  *nr = the step the file was written at.                       */
int icls_read_checkpoint(icls_ctx* ctx, const char* path, int* nr);
/* Returns ICLS_E_DIVERGENCE when max|div| > 1e-12 and istep != 0.        */
int icls_chkdiv(icls_ctx* ctx, int istep, double* divtot, double* divmax,
                int ijk[3]);                                /* chkdiv.f90:10-90     */
int icls_chkdt(icls_ctx* ctx, double* dtmax);               /* chkdt.f90:11-105     */
int icls_ipot(icls_ctx* ctx, double* dmin);                 /* interface.f90:225-277; dmin(lmax,lmax) column-major */
/* Value of one element of a field (the NaN probe of main.f90:207).       */
int icls_probe(icls_ctx* ctx, int field_id, int l, int i, int j, int k, double* value);

/* One full main-loop iteration, main.f90:107-210 (time += dt, ls_main,
 * average_stream_vel, ab2, fillps, gfm4p, p += p_jump, solver2d, boundp,
 * correc, bounduvw, pressure update, average_vel_at_center, NaN check),
 * issued as one stream-ordered sequence with no host synchronisation
 * except where the reference's branches depend on a device scalar.     */
int icls_step(icls_ctx* ctx, int istep, int begin);

/* ---- the routines those subroutines are built from -------------------- */
int icls_tube_construction(icls_ctx* ctx, int l);           /* levelset.f90:87-197  */
int icls_ls_advection(icls_ctx* ctx, int l);                /* levelset.f90:208-335 */
int icls_ls_mass_correction(icls_ctx* ctx, int istep, int l); /* levelset.f90:377-400 */
int icls_ls_reinit_main(icls_ctx* ctx, int istep, int l);   /* levelset.f90:592-612 */
int icls_update_materials(icls_ctx* ctx);                   /* misc.f90:79-290      */
int icls_get_curvature(icls_ctx* ctx, int l);               /* interface.f90:20-119 -> CURV, NORMAL_M */
/* (with curvature_model ICLS_CURV_MLP and a network attached, CURV near drop
 * l's interface is the network's, with the per-cell fallback gfm4p uses) */
/* Number of band cells of drop l after the last tube_construction
 * (nb_cnt, levelset.f90:158).                                           */
int icls_band_count(icls_ctx* ctx, int l, long long* nb_cnt);

/* ---- learned interface curvature ----
 * No counterpart in the reference: the network that replaces the
 * get_curvature stencil (interface.f90:20-119) near the interface in the
 * learned form.  27 -> 128 -> 128 -> 64 -> 1 SiLU MLP, BF16 weights and
 * activations on tcgen05 tiles (the FP32 inputs enter as BF16 hi + lo
 * pairs), FP32 accumulation and FP32 Adam; input the features of the
 * stencil (phi(x + o dx) - phi(x)) / dx, o in {-1,0,1}^3 (z outer, x inner):
 * the stencil minus its least-squares linear part and the unit gradient,
 * output the correction to the stencil's kappa * dx (learned kappa =
 * kappa_stencil + output / dx).  Training samples come from seeded spheres and
 * ellipsoids (exact signed distance) with the least-squares curvature of a
 * 4x refined stencil as label.  All arrays named "device" live in GPU memory. */
typedef struct icls_mlp icls_mlp;
#define ICLS_MLP_PARAMS 29057
int icls_mlp_create(icls_mlp** out, unsigned long long seed);
int icls_mlp_destroy(icls_mlp* m);
/* training and held-out samples; n_train a power of two */
int icls_mlp_make_data(icls_mlp* m, unsigned long long seed, long long n_train, long long n_hold);
/* Adam on the squared error weighted by (0.1 / (|kappa dx| + 0.02))^2 (relative accuracy),
 * step size from lr to lr_final along a half cosine; loss_out[epochs] (optional): mean
 * weighted squared error per epoch */
int icls_mlp_train(icls_mlp* m, int epochs, int batch, double lr, double lr_final, unsigned long long seed,
                   double* loss_out);
/* held-out statistics (kappa*dx): rms(mlp-label), rms(mlp-analytic), rms(plain-analytic),
 * rms(label-analytic), max|mlp-analytic|, max|plain-analytic|, rms|analytic|, samples */
int icls_mlp_eval(icls_mlp* m, double stats[8]);
/* y (device FP32 [n]) = network(X (device FP32 [n][32], 16-byte aligned)); stream 0:
 * synchronous */
int icls_mlp_infer(icls_mlp* m, const void* X, float* y, long long n, void* stream);
/* parameters to (get = 1) or from (get = 0) host float[ICLS_MLP_PARAMS] */
int icls_mlp_params(icls_mlp* m, float* host, int get);
/* gradient of scale * sum (y - label)^2 over n samples (power of two >= 128) into host grad */
int icls_mlp_grad(icls_mlp* m, const void* X, const float* label, long long n, float scale, float* grad,
                  double* loss);

/* Attach a trained network to a context created with curvature_model =
 * ICLS_CURV_MLP (grid spacing isotropic): gfm4p then uses the network's
 * curvature at the cells with |phi| <= 4dz and falls back to the stencil
 * per cell when the correction |kappa_mlp - kappa_stencil| dx > mlp_fallback_tol or
 * |kappa_stencil| dx > 2/3 (curvature radius below 3 cells).  The network
 * must outlive its use by the context. */
int icls_set_curvature_net(icls_ctx* ctx, icls_mlp* net);
/* cells the network evaluated and the fallbacks among them since the last reset */
int icls_curvature_stats(icls_ctx* ctx, long long* evaluated, long long* fallbacks, int reset);

/* ---- tensor-core tile check ----
 * No counterpart in the reference.  d (128 x n FP32, row-major) = a (128 x k
 * BF16, row-major) * b (n x k BF16, row-major)^T on one tcgen05 tile, the
 * building block of the learned curvature's network; device pointers,
 * n and k multiples of 16 in [16, 128]; synchronous on `stream`. */
int icls_tc_gemm_bf16(const void* a, const void* b, float* d, int n, int k, void* stream);

/* ---- divergence check without device allocation -----------------------
 * No counterpart in the reference.  The chkdiv reduction for callers that
 * cannot let the library allocate device memory (their device memory is
 * claimed by their own pool, or a failed allocation inside a check is not
 * acceptable).  u, v, w: device arrays of shape (0:imax+1,0:jmax+1,0:kmax+1),
 * column-major; result: caller's device buffer of 5 doubles, set to
 * [sum of div, max|div|, i, j, k of the first maximum].  The per-block
 * partial sums live in a fixed file-scope device array (about 28 KB on every
 * GPU that loads the library, until exit); the first call on a device looks
 * up its address, so make it before any stream capture.  Calls share that
 * array: calls that overlap on the GPU race.  Grids above
 * ICLS_NOALLOC_MAX_CELLS interior cells return ICLS_E_SIZE; up to it the
 * kernel indexes cells with 64-bit integers.  Nothing is
 * allocated; the call is asynchronous on `stream` (a cudaStream_t, 0 for
 * the default stream).                                                   */
#define ICLS_NOALLOC_MAX_CELLS 2147483647LL
int icls_chkdiv_noalloc(const double* u, const double* v, const double* w, int imax, int jmax, int kmax,
                        double dxi, double dyi, double dzi, double* result, void* stream);

/* ---- instrumentation (not part of the reference interface) ------------
 * Per-launcher device time measured with CUDA events on the context's
 * stream while profiling is on, and kernel launch counts (always kept).  */
int icls_profile_enable(icls_ctx* ctx, int on);
int icls_profile_reset(icls_ctx* ctx);
int icls_profile_count(icls_ctx* ctx, int* n);
int icls_profile_entry(icls_ctx* ctx, int idx, char* name, int name_len, double* total_ms,
                       long long* launches, long long* timed);
int icls_launch_count(icls_ctx* ctx, long long* n);
/* The cudaStream_t every kernel of this context is launched on.          */
int icls_get_stream(icls_ctx* ctx, void** stream);

#ifdef __cplusplus
}
#endif
#endif /* ICLS_GPU_H */
