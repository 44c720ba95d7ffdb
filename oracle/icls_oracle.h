/*
 * icls_oracle.h — CPU restatement of the ICLS per-timestep hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the CUDA path is compared
 * against (tests/, __graft_entry__.smoke(), and bench.py's cpu_baseline /
 * --impl reference legs).  Nothing in the product links or calls it.
 *
 * The entry points mirror include/icls_gpu.h one for one (prefix ora_
 * instead of icls_), operate on the same Fortran-layout arrays and use the
 * same icls_config, so a test can drive both with identical calls.
 */
#ifndef ICLS_ORACLE_H
#define ICLS_ORACLE_H
#include "../include/icls_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ora_ctx ora_ctx;

int ora_create(const icls_config* cfg, ora_ctx** out);
int ora_destroy(ora_ctx* ctx);
int ora_set_threads(int n);
int ora_field_bounds(const ora_ctx* ctx, int field_id, int lo[3], int hi[3]);
int ora_upload_field(ora_ctx* ctx, int field_id, int l, const double* host);
int ora_download_field(ora_ctx* ctx, int field_id, int l, double* host);
int ora_get_scalars(ora_ctx* ctx, icls_scalars* out);
int ora_set_dt(ora_ctx* ctx, double dt);
int ora_get_volumes(ora_ctx* ctx, double* volume, double* init_volume);
/* exact, order-independent sum of n doubles (the volume integral's sum) */
double ora_exact_sum(const double* x, long long n);
int ora_get_pseudo_inv(ora_ctx* ctx, double* P /* 10x27 row-major */);

int ora_init_program(ora_ctx* ctx);
int ora_ls_main(ora_ctx* ctx, int istep);
int ora_average_stream_vel(ora_ctx* ctx, double* v_bulk);
int ora_ab2(ora_ctx* ctx);
int ora_fillps(ora_ctx* ctx);
int ora_gfm4p(ora_ctx* ctx);
int ora_add_pjump(ora_ctx* ctx);
int ora_solver2d(ora_ctx* ctx);
int ora_boundp(ora_ctx* ctx, int field_id);
int ora_correc(ora_ctx* ctx);
int ora_bounduvw(ora_ctx* ctx, int field_id_u);
int ora_pressure_update(ora_ctx* ctx, int istep, int begin);
int ora_average_vel_at_center(ora_ctx* ctx);
int ora_max_vel_at_center(ora_ctx* ctx, double* vel_max);
int ora_disp(ora_ctx* ctx, int l, double cg[3], double vel[3]);
int ora_set_inflow(ora_ctx* ctx, const double* v_inflow);
int ora_download_plane_x(ora_ctx* ctx, int id, int l, int i, double* out);
int ora_timestep_record(ora_ctx* ctx, int istep, double rec[6]);
int ora_write_checkpoint(ora_ctx* ctx, const char* path, int nr, int history);
int ora_read_checkpoint(ora_ctx* ctx, const char* path, int* nr);
int ora_chkdiv(ora_ctx* ctx, int istep, double* divtot, double* divmax, int ijk[3]);
int ora_chkdt(ora_ctx* ctx, double* dtmax);
int ora_ipot(ora_ctx* ctx, double* dmin);
int ora_step(ora_ctx* ctx, int istep, int begin);

int ora_tube_construction(ora_ctx* ctx, int l);
int ora_ls_advection(ora_ctx* ctx, int l);
int ora_ls_mass_correction(ora_ctx* ctx, int istep, int l);
int ora_ls_reinit_main(ora_ctx* ctx, int istep, int l);
int ora_update_materials(ora_ctx* ctx);
int ora_get_curvature(ora_ctx* ctx, int l);
int ora_band_count(ora_ctx* ctx, int l, long long* nb_cnt);

/* VFFTPACK contract (libs/fft/fft.f:1123-1142 forward, 403-452 backward):
 * m sequences of length n, sequence s stored contiguously at r + s*n.    */
int ora_vrfftf(int m, int n, double* r);
int ora_vrfftb(int m, int n, double* r);
int ora_vcosqf(int m, int n, double* r);  /* fft.f:68-216, per row */
int ora_vcosqb(int m, int n, double* r);  /* fft.f:218-372, per row */

/* Initial level sets of init.f90 'drp' (717-753) and 'mdp' (901-984)
 * generalised to arbitrary centres/radii: writes lvset(:,:,:,l) for
 * l=1..ndrop (shape L) into out, drop after drop.                        */
int ora_init_drops(const icls_config* cfg, int ndrop, const double* xc,
                   const double* yc, const double* zc, const double* radius,
                   double* out);

#ifdef __cplusplus
}
#endif
#endif
