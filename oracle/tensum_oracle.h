/*
 * tensum_oracle.h -- CPU restatement of TENSUM's explicit residual/update path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker the CUDA path is
 * compared against; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline load it.  The product (libtensum_b200.so) never links or calls it.
 *
 * It restates, in plain C and in the reference's own operation order, the
 * functions FiniteVolume::solve calls per stage (src/fv.cc:699-1879) on the
 * reference's array-of-structures data, so that it reproduces the compiled
 * reference bit for bit (checked by tests/test_oracle_pinned.py against
 * fixtures produced by oracle/_ref/tensum_harness).
 *
 * Layouts match the reference: primitive (T,p,u,v,w, the PrimVar memory order), residual (mass,mx,my,mz,
 * energy), gradient dE[v][var][xyz] with var order (V1,V2,V3,V4,V5).
 */
#ifndef TENSUM_ORACLE_H
#define TENSUM_ORACLE_H

#include "../include/tensum_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct tor_state tor_state;

tor_state* tor_create(const tg_mesh* mesh, const tg_material* mat, const tg_bc_table* bc,
                      const tg_options* opt);
void tor_destroy(tor_state* s);
int tor_n_vertex(const tor_state* s);

void tor_set_prim(tor_state* s, const double* prim_aos, double t0);
void tor_get_prim(const tor_state* s, double* prim_aos);
void tor_store_conserved_old(tor_state* s);
double tor_compute_dt(tor_state* s, double* dt_out);
void tor_compute_gradients(tor_state* s, double* dE_out);
void tor_compute_residual(tor_state* s, double* res_out, double* dE_out);
void tor_update(tor_state* s, int r);
void tor_residual_norm(tor_state* s, long iter, double* out6);
void tor_end_step(tor_state* s);
/* Runs n_steps of the solve loop; returns the number of steps actually taken
 * (stops at final_time).  info4 = {elapsed, dt_global, residual_total, iter}. */
long tor_step(tor_state* s, long n_steps, double* info4);
void tor_global(const tor_state* s, double* ke, double* entropy);

/* Single-edge flux kernel access for unit tests: states are (T,u,v,w,p),
 * gradients 5x3 (var-major), coordinates and normal 2D. */
void tor_num_flux(const tor_state* s, const double* cl, const double* cr, const double* left,
                  const double* right, const double* dEl, const double* dEr, const double* normal,
                  double* flux5);
double tor_logavg(double a, double b);

/* Monte Carlo moments (increment_moments src/fv.cc:595-694, reduce_moments
 * src/reduce_moments.cc:14-221).  Records per vertex: PrimVar (T,p,u,v,w),
 * then density, mach, entropy, vorticity as selected by the bits of extras. */
void tor_forces(tor_state* s, int n_forces, const int* n_tags, const int* tags, double* out4);
void tor_get_residual(const tor_state* s, double* out5);
int tor_counter(const tor_state* s);   /* next output-time index (FiniteVolume::counter) */
int tor_moment_nvars(int extras);
void tor_moments_increment(const tor_state* s, long k, int extras, double* fm, double* sm, double* m2);
long tor_moments_merge(int nv, int nvar, long n_old, double* fm, double* sm, double* m2, long n_other,
                       const double* fm_o, const double* sm_o, const double* m2_o);
void tor_moments_finalize(int nv, int nvar, long n, double* sm, double* m2);

#ifdef __cplusplus
}

#endif
#endif
