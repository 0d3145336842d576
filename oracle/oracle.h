/*
 * oracle.h -- CPU FP64 restatement of the reference's hot path, used ONLY
 * as test infrastructure: the parity tests, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py call it as the checker.  The product library
 * (anelastic_solve_b200/libanel.so) never links, loads or calls it.
 *
 * Parity status: the Fortran reference cannot be compiled in this
 * environment (no Fortran front end, no MPI), so this restatement is pinned
 * by the reference's own known-answer cases (the six analytic problems of
 * ANELASTIC_SL/mgMK/test/test.F90:149-382, whose exact solutions are at
 * :471-564) and by manufactured solutions, not by reference binaries.
 *
 * Evaluation order follows the Fortran source left to right and the
 * library is built with -ffp-contract=off so no FMA changes a rounding.
 */
#ifndef ANEL_ORACLE_H
#define ANEL_ORACLE_H

#include "../include/anel.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_mg orc_mg;

/* MG_init + mg_read_params (values passed in directly).  *stat = 0 ok,
 * the mg_check_size code (1..12) or -1 for a bad BC. */
orc_mg* orc_mg_create(const anel_grid_desc* g, const anel_mg_params* p, int* stat);
void orc_mg_destroy(orc_mg* m);

/* Density Flow::r on the fine ghosted grid; default r == 1. */
void orc_mg_set_density(orc_mg* m, const double* r);

/* mg_solver(phif, rhsf, iter, relmax) with the reference semantics,
 * including the clobbering of rhsf (mg_cycle.F90:84-85). */
void orc_mg_solve(orc_mg* m, double* phif, double* rhsf, int* iter, double* relmax);

/* Single passes on the finest level (for kernel parity tests).
 * which: 0 = one mg_relaxRB iteration (iters=1), 1 = mg_bdry,
 *        2 = one mg_cycle (with coefficients built first). */
void orc_mg_debug_pass(orc_mg* m, int which, double* phi, double* src);

/* Level table in the layout of anel_mg_ctx_levels(); returns ngrid. */
int orc_mg_levels(const orc_mg* m, int* out, int cap);

/* ||f - A phi||_2 / ||f||_2 over the fine interior with the fine operator
 * of the context's mode (coefficients built from the current density). */
double orc_mg_true_resid(orc_mg* m, const double* phi, const double* f);

/* Apply the fine operator: out(interior) = A phi (phi ghosts must be set). */
void orc_mg_apply(orc_mg* m, const double* phi, double* out);

/* ---- RK3 stepper (ns_oracle.c) ---- */
typedef struct orc_ns orc_ns;
orc_ns* orc_ns_create(const anel_grid_desc* g, const anel_mg_params* mgp, const anel_ns_params* np,
                      int* stat);
void orc_ns_destroy(orc_ns* s);
/* the oracle works in place on the caller's host arrays */
void orc_ns_bind(orc_ns* s, const anel_fields* f);
void orc_ns_set_clock(orc_ns* s, double time, int nstep);
int orc_ns_substep(orc_ns* s, double a1, double a2, double a3, double dt_rk, double dt, int* iters,
                   double* relmax);
int orc_ns_step(orc_ns* s, anel_step_report* rep);
int orc_ns_project(orc_ns* s, int* iters, double* relmax);
void orc_ns_divergence(orc_ns* s, double* out);
/* vt: 0 u 1 v 2 w 3 p 4 rho 5 cfluc 6 psource 7 utemp 8 vtemp 9 wtemp
 *     10 rtemp 11 s1temp 12 scal1 13 scal1temp */
void orc_ns_ghost(orc_ns* s, double* var, int vt);
/* explicit right-hand side of one field on the bound fields (tests):
 * which 0..4 = u1_rhs, u2_rhs, u3_rhs, rho_rhs, scal1_rhs, into the ghosted
 * array out (gravity at the context's current time) */
void orc_ns_rhs(orc_ns* s, int which, double* out);
/* var_advance_CN_PL(q, u, 1, a3, 1, rkdt, var) (tests): u is replaced by
 * the solved, ghosted field; var 1 u, 2 v, 3 w, 5 rho, 8 scal1 */
void orc_ns_cn(orc_ns* s, const double* q, double* u, double a3, double rkdt, int var);
/* the LES update on the bound fields (tests): model coefficients, then
 * SGSdiff's nuT, kappaT, nappaT */
void orc_ns_les_update(orc_ns* s);
/* the driver's per-step plane statistics (NSsolver.F90:288-395) on the
 * current fields: 16 profiles of nz+2 values into out */
int orc_ns_diagnostics(orc_ns* s, int corrected, const int* stretched, double* out);

#ifdef __cplusplus
}
#endif
#endif
