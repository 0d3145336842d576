/*
 * anel.h -- C-ABI of the B200 (sm_100a) anelastic/Boussinesq hot path:
 * the multigrid pressure-Poisson solve (mgMK) and the RK3 sub-step.
 *
 * Every entry point takes plain pointers and sizes.  Field arrays are the
 * reference's ghost-layered, column-major (i fastest) FP64 arrays:
 *   element (i,j,k), 1-based with ghosts, i = 1..nx+2 (interior 2..nx+1),
 *   sits at offset (i-1) + (nx+2)*((j-1) + (ny+2)*(k-1)).
 * 1-D grid metric arrays (xe, xc, dxe, dxc, rdxe, rdxc, ...) have n+2
 * entries, entry 0 being the Fortran index 1, exactly as read from the
 * reference's x?_grid.in files (ANELASTIC_SL/utils/loadGrid.F90:38-90).
 *
 * Two families of calls exist:
 *  - drop-in calls with the reference's names and by-reference arguments
 *    (anel_mg_init / anel_mg_solve / anel_mg_finalize, anel_rk_substep),
 *    operating on one library-owned default context and on HOST arrays;
 *  - context calls (anel_mg_ctx_*, anel_ns_ctx_*) that take a context
 *    handle, a memory-space flag (host or device pointers) and a CUDA
 *    stream, for device-resident use and for many independent members.
 *
 * Return codes are ANEL_OK (0) or a negative ANEL_ERR_*; no call exits the
 * process.  anel_last_error() returns a message for the calling thread.
 */
#ifndef ANEL_H
#define ANEL_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ANEL_MAX_LEVELS 16

/* ---- status codes ---------------------------------------------------- */
enum {
  ANEL_OK = 0,
  ANEL_ERR_SIZE = -1,        /* level/size constraints (mg_check_size.F90:77-151) */
  ANEL_ERR_BC = -2,          /* bad boundary-condition code (mg_init.F90:317-328) */
  ANEL_ERR_NOCONV = -3,      /* maxcy reached before tolmax (mg_solver.F90:130-133) */
  ANEL_ERR_CUDA = -4,        /* a CUDA runtime call failed */
  ANEL_ERR_TIMEOUT = -5,     /* a bounded device-side loop gave up */
  ANEL_ERR_ARG = -6,         /* null pointer / bad enum / not initialised */
  ANEL_ERR_NOMEM = -7,       /* device allocation failed */
  ANEL_ERR_UNSUPPORTED = -8, /* valid in the reference, not handled by this build */
  ANEL_ERR_NONFINITE = -9    /* NaN/Inf found in an input field */
};

/* ---- enums ------------------------------------------------------------ */
/* RBPGS: red-black point Gauss-Seidel (mg_relax.F90:85-179, the runfile's
 *        choice).  LJ: the reference's (i+j) red-black z-line smoother with
 *        the pcf_* coefficients (mg_relax.F90:423-538).  ZLINE: (i+j)
 *        red-black z-line Gauss-Seidel with the level's own 7-point
 *        operator (an extension for stretched z grids). */
enum { ANEL_SMOOTHER_RBPGS = 0, ANEL_SMOOTHER_LJ = 1, ANEL_SMOOTHER_ZLINE = 2 };
/* LITERAL: the reference's RBPGS operator (uniform spacing xL/nx, zL/nz,
 *          mg_pfpde.F90 / mg_phpde.F90).  METRIC: the same V-cycle with
 *          every level's 7-point operator built from the stretched metric:
 *          the fine level is exactly Psource(Pgrad(p)), coarse levels use
 *          1/(dzc*dze) products (mg_coeff.F90 form) on a cell-centred
 *          agglomeration of the grid, with consistent Neumann walls. */
enum { ANEL_MODE_LITERAL = 0, ANEL_MODE_METRIC = 1 };
/* FP64: every MG array FP64.  MIXED: FP32 V-cycle inside an FP64 defect-
 *       correction loop (FP64 fine residual, correction and norms). */
enum { ANEL_PREC_FP64 = 0, ANEL_PREC_MIXED = 1 };
/* RELMAX: the reference's stop test max|phi_new-phi_old|/max|phi_new| <=
 *         tolmax (mg_residual.F90:60-94).  RESID: ||f - A phi||_2/||f||_2
 *         <= tolmax with the fine operator. */
enum { ANEL_STOP_RELMAX = 0, ANEL_STOP_RESID = 1 };
enum { ANEL_MEM_HOST = 0, ANEL_MEM_DEVICE = 1 };
/* boundary types, tbc[] (mg_read_params.F90:96-99) */
enum { ANEL_BC_PERIODIC = 0, ANEL_BC_NEUMANN = 1, ANEL_BC_DIRICHLET = 2 };

/* ---- descriptors -------------------------------------------------------
 * anel_grid_desc replaces the Domain and Grid modules
 * (ANELASTIC_SL/include/modules.F90:17-39): interior sizes, domain lengths
 * and the 18 metric arrays of length n+2. */
typedef struct {
  int32_t nx, ny, nz;
  double xL, yL, zL;
  const double *xe, *xc, *dxe, *dxc, *rdxe, *rdxc;
  const double *ye, *yc, *dye, *dyc, *rdye, *rdyc;
  const double *ze, *zc, *dze, *dzc, *rdze, *rdzc;
} anel_grid_desc;

/* anel_mg_params replaces the mgVars module inputs read by mg_read_params
 * (ANELASTIC_SL/mgMK/mg_read_params.F90:43-214).  pre_relax/post_relax are
 * indexed by level-1, level 1 = coarsest, exactly as the ini lists them.
 * tbc/vbc use the reference face order 1=X2max 2=X3min 3=X2min 4=X3max
 * 5=X1min 6=X1max (index 0..5 here). */
typedef struct {
  int32_t levels[3];               /* nxlevels, nylevels, nzlevels */
  int32_t maxcy;                   /* maximum V-cycles */
  double tolmax;                   /* stop tolerance */
  int32_t smoother;                /* ANEL_SMOOTHER_* */
  int32_t pre_relax[ANEL_MAX_LEVELS];
  int32_t post_relax[ANEL_MAX_LEVELS];
  int32_t tbc[6];
  double vbc[6];
  int32_t mode;                    /* ANEL_MODE_* */
  int32_t precision;               /* ANEL_PREC_* */
  int32_t stop;                    /* ANEL_STOP_* */
  int32_t verbose;                 /* print per-cycle residuals to stderr */
} anel_mg_params;

/* Per-solve report (the reference prints the same numbers,
 * NSsolver.F90:524 and mg_solver.F90:123). */
typedef struct {
  int32_t iter;        /* V-cycles (MIXED: defect-correction iterations) */
  int32_t status;      /* ANEL_OK or ANEL_ERR_NOCONV / _TIMEOUT */
  double relmax;       /* reference stop metric of the last cycle */
  double resid;        /* ||f - A phi||_2 / ||f||_2 (fine operator) after the solve */
  double ms;           /* device time of the solve (CUDA events) */
  int64_t launches;    /* kernels of this library launched by the solve */
  int32_t fine_sweeps; /* finest-level smoother launches timed (profiling on) */
  int32_t reserved;
  double fine_sweep_ms;/* their summed device time (CUDA events, profiling on) */
} anel_mg_report;

typedef struct anel_mg_ctx anel_mg_ctx;

/* ---- library ------------------------------------------------------------ */
const char* anel_last_error(void);
int anel_version(void);
/* Number of this library's kernels launched since load (all contexts). */
int64_t anel_kernel_launch_count(void);
/* The autotuner's choices so far, one line per tuned kernel shape:
 * "<kernel> dev<d> <shape>: variant <v> (<ms of each variant> ms)".  Kernels
 * with several launch shapes are timed once per device and shape (when a
 * context that uses them is created) and the fastest is kept for the
 * process; ANEL_TUNE=0 in the environment keeps every default.  Copies at
 * most cap-1 characters and a NUL into buf; returns the report's length.
 * Library introspection: no counterpart in the reference. */
int32_t anel_tuning_report(char* buf, int32_t cap);

/* ---- multigrid: drop-in calls ------------------------------------------ */

/* Replaces mg_read_params + MG_init (mg_read_params.F90:1-218,
 * mg_init.F90:1-351): level maps, workspace, coarse metrics.  Returns the
 * reference's stat meaning as ANEL_OK / ANEL_ERR_SIZE / ANEL_ERR_BC. */
int anel_mg_init(const anel_grid_desc* grid, const anel_mg_params* params);

/* Sets the density Flow::r (host, ghosted G array) used to build the level
 * coefficients (mg_solver.F90:81-97 rebuilds them from r on every call;
 * here they are rebuilt only when r changes).  Before the first call r == 1. */
int anel_mg_set_density(const double* r);

/* Replaces mg_solver(phif,rhsf,iter,relmax) (mg_solver.F90:1-141), same
 * argument order, Fortran by-reference, host arrays.  phif: inout, ghosted;
 * its ghosts are set by the final boundary pass.  rhsf: in; the reference
 * uses it as V-cycle scratch (mg_cycle.F90:33,84-85), so its contents on
 * return are unspecified here as well.  iter: cycles used (maxcy+1 when not
 * converged, the value the reference's DO loop leaves).  relmax: last
 * max|dphi|/max|phi|. */
void anel_mg_solve(double* phif, double* rhsf, int32_t* iter, double* relmax);

/* Replaces mg_end (mg_end.F90:1-42). */
int anel_mg_finalize(void);

/* ---- multigrid: context calls ------------------------------------------- */
anel_mg_ctx* anel_mg_create(const anel_grid_desc* grid, const anel_mg_params* params,
                            int32_t device, int32_t* status);
void anel_mg_destroy(anel_mg_ctx* ctx);
int anel_mg_ctx_set_density(anel_mg_ctx* ctx, const double* r, int32_t mem);
/* phif/rhsf are host (ANEL_MEM_HOST) or device (ANEL_MEM_DEVICE) ghosted
 * FP64 arrays; stream is a cudaStream_t (NULL = the context's stream).
 * rhsf is read only (unlike the reference, it is not clobbered). */
int anel_mg_ctx_solve(anel_mg_ctx* ctx, double* phif, const double* rhsf, int32_t mem,
                      void* stream, anel_mg_report* report);
/* Batched solve (no reference counterpart: the reference solves one
 * problem per call): n independent problems on the context's grid, device
 * arrays d_phis[b] (inout) / d_rhss[b], solved together -- every kernel of
 * the mixed-precision z-line cycle runs over all members still iterating,
 * the defect-correction loop is one CUDA graph per batch size, and each
 * member stops at its own tolerance.  Member b ends bit-identical to
 * anel_mg_ctx_solve of it alone; reports[b] is its report (ms: the whole
 * batch).  Needs a mixed-precision ZLINE context on the column layout
 * (x/y semi-coarsened levels, nz = 32*M), else ANEL_ERR_UNSUPPORTED.
 * Returns ANEL_ERR_NOCONV if any member did not converge. */
int anel_mg_ctx_solve_batch(anel_mg_ctx* ctx, int32_t n, double* const* d_phis, const double* const* d_rhss,
                            void* stream, anel_mg_report* reports);
/* Profiling: when on, every finest-level smoother launch of the following
 * solves is bracketed by CUDA events on its stream, and the report carries
 * their count and summed time (fine_sweeps, fine_sweep_ms). */
int anel_mg_ctx_set_profiling(anel_mg_ctx* ctx, int32_t on);
/* Level table, for tests of the bit-exact index maps (mg_init.F90:125-220):
 * out[l*12 + 0..11] = nxk nyk nzk sxk exk syk eyk szk ezk kp3d kpx1 kpx2
 * for l = 0..ngrid-1 (level l+1); returns ngrid. */
int anel_mg_ctx_levels(const anel_mg_ctx* ctx, int32_t* out, int32_t cap);

/* Primitive passes on the finest level, device pointers, for parity tests
 * of single kernels.  which: 0 = one RB-GS iteration (both colours + the
 * boundary pass after each, mg_relax.F90:146-172), 1 = boundary pass only
 * (mg_bdry.F90), 2 = one V-cycle with phif as initial guess
 * (mg_cycle.F90), 3 = the FP64 direct solve that the mixed z-line cycle
 * uses on its coarse level, applied to the fine level itself (A phi = f
 * with the gauge pinned, then the boundary pass; needs a context of the
 * column-layout cycle and a fine level of at most 64 x 64 columns and 512
 * of them in all: ANEL_ERR_UNSUPPORTED otherwise; no reference
 * counterpart). */
int anel_mg_ctx_debug_pass(anel_mg_ctx* ctx, int32_t which, double* d_phi,
                           const double* d_src, void* stream);

/* ======================================================================
 * RK3 time stepper (rk_ss / NSsolver, ANELASTIC_SL/dns/NSsolver.F90)
 * ==================================================================== */

/* velocity / scalar models (the Vmodel/Rmodel/Smodel ini keys,
 * ANELASTIC_SL/dns/input.F90): DNS, or the constant-coefficient
 * Smagorinsky model (SSM, SSMrho, SSMscal1), or the dynamic Smagorinsky
 * model (DSM, DSMrho, DSMscal1, les/DSM*.F90) with x-y plane-averaged
 * coefficients (their C_avg_dir = 12). */
enum { ANEL_MODEL_DNS = 0, ANEL_MODEL_SSM = 1, ANEL_MODEL_DSM = 2 };
/* LES filter width (les_grid_size, straincal.F90:126-134) */
enum { ANEL_DELTA_3ROOT = 0, ANEL_DELTA_2ROOT = 1 };
/* LES wall damping: LITERAL = Mason damping of SSM.F90:27,60 with its
 * REAL(4) literals; NONE = f_damp == 1, i.e. Csgs = SSM_const. */
enum { ANEL_DAMP_LITERAL = 0, ANEL_DAMP_NONE = 1 };

/* Field variables of the boundC tables TB(3,2,8)/VB(3,2,8)
 * (ANELASTIC_SL/include/modules.F90:80-86): index l-1 of
 * 1=U1 2=U2 3=U3 4=P 5=RHO 6=FLUC 7=temporaries/psource 8=SCAL1.
 * Types: 1 Dirichlet, 2 Neumann, 3 periodic, 4 one-point Neumann,
 * 6 wall6, 7 wall7, 8 linear extrapolation (ANELASTIC_SL/dns/BC.F90:334-585). */
typedef struct {
  double Re, Pr, Sc;                  /* rRe = 1/Re, rPr = 1/Pr, rSc = 1/Sc */
  double cfl, dtmax;                  /* calcdt (Routines.F90:186-258), DeltaT_max */
  double g_init, g_final, gt1, gt2;   /* gravity ramp (Routines.F90:2-52) */
  int32_t vmodel, rmodel, smodel;     /* ANEL_MODEL_* */
  int32_t les_delta;                  /* ANEL_DELTA_* */
  int32_t les_damp;                   /* ANEL_DAMP_* */
  double ssm_const, pr_sgs;           /* SSM_const, Pr_eddy (Pr_sgs) */
  int32_t les_start, les_freq;        /* les_start_step, les_call_freq */
  int32_t tb[3][2][8];                /* TB(dir,face,var) */
  double vb[3][2][8];                 /* VB(dir,face,var) */
  /* EW edge-node flag of the w field (Domain module).  0: as Sturb.F90:
   * 110-112 forces it -- w at the top wall face (k = nz+1) is advanced as
   * an unknown, which leaves the Neumann pressure problem incompatible.
   * 1: the edge-node mode the code is written for -- u3_rhs and Pgrad stop
   * at nz, and the w ghost sets w(nz+1) to the wall value and w(nz+2) to 0
   * (BC.F90:471-527). */
  int32_t ew;
  /* 1: advance scal1 as rk_ss always does.  0: hold scal1 (and its
   * accumulator) at zero, valid when scal1 starts at zero with zero wall
   * values -- it then stays zero in the reference as well. */
  int32_t scal1_on;
  /* Dynamic models: TestGrid_ratio (r_dgt_dg), the test filter's
   * directions xfilter/yfilter/zfilter, and for center_velocity the
   * Gridtype of each axis (1 = stretched) and the interpolation mode on a
   * stretched axis (ANEL_DIAG_LITERAL / ANEL_DIAG_CORRECTED, see the plane
   * statistics). */
  double test_ratio;
  int32_t filt[3];
  int32_t stretched[3];
  int32_t interp;
  /* Clip (Parameters::clip, NSsolver.F90:206-211, 235-240, 264-269):
   * after every sub-step rho and then scal1 are clipped to [min, max]
   * on the interior (clipVS, Routines.F90:301-380: below min -> min,
   * then above max -> max) and ghosted.  0 (the runfiles' Clip=no): off.
   * With scal1_on = 0 the scal1 range must contain 0. */
  int32_t clip;
  /* Initial guess of each sub-step's pressure solve (an extension; the
   * reference starts from the current p, pguess = 0).  1: the linear
   * extrapolation 2 p(n-1) - p(n-2) of the member's solutions of the same
   * sub-step in the last two steps, when both exist.  The solve still
   * runs to the same stopping test, so it changes which iterate is
   * returned (within the tolerance), not the accuracy. */
  int32_t pguess;
  double rho_min, rho_max, scal1_min, scal1_max;
} anel_ns_params;

/* Host (or device) pointers to the ghosted FP64 fields of the Flow and
 * LESmod modules.  u at (xe,yc,zc), v at (xc,ye,zc), w at (xc,yc,ze),
 * the others at cell centres.  q_* are the RK3 accumulators u1_tmp2,
 * u2_tmp2, u3_tmp2, r_tmp2, scal1_tmp2; psrc is r_tmp1 (the Poisson right-
 * hand side scratch).  nuT/kappaT/nappaT may be NULL for DNS. */
typedef struct {
  double *u, *v, *w, *p, *rho, *scal1;
  double *r, *densityBG;
  double *q_u, *q_v, *q_w, *q_rho, *q_s;
  double *psrc;
  double *nuT, *kappaT, *nappaT;
} anel_fields;

/* Per-step report */
typedef struct {
  int32_t nstep;        /* step number just completed */
  int32_t mg_iter[3];   /* MG cycles of the three sub-steps */
  double dt;            /* delt used */
  double time;          /* time after the step */
  double mg_relmax[3];  /* MG stop metric of each sub-step */
  double max_div;       /* max |div u| after the step (divergence()) */
  double avg_div;       /* volume-weighted mean |div u| */
  double ms;            /* device time of the steps of the call */
  double mg_ms;         /* part of it spent in the multigrid solves */
  int64_t launches;     /* kernels of this library launched by the call */
  int32_t fine_sweeps;  /* finest-level smoother launches timed (profiling on) */
  int32_t reserved;
  double fine_sweep_ms; /* their summed device time (profiling on) */
  double diag_ms;       /* device time of the plane statistics (diagnostics on) */
} anel_step_report;

typedef struct anel_ns_ctx anel_ns_ctx;

/* Context calls: fields live on the device inside the context. */
anel_ns_ctx* anel_ns_create(const anel_grid_desc* grid, const anel_mg_params* mg,
                            const anel_ns_params* ns, int32_t device, int32_t* status);
void anel_ns_destroy(anel_ns_ctx* ctx);
/* Copy fields in/out (mem = ANEL_MEM_HOST or ANEL_MEM_DEVICE pointers).
 * Null members are skipped.  r and densityBG must be horizontally
 * uniform (functions of z only). */
int anel_ns_set_fields(anel_ns_ctx* ctx, const anel_fields* f, int32_t mem);
int anel_ns_get_fields(anel_ns_ctx* ctx, const anel_fields* f, int32_t mem);
/* One RK sub-step, rk_ss(a1,a2,a3,ec,dt_rk,dt,psolve,stat)
 * (NSsolver.F90:418-583), on the context's fields. */
int anel_ns_ctx_substep(anel_ns_ctx* ctx, double a1, double a2, double a3, double dt_rk,
                        double dt, void* stream, int32_t* mg_iter, double* mg_relmax);
/* nsteps full time steps of NSsolver (NSsolver.F90:63-283 without the
 * output/statistics diagnostics): calcdt, gravity, LES update, three
 * sub-steps.  report (may be NULL) describes the last step. */
int anel_ns_ctx_step(anel_ns_ctx* ctx, int32_t nsteps, void* stream, anel_step_report* report);
/* nsteps steps of n contexts together (an ensemble cohort; no reference
 * counterpart): the contexts share grid, boundary setup and multigrid
 * parameters (physics, time step and fields are their own), run on one
 * stream, and every sub-step's n pressure solves are one batched solve
 * (anel_mg_ctx_solve_batch) of `batch` -- a multigrid context of the same
 * grid and parameters, or NULL for the first member's own.  Each member's
 * fields and report equal those of anel_ns_ctx_step on it alone (report
 * ms and launches: the whole cohort's; mg ms: the batch's shared out). */
int anel_ns_ctx_step_cohort(anel_ns_ctx* const* ctxs, int32_t n, int32_t nsteps, anel_mg_ctx* batch,
                            void* stream, anel_step_report* reports);
/* nsteps from host fields `in` to host fields `out` (the same arrays
 * allowed; null members are skipped): the caller's state stays in host
 * memory, as with the reference's rk_ss on its module arrays.  The copy
 * of p in overlaps sub-step 1 up to its pressure solve, the copies of rho,
 * scal1 and p out overlap the last sub-step's pressure solve and Pgrad;
 * the results equal set_fields + step + get_fields.  Pinned host memory
 * lets the copies run asynchronously. */
int anel_ns_ctx_step_host(anel_ns_ctx* ctx, const anel_fields* in, const anel_fields* out, int32_t nsteps,
                          void* stream, anel_step_report* report);
/* Profiling of the multigrid inside the steps (see
 * anel_mg_ctx_set_profiling); totals land in the step report. */
int anel_ns_ctx_set_profiling(anel_ns_ctx* ctx, int32_t on);
/* time and step counter (time, nstep of the Parameters module) */
int anel_ns_ctx_set_clock(anel_ns_ctx* ctx, double time, int32_t nstep);
/* Projection of the current velocity onto divergence-free fields (used to
 * prepare initial conditions): the velocity ghost passes, Psource with
 * dt = 1, one MG solve starting from p, Pgrad with dt = 1 and the velocity
 * ghost passes. */
int anel_ns_ctx_project(anel_ns_ctx* ctx, int32_t* mg_iter, double* mg_relmax);
/* Plane statistics of the driver's per-step dk/dt block
 * (NSsolver.F90:288-395): cell-centred velocities (center_velocity,
 * StatTools.F90:87-289), x-y plane averages (avgX1X2, Average.F90:279-368),
 * the mean profiles U1, U2, T, S and MKE = U1 + U2, the second moments of
 * the fluctuations (TKE = (<u'u'> + <v'v'> + <w'w'>)/2, t2 = <t't'>,
 * s2 = <s's'>) and the time derivative of each over the last step
 * ((new - old)/(time - told)).  The previous profiles start at 0.
 * stretched[d] = 1 where axis d's grid file says 'stretched': there
 * center_velocity interpolates over five points.  mode LITERAL keeps the
 * reference's interpolation as written (StatTools.F90:611-653 hands the
 * values to divdiffs as abscissae: the inverse interpolant, which divides
 * by differences of the values and is Inf/NaN where two of them are
 * equal); CORRECTED interpolates the values over the coordinates.
 * With on = 1, anel_ns_ctx_step runs the block after every step
 * (as the reference driver does); the report's diag_ms is its time. */
enum { ANEL_DIAG_LITERAL = 0, ANEL_DIAG_CORRECTED = 1 };
enum { ANEL_DIAG_PROFILES = 16 };
int anel_ns_ctx_set_diagnostics(anel_ns_ctx* ctx, int32_t on, int32_t mode, const int32_t* stretched);
/* Run the block once on the current fields (between steps). */
int anel_ns_ctx_compute_diagnostics(anel_ns_ctx* ctx, void* stream);
/* Copy the 16 profiles of nz+2 values (k = 1..nz+2), in the order U1, U2,
 * T, S, MKE, TKE, t2, s2, dU1dt, dU2dt, dTdt, dSdt, dMKEdt, dkdt, dt2dt,
 * ds2dt, to out (mem = ANEL_MEM_HOST or ANEL_MEM_DEVICE). */
int anel_ns_ctx_get_diagnostics(anel_ns_ctx* ctx, double* out, int32_t mem);
/* Restart files in the reference's layout (Restart.F90): Fortran
 * sequential unformatted records (4-byte little-endian length markers)
 * holding the header nstep, time, delt, g, rho_0, scal1_0, Re, Pr, Sc; the
 * extents; then u, v, w, p, rho, scal1, each the whole ghosted array.
 * SMALL is the serial dump of write_flow_small / Greadfile (extents nx+2,
 * ny+2, nz+2; file name basename//nstep); BIG is one rank's file of
 * write_flow_big / start_big (extents sx, ex, sy, ey, sz, ez = 2, nx+1,
 * 2, ny+1, 2, nz+1 for the single rank; file name
 * basename//c1_c2_c3.nstep).  Readers refuse other extents
 * (ANEL_ERR_SIZE) and malformed records; a field record above 2^31-1
 * bytes is refused. */
enum { ANEL_RESTART_SMALL = 0, ANEL_RESTART_BIG = 1 };
typedef struct {
  int32_t nstep;
  double time, delt, g, rho_0, scal1_0, Re, Pr, Sc;
} anel_restart_header;
/* Host arrays u, v, w, p, rho, scal1 ((nx+2)(ny+2)(nz+2) each, Fortran
 * order); no GPU involved. */
int anel_restart_write(const char* path, int32_t layout, const anel_restart_header* hdr, int32_t nx,
                       int32_t ny, int32_t nz, const double* const* fields);
int anel_restart_read(const char* path, int32_t layout, anel_restart_header* hdr, int32_t nx, int32_t ny,
                      int32_t nz, double* const* fields);
/* The context's fields to / from a restart file.  Reading ghosts the six
 * fields as start_small / start_big do; icparam = 1 also takes the clock
 * (time, nstep) from the header, as the reference's icparam does for its
 * Parameters (Re, Pr, Sc, g are returned in hdr: a context is built with
 * its physics). */
int anel_ns_ctx_write_restart(anel_ns_ctx* ctx, const char* path, int32_t layout,
                              const anel_restart_header* hdr);
int anel_ns_ctx_read_restart(anel_ns_ctx* ctx, const char* path, int32_t layout, int32_t icparam,
                             anel_restart_header* hdr);
/* divergence() (Routines.F90:54-183) of the current velocity:
 * out[0] = volume-weighted mean |div|, out[1] = max |div|. */
int anel_ns_ctx_divergence(anel_ns_ctx* ctx, double* out);

/* The same divergence diagnostic for callers that must not have the
 * library allocate device memory (a driver that pools or pins all of its
 * device memory up front, or runs under a fully committed memory budget):
 * it allocates nothing.  This entry point has no counterpart in the
 * reference.  u, v, w are the caller's ghosted device fields
 * ((nx+2)(ny+2)(nz+2) doubles, Fortran order), rdxc/rdyc/rdzc its device
 * metric arrays (n+2 each); out (host, 2 doubles) receives the mean and
 * max |div| as anel_ns_ctx_divergence does (the mean may differ in the
 * last bits: its sums run per z-plane).  Partial sums live in a fixed
 * array inside the library's device image, which limits nz to 4096
 * (larger: ANEL_ERR_SIZE) and is shared by all calls on a device, so
 * calls whose GPU work overlaps race; run them on one stream.  The first
 * call on a device looks up that array's address and keeps it: make it
 * before any stream capture on the device.  The kept address belongs to
 * the device's primary context: after cudaDeviceReset (or any teardown of
 * that context) it is stale, so a process that resets the device must not
 * call this entry point again.  Waits for stream. */
int anel_divergence_noalloc(int32_t nx, int32_t ny, int32_t nz, const double* u, const double* v,
                            const double* w, const double* rdxc, const double* rdyc,
                            const double* rdzc, double* out, void* stream);

/* ---- serving: continuous batching of independent members ----------------
 * An engine that runs many short, independent shear-layer members (an
 * ensemble, or a request stream) on one GPU.  Not a reference routine:
 * each reference run is its own job.  Requests queue in FIFO order;
 * max_active host threads each drive a cohort: the members of one bucket
 * (grid, models, multigrid setup) stepping together, joined by the
 * bucket's new requests and left by finished members at step boundaries,
 * with each sub-step's pressure solves batched into one multigrid solve
 * (up to 16 members; buckets whose multigrid is not the column-layout
 * mixed z-line cycle run member by member).  Cohorts of different buckets
 * overlap on the device.  A member is admitted when its device memory
 * fits the HBM budget, re-using an idle context of the same bucket or
 * releasing idle contexts of other buckets (least recently used first).
 * A member's fields do not depend on what else runs.  Caller arrays named in a request (fields_in, fields_out) must
 * stay alive until its result is polled. */
typedef struct anel_serve anel_serve;
enum { ANEL_INIT_SHEAR = 0, ANEL_INIT_FIELDS = 1, ANEL_INIT_POISSON = 2 };
typedef struct {
  anel_grid_desc grid;   /* host metric arrays: copied at submit */
  anel_mg_params mg;
  anel_ns_params ns;
  int32_t nsteps;        /* RK3 steps after the initial projection */
  int32_t init;          /* ANEL_INIT_SHEAR: shear layer U = tanh(zc), rho = -tanh(zc), noise
                          * amp*(2U-1) on |zc| < 2 from the Park-Miller sequence of seed;
                          * ANEL_INIT_FIELDS: the host fields of fields_in;
                          * ANEL_INIT_POISSON: a standalone pressure solve with the
                          * request's grid and mg parameters (ns, nsteps, seed unused):
                          * right-hand side fields_in->psrc, initial guess fields_in->p
                          * (NULL: zero), solution to fields_out->p (may be NULL).
                          * Requests of one bucket are solved together, up to 16 per
                          * batched solve. */
  uint32_t seed;
  int32_t reserved;
  double amp;
  const anel_fields* fields_in;  /* host; ANEL_INIT_FIELDS only */
  anel_fields* fields_out;       /* host, may be NULL: fields after the last step */
} anel_request;
typedef struct {
  int64_t id;
  int32_t status;        /* ANEL_OK or the member's error (ANEL_ERR_NOMEM: larger than the budget) */
  int32_t nsteps;
  int64_t cells;         /* interior cells */
  double queue_ms;       /* submit -> start (host steady clock) */
  double run_ms;         /* start -> fields ready */
  double latency_ms;     /* submit -> fields ready */
  double dt_last;        /* time step of the last step */
  double max_div;        /* max |div u| after the last step */
  int32_t mg_iter;       /* Poisson requests: V-cycles of the solve */
  int32_t reserved;
  double resid;          /* Poisson requests: final relative residual */
} anel_result;
typedef struct {
  int64_t submitted, completed, failed;
  int64_t bytes_in_use, peak_bytes;  /* admitted context memory (estimates) */
  int32_t active, peak_active, contexts, queued;
  int32_t peak_cohort;               /* most members stepped together in one cohort */
  int32_t reserved;
} anel_serve_stats;

anel_serve* anel_serve_create(int32_t device, int64_t hbm_budget_bytes, int32_t max_active,
                              int32_t* status);
/* queue a member; returns at once with its id */
int anel_serve_submit(anel_serve* e, const anel_request* req, int64_t* id);
/* up to cap finished members into out (n of them); waits up to wait_ms
 * for the first when none is ready */
int anel_serve_poll(anel_serve* e, anel_result* out, int32_t cap, int32_t* n, int32_t wait_ms);
/* wait until every submitted member has finished */
int anel_serve_drain(anel_serve* e);
int anel_serve_stats_get(anel_serve* e, anel_serve_stats* st);
/* finishes queued and running members, then frees every context */
void anel_serve_destroy(anel_serve* e);

/* Drop-in form for the Fortran driver: bind the module arrays (host)
 * once, then call anel_rk_substep with the reference's rk_ss arguments;
 * every call copies the bound fields to the device and back. */
int anel_ns_init(const anel_grid_desc* grid, const anel_mg_params* mg, const anel_ns_params* ns);
int anel_bind_fields(const anel_fields* f);
void anel_rk_substep(const double* a1, const double* a2, const double* a3, const double* ec,
                     const double* dt_rk, const double* dt, const int32_t* psolve,
                     int32_t* stat);
int anel_ns_finalize(void);

#ifdef __cplusplus
}
#endif
#endif /* ANEL_H */
