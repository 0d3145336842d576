// ns_launch.h -- host launchers of the RK3 sub-step kernels.
#pragma once

#include "anel_internal.h"
#include "ns_device.cuh"

namespace anel {

// Device pointers of the column-independent CN factors of one variable.
// Column-independent CN data per row k = 1..nz+2 (index k-1): eliminated
// sub-diagonal ap and diagonal bp, super-diagonal c, explicit weights t1,
// t2, wall-row right-hand side rb and flag isbc, and the raw sub-diagonal
// and diagonal (the LES solve adds its eddy terms to these).
struct CNFacHost {
  const double *ap, *bp, *c, *t1, *t2, *rb, *isbc, *sub, *diag;
};

void launch_rhs_accum(const NSDev& D, double a1, double a2, double dt, bool first, cudaStream_t s);
// variant: rows per load batch and columns per block of the column solve
// (0: 8 rows, 256; 1: 16, 128; 2: 16, 256; 3: 32, 128), chosen by the
// autotuner; every variant computes the same bits
constexpr int kCNVariants = 4;
void launch_cn(const NSDev& D, int var, double* fld, const double* q, const CNFacHost& F, double a3,
               double rkdt, const ZRule& R, int variant, cudaStream_t s);
// var_advance_CN_PL with the eddy terms (Vmodel = SSM): per-column
// elimination; b: G-sized scratch for the eliminated diagonal (the
// super-diagonal is formed again from kT in the back substitution).
// kT = nuT (u, v, w), kappaT (rho), nappaT (scal1).
// variant: rows per load batch and columns per block (0: 8 rows, 256;
// 1: 4, 128; 2: 8, 128; 3: 16, 128), chosen by the autotuner; every
// variant computes the same bits
constexpr int kCNLesVariants = 4;
void launch_cn_les(const NSDev& D, int var, double* fld, const double* q, const CNFacHost& F, double a3,
                   double rkdt, const ZRule& R, const double* kT, double* b, int variant, cudaStream_t s);
// SGSdiff (straincal.F90:339-414): modS, nuT, kappaT, nappaT on the
// interior from the model profiles, then their ghosts ('cfluc').
void launch_sgs(const NSDev& D, const ZRule& cfluc, cudaStream_t s);
void launch_psource(const NSDev& D, double dt, cudaStream_t s);
// shear-layer initial state (NSSolver::init_shear): prof = tanh(zc)[Z],
// |zc|[Z]; noise from the Park-Miller sequence of seed, element q*G + c
// for u (q = 0), v (1), w (2) at Fortran linear index c.
void launch_init_shear(const NSDev& D, const double* prof, uint32_t seed, double amp, double zmax,
                       cudaStream_t s);
// hist (may be null): a copy of p's interior (pressure guess history)
void launch_pgrad(const NSDev& D, double dt, const ZRule& Ru, const ZRule& Rv, const ZRule& Rw,
                  cudaStream_t s, double* hist = nullptr);
// p = 2 h1 - h2 on the interior (the extrapolated pressure guess)
void launch_extrap(const NSDev& D, double* p, const double* h1, const double* h2, cudaStream_t s);
void launch_ghost_field(const NSDev& D, double* a, const ZRule& R, cudaStream_t s);
// clipVS (Routines.F90:301-380) of a cell-centred field's interior
void launch_clip(const NSDev& D, double* a, double vmin, double vmax, cudaStream_t s);
void launch_cfl_max(const NSDev& D, unsigned long long* out, cudaStream_t s);
int64_t divergence_blocks(const NSDev& D);
// plane statistics (NSsolver.F90:288-395): center_velocity of one
// component, squared fluctuations, weighted x-y plane averages of every
// plane (part: plane_part_doubles scratch) and the profile update
void launch_center(const NSDev& D, const double* in, double* out, int dir, int stretched, int corrected,
                   const double* e, const double* c, cudaStream_t s);
void launch_fluct_sq(const NSDev& D, const double* a, const double* mean, double* out, cudaStream_t s);
int64_t plane_part_doubles(const NSDev& D);
void launch_plane_avg(const NSDev& D, const double* a, const double* wx, const double* wy, double area,
                      double* part, double* out, cudaStream_t s);
void launch_diag_update(int Z, double dtt, const double* m, double* dg, cudaStream_t s);
// cfl (may be null): also calcdt's CFL maximum of the same fields, as the
// bit pattern of a non-negative double, atomically maxed into *cfl
void launch_divergence(const NSDev& D, unsigned long long* mx, double* part, cudaStream_t s,
                       unsigned long long* cfl = nullptr);

}  // namespace anel
