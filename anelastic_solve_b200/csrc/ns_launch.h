// ns_launch.h -- host launchers of the RK3 sub-step kernels.
#pragma once

#include "anel_internal.h"
#include "ns_device.cuh"

namespace anel {

// Device pointers of the column-independent CN factors of one variable.
struct CNFacHost {
  const double *ap, *bp, *c, *t1, *t2, *rb, *isbc;
};

void launch_rhs_accum(const NSDev& D, double a1, double a2, double dt, bool first, cudaStream_t s);
void launch_cn(const NSDev& D, int var, double* fld, const double* q, const CNFacHost& F, double a3,
               double rkdt, const ZRule& R, cudaStream_t s);
void launch_psource(const NSDev& D, double dt, cudaStream_t s);
void launch_pgrad(const NSDev& D, double dt, const ZRule& Ru, const ZRule& Rv, const ZRule& Rw,
                  cudaStream_t s);
void launch_ghost_field(const NSDev& D, double* a, const ZRule& R, cudaStream_t s);
void launch_cfl_max(const NSDev& D, unsigned long long* out, cudaStream_t s);
int64_t divergence_blocks(const NSDev& D);
void launch_divergence(const NSDev& D, unsigned long long* mx, double* part, cudaStream_t s);

}  // namespace anel
