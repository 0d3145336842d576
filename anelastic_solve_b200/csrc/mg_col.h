// mg_col.h -- launchers of the column-layout FP32 cycle (mg_col.cuh) and of
// the FP64 <-> column transfers of the defect correction.
#pragma once

#include "mg_col.cuh"

namespace anel {

// rows per lane the column sweep is built for (nz = 32 * M)
inline bool col_rows_supported(int M) {
  return M == 2 || M == 3 || M == 4 || M == 6 || M == 8 || M == 12 || M == 16;
}
// variants of the sweep: k_col_sweep<M, NL, MINB> with 0 = one line per
// warp step, 3 CTAs/SM; 1 = one line, 4 CTAs/SM; 2 = two lines, 2 CTAs/SM;
// 3 = k_col_sweep_tma (source columns staged by bulk copies; err: a
// host-mapped int set to 1 if a copy wait ran out); 4 = k_col_sweep_rf
// (factors in registers, persistent, next line prefetched into L2)
constexpr int kColSweepVariants = 5;
void launch_col_sweep(const ColLevel& L, int color, const float* fac, int M, int variant, int* err,
                      cudaStream_t s);
// sets the launch attributes every sweep variant for M needs (call before
// any stream capture)
void col_sweep_prepare(int M);
// coarse f from the fine residual (cdir: bit 0 x, bit 1 y coarsened); the
// caller zeroes coarse phi first
void launch_col_restrict(const ColLevel& F, const ColLevel& C, int cdir, cudaStream_t s);
// fine phi += interpolated coarse correction, ghost copies included
void launch_col_prolong(const ColLevel& F, const ColLevel& C, int cdir, cudaStream_t s);

// FP64 fine residual r = f - A phi (reference layout) stored as FP32 into
// E.src (column layout), with the squared norms of r and f folded into
// out[0], out[1] in a fixed order.
void launch_col_resid_store(const DevLevel<double>& L, const double* phi, const double* f,
                            const ColLevel& E, double* part, double* out, cudaStream_t s);
int64_t col_resid_part_doubles(const DevLevel<double>& L);
// phi += (double) E.phi on the interior (phi in the reference layout)
void launch_col_add_correction(const DevLevel<double>& L, double* phi, const ColLevel& E, cudaStream_t s);

// The same for the E.nm members of a batch, member b's FP64 arrays in mt[b]
// (a device table) and E.act masking the inactive ones: the residual's
// norms go to out[2b], out[2b+1], folded in the one-member order; part
// holds col_resid_part_doubles_members(L, E.nm) doubles.  The ghost pass
// needs the homogeneous ghost table of L (L.gtab).
int64_t col_resid_part_doubles_members(const DevLevel<double>& L, int nm);
void launch_col_resid_store_members(const DevLevel<double>& L, const MemberIO* mt, const ColLevel& E,
                                    double* part, double* out, cudaStream_t s);
void launch_col_add_correction_members(const DevLevel<double>& L, const MemberIO* mt, const ColLevel& E,
                                       cudaStream_t s);
void launch_bdry_members(const DevLevel<double>& L, const MemberIO* mt, const int* act, int nm, cudaStream_t s);

}  // namespace anel
