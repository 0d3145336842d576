// mg_coarse.h -- host side of the FP64 coarse-level direct solve (mg_coarse.cuh).
#pragma once

#include "mg_coarse.cuh"

namespace anel {

// Device buffers of one directly solved level.
struct DirectHost {
  DirectFac f{};
  double* d_buf = nullptr;
  size_t bytes = 0;
};

// Builds the basis, per-mode Thomas factors and work space of a level with
// nx x ny interior columns (x, y periodic) and nz rows: line coefficients
// a1..a4 (a1 == a2, a3 == a4 required), z coefficients cz5, cz6, dz5, dz6
// indexed k-1, z-ghost codes z1/zZ of the homogeneous rule (0 zero, 1 copy
// of row k=2, 2 copy of row k=nz+1; a periodic z is not supported).
// Returns ANEL_ERR_UNSUPPORTED when the level does not qualify.
int direct_build(DirectHost& D, int nx, int ny, int nz, double a1, double a2, double a3, double a4,
                 const double* cz5, const double* cz6, const double* dz5, const double* dz6, int z1, int zZ);
void direct_free(DirectHost& D);
// solve of the level in the cycle: L.src -> L.phi (FP32 column layout, ghosts
// written), for each of L's L.nm members (act: L.act); work: nm * nx*ny*nz
// doubles for a batch (null: the level's own block, one member)
void launch_direct_col(const DirectFac& F, const ColLevel& L, double* work, cudaStream_t s);
// the same on FP64 reference-layout arrays (interior of phi written)
void launch_direct_row(const DirectFac& F, const double* f, double* phi, int X, int64_t XY, cudaStream_t s);

}  // namespace anel
