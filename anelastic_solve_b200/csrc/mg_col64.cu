// mg_col64.cu -- the FP64 side of the column-layout cycle: the fine
// residual of the defect correction written into the FP32 column layout,
// and the correction added back into the reference layout.  Both move
// tiles of 32 (i) x 8 (j) x 32 (k) cells through shared memory, so the
// FP64 accesses run along i and the FP32 ones along k, each coalesced.
// Compiled with -fmad=false: the FP64 residual is the value fine_resid
// gives in the reference's order (the same numbers as the row-major path).
#include "mg_col.h"

namespace anel {

constexpr int kTI = 32, kTJ = 8, kTK = 32;

__device__ __forceinline__ double col_block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) s += sh[q];
  return s;
}

__global__ void __launch_bounds__(kTI * kTJ) k_col_resid_store(DevLevel<double> L, const double* __restrict__ phi,
                                                             const double* __restrict__ f, ColLevel E,
                                                             double* __restrict__ part) {
  __shared__ float tile[kTJ][kTI][kTK + 1];
  __shared__ double sh[kTJ];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int i0 = 2 + blockIdx.x * kTI, j = 2 + blockIdx.y * kTJ + ty, k0 = 2 + blockIdx.z * kTK;
  const int i = i0 + tx;
  const bool row = j <= L.ny + 1;
  double rr = 0.0, ff = 0.0;
  if (row && i <= L.nx + 1) {
    DevLevel<double> Lp = L;
    Lp.phi = const_cast<double*>(phi);
    Lp.src = const_cast<double*>(f);
    const int kn = min(kTK, L.nz + 2 - k0);
#pragma unroll 4
    for (int kk = 0; kk < kn; ++kk) {
      const int k = k0 + kk;
      const double r = fine_resid(Lp, i, j, k);
      const double fv = f[cidx(i, j, k, L.X, L.XY)];
      tile[ty][tx][kk] = (float)r;
      rr += r * r;
      ff += fv * fv;
    }
  }
  __syncthreads();
  // warp ty writes the columns of its row j, lane = k offset
  if (row && k0 + tx <= L.nz + 1) {
    const int in = min(kTI, L.nx + 2 - i0);
    for (int ii = 0; ii < in; ++ii) E.src[col_cell(E, i0 + ii, j, k0 + tx)] = tile[ty][ii][tx];
  }
  const double s1 = col_block_sum(rr, sh);
  const double s2 = col_block_sum(ff, sh);
  if (threadIdx.x == 0) {
    const int64_t b = blockIdx.x + (int64_t)gridDim.x * (blockIdx.y + (int64_t)gridDim.y * blockIdx.z);
    part[2 * b] = s1;
    part[2 * b + 1] = s2;
  }
}

__global__ void __launch_bounds__(kTI * kTJ) k_col_add_correction(DevLevel<double> L, double* __restrict__ phi,
                                                                ColLevel E) {
  __shared__ float tile[kTJ][kTI][kTK + 1];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int i0 = 2 + blockIdx.x * kTI, j = 2 + blockIdx.y * kTJ + ty, k0 = 2 + blockIdx.z * kTK;
  const bool row = j <= L.ny + 1;
  if (row && k0 + tx <= L.nz + 1) {
    const int in = min(kTI, L.nx + 2 - i0);
    for (int ii = 0; ii < in; ++ii) tile[ty][ii][tx] = E.phi[col_cell(E, i0 + ii, j, k0 + tx)];
  }
  __syncthreads();
  const int i = i0 + tx;
  if (row && i <= L.nx + 1) {
    const int kn = min(kTK, L.nz + 2 - k0);
#pragma unroll 4
    for (int kk = 0; kk < kn; ++kk) {
      const int64_t c = cidx(i, j, k0 + kk, L.X, L.XY);
      phi[c] = phi[c] + (double)tile[ty][tx][kk];
    }
  }
}

static dim3 col_tiles(const DevLevel<double>& L) {
  return dim3((unsigned)((L.nx + kTI - 1) / kTI), (unsigned)((L.ny + kTJ - 1) / kTJ),
              (unsigned)((L.nz + kTK - 1) / kTK));
}

int64_t col_resid_part_doubles(const DevLevel<double>& L) {
  const dim3 g = col_tiles(L);
  return 2 * (int64_t)g.x * g.y * g.z + fold_scratch_doubles();
}

void launch_col_resid_store(const DevLevel<double>& L, const double* phi, const double* f,
                            const ColLevel& E, double* part, double* out, cudaStream_t s) {
  const dim3 g = col_tiles(L);
  const int64_t n = (int64_t)g.x * g.y * g.z;
  k_col_resid_store<<<g, kTI * kTJ, 0, s>>>(L, phi, f, E, part);
  count_launch();
  launch_fold_pairs(part, n, part + 2 * n, out, s);
}

void launch_col_add_correction(const DevLevel<double>& L, double* phi, const ColLevel& E, cudaStream_t s) {
  k_col_add_correction<<<col_tiles(L), kTI * kTJ, 0, s>>>(L, phi, E);
  count_launch();
}

}  // namespace anel
