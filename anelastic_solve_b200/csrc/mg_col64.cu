// mg_col64.cu -- the FP64 side of the column-layout cycle: the fine
// residual of the defect correction written into the FP32 column layout,
// and the correction added back into the reference layout.  A thread owns
// kColRows consecutive z-cells of one (i,j) column: its FP64 accesses run
// along i across the warp (coalesced) and march along k with the z
// neighbours kept in registers, and its FP32 accesses are two 16-byte
// vectors of one column that together fill a 32-byte sector.
// Compiled with -fmad=false: the FP64 residual is the value fine_resid
// gives in the reference's order (the same numbers as the row-major path).
#include "mg_col.h"
#include "mg_launch.h"

namespace anel {

constexpr int kTI = 32, kTJ = 8, kColRows = 8;

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

// grid (ceil(nx/32), ceil(ny/8), nz/kColRows * members), block 32 x 8.
// Member b of a batch (mt non-null) takes its phi and f from mt[b], its
// FP32 columns from E's member b and its partial sums from the b-th block
// of part; an inactive member's blocks return at once.
__global__ void __launch_bounds__(kTI * kTJ) k_col_resid_store(DevLevel<double> L, const double* __restrict__ phi,
                                                             const double* __restrict__ f, ColLevel Eb,
                                                             double* __restrict__ part,
                                                             const MemberIO* __restrict__ mt) {
  __shared__ double sh[kTJ];
  const int nzb = L.nz / kColRows;
  const int b = blockIdx.z / nzb;
  if (!col_active(Eb, b)) return;  // the whole block
  if (mt) {
    phi = mt[b].phi;
    f = mt[b].rhs;
  }
  const ColLevel E = col_member(Eb, b);
  const int i = 2 + blockIdx.x * kTI + (threadIdx.x & 31);
  const int j = 2 + blockIdx.y * kTJ + (threadIdx.x >> 5);
  const int k0 = 2 + (blockIdx.z - b * nzb) * kColRows;
  double rr = 0.0, ff = 0.0;
  if (i <= L.nx + 1 && j <= L.ny + 1) {
    const double* cx1 = cx1p(L);
    const double* cx2 = cx2p(L);
    const double* cy3 = cy3p(L);
    const double* cy4 = cy4p(L);
    const double* cz5 = cz5p(L);
    const double* cz6 = cz6p(L);
    const double* dz5 = dz5p(L);
    const double* dz6 = dz6p(L);
    const double a1 = cx1[i - 1], a2 = cx2[i - 1], a3 = cy3[j - 1], a4 = cy4[j - 1];
    const int64_t X = L.X, XY = L.XY;
    int64_t c = cidx(i, j, k0, L.X, L.XY);
    double pm = phi[c - XY], pc = phi[c];
    float r[kColRows];
#pragma unroll
    for (int q = 0; q < kColRows; ++q) {
      const int k = k0 + q;
      const double pp = phi[c + XY];
      // fine_resid's order: c1 W + c2 E + c3 S + c4 N + c5 B + c6 T + c7 P
      const double diag = -(a1 + a2 + a3 + a4 + dz5[k - 1] + dz6[k - 1]);
      double acc = a1 * phi[c - 1];
      acc = acc + a2 * phi[c + 1];
      acc = acc + a3 * phi[c - X];
      acc = acc + a4 * phi[c + X];
      acc = acc + cz5[k - 1] * pm;
      acc = acc + cz6[k - 1] * pp;
      acc = acc + diag * pc;
      const double fv = f[c];
      const double res = fv - acc;
      r[q] = (float)res;
      rr += res * res;
      ff += fv * fv;
      pm = pc;
      pc = pp;
      c += XY;
    }
    float4* o = reinterpret_cast<float4*>(E.src + col_cell(E, i, j, k0));
#pragma unroll
    for (int q = 0; q < kColRows / 4; ++q) o[q] = make_float4(r[4 * q], r[4 * q + 1], r[4 * q + 2], r[4 * q + 3]);
  }
  const double s1 = col_block_sum(rr, sh);
  const double s2 = col_block_sum(ff, sh);
  if (threadIdx.x == 0) {
    const int64_t q = blockIdx.x + (int64_t)gridDim.x * (blockIdx.y + (int64_t)gridDim.y * blockIdx.z);
    part[2 * q] = s1;
    part[2 * q + 1] = s2;
  }
}

__global__ void __launch_bounds__(kTI * kTJ) k_col_add_correction(DevLevel<double> L, double* __restrict__ phi,
                                                                ColLevel Eb, const MemberIO* __restrict__ mt) {
  const int nzb = L.nz / kColRows;
  const int b = blockIdx.z / nzb;
  if (!col_active(Eb, b)) return;
  if (mt) phi = mt[b].phi;
  const ColLevel E = col_member(Eb, b);
  const int i = 2 + blockIdx.x * kTI + (threadIdx.x & 31);
  const int j = 2 + blockIdx.y * kTJ + (threadIdx.x >> 5);
  const int k0 = 2 + (blockIdx.z - b * nzb) * kColRows;
  if (i > L.nx + 1 || j > L.ny + 1) return;
  const float4* e4 = reinterpret_cast<const float4*>(E.phi + col_cell(E, i, j, k0));
  float e[kColRows];
#pragma unroll
  for (int q = 0; q < kColRows / 4; ++q) {
    const float4 v = e4[q];
    e[4 * q] = v.x;
    e[4 * q + 1] = v.y;
    e[4 * q + 2] = v.z;
    e[4 * q + 3] = v.w;
  }
  const int64_t c = cidx(i, j, k0, L.X, L.XY), XY = L.XY;
  double p[kColRows];
#pragma unroll
  for (int q = 0; q < kColRows; ++q) p[q] = phi[c + q * XY];
#pragma unroll
  for (int q = 0; q < kColRows; ++q) phi[c + q * XY] = p[q] + (double)e[q];
}

static dim3 col_tiles(const DevLevel<double>& L, int nm = 1) {
  return dim3((unsigned)((L.nx + kTI - 1) / kTI), (unsigned)((L.ny + kTJ - 1) / kTJ),
              (unsigned)(L.nz / kColRows * nm));
}

int64_t col_resid_part_doubles(const DevLevel<double>& L) {
  const dim3 g = col_tiles(L);
  return 2 * (int64_t)g.x * g.y * g.z + fold_scratch_doubles();
}

void launch_col_resid_store(const DevLevel<double>& L, const double* phi, const double* f,
                            const ColLevel& E, double* part, double* out, cudaStream_t s) {
  const dim3 g = col_tiles(L);
  const int64_t n = (int64_t)g.x * g.y * g.z;
  k_col_resid_store<<<g, kTI * kTJ, 0, s>>>(L, phi, f, E, part, nullptr);
  count_launch();
  launch_fold_pairs(part, n, part + 2 * n, out, s);
}

void launch_col_add_correction(const DevLevel<double>& L, double* phi, const ColLevel& E, cudaStream_t s) {
  k_col_add_correction<<<col_tiles(L), kTI * kTJ, 0, s>>>(L, phi, E, nullptr);
  count_launch();
}

int64_t col_resid_part_doubles_members(const DevLevel<double>& L, int nm) {
  const dim3 g = col_tiles(L);
  return nm * (2 * (int64_t)g.x * g.y * g.z + fold_scratch_doubles());
}

void launch_col_resid_store_members(const DevLevel<double>& L, const MemberIO* mt, const ColLevel& E,
                                    double* part, double* out, cudaStream_t s) {
  const dim3 g1 = col_tiles(L);
  const int64_t n = (int64_t)g1.x * g1.y * g1.z;  // blocks of one member
  k_col_resid_store<<<col_tiles(L, E.nm), kTI * kTJ, 0, s>>>(L, nullptr, nullptr, E, part, mt);
  count_launch();
  // member b's partials are the b-th run of n pairs (blockIdx.z runs over
  // the members' z-blocks in member order)
  launch_fold_pairs_members(part, n, 2 * n, part + 2 * n * E.nm, out, E.nm, s);
}

void launch_col_add_correction_members(const DevLevel<double>& L, const MemberIO* mt, const ColLevel& E,
                                       cudaStream_t s) {
  k_col_add_correction<<<col_tiles(L, E.nm), kTI * kTJ, 0, s>>>(L, nullptr, E, mt);
  count_launch();
}

// ghost pass of every active member's FP64 phi (blockIdx.y: member)
__global__ void k_bdry_members(DevLevel<double> L, const MemberIO* __restrict__ mt, const int* __restrict__ act) {
  const int b = blockIdx.y;
  if (act && !act[b]) return;
  bdry_range(L, mt[b].phi, blockIdx.x * (int64_t)blockDim.x + threadIdx.x, (int64_t)gridDim.x * blockDim.x);
}

void launch_bdry_members(const DevLevel<double>& L, const MemberIO* mt, const int* act, int nm, cudaStream_t s) {
  const int64_t ng = L.G - (int64_t)L.nx * L.ny * L.nz;
  k_bdry_members<<<dim3((unsigned)gs_blocks(ng), (unsigned)nm), 256, 0, s>>>(L, mt, act);
  count_launch();
}

}  // namespace anel
