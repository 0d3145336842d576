// mg_kernels64.cu -- FP64 instantiation of the multigrid kernels plus the
// FP64-only reductions.  Compiled with -fmad=false: no multiply-add
// contraction, so every value is rounded exactly as the reference's
// expressions evaluated left to right.
#include "mg_launch_impl.cuh"

namespace anel {

template void launch_bdry<double>(const DevLevel<double>&, double*, cudaStream_t);
template void launch_rb_sweep<double>(const DevLevel<double>&, int, cudaStream_t);
template void launch_zline<double>(const DevLevel<double>&, int, const double*, const double*, cudaStream_t);
template void launch_zline_lj<double>(const DevLevel<double>&, int, const double*, const double*, cudaStream_t);
template void launch_restrict<double>(const DevLevel<double>&, const DevLevel<double>&, int,
                                      cudaStream_t);
template void launch_prolong<double>(const DevLevel<double>&, const DevLevel<double>&, int,
                                     cudaStream_t);

// ------------------------------------------------------------- reductions
__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long v) {
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w > v ? w : v;
  }
  return v;
}

// Non-negative doubles order like their bit patterns, so the maxima are
// accumulated exactly (and order-independently) with integer atomicMax.
__global__ void k_relmax_copy(DevLevel<double> L, const double* __restrict__ phin,
                              double* __restrict__ phio, unsigned long long* out) {
  unsigned long long m1 = 0, m2 = 0;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < L.G;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int i = 1 + (int)(t % L.X);
    const int64_t r = t / L.X;
    const int j = 1 + (int)(r % L.Y);
    const int k = 1 + (int)(r / L.Y);
    const double n = phin[t];
    if (i >= 2 && i <= L.nx + 1 && j >= 2 && j <= L.ny + 1 && k >= 2 && k <= L.nz + 1) {
      const unsigned long long a = __double_as_longlong(fabs(n));
      const unsigned long long d = __double_as_longlong(fabs(n - phio[t]));
      m1 = a > m1 ? a : m1;
      m2 = d > m2 ? d : m2;
    }
    phio[t] = n;
  }
  m1 = warp_max_u64(m1);
  m2 = warp_max_u64(m2);
  if ((threadIdx.x & 31) == 0) {
    atomicMax(out, m1);
    atomicMax(out + 1, m2);
  }
}

void launch_relmax_copy(const DevLevel<double>& L, const double* phin, double* phio,
                        unsigned long long* out, cudaStream_t s) {
  k_relmax_copy<<<gs_blocks(L.G), 256, 0, s>>>(L, phin, phio, out);
  count_launch();
}

static constexpr int kNormThreads = 256;

__device__ __forceinline__ double block_sum(double v, double* sh) {
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

// kZBatch interior cells per thread (consecutive k): grid (ceil(nx/kResidX),
// ny, ceil(nz/kZBatch)), their stencil loads in flight together.  Each CTA
// writes its partial sums (fixed order); two fixed-order fold stages
// follow, so the norms are deterministic.
constexpr int kResidX = 128;
constexpr int kFoldBlocks = 1024;

template <bool kStore>
__global__ void __launch_bounds__(kResidX) k_resid_norm(DevLevel<double> L, const double* __restrict__ phi,
                                                       const double* __restrict__ f,
                                                       float* __restrict__ r32,
                                                       double* __restrict__ part) {
  __shared__ double sh[kResidX / 32];
  const int i = 2 + blockIdx.x * kResidX + threadIdx.x;
  const int j = 2 + blockIdx.y;
  const int k0 = 2 + blockIdx.z * kZBatch;
  double rr = 0.0, ff = 0.0;
  if (i <= L.nx + 1) {
    DevLevel<double> Lp = L;
    Lp.phi = const_cast<double*>(phi);
    Lp.src = const_cast<double*>(f);
    double res[kZBatch], fv[kZBatch];
#pragma unroll
    for (int q = 0; q < kZBatch; ++q) {
      const int k = k0 + q;
      if (k <= L.nz + 1) {
        res[q] = fine_resid(Lp, i, j, k);
        fv[q] = f[cidx(i, j, k, L.X, L.XY)];
      }
    }
#pragma unroll
    for (int q = 0; q < kZBatch; ++q) {
      const int k = k0 + q;
      if (k <= L.nz + 1) {
        if (kStore) r32[cidx(i, j, k, L.X, L.XY)] = (float)res[q];
        rr += res[q] * res[q];
        ff += fv[q] * fv[q];
      }
    }
  }
  const double s1 = block_sum(rr, sh);
  const double s2 = block_sum(ff, sh);
  if (threadIdx.x == 0) {
    const int64_t b = blockIdx.x + (int64_t)gridDim.x * (blockIdx.y + (int64_t)gridDim.y * blockIdx.z);
    part[2 * b] = s1;
    part[2 * b + 1] = s2;
  }
}

// part[0..2n) -> out2[0..2*gridDim.x): CTA b sums its contiguous chunk
// (blockIdx.y: member of a batch, its arrays pstride / ostride doubles on)
__global__ void k_fold_chunks(const double* __restrict__ part, int64_t n, double* __restrict__ out2,
                              int64_t pstride = 0, int64_t ostride = 0) {
  __shared__ double sh[kNormThreads / 32];
  part += blockIdx.y * pstride;
  out2 += blockIdx.y * ostride;
  const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
  const int64_t b0 = blockIdx.x * chunk;
  const int64_t b1 = b0 + chunk < n ? b0 + chunk : n;
  double a = 0.0, c = 0.0;
  for (int64_t q = b0 + threadIdx.x; q < b1; q += blockDim.x) {
    a += part[2 * q];
    c += part[2 * q + 1];
  }
  const double s1 = block_sum(a, sh);
  const double s2 = block_sum(c, sh);
  if (threadIdx.x == 0) {
    out2[2 * blockIdx.x] = s1;
    out2[2 * blockIdx.x + 1] = s2;
  }
}

__global__ void k_fold(const double* __restrict__ part, int nb, double* out, int64_t pstride = 0) {
  __shared__ double sh[kNormThreads / 32];
  part += blockIdx.x * pstride;
  out += 2 * blockIdx.x;
  double a = 0.0, b = 0.0;
  for (int q = threadIdx.x; q < nb; q += blockDim.x) {
    a += part[2 * q];
    b += part[2 * q + 1];
  }
  const double s1 = block_sum(a, sh);
  const double s2 = block_sum(b, sh);
  if (threadIdx.x == 0) {
    out[0] = s1;
    out[1] = s2;
  }
}

static dim3 resid_grid(const DevLevel<double>& L) {
  return dim3((unsigned)((L.nx + kResidX - 1) / kResidX), (unsigned)L.ny,
              (unsigned)((L.nz + kZBatch - 1) / kZBatch));
}

int64_t resid_part_doubles(const DevLevel<double>& L) {
  const dim3 g = resid_grid(L);
  return 2 * (int64_t)g.x * g.y * g.z + 2 * kFoldBlocks;
}

template <bool kStore>
static void launch_resid(const DevLevel<double>& L, const double* phi, const double* f, float* r32,
                         double* part, double* out, cudaStream_t s) {
  const dim3 g = resid_grid(L);
  const int64_t n = (int64_t)g.x * g.y * g.z;
  k_resid_norm<kStore><<<g, kResidX, 0, s>>>(L, phi, f, r32, part);
  double* part2 = part + 2 * n;
  k_fold_chunks<<<kFoldBlocks, kNormThreads, 0, s>>>(part, n, part2);
  k_fold<<<1, kNormThreads, 0, s>>>(part2, kFoldBlocks, out);
  count_launch(3);
}

int64_t fold_scratch_doubles() { return 2 * (int64_t)kFoldBlocks; }

void launch_fold_pairs(const double* part, int64_t n, double* scratch, double* out, cudaStream_t s) {
  k_fold_chunks<<<kFoldBlocks, kNormThreads, 0, s>>>(part, n, scratch);
  k_fold<<<1, kNormThreads, 0, s>>>(scratch, kFoldBlocks, out);
  count_launch(2);
}

void launch_fold_pairs_members(const double* part, int64_t n, int64_t pstride, double* scratch, double* out,
                               int nm, cudaStream_t s) {
  k_fold_chunks<<<dim3(kFoldBlocks, nm), kNormThreads, 0, s>>>(part, n, scratch, pstride, 2 * kFoldBlocks);
  k_fold<<<nm, kNormThreads, 0, s>>>(scratch, kFoldBlocks, out, 2 * kFoldBlocks);
  count_launch(2);
}

void launch_resid_norm(const DevLevel<double>& L, const double* phi, const double* f, double* part,
                       double* out, cudaStream_t s) {
  launch_resid<false>(L, phi, f, nullptr, part, out, s);
}

void launch_resid_store(const DevLevel<double>& L, const double* phi, const double* f, float* r32,
                        double* part, double* out, cudaStream_t s) {
  launch_resid<true>(L, phi, f, r32, part, out, s);
}

// phi += e on the interior: rows (j,k) walked kACRows at a time, the loads
// of all those rows issued before their stores.
constexpr int kACRows = 4;
__global__ void __launch_bounds__(256) k_add_correction(DevLevel<double> L, double* __restrict__ phi,
                                                       const float* __restrict__ e) {
  const int nrow = L.ny * L.nz;
  for (int row0 = blockIdx.x * kACRows; row0 < nrow; row0 += gridDim.x * kACRows) {
    int64_t base[kACRows];
#pragma unroll
    for (int u = 0; u < kACRows; ++u) {
      const int row = row0 + u < nrow ? row0 + u : nrow - 1;
      base[u] = cidx(0, 2 + row % L.ny, 2 + row / L.ny, L.X, L.XY);
    }
    for (int i = 2 + threadIdx.x; i <= L.nx + 1; i += blockDim.x) {
      double pv[kACRows];
      float ev[kACRows];
#pragma unroll
      for (int u = 0; u < kACRows; ++u) {
        pv[u] = phi[base[u] + i];
        ev[u] = e[base[u] + i];
      }
#pragma unroll
      for (int u = 0; u < kACRows; ++u)
        if (row0 + u < nrow) phi[base[u] + i] = pv[u] + (double)ev[u];
    }
  }
}

void launch_add_correction(const DevLevel<double>& L, double* phi, const float* e, cudaStream_t s) {
  const int64_t groups = ((int64_t)L.ny * L.nz + kACRows - 1) / kACRows;
  k_add_correction<<<(unsigned)(groups < 148 * 8 ? groups : 148 * 8), 256, 0, s>>>(L, phi, e);
  count_launch();
}

}  // namespace anel
