// noalloc.cu -- divergence diagnostic that allocates no device memory.
//
// Who needs it: a host code that owns every device buffer itself and must
// not have a library allocate behind its back -- a Fortran driver whose
// device memory is pooled or pinned up front, a code running under a
// memory budget that is fully committed, or a caller inside a region where
// allocation is not allowed.  anel_ns_ctx_divergence works on an NS context
// (which allocates its fields and, on first use, a buffer of block
// partial sums); this entry point takes the caller's device arrays and
// keeps its partial sums in a fixed array in the library's own device
// memory image (a file-scope __device__ array, loaded with the module),
// so no cudaMalloc, cudaFree or allocating library routine is ever called.
//
// Limits and rules (also in include/anel.h):
//   * nz <= kNoAllocMaxPlanes: one partial pair per z-plane lives in the
//     fixed array; larger nz is rejected with ANEL_ERR_SIZE.
//   * The array is shared by every call on a device: calls whose GPU work
//     overlaps (different streams, or several host threads) race on it.
//     Order them on one stream, or synchronise between them.
//   * The first call on each device looks up the array's device address
//     (cudaGetSymbolAddress) and keeps it; make that first call before any
//     stream capture is started on the device.
//   * The maximum accumulator must start at zero: every call clears it
//     (cudaMemsetAsync on the fixed array) before the kernels run.
#include <mutex>

#include "anel_internal.h"

namespace anel {

constexpr int kNoAllocMaxPlanes = 4096;
constexpr int kNoAllocMaxDevices = 64;
// [0, 2P): per-plane sums of |div|*vol and vol; [2P]: bit pattern of the
// maximum |div| (non-negative doubles order like their bit patterns);
// [2P+1], [2P+2]: the results (mean, max)
constexpr int kNoAllocDoubles = 2 * kNoAllocMaxPlanes + 3;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

__global__ void k_div_planes(int nx, int ny, int nz, const double* __restrict__ u,
                             const double* __restrict__ v, const double* __restrict__ w,
                             const double* __restrict__ rdxc, const double* __restrict__ rdyc,
                             const double* __restrict__ rdzc, double* __restrict__ scratch) {
  // one CTA per z-plane k = 2 + blockIdx.x; fixed per-thread order, then a
  // fixed-order block reduction: the plane sums are deterministic
  __shared__ double sh[2][32];
  const int k = 2 + blockIdx.x;
  const int64_t X = nx + 2, XY = X * (ny + 2);
  const int64_t nxy = (int64_t)nx * ny;
  double s1 = 0.0, s2 = 0.0;
  unsigned long long m = 0;
  for (int64_t t = threadIdx.x; t < nxy; t += blockDim.x) {
    const int i = 2 + (int)(t % nx), j = 2 + (int)(t / nx);
    const int64_t c = (i - 1) + X * (j - 1) + XY * (k - 1);
    const double d = (u[c] - u[c - 1]) * rdxc[i - 1] + (v[c] - v[c - X]) * rdyc[j - 1] +
                     (w[c] - w[c - XY]) * rdzc[k - 1];
    const double vol = 1.0 / (rdxc[i - 1] * rdyc[j - 1] * rdzc[k - 1]);
    s1 += fabs(d) * vol;
    s2 += vol;
    const unsigned long long b = __double_as_longlong(fabs(d));
    m = b > m ? b : m;
  }
  for (int o = 16; o > 0; o >>= 1) {
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    const unsigned long long q = __shfl_xor_sync(0xffffffffu, m, o);
    m = q > m ? q : m;
  }
  const int wid = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    sh[0][wid] = s1;
    sh[1][wid] = s2;
    atomicMax(reinterpret_cast<unsigned long long*>(scratch + 2 * kNoAllocMaxPlanes), m);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) {
      a += sh[0][q];
      b += sh[1][q];
    }
    scratch[2 * blockIdx.x] = a;
    scratch[2 * blockIdx.x + 1] = b;
  }
}

__global__ void k_div_fold(int nz, double* __restrict__ scratch) {
  // plane partials summed in plane order by one thread (nz <= 4096)
  if (threadIdx.x != 0) return;
  double a = 0.0, b = 0.0;
  for (int k = 0; k < nz; ++k) {
    a += scratch[2 * k];
    b += scratch[2 * k + 1];
  }
  scratch[2 * kNoAllocMaxPlanes + 1] = a / b;
  scratch[2 * kNoAllocMaxPlanes + 2] =
      __longlong_as_double(*reinterpret_cast<const long long*>(scratch + 2 * kNoAllocMaxPlanes));
}

static std::mutex g_noalloc_mu;
static double* g_noalloc_ptr[kNoAllocMaxDevices] = {nullptr};

}  // namespace anel

extern "C" int anel_divergence_noalloc(int32_t nx, int32_t ny, int32_t nz, const double* u,
                                       const double* v, const double* w, const double* rdxc,
                                       const double* rdyc, const double* rdzc, double* out,
                                       void* stream) {
  using namespace anel;
  if (!u || !v || !w || !rdxc || !rdyc || !rdzc || !out) {
    set_error("anel_divergence_noalloc: null pointer argument");
    return ANEL_ERR_ARG;
  }
  if (nx < 1 || ny < 1 || nz < 1) {
    set_error("anel_divergence_noalloc: grid sizes must be positive (got %d %d %d)", nx, ny, nz);
    return ANEL_ERR_SIZE;
  }
  if (nz > kNoAllocMaxPlanes) {
    set_error("anel_divergence_noalloc: nz = %d exceeds the fixed scratch limit of %d z-planes", nz,
              kNoAllocMaxPlanes);
    return ANEL_ERR_SIZE;
  }
  int dev = -1;
  ANEL_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices) {
    set_error("anel_divergence_noalloc: device ordinal %d out of range", dev);
    return ANEL_ERR_ARG;
  }
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
      const cudaError_t e = cudaGetSymbolAddress((void**)&g_noalloc_ptr[dev], g_noalloc_scratch);
      if (e != cudaSuccess) {
        g_noalloc_ptr[dev] = nullptr;
        set_error("anel_divergence_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
        return ANEL_ERR_CUDA;
      }
    }
    scratch = g_noalloc_ptr[dev];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // the maximum accumulator starts at zero on every call
  ANEL_CUDA_TRY(cudaMemsetAsync(scratch + 2 * kNoAllocMaxPlanes, 0, sizeof(double), s));
  k_div_planes<<<nz, 256, 0, s>>>(nx, ny, nz, u, v, w, rdxc, rdyc, rdzc, scratch);
  k_div_fold<<<1, 32, 0, s>>>(nz, scratch);
  count_launch(2);
  const int st = check_launch("anel_divergence_noalloc");
  if (st != ANEL_OK) return st;
  ANEL_CUDA_TRY(cudaMemcpyAsync(out, scratch + 2 * kNoAllocMaxPlanes + 1, 2 * sizeof(double),
                                cudaMemcpyDeviceToHost, s));
  ANEL_CUDA_TRY(cudaStreamSynchronize(s));
  return ANEL_OK;
}
