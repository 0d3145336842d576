// anel_internal.h -- shared declarations of the B200 library (not installed).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/anel.h"

namespace anel {

// ---------------------------------------------------------------- errors
void set_error(const char* fmt, ...);
const char* last_error();

#define ANEL_CUDA_TRY(expr)                                                              \
  do {                                                                                   \
    cudaError_t _e = (expr);                                                             \
    if (_e != cudaSuccess) {                                                             \
      ::anel::set_error("%s failed: %s (%s:%d)", #expr, cudaGetErrorString(_e), __FILE__, \
                        __LINE__);                                                       \
      return ANEL_ERR_CUDA;                                                              \
    }                                                                                    \
  } while (0)

// Every kernel launch of this library goes through count_launch() so the
// total is observable through anel_kernel_launch_count().
// The thread-local count gives per-call reports (solve, step) that are
// right when several host threads drive contexts at once.
extern std::atomic<int64_t> g_launches;
extern thread_local int64_t t_launches;
inline void count_launch(int64_t n = 1) {
  g_launches.fetch_add(n, std::memory_order_relaxed);
  t_launches += n;
}
int check_launch(const char* what);
// Raise a kernel's dynamic shared-memory limit on the current device to at
// least `bytes` (set once per device and kernel, raised again only when a
// larger launch asks); safe to call from several host threads.
void set_smem_limit_once(const void* func, int bytes);
// Copy nwords 8-byte words by a kernel, between device memory and pinned
// host memory allocated with cudaHostAllocMapped (either direction).  Small
// readbacks and uploads of the step path go this way instead of through a
// copy engine, so they never queue behind large copies that other streams
// have in flight; the host reads a readback after synchronising the stream.
void copy_words(const void* src, void* dst, int64_t nwords, cudaStream_t s);
// Fixed-order fold of n (a, b) partial pairs into out[0..1] on the device;
// scratch holds fold_scratch_doubles() doubles.
int64_t fold_scratch_doubles();
void launch_fold_pairs(const double* part, int64_t n, double* scratch, double* out, cudaStream_t s);
// the same for nm members at once: member b's n pairs at part + b*pstride,
// its sums to out[2b], out[2b+1] (the order of each member's fold is the
// one-member order); scratch holds nm * fold_scratch_doubles() doubles
void launch_fold_pairs_members(const double* part, int64_t n, int64_t pstride, double* scratch, double* out,
                               int nm, cudaStream_t s);

// ------------------------------------------------------------ level maps
// One multigrid level, 1-based Fortran conventions of mg_init.F90:
// nk = interior+1, interior indices s..e (s = 2), ghosted dims X,Y,Z = e+1.
struct LevelGeom {
  int n[3];       // interior cells
  int nk[3];      // nxk (= n+1)
  int s[3], e[3]; // sxk..exk
  int X, Y, Z;    // ghosted dims
  int64_t G;      // X*Y*Z
  int64_t kp3d;   // 1-based workspace offset (reference layout, reported only)
  int kpx[3];     // 1-based 1-D metric offsets
};

// Ghost-cell rule of one level: wall types of the six faces in the
// reference's mg_bdry order and the additive constants of Neumann faces.
// face: 0=X2max 1=X3min 2=X2min 3=X3max 4=X1min 5=X1max.
struct BdryRule {
  int type[6];    // 0 periodic/none, 1 Neumann, 2 Dirichlet
  double val[6];  // phibc(level, face)
  double dist[6]; // spacing multiplying phibc (dyck(eym), dzck(szm), ...)
};

// Coefficients of one level in separable form (density r = r(z)):
//   c1 = cx1[i], c2 = cx2[i], c3 = cy3[j], c4 = cy4[j], c5 = cz5[k],
//   c6 = cz6[k], c7 = -(c1 + c2 + c3 + c4 + dz5[k] + dz6[k]).
// All arrays are indexed by the 1-based ghosted index minus one.
struct LevelCoef {
  std::vector<double> cx1, cx2, cy3, cy4, cz5, cz6, dz5, dz6;
};

}  // namespace anel
