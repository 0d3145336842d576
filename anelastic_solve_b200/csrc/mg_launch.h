// mg_launch.h -- host-side launchers of the multigrid kernels.
#pragma once

#include "mg_device.cuh"

namespace anel {

// Grid size for a grid-stride kernel over `work` items: enough CTAs to
// cover the work, capped at 148 SMs x 8 resident CTAs of 256 threads.
inline int gs_blocks(int64_t work, int threads = 256) {
  int64_t b = (work + threads - 1) / threads;
  const int64_t cap = 148 * 8;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

template <typename T>
void launch_bdry(const DevLevel<T>& L, T* phi, cudaStream_t s);
template <typename T>
void launch_rb_sweep(const DevLevel<T>& L, int color, cudaStream_t s);
template <typename T>
void launch_zline(const DevLevel<T>& L, int color, const T* ap, const T* bp, cudaStream_t s);
// LJ z-line sweep (L.coef = the pcf line coefficients)
template <typename T>
void launch_zline_lj(const DevLevel<T>& L, int color, const T* ap, const T* bp, cudaStream_t s);
// partitioned FP32 z-line solver: kZSeg segments per line, each of
// 2..kZSegRows rows (lines of nz = kZSeg * m rows)
constexpr int kZSeg = 16;
constexpr int kZSegRows = 32;
// levels with at most this many lines of a colour use the cyclic-reduction
// line solve (one CTA per line) when its multipliers exist: about 6 us per
// sweep up to a few hundred lines, where the partitioned solver's per-CTA
// chain costs about 20 us; from ~1000 lines on the partitioned one is faster
constexpr int64_t kCRMaxLines = 512;
template <typename T>
void launch_zline_seg(const DevLevel<T>& L, int color, const SegFac<T>& F, cudaStream_t s);
// ghost table of an FP32 level with a homogeneous rule (L.gtab ignored)
void launch_ghost_table(const DevLevel<float>& L, int2* tab, cudaStream_t s);
template <typename T>
void launch_restrict(const DevLevel<T>& F, const DevLevel<T>& C, int cdir, cudaStream_t s);
template <typename T>
void launch_prolong(const DevLevel<T>& F, const DevLevel<T>& C, int cdir, cudaStream_t s);

// max|phin|, max|phin - phio| over the interior (bit patterns of the two
// non-negative maxima accumulated in out[0], out[1]), then phio <- phin on
// the whole ghosted array (mg_residual.F90:60-105).
void launch_relmax_copy(const DevLevel<double>& L, const double* phin, double* phio,
                        unsigned long long* out, cudaStream_t s);

// Deterministic sums over the interior of the FP64 fine level:
//   part[b] = per-block partial of (f - A phi)^2 and f^2; then one block
//   folds the partials in index order into out[0], out[1].
void launch_resid_norm(const DevLevel<double>& L, const double* phi, const double* f, double* part,
                       double* out, cudaStream_t s);
// doubles of partial sums the two launches below need
int64_t resid_part_doubles(const DevLevel<double>& L);

// FP64 fine residual r = f - A phi written to r (interior; ghosts 0) and
// its squared norm partials, for the mixed-precision defect correction.
void launch_resid_store(const DevLevel<double>& L, const double* phi, const double* f, float* r32,
                        double* part, double* out, cudaStream_t s);
// phi += (double) e on the interior (e FP32, same ghosted shape).
void launch_add_correction(const DevLevel<double>& L, double* phi, const float* e, cudaStream_t s);

}  // namespace anel
