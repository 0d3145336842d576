// mg_launch_impl.cuh -- launcher templates shared by the FP64 and FP32
// kernel translation units (each instantiates its own type).
#pragma once

#include "mg_launch.h"

namespace anel {

template <typename T>
void launch_bdry(const DevLevel<T>& L, T* phi, cudaStream_t s) {
  const int64_t ng = L.G - (int64_t)L.nx * L.ny * L.nz;
  k_bdry<T><<<gs_blocks(ng), 256, 0, s>>>(L, phi);
  count_launch();
}
template <typename T>
void launch_rb_sweep(const DevLevel<T>& L, int color, cudaStream_t s) {
  const int64_t w = (int64_t)((L.nx + 1) / 2) * L.ny * L.nz;
  k_rb_sweep<T><<<gs_blocks(w), 256, 0, s>>>(L, color);
  count_launch();
}
template <typename T>
void launch_zline(const DevLevel<T>& L, int color, const T* ap, const T* bp, cudaStream_t s) {
  const int pairs = (L.nx + 1) / 2;
  const int64_t cols = (int64_t)pairs * L.ny;
  // few long lines (coarse levels of the FP32 cycle): one warp per line
  if (sizeof(T) == 4 && cols < 16384 && L.nz <= 512 && L.nz >= 2) {
    constexpr int NMAX = 512;
    const int warps = 4;
    const size_t sm = (size_t)warps * 4 * NMAX * sizeof(T);
    const unsigned blocks = (unsigned)((cols + warps - 1) / warps);
    set_smem_limit_once((const void*)k_zline_pcr<T, NMAX>, (int)sm);
    k_zline_pcr<T, NMAX><<<blocks, 32 * warps, sm, s>>>(L, color);
    count_launch();
    return;
  }
  const int tx = 64;
  dim3 grid((unsigned)((pairs + tx - 1) / tx), (unsigned)L.ny, 1u);
  k_zline<T, false><<<grid, tx, 0, s>>>(L, color, ZFac<T>{ap, bp});
  count_launch();
}
template <typename T>
void launch_zline_lj(const DevLevel<T>& L, int color, const T* ap, const T* bp, cudaStream_t s) {
  const int pairs = (L.nx + 1) / 2;
  const int tx = 64;
  dim3 grid((unsigned)((pairs + tx - 1) / tx), (unsigned)L.ny, 1u);
  k_zline<T, true><<<grid, tx, 0, s>>>(L, color, ZFac<T>{ap, bp});
  count_launch();
}
template <typename T>
void launch_zline_seg(const DevLevel<T>& L, int color, const SegFac<T>& F, cudaStream_t s) {
  const int64_t cols = (int64_t)((L.nx + 1) / 2) * L.ny;
  if (F.cr && cols <= kCRMaxLines && L.nz <= kCRMaxRows) {
    k_zline_cr<T><<<(unsigned)cols, (unsigned)((L.nz + 31) / 32 * 32), 0, s>>>(L, color, F);
    count_launch();
    return;
  }
  const size_t sm = (size_t)kZSegRows * kZSeg * 32 * sizeof(T);
  set_smem_limit_once((const void*)k_zline_seg<T, kZSeg, kZSegRows>, (int)sm);
  dim3 block(32, kZSeg, 1);
  k_zline_seg<T, kZSeg, kZSegRows><<<(unsigned)((cols + 31) / 32), block, sm, s>>>(L, color, F);
  count_launch();
}
template <typename T>
void launch_restrict(const DevLevel<T>& F, const DevLevel<T>& C, int cdir, cudaStream_t s) {
  const dim3 g((unsigned)((C.nx + 127) / 128), (unsigned)C.Y, (unsigned)((C.Z + kZBatch - 1) / kZBatch));
  switch (cdir & 7) {
    case 0: k_restrict<T, 0><<<g, 128, 0, s>>>(F, C); break;
    case 1: k_restrict<T, 1><<<g, 128, 0, s>>>(F, C); break;
    case 2: k_restrict<T, 2><<<g, 128, 0, s>>>(F, C); break;
    case 3: k_restrict<T, 3><<<g, 128, 0, s>>>(F, C); break;
    case 4: k_restrict<T, 4><<<g, 128, 0, s>>>(F, C); break;
    case 5: k_restrict<T, 5><<<g, 128, 0, s>>>(F, C); break;
    case 6: k_restrict<T, 6><<<g, 128, 0, s>>>(F, C); break;
    default: k_restrict<T, 7><<<g, 128, 0, s>>>(F, C); break;
  }
  count_launch();
}
template <typename T>
void launch_prolong(const DevLevel<T>& F, const DevLevel<T>& C, int cdir, cudaStream_t s) {
  const dim3 g((unsigned)((F.nx + 127) / 128), (unsigned)F.ny, (unsigned)((F.nz + kZBatch - 1) / kZBatch));
  switch (cdir & 7) {
    case 0: k_prolong<T, 0><<<g, 128, 0, s>>>(F, C); break;
    case 1: k_prolong<T, 1><<<g, 128, 0, s>>>(F, C); break;
    case 2: k_prolong<T, 2><<<g, 128, 0, s>>>(F, C); break;
    case 3: k_prolong<T, 3><<<g, 128, 0, s>>>(F, C); break;
    case 4: k_prolong<T, 4><<<g, 128, 0, s>>>(F, C); break;
    case 5: k_prolong<T, 5><<<g, 128, 0, s>>>(F, C); break;
    case 6: k_prolong<T, 6><<<g, 128, 0, s>>>(F, C); break;
    default: k_prolong<T, 7><<<g, 128, 0, s>>>(F, C); break;
  }
  count_launch();
}

}  // namespace anel
