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
void launch_restrict(const DevLevel<T>& F, const DevLevel<T>& C, int cdir, cudaStream_t s) {
  k_restrict<T><<<gs_blocks(C.G), 256, 0, s>>>(F, C, cdir);
  count_launch();
}
template <typename T>
void launch_prolong(const DevLevel<T>& F, const DevLevel<T>& C, int cdir, cudaStream_t s) {
  const int64_t w = (int64_t)F.nx * F.ny * F.nz;
  k_prolong<T><<<gs_blocks(w), 256, 0, s>>>(F, C, cdir);
  count_launch();
}

}  // namespace anel
