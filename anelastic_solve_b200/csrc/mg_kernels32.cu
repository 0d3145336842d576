// mg_kernels32.cu -- FP32 instantiation of the multigrid kernels, used by
// the inner V-cycle of the mixed-precision defect correction.  Compiled
// with multiply-add contraction allowed (this path is not bit-matched to
// the reference; its accuracy is set by the FP64 outer loop).
#include "mg_launch_impl.cuh"

namespace anel {

template void launch_bdry<float>(const DevLevel<float>&, float*, cudaStream_t);
template void launch_rb_sweep<float>(const DevLevel<float>&, int, cudaStream_t);
template void launch_zline<float>(const DevLevel<float>&, int, const float*, const float*, cudaStream_t);
template void launch_zline_lj<float>(const DevLevel<float>&, int, const float*, const float*, cudaStream_t);
template void launch_zline_seg<float>(const DevLevel<float>&, int, const SegFac<float>&, cudaStream_t);

void launch_ghost_table(const DevLevel<float>& L, int2* tab, cudaStream_t s) {
  const int64_t ng = L.G - (int64_t)L.nx * L.ny * L.nz;
  k_ghost_table<float><<<gs_blocks(ng), 256, 0, s>>>(L, tab);
  count_launch();
}

template void launch_restrict<float>(const DevLevel<float>&, const DevLevel<float>&, int,
                                     cudaStream_t);
template void launch_prolong<float>(const DevLevel<float>&, const DevLevel<float>&, int,
                                    cudaStream_t);

}  // namespace anel
