// mg_col.cu -- FP32 column-layout cycle kernels (sweep, restriction,
// prolongation).  Compiled with multiply-add contraction allowed, like the
// row-major FP32 cycle: its accuracy is set by the FP64 defect correction.
#include "mg_col.h"

namespace anel {

void launch_col_sweep(const ColLevel& L, int color, const float* fac, int M, cudaStream_t s) {
  const int64_t nlines = (int64_t)((L.nx + 1) / 2) * L.ny;
  int64_t b = (nlines + kColWarps - 1) / kColWarps;
  const int64_t cap = 148 * 6;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  const dim3 grid((unsigned)b), block(32 * kColWarps);
  switch (M) {
    case 2: k_col_sweep<2><<<grid, block, 0, s>>>(L, color, fac); break;
    case 3: k_col_sweep<3><<<grid, block, 0, s>>>(L, color, fac); break;
    case 4: k_col_sweep<4><<<grid, block, 0, s>>>(L, color, fac); break;
    case 6: k_col_sweep<6><<<grid, block, 0, s>>>(L, color, fac); break;
    case 8: k_col_sweep<8><<<grid, block, 0, s>>>(L, color, fac); break;
    case 12: k_col_sweep<12><<<grid, block, 0, s>>>(L, color, fac); break;
    default: k_col_sweep<16><<<grid, block, 0, s>>>(L, color, fac); break;
  }
  count_launch();
}

void launch_col_restrict(const ColLevel& F, const ColLevel& C, int cdir, cudaStream_t s) {
  const dim3 g((unsigned)((int64_t)C.nx * C.ny), (unsigned)((C.nz + 127) / 128));
  switch (cdir & 3) {
    case 1: k_col_restrict<1><<<g, 128, 0, s>>>(F, C); break;
    case 2: k_col_restrict<2><<<g, 128, 0, s>>>(F, C); break;
    default: k_col_restrict<3><<<g, 128, 0, s>>>(F, C); break;
  }
  count_launch();
}

void launch_col_prolong(const ColLevel& F, const ColLevel& C, int cdir, cudaStream_t s) {
  const dim3 g((unsigned)((int64_t)F.nx * F.ny), (unsigned)((F.nz + 127) / 128));
  switch (cdir & 3) {
    case 1: k_col_prolong<1><<<g, 128, 0, s>>>(F, C); break;
    case 2: k_col_prolong<2><<<g, 128, 0, s>>>(F, C); break;
    default: k_col_prolong<3><<<g, 128, 0, s>>>(F, C); break;
  }
  count_launch();
}

}  // namespace anel
