// mg_col.cu -- FP32 column-layout cycle kernels (sweep, restriction,
// prolongation).  Compiled with multiply-add contraction allowed, like the
// row-major FP32 cycle: its accuracy is set by the FP64 defect correction.
#include "mg_col.h"

namespace anel {

template <int M, int NL, int MINB>
static void col_sweep_launch(const ColLevel& L, int color, const float* fac, cudaStream_t s) {
  const int64_t nlines = (int64_t)((L.nx + 1) / 2) * L.ny * L.nm;
  const int64_t per = (int64_t)kColWarps * NL;
  int64_t b = (nlines + per - 1) / per;
  const int64_t cap = 148 * MINB * 2;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  k_col_sweep<M, NL, MINB><<<(unsigned)b, 32 * kColWarps, 0, s>>>(L, color, fac);
}

template <int M>
static void col_sweep_tma_launch(const ColLevel& L, int color, const float* fac, int* err, cudaStream_t s) {
  const int64_t nlines = (int64_t)((L.nx + 1) / 2) * L.ny * L.nm;
  int64_t b = (nlines + kColTmaWarps - 1) / kColTmaWarps;
  const int64_t cap = 148 * 2 * 4;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  const size_t sm = col_tma_smem<M>(kColTmaWarps);
  set_smem_limit_once((const void*)k_col_sweep_tma<M>, (int)sm);
  k_col_sweep_tma<M><<<(unsigned)b, 32 * kColTmaWarps, sm, s>>>(L, color, fac, err);
}

// resident blocks per SM of k_col_sweep_rf<M> (set by col_sweep_prepare,
// outside any capture)
static int g_rf_occ[17];

template <int M>
static void col_sweep_rf_occupancy() {
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_col_sweep_rf<M>, 32 * kColWarps, 0) != cudaSuccess ||
      occ < 1)
    occ = 1;
  g_rf_occ[M] = occ;
}

template <int M>
static void col_sweep_rf_launch(const ColLevel& L, int color, const float* fac, cudaStream_t s) {
  const int64_t nlines = (int64_t)((L.nx + 1) / 2) * L.ny * L.nm;
  int64_t b = (nlines + kColWarps - 1) / kColWarps;
  const int64_t cap = 148 * (int64_t)(g_rf_occ[M] > 0 ? g_rf_occ[M] : 1);
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  k_col_sweep_rf<M><<<(unsigned)b, 32 * kColWarps, 0, s>>>(L, color, fac);
}

template <int M>
static void col_sweep_variant(const ColLevel& L, int color, const float* fac, int variant, int* err,
                              cudaStream_t s) {
  // the TMA-staged kernel needs every line of a colour to exist (even nx)
  if (variant == 3 && (L.nx % 2 != 0 || !err)) variant = 0;
  switch (variant) {
    case 1: col_sweep_launch<M, 1, 4>(L, color, fac, s); break;
    case 2: col_sweep_launch<M, 2, 2>(L, color, fac, s); break;
    case 3: col_sweep_tma_launch<M>(L, color, fac, err, s); break;
    case 4: col_sweep_rf_launch<M>(L, color, fac, s); break;
    default: col_sweep_launch<M, 1, 3>(L, color, fac, s); break;
  }
}

void col_sweep_prepare(int M) {
  switch (M) {
    case 2: col_sweep_rf_occupancy<2>(); break;
    case 3: col_sweep_rf_occupancy<3>(); break;
    case 4: col_sweep_rf_occupancy<4>(); break;
    case 6: col_sweep_rf_occupancy<6>(); break;
    case 8: col_sweep_rf_occupancy<8>(); break;
    case 12: col_sweep_rf_occupancy<12>(); break;
    default: col_sweep_rf_occupancy<16>(); break;
  }
  switch (M) {
    case 2: set_smem_limit_once((const void*)k_col_sweep_tma<2>, (int)col_tma_smem<2>(kColTmaWarps)); break;
    case 3: set_smem_limit_once((const void*)k_col_sweep_tma<3>, (int)col_tma_smem<3>(kColTmaWarps)); break;
    case 4: set_smem_limit_once((const void*)k_col_sweep_tma<4>, (int)col_tma_smem<4>(kColTmaWarps)); break;
    case 6: set_smem_limit_once((const void*)k_col_sweep_tma<6>, (int)col_tma_smem<6>(kColTmaWarps)); break;
    case 8: set_smem_limit_once((const void*)k_col_sweep_tma<8>, (int)col_tma_smem<8>(kColTmaWarps)); break;
    case 12: set_smem_limit_once((const void*)k_col_sweep_tma<12>, (int)col_tma_smem<12>(kColTmaWarps)); break;
    default: set_smem_limit_once((const void*)k_col_sweep_tma<16>, (int)col_tma_smem<16>(kColTmaWarps)); break;
  }
}

void launch_col_sweep(const ColLevel& L, int color, const float* fac, int M, int variant, int* err,
                      cudaStream_t s) {
  switch (M) {
    case 2: col_sweep_variant<2>(L, color, fac, variant, err, s); break;
    case 3: col_sweep_variant<3>(L, color, fac, variant, err, s); break;
    case 4: col_sweep_variant<4>(L, color, fac, variant, err, s); break;
    case 6: col_sweep_variant<6>(L, color, fac, variant, err, s); break;
    case 8: col_sweep_variant<8>(L, color, fac, variant, err, s); break;
    case 12: col_sweep_variant<12>(L, color, fac, variant, err, s); break;
    default: col_sweep_variant<16>(L, color, fac, variant, err, s); break;
  }
  count_launch();
}

static dim3 col_xfer_grid(int64_t per_row, int rows, int nm) {
  return dim3((unsigned)((per_row + kColXferThreads - 1) / kColXferThreads), (unsigned)rows, (unsigned)nm);
}

void launch_col_restrict(const ColLevel& F, const ColLevel& C, int cdir, cudaStream_t s) {
  const dim3 g = col_xfer_grid((int64_t)C.nx * (C.nz / 4), C.ny, C.nm);
  switch (cdir & 3) {
    case 1: k_col_restrict<1><<<g, kColXferThreads, 0, s>>>(F, C); break;
    case 2: k_col_restrict<2><<<g, kColXferThreads, 0, s>>>(F, C); break;
    default: k_col_restrict<3><<<g, kColXferThreads, 0, s>>>(F, C); break;
  }
  count_launch();
}

void launch_col_prolong(const ColLevel& F, const ColLevel& C, int cdir, cudaStream_t s) {
  // groups of fine columns sharing their coarse columns (k_col_prolong)
  const int cd = (cdir & 3) ? (cdir & 3) : 3;  // the kernel chosen below
  const bool cx = cd & 1, cy = cd & 2;
  const int64_t gx = cx ? F.nx / 2 + 1 : F.nx;
  const int gy = cy ? F.ny / 2 + 1 : F.ny;
  const dim3 g = col_xfer_grid(gx * (F.nz / 4), gy, F.nm);
  switch (cdir & 3) {
    case 1: k_col_prolong<1><<<g, kColXferThreads, 0, s>>>(F, C); break;
    case 2: k_col_prolong<2><<<g, kColXferThreads, 0, s>>>(F, C); break;
    default: k_col_prolong<3><<<g, kColXferThreads, 0, s>>>(F, C); break;
  }
  count_launch();
}

}  // namespace anel
