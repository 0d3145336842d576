// mg_solver.cu -- host side of the B200 multigrid pressure solver: level
// maps (mg_init.F90), coarse metric hierarchy (mg_grids.F90, mg_coeff.F90),
// level coefficients (mg_pfpde.F90, mg_phpde.F90), the V-cycle schedule
// (mg_cycle.F90) and the solve loop (mg_solver.F90), all driving the
// sm_100a kernels of mg_device.cuh.  Built with -ffp-contract=off for the
// host compiler so the coefficients round exactly as the reference's.
#include "mg_solver.h"
#include "tune.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

namespace anel {

static inline int imax(int a, int b) { return a > b ? a : b; }
int zline_segment_factors(int n, int P, const std::vector<double>& sub, const std::vector<double>& dia,
                          const std::vector<double>& sup, std::vector<double>& out);
int zline_cr_factors(int n, int S, const std::vector<double>& sub, const std::vector<double>& dia,
                     const std::vector<double>& sup, std::vector<double>& out);
int col_sweep_factors(int n, int M, const std::vector<double>& sub, const std::vector<double>& dia,
                      const std::vector<double>& sup, std::vector<float>& out);
int col_sweep_factors_d(int n, int M, const std::vector<double>& sub, const std::vector<double>& dia,
                        const std::vector<double>& sup, std::vector<double>& out);
static bool graph_solve_enabled();

// ------------------------------------------------------------------ init
MGSolver* MGSolver::create(const anel_grid_desc* g, const anel_mg_params* p, int device,
                           int* status) {
  MGSolver* s = new MGSolver();
  const int st = s->init(g, p, device);
  if (status) *status = st;
  if (st != ANEL_OK) {
    delete s;
    return nullptr;
  }
  return s;
}

int MGSolver::init(const anel_grid_desc* g, const anel_mg_params* p, int device) {
  if (!g || !p) {
    set_error("null grid or params");
    return ANEL_ERR_ARG;
  }
  prm_ = *p;
  device_ = device;
  nx_ = g->nx;
  ny_ = g->ny;
  nz_ = g->nz;
  L_[0] = g->xL;
  L_[1] = g->yL;
  L_[2] = g->zL;
  const int n[3] = {nx_, ny_, nz_};
  if (nx_ < 1 || ny_ < 1 || nz_ < 1) {
    set_error("grid sizes must be positive (got %d %d %d)", nx_, ny_, nz_);
    return ANEL_ERR_SIZE;
  }
  if (p->smoother != ANEL_SMOOTHER_RBPGS && p->smoother != ANEL_SMOOTHER_LJ &&
      p->smoother != ANEL_SMOOTHER_ZLINE) {
    set_error("unknown smoother %d", p->smoother);
    return ANEL_ERR_ARG;
  }
  if (p->mode != ANEL_MODE_LITERAL && p->mode != ANEL_MODE_METRIC) {
    set_error("unknown mode %d", p->mode);
    return ANEL_ERR_ARG;
  }
  if (p->precision != ANEL_PREC_FP64 && p->precision != ANEL_PREC_MIXED) {
    set_error("unknown precision %d", p->precision);
    return ANEL_ERR_ARG;
  }
  if (p->maxcy < 1) {
    set_error("maxcy must be >= 1");
    return ANEL_ERR_ARG;
  }
  const double* src[3][6] = {{g->xe, g->xc, g->dxe, g->dxc, g->rdxe, g->rdxc},
                             {g->ye, g->yc, g->dye, g->dyc, g->rdye, g->rdyc},
                             {g->ze, g->zc, g->dze, g->dzc, g->rdze, g->rdzc}};
  for (int d = 0; d < 3; ++d)
    for (int a = 0; a < 6; ++a) {
      if (!src[d][a]) {
        set_error("grid metric array %d of direction %d is null", a, d);
        return ANEL_ERR_ARG;
      }
      fm_[d][a].assign(src[d][a], src[d][a] + n[d] + 2);
    }
  // ---- level sizes and index maps (mg_init.F90:86-220) ----
  ngrid_ = imax(p->levels[0], imax(p->levels[1], p->levels[2]));
  if (ngrid_ < 2 || ngrid_ > ANEL_MAX_LEVELS) {
    set_error("ngrid = %d; need 2..%d levels (a single level has no coarse grid)", ngrid_,
              ANEL_MAX_LEVELS);
    return ANEL_ERR_SIZE;
  }
  for (int d = 0; d < 3; ++d) {
    const int Ld = p->levels[d];
    // ZLINE may keep z unrefined (horizontal semi-coarsening, an extension)
    if (Ld < 2 && !(d == 2 && p->smoother == ANEL_SMOOTHER_ZLINE)) {
      set_error("no coarsening in direction %d at the finest level (mg_check_size codes 10-12)",
                d + 1);
      return ANEL_ERR_SIZE;
    }
    nC_[d] = n[d] >> (Ld - 1);
    if (nC_[d] < 1 || (nC_[d] << (Ld - 1)) != n[d]) {
      set_error("n%d = %d is not nC*2^(levels-1) (mg_check_size codes 4-6)", d + 1, n[d]);
      return ANEL_ERR_SIZE;
    }
  }
  for (int l = 1; l <= ngrid_; ++l)
    for (int d = 0; d < 3; ++d)
      geo_[l].nk[d] = (nC_[d] << (imax(l + p->levels[d] - ngrid_, 1) - 1)) + 1;
  for (int d = 0; d < 3; ++d) {
    geo_[ngrid_].s[d] = 2;
    geo_[ngrid_].e[d] = n[d] + 1;
  }
  for (int l = ngrid_ - 1; l >= 1; --l)
    for (int d = 0; d < 3; ++d) {
      const bool coarser = geo_[l].nk[d] < geo_[l + 1].nk[d];
      geo_[l].s[d] = coarser ? geo_[l + 1].s[d] / 2 + 1 : geo_[l + 1].s[d];
      geo_[l].e[d] = coarser ? (geo_[l + 1].e[d] - 1) / 2 + 1 : geo_[l + 1].e[d];
    }
  int64_t kp3 = 1;
  int kx[3] = {1, 1, 1};
  for (int l = ngrid_; l >= 1; --l) {
    LevelGeom& G = geo_[l];
    for (int d = 0; d < 3; ++d) G.n[d] = G.e[d] - G.s[d] + 1;
    G.X = G.e[0] + 1;
    G.Y = G.e[1] + 1;
    G.Z = G.e[2] + 1;
    G.G = (int64_t)G.X * G.Y * G.Z;
    G.kp3d = kp3;
    kp3 += G.G;
    for (int d = 0; d < 3; ++d) {
      G.kpx[d] = kx[d];
      kx[d] += G.nk[d] + 1;
    }
  }
  // ---- boundary codes (mg_init.F90:265-328) ----
  for (int f = 0; f < 6; ++f)
    if (p->tbc[f] < 0 || p->tbc[f] > 2) {
      set_error("bad boundary type tbc(%d) = %d", f + 1, p->tbc[f]);
      return ANEL_ERR_BC;
    }
  // periodic must be paired
  if ((p->tbc[4] == 0) != (p->tbc[5] == 0) || (p->tbc[2] == 0) != (p->tbc[0] == 0) ||
      (p->tbc[1] == 0) != (p->tbc[3] == 0)) {
    set_error("a direction mixes periodic and wall faces");
    return ANEL_ERR_BC;
  }
  std::memset(bd_, 0, sizeof(bd_));
  bd_[9] = p->tbc[4];
  bd_[18] = p->tbc[5];
  bd_[5] = p->tbc[2];
  bd_[1] = p->tbc[0];
  bd_[3] = p->tbc[1];
  bd_[7] = p->tbc[3];
  for (int f = 0; f < 6; ++f) {
    phibc_[ngrid_][f] = p->vbc[f];
    for (int l = ngrid_ - 1; l >= 1; --l) phibc_[l][f] = 0.0;
  }
  build_metric_hierarchy();
  if (p->smoother == ANEL_SMOOTHER_LJ) build_lj_coefficients();
  build_agglomerated();
  // boundary rules; spacings indexed without the level offset, exactly as
  // mg_bdry.F90:106-181 (dyck(eym) etc.)
  for (int l = 1; l <= ngrid_; ++l) {
    const LevelGeom& G = geo_[l];
    BdryRule R;
    const int bdf[6] = {bd_[1], bd_[3], bd_[5], bd_[7], bd_[9], bd_[18]};
    const double dist[6] = {hDC_[1][G.e[1]], hDC_[2][G.s[2]], hDC_[1][G.s[1]],
                            hDC_[2][G.e[2]], hDC_[0][G.s[0]], hDC_[0][G.e[0]]};
    for (int f = 0; f < 6; ++f) {
      R.type[f] = bdf[f];
      R.val[f] = phibc_[l][f];
      R.dist[f] = dist[f];
    }
    rule_[l] = R;
    for (int f = 0; f < 6; ++f) R.val[f] = 0.0;
    rule_hom_[l] = R;
  }
  // ---- device ----
  ANEL_CUDA_TRY(cudaSetDevice(device_));
  ANEL_CUDA_TRY(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  ANEL_CUDA_TRY(cudaEventCreate(&ev0_));
  ANEL_CUDA_TRY(cudaEventCreate(&ev1_));
  const bool mixed = p->precision == ANEL_PREC_MIXED;
  // column layout of the FP32 levels: z never coarsened, nz = 32*M
  bool col_ok = mixed && p->smoother == ANEL_SMOOTHER_ZLINE && nz_ % 32 == 0 &&
                col_rows_supported(nz_ / 32);
  for (int l = 1; l <= ngrid_ && col_ok; ++l) col_ok = geo_[l].n[2] == nz_;
  for (int l = 1; l <= ngrid_; ++l) {
    const int64_t G = geo_[l].G;
    // FP32 arrays are sized for either layout, so the choice can still
    // fall back to the row-major one below
    const int64_t G32 = col_ok ? std::max<int64_t>(G, (int64_t)geo_[l].X * geo_[l].Y * col_stride(nz_)) : G;
    const size_t ncoef = 2 * (size_t)geo_[l].X + 2 * (size_t)geo_[l].Y + 4 * (size_t)geo_[l].Z;
    if (!mixed || l == ngrid_) {
      ANEL_CUDA_TRY(cudaMalloc(&d_phi64_[l], G * sizeof(double)));
      ANEL_CUDA_TRY(cudaMalloc(&d_src64_[l], G * sizeof(double)));
      ANEL_CUDA_TRY(cudaMemset(d_phi64_[l], 0, G * sizeof(double)));
      ANEL_CUDA_TRY(cudaMemset(d_src64_[l], 0, G * sizeof(double)));
    }
    ANEL_CUDA_TRY(cudaMalloc(&d_coef64_[l], ncoef * sizeof(double)));
    if (p->smoother == ANEL_SMOOTHER_LJ) {
      ANEL_CUDA_TRY(cudaMalloc(&d_zf64_[l], 2 * (size_t)geo_[l].Z * sizeof(double)));
      ANEL_CUDA_TRY(cudaMalloc(&d_zf32_[l], 2 * (size_t)geo_[l].Z * sizeof(float)));
      ANEL_CUDA_TRY(cudaMalloc(&d_ljc64_[l], ncoef * sizeof(double)));
      if (mixed) ANEL_CUDA_TRY(cudaMalloc(&d_ljc32_[l], ncoef * sizeof(float)));
    }
    if (p->smoother == ANEL_SMOOTHER_ZLINE) {
      ANEL_CUDA_TRY(cudaMalloc(&d_zf64_[l], 2 * (size_t)geo_[l].Z * sizeof(double)));
      ANEL_CUDA_TRY(cudaMalloc(&d_zf32_[l], 2 * (size_t)geo_[l].Z * sizeof(float)));
      const int nz = geo_[l].n[2];
      // (the kernel indexes a segment's rows with 32-bit offsets m * X * Y)
      if (mixed && nz % kZSeg == 0 && nz >= 2 * kZSeg && nz <= kZSeg * kZSegRows &&
          (int64_t)(nz / kZSeg + 1) * geo_[l].X * geo_[l].Y < (int64_t)1 << 31)
      {
        ANEL_CUDA_TRY(cudaMalloc(&d_zseg32_[l], (4 * (size_t)geo_[l].Z + 4 * kZSeg * kZSeg) *
                                                    sizeof(float)));
        if (nz <= kCRMaxRows) {
          int st = 0;
          while ((1 << st) < nz) ++st;
          zcr_steps_[l] = st;
          ANEL_CUDA_TRY(cudaMalloc(&d_zcr32_[l], (2 * (size_t)st + 1) * nz * sizeof(float)));
        }
      }
    }
    if (mixed) {
      ANEL_CUDA_TRY(cudaMalloc(&d_phi32_[l], G32 * sizeof(float)));
      ANEL_CUDA_TRY(cudaMalloc(&d_src32_[l], G32 * sizeof(float)));
      ANEL_CUDA_TRY(cudaMemset(d_phi32_[l], 0, G32 * sizeof(float)));
      ANEL_CUDA_TRY(cudaMemset(d_src32_[l], 0, G32 * sizeof(float)));
      ANEL_CUDA_TRY(cudaMalloc(&d_coef32_[l], ncoef * sizeof(float)));
      // ghost table of the FP32 cycle's homogeneous rule (32-bit indices)
      if (G < ((int64_t)1 << 31)) {
        const int64_t ngh = G - (int64_t)geo_[l].n[0] * geo_[l].n[1] * geo_[l].n[2];
        ANEL_CUDA_TRY(cudaMalloc(&d_gtab32_[l], (size_t)ngh * sizeof(int2)));
        launch_ghost_table(L32(l, true), d_gtab32_[l], stream_);
      }
    }
  }
  ANEL_CUDA_TRY(cudaStreamSynchronize(stream_));
  for (int l = 1; l <= ngrid_; ++l)
    if ((d_zseg32_[l] || col_ok) && d_gtab32_[l]) {
      const int st = build_self_ghosting(l);
      if (st != ANEL_OK) return st;
    }
  for (int l = 1; l <= ngrid_ && col_ok; ++l) col_ok = d_img32_[l] != nullptr;
  col_ = col_ok;
  if (col_) {
    ANEL_CUDA_TRY(cudaHostAlloc(&h_err_, sizeof(int), cudaHostAllocMapped));
    *h_err_ = 0;
    ANEL_CUDA_TRY(cudaHostGetDevicePointer((void**)&d_err_, h_err_, 0));
    colM_ = nz_ / 32;
    for (int l = 1; l <= ngrid_; ++l)
      ANEL_CUDA_TRY(cudaMalloc(&d_colfac_[l], (size_t)col_fac_floats(colM_) * sizeof(float)));
  }
  ANEL_CUDA_TRY(cudaMalloc(&d_max_, 2 * sizeof(unsigned long long)));
  int64_t npart = resid_part_doubles(L64(ngrid_));
  if (col_) npart = std::max(npart, col_resid_part_doubles(L64(ngrid_)));
  ANEL_CUDA_TRY(cudaMalloc(&d_part_, (size_t)npart * sizeof(double)));
  ANEL_CUDA_TRY(cudaMalloc(&d_norm_, 2 * sizeof(double)));
  ANEL_CUDA_TRY(cudaHostAlloc(&h_pin_, 4 * sizeof(double), cudaHostAllocMapped));
  choose_direct_level();
  // default density r == 1
  std::vector<double> rz(geo_[ngrid_].Z, 1.0);
  int st = build_coefficients(rz);
  if (st != ANEL_OK) return st;
  st = upload_coefficients();
  if (st != ANEL_OK) return st;
  return col_ ? tune_col() : ANEL_OK;
}

// Autotuning of the column sweep: every variant of launch_col_sweep timed
// on each level's own arrays (scratch at this point: the cycle overwrites
// them) with CUDA events, one warm-up sweep pair and then kTuneReps pairs;
// the fastest is kept per (device, rows per lane, level columns) for the
// whole process.
// A sweep that gave up on a copy wait leaves *h_err_ = 1 (after the stream
// has been synchronised): report it once as a timeout.
int MGSolver::take_kernel_error(const char* what) {
  if (h_err_ && *reinterpret_cast<volatile int*>(h_err_) != 0) {
    *reinterpret_cast<volatile int*>(h_err_) = 0;
    set_error("%s: a bounded wait for a bulk copy ran out in the column sweep", what);
    return ANEL_ERR_TIMEOUT;
  }
  return ANEL_OK;
}

int MGSolver::tune_col() {
  constexpr int kTuneReps = 4;
  // kernel attributes of every variant are set here, outside any capture
  col_sweep_prepare(colM_);
  // ANEL_COL_VARIANT=v forces one variant everywhere (no timing): for tests
  const char* force = std::getenv("ANEL_COL_VARIANT");
  if (force && *force) {
    const int v = std::atoi(force);
    if (v < 0 || v >= kColSweepVariants) {
      set_error("ANEL_COL_VARIANT=%s: variants are 0..%d", force, kColSweepVariants - 1);
      return ANEL_ERR_ARG;
    }
    for (int l = 1; l <= ngrid_; ++l) colvar_[l] = v;
    return ANEL_OK;
  }
  for (int l = 1; l <= ngrid_; ++l) {
    char key[128];
    std::snprintf(key, sizeof(key), "k_col_sweep dev%d M=%d lines=%dx%d", device_, colM_, geo_[l].n[0],
                  geo_[l].n[1]);
    int v = tune_lookup(key);
    if (v < 0 && !tune_enabled()) v = 0;
    if (v < 0) {
      const ColLevel L = C32(l);
      std::vector<double> ms(kColSweepVariants, 0.0);
      for (int q = 0; q < kColSweepVariants; ++q) {
        for (int c = 0; c < 2; ++c) launch_col_sweep(L, c, d_colfac_[l], colM_, q, d_err_, stream_);
        ANEL_CUDA_TRY(cudaEventRecord(ev0_, stream_));
        for (int r = 0; r < kTuneReps; ++r)
          for (int c = 0; c < 2; ++c) launch_col_sweep(L, c, d_colfac_[l], colM_, q, d_err_, stream_);
        ANEL_CUDA_TRY(cudaEventRecord(ev1_, stream_));
        ANEL_CUDA_TRY(cudaEventSynchronize(ev1_));
        float t = 0.f;
        ANEL_CUDA_TRY(cudaEventElapsedTime(&t, ev0_, ev1_));
        ms[q] = t / (2.0 * kTuneReps);
      }
      const int le = check_launch("column sweep tuning");
      if (le != ANEL_OK) return le;
      const int ke = take_kernel_error("column sweep tuning");
      if (ke != ANEL_OK) return ke;
      v = 0;
      for (int q = 1; q < kColSweepVariants; ++q)
        if (ms[q] < ms[v]) v = q;
      tune_store(key, v, ms);
    }
    colvar_[l] = v;
  }
  return ANEL_OK;
}

MGSolver::~MGSolver() {
  if (device_ >= 0) cudaSetDevice(device_);
  if (g32x_) cudaGraphExecDestroy(g32x_);
  for (int l = 0; l <= ANEL_MAX_LEVELS; ++l) {
    cudaFree(d_phi64_[l]);
    cudaFree(d_src64_[l]);
    cudaFree(d_coef64_[l]);
    cudaFree(d_phi32_[l]);
    cudaFree(d_src32_[l]);
    cudaFree(d_coef32_[l]);
    cudaFree(d_zf64_[l]);
    cudaFree(d_ljc64_[l]);
    cudaFree(d_ljc32_[l]);
    cudaFree(d_zf32_[l]);
    cudaFree(d_zseg32_[l]);
    cudaFree(d_zcr32_[l]);
    cudaFree(d_gtab32_[l]);
    cudaFree(d_img32_[l]);
    cudaFree(d_colfac_[l]);
  }
  direct_free(dir_);
  direct_free(dirfine_);
  batch_free();
  if (h_err_) cudaFreeHost(h_err_);
  if (gsolve_) cudaGraphExecDestroy(gsolve_);
  if (side_) cudaStreamDestroy(side_);
  cudaFree(d_conv_);
  cudaFree(d_max_);
  cudaFree(d_part_);
  cudaFree(d_norm_);
  cudaFree(d_io_phi_);
  cudaFree(d_io_rhs_);
  if (h_pin_) cudaFreeHost(h_pin_);
  for (cudaEvent_t e : prof_ev_) cudaEventDestroy(e);
  if (ev0_) cudaEventDestroy(ev0_);
  if (ev1_) cudaEventDestroy(ev1_);
  if (stream_) cudaStreamDestroy(stream_);
}

// ------------------------------------------------- coarse metric hierarchy
// mg_grids.F90:54-448 and mg_coeff.F90:77-145.  Arrays are 1-based
// (index 0 unused) over the concatenated per-level 1-D workspace.
void MGSolver::build_metric_hierarchy() {
  const int tmin[3] = {prm_.tbc[4], prm_.tbc[2], prm_.tbc[1]};
  const int tmax[3] = {prm_.tbc[5], prm_.tbc[0], prm_.tbc[3]};
  for (int d = 0; d < 3; ++d) {
    const int nw = geo_[1].kpx[d] + geo_[1].nk[d] + 1;  // nworkx
    std::vector<double>& E = hE_[d];
    std::vector<double>& C = hC_[d];
    std::vector<double>& DC = hDC_[d];
    std::vector<double>& DE = hDE_[d];
    E.assign(nw + 1, 0.0);
    C.assign(nw + 1, 0.0);
    DC.assign(nw + 1, 99999999999.0);
    DE.assign(nw + 1, 99999999999.0);
    const int nf = geo_[ngrid_].nk[d];
    const int k0 = geo_[ngrid_].kpx[d];
    for (int q = 1; q <= nf + 1; ++q) {
      E[q + k0 - 1] = fm_[d][0][q - 1];
      C[q + k0 - 1] = fm_[d][1][q - 1];
      DE[q + k0 - 1] = fm_[d][2][q - 1];
      DC[q + k0 - 1] = fm_[d][3][q - 1];
    }
    const double LL = fm_[d][0][nf] - fm_[d][0][0];
    const int Ld = prm_.levels[d];
    for (int lvl = ngrid_; lvl >= ngrid_ - Ld + 2; --lvl) {
      const int lC = lvl - 1;
      const int nc = geo_[lC].nk[d], nfl = geo_[lvl].nk[d];
      const int kc = geo_[lC].kpx[d], kf = geo_[lvl].kpx[d];
      if (tmin[d] == 0) {
        const double h = LL / (double)nc;
        for (int q = 1; q <= nc + 1; ++q) E[q + kc - 1] = -h + h * (double)q;
        for (int q = 2; q <= nc + 1; ++q) C[q + kc - 1] = (E[q + kc - 1] + E[q + kc - 2]) / 2.0;
        C[kc] = E[kc] - 0.5 * h;
        for (int q = 1; q <= nc + 1; ++q) {
          DC[q + kc - 1] = h;
          DE[q + kc - 1] = h;
        }
        continue;
      }
      E[kc] = E[kf];
      for (int q = 2; q <= nc; ++q) {
        const int f = (kf - 1) + 2 * q - 2, c = (kc - 1) + q;
        C[c] = C[f] + DC[f] * 0.5;
        E[c] = C[c] + DC[f];
      }
      C[kc] = (tmin[d] == 2) ? C[kf] : C[kf] - 0.5 * DE[kf + 1];
      {
        const int c = kc + nc, f = kf + nfl;
        if (tmax[d] == 2) {
          C[c] = C[f];
          E[c] = E[f];
        } else {
          C[c] = C[f] + 0.5 * DE[f - 1];
          E[c] = E[f] + 0.5 * DC[f - 1];
        }
      }
      for (int q = 2; q <= nc; ++q) {
        const int c = (kc - 1) + q;
        DE[c] = C[c + 1] - C[c];
        DC[c] = E[c] - E[c - 1];
      }
      DC[kc] = 0.0;
      DE[kc] = (tmin[d] == 2) ? C[kc + 1] - C[kc] : DE[kc + 1];
      {
        const int c = kc + nc;
        if (tmax[d] == 2) {
          DE[c] = C[c] - C[c - 1];
          DC[c] = E[c] - E[c - 1];
        } else {
          DE[c] = DE[c - 1];
          DC[c] = DC[c - 1];
        }
      }
    }
    for (int lvl = ngrid_ - Ld + 1; lvl >= 2; --lvl) {
      const int lC = lvl - 1;
      const int nc = geo_[lC].nk[d];
      const int kc = geo_[lC].kpx[d], kf = geo_[lvl].kpx[d];
      for (int q = 1; q <= nc + 1; ++q) {
        E[(kc - 1) + q] = E[(kf - 1) + q];
        C[(kc - 1) + q] = C[(kf - 1) + q];
        DE[(kc - 1) + q] = DE[(kf - 1) + q];
        DC[(kc - 1) + q] = DC[(kf - 1) + q];
      }
    }
    // pcf_(2d+1), pcf_(2d+2) of mg_coeff.F90:77-99
    pA_[d].assign(nw + 1, 0.0);
    pB_[d].assign(nw + 1, 0.0);
    for (int l = 1; l <= ngrid_; ++l) {
      const int s0 = geo_[l].kpx[d];
      for (int q = 2; q <= geo_[l].nk[d]; ++q) {
        const int gq = s0 + q - 1;
        pA_[d][gq] = 1.0 / (DC[gq] * DE[gq - 1]);
        pB_[d][gq] = 1.0 / (DC[gq] * DE[gq]);
      }
    }
  }
}

// METRIC mode coarse metrics: cell-centred agglomeration (coarse edge q
// is fine edge 2q-1; widths and centres from the edges; ghosts mirror their
// interior neighbour).  The reference's mg_grids recursion is not used
// here because its edges drift on strongly stretched grids.
void MGSolver::build_agglomerated() {
  const int ng = ngrid_;
  for (int d = 0; d < 3; ++d) {
    ag_[ng][d][0] = fm_[d][0];
    ag_[ng][d][1] = fm_[d][1];
    ag_[ng][d][2] = fm_[d][3];
    ag_[ng][d][3] = fm_[d][2];
    for (int l = ng - 1; l >= 1; --l) {
      if (geo_[l].nk[d] == geo_[l + 1].nk[d]) {
        for (int a = 0; a < 4; ++a) ag_[l][d][a] = ag_[l + 1][d][a];
        continue;
      }
      const int n = geo_[l].nk[d] - 1;
      std::vector<double> E(n + 2), C(n + 2), DC(n + 2), DE(n + 2);
      const std::vector<double>& Ef = ag_[l + 1][d][0];
      for (int q = 1; q <= n + 1; ++q) E[q - 1] = Ef[2 * q - 2];
      for (int q = 2; q <= n + 1; ++q) {
        DC[q - 1] = E[q - 1] - E[q - 2];
        C[q - 1] = 0.5 * (E[q - 1] + E[q - 2]);
      }
      DC[0] = DC[1];
      DC[n + 1] = DC[n];
      C[0] = E[0] - 0.5 * DC[0];
      E[n + 1] = E[n] + DC[n + 1];
      C[n + 1] = E[n] + 0.5 * DC[n + 1];
      for (int q = 1; q <= n + 1; ++q) DE[q - 1] = C[q] - C[q - 1];
      DE[n + 1] = DE[n];
      // a direction whose finer spacings are one value is coarsened
      // exactly: every coarse spacing is twice it
      const std::vector<double>& DCf = ag_[l + 1][d][2];
      const std::vector<double>& DEf = ag_[l + 1][d][3];
      bool uni = true;
      for (size_t q = 0; q < DCf.size(); ++q)
        if (!(DCf[q] == DCf[0] && DEf[q] == DCf[0])) uni = false;
      if (uni)
        for (int q = 0; q < n + 2; ++q) DC[q] = DE[q] = 2.0 * DCf[0];
      ag_[l][d][0] = E;
      ag_[l][d][1] = C;
      ag_[l][d][2] = DC;
      ag_[l][d][3] = DE;
    }
  }
}

// ------------------------------------------------------- coefficients
// rz[k-1] = r(:,:,k) on the fine level, k = 1..nz+2.
int MGSolver::build_coefficients(const std::vector<double>& rz) {
  const int ng = ngrid_;
  const int Zf = geo_[ng].Z;
  auto R = [&](int k) {  // fine r at 1-based k; k < 1 clamps to the ghost plane
    if (k < 1) k = 1;
    if (k > Zf) k = Zf;
    return rz[k - 1];
  };
  for (int l = 1; l <= ng; ++l) {
    const LevelGeom& G = geo_[l];
    LevelCoef& c = coef_[l];
    c.cx1.assign(G.X, 0.0);
    c.cx2.assign(G.X, 0.0);
    c.cy3.assign(G.Y, 0.0);
    c.cy4.assign(G.Y, 0.0);
    c.cz5.assign(G.Z, 0.0);
    c.cz6.assign(G.Z, 0.0);
    c.dz5.assign(G.Z, 0.0);
    c.dz6.assign(G.Z, 0.0);
    const int kstep = (geo_[ng].nk[2] - 1) / (G.nk[2] - 1);
    if (prm_.mode == ANEL_MODE_LITERAL) {
      const double dlx = L_[0] / (double)(float)(G.nk[0] - 1);
      const double ex = 1.0 / (dlx * dlx);
      const double dly = L_[1] / (double)(float)(G.nk[1] - 1);
      const double ey = 1.0 / (dly * dly);
      const double dlz = L_[2] / (double)(float)(G.nk[2] - 1);
      const double ez = 1.0 / (dlz * dlz);
      for (int i = 1; i <= G.X; ++i) c.cx1[i - 1] = c.cx2[i - 1] = ex;
      for (int j = 1; j <= G.Y; ++j) c.cy3[j - 1] = c.cy4[j - 1] = ey;
      if (l == ng) {  // mgdpfpde (mg_pfpde.F90:41-60)
        for (int k = G.s[2]; k <= G.e[2]; ++k) {
          c.cz5[k - 1] = ez * 0.5 * (R(k) + R(k - 1)) / R(k - 1);
          c.cz6[k - 1] = ez * 0.5 * (R(k) + R(k + 1)) / R(k + 1);
          c.dz5[k - 1] = ez * 0.5 * (R(k) + R(k - 1)) / R(k);
          c.dz6[k - 1] = ez * 0.5 * (R(k) + R(k + 1)) / R(k);
        }
      } else {  // mgdphpde (mg_phpde.F90:111-199)
        int ks = 0;
        for (int k = G.s[2]; k <= G.e[2]; ++k) {
          const int km = 2 * kstep * k - 3 * (kstep - 1);
          int q = (km - kstep) / 2;
          c.cz5[k - 1] = ez * 0.5 * (R(q) + R(q - 1)) / R(q - 1);
          q = (km + kstep) / 2;
          c.cz6[k - 1] = ez * 0.5 * (R(q) + R(q + 1)) / R(q + 1);
          ks = q;  // the value left over for the diagonal loop
        }
        if (bd_[9] == 1) c.cx1[G.s[0] - 1] = 0.0;
        if (bd_[18] == 1) c.cx2[G.e[0] - 1] = 0.0;
        if (bd_[5] == 1) c.cy3[G.s[1] - 1] = 0.0;
        if (bd_[1] == 1) c.cy4[G.e[1] - 1] = 0.0;
        if (bd_[3] == 1) c.cz5[G.s[2] - 1] = 0.0;
        if (bd_[7] == 1) c.cz6[G.e[2] - 1] = 0.0;
        const double d5 = ez * 0.5 * (R(ks) + R(ks - 1)) / R(ks);
        const double d6 = ez * 0.5 * (R(ks) + R(ks + 1)) / R(ks);
        for (int k = G.s[2]; k <= G.e[2]; ++k) {
          c.dz5[k - 1] = d5;
          c.dz6[k - 1] = d6;
        }
      }
    } else {  // METRIC
      const bool fine = (l == ng);
      // 1/(dxc(q)*dxe(q-1)) and 1/(dxc(q)*dxe(q)) on the agglomerated level
      auto pcf = [&](int d, bool a, int q) {
        const std::vector<double>& DC = ag_[l][d][2];
        const std::vector<double>& DE = ag_[l][d][3];
        return a ? 1.0 / (DC[q - 1] * DE[q - 2]) : 1.0 / (DC[q - 1] * DE[q - 1]);
      };
      for (int i = G.s[0]; i <= G.e[0]; ++i) {
        double a1 = fine ? fm_[0][5][i - 1] * fm_[0][4][i - 2] : pcf(0, true, i);
        double a2 = fine ? fm_[0][5][i - 1] * fm_[0][4][i - 1] : pcf(0, false, i);
        if (bd_[9] == 1 && i == G.s[0]) a1 = 0.0;
        if (bd_[18] == 1 && i == G.e[0]) a2 = 0.0;
        c.cx1[i - 1] = a1;
        c.cx2[i - 1] = a2;
      }
      for (int j = G.s[1]; j <= G.e[1]; ++j) {
        double a3 = fine ? fm_[1][5][j - 1] * fm_[1][4][j - 2] : pcf(1, true, j);
        double a4 = fine ? fm_[1][5][j - 1] * fm_[1][4][j - 1] : pcf(1, false, j);
        if (bd_[5] == 1 && j == G.s[1]) a3 = 0.0;
        if (bd_[1] == 1 && j == G.e[1]) a4 = 0.0;
        c.cy3[j - 1] = a3;
        c.cy4[j - 1] = a4;
      }
      for (int k = G.s[2]; k <= G.e[2]; ++k) {
        double a5 = fine ? fm_[2][5][k - 1] * fm_[2][4][k - 2] : pcf(2, true, k);
        double a6 = fine ? fm_[2][5][k - 1] * fm_[2][4][k - 1] : pcf(2, false, k);
        if (bd_[3] == 1 && k == G.s[2]) a5 = 0.0;
        if (bd_[7] == 1 && k == G.e[2]) a6 = 0.0;
        const int km = 2 * kstep * k - 3 * (kstep - 1);
        const int fk = fine ? k : km / 2;
        const double rp = R(fk), rb = R(fk - 1), rt = R(fk + 1);
        const double w5 = 0.5 * (rp + rb), w6 = 0.5 * (rp + rt);
        c.cz5[k - 1] = a5 * w5 / rb;
        c.cz6[k - 1] = a6 * w6 / rt;
        c.dz5[k - 1] = a5 * w5 / rp;
        c.dz6[k - 1] = a6 * w6 / rp;
      }
    }
  }
  coef_ready_ = true;
  return ANEL_OK;
}

// ZLINE: the line system of column (i,j) is (a, b, c) = (c5, c7, c6)
// with c7 = -(c1+c2+c3+c4+d5+d6).  With x/y-uniform coefficients every
// column has the same system, so the Thomas elimination (mg_relax.F90:
// 563-566) is done once per level here; the kernel runs the substitution.
// LJ (mg_relaxLz, mg_relax.F90:423-538) solves its lines with the 1-D
// coefficients pcf_1..6 of mg_coeff.F90:77-145 (not the level operator):
// x: pcf_1, pcf_2; y: pcf_3, pcf_4; z: sub pcf_5, super pcf_6 and diagonal
// -(pcf_1+pcf_2+pcf_3+pcf_4+pcf_5+pcf_6).  Kept in the level-coefficient
// layout (dz5 = cz5 = pcf_5, dz6 = cz6 = pcf_6) so the z-line kernel reads
// them in place of the operator; the finest level's Neumann faces are
// zeroed as mg_coeff.F90:123-145 does.
void MGSolver::build_lj_coefficients() {
  for (int l = 1; l <= ngrid_; ++l) {
    const LevelGeom& G = geo_[l];
    LevelCoef& c = ljc_[l];
    const int dims[3] = {G.X, G.Y, G.Z};
    std::vector<double>* A[3] = {&c.cx1, &c.cy3, &c.cz5};
    std::vector<double>* B[3] = {&c.cx2, &c.cy4, &c.cz6};
    for (int d = 0; d < 3; ++d) {
      A[d]->assign(dims[d], 0.0);
      B[d]->assign(dims[d], 0.0);
      const int s0 = G.kpx[d];
      for (int q = 2; q <= G.nk[d]; ++q) {
        (*A[d])[q - 1] = pA_[d][s0 + q - 1];
        (*B[d])[q - 1] = pB_[d][s0 + q - 1];
      }
    }
    if (l == ngrid_) {
      const int* t = prm_.tbc;
      if (t[4] == 1) c.cx1[1] = 0.0;
      if (t[5] == 1) c.cx2[G.nk[0] - 1] = 0.0;
      if (t[2] == 1) c.cy3[1] = 0.0;
      if (t[0] == 1) c.cy4[G.nk[1] - 1] = 0.0;
      if (t[1] == 1) c.cz5[1] = 0.0;
      if (t[3] == 1) c.cz6[G.nk[2] - 1] = 0.0;
    }
    c.dz5 = c.cz5;
    c.dz6 = c.cz6;
  }
}

// The coarsest level the column cycle solves directly: the finest level
// below the fine one whose columns fit the direct solver, with x and y
// periodic.  ANEL_DIRECT_COARSE=0 in the environment keeps the relaxation
// down to level 1 (the reference's schedule).
void MGSolver::choose_direct_level() {
  dirL_ = 0;
  if (!col_) return;
  const char* env = std::getenv("ANEL_DIRECT_COARSE");
  if (env && std::strcmp(env, "0") == 0) return;
  const int* t = prm_.tbc;
  if (!(t[4] == 0 && t[5] == 0 && t[0] == 0 && t[2] == 0)) return;
  for (int l = ngrid_ - 1; l >= 1; --l) {
    const int nx = geo_[l].n[0], ny = geo_[l].n[1];
    if (nx <= kDirMaxN && ny <= kDirMaxN && nx * ny <= kDirMaxModes) {
      dirL_ = l;
      return;
    }
  }
}

int MGSolver::build_direct(int l, DirectHost& D) {
  const LevelGeom& G = geo_[l];
  const LevelCoef& c = coef_[l];
  return direct_build(D, G.n[0], G.n[1], G.n[2], c.cx1[G.s[0] - 1], c.cx2[G.s[0] - 1], c.cy3[G.s[1] - 1],
                      c.cy4[G.s[1] - 1], c.cz5.data(), c.cz6.data(), c.dz5.data(), c.dz6.data(),
                      zcode_[l][0], zcode_[l][1]);
}

int MGSolver::build_zline_factors() {
  const bool lj = prm_.smoother == ANEL_SMOOTHER_LJ;
  if (dirL_ > 0) {
    // coefficients changed (density): rebuild the direct solve; a level
    // that does not qualify keeps the relaxation
    const int st = build_direct(dirL_, dir_);
    if (st == ANEL_ERR_UNSUPPORTED) {
      direct_free(dir_);
      dirL_ = 0;
    } else if (st != ANEL_OK) {
      return st;
    }
  }
  direct_free(dirfine_);
  for (int l = 1; l <= ngrid_; ++l) {
    const LevelGeom& G = geo_[l];
    const LevelCoef& c = lj ? ljc_[l] : coef_[l];
    for (int i = G.s[0]; i <= G.e[0]; ++i)
      if (!(c.cx1[i - 1] == c.cx1[G.s[0] - 1] && c.cx2[i - 1] == c.cx2[G.s[0] - 1])) {
        set_error("the z-line smoothers need x-uniform line coefficients (level %d)", l);
        return ANEL_ERR_UNSUPPORTED;
      }
    for (int j = G.s[1]; j <= G.e[1]; ++j)
      if (!(c.cy3[j - 1] == c.cy3[G.s[1] - 1] && c.cy4[j - 1] == c.cy4[G.s[1] - 1])) {
        set_error("the z-line smoothers need y-uniform line coefficients (level %d)", l);
        return ANEL_ERR_UNSUPPORTED;
      }
    const double a1 = c.cx1[G.s[0] - 1], a2 = c.cx2[G.s[0] - 1];
    const double a3 = c.cy3[G.s[1] - 1], a4 = c.cy4[G.s[1] - 1];
    const int n = G.n[2];
    std::vector<double> ap(G.Z, 0.0), bp(G.Z, 0.0);
    // rows r = 0..n-1 <-> k = r+2; stored at index k-1
    double bprev = 0.0;
    for (int r = 0; r < n; ++r) {
      const int k = r + 2;
      const double b = -(a1 + a2 + a3 + a4 + c.dz5[k - 1] + c.dz6[k - 1]);
      if (r == 0) {
        bp[k - 1] = b;
      } else {
        const double a = -c.cz5[k - 1] / bprev;
        ap[k - 1] = a;
        bp[k - 1] = b + a * c.cz6[k - 2];
      }
      bprev = bp[k - 1];
    }
    std::vector<double> both(ap);
    both.insert(both.end(), bp.begin(), bp.end());
    ANEL_CUDA_TRY(cudaMemcpy(d_zf64_[l], both.data(), both.size() * sizeof(double), cudaMemcpyHostToDevice));
    std::vector<float> b32(both.begin(), both.end());
    ANEL_CUDA_TRY(cudaMemcpy(d_zf32_[l], b32.data(), b32.size() * sizeof(float), cudaMemcpyHostToDevice));
    if (d_colfac_[l]) {
      std::vector<double> sub(n), dia(n), sup(n);
      for (int r = 0; r < n; ++r) {
        const int k = r + 2;
        sub[r] = c.cz5[k - 1];
        sup[r] = c.cz6[k - 1];
        dia[r] = -(a1 + a2 + a3 + a4 + c.dz5[k - 1] + c.dz6[k - 1]);
      }
      std::vector<float> cf;
      const int st = col_sweep_factors(n, colM_, sub, dia, sup, cf);
      if (st != ANEL_OK) return st;
      ANEL_CUDA_TRY(cudaMemcpy(d_colfac_[l], cf.data(), cf.size() * sizeof(float), cudaMemcpyHostToDevice));
    }
    if (d_zseg32_[l]) {
      std::vector<double> sub(n), dia(n), sup(n);
      for (int r = 0; r < n; ++r) {
        const int k = r + 2;
        sub[r] = c.cz5[k - 1];
        sup[r] = c.cz6[k - 1];
        dia[r] = -(a1 + a2 + a3 + a4 + c.dz5[k - 1] + c.dz6[k - 1]);
      }
      std::vector<double> seg;
      const int st = zline_segment_factors(n, kZSeg, sub, dia, sup, seg);
      if (st != ANEL_OK) return st;
      // rows r <-> index r+1 (the layout of the Thomas factors above)
      std::vector<float> f32(4 * (size_t)G.Z + 4 * kZSeg * kZSeg, 0.0f);
      for (int a = 0; a < 4; ++a)
        for (int r = 0; r < n; ++r) {
          const double f = seg[(size_t)a * n + r];
          f32[(size_t)a * G.Z + r + 1] = (float)(a == 1 ? 1.0 / f : f);  // bp -> 1/bp
        }
      for (int q = 0; q < 4 * kZSeg * kZSeg; ++q) f32[4 * (size_t)G.Z + q] = (float)seg[4 * (size_t)n + q];
      ANEL_CUDA_TRY(cudaMemcpy(d_zseg32_[l], f32.data(), f32.size() * sizeof(float),
                               cudaMemcpyHostToDevice));
      if (d_zcr32_[l]) {
        std::vector<double> cr;
        const int st2 = zline_cr_factors(n, zcr_steps_[l], sub, dia, sup, cr);
        if (st2 != ANEL_OK) return st2;
        std::vector<float> c32(cr.begin(), cr.end());
        ANEL_CUDA_TRY(cudaMemcpy(d_zcr32_[l], c32.data(), c32.size() * sizeof(float),
                                 cudaMemcpyHostToDevice));
      }
    }
  }
  return ANEL_OK;
}

// Factors of the partitioned line solver: the n rows of the tridiagonal
// system (sub, dia, sup) are cut into P segments of m = n/P rows.  Output,
// each array of n values followed by the (2P)^2 interface inverse:
//   ap, bp  Thomas factors of every segment taken alone (first row of a
//           segment: bp = dia, ap unused);
//   u, v    the segment's solution for a unit value in the row before it
//           (u, coupling -sub[lo]) and in the row after it (v, -sup[hi-1]);
//   minv    inverse of I - K, K coupling the interface unknowns
//           (F_0, L_0, F_1, L_1, ...) = first/last row of each segment.
// Multipliers of parallel cyclic reduction for the tridiagonal system
// (sub, dia, sup) of n rows (sub[0] and sup[n-1] unused): for steps
// q = 0..S-1 (stride 2^q) alpha_q[r] = -a_r / b_(r-2^q) and gamma_q[r] =
// -c_r / b_(r+2^q) of the current reduced system (0 past either end), then
// the reciprocal of the final diagonal.  out = alpha_0, gamma_0, ...,
// alpha_(S-1), gamma_(S-1), 1/b, n values each.
int zline_cr_factors(int n, int S, const std::vector<double>& sub, const std::vector<double>& dia,
                     const std::vector<double>& sup, std::vector<double>& out) {
  out.assign((2 * (size_t)S + 1) * n, 0.0);
  std::vector<double> a(sub), b(dia), c(sup), na(n), nb(n), nc(n);
  a[0] = 0.0;
  c[n - 1] = 0.0;
  for (int q = 0; q < S; ++q) {
    const int st = 1 << q;
    double* al = out.data() + (size_t)(2 * q) * n;
    double* ga = al + n;
    for (int r = 0; r < n; ++r) {
      const bool lo = r - st >= 0, hi = r + st < n;
      al[r] = lo ? -a[r] / b[r - st] : 0.0;
      ga[r] = hi ? -c[r] / b[r + st] : 0.0;
      nb[r] = b[r] + (lo ? al[r] * c[r - st] : 0.0) + (hi ? ga[r] * a[r + st] : 0.0);
      na[r] = lo ? al[r] * a[r - st] : 0.0;
      nc[r] = hi ? ga[r] * c[r + st] : 0.0;
    }
    a.swap(na);
    b.swap(nb);
    c.swap(nc);
  }
  double* rb = out.data() + (size_t)(2 * S) * n;
  for (int r = 0; r < n; ++r) {
    if (!(std::isfinite(b[r]) && b[r] != 0.0)) {
      set_error("z-line cyclic reduction is singular at row %d", r);
      return ANEL_ERR_NONFINITE;
    }
    rb[r] = 1.0 / b[r];
  }
  for (double v : out)
    if (!std::isfinite(v)) {
      set_error("z-line cyclic reduction multipliers are not finite");
      return ANEL_ERR_NONFINITE;
    }
  return ANEL_OK;
}

// Factors of the column sweep (k_col_sweep) for a line of n = 32*M rows
// (sub, dia, sup; sub[0] and sup[n-1] belong to the z ghosts and are not
// part of the system): lane s owns rows s*M .. s*M+M-1, the last of them a
// separator.  Per lane and inner row w (rows s*M+w, w < M-1): the Thomas
// factors ap, 1/bp and sup of the inner rows taken alone, and the spikes L
// (their solution for a unit value in the previous separator, coupling
// -sub of the first inner row; 0 on lane 0) and R (for a unit value in the
// own separator, coupling -sup of the last inner row).  Eliminating the
// inner rows leaves, in the separators X_s,
//   sub[h] L_s(last) X_(s-1) + (dia[h] + sub[h] R_s(last) + sup[h] L_(s+1)(first)) X_s
//     + sup[h] R_(s+1)(first) X_(s+1) = rhs[h] - sub[h] y_s(last) - sup[h] y_(s+1)(first)
// (h the separator row, y the inner rows' local solution), whose cyclic
// reduction multipliers come from zline_cr_factors.  Layout: see
// col_fac_floats.
int col_sweep_factors(int n, int M, const std::vector<double>& sub, const std::vector<double>& dia,
                      const std::vector<double>& sup, std::vector<float>& out) {
  std::vector<double> d;
  const int st = col_sweep_factors_d(n, M, sub, dia, sup, d);
  if (st != ANEL_OK) return st;
  out.assign(d.begin(), d.end());
  for (float v : out)
    if (!std::isfinite(v)) {
      set_error("column sweep factors are not finite in FP32");
      return ANEL_ERR_NONFINITE;
    }
  return ANEL_OK;
}

// the same factors in FP64 (the coarse direct solve uses them per mode)
int col_sweep_factors_d(int n, int M, const std::vector<double>& sub, const std::vector<double>& dia,
                        const std::vector<double>& sup, std::vector<double>& out) {
  constexpr int P = 32;
  if (M < 2 || n != P * M) {
    set_error("column sweep needs nz = 32*M rows with M >= 2 (nz = %d)", n);
    return ANEL_ERR_UNSUPPORTED;
  }
  const int I = M - 1;  // inner rows per lane
  std::vector<double> ap((size_t)I * P, 0.0), rbp((size_t)I * P, 0.0), sp((size_t)I * P, 0.0),
      Ls((size_t)I * P, 0.0), Rs((size_t)I * P, 0.0);
  auto at = [&](std::vector<double>& a, int w, int s) -> double& { return a[(size_t)w * P + s]; };
  std::vector<double> bp(I), w1(I), w2(I);
  for (int s = 0; s < P; ++s) {
    const int lo = s * M;
    bp[0] = dia[lo];
    for (int w = 1; w < I; ++w) {
      at(ap, w, s) = -sub[lo + w] / bp[w - 1];
      bp[w] = dia[lo + w] + at(ap, w, s) * sup[lo + w - 1];
    }
    for (int w = 0; w < I; ++w) {
      if (!(std::isfinite(bp[w]) && bp[w] != 0.0)) {
        set_error("column sweep: inner rows of lane %d are singular", s);
        return ANEL_ERR_NONFINITE;
      }
      at(rbp, w, s) = 1.0 / bp[w];
      at(sp, w, s) = sup[lo + w];
    }
    // solve T x = e on the inner rows
    auto solve = [&](std::vector<double>& e) {
      double g = e[0];
      e[0] = g;
      for (int w = 1; w < I; ++w) {
        g = e[w] + at(ap, w, s) * g;
        e[w] = g;
      }
      double x = g / bp[I - 1];
      e[I - 1] = x;
      for (int w = I - 2; w >= 0; --w) {
        x = (e[w] - sup[lo + w] * x) / bp[w];
        e[w] = x;
      }
    };
    std::fill(w1.begin(), w1.end(), 0.0);
    if (s > 0) {
      w1[0] = -sub[lo];
      solve(w1);
    }
    std::fill(w2.begin(), w2.end(), 0.0);
    w2[I - 1] = -sup[lo + I - 1];
    solve(w2);
    for (int w = 0; w < I; ++w) {
      at(Ls, w, s) = w1[w];
      at(Rs, w, s) = w2[w];
    }
  }
  std::vector<double> A(P, 0.0), B(P, 0.0), C(P, 0.0), subh(P, 0.0), suph(P, 0.0);
  for (int s = 0; s < P; ++s) {
    const int h = s * M + I;
    subh[s] = sub[h];
    suph[s] = s < P - 1 ? sup[h] : 0.0;
    A[s] = s > 0 ? sub[h] * at(Ls, I - 1, s) : 0.0;
    B[s] = dia[h] + sub[h] * at(Rs, I - 1, s) + (s < P - 1 ? sup[h] * at(Ls, 0, s + 1) : 0.0);
    C[s] = s < P - 1 ? sup[h] * at(Rs, 0, s + 1) : 0.0;
  }
  std::vector<double> cr;
  const int st = zline_cr_factors(P, 5, A, B, C, cr);
  if (st != ANEL_OK) return st;
  out.assign((size_t)col_fac_floats(M), 0.0);
  size_t o = 0;
  for (const std::vector<double>* a : {&ap, &rbp, &sp, &Ls, &Rs})
    for (double v : *a) out[o++] = v;
  for (int s = 0; s < P; ++s) out[o + s] = subh[s];
  for (int s = 0; s < P; ++s) out[o + P + s] = suph[s];
  for (int q = 0; q < 5; ++q)
    for (int s = 0; s < P; ++s) {
      out[o + (2 + q) * P + s] = cr[(size_t)(2 * q) * P + s];
      out[o + (7 + q) * P + s] = cr[(size_t)(2 * q + 1) * P + s];
    }
  for (int s = 0; s < P; ++s) out[o + 12 * P + s] = cr[(size_t)10 * P + s];
  for (double v : out)
    if (!std::isfinite(v)) {
      set_error("column sweep factors are not finite");
      return ANEL_ERR_NONFINITE;
    }
  return ANEL_OK;
}

int zline_segment_factors(int n, int P, const std::vector<double>& sub, const std::vector<double>& dia,
                          const std::vector<double>& sup, std::vector<double>& out) {
  const int m = n / P;
  const int P2 = 2 * P;
  out.assign(4 * (size_t)n + (size_t)P2 * P2, 0.0);
  double* ap = out.data();
  double* bp = ap + n;
  double* u = bp + n;
  double* v = u + n;
  double* minv = v + n;
  auto solve_seg = [&](int lo, int hi, std::vector<double>& rhs) {
    double g = rhs[lo];
    std::vector<double> gs(hi - lo);
    gs[0] = g;
    for (int q = lo + 1; q < hi; ++q) {
      g = rhs[q] + ap[q] * g;
      gs[q - lo] = g;
    }
    double x = g / bp[hi - 1];
    rhs[hi - 1] = x;
    for (int q = hi - 2; q >= lo; --q) {
      x = (gs[q - lo] - sup[q] * x) / bp[q];
      rhs[q] = x;
    }
  };
  std::vector<double> M((size_t)P2 * P2, 0.0);
  for (int s = 0; s < P; ++s) {
    const int lo = s * m, hi = lo + m;
    bp[lo] = dia[lo];
    for (int q = lo + 1; q < hi; ++q) {
      ap[q] = -sub[q] / bp[q - 1];
      bp[q] = dia[q] + ap[q] * sup[q - 1];
    }
    for (int q = lo; q < hi; ++q)
      if (!(std::isfinite(bp[q]) && bp[q] != 0.0)) {
        set_error("z-line segment %d is singular at row %d", s, q);
        return ANEL_ERR_NONFINITE;
      }
    std::vector<double> w(n, 0.0);
    if (s > 0) {
      w[lo] = -sub[lo];
      solve_seg(lo, hi, w);
      for (int q = lo; q < hi; ++q) u[q] = w[q];
    }
    if (s < P - 1) {
      std::fill(w.begin(), w.end(), 0.0);
      w[hi - 1] = -sup[hi - 1];
      solve_seg(lo, hi, w);
      for (int q = lo; q < hi; ++q) v[q] = w[q];
    }
    M[(size_t)(2 * s) * P2 + 2 * s] = 1.0;
    M[(size_t)(2 * s + 1) * P2 + 2 * s + 1] = 1.0;
    if (s > 0) {
      M[(size_t)(2 * s) * P2 + 2 * s - 1] -= u[lo];
      M[(size_t)(2 * s + 1) * P2 + 2 * s - 1] -= u[hi - 1];
    }
    if (s < P - 1) {
      M[(size_t)(2 * s) * P2 + 2 * s + 2] -= v[lo];
      M[(size_t)(2 * s + 1) * P2 + 2 * s + 2] -= v[hi - 1];
    }
  }
  // Gauss-Jordan with partial pivoting
  for (int r = 0; r < P2; ++r) minv[(size_t)r * P2 + r] = 1.0;
  for (int c = 0; c < P2; ++c) {
    int piv = c;
    for (int r = c + 1; r < P2; ++r)
      if (std::fabs(M[(size_t)r * P2 + c]) > std::fabs(M[(size_t)piv * P2 + c])) piv = r;
    if (!(std::fabs(M[(size_t)piv * P2 + c]) > 0.0)) {
      set_error("z-line interface system is singular");
      return ANEL_ERR_NONFINITE;
    }
    if (piv != c)
      for (int q = 0; q < P2; ++q) {
        std::swap(M[(size_t)c * P2 + q], M[(size_t)piv * P2 + q]);
        std::swap(minv[(size_t)c * P2 + q], minv[(size_t)piv * P2 + q]);
      }
    const double d = M[(size_t)c * P2 + c];
    for (int q = 0; q < P2; ++q) {
      M[(size_t)c * P2 + q] /= d;
      minv[(size_t)c * P2 + q] /= d;
    }
    for (int r = 0; r < P2; ++r) {
      if (r == c) continue;
      const double f = M[(size_t)r * P2 + c];
      if (f == 0.0) continue;
      for (int q = 0; q < P2; ++q) {
        M[(size_t)r * P2 + q] -= f * M[(size_t)c * P2 + q];
        minv[(size_t)r * P2 + q] -= f * minv[(size_t)c * P2 + q];
      }
    }
  }
  return ANEL_OK;
}

int MGSolver::upload_coefficients() {
  ANEL_CUDA_TRY(cudaSetDevice(device_));
  if (prm_.smoother == ANEL_SMOOTHER_ZLINE || prm_.smoother == ANEL_SMOOTHER_LJ) {
    const int st = build_zline_factors();
    if (st != ANEL_OK) return st;
  }
  if (prm_.smoother == ANEL_SMOOTHER_LJ)
    for (int l = 1; l <= ngrid_; ++l) {
      const LevelCoef& c = ljc_[l];
      std::vector<double> packed;
      for (const std::vector<double>* v :
           {&c.cx1, &c.cx2, &c.cy3, &c.cy4, &c.cz5, &c.cz6, &c.dz5, &c.dz6})
        packed.insert(packed.end(), v->begin(), v->end());
      ANEL_CUDA_TRY(cudaMemcpy(d_ljc64_[l], packed.data(), packed.size() * sizeof(double),
                               cudaMemcpyHostToDevice));
      if (d_ljc32_[l]) {
        std::vector<float> p32(packed.begin(), packed.end());
        ANEL_CUDA_TRY(cudaMemcpy(d_ljc32_[l], p32.data(), p32.size() * sizeof(float),
                                 cudaMemcpyHostToDevice));
      }
    }
  uint64_t h = 1469598103934665603ull;  // FNV-1a over every level's coefficients
  for (int l = 1; l <= ngrid_; ++l) {
    const LevelCoef& c = coef_[l];
    std::vector<double> packed;
    for (const std::vector<double>* v :
         {&c.cx1, &c.cx2, &c.cy3, &c.cy4, &c.cz5, &c.cz6, &c.dz5, &c.dz6})
      packed.insert(packed.end(), v->begin(), v->end());
    const unsigned char* pb = reinterpret_cast<const unsigned char*>(packed.data());
    for (size_t q = 0; q < packed.size() * sizeof(double); ++q) {
      h ^= pb[q];
      h *= 1099511628211ull;
    }
    ANEL_CUDA_TRY(cudaMemcpy(d_coef64_[l], packed.data(), packed.size() * sizeof(double),
                             cudaMemcpyHostToDevice));
    if (d_coef32_[l]) {
      std::vector<float> p32(packed.begin(), packed.end());
      ANEL_CUDA_TRY(cudaMemcpy(d_coef32_[l], p32.data(), p32.size() * sizeof(float),
                               cudaMemcpyHostToDevice));
    }
  }
  op_hash_ = h;
  return ANEL_OK;
}

int MGSolver::set_density_host(const double* r) {
  if (!r) {
    set_error("null density");
    return ANEL_ERR_ARG;
  }
  const LevelGeom& F = geo_[ngrid_];
  const int64_t XY = (int64_t)F.X * F.Y;
  std::vector<double> rz(F.Z);
  for (int k = 0; k < F.Z; ++k) {
    const double* plane = r + (int64_t)k * XY;
    const double v = plane[0];
    for (int64_t q = 1; q < XY; ++q)
      if (!(plane[q] == v)) {
        set_error(
            "density must be horizontally uniform r = r(z); plane k=%d differs at offset %lld",
            k + 1, (long long)q);
        return ANEL_ERR_UNSUPPORTED;
      }
    if (!std::isfinite(v) || v == 0.0) {
      set_error("density plane k=%d is zero or not finite", k + 1);
      return ANEL_ERR_NONFINITE;
    }
    rz[k] = v;
  }
  int st = build_coefficients(rz);
  if (st != ANEL_OK) return st;
  return upload_coefficients();
}

int MGSolver::set_density_device(const double* r, cudaStream_t s) {
  const LevelGeom& F = geo_[ngrid_];
  std::vector<double> h(F.G);
  ANEL_CUDA_TRY(cudaMemcpyAsync(h.data(), r, F.G * sizeof(double), cudaMemcpyDeviceToHost,
                                s ? s : stream_));
  ANEL_CUDA_TRY(cudaStreamSynchronize(s ? s : stream_));
  return set_density_host(h.data());
}

// ------------------------------------------------------------ views
DevLevel<double> MGSolver::L64(int l) const {
  const LevelGeom& G = geo_[l];
  DevLevel<double> L;
  L.nx = G.n[0];
  L.ny = G.n[1];
  L.nz = G.n[2];
  L.X = G.X;
  L.Y = G.Y;
  L.Z = G.Z;
  L.XY = (int64_t)G.X * G.Y;
  L.G = G.G;
  L.phi = d_phi64_[l];
  L.src = d_src64_[l];
  L.coef = d_coef64_[l];
  L.rule = rule_[l];
  L.gtab = nullptr;
  return L;
}

DevLevel<float> MGSolver::L32(int l, bool hom) const {
  const LevelGeom& G = geo_[l];
  DevLevel<float> L;
  L.nx = G.n[0];
  L.ny = G.n[1];
  L.nz = G.n[2];
  L.X = G.X;
  L.Y = G.Y;
  L.Z = G.Z;
  L.XY = (int64_t)G.X * G.Y;
  L.G = G.G;
  L.phi = d_phi32_[l];
  L.src = d_src32_[l];
  L.coef = d_coef32_[l];
  L.rule = hom ? rule_hom_[l] : rule_[l];
  L.gtab = hom ? d_gtab32_[l] : nullptr;
  return L;
}

ColLevel MGSolver::C32(int l) const {
  const LevelGeom& G = geo_[l];
  const LevelCoef& c = coef_[l];
  ColLevel L;
  L.nx = G.n[0];
  L.ny = G.n[1];
  L.nz = G.n[2];
  L.X = G.X;
  L.Y = G.Y;
  L.CS = col_stride(G.n[2]);
  L.phi = d_phi32_[l];
  L.src = d_src32_[l];
  // x/y-uniform line coefficients (checked by build_zline_factors)
  L.a1 = (float)c.cx1[G.s[0] - 1];
  L.a2 = (float)c.cx2[G.s[0] - 1];
  L.a3 = (float)c.cy3[G.s[1] - 1];
  L.a4 = (float)c.cy4[G.s[1] - 1];
  const float* z = d_coef32_[l] + 2 * (size_t)G.X + 2 * (size_t)G.Y;
  L.cz5 = z;
  L.cz6 = z + G.Z;
  L.dz5 = z + 2 * G.Z;
  L.dz6 = z + 3 * G.Z;
  L.img = d_img32_[l];
  L.z1 = zcode_[l][0];
  L.zZ = zcode_[l][1];
  return L;
}

int64_t MGSolver::fp32_elems(int l) const {
  return col_ ? (int64_t)geo_[l].X * geo_[l].Y * col_stride(geo_[l].n[2]) : geo_[l].G;
}

DevLevel<double> MGSolver::fine_view(double* phi, const double* src) const {
  DevLevel<double> L = L64(ngrid_);
  L.phi = phi;
  L.src = const_cast<double*>(src);
  return L;
}

int MGSolver::coarsen_dirs(int lC) const {
  int m = 0;
  for (int d = 0; d < 3; ++d)
    if (geo_[lC].nk[d] < geo_[lC + 1].nk[d]) m |= 1 << d;
  return m;
}

// ----------------------------------------------------------- V-cycle
// mg_relaxRB: per iteration colour 0, boundary pass, colour 1, boundary
// pass (mg_relax.F90:146-172); the extra final boundary pass of :176 is a
// no-op after an iteration and is kept only when iters == 0.
void MGSolver::relax64(int l, int iters, cudaStream_t s) {
  const DevLevel<double> L = L64(l);
  const bool prof = prof_ && l == ngrid_;
  const bool zl = prm_.smoother == ANEL_SMOOTHER_ZLINE;
  const bool lj = prm_.smoother == ANEL_SMOOTHER_LJ;
  const double* zf = d_zf64_[l];
  DevLevel<double> Lj = L;  // LJ lines use the pcf coefficients
  if (lj) Lj.coef = d_ljc64_[l];
  for (int it = 0; it < iters; ++it) {
    for (int color = 0; color < 2; ++color) {
      if (prof) prof_begin(s);
      if (zl) launch_zline(L, color, zf, zf + geo_[l].Z, s);
      else if (lj) launch_zline_lj(Lj, color, zf, zf + geo_[l].Z, s);
      else launch_rb_sweep(L, color, s);
      if (prof) prof_end(s);
      launch_bdry(L, L.phi, s);
    }
  }
  if (iters == 0) launch_bdry(L, L.phi, s);
}

// mg_cycle.F90:186-325
void MGSolver::cycle64(cudaStream_t s) {
  const int ng = ngrid_;
  const int* pre = prm_.pre_relax;
  const int* post = prm_.post_relax;
  relax64(ng, pre[ng - 1], s);
  launch_restrict(L64(ng), L64(ng - 1), coarsen_dirs(ng - 1), s);
  for (int l = ng - 1; l >= 2; --l) {
    relax64(l, pre[l - 1], s);
    launch_restrict(L64(l), L64(l - 1), coarsen_dirs(l - 1), s);
  }
  relax64(1, pre[0], s);
  for (int l = 1; l <= ng - 1; ++l) {
    relax64(l, post[l - 1], s);
    const DevLevel<double> F = L64(l + 1);
    launch_prolong(F, L64(l), coarsen_dirs(l), s);
    launch_bdry(F, F.phi, s);
  }
  relax64(ng, post[ng - 1], s);
}

void MGSolver::relax32(int l, int iters, cudaStream_t s) {
  const DevLevel<float> L = L32(l, true);
  const bool prof = prof_ && l == ngrid_;
  const bool zl = prm_.smoother == ANEL_SMOOTHER_ZLINE;
  const bool lj = prm_.smoother == ANEL_SMOOTHER_LJ;
  const float* zf = d_zf32_[l];
  const float* zs = d_zseg32_[l];
  const SegFac<float> sf = segfac32(l);
  DevLevel<float> Lj = L;
  if (lj) Lj.coef = d_ljc32_[l];
  for (int it = 0; it < iters; ++it) {
    for (int color = 0; color < 2; ++color) {
      if (prof) prof_begin(s);
      if (zl && zs) launch_zline_seg(L, color, sf, s);
      else if (zl) launch_zline(L, color, zf, zf + geo_[l].Z, s);
      else if (lj) launch_zline_lj(Lj, color, zf, zf + geo_[l].Z, s);
      else launch_rb_sweep(L, color, s);
      if (prof) prof_end(s);
      if (!(zl && zs && sf.img)) launch_bdry(L, L.phi, s);
    }
  }
  if (iters == 0) launch_bdry(L, L.phi, s);
}

void MGSolver::cycle32(cudaStream_t s) {
  const int ng = ngrid_;
  const int* pre = prm_.pre_relax;
  const int* post = prm_.post_relax;
  relax32(ng, pre[ng - 1], s);
  launch_restrict(L32(ng, true), L32(ng - 1, true), coarsen_dirs(ng - 1), s);
  for (int l = ng - 1; l >= 2; --l) {
    relax32(l, pre[l - 1], s);
    launch_restrict(L32(l, true), L32(l - 1, true), coarsen_dirs(l - 1), s);
  }
  relax32(1, pre[0], s);
  for (int l = 1; l <= ng - 1; ++l) {
    relax32(l, post[l - 1], s);
    const DevLevel<float> F = L32(l + 1, true);
    launch_prolong(F, L32(l, true), coarsen_dirs(l), s);
    launch_bdry(F, F.phi, s);
  }
  relax32(ng, post[ng - 1], s);
}

// The FP32 cycle on the column layout: cycle32's schedule, the boundary
// pass after each prolongation folded into the prolongation, the coarse
// correction zeroed before each restriction.
void MGSolver::relax_col(int l, int iters, cudaStream_t s, int nb) {
  const ColLevel L = nb > 0 ? C32b(l, nb) : C32(l);
  const bool prof = prof_ && l == ngrid_ && nb == 0;
  for (int it = 0; it < iters; ++it)
    for (int color = 0; color < 2; ++color) {
      if (prof) prof_begin(s);
      launch_col_sweep(L, color, d_colfac_[l], colM_, colvar_[l], d_err_, s);
      if (prof) prof_end(s);
    }
}

void MGSolver::cycle_col(cudaStream_t s, int nb) {
  const int ng = ngrid_;
  const int* pre = prm_.pre_relax;
  const int* post = prm_.post_relax;
  auto C = [&](int l) { return nb > 0 ? C32b(l, nb) : C32(l); };
  auto down = [&](int l) {
    float* ph = nb > 0 ? d_bphi32_[l - 1] : d_phi32_[l - 1];
    cudaMemsetAsync(ph, 0, fp32_elems(l - 1) * (nb > 0 ? nb : 1) * sizeof(float), s);
    launch_col_restrict(C(l), C(l - 1), coarsen_dirs(l - 1), s);
  };
  // with a direct level L0 the levels below it are never visited: L0 is
  // solved exactly in place of its relaxation and of the coarser cycle
  const int L0 = dirL_ > 0 ? dirL_ : 1;
  relax_col(ng, pre[ng - 1], s, nb);
  for (int l = ng; l > L0; --l) {
    if (l < ng) relax_col(l, pre[l - 1], s, nb);
    down(l);
  }
  if (dirL_ > 0) {
    launch_direct_col(dir_.f, C(L0), nb > 0 ? d_bdir_ : nullptr, s);
  } else {
    relax_col(1, pre[0], s, nb);
    relax_col(1, post[0], s, nb);
  }
  for (int l = L0; l < ng; ++l) {
    if (l > L0) relax_col(l, post[l - 1], s, nb);
    launch_col_prolong(C(l + 1), C(l), coarsen_dirs(l), s);
  }
  relax_col(ng, post[ng - 1], s, nb);
}

ColLevel MGSolver::C32b(int l, int nb) const {
  ColLevel L = C32(l);
  L.phi = d_bphi32_[l];
  L.src = d_bsrc32_[l];
  L.nm = nb;
  L.ms = fp32_elems(l);
  L.act = d_bact_;
  return L;
}

SegFac<float> MGSolver::segfac32(int l) const {
  const float* zs = d_zseg32_[l];
  SegFac<float> f{};
  if (!zs) return f;
  const int Z = geo_[l].Z;
  f.ap = zs;
  f.rbp = zs + Z;
  f.u = zs + 2 * Z;
  f.v = zs + 3 * Z;
  f.minv = zs + 4 * Z;
  f.img = d_img32_[l];
  f.z1 = zcode_[l][0];
  f.zZ = zcode_[l][1];
  f.cr = d_zcr32_[l];
  f.crs = zcr_steps_[l];
  return f;
}

// Derive from the level's ghost table which ghost cells copy which line, so
// the z-line sweep can write them itself: every ghost column must copy one
// interior line row by row (or be 0), every line may have at most three
// such image columns, and the k=1 / k=Z ghosts of all columns must follow
// one rule (0, row k=2 or row k=nz+1 of the column they image).  A level
// that does not fit keeps the boundary pass.
int MGSolver::build_self_ghosting(int l) {
  const LevelGeom& G = geo_[l];
  const int X = G.X, Y = G.Y, Z = G.Z, nx = G.n[0], ny = G.n[1], nz = G.n[2];
  const int64_t XY = (int64_t)X * Y;
  const int64_t ngh = G.G - (int64_t)nx * ny * nz;
  std::vector<int2> tab(ngh);
  ANEL_CUDA_TRY(cudaMemcpy(tab.data(), d_gtab32_[l], ngh * sizeof(int2), cudaMemcpyDeviceToHost));
  // source column (interior (i,j) as index, -1 zero) of every column of
  // the ghosted plane for the interior rows, and the z rule per column
  std::vector<int64_t> colsrc(XY, -2);
  int zc[2] = {-1, -1};
  bool ok = true;
  auto col_of = [&](int64_t c) { return c % XY; };
  for (int64_t g = 0; g < ngh && ok; ++g) {
    const int64_t d = tab[g].x, src = tab[g].y;
    const int64_t dcol = col_of(d);
    const int dk = 1 + (int)(d / XY);
    if (dk >= 2 && dk <= nz + 1) {
      int64_t sc = -1;
      if (src >= 0) {
        if (1 + src / XY != dk) ok = false;
        sc = col_of(src);
      }
      if (colsrc[dcol] == -2) colsrc[dcol] = sc;
      else if (colsrc[dcol] != sc) ok = false;
    }
  }
  for (int64_t c = 0; c < XY && ok; ++c) {
    const int i = 1 + (int)(c % X), j = 1 + (int)(c / X);
    const bool interior = i >= 2 && i <= nx + 1 && j >= 2 && j <= ny + 1;
    if (interior) colsrc[c] = c;
    else if (colsrc[c] == -2) ok = false;
  }
  // z ghosts
  for (int64_t g = 0; g < ngh && ok; ++g) {
    const int64_t d = tab[g].x, src = tab[g].y;
    const int dk = 1 + (int)(d / XY);
    if (dk != 1 && dk != Z) continue;
    const int64_t sc = colsrc[col_of(d)];
    int code;
    if (src < 0) {
      code = 0;
    } else {
      if (col_of(src) != sc) { ok = false; break; }
      const int sk = 1 + (int)(src / XY);
      code = (sk == 2) ? 1 : (sk == nz + 1 ? 2 : -1);
      if (code < 0) { ok = false; break; }
    }
    if (sc < 0 && code != 0) { ok = false; break; }
    if (sc < 0) continue;  // a zero column: its z ghosts are zero as well
    int& z = zc[dk == 1 ? 0 : 1];
    if (z == -1) z = code;
    else if (z != code) ok = false;
  }
  std::vector<int> img(3 * (size_t)nx * ny, kNoImage);
  for (int64_t c = 0; c < XY && ok; ++c) {
    const int64_t sc = colsrc[c];
    if (sc < 0 || sc == c) continue;
    const int si = 1 + (int)(sc % X), sj = 1 + (int)(sc / X);
    int* e = &img[3 * ((size_t)(si - 2) + (size_t)nx * (sj - 2))];
    int q = 0;
    while (q < 3 && e[q] != kNoImage) ++q;
    if (q == 3) { ok = false; break; }
    e[q] = (int)(c - sc);
  }
  if (!ok || zc[0] < 0 || zc[1] < 0) return ANEL_OK;  // keep the boundary pass
  ANEL_CUDA_TRY(cudaMalloc(&d_img32_[l], img.size() * sizeof(int)));
  ANEL_CUDA_TRY(cudaMemcpy(d_img32_[l], img.data(), img.size() * sizeof(int), cudaMemcpyHostToDevice));
  zcode_[l][0] = zc[0];
  zcode_[l][1] = zc[1];
  return ANEL_OK;
}


// ------------------------------------------------------------ solves
double MGSolver::true_resid(const double* d_phi, const double* d_rhs, cudaStream_t s,
                            double* fnorm) {
  const DevLevel<double> F = fine_view(const_cast<double*>(d_phi), d_rhs);
  launch_resid_norm(F, d_phi, d_rhs, d_part_, d_norm_, s);
  copy_words(d_norm_, h_pin_, 2, s);
  cudaStreamSynchronize(s);
  if (fnorm) *fnorm = std::sqrt(h_pin_[1]);
  return h_pin_[1] > 0.0 ? std::sqrt(h_pin_[0] / h_pin_[1]) : std::sqrt(h_pin_[0]);
}

int MGSolver::solve_device(double* d_phi, const double* d_rhs, cudaStream_t s,
                           anel_mg_report* rep) {
  if (!d_phi || !d_rhs) {
    set_error("null phi or rhs");
    return ANEL_ERR_ARG;
  }
  ANEL_CUDA_TRY(cudaSetDevice(device_));
  if (!s) s = stream_;
  anel_mg_report r{};
  const int64_t launches0 = t_launches;
  prof_n_ = 0;
  ANEL_CUDA_TRY(cudaEventRecord(ev0_, s));
  // the graph solve when it applies: column cycle, no per-sweep profiling,
  // no per-cycle printing, a capturable stream
  const bool graph_ok = col_ && !prof_ && !prm_.verbose && gsolve_state_ >= 0 && s != nullptr &&
                        s != cudaStreamLegacy && s != cudaStreamPerThread && !g32_off_ && graph_solve_enabled();
  const int st = prm_.precision != ANEL_PREC_MIXED ? solve_fp64(d_phi, d_rhs, s, &r)
                 : graph_ok                        ? solve_mixed_graph(d_phi, d_rhs, s, &r)
                                                   : solve_mixed(d_phi, d_rhs, s, &r);
  ANEL_CUDA_TRY(cudaEventRecord(ev1_, s));
  ANEL_CUDA_TRY(cudaEventSynchronize(ev1_));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ev0_, ev1_);
  r.ms = ms;
  if (st != ANEL_OK && st != ANEL_ERR_NOCONV) return st;
  const int le = check_launch("mg solve");
  if (le != ANEL_OK) return le;
  const int ke = take_kernel_error("mg solve");
  if (ke != ANEL_OK) return ke;
  r.launches = t_launches - launches0;
  const int pe = prof_collect(&r);
  if (pe != ANEL_OK) return pe;
  // the mixed solve's last defect is the true residual of the returned phi
  // (computed after the last correction and boundary pass); the FP64 solve
  // stopped on relmax needs its own pass
  if (prm_.precision != ANEL_PREC_MIXED) r.resid = true_resid(d_phi, d_rhs, s, nullptr);
  r.status = st;
  if (rep) *rep = r;
  return st;
}

int MGSolver::solve_fp64(double* d_phi, const double* d_rhs, cudaStream_t s,
                         anel_mg_report* rep) {
  const int ng = ngrid_;
  const DevLevel<double> Fu = fine_view(d_phi, d_rhs);
  const DevLevel<double> W = L64(ng);
  launch_bdry(Fu, d_phi, s);  // mg_solver.F90:101
  ANEL_CUDA_TRY(cudaMemcpyAsync(W.phi, d_phi, W.G * sizeof(double), cudaMemcpyDeviceToDevice, s));
  ANEL_CUDA_TRY(cudaMemcpyAsync(W.src, d_rhs, W.G * sizeof(double), cudaMemcpyDeviceToDevice, s));
  double relmax = 0.0, fn = 0.0;
  int iter = 0;
  bool conv = false;
  const bool by_resid = prm_.stop == ANEL_STOP_RESID;
  if (by_resid) {
    // ||f|| once; ||f - A phi|| is taken on the work array after each cycle
    true_resid(d_phi, d_rhs, s, &fn);
  }
  for (iter = 1; iter <= prm_.maxcy; ++iter) {
    cycle64(s);
    if (by_resid) {
      const double res = true_resid(W.phi, d_rhs, s, nullptr);
      relmax = res;
      if (prm_.verbose) std::fprintf(stderr, "       Iteration: %5d  RESID= %22.15e\n", iter, res);
      if (res <= prm_.tolmax) {
        conv = true;
        break;
      }
    } else {
      ANEL_CUDA_TRY(cudaMemsetAsync(d_max_, 0, 2 * sizeof(unsigned long long), s));
      launch_relmax_copy(W, W.phi, d_phi, d_max_, s);
      copy_words(d_max_, h_pin_, 2, s);
      ANEL_CUDA_TRY(cudaStreamSynchronize(s));
      const double v1 = h_pin_[0], v2 = h_pin_[1];  // bit patterns of the maxima
      relmax = v1 > 0.0 ? v2 / v1 : 0.0;
      if (prm_.verbose)
        std::fprintf(stderr, "       Iteration: %5d  RESIDUAL= %22.15e\n", iter, relmax);
      if (relmax <= prm_.tolmax) {
        conv = true;
        break;
      }
    }
  }
  if (by_resid)
    ANEL_CUDA_TRY(cudaMemcpyAsync(d_phi, W.phi, W.G * sizeof(double), cudaMemcpyDeviceToDevice, s));
  launch_bdry(Fu, d_phi, s);  // mg_solver.F90:139
  if (!conv) {
    if (prm_.verbose)
      std::fprintf(stderr, "WARNING: failed to achieve convergence in %6d cycles, RESIDUAL=%22.16f\n",
                   prm_.maxcy, relmax);
    iter = prm_.maxcy + 1;  // value of the Fortran DO variable after the loop
  }
  rep->iter = iter;
  rep->relmax = relmax;
  return conv ? ANEL_OK : ANEL_ERR_NOCONV;
}

// Mixed precision: FP64 defect correction around one FP32 V-cycle per
// iteration.  FP64: fine residual, correction update, norms, boundary
// pass of the solution.  FP32: smoothing, restriction, prolongation and
// every coarse level, on the error equation (homogeneous wall values).
// The FP32 cycle is ~100-200 small launches whose arguments never change
// for a solver, so from the second call on it is captured once (thread-
// local capture mode: other host threads driving other contexts are not
// affected) and replayed as one graph launch.  The same kernels run in the
// same order, so results are unchanged.  Profiling runs (events between
// sweeps) and the legacy default stream stay uncaptured.
void MGSolver::run_cycle32(cudaStream_t s) {
  float* const e = d_phi32_[ngrid_];
  const int64_t ne = fp32_elems(ngrid_);
  auto cycle = [&]() {
    cudaMemsetAsync(e, 0, ne * sizeof(float), s);
    if (col_) cycle_col(s);
    else cycle32(s);
  };
  const bool can = !prof_ && !g32_off_ && s != nullptr && s != cudaStreamLegacy &&
                   s != cudaStreamPerThread;
  if (!can || (++g32_calls_ < 2 && !g32x_)) {
    cycle();
    return;
  }
  if (!g32x_) {
    const int64_t l0 = t_launches;
    bool ok = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
      cycle();
      cudaGraph_t g = nullptr;
      ok = cudaStreamEndCapture(s, &g) == cudaSuccess && g;
      const int64_t n = t_launches - l0;  // counted while capturing, not run
      g_launches.fetch_sub(n, std::memory_order_relaxed);
      t_launches -= n;
      g32_launches_ = n;
      if (ok) ok = cudaGraphInstantiate(&g32x_, g, 0) == cudaSuccess;
      if (g) cudaGraphDestroy(g);
    }
    if (!ok) {
      cudaGetLastError();
      g32x_ = nullptr;
      g32_off_ = true;
      cycle();
      return;
    }
  }
  cudaGraphLaunch(g32x_, s);
  count_launch(g32_launches_);
}

// ------------------------------------------- device-side convergence loop
// ANEL_GRAPH_SOLVE=0 in the environment keeps the host-driven loop
static bool graph_solve_enabled() {
  const char* v = std::getenv("ANEL_GRAPH_SOLVE");
  return !(v && std::strcmp(v, "0") == 0);
}

struct ConvState {
  double rel;
  int iter;
  int conv;
};

__device__ __forceinline__ double conv_rel(const double* n) {
  return n[1] > 0.0 ? sqrt(n[0] / n[1]) : sqrt(n[0]);
}

// the first defect: stop before any cycle if it already meets the tolerance
__global__ void k_conv_init(const double* norm, ConvState* st, double tol, int maxcy,
                            cudaGraphConditionalHandle h) {
  const double rel = conv_rel(norm);
  const int c = rel <= tol;
  st->rel = rel;
  st->iter = 0;
  st->conv = c;
  cudaGraphSetConditional(h, (!c && maxcy > 0) ? 1u : 0u);
}

// after a cycle: the loop of solve_mixed (iteration count, stop at the
// tolerance or after maxcy cycles), decided on the device
__global__ void k_conv_step(const double* norm, ConvState* st, double tol, int maxcy,
                            cudaGraphConditionalHandle h) {
  const double rel = conv_rel(norm);
  const int it = st->iter + 1;
  const int c = rel <= tol;
  st->rel = rel;
  st->iter = it;
  st->conv = c;
  cudaGraphSetConditional(h, (!c && it < maxcy) ? 1u : 0u);
}

int MGSolver::build_solve_graph(double* d_phi, const double* d_rhs, cudaStream_t s) {
  if (gsolve_) {
    cudaGraphExecDestroy(gsolve_);
    gsolve_ = nullptr;
  }
  if (!side_) ANEL_CUDA_TRY(cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking));
  if (!d_conv_) ANEL_CUDA_TRY(cudaMalloc(&d_conv_, sizeof(ConvState)));
  const int ng = ngrid_;
  const DevLevel<double> Fu = fine_view(d_phi, d_rhs);
  const ColLevel Ec = C32(ng);
  ConvState* cs = static_cast<ConvState*>(d_conv_);
  const double tol = prm_.tolmax;
  const int maxcy = prm_.maxcy;
  cudaGraph_t g = nullptr;
  bool ok = cudaGraphCreate(&g, 0) == cudaSuccess;
  cudaGraphConditionalHandle h{};
  if (ok) ok = cudaGraphConditionalHandleCreate(&h, g, 0, 0) == cudaSuccess;
  // head: boundary pass, first defect, the loop's entry test
  const int64_t l0 = t_launches;
  if (ok) ok = cudaStreamBeginCaptureToGraph(s, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) ==
               cudaSuccess;
  cudaGraphNode_t cnode = nullptr;
  cudaGraph_t body = nullptr;
  if (ok) {
    launch_bdry(Fu, d_phi, s);
    launch_col_resid_store(Fu, d_phi, d_rhs, Ec, d_part_, d_norm_, s);
    k_conv_init<<<1, 1, 0, s>>>(d_norm_, cs, tol, maxcy, h);
    count_launch();
    cudaStreamCaptureStatus cst;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    ok = cudaStreamGetCaptureInfo(s, &cst, nullptr, nullptr, &deps, &ndeps) == cudaSuccess &&
         cst == cudaStreamCaptureStatusActive;
    if (ok) {
      cudaGraphNodeParams cp{};
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = h;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      ok = cudaGraphAddNode(&cnode, g, deps, ndeps, &cp) == cudaSuccess;
      if (ok) body = cp.conditional.phGraph_out[0];
      if (ok) ok = cudaStreamUpdateCaptureDependencies(s, &cnode, 1, cudaStreamSetCaptureDependencies) ==
                   cudaSuccess;
    }
    cudaGraph_t gout = nullptr;
    const bool ended = cudaStreamEndCapture(s, &gout) == cudaSuccess;
    ok = ok && ended;
  }
  gsolve_head_launches_ = t_launches - l0;
  // body: one FP32 cycle, the correction, the next defect and its test
  const int64_t l1 = t_launches;
  if (ok) ok = cudaStreamBeginCaptureToGraph(side_, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) ==
               cudaSuccess;
  if (ok) {
    cudaMemsetAsync(d_phi32_[ng], 0, fp32_elems(ng) * sizeof(float), side_);
    cycle_col(side_);
    launch_col_add_correction(Fu, d_phi, Ec, side_);
    launch_bdry(Fu, d_phi, side_);
    launch_col_resid_store(Fu, d_phi, d_rhs, Ec, d_part_, d_norm_, side_);
    k_conv_step<<<1, 1, 0, side_>>>(d_norm_, cs, tol, maxcy, h);
    count_launch();
    cudaGraph_t gout = nullptr;
    ok = cudaStreamEndCapture(side_, &gout) == cudaSuccess;
  }
  gsolve_body_launches_ = t_launches - l1;
  // launches counted while capturing did not run
  g_launches.fetch_sub(gsolve_head_launches_ + gsolve_body_launches_, std::memory_order_relaxed);
  t_launches -= gsolve_head_launches_ + gsolve_body_launches_;
  if (ok) ok = cudaGraphInstantiate(&gsolve_, g, 0) == cudaSuccess;
  if (g) cudaGraphDestroy(g);
  if (!ok) {
    cudaGetLastError();
    gsolve_ = nullptr;
    gsolve_state_ = -1;
    return ANEL_OK;
  }
  gsolve_phi_ = d_phi;
  gsolve_rhs_ = d_rhs;
  gsolve_state_ = 1;
  return ANEL_OK;
}

int MGSolver::solve_mixed_graph(double* d_phi, const double* d_rhs, cudaStream_t s, anel_mg_report* rep) {
  if (!gsolve_ || gsolve_phi_ != d_phi || gsolve_rhs_ != d_rhs) {
    const int st = build_solve_graph(d_phi, d_rhs, s);
    if (st != ANEL_OK) return st;
    if (gsolve_state_ < 0) return solve_mixed(d_phi, d_rhs, s, rep);
  }
  ANEL_CUDA_TRY(cudaGraphLaunch(gsolve_, s));
  copy_words(d_conv_, h_pin_, 2, s);  // rel, then (iter, conv)
  ANEL_CUDA_TRY(cudaStreamSynchronize(s));
  const double rel = h_pin_[0];
  int iv[2];
  std::memcpy(iv, &h_pin_[1], sizeof(iv));
  const int iter = iv[0];
  const bool conv = iv[1] != 0;
  count_launch(gsolve_head_launches_ + (int64_t)iter * gsolve_body_launches_);
  rep->iter = conv ? iter : prm_.maxcy + 1;
  rep->relmax = rel;
  rep->resid = rel;
  return conv ? ANEL_OK : ANEL_ERR_NOCONV;
}

// ------------------------------------------------------- batched solve
// Members of a batch share this solver's levels, coefficients, factors and
// tuned launch variants; each has its own FP32 levels (d_bphi32_ /
// d_bsrc32_, member b at b * fp32_elems(l)), direct-solve work, partial
// sums, norms and convergence state.  Every kernel takes the member from
// its work index and skips members whose act flag is 0, so a member's
// arithmetic is that of the one-member solve, whatever else is in the
// batch.

struct BatchConv {
  double rel;
  int iter;
  int conv;
};

__global__ void k_fill_int(int* a, int n, int v) {
  for (int q = threadIdx.x; q < n; q += blockDim.x) a[q] = v;
}

__global__ void k_bconv_init(const double* norm, BatchConv* st, int* act, int n, double tol, int maxcy,
                             cudaGraphConditionalHandle h) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  for (int b = threadIdx.x; b < n; b += blockDim.x) {
    const double rel = conv_rel(norm + 2 * b);
    const int c = rel <= tol;
    st[b].rel = rel;
    st[b].iter = 0;
    st[b].conv = c;
    const int a = (!c && maxcy > 0) ? 1 : 0;
    act[b] = a;
    if (a) atomicOr(&any, 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) cudaGraphSetConditional(h, any ? 1u : 0u);
}

__global__ void k_bconv_step(const double* norm, BatchConv* st, int* act, int n, double tol, int maxcy,
                             cudaGraphConditionalHandle h) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  for (int b = threadIdx.x; b < n; b += blockDim.x) {
    if (!act[b]) continue;  // stopped in an earlier cycle: its state stays
    const double rel = conv_rel(norm + 2 * b);
    const int it = st[b].iter + 1;
    const int c = rel <= tol;
    st[b].rel = rel;
    st[b].iter = it;
    st[b].conv = c;
    const int a = (!c && it < maxcy) ? 1 : 0;
    act[b] = a;
    if (a) atomicOr(&any, 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) cudaGraphSetConditional(h, any ? 1u : 0u);
}

bool MGSolver::batch_capable() const {
  return col_ && prm_.precision == ANEL_PREC_MIXED && gsolve_state_ >= 0;
}

void MGSolver::batch_free() {
  if (bgraph_) cudaGraphExecDestroy(bgraph_);
  bgraph_ = nullptr;
  bgraph_n_ = 0;
  for (int l = 0; l <= ANEL_MAX_LEVELS; ++l) {
    cudaFree(d_bphi32_[l]);
    cudaFree(d_bsrc32_[l]);
    d_bphi32_[l] = d_bsrc32_[l] = nullptr;
  }
  cudaFree(d_bdir_);
  cudaFree(d_bpart_);
  cudaFree(d_bnorm_);
  cudaFree(d_bmt_);
  cudaFree(d_bact_);
  cudaFree(d_bconv_);
  if (h_bmt_) cudaFreeHost(h_bmt_);
  if (h_bconv_) cudaFreeHost(h_bconv_);
  d_bdir_ = d_bpart_ = d_bnorm_ = nullptr;
  d_bmt_ = h_bmt_ = nullptr;
  d_bact_ = nullptr;
  d_bconv_ = h_bconv_ = nullptr;
  bcap_ = 0;
}

int MGSolver::batch_reserve(int n) {
  if (n <= bcap_) return ANEL_OK;
  ANEL_CUDA_TRY(cudaStreamSynchronize(stream_));
  batch_free();
  for (int l = 1; l <= ngrid_; ++l) {
    const size_t b = (size_t)fp32_elems(l) * n * sizeof(float);
    ANEL_CUDA_TRY(cudaMalloc(&d_bphi32_[l], b));
    ANEL_CUDA_TRY(cudaMalloc(&d_bsrc32_[l], b));
    ANEL_CUDA_TRY(cudaMemset(d_bphi32_[l], 0, b));
    ANEL_CUDA_TRY(cudaMemset(d_bsrc32_[l], 0, b));
  }
  if (dirL_ > 0) {
    const DirectFac& F = dir_.f;
    ANEL_CUDA_TRY(cudaMalloc(&d_bdir_, (size_t)n * F.nm * F.nz * sizeof(double)));
  }
  ANEL_CUDA_TRY(cudaMalloc(&d_bpart_, (size_t)col_resid_part_doubles_members(L64(ngrid_), n) * sizeof(double)));
  ANEL_CUDA_TRY(cudaMalloc(&d_bnorm_, (size_t)2 * n * sizeof(double)));
  ANEL_CUDA_TRY(cudaMalloc(&d_bmt_, (size_t)n * sizeof(MemberIO)));
  ANEL_CUDA_TRY(cudaMalloc(&d_bact_, (size_t)n * sizeof(int)));
  ANEL_CUDA_TRY(cudaMalloc(&d_bconv_, (size_t)n * sizeof(BatchConv)));
  ANEL_CUDA_TRY(cudaHostAlloc(&h_bmt_, (size_t)n * sizeof(MemberIO), cudaHostAllocDefault));
  ANEL_CUDA_TRY(cudaHostAlloc(&h_bconv_, (size_t)n * sizeof(BatchConv), cudaHostAllocDefault));
  bcap_ = n;
  return ANEL_OK;
}

int MGSolver::build_batch_graph(int n, cudaStream_t s) {
  if (bgraph_) {
    cudaGraphExecDestroy(bgraph_);
    bgraph_ = nullptr;
    bgraph_n_ = 0;
  }
  if (!side_) ANEL_CUDA_TRY(cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking));
  const int ng = ngrid_;
  const DevLevel<double> Fu = L64(ng);  // geometry only: the arrays come from the member table
  const ColLevel Ec = C32b(ng, n);
  BatchConv* cs = static_cast<BatchConv*>(d_bconv_);
  const double tol = prm_.tolmax;
  const int maxcy = prm_.maxcy;
  cudaGraph_t g = nullptr;
  bool ok = cudaGraphCreate(&g, 0) == cudaSuccess;
  cudaGraphConditionalHandle h{};
  if (ok) ok = cudaGraphConditionalHandleCreate(&h, g, 0, 0) == cudaSuccess;
  const int64_t l0 = t_launches;
  if (ok) ok = cudaStreamBeginCaptureToGraph(s, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) ==
               cudaSuccess;
  cudaGraph_t body = nullptr;
  if (ok) {
    // head: every member active for the boundary pass and first defect
    k_fill_int<<<1, 256, 0, s>>>(d_bact_, n, 1);
    launch_bdry_members(Fu, d_bmt_, d_bact_, n, s);
    launch_col_resid_store_members(Fu, d_bmt_, Ec, d_bpart_, d_bnorm_, s);
    k_bconv_init<<<1, 256, 0, s>>>(d_bnorm_, cs, d_bact_, n, tol, maxcy, h);
    count_launch(2);
    cudaStreamCaptureStatus cst;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    ok = cudaStreamGetCaptureInfo(s, &cst, nullptr, nullptr, &deps, &ndeps) == cudaSuccess &&
         cst == cudaStreamCaptureStatusActive;
    cudaGraphNode_t cnode = nullptr;
    if (ok) {
      cudaGraphNodeParams cp{};
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = h;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      ok = cudaGraphAddNode(&cnode, g, deps, ndeps, &cp) == cudaSuccess;
      if (ok) body = cp.conditional.phGraph_out[0];
      if (ok) ok = cudaStreamUpdateCaptureDependencies(s, &cnode, 1, cudaStreamSetCaptureDependencies) ==
                   cudaSuccess;
    }
    cudaGraph_t gout = nullptr;
    const bool ended = cudaStreamEndCapture(s, &gout) == cudaSuccess;
    ok = ok && ended;
  }
  bgraph_head_launches_ = t_launches - l0;
  // body: one FP32 cycle of every active member, its correction, its next
  // defect and the per-member tests
  const int64_t l1 = t_launches;
  if (ok) ok = cudaStreamBeginCaptureToGraph(side_, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) ==
               cudaSuccess;
  if (ok) {
    cudaMemsetAsync(d_bphi32_[ng], 0, fp32_elems(ng) * n * sizeof(float), side_);
    cycle_col(side_, n);
    launch_col_add_correction_members(Fu, d_bmt_, Ec, side_);
    launch_bdry_members(Fu, d_bmt_, d_bact_, n, side_);
    launch_col_resid_store_members(Fu, d_bmt_, Ec, d_bpart_, d_bnorm_, side_);
    k_bconv_step<<<1, 256, 0, side_>>>(d_bnorm_, cs, d_bact_, n, tol, maxcy, h);
    count_launch();
    cudaGraph_t gout = nullptr;
    ok = cudaStreamEndCapture(side_, &gout) == cudaSuccess;
  }
  bgraph_body_launches_ = t_launches - l1;
  g_launches.fetch_sub(bgraph_head_launches_ + bgraph_body_launches_, std::memory_order_relaxed);
  t_launches -= bgraph_head_launches_ + bgraph_body_launches_;
  if (ok) ok = cudaGraphInstantiate(&bgraph_, g, 0) == cudaSuccess;
  if (g) cudaGraphDestroy(g);
  if (!ok) {
    cudaGetLastError();
    bgraph_ = nullptr;
    set_error("batched solve: CUDA graph capture failed");
    return ANEL_ERR_CUDA;
  }
  bgraph_n_ = n;
  return ANEL_OK;
}

int MGSolver::solve_batch(int n, double* const* phis, const double* const* rhss, cudaStream_t s,
                          anel_mg_report* reps) {
  if (n < 1 || !phis || !rhss || !reps) {
    set_error("solve_batch: n >= 1 and non-null member arrays required");
    return ANEL_ERR_ARG;
  }
  if (!batch_capable()) {
    set_error("solve_batch: needs the column-layout mixed-precision z-line cycle");
    return ANEL_ERR_UNSUPPORTED;
  }
  ANEL_CUDA_TRY(cudaSetDevice(device_));
  if (!s) s = stream_;
  for (int b = 0; b < n; ++b)
    if (!phis[b] || !rhss[b]) {
      set_error("solve_batch: member %d has a null array", b);
      return ANEL_ERR_ARG;
    }
  int st = batch_reserve(n);
  if (st != ANEL_OK) return st;
  if (bgraph_n_ != n) {
    st = build_batch_graph(n, s);
    if (st != ANEL_OK) return st;
  }
  for (int b = 0; b < n; ++b) h_bmt_[b] = MemberIO{phis[b], rhss[b]};
  ANEL_CUDA_TRY(cudaMemcpyAsync(d_bmt_, h_bmt_, (size_t)n * sizeof(MemberIO), cudaMemcpyHostToDevice, s));
  ANEL_CUDA_TRY(cudaEventRecord(ev0_, s));
  ANEL_CUDA_TRY(cudaGraphLaunch(bgraph_, s));
  ANEL_CUDA_TRY(cudaEventRecord(ev1_, s));
  ANEL_CUDA_TRY(cudaMemcpyAsync(h_bconv_, d_bconv_, (size_t)n * sizeof(BatchConv), cudaMemcpyDeviceToHost, s));
  ANEL_CUDA_TRY(cudaStreamSynchronize(s));
  float ms = 0.f;
  ANEL_CUDA_TRY(cudaEventElapsedTime(&ms, ev0_, ev1_));
  st = take_kernel_error("batched solve");
  if (st != ANEL_OK) return st;
  const BatchConv* cv = static_cast<const BatchConv*>(h_bconv_);
  int itmax = 0, rc = ANEL_OK;
  for (int b = 0; b < n; ++b) {
    anel_mg_report& r = reps[b];
    r = anel_mg_report{};
    const bool conv = cv[b].conv != 0;
    r.iter = conv ? cv[b].iter : prm_.maxcy + 1;
    r.relmax = cv[b].rel;
    r.resid = cv[b].rel;
    r.status = conv ? ANEL_OK : ANEL_ERR_NOCONV;
    r.ms = ms;
    itmax = std::max(itmax, cv[b].iter);
    if (!conv) rc = ANEL_ERR_NOCONV;
  }
  count_launch(bgraph_head_launches_ + (int64_t)itmax * bgraph_body_launches_);
  return rc;
}

int MGSolver::solve_mixed(double* d_phi, const double* d_rhs, cudaStream_t s,
                          anel_mg_report* rep) {
  const int ng = ngrid_;
  const DevLevel<double> Fu = fine_view(d_phi, d_rhs);
  const DevLevel<float> E = L32(ng, true);
  launch_bdry(Fu, d_phi, s);
  double rel = 0.0;
  int iter = 0;
  bool conv = false;
  const ColLevel Ec = col_ ? C32(ng) : ColLevel{};
  for (iter = 0; iter <= prm_.maxcy; ++iter) {
    if (col_) launch_col_resid_store(Fu, d_phi, d_rhs, Ec, d_part_, d_norm_, s);
    else launch_resid_store(Fu, d_phi, d_rhs, E.src, d_part_, d_norm_, s);
    copy_words(d_norm_, h_pin_, 2, s);
    ANEL_CUDA_TRY(cudaStreamSynchronize(s));
    rel = h_pin_[1] > 0.0 ? std::sqrt(h_pin_[0] / h_pin_[1]) : std::sqrt(h_pin_[0]);
    if (prm_.verbose) std::fprintf(stderr, "       Defect: %5d  RESID= %22.15e\n", iter, rel);
    if (rel <= prm_.tolmax) {
      conv = true;
      break;
    }
    if (iter == prm_.maxcy) break;
    run_cycle32(s);
    if (col_) launch_col_add_correction(Fu, d_phi, Ec, s);
    else launch_add_correction(Fu, d_phi, E.phi, s);
    launch_bdry(Fu, d_phi, s);
  }
  rep->iter = conv ? iter : prm_.maxcy + 1;
  rep->relmax = rel;
  rep->resid = rel;
  return conv ? ANEL_OK : ANEL_ERR_NOCONV;
}

int MGSolver::solve_host(double* phi, const double* rhs, cudaStream_t s, anel_mg_report* rep) {
  if (!phi || !rhs) {
    set_error("null phi or rhs");
    return ANEL_ERR_ARG;
  }
  ANEL_CUDA_TRY(cudaSetDevice(device_));
  if (!s) s = stream_;
  const size_t bytes = geo_[ngrid_].G * sizeof(double);
  if (!d_io_phi_) {
    ANEL_CUDA_TRY(cudaMalloc(&d_io_phi_, bytes));
    ANEL_CUDA_TRY(cudaMalloc(&d_io_rhs_, bytes));
  }
  ANEL_CUDA_TRY(cudaMemcpyAsync(d_io_phi_, phi, bytes, cudaMemcpyHostToDevice, s));
  ANEL_CUDA_TRY(cudaMemcpyAsync(d_io_rhs_, rhs, bytes, cudaMemcpyHostToDevice, s));
  const int st = solve_device(d_io_phi_, d_io_rhs_, s, rep);
  if (st != ANEL_OK && st != ANEL_ERR_NOCONV) return st;
  ANEL_CUDA_TRY(cudaMemcpyAsync(phi, d_io_phi_, bytes, cudaMemcpyDeviceToHost, s));
  ANEL_CUDA_TRY(cudaStreamSynchronize(s));
  return st;
}

int MGSolver::debug_pass(int which, double* d_phi, const double* d_src, cudaStream_t s) {
  ANEL_CUDA_TRY(cudaSetDevice(device_));
  if (!s) s = stream_;
  const int ng = ngrid_;
  const DevLevel<double> W = L64(ng);
  if (which == 1) {
    DevLevel<double> F = fine_view(d_phi, d_src);
    launch_bdry(F, d_phi, s);
  } else if (which == 0) {
    ANEL_CUDA_TRY(cudaMemcpyAsync(W.phi, d_phi, W.G * sizeof(double), cudaMemcpyDeviceToDevice, s));
    ANEL_CUDA_TRY(cudaMemcpyAsync(W.src, d_src, W.G * sizeof(double), cudaMemcpyDeviceToDevice, s));
    relax64(ng, 1, s);
    ANEL_CUDA_TRY(cudaMemcpyAsync(d_phi, W.phi, W.G * sizeof(double), cudaMemcpyDeviceToDevice, s));
  } else if (which == 2) {
    ANEL_CUDA_TRY(cudaMemcpyAsync(W.phi, d_phi, W.G * sizeof(double), cudaMemcpyDeviceToDevice, s));
    ANEL_CUDA_TRY(cudaMemcpyAsync(W.src, d_src, W.G * sizeof(double), cudaMemcpyDeviceToDevice, s));
    cycle64(s);
    ANEL_CUDA_TRY(cudaMemcpyAsync(d_phi, W.phi, W.G * sizeof(double), cudaMemcpyDeviceToDevice, s));
  } else if (which == 3) {
    // the FP64 direct solve applied to the fine level itself (A phi = src,
    // gauge pinned), then the fine boundary pass: for testing the solver
    if (!col_) {
      set_error("debug pass 3 needs the column-layout cycle (mixed ZLINE, z not coarsened)");
      return ANEL_ERR_UNSUPPORTED;
    }
    if (!dirfine_.d_buf) {
      const int st = build_direct(ng, dirfine_);
      if (st != ANEL_OK) return st;
    }
    const DevLevel<double> F = fine_view(d_phi, d_src);
    launch_direct_row(dirfine_.f, d_src, d_phi, F.X, F.XY, s);
    launch_bdry(F, d_phi, s);
  } else {
    set_error("unknown debug pass %d", which);
    return ANEL_ERR_ARG;
  }
  ANEL_CUDA_TRY(cudaStreamSynchronize(s));
  return check_launch("debug pass");
}

int MGSolver::set_profiling(bool on) {
  prof_ = on;
  return ANEL_OK;
}

void MGSolver::prof_begin(cudaStream_t s) {
  if (prof_ev_.size() < 2 * prof_n_ + 2) {
    for (int q = 0; q < 64; ++q) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      prof_ev_.push_back(e);
    }
  }
  cudaEventRecord(prof_ev_[2 * prof_n_], s);
}

void MGSolver::prof_end(cudaStream_t s) {
  cudaEventRecord(prof_ev_[2 * prof_n_ + 1], s);
  ++prof_n_;
}

int MGSolver::prof_collect(anel_mg_report* r) {
  double ms = 0.0;
  for (size_t q = 0; q < prof_n_; ++q) {
    float t = 0.f;
    ANEL_CUDA_TRY(cudaEventElapsedTime(&t, prof_ev_[2 * q], prof_ev_[2 * q + 1]));
    ms += t;
  }
  r->fine_sweeps = (int32_t)prof_n_;
  r->fine_sweep_ms = ms;
  prof_n_ = 0;
  return ANEL_OK;
}

int MGSolver::levels_table(int32_t* out, int cap) const {
  for (int l = 1; l <= ngrid_ && l <= cap; ++l) {
    const LevelGeom& G = geo_[l];
    int32_t* o = out + (l - 1) * 12;
    o[0] = G.nk[0];
    o[1] = G.nk[1];
    o[2] = G.nk[2];
    o[3] = G.s[0];
    o[4] = G.e[0];
    o[5] = G.s[1];
    o[6] = G.e[1];
    o[7] = G.s[2];
    o[8] = G.e[2];
    o[9] = (int32_t)G.kp3d;
    o[10] = G.kpx[0];
    o[11] = G.kpx[1];
  }
  return ngrid_;
}

}  // namespace anel
