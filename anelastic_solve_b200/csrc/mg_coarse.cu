// mg_coarse.cu -- FP64 direct solve of a coarse level (see mg_coarse.cuh):
// host-side basis and factors, launchers.
#include "mg_coarse.h"
#include "mg_col.h"

#include <cmath>
#include <vector>

namespace anel {

// Real orthonormal Fourier basis of n periodic points: row p over i.
// p = 0 constant; p = 2m-1, 2m the cosine and sine of wavenumber m; for
// even n the last row alternates.  theta[p] is the mode's angle, so that
// phi(i-1) + phi(i+1) = 2 cos(theta[p]) phi(i) for basis function p.
static void fourier_basis(int n, std::vector<double>& B, std::vector<double>& theta) {
  const double pi = 3.14159265358979323846;
  B.assign((size_t)n * n, 0.0);
  theta.assign(n, 0.0);
  for (int i = 0; i < n; ++i) B[i] = 1.0 / std::sqrt((double)n);
  const int half = (n - 1) / 2;
  for (int m = 1; m <= half; ++m) {
    const double th = 2.0 * pi * m / n;
    for (int i = 0; i < n; ++i) {
      B[(size_t)(2 * m - 1) * n + i] = std::sqrt(2.0 / n) * std::cos(th * i);
      B[(size_t)(2 * m) * n + i] = std::sqrt(2.0 / n) * std::sin(th * i);
    }
    theta[2 * m - 1] = theta[2 * m] = th;
  }
  if (n % 2 == 0 && n > 1) {
    for (int i = 0; i < n; ++i) B[(size_t)(n - 1) * n + i] = (i % 2 ? -1.0 : 1.0) / std::sqrt((double)n);
    theta[n - 1] = pi;
  }
}

int col_sweep_factors_d(int n, int M, const std::vector<double>& sub, const std::vector<double>& dia,
                        const std::vector<double>& sup, std::vector<double>& out);

int direct_build(DirectHost& D, int nx, int ny, int nz, double a1, double a2, double a3, double a4,
                 const double* cz5, const double* cz6, const double* dz5, const double* dz6, int z1, int zZ) {
  if (nx < 1 || ny < 1 || nx > kDirMaxN || ny > kDirMaxN || nx * ny > kDirMaxModes || nz % 32 != 0 ||
      !col_rows_supported(nz / 32)) {
    set_error("direct coarse solve: level %dx%dx%d out of range", nx, ny, nz);
    return ANEL_ERR_UNSUPPORTED;
  }
  if (!(a1 == a2 && a3 == a4)) {
    set_error("direct coarse solve needs symmetric x/y line coefficients");
    return ANEL_ERR_UNSUPPORTED;
  }
  if (z1 == 2 || zZ == 1 || z1 < 0 || zZ < 0) {
    set_error("direct coarse solve: periodic z is not supported");
    return ANEL_ERR_UNSUPPORTED;
  }
  const int M = nz / 32;
  const int fpm = dir_fac_per_mode(M);
  std::vector<double> Bx, By, tx, ty;
  fourier_basis(nx, Bx, tx);
  fourier_basis(ny, By, ty);
  const int nm = nx * ny;
  std::vector<double> fac((size_t)nm * fpm, 0.0);
  std::vector<double> sub(nz), dia0(nz), sup(nz), dia(nz), sb(nz), mf;
  for (int r = 0; r < nz; ++r) {
    const int k = r + 2;
    sub[r] = cz5[k - 1];
    sup[r] = cz6[k - 1];
    dia0[r] = -(a1 + a2 + a3 + a4 + dz5[k - 1] + dz6[k - 1]);
  }
  // the level's z-ghost rule: a copy of the adjacent row folds into it
  if (z1 == 1) dia0[0] += sub[0];
  if (zZ == 2) dia0[nz - 1] += sup[nz - 1];
  double scale = 0.0;
  for (int r = 0; r < nz; ++r) scale = std::fmax(scale, std::fabs(dia0[r]));
  for (int q = 0; q < ny; ++q)
    for (int p = 0; p < nx; ++p) {
      const int m = p + nx * q;
      const double shift = 2.0 * a1 * std::cos(tx[p]) + 2.0 * a3 * std::cos(ty[q]);
      for (int r = 0; r < nz; ++r) dia[r] = dia0[r] + shift;
      sb = sub;
      double rhs_scale = 1.0;
      if (m == 0) {
        // singular under Neumann walls (rows sum to zero): pin the gauge by
        // replacing the last row with phi = 0
        double worst = 0.0;
        for (int r = 0; r < nz; ++r)
          worst = std::fmax(worst, std::fabs(dia[r] + (r > 0 ? sub[r] : 0.0) + (r < nz - 1 ? sup[r] : 0.0)));
        if (worst <= 1e-12 * scale) {
          sb[nz - 1] = 0.0;
          dia[nz - 1] = 1.0;
          rhs_scale = 0.0;
        }
      }
      const int st = col_sweep_factors_d(nz, M, sb, dia, sup, mf);
      if (st != ANEL_OK) {
        set_error("direct coarse solve: mode %d: %s", m, last_error());
        return ANEL_ERR_UNSUPPORTED;
      }
      double* o = fac.data() + (size_t)m * fpm;
      for (size_t t = 0; t < mf.size(); ++t) o[t] = mf[t];
      o[col_fac_floats(M)] = rhs_scale;
    }
  direct_free(D);
  const size_t nd = Bx.size() + By.size() + fac.size() + (size_t)nz * nm;
  ANEL_CUDA_TRY(cudaMalloc(&D.d_buf, nd * sizeof(double)));
  D.bytes = nd * sizeof(double);
  double* p = D.d_buf;
  auto put = [&](const std::vector<double>& v) -> double* {
    double* at = p;
    cudaMemcpy(at, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice);
    p += v.size();
    return at;
  };
  D.f.nx = nx;
  D.f.ny = ny;
  D.f.nz = nz;
  D.f.nm = nm;
  D.f.M = M;
  D.f.Bx = put(Bx);
  D.f.By = put(By);
  D.f.fac = put(fac);
  D.f.work = p;
  // launch attributes set here, outside any stream capture
  const int sm = (int)dir_smem_bytes(nx, ny);
  set_smem_limit_once((const void*)k_dir_forward<DirColIn>, sm);
  set_smem_limit_once((const void*)k_dir_inverse<DirColOut>, sm);
  set_smem_limit_once((const void*)k_dir_forward<DirRowIn>, sm);
  set_smem_limit_once((const void*)k_dir_inverse<DirRowOut>, sm);
  ANEL_CUDA_TRY(cudaGetLastError());
  return ANEL_OK;
}

void direct_free(DirectHost& D) {
  if (D.d_buf) cudaFree(D.d_buf);
  D.d_buf = nullptr;
  D.bytes = 0;
  D.f = DirectFac{};
}

// One warp per mode of a member: the mode's z-system (mode-major rows), in
// place, by the column sweep's partitioned solve in FP64.
template <int M>
__global__ void __launch_bounds__(128) k_dir_solve(DirectFac F) {
  const int lane = threadIdx.x & 31;
  const int q0 = blockIdx.x * 4 + (threadIdx.x >> 5);
  if (q0 >= F.nm * F.nmem) return;  // the whole warp
  const int b = q0 / F.nm, m = q0 - b * F.nm;
  if (F.act && !F.act[b]) return;
  constexpr int NF = col_fac_floats(M);
  const double* f = F.fac + (int64_t)m * dir_fac_per_mode(M);
  const double* Fap = f;
  const double* Frbp = f + (M - 1) * 32;
  const double* Fsup = f + 2 * (M - 1) * 32;
  const double* FL = f + 3 * (M - 1) * 32;
  const double* FR = f + 4 * (M - 1) * 32;
  const double* Fg = f + 5 * (M - 1) * 32;
  double* w = F.work + ((int64_t)b * F.nm + m) * F.nz;
  double y[M];
#pragma unroll
  for (int q = 0; q < M; ++q) y[q] = w[lane * M + q];
  if (lane == 31) y[M - 1] *= f[NF];  // 0 on the pinned row
  double g = y[0];
#pragma unroll
  for (int q = 1; q < M - 1; ++q) {
    g = y[q] + Fap[q * 32 + lane] * g;
    y[q] = g;
  }
  double x = g * Frbp[(M - 2) * 32 + lane];
  y[M - 2] = x;
#pragma unroll
  for (int q = M - 3; q >= 0; --q) {
    x = (y[q] - Fsup[q * 32 + lane] * x) * Frbp[q * 32 + lane];
    y[q] = x;
  }
  const double ynext = __shfl_down_sync(0xffffffffu, y[0], 1);
  double h = y[M - 1] - Fg[lane] * y[M - 2] - (lane < 31 ? Fg[32 + lane] * ynext : 0.0);
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    const int st = 1 << q;
    const double up = __shfl_up_sync(0xffffffffu, h, st);
    const double dn = __shfl_down_sync(0xffffffffu, h, st);
    h = h + Fg[(2 + q) * 32 + lane] * up + Fg[(7 + q) * 32 + lane] * dn;
  }
  const double xs = h * Fg[12 * 32 + lane];
  const double xprev = __shfl_up_sync(0xffffffffu, xs, 1);
#pragma unroll
  for (int q = 0; q < M - 1; ++q) y[q] = y[q] + FL[q * 32 + lane] * xprev + FR[q * 32 + lane] * xs;
  y[M - 1] = xs;
  if (m == 0) {
    // the constant mode's profile is fixed only up to a constant (the
    // pinned row picks one): return it with zero mean, so that successive
    // coarse corrections add no drifting constant to the solution
    double sum = 0.0;
#pragma unroll
    for (int q = 0; q < M; ++q) sum += y[q];
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    const double mean = sum / (double)(32 * M);
#pragma unroll
    for (int q = 0; q < M; ++q) y[q] -= mean;
  }
#pragma unroll
  for (int q = 0; q < M; ++q) w[lane * M + q] = y[q];
}

static void dir_solve_launch(const DirectFac& F, cudaStream_t s) {
  const unsigned g = (unsigned)((F.nm * F.nmem + 3) / 4);
  switch (F.M) {
    case 2: k_dir_solve<2><<<g, 128, 0, s>>>(F); break;
    case 3: k_dir_solve<3><<<g, 128, 0, s>>>(F); break;
    case 4: k_dir_solve<4><<<g, 128, 0, s>>>(F); break;
    case 6: k_dir_solve<6><<<g, 128, 0, s>>>(F); break;
    case 8: k_dir_solve<8><<<g, 128, 0, s>>>(F); break;
    case 12: k_dir_solve<12><<<g, 128, 0, s>>>(F); break;
    default: k_dir_solve<16><<<g, 128, 0, s>>>(F); break;
  }
}

template <class In, class Out>
static void direct_launch(const DirectFac& F, const In& in, const Out& out, cudaStream_t s) {
  const size_t sm = dir_smem_bytes(F.nx, F.ny);
  set_smem_limit_once((const void*)k_dir_forward<In>, (int)sm);
  set_smem_limit_once((const void*)k_dir_inverse<Out>, (int)sm);
  k_dir_forward<In><<<F.nz * F.nmem, 256, sm, s>>>(F, in);
  dir_solve_launch(F, s);
  k_dir_inverse<Out><<<F.nz * F.nmem, 256, sm, s>>>(F, out);
  count_launch(3);
}

void launch_direct_col(const DirectFac& F, const ColLevel& L, double* work, cudaStream_t s) {
  DirectFac Fb = F;
  Fb.nmem = L.nm;
  Fb.act = L.act;
  if (work) Fb.work = work;
  direct_launch(Fb, DirColIn{L}, DirColOut{L}, s);
}

void launch_direct_row(const DirectFac& F, const double* f, double* phi, int X, int64_t XY, cudaStream_t s) {
  direct_launch(F, DirRowIn{f, X, XY}, DirRowOut{phi, X, XY}, s);
}

}  // namespace anel
