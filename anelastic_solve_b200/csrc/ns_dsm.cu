// ns_dsm.cu -- the dynamic Smagorinsky models: DSM (les/DSM.F90:1-258),
// DSMrho and DSMscal1 (les/DSMrho.F90, les/DSMscal1.F90), with the
// reference's C_avg_dir = 12 (x-y plane averages of the model
// coefficients; LagAvg is not reached).  Compiled with -fmad=false: every
// per-cell expression is evaluated in the source's order, so everything
// up to the plane averages equals the oracle bit for bit; the averages are
// fixed-order parallel sums.
//
// Test filter: filter(.., 2, xfil, yfil, zfil, ..) (les/filter.F90:1-149),
// one direction at a time with the source's zero weights and boundary
// formulas, each followed by the ghost pass of the filtered field's type.
// Smoothing of the coefficient: filterHF(.., 2, 1, 1, 1, ..) (:152-288).
// A plane-constant coefficient stays plane-constant through filterHF, so
// each model yields a profile of k that SGSdiff (k_sgs) consumes like the
// Smagorinsky profiles.
#include <cstring>
#include <vector>

#include "ns_solver.h"

namespace anel {

namespace {

dim3 interior_grid(const NSDev& D) {
  return dim3((unsigned)((D.nx + 127) / 128), (unsigned)D.ny, (unsigned)D.nz);
}

#define DYN_CELL()                                       \
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x; \
  const int j = 2 + blockIdx.y;                          \
  const int k = 2 + blockIdx.z;                          \
  if (i > D.nx + 1) return;                              \
  const int64_t o = NS_IX(i, j, k)

__global__ void k_dyn_modS(NSDev D, const double* __restrict__ l1, const double* __restrict__ l2,
                           const double* __restrict__ l3, double* __restrict__ out) {
  DYN_CELL();
  out[o] = strain_mag(D, l1, l2, l3, i, j, k);
}

// DSM's lestmp1 of component ij (DSM.F90:38-86): the diagonal strain, and
// for ij = 4..6 half the difference of the two cross derivatives (the
// source subtracts where straincal adds).
__global__ void k_dyn_comp(NSDev D, int ij, double* __restrict__ out) {
  DYN_CELL();
  const double *l1 = D.u, *l2 = D.v, *l3 = D.w;
  double r, t1, t2, t3, t4;
  switch (ij) {
    case 1: r = (FA(l1, i + 1, j, k) - FA(l1, i, j, k)) * MT(D.rdxc, i); break;
    case 2: r = (FA(l2, i, j + 1, k) - FA(l2, i, j, k)) * MT(D.rdyc, j); break;
    case 3: r = (FA(l3, i, j, k + 1) - FA(l3, i, j, k)) * MT(D.rdzc, k); break;
    case 4:
      t1 = 0.25 * (FA(l1, i, j, k) + FA(l1, i + 1, j, k) + FA(l1, i, j + 1, k) + FA(l1, i + 1, j + 1, k));
      t2 = 0.25 * (FA(l1, i, j, k) + FA(l1, i + 1, j, k) + FA(l1, i, j - 1, k) + FA(l1, i + 1, j - 1, k));
      t3 = 0.25 * (FA(l2, i, j, k) + FA(l2, i, j + 1, k) + FA(l2, i + 1, j, k) + FA(l2, i + 1, j + 1, k));
      t4 = 0.25 * (FA(l2, i, j, k) + FA(l2, i, j + 1, k) + FA(l2, i - 1, j, k) + FA(l2, i - 1, j + 1, k));
      r = 0.5 * ((t1 - t2) * MT(D.rdyc, j) - (t3 - t4) * MT(D.rdxc, i));
      break;
    case 5:
      t1 = 0.25 * (FA(l1, i, j, k) + FA(l1, i + 1, j, k) + FA(l1, i, j, k + 1) + FA(l1, i + 1, j, k + 1));
      t2 = 0.25 * (FA(l1, i, j, k) + FA(l1, i + 1, j, k) + FA(l1, i, j, k - 1) + FA(l1, i + 1, j, k - 1));
      t3 = 0.25 * (FA(l3, i, j, k) + FA(l3, i, j, k + 1) + FA(l3, i + 1, j, k) + FA(l3, i + 1, j, k + 1));
      t4 = 0.25 * (FA(l3, i, j, k) + FA(l3, i, j, k + 1) + FA(l3, i - 1, j, k) + FA(l3, i - 1, j, k + 1));
      r = 0.5 * ((t1 - t2) * MT(D.rdzc, k) - (t3 - t4) * MT(D.rdxc, i));
      break;
    default:
      t1 = 0.25 * (FA(l2, i, j, k) + FA(l2, i, j + 1, k) + FA(l2, i, j, k + 1) + FA(l2, i, j + 1, k + 1));
      t2 = 0.25 * (FA(l2, i, j, k) + FA(l2, i, j + 1, k) + FA(l2, i, j, k - 1) + FA(l2, i, j + 1, k - 1));
      t3 = 0.25 * (FA(l3, i, j, k) + FA(l3, i, j, k + 1) + FA(l3, i, j + 1, k) + FA(l3, i, j + 1, k + 1));
      t4 = 0.25 * (FA(l3, i, j, k) + FA(l3, i, j, k + 1) + FA(l3, i, j - 1, k) + FA(l3, i, j - 1, k + 1));
      r = 0.5 * ((t1 - t2) * MT(D.rdzc, k) - (t3 - t4) * MT(D.rdyc, j));
  }
  out[o] = r;
}

// One direction of the test filter (HF = false: filter with weights 1/4,
// 1/2, 1/4, written with the source's zero weights, sx and ex boundary
// formulas) or of filterHF (HF = true: a strict local extremum of the
// pencil takes the 3-point average when that is still an extremum of the
// same kind), src -> dst on the interior.  A thread does kDynK planes of
// one (i, j): for the z direction the planes its next cell reads are the
// ones it has just read, so they come from L1.
constexpr int kDynK = 8;
template <int DIR, bool HF>
__global__ void __launch_bounds__(128) k_dyn_pass(NSDev D, const double* __restrict__ src,
                                                  double* __restrict__ dst) {
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y;
  const int k0 = 2 + blockIdx.z * kDynK;
  if (i > D.nx + 1) return;
  const int kend = min(k0 + kDynK, D.nz + 2);  // exclusive
  const int n = DIR == 0 ? D.nx : (DIR == 1 ? D.ny : D.nz);
  const int64_t st = DIR == 0 ? 1 : (DIR == 1 ? (int64_t)D.X : D.XY);
  for (int k = k0; k < kend; ++k) {
    const int64_t o = NS_IX(i, j, k);
    const int q = DIR == 0 ? i : (DIR == 1 ? j : k);
    const double* p = src + o;
    if constexpr (!HF) {
      const double w0 = 0.0, w1 = 1.0 / 4.0, w2 = 1.0 / 2.0, w3 = 1.0 / 4.0, w4 = 0.0;
      double r;
      if (q == 2)
        r = w1 * p[-st] + w2 * p[0] + w3 * p[st] + w4 * p[2 * st] + w0 * p[3 * st];
      else if (q == n + 1)
        r = w1 * p[st] + w2 * p[0] + w3 * p[-st] + w4 * p[-2 * st] + w0 * p[-3 * st];
      else
        r = w0 * p[-2 * st] + w1 * p[-st] + w2 * p[0] + w3 * p[st] + w4 * p[2 * st];
      dst[o] = r;
    } else {
      const double p0 = p[0], pm = p[-st], pp = p[st];
      double r = p0;
      if (p0 < pp && p0 < pm) {
        const double x = 1.0 / 4.0 * pm + 1.0 / 2.0 * p0 + 1.0 / 4.0 * pp;
        if (x < pp && x < pm) r = x;
      } else if (p0 > pp && p0 > pm) {
        const double x = 1.0 / 4.0 * pm + 1.0 / 2.0 * p0 + 1.0 / 4.0 * pp;
        if (x > pp && x > pm) r = x;
      }
      dst[o] = r;
    }
  }
}

template <int DIR>
void dyn_pass_launch(const NSDev& D, const double* src, double* dst, int hf, cudaStream_t s) {
  const dim3 g((unsigned)((D.nx + 127) / 128), (unsigned)D.ny, (unsigned)((D.nz + kDynK - 1) / kDynK));
  if (hf)
    k_dyn_pass<DIR, true><<<g, 128, 0, s>>>(D, src, dst);
  else
    k_dyn_pass<DIR, false><<<g, 128, 0, s>>>(D, src, dst);
}

void launch_dyn_pass(const NSDev& D, const double* src, double* dst, int dir, int hf, cudaStream_t s) {
  if (dir == 0)
    dyn_pass_launch<0>(D, src, dst, hf, s);
  else if (dir == 1)
    dyn_pass_launch<1>(D, src, dst, hf, s);
  else
    dyn_pass_launch<2>(D, src, dst, hf, s);
}

// whole-array assignments of the source (ghost cells included)
enum { EW_SUB, EW_MUL, EW_ACC, EW_ACC2, EW_DEC1, EW_DEC, EW_DEC2 };
// (out may alias a or b: no __restrict__)
__global__ void k_dyn_ew(int op, int64_t n, double* out, const double* a, const double* b, const double* c) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    switch (op) {
      case EW_SUB: out[t] = a[t] - b[t]; break;                          // l3 = l3 - l2
      case EW_MUL: out[t] = a[t] * b[t]; break;                          // l1 = l1*l2
      case EW_ACC: out[t] = out[t] + a[t] * b[t]; break;                 // l4 = l4 + l3*l2
      case EW_ACC2: out[t] = out[t] + 2.0 * a[t] * b[t]; break;          // l4 = l4 + 2.d0*l3*l2
      case EW_DEC1: out[t] = out[t] - a[t] * b[t]; break;                // l3 = l3 - lestmp*l1
      case EW_DEC: out[t] = out[t] - a[t] * b[t] * c[t]; break;          // l4 = l4 - l3*l2*l2
      default: out[t] = out[t] - 2.0 * a[t] * b[t] * c[t];               // l4 = l4 - 2.d0*l3*l1*l2
    }
  }
}

// interior products with the filter width delg(k):
//   SC_A: out = delg**2 * modS * a                 (DSM.F90:91)
//   SC_B: out = (rt*delg)**2 * a * b               (DSM.F90:101)
//   SC_C: out = out - (rt*delg)**2 * a * b         (DSMrho.F90:92)
enum { SC_A, SC_B, SC_C };
__global__ void k_dyn_scale(NSDev D, int op, double* out, const double* a, const double* b, const double* dg,
                            double rt) {
  DYN_CELL();
  const double g = dg[k - 1];
  if (op == SC_A) {
    out[o] = g * g * b[o] * a[o];
  } else {
    const double rd = rt * g;
    if (op == SC_B) out[o] = rd * rd * a[o] * b[o];
    else out[o] = out[o] - rd * rd * a[o] * b[o];
  }
}

// DSMrho's gradient of the scalar c in direction dir (DSMrho.F90:30-75):
// weighted: delg**2 * modS * (tmp2 - tmp1) * rd, else (tmp2 - tmp1) * rd
__global__ void k_dyn_sgrad(NSDev D, const double* __restrict__ c, const double* __restrict__ modS,
                            const double* __restrict__ dg, int dir, int weighted, double* __restrict__ out) {
  DYN_CELL();
  const int64_t st = dir == 0 ? 1 : (dir == 1 ? (int64_t)D.X : D.XY);
  const double t1 = 0.5 * (c[o] + c[o - st]);
  const double t2 = 0.5 * (c[o] + c[o + st]);
  const double rd = dir == 0 ? MT(D.rdxc, i) : (dir == 1 ? MT(D.rdyc, j) : MT(D.rdzc, k));
  const double g = dg[k - 1];
  out[o] = weighted ? g * g * modS[o] * (t2 - t1) * rd : (t2 - t1) * rd;
}

// DSMrho's flux c * 0.5 * (vel(prev) + vel) (DSMrho.F90:100-125)
__global__ void k_dyn_flux(NSDev D, const double* __restrict__ c, const double* __restrict__ vel, int dir,
                           double* __restrict__ out) {
  DYN_CELL();
  const int64_t st = dir == 0 ? 1 : (dir == 1 ? (int64_t)D.X : D.XY);
  out[o] = c[o] * 0.5 * (vel[o - st] + vel[o]);
}

// interior = the plane value (clip: negative values to 0)
__global__ void k_dyn_bcast(NSDev D, const double* __restrict__ prof, int clip, double* __restrict__ out) {
  DYN_CELL();
  double v = prof[k - 1];
  if (clip && v < 0.0) v = 0.0;
  out[o] = v;
}

// out = 0.5 num / den, 1e-20 where den == 0 (DSM.F90:242-250)
__global__ void k_dyn_ratio(NSDev D, const double* __restrict__ num, const double* __restrict__ den,
                            double* __restrict__ out) {
  DYN_CELL();
  out[o] = den[o] == 0.0 ? 1.0e-20 : 0.5 * num[o] / den[o];
}

// the column (2, 2, k), k = 1..Z, of a plane-constant field
__global__ void k_dyn_column(NSDev D, const double* __restrict__ a, double* __restrict__ prof) {
  const int k = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (k > D.Z) return;
  prof[k - 1] = a[NS_IX(2, 2, k)];
}

#undef DYN_CELL

}  // namespace

// ------------------------------------------------------------ host side
enum { DY_MODS, DY_FMODS, DY_C0, DY_FC0 = DY_C0 + 3, DY_L1 = DY_FC0 + 3, DY_L2, DY_L3, DY_L4, DY_A, DY_B, DY_P,
       DY_TMP, DY_N };

int NSSolver::ensure_dyn() {
  if (d_dyn_) return ANEL_OK;
  const int X = nx_ + 2, Y = ny_ + 2, Z = nz_ + 2;
  ANEL_CUDA_TRY(cudaMalloc(&d_dyn_, (size_t)DY_N * G_ * sizeof(double)));
  ANEL_CUDA_TRY(cudaMemset(d_dyn_, 0, (size_t)DY_N * G_ * sizeof(double)));
  // dxc[X] dyc[Y] delg[Z] profiles[2Z], then the plane partial sums
  std::vector<double> h;
  h.insert(h.end(), m_[0][3].begin(), m_[0][3].end());
  h.insert(h.end(), m_[1][3].begin(), m_[1][3].end());
  std::vector<double> dg(Z, 0.0);
  const double dxc = m_[0][3][1], dyc = m_[1][3][1];
  for (int k = 2; k <= nz_ + 1; ++k) {
    const double dzc = m_[2][3][k - 1];
    dg[k - 1] = prm_.les_delta == ANEL_DELTA_3ROOT ? std::pow(dxc * dyc * dzc, 1.0 / 3.0)
                                                   : std::pow(dxc * dxc + dyc * dyc + dzc * dzc, 1.0 / 2.0);
  }
  h.insert(h.end(), dg.begin(), dg.end());
  h.resize(h.size() + 2 * (size_t)Z, 0.0);
  const size_t nm = h.size();
  ANEL_CUDA_TRY(cudaMalloc(&d_dyn_m_, (nm + (size_t)plane_part_doubles(D_)) * sizeof(double)));
  ANEL_CUDA_TRY(cudaMemcpy(d_dyn_m_, h.data(), nm * sizeof(double), cudaMemcpyHostToDevice));
  dyn_part_ = d_dyn_m_ + nm;
  // coordinates for center_velocity: xe xc ye yc ze zc
  std::vector<double> ax;
  for (int d = 0; d < 3; ++d)
    for (int q = 0; q < 2; ++q) ax.insert(ax.end(), m_[d][q].begin(), m_[d][q].end());
  ANEL_CUDA_TRY(cudaMalloc(&d_dyn_axes_, ax.size() * sizeof(double)));
  ANEL_CUDA_TRY(cudaMemcpy(d_dyn_axes_, ax.data(), ax.size() * sizeof(double), cudaMemcpyHostToDevice));
  {
    const int len[3] = {X, Y, Z};
    double* p = d_dyn_axes_;
    for (int d = 0; d < 3; ++d)
      for (int q = 0; q < 2; ++q) {
        d_dyn_ax_[2 * d + q] = p;
        p += len[d];
      }
  }
  double area = 0.0;
  for (int j = 2; j <= ny_ + 1; ++j)
    for (int i = 2; i <= nx_ + 1; ++i) area = area + m_[0][3][i - 1] * m_[1][3][j - 1];
  dyn_area_ = area;
  (void)X;
  (void)Y;
  return ANEL_OK;
}

// filter(in, out, 2, xfil, yfil, zfil, vt) (hf = 0) or filterHF(in, out,
// 2, 1, 1, 1, vt) (hf = 1): in is not modified
void NSSolver::dyn_filter(const double* in, double* out, int vt, int hf, cudaStream_t s, double* tmp) {
  if (!tmp) tmp = d_dyn_ + (size_t)DY_TMP * G_;
  const double* cur = in;
  for (int d = 0; d < 3; ++d) {
    if (hf || prm_.filt[d]) {
      double* dst = (cur == out) ? tmp : out;
      launch_dyn_pass(D_, cur, dst, d, hf, s);
      count_launch();
      cur = dst;
    } else if (cur == in) {
      cudaMemcpyAsync(out, in, G_ * sizeof(double), cudaMemcpyDeviceToDevice, s);
      cur = out;
    }
    launch_ghost_field(D_, const_cast<double*>(cur), zrule(vt), s);
  }
  if (cur != out) cudaMemcpyAsync(out, cur, G_ * sizeof(double), cudaMemcpyDeviceToDevice, s);
}

// Every 50 steps the driver smooths the scalars of the LES scalar models
// with filterHF(.., 2, 1, 1, 1, 'rho' / 'scal1', ..) (NSsolver.F90:144-164;
// its EDIFF and tol arguments are unused, filter.F90:209,237,266): a
// whole-array copy back, then the field's ghost pass.  q_rho and q_s are
// the scratch (the driver's zero_temps comes first) and are zeroed again.
int NSSolver::smooth_scalars(cudaStream_t s) {
  double* a = D_.qr;
  double* b = D_.qs;
  double* f[2] = {D_.rles ? D_.rho : nullptr, D_.sles ? D_.s : nullptr};
  const int vt[2] = {NV_RHO, NV_SCAL1};
  for (int q = 0; q < 2; ++q) {
    if (!f[q]) continue;
    dyn_filter(f[q], a, vt[q], 1, s, b);
    ANEL_CUDA_TRY(cudaMemcpyAsync(f[q], a, G_ * sizeof(double), cudaMemcpyDeviceToDevice, s));
    launch_ghost_field(D_, f[q], zrule(vt[q]), s);
  }
  ANEL_CUDA_TRY(cudaMemsetAsync(a, 0, G_ * sizeof(double), s));
  ANEL_CUDA_TRY(cudaMemsetAsync(b, 0, G_ * sizeof(double), s));
  return ANEL_OK;
}

void NSSolver::dyn_ew(int op, double* out, const double* a, const double* b, const double* c, cudaStream_t s) {
  int64_t blocks = (G_ + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_dyn_ew<<<(unsigned)blocks, 256, 0, s>>>(op, G_, out, a, b, c);
  count_launch();
}

// modS, fmodS (get_fmodS, straincal.F90:166-229), the centred velocities
// and their test-filtered forms (DSM.F90:126-196 recomputes these per use;
// the values are the same)
int NSSolver::dyn_prepare(cudaStream_t s) {
  if (dyn_ready_) return ANEL_OK;
  dyn_ready_ = true;
  double* F = d_dyn_;
  const dim3 g = interior_grid(D_);
  double* modS = F + (size_t)DY_MODS * G_;
  double* fmodS = F + (size_t)DY_FMODS * G_;
  double *l1 = F + (size_t)DY_L1 * G_, *l2 = F + (size_t)DY_L2 * G_, *l3 = F + (size_t)DY_L3 * G_;
  k_dyn_modS<<<g, 128, 0, s>>>(D_, D_.u, D_.v, D_.w, modS);
  count_launch();
  launch_ghost_field(D_, modS, zrule(NV_CFLUC), s);
  dyn_filter(D_.u, l1, NV_U, 0, s);
  dyn_filter(D_.v, l2, NV_V, 0, s);
  dyn_filter(D_.w, l3, NV_W, 0, s);
  k_dyn_modS<<<g, 128, 0, s>>>(D_, l1, l2, l3, fmodS);
  count_launch();
  launch_ghost_field(D_, fmodS, zrule(NV_CFLUC), s);
  const double* vel[3] = {D_.u, D_.v, D_.w};
  const double* ax_e[3] = {d_dyn_ax_[0], d_dyn_ax_[2], d_dyn_ax_[4]};
  const double* ax_c[3] = {d_dyn_ax_[1], d_dyn_ax_[3], d_dyn_ax_[5]};
  for (int d = 0; d < 3; ++d) {
    double* c = F + (size_t)(DY_C0 + d) * G_;
    launch_center(D_, vel[d], c, d + 1, prm_.stretched[d], prm_.interp == ANEL_DIAG_CORRECTED, ax_e[d], ax_c[d],
                  s);
    launch_ghost_field(D_, c, zrule(d == 0 ? NV_U : (d == 1 ? NV_V : NV_W)), s);
    dyn_filter(c, F + (size_t)(DY_FC0 + d) * G_, NV_CFLUC, 0, s);
  }
  ANEL_CUDA_TRY(cudaGetLastError());
  return ANEL_OK;
}

// plane averages of num and den, plane values on the interior (num
// clipped at 0), out = 0.5 num / den, filterHF (DSM.F90:196-256)
int NSSolver::dyn_ratio(double* num, double* den, double* out, cudaStream_t s) {
  const int X = nx_ + 2, Y = ny_ + 2, Z = nz_ + 2;
  const double* dxc = d_dyn_m_;
  const double* dyc = dxc + X;
  double* pn = d_dyn_m_ + X + Y + Z;
  double* pd = pn + Z;
  const dim3 g = interior_grid(D_);
  const ZRule cf = zrule(NV_CFLUC);
  launch_ghost_field(D_, num, cf, s);
  launch_ghost_field(D_, den, cf, s);
  launch_plane_avg(D_, num, dxc, dyc, dyn_area_, dyn_part_, pn, s);
  launch_plane_avg(D_, den, dxc, dyc, dyn_area_, dyn_part_, pd, s);
  k_dyn_bcast<<<g, 128, 0, s>>>(D_, pn, 1, num);
  k_dyn_bcast<<<g, 128, 0, s>>>(D_, pd, 0, den);
  count_launch(2);
  launch_ghost_field(D_, num, cf, s);
  launch_ghost_field(D_, den, cf, s);
  k_dyn_ratio<<<g, 128, 0, s>>>(D_, num, den, out);
  count_launch();
  launch_ghost_field(D_, out, cf, s);
  double* P = d_dyn_ + (size_t)DY_P * G_;
  dyn_filter(out, P, NV_CFLUC, 1, s);
  ANEL_CUDA_TRY(cudaMemcpyAsync(out, P, G_ * sizeof(double), cudaMemcpyDeviceToDevice, s));
  launch_ghost_field(D_, out, cf, s);
  ANEL_CUDA_TRY(cudaGetLastError());
  return ANEL_OK;
}

int NSSolver::dyn_profile(const double* a, double* host, cudaStream_t s) {
  const int Z = nz_ + 2;
  double* pr = d_dyn_m_ + (nx_ + 2) + (ny_ + 2) + Z;
  k_dyn_column<<<(Z + 127) / 128, 128, 0, s>>>(D_, a, pr);
  count_launch();
  ANEL_CUDA_TRY(cudaMemcpyAsync(host, pr, Z * sizeof(double), cudaMemcpyDeviceToHost, s));
  ANEL_CUDA_TRY(cudaStreamSynchronize(s));
  return ANEL_OK;
}

// DSM (DSM.F90:1-258): the Csgs profile into cs (Z values)
int NSSolver::dsm_velocity(cudaStream_t s, double* cs) {
  int st = ensure_dyn();
  if (st != ANEL_OK) return st;
  if ((st = dyn_prepare(s)) != ANEL_OK) return st;
  double* F = d_dyn_;
  const dim3 g = interior_grid(D_);
  const double* dg = d_dyn_m_ + (nx_ + 2) + (ny_ + 2);
  const double* modS = F + (size_t)DY_MODS * G_;
  const double* fmodS = F + (size_t)DY_FMODS * G_;
  double *l1 = F + (size_t)DY_L1 * G_, *l2 = F + (size_t)DY_L2 * G_, *l3 = F + (size_t)DY_L3 * G_;
  double *l4 = F + (size_t)DY_L4 * G_, *A = F + (size_t)DY_A * G_, *C = F + (size_t)DY_B * G_;
  const ZRule cf = zrule(NV_CFLUC);
  ANEL_CUDA_TRY(cudaMemsetAsync(l4, 0, G_ * sizeof(double), s));
  ANEL_CUDA_TRY(cudaMemsetAsync(C, 0, G_ * sizeof(double), s));
  static const int pa[7] = {0, 0, 1, 2, 0, 0, 1}, pb[7] = {0, 0, 1, 2, 1, 2, 2};
  for (int ij = 1; ij <= 6; ++ij) {
    k_dyn_comp<<<g, 128, 0, s>>>(D_, ij, l1);
    count_launch();
    launch_ghost_field(D_, l1, cf, s);
    k_dyn_scale<<<g, 128, 0, s>>>(D_, SC_A, l2, l1, modS, dg, 0.0);
    count_launch();
    launch_ghost_field(D_, l2, cf, s);
    dyn_filter(l2, l3, NV_CFLUC, 0, s);
    dyn_filter(l1, l2, NV_CFLUC, 0, s);
    ANEL_CUDA_TRY(cudaMemcpyAsync(l1, fmodS, G_ * sizeof(double), cudaMemcpyDeviceToDevice, s));
    k_dyn_scale<<<g, 128, 0, s>>>(D_, SC_B, l2, l1, l2, dg, prm_.test_ratio);
    count_launch();
    launch_ghost_field(D_, l2, cf, s);
    dyn_ew(EW_SUB, l3, l3, l2, nullptr, s);
    launch_ghost_field(D_, l3, cf, s);
    const double* ca = F + (size_t)(DY_C0 + pa[ij]) * G_;
    const double* cb = F + (size_t)(DY_C0 + pb[ij]) * G_;
    dyn_ew(EW_MUL, A, ca, cb, nullptr, s);
    dyn_filter(A, l2, NV_CFLUC, 0, s);
    const double* fa = F + (size_t)(DY_FC0 + pa[ij]) * G_;
    const double* fb = F + (size_t)(DY_FC0 + pb[ij]) * G_;
    if (ij <= 3) {
      dyn_ew(EW_ACC, l4, l3, l2, nullptr, s);
      dyn_ew(EW_DEC, l4, l3, fa, fb, s);
      dyn_ew(EW_ACC, C, l3, l3, nullptr, s);
    } else {
      dyn_ew(EW_ACC2, l4, l3, l2, nullptr, s);
      dyn_ew(EW_DEC2, l4, l3, fa, fb, s);
      dyn_ew(EW_ACC2, C, l3, l3, nullptr, s);
    }
  }
  // Csgs = 0.5 <LM> / <MM>: num = l4, den = a copy of C, out = C
  double* den = F + (size_t)DY_A * G_;
  ANEL_CUDA_TRY(cudaMemcpyAsync(den, C, G_ * sizeof(double), cudaMemcpyDeviceToDevice, s));
  if ((st = dyn_ratio(l4, den, C, s)) != ANEL_OK) return st;
  return dyn_profile(C, cs, s);
}

// DSMrho / DSMscal1 (DSMrho.F90:1-240) of the scalar c: the CTsgs / CSsgs
// profile into out (Z values)
int NSSolver::dsm_scalar(const double* c, cudaStream_t s, double* out) {
  int st = ensure_dyn();
  if (st != ANEL_OK) return st;
  if ((st = dyn_prepare(s)) != ANEL_OK) return st;
  double* F = d_dyn_;
  const dim3 g = interior_grid(D_);
  const double* dg = d_dyn_m_ + (nx_ + 2) + (ny_ + 2);
  const double* modS = F + (size_t)DY_MODS * G_;
  const double* fmodS = F + (size_t)DY_FMODS * G_;
  double *l1 = F + (size_t)DY_L1 * G_, *l2 = F + (size_t)DY_L2 * G_, *l3 = F + (size_t)DY_L3 * G_;
  double *l4 = F + (size_t)DY_L4 * G_, *A = F + (size_t)DY_A * G_, *C = F + (size_t)DY_B * G_;
  const ZRule cf = zrule(NV_CFLUC);
  ANEL_CUDA_TRY(cudaMemsetAsync(l4, 0, G_ * sizeof(double), s));
  ANEL_CUDA_TRY(cudaMemsetAsync(C, 0, G_ * sizeof(double), s));
  const double* vel[3] = {D_.u, D_.v, D_.w};
  for (int d = 0; d < 3; ++d) {
    k_dyn_sgrad<<<g, 128, 0, s>>>(D_, c, modS, dg, d, 1, l1);
    count_launch();
    launch_ghost_field(D_, l1, cf, s);
    dyn_filter(l1, l2, NV_CFLUC, 0, s);
    k_dyn_sgrad<<<g, 128, 0, s>>>(D_, c, modS, dg, d, 0, l1);
    count_launch();
    launch_ghost_field(D_, l1, cf, s);
    dyn_filter(l1, l3, NV_CFLUC, 0, s);
    ANEL_CUDA_TRY(cudaMemcpyAsync(l1, fmodS, G_ * sizeof(double), cudaMemcpyDeviceToDevice, s));
    k_dyn_scale<<<g, 128, 0, s>>>(D_, SC_C, l2, l1, l3, dg, prm_.test_ratio);
    count_launch();
    launch_ghost_field(D_, l2, cf, s);
    k_dyn_flux<<<g, 128, 0, s>>>(D_, c, vel[d], d, l1);
    count_launch();
    launch_ghost_field(D_, l1, cf, s);
    dyn_filter(l1, l3, NV_CFLUC, 0, s);
    dyn_filter(c, A, NV_CFLUC, 0, s);
    dyn_ew(EW_DEC1, l3, A, F + (size_t)(DY_FC0 + d) * G_, nullptr, s);
    launch_ghost_field(D_, l3, cf, s);
    dyn_ew(EW_ACC, l4, l2, l2, nullptr, s);
    dyn_ew(EW_ACC, C, l2, l3, nullptr, s);
  }
  // C = 0.5 <N> / <D>: num = a copy of C, den = l4, out = C
  ANEL_CUDA_TRY(cudaMemcpyAsync(A, C, G_ * sizeof(double), cudaMemcpyDeviceToDevice, s));
  if ((st = dyn_ratio(A, l4, C, s)) != ANEL_OK) return st;
  return dyn_profile(C, out, s);
}

}  // namespace anel
