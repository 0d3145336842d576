// ns_solver.cu -- host side of the B200 RK3 time stepper: field storage,
// boundary rules, the column-independent Crank-Nicolson factors and the
// sub-step / step schedule of rk_ss and NSsolver (NSsolver.F90:63-583).
// Host code is compiled with -ffp-contract=off so the factors round as
// the reference's expressions.
#include "ns_solver.h"
#include "tune.h"

#include <cmath>
#include <cstdlib>
#include <cstring>

namespace anel {

static const int kVarCode[5] = {1, 2, 3, 5, 8};  // u v w rho scal1 (boundC index)

NSSolver* NSSolver::create(const anel_grid_desc* g, const anel_mg_params* mg,
                           const anel_ns_params* ns, int device, int* status) {
  NSSolver* s = new NSSolver();
  const int st = s->init(g, mg, ns, device);
  if (status) *status = st;
  if (st != ANEL_OK) {
    delete s;
    return nullptr;
  }
  return s;
}

NSSolver::~NSSolver() {
  cudaSetDevice(device_);
  delete mg_;
  for (double* p : d_fields_) cudaFree(p);
  cudaFree(d_metric_);
  cudaFree(d_prof_);
  cudaFree(d_cn_);
  cudaFree(d_les_);
  cudaFree(d_ic_);
  cudaFree(d_cnb_);
  cudaFree(d_red_);
  cudaFree(d_part_);
  for (auto& h : hist_)
    for (double* a : h) cudaFree(a);
  if (h_cn_) cudaFreeHost(h_cn_);
  if (h_red_) cudaFreeHost(h_red_);
  if (ev0_) cudaEventDestroy(ev0_);
  if (ev1_) cudaEventDestroy(ev1_);
  cudaFree(d_diag_);
  cudaFree(d_dgA_);
  cudaFree(d_dgB_);
  cudaFree(d_dgm_);
  cudaFree(d_dgpart_);
  cudaFree(d_dyn_);
  cudaFree(d_dyn_m_);
  cudaFree(d_dyn_axes_);
  if (dev0_) cudaEventDestroy(dev0_);
  if (dev1_) cudaEventDestroy(dev1_);
  for (cudaEvent_t e : io_ev_)
    if (e) cudaEventDestroy(e);
  if (io_stream_) cudaStreamDestroy(io_stream_);
  if (stream_) cudaStreamDestroy(stream_);
}

// clip: with scal1 held at zero (scal1_on = 0) its range must keep it there
static int check_clip(const anel_ns_params* ns) {
  if (ns->clip && !ns->scal1_on && !(ns->scal1_min <= 0.0 && 0.0 <= ns->scal1_max)) {
    set_error("clip: with scal1_on = 0 the scal1 range [%g, %g] must contain 0", ns->scal1_min, ns->scal1_max);
    return ANEL_ERR_ARG;
  }
  return ANEL_OK;
}

int NSSolver::init(const anel_grid_desc* g, const anel_mg_params* mgp, const anel_ns_params* ns,
                   int device) {
  if (!g || !mgp || !ns) {
    set_error("null grid, mg or ns parameters");
    return ANEL_ERR_ARG;
  }
  if (check_clip(ns) != ANEL_OK) return ANEL_ERR_ARG;
  prm_ = *ns;
  device_ = device;
  nx_ = g->nx;
  ny_ = g->ny;
  nz_ = g->nz;
  // this implementation: x and y periodic for every field
  for (int d = 0; d < 2; ++d)
    for (int f = 0; f < 2; ++f)
      for (int v = 0; v < 8; ++v)
        if (ns->tb[d][f][v] != 3) {
          set_error("the GPU stepper needs x and y periodic for every field (TB(%d,%d,%d)=%d)", d + 1,
                    f + 1, v + 1, ns->tb[d][f][v]);
          return ANEL_ERR_UNSUPPORTED;
        }
  // z wall types the CN rows of var_advance_CN_PL accept (NSsolver.F90:3297-3429)
  for (int vi = 0; vi < 5; ++vi) {
    const int v = kVarCode[vi] - 1;
    const int t0 = ns->tb[2][0][v], t1 = ns->tb[2][1][v];
    if (!(t0 == 1 || t0 == 2 || t0 == 6) || !(t1 == 1 || t1 == 2 || t1 == 6 || t1 == 7)) {
      set_error("z boundary types %d/%d of variable %d have no Crank-Nicolson row in the reference",
                t0, t1, v + 1);
      return ANEL_ERR_BC;
    }
  }
  for (int m : {ns->vmodel, ns->rmodel, ns->smodel})
    if (m != ANEL_MODEL_DNS && m != ANEL_MODEL_SSM && m != ANEL_MODEL_DSM) {
      set_error("unknown subgrid model %d", m);
      return ANEL_ERR_ARG;
    }
  les_any_ = ns->vmodel != ANEL_MODEL_DNS || ns->rmodel != ANEL_MODEL_DNS || ns->smodel != ANEL_MODEL_DNS;
  if (ns->vmodel == ANEL_MODEL_DSM || ns->rmodel == ANEL_MODEL_DSM || ns->smodel == ANEL_MODEL_DSM) {
    // the test filter's boundary formulas reach three cells in; the
    // centring interpolation needs four
    const int n[3] = {g->nx, g->ny, g->nz};
    for (int d = 0; d < 3; ++d)
      if (n[d] < 4) {
        set_error("the dynamic models need at least 4 cells in every direction");
        return ANEL_ERR_SIZE;
      }
    if (!(ns->test_ratio > 0.0) || (ns->interp != ANEL_DIAG_LITERAL && ns->interp != ANEL_DIAG_CORRECTED)) {
      set_error("dynamic model: test_ratio must be positive and interp LITERAL or CORRECTED");
      return ANEL_ERR_ARG;
    }
  }
  if (ns->vmodel != ANEL_MODEL_DNS) {
    if (ns->les_freq < 1) {
      set_error("les_freq must be >= 1");
      return ANEL_ERR_ARG;
    }
    if (ns->les_delta != ANEL_DELTA_3ROOT && ns->les_delta != ANEL_DELTA_2ROOT) {
      set_error("unknown les_delta %d", ns->les_delta);
      return ANEL_ERR_ARG;
    }
    // the model coefficients are kept as profiles of k: x and y spacing
    // must be uniform (the filter width delg then depends on k only)
    for (int d = 0; d < 2; ++d) {
      const double* dxc = d == 0 ? g->dxc : g->dyc;
      const int n = d == 0 ? nx_ : ny_;
      for (int i = 2; i <= n + 1; ++i)
        if (!(dxc[i - 1] == dxc[1])) {
          set_error("the GPU LES model needs uniform %s spacing (dxc(%d) differs)", d == 0 ? "x" : "y", i);
          return ANEL_ERR_UNSUPPORTED;
        }
    }
  }
  if (ns->ew != 0 && ns->ew != 1) {
    set_error("ew must be 0 or 1");
    return ANEL_ERR_ARG;
  }
  // the Crank-Nicolson kernels stage up to 10 column profiles of nz+3
  // doubles in shared memory (200 KB at most)
  if (10 * (int64_t)(nz_ + 3) * 8 > 200 * 1024) {
    set_error("nz = %d exceeds the column solver's limit of 2557", nz_);
    return ANEL_ERR_UNSUPPORTED;
  }
  const int n[3] = {nx_, ny_, nz_};
  const double* src[3][6] = {{g->xe, g->xc, g->dxe, g->dxc, g->rdxe, g->rdxc},
                             {g->ye, g->yc, g->dye, g->dyc, g->rdye, g->rdyc},
                             {g->ze, g->zc, g->dze, g->dzc, g->rdze, g->rdzc}};
  for (int d = 0; d < 3; ++d)
    for (int a = 0; a < 6; ++a) m_[d][a].assign(src[d][a], src[d][a] + n[d] + 2);
  rRe_ = 1.0 / ns->Re;
  rPr_ = 1.0 / ns->Pr;
  rSc_ = 1.0 / ns->Sc;
  g_orig_ = ns->g_final;
  gnow_ = ns->g_init;
  int st = ANEL_OK;
  mg_ = MGSolver::create(g, mgp, device, &st);
  if (!mg_) return st;
  ANEL_CUDA_TRY(cudaSetDevice(device_));
  ANEL_CUDA_TRY(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  ANEL_CUDA_TRY(cudaEventCreate(&ev0_));
  ANEL_CUDA_TRY(cudaEventCreate(&ev1_));
  const int X = nx_ + 2, Y = ny_ + 2, Z = nz_ + 2;
  G_ = (int64_t)X * Y * Z;
  for (int q = 0; q < 17; ++q) {
    if (q == 6 || q == 7) continue;  // r, densityBG: allocated below
    if (q >= 14 && !les_any_) continue;  // nuT, kappaT, nappaT: LES only
    ANEL_CUDA_TRY(cudaMalloc(&d_fields_[q], G_ * sizeof(double)));
    ANEL_CUDA_TRY(cudaMemset(d_fields_[q], 0, G_ * sizeof(double)));
  }
  if (les_any_) {
    // model profiles Csgs, CTsgs, CSsgs, delg^2 (zero until the first
    // les_coeffs of the step cadence)
    ANEL_CUDA_TRY(cudaMalloc(&d_les_, 4 * (size_t)Z * sizeof(double)));
    ANEL_CUDA_TRY(cudaMemset(d_les_, 0, 4 * (size_t)Z * sizeof(double)));
  }
  if (ns->vmodel != ANEL_MODEL_DNS) {
    // per-column eliminated diagonal of the LES CN solve
    ANEL_CUDA_TRY(cudaMalloc(&d_cnb_, G_ * sizeof(double)));
  }
  // metrics
  std::vector<double> met;
  for (int a : {4, 5}) met.insert(met.end(), m_[0][a].begin(), m_[0][a].end());
  for (int a : {4, 5}) met.insert(met.end(), m_[1][a].begin(), m_[1][a].end());
  for (int a : {4, 5}) met.insert(met.end(), m_[2][a].begin(), m_[2][a].end());
  met.insert(met.end(), m_[2][2].begin(), m_[2][2].end());  // dze
  met.insert(met.end(), m_[2][3].begin(), m_[2][3].end());  // dzc
  ANEL_CUDA_TRY(cudaMalloc(&d_metric_, met.size() * sizeof(double)));
  ANEL_CUDA_TRY(cudaMemcpy(d_metric_, met.data(), met.size() * sizeof(double), cudaMemcpyHostToDevice));
  ANEL_CUDA_TRY(cudaMalloc(&d_prof_, 2 * (size_t)Z * sizeof(double)));
  const size_t ncn = 3 * 5 * 9 * (size_t)Z;
  ANEL_CUDA_TRY(cudaMalloc(&d_cn_, ncn * sizeof(double)));
  ANEL_CUDA_TRY(cudaHostAlloc(&h_cn_, ncn * sizeof(double), cudaHostAllocMapped));
  ANEL_CUDA_TRY(cudaMalloc(&d_red_, 4 * sizeof(unsigned long long)));
  ANEL_CUDA_TRY(cudaHostAlloc(&h_red_, 4 * sizeof(double), cudaHostAllocMapped));
  // device view
  D_.nx = nx_;
  D_.ny = ny_;
  D_.nz = nz_;
  D_.X = X;
  D_.Y = Y;
  D_.Z = Z;
  D_.XY = (int64_t)X * Y;
  D_.G = G_;
  const double* mp = d_metric_;
  D_.rdxe = mp;
  D_.rdxc = mp + X;
  D_.rdye = mp + 2 * X;
  D_.rdyc = mp + 2 * X + Y;
  D_.rdze = mp + 2 * X + 2 * Y;
  D_.rdzc = mp + 2 * X + 2 * Y + Z;
  D_.dze = mp + 2 * X + 2 * Y + 2 * Z;
  D_.dzc = mp + 2 * X + 2 * Y + 3 * Z;
  D_.rz = d_prof_;
  D_.bgz = d_prof_ + Z;
  D_.u = d_fields_[0];
  D_.v = d_fields_[1];
  D_.w = d_fields_[2];
  D_.p = d_fields_[3];
  D_.rho = d_fields_[4];
  D_.s = d_fields_[5];
  D_.qu = d_fields_[8];
  D_.qv = d_fields_[9];
  D_.qw = d_fields_[10];
  D_.qr = d_fields_[11];
  D_.qs = d_fields_[12];
  D_.psrc = d_fields_[13];
  D_.nuT = d_fields_[14];
  D_.kT = d_fields_[15];
  D_.nT = d_fields_[16];
  D_.Cs = d_les_;
  D_.CTs = d_les_ ? d_les_ + Z : nullptr;
  D_.CSs = d_les_ ? d_les_ + 2 * Z : nullptr;
  D_.delg2 = d_les_ ? d_les_ + 3 * Z : nullptr;
  D_.rRe = rRe_;
  D_.rPr = rPr_;
  D_.rSc = rSc_;
  D_.g = gnow_;
  D_.vles = ns->vmodel != ANEL_MODEL_DNS;
  D_.rles = ns->rmodel != ANEL_MODEL_DNS;
  D_.sles = ns->smodel != ANEL_MODEL_DNS;
  D_.ew = ns->ew;
  D_.scal1_on = ns->scal1_on;
  // r = densityBG = 1 until set
  rz_.assign(Z, 1.0);
  bgz_.assign(Z, 1.0);
  // full r / densityBG arrays kept for get_fields
  for (int q : {6, 7}) {
    ANEL_CUDA_TRY(cudaMalloc(&d_fields_[q], G_ * sizeof(double)));
    std::vector<double> one(G_, 1.0);
    ANEL_CUDA_TRY(cudaMemcpy(d_fields_[q], one.data(), G_ * sizeof(double), cudaMemcpyHostToDevice));
  }
  const int ps = upload_profiles();
  if (ps != ANEL_OK) return ps;
  return tune_cn();
}

// Autotuning of the DNS column solve: every launch variant of launch_cn
// timed with CUDA events on this context's own u and q (all zero at this
// point; the factors of a placeholder rkdt are dropped afterwards), the
// fastest kept per (device, grid) for the process.  The variants compute
// the same bits.
int NSSolver::tune_cn() {
  // one kernel's variants: forced by the environment variable (no timing;
  // for tests), looked up in the registry, or timed here on this
  // context's own u and q (all zero at this point; the factors of a
  // placeholder rkdt are dropped afterwards)
  bool timed = false;
  auto pick = [&](const char* name, int nvar, const char* env, auto run, int* out) -> int {
    const char* force = std::getenv(env);
    if (force && *force) {
      const int v = std::atoi(force);
      if (v < 0 || v >= nvar) {
        set_error("%s=%s: variants are 0..%d", env, force, nvar - 1);
        return ANEL_ERR_ARG;
      }
      *out = v;
      return ANEL_OK;
    }
    char key[128];
    std::snprintf(key, sizeof(key), "%s dev%d %dx%dx%d", name, device_, nx_, ny_, nz_);
    int v = tune_lookup(key);
    if (v < 0 && !tune_enabled()) v = 0;
    if (v < 0) {
      constexpr int kReps = 3;
      if (!timed) {
        const int st = cn_factors(0, 1e-3, stream_);
        if (st != ANEL_OK) return st;
        timed = true;
      }
      std::vector<double> ms(nvar, 0.0);
      for (int q = 0; q < nvar; ++q) {
        run(q);
        ANEL_CUDA_TRY(cudaEventRecord(ev0_, stream_));
        for (int r = 0; r < kReps; ++r) run(q);
        ANEL_CUDA_TRY(cudaEventRecord(ev1_, stream_));
        ANEL_CUDA_TRY(cudaEventSynchronize(ev1_));
        float t = 0.f;
        ANEL_CUDA_TRY(cudaEventElapsedTime(&t, ev0_, ev1_));
        ms[q] = t / kReps;
      }
      const int le = check_launch("column solve tuning");
      if (le != ANEL_OK) return le;
      v = 0;
      for (int q = 1; q < nvar; ++q)
        if (ms[q] < ms[v]) v = q;
      tune_store(key, v, ms);
    }
    *out = v;
    return ANEL_OK;
  };
  const ZRule R = zrule(NV_U);
  int st = pick("k_cn_column", kCNVariants, "ANEL_CN_VARIANT", [&](int q) {
    launch_cn(D_, 1, D_.u, D_.qu, fac(0, 0), 1.0 / 3.0, 1e-3, R, q, stream_);
  }, &cnvar_);
  if (st == ANEL_OK && D_.vles)
    st = pick("k_cn_column_les", kCNLesVariants, "ANEL_CN_LES_VARIANT", [&](int q) {
      launch_cn_les(D_, 1, D_.u, D_.qu, fac(0, 0), 1.0 / 3.0, 1e-3, R, D_.nuT, d_cnb_, q, stream_);
    }, &cnlesvar_);
  if (st != ANEL_OK) return st;
  if (timed) {
    // back to the state of a fresh context
    ANEL_CUDA_TRY(cudaMemsetAsync(D_.u, 0, G_ * sizeof(double), stream_));
    ANEL_CUDA_TRY(cudaStreamSynchronize(stream_));
    cn_rkdt_[0] = -1.0;
  }
  return ANEL_OK;
}

int NSSolver::upload_profiles() {
  D_.unit_r = 1;
  for (int k = 0; k < (int)rz_.size(); ++k)
    if (!(rz_[k] == 1.0 && bgz_[k] == 1.0)) D_.unit_r = 0;
  std::vector<double> pr(rz_);
  pr.insert(pr.end(), bgz_.begin(), bgz_.end());
  ANEL_CUDA_TRY(cudaMemcpy(d_prof_, pr.data(), pr.size() * sizeof(double), cudaMemcpyHostToDevice));
  for (double& v : cn_rkdt_) v = -1.0;  // factors depend on r
  return ANEL_OK;
}

// vtype -> z rule (ghost/bound_update, BC.F90:67-95 and 334-420)
ZRule NSSolver::zrule(int vt) const {
  ZRule R{};
  int l = 7, stag = 0;
  switch (vt) {
    case NV_U: l = 1; stag = 1; break;
    case NV_V: l = 2; stag = 2; break;
    case NV_W: l = 3; stag = 3; break;
    case NV_P: l = 4; break;
    case NV_RHO: l = 5; R.rt = 1; break;
    case NV_CFLUC: l = 6; break;
    case NV_SCAL1: l = 8; R.rt = 1; break;
    case NV_SCAL1TEMP: l = 8; break;
    default: l = 7; stag = (vt == NV_UTEMP) ? 1 : (vt == NV_VTEMP) ? 2 : (vt == NV_WTEMP) ? 3 : 0;
  }
  for (int f = 0; f < 2; ++f) {
    R.type[f] = prm_.tb[2][f][l - 1];
    R.val[f] = prm_.vb[2][f][l - 1];
  }
  if (stag == 0) {
    R.of1 = -1;
    R.of2 = 0;
    R.dzt_is_zc = 0;
  } else {
    R.of1 = 0;
    R.of2 = 1;
    R.dzt_is_zc = (stag == 3) ? 1 : 0;
  }
  R.iw = (stag == 3) ? prm_.ew : 0;
  return R;
}

// Column-independent factors of the CN system of each variable for one
// rkdt (var_advance_CN_PL, NSsolver.F90:3102-3296), then the elimination
// of the Thomas routine (mg_relax.F90:563-568) applied to them.
int NSSolver::cn_factors(int slot, double rkdt, cudaStream_t s) {
  if (cn_rkdt_[slot] == rkdt) return ANEL_OK;
  // the pinned staging slot may still feed an earlier asynchronous copy
  ANEL_CUDA_TRY(cudaStreamSynchronize(s));
  const int Z = nz_ + 2, n = Z, sz = 2, ez = nz_ + 1;
  const double H = 0.5;
  auto R = [&](int k) { return rz_[k - 1]; };
  auto rdze = [&](int k) { return m_[2][4][k - 1]; };
  auto rdzc = [&](int k) { return m_[2][5][k - 1]; };
  auto dze = [&](int k) { return m_[2][2][k - 1]; };
  auto dzc = [&](int k) { return m_[2][3][k - 1]; };
  for (int vi = 0; vi < 5; ++vi) {
    const int var = kVarCode[vi];
    double* base = h_cn_ + ((size_t)(slot * 5 + vi) * 9) * Z;
    double *ap = base, *bp = base + Z, *c = base + 2 * Z, *t1a = base + 3 * Z, *t2a = base + 4 * Z,
           *rb = base + 5 * Z, *isbc = base + 6 * Z, *suba = base + 7 * Z, *diaga = base + 8 * Z;
    std::vector<double> sub(n, 0.0), diag(n, 0.0), sup(n, 0.0);
    for (int q = 0; q < n; ++q) {
      t1a[q] = t2a[q] = rb[q] = isbc[q] = 0.0;
    }
    for (int k = sz; k <= ez; ++k) {
      double t1, t2;
      if (var != 3) {
        const double ra1 = H * (R(k + 1) + R(k));
        const double ra2 = H * (R(k) + R(k - 1));
        if (var == 1 || var == 2) {
          t1 = (rRe_ + 0.0) * ra1 / R(k);
          t2 = (rRe_ + 0.0) * ra2 / R(k);
        } else if (var == 5) {
          t1 = (rRe_ * rPr_ + 0.0) * ra1 / R(k);
          t2 = (rRe_ * rPr_ + 0.0) * ra2 / R(k);
        } else {
          t1 = rRe_ * rSc_ + 0.0;
          t2 = rRe_ * rSc_ + 0.0;
        }
        sub[k - 1] = -0.5 * rkdt * t1 * rdze(k - 1) * rdzc(k);
        sup[k - 1] = -0.5 * rkdt * t2 * rdze(k) * rdzc(k);
        diag[k - 1] = 1.0 + 0.5 * rkdt * (t1 * rdze(k - 1) + t2 * rdze(k)) * rdzc(k);
      } else {
        t1 = (rRe_ + 0.0) * R(k) / (H * (R(k + 1) + R(k)));
        t2 = (rRe_ + 0.0) * R(k + 1) / (H * (R(k + 1) + R(k)));
        sub[k - 1] = -0.5 * rkdt * t1 * rdze(k) * rdzc(k);
        sup[k - 1] = -0.5 * rkdt * t2 * rdze(k) * rdzc(k + 1);
        diag[k - 1] = 1.0 + 0.5 * rkdt * (t1 * rdzc(k) + t2 * rdzc(k + 1)) * rdze(k);
      }
      t1a[k - 1] = t1;
      t2a[k - 1] = t2;
    }
    // wall rows (NSsolver.F90:3297-3429)
    const int tbmin = prm_.tb[2][0][var - 1], tbmax = prm_.tb[2][1][var - 1];
    const double vbmin = prm_.vb[2][0][var - 1], vbmax = prm_.vb[2][1][var - 1];
    auto set = [&](int k, double a, double b, double cc, double d) {
      sub[k - 1] = a;
      diag[k - 1] = b;
      sup[k - 1] = cc;
      rb[k - 1] = d;
      isbc[k - 1] = 1.0;
    };
    if (tbmin == 1) set(sz - 1, 0.0, 1.0, 0.0, vbmin);
    else if (tbmin == 2) {
      if (var == 3) set(sz - 1, 0.0, -1.0, 1.0, dzc(sz - 1) * vbmin);
      else if (var == 5 || var == 8) {
        set(sz - 1, 0.0, -1.0, 1.0, dze(sz - 1) * vbmin);
        set(sz, 0.0, -1.0, 1.0, dze(sz) * vbmin);
      } else set(sz - 1, 0.0, -1.0, 1.0, dze(sz - 1) * vbmin);
    } else if (tbmin == 6) set(sz - 1, 0.0, 1.0, 1.0, 2.0 * vbmin);
    if (tbmax == 1) set(ez + 1, 0.0, 1.0, 0.0, vbmax);
    else if (tbmax == 2) {
      if (var == 3) set(ez + 1, -1.0, 1.0, 0.0, dzc(ez + 1) * vbmax);
      else if (var == 5 || var == 8) {
        set(ez + 1, -1.0, 1.0, 0.0, dze(ez + 1) * vbmax);
        set(ez, -1.0, 1.0, 0.0, dze(ez) * vbmax);
      } else set(ez + 1, -1.0, 1.0, 0.0, dze(ez + 1) * vbmax);
    } else if (tbmax == 6) set(ez + 1, 1.0, 1.0, 0.0, 2.0 * vbmax);
    else if (tbmax == 7) {
      set(ez + 1, 0.0, 1.0, 0.0, 0.0);
      set(ez, 0.0, 1.0, 0.0, 0.0);
    }
    // elimination (a, b overwritten, c untouched)
    std::vector<double> a(sub), b(diag);
    for (int j = 1; j <= n - 1; ++j) {
      a[j] = -a[j] / b[j - 1];
      b[j] = b[j] + a[j] * sup[j - 1];
    }
    for (int q = 0; q < n; ++q) {
      ap[q] = (q == 0) ? 0.0 : a[q];
      bp[q] = b[q];
      c[q] = sup[q];
      suba[q] = sub[q];
      diaga[q] = diag[q];
    }
  }
  double* dst = d_cn_ + (size_t)slot * 5 * 9 * Z;
  // by a kernel from the mapped staging slot: a copy-engine upload would
  // queue behind large uploads other streams have in flight
  copy_words(h_cn_ + (size_t)slot * 5 * 9 * Z, dst, 5 * 9 * (int64_t)Z, s);
  cn_rkdt_[slot] = rkdt;
  return ANEL_OK;
}

CNFacHost NSSolver::fac(int slot, int vi) const {
  const int Z = nz_ + 2;
  const double* base = d_cn_ + ((size_t)(slot * 5 + vi) * 9) * Z;
  return CNFacHost{base,         base + Z,     base + 2 * Z, base + 3 * Z, base + 4 * Z,
                   base + 5 * Z, base + 6 * Z, base + 7 * Z, base + 8 * Z};
}

// --------------------------------------------------------------- fields
int NSSolver::set_fields(const anel_fields* f, int mem, cudaStream_t s) {
  if (!f) return ANEL_ERR_ARG;
  ANEL_CUDA_TRY(cudaSetDevice(device_));
  if (!s) s = stream_;
  double* const* src = reinterpret_cast<double* const*>(f);
  const cudaMemcpyKind kind = mem == ANEL_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  bool density = false;
  fields_changed();
  for (int q = 0; q < 17; ++q) {
    if (!src[q] || !d_fields_[q]) continue;  // LES fields exist only with a subgrid model
    ANEL_CUDA_TRY(cudaMemcpyAsync(d_fields_[q], src[q], G_ * sizeof(double), kind, s));
    if (q == 6 || q == 7) density = true;
    if (q >= 8 && q <= 12) temps_clean_ = false;
  }
  if (density) {
    // profiles of r and densityBG: both must be functions of z only
    std::vector<double> h(G_);
    const int64_t XY = (int64_t)(nx_ + 2) * (ny_ + 2);
    for (int q : {6, 7}) {
      if (!src[q]) continue;
      ANEL_CUDA_TRY(cudaMemcpyAsync(h.data(), d_fields_[q], G_ * sizeof(double), cudaMemcpyDeviceToHost, s));
      ANEL_CUDA_TRY(cudaStreamSynchronize(s));
      std::vector<double>& prof = (q == 6) ? rz_ : bgz_;
      for (int k = 0; k < nz_ + 2; ++k) {
        const double v = h[(int64_t)k * XY];
        for (int64_t o = 1; o < XY; ++o)
          if (!(h[(int64_t)k * XY + o] == v)) {
            set_error("%s must be horizontally uniform (a function of z); plane k=%d differs",
                      q == 6 ? "r" : "densityBG", k + 1);
            return ANEL_ERR_UNSUPPORTED;
          }
        prof[k] = v;
      }
      if (q == 6) {
        const int st = mg_->set_density_host(h.data());
        if (st != ANEL_OK) return st;
      }
    }
    const int st = upload_profiles();
    if (st != ANEL_OK) return st;
  }
  ANEL_CUDA_TRY(cudaStreamSynchronize(s));
  return ANEL_OK;
}

int NSSolver::get_fields(const anel_fields* f, int mem, cudaStream_t s) {
  if (!f) return ANEL_ERR_ARG;
  ANEL_CUDA_TRY(cudaSetDevice(device_));
  if (!s) s = stream_;
  double* const* dst = reinterpret_cast<double* const*>(f);
  const cudaMemcpyKind kind = mem == ANEL_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  for (int q = 0; q < 17; ++q)
    if (dst[q] && d_fields_[q])
      ANEL_CUDA_TRY(cudaMemcpyAsync(dst[q], d_fields_[q], G_ * sizeof(double), kind, s));
  ANEL_CUDA_TRY(cudaStreamSynchronize(s));
  return ANEL_OK;
}

int NSSolver::ensure_hist() {
  if (hist_[0][0]) return ANEL_OK;
  for (auto& h : hist_)
    for (double*& a : h) {
      ANEL_CUDA_TRY(cudaMalloc(&a, G_ * sizeof(double)));
      ANEL_CUDA_TRY(cudaMemset(a, 0, G_ * sizeof(double)));
    }
  return ANEL_OK;
}

// --------------------------------------------------------------- rk_ss
// rk_ss (NSsolver.F90:418-583) in two halves around the pressure solve:
// RHS, Crank-Nicolson columns and Psource, then (after the solve) Pgrad.
int NSSolver::substep_pre(double a1, double a2, double a3, double dt_rk, double dt, cudaStream_t s,
                          bool q_zero) {
  // slot of the factor cache (three rkdt values per step)
  int slot = -1;
  for (int q = 0; q < 3; ++q)
    if (cn_rkdt_[q] == dt_rk) slot = q;
  if (slot < 0) {
    slot = cn_next_;
    cn_next_ = (cn_next_ + 1) % 3;
    const int st = cn_factors(slot, dt_rk, s);
    if (st != ANEL_OK) return st;
  }
  D_.g = gnow_;
  launch_rhs_accum(D_, a1, a2, dt, q_zero && a1 == 0.0, s);
  const ZRule ru = zrule(NV_U), rv = zrule(NV_V), rw = zrule(NV_W);
  // var_advance_CN_PL: with Vmodel = SSM every variable gets the eddy
  // terms (the LES block is gated on Vmodel, NSsolver.F90:3160-3190)
  auto cn = [&](int var, double* f, const double* q, int vi, const ZRule& R, const double* kT, cudaStream_t st) {
    if (D_.vles) launch_cn_les(D_, var, f, q, fac(slot, vi), a3, dt_rk, R, kT, d_cnb_, cnlesvar_, st);
    else launch_cn(D_, var, f, q, fac(slot, vi), a3, dt_rk, R, cnvar_, st);
  };
  cn(1, D_.u, D_.qu, 0, ru, D_.nuT, s);
  cn(2, D_.v, D_.qv, 1, rv, D_.nuT, s);
  cn(3, D_.w, D_.qw, 2, rw, D_.nuT, s);
  launch_psource(D_, dt_rk, s);
  if (prm_.pguess && cur_sub_ >= 0 && nhist_[cur_sub_] >= 2) {
    const int q = cur_sub_;
    launch_extrap(D_, D_.p, hist_[q][last_[q]], hist_[q][last_[q] ^ 1], s);
  }
  cn(5, D_.rho, D_.qr, 3, zrule(NV_RHO), D_.kT, s);
  if (prm_.scal1_on) cn(8, D_.s, D_.qs, 4, zrule(NV_SCAL1), D_.nT, s);
  const size_t fb = G_ * sizeof(double);
  if (io_last_sub_ && io_out_) {
    // rho and scal1 are final: copy them out during the pressure solve
    ANEL_CUDA_TRY(cudaEventRecord(io_ev_[1], s));
    ANEL_CUDA_TRY(cudaStreamWaitEvent(io_stream_, io_ev_[1], 0));
    if (io_out_->rho) ANEL_CUDA_TRY(cudaMemcpyAsync(io_out_->rho, D_.rho, fb, cudaMemcpyDeviceToHost, io_stream_));
    if (io_out_->scal1)
      ANEL_CUDA_TRY(cudaMemcpyAsync(io_out_->scal1, D_.s, fb, cudaMemcpyDeviceToHost, io_stream_));
  }
  if (io_wait_p_) {  // p (the solve's initial guess) arrives on the copy stream
    ANEL_CUDA_TRY(cudaStreamWaitEvent(s, io_ev_[0], 0));
    io_wait_p_ = false;
  }
  pend_dtrk_ = dt_rk;
  return ANEL_OK;
}

int NSSolver::substep_post(const anel_mg_report& rep, cudaStream_t s, int* iters, double* relmax) {
  if (io_last_sub_ && io_out_ && io_out_->p) {  // p is final: copy it out during Pgrad
    ANEL_CUDA_TRY(cudaEventRecord(io_ev_[2], s));
    ANEL_CUDA_TRY(cudaStreamWaitEvent(io_stream_, io_ev_[2], 0));
    ANEL_CUDA_TRY(cudaMemcpyAsync(io_out_->p, D_.p, G_ * sizeof(double), cudaMemcpyDeviceToHost, io_stream_));
  }
  acc_mg_ms_ += rep.ms;
  acc_sweep_ms_ += rep.fine_sweep_ms;
  acc_sweeps_ += rep.fine_sweeps;
  double* hist = nullptr;
  if (prm_.pguess && cur_sub_ >= 0) {
    const int st = ensure_hist();
    if (st != ANEL_OK) return st;
    const int q = cur_sub_;
    last_[q] ^= 1;  // the older buffer takes this solution
    hist = hist_[q][last_[q]];
    nhist_[q] = nhist_[q] < 2 ? nhist_[q] + 1 : 2;
  }
  launch_pgrad(D_, pend_dtrk_, zrule(NV_U), zrule(NV_V), zrule(NV_W), s, hist);
  fields_changed();
  if (iters) *iters = rep.iter;
  if (relmax) *relmax = rep.relmax;
  return check_launch("rk substep");
}

int NSSolver::substep(double a1, double a2, double a3, double dt_rk, double dt, cudaStream_t s,
                      int* iters, double* relmax, bool q_zero) {
  ANEL_CUDA_TRY(cudaSetDevice(device_));
  if (!s) s = stream_;
  int st = substep_pre(a1, a2, a3, dt_rk, dt, s, q_zero);
  if (st != ANEL_OK) return st;
  anel_mg_report rep{};
  st = mg_->solve_device(D_.p, D_.psrc, s, &rep);
  if (st != ANEL_OK && st != ANEL_ERR_NOCONV) return st;
  return substep_post(rep, s, iters, relmax);
}

int NSSolver::reset(const anel_ns_params* ns, cudaStream_t s) {
  ANEL_CUDA_TRY(cudaSetDevice(device_));
  if (!s) s = stream_;
  const bool les = ns->vmodel != ANEL_MODEL_DNS || ns->rmodel != ANEL_MODEL_DNS ||
                   ns->smodel != ANEL_MODEL_DNS;
  const bool dyn = ns->vmodel == ANEL_MODEL_DSM || ns->rmodel == ANEL_MODEL_DSM || ns->smodel == ANEL_MODEL_DSM;
  if (les != les_any_ || (ns->vmodel != ANEL_MODEL_DNS) != (D_.vles != 0) || ns->ew != prm_.ew ||
      (dyn && (ns->test_ratio != prm_.test_ratio || std::memcmp(ns->filt, prm_.filt, sizeof(prm_.filt)) != 0 ||
               std::memcmp(ns->stretched, prm_.stretched, sizeof(prm_.stretched)) != 0 ||
               ns->interp != prm_.interp)) ||
      std::memcmp(ns->tb, prm_.tb, sizeof(prm_.tb)) != 0 ||
      std::memcmp(ns->vb, prm_.vb, sizeof(prm_.vb)) != 0) {
    set_error("reset: models, edge-node flag and boundary conditions must match the context");
    return ANEL_ERR_ARG;
  }
  if (check_clip(ns) != ANEL_OK) return ANEL_ERR_ARG;
  prm_ = *ns;
  temps_clean_ = false;
  fields_changed();
  for (int q = 0; q < 3; ++q) nhist_[q] = 0;
  rRe_ = 1.0 / ns->Re;
  rPr_ = 1.0 / ns->Pr;
  rSc_ = 1.0 / ns->Sc;
  g_orig_ = ns->g_final;
  gnow_ = ns->g_init;
  D_.rRe = rRe_;
  D_.rPr = rPr_;
  D_.rSc = rSc_;
  D_.g = gnow_;
  D_.rles = ns->rmodel != ANEL_MODEL_DNS;
  D_.sles = ns->smodel != ANEL_MODEL_DNS;
  D_.scal1_on = ns->scal1_on;
  for (double& r : cn_rkdt_) r = -1.0;  // the CN factors depend on Re, Pr, Sc
  time_ = 0.0;
  told_ = 1.0e-16;
  nstep_ = 1;
  if (d_diag_) ANEL_CUDA_TRY(cudaMemsetAsync(d_diag_, 0, 26 * (size_t)(nz_ + 2) * sizeof(double), s));
  for (int q = 8; q < 17; ++q)
    if (d_fields_[q]) ANEL_CUDA_TRY(cudaMemsetAsync(d_fields_[q], 0, G_ * sizeof(double), s));
  if (d_les_) ANEL_CUDA_TRY(cudaMemsetAsync(d_les_, 0, 4 * (size_t)(nz_ + 2) * sizeof(double), s));
  les_coeffs_done_ = false;
  return ANEL_OK;
}

int NSSolver::init_shear(uint32_t seed, double amp, double zmax, cudaStream_t s) {
  ANEL_CUDA_TRY(cudaSetDevice(device_));
  if (!s) s = stream_;
  fields_changed();
  const int Z = nz_ + 2;
  if (!d_ic_) ANEL_CUDA_TRY(cudaMalloc(&d_ic_, 2 * (size_t)Z * sizeof(double)));
  std::vector<double> prof(2 * (size_t)Z);
  for (int k = 0; k < Z; ++k) {
    prof[k] = std::tanh(m_[2][1][k]);
    prof[Z + k] = std::fabs(m_[2][1][k]);
  }
  ANEL_CUDA_TRY(cudaMemcpyAsync(d_ic_, prof.data(), prof.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  launch_init_shear(D_, d_ic_, seed, amp, zmax, s);
  ANEL_CUDA_TRY(cudaStreamSynchronize(s));  // prof lives on the host stack
  return check_launch("init_shear");
}

// les_coeffs: the filter width delg (straincal.F90:126-134) and the
// model coefficients Csgs, CTsgs, CSsgs (SSM.F90:27,60,97) are functions of
// the grid only; with uniform x/y spacing they depend on k alone and are
// kept as profiles (evaluated on the host with the same libm as the
// reference's build).  Recomputed on the reference's cadence; the values do
// not change between calls.
int NSSolver::les_coeffs(cudaStream_t s) {
  if (les_coeffs_done_) return ANEL_OK;
  const bool dyn = prm_.vmodel == ANEL_MODEL_DSM || prm_.rmodel == ANEL_MODEL_DSM || prm_.smodel == ANEL_MODEL_DSM;
  const int Z = nz_ + 2;
  std::vector<double> prof(4 * (size_t)Z, 0.0), damp_u(Z, 1.0), damp_t(Z, 1.0);
  const double dxc = m_[0][3][1], dyc = m_[1][3][1];
  const double c = prm_.ssm_const;
  for (int k = 2; k <= nz_ + 1; ++k) {
    const double dzc = m_[2][3][k - 1];
    double dg;
    if (prm_.les_delta == ANEL_DELTA_3ROOT) dg = std::pow(dxc * dyc * dzc, 1.0 / 3.0);
    else dg = std::pow(dxc * dxc + dyc * dyc + dzc * dzc, 1.0 / 2.0);
    if (prm_.les_damp == ANEL_DAMP_LITERAL) {
      // REAL(4) literals 0.41 and 0.3 (SSMrho); 0.3d0 in SSM
      const double k41 = (double)(float)0.41;
      const double zo_u = 0.3, zo_t = (double)(float)0.3;
      const double zc = m_[2][1][k - 1];
      const double a = k41 * (zc + zo_u);
      damp_u[k - 1] = (a * a) / ((a * a) + c * (dg * dg));
      const double b = k41 * (zc + zo_t);
      damp_t[k - 1] = (b * b) / ((b * b) + c * (dg * dg));
    }
    prof[k - 1] = c * damp_u[k - 1];
    prof[3 * (size_t)Z + k - 1] = dg * dg;
  }
  // the driver's order (NSsolver.F90:83-130): the velocity model's Csgs,
  // then SSMrho / SSMscal1 from that Csgs, or their dynamic forms
  std::vector<double> dynp(Z, 0.0);
  int st = ANEL_OK;
  dyn_ready_ = false;  // the models of this update share one dyn_prepare
  if (prm_.vmodel == ANEL_MODEL_DSM) {
    if ((st = dsm_velocity(s, dynp.data())) != ANEL_OK) return st;
    for (int k = 2; k <= nz_ + 1; ++k) prof[k - 1] = dynp[k - 1];
  }
  for (int q = 0; q < 2; ++q) {
    const int model = q == 0 ? prm_.rmodel : prm_.smodel;
    double* dst = prof.data() + (size_t)(q + 1) * Z;
    if (model == ANEL_MODEL_DSM) {
      const double* field = q == 0 ? D_.rho : D_.s;
      if ((st = dsm_scalar(field, s, dynp.data())) != ANEL_OK) return st;
      for (int k = 2; k <= nz_ + 1; ++k) dst[k - 1] = dynp[k - 1];
    } else {
      const std::vector<double>& dmp = q == 0 ? damp_t : damp_u;
      for (int k = 2; k <= nz_ + 1; ++k) dst[k - 1] = prof[k - 1] / prm_.pr_sgs * dmp[k - 1];
    }
  }
  ANEL_CUDA_TRY(cudaMemcpyAsync(d_les_, prof.data(), prof.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  ANEL_CUDA_TRY(cudaStreamSynchronize(s));
  les_coeffs_done_ = !dyn;  // the dynamic coefficients follow the fields
  return ANEL_OK;
}

// calcdt (Routines.F90:186-258) in two halves: the CFL maximum to the
// host-mapped word (issue), then, after the stream is synchronised, the
// time step from it (take)
void NSSolver::calcdt_issue(cudaStream_t s) {
  if (cfl_ready_) {
    // the previous step's divergence pass took it from these fields
    copy_words(d_red_ + 2, h_red_, 1, s);
    cfl_ready_ = false;
  } else {
    cudaMemsetAsync(d_red_, 0, sizeof(unsigned long long), s);
    launch_cfl_max(D_, d_red_, s);
    copy_words(d_red_, h_red_, 1, s);
  }
}

double NSSolver::calcdt_take() const {
  double dt = prm_.cfl / h_red_[0];
  if (dt >= prm_.dtmax) dt = prm_.dtmax;
  return dt;
}

double NSSolver::calcdt(cudaStream_t s, int* st) {
  calcdt_issue(s);
  if (cudaStreamSynchronize(s) != cudaSuccess) {
    *st = ANEL_ERR_CUDA;
    return 0.0;
  }
  *st = ANEL_OK;
  return calcdt_take();
}

// The driver's optional clip after each rk_ss (NSsolver.F90:206-211,
// 235-240, 264-269): clipVS of rho, its ghost pass, clipVS of scal1, its
// ghost pass.
void NSSolver::clip_scalars(cudaStream_t s) {
  if (!prm_.clip) return;
  launch_clip(D_, D_.rho, prm_.rho_min, prm_.rho_max, s);
  launch_ghost_field(D_, D_.rho, zrule(NV_RHO), s);
  launch_clip(D_, D_.s, prm_.scal1_min, prm_.scal1_max, s);
  launch_ghost_field(D_, D_.s, zrule(NV_SCAL1), s);
}

static const double kA1[3] = {0.0, -5.0 / 9.0, -153.0 / 128.0};
static const double kA3[3] = {1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0};

// Start of a step (NSsolver.F90:63-164): zero_temps, calcdt, gravity, the
// LES coefficients on their cadence and the scalar smoothing.
int NSSolver::step_begin(cudaStream_t s, double* delt_out) {
  step_begin_issue(s);
  ANEL_CUDA_TRY(cudaStreamSynchronize(s));
  return step_begin_finish(s, delt_out);
}

void NSSolver::step_begin_issue(cudaStream_t s) {
  // zero_temps (memManage.F90:844-853).  The accumulators q_u, q_v,
  // q_w, q_rho, q_s are written, never read, by the first sub-step
  // (a1 = 0) on every interior cell, and no kernel writes their ghost
  // cells, so once zeroed they need no zeroing again until set_fields,
  // reset or a scratch use touches them (temps_clean_); the Poisson
  // right-hand side is zeroed every step.
  for (int q : {8, 9, 10, 11, 12, 13})
    if (q == 13 || !temps_clean_) cudaMemsetAsync(d_fields_[q], 0, G_ * sizeof(double), s);
  temps_clean_ = true;
  calcdt_issue(s);
}

// (after step_begin_issue and a synchronisation of its stream)
int NSSolver::step_begin_finish(cudaStream_t s, double* delt_out) {
  int st = check_launch("step start");
  if (st != ANEL_OK) return st;
  const double delt = calcdt_take();
  // gravity (Routines.F90:27-52)
  if (time_ < prm_.gt1) gnow_ = 0.0;
  else if (time_ > prm_.gt1 && time_ < prm_.gt2) gnow_ = g_orig_ * (time_ - prm_.gt1) / (prm_.gt2 - prm_.gt1);
  else if (time_ >= prm_.gt2) gnow_ = g_orig_;
  // LES model coefficients and eddy viscosities (NSsolver.F90:86-100):
  // les_coeffs on the step cadence, SGSdiff before every sub-step
  const bool les = D_.vles != 0;
  if (les && nstep_ >= prm_.les_start && nstep_ % prm_.les_freq == 0) {
    st = les_coeffs(s);
    if (st != ANEL_OK) return st;
  }
  // the scalar models' smoothing of rho and scal1 every 50 steps
  // (NSsolver.F90:144-164), after the coefficients, before SGSdiff
  if (time_ > 0.0 && nstep_ % 50 == 0 && (D_.rles || D_.sles)) {
    st = smooth_scalars(s);
    if (st != ANEL_OK) return st;
  }
  *delt_out = delt;
  return ANEL_OK;
}

// End of a step: the clock (NSsolver.F90:272-274) and the diagnostics.
int NSSolver::step_end(double delt, cudaStream_t s, anel_step_report* r) {
  told_ = time_;  // told = time; time = time + delt
  time_ = time_ + delt;
  if (diag_on_) {
    int st = ensure_diag();
    if (st != ANEL_OK) return st;
    ANEL_CUDA_TRY(cudaEventRecord(dev0_, s));
    st = compute_diagnostics(s);
    if (st != ANEL_OK) return st;
    ANEL_CUDA_TRY(cudaEventRecord(dev1_, s));
    ANEL_CUDA_TRY(cudaEventSynchronize(dev1_));
    float dms = 0.f;
    cudaEventElapsedTime(&dms, dev0_, dev1_);
    acc_diag_ms_ += dms;
  }
  r->nstep = nstep_;
  r->dt = delt;
  r->time = time_;
  nstep_ += 1;
  // divergence of the step's result and the next step's CFL maximum
  const int st = divergence_pass(s, true);
  if (st != ANEL_OK) return st;
  cfl_ready_ = div_ready_ = true;
  return ANEL_OK;
}

// After the last step: accumulated times and the divergence check.
int NSSolver::step_finish(cudaStream_t s, int64_t launches0, anel_step_report* r) {
  r->mg_ms = acc_mg_ms_;
  r->fine_sweep_ms = acc_sweep_ms_;
  r->fine_sweeps = acc_sweeps_;
  r->diag_ms = acc_diag_ms_;
  r->launches = t_launches - launches0;
  double dv[2];
  const int st = div_ready_ ? divergence_read(s, dv) : divergence(s, dv);
  if (st != ANEL_OK) return st;
  r->avg_div = dv[0];
  r->max_div = dv[1];
  return ANEL_OK;
}

int NSSolver::step(int nsteps, cudaStream_t s, anel_step_report* rep) {
  ANEL_CUDA_TRY(cudaSetDevice(device_));
  if (!s) s = stream_;
  anel_step_report r{};
  acc_mg_ms_ = acc_sweep_ms_ = 0.0;
  acc_diag_ms_ = 0.0;
  acc_sweeps_ = 0;
  const int64_t launches0 = t_launches;
  ANEL_CUDA_TRY(cudaEventRecord(ev0_, s));
  for (int n = 0; n < nsteps; ++n) {
    double delt = 0.0;
    int st = step_begin(s, &delt);
    if (st != ANEL_OK) return st;
    const bool les = D_.vles != 0;
    const double DTR[3] = {1.0 / 3.0 * delt, 5.0 / 12.0 * delt, 1.0 / 4.0 * delt};
    for (int q = 0; q < 3; ++q) {
      if (les && nstep_ > prm_.les_start) launch_sgs(D_, zrule(NV_CFLUC), s);
      io_last_sub_ = io_out_ && n == nsteps - 1 && q == 2;
      cur_sub_ = q;
      st = substep(kA1[q], 1.0, kA3[q], DTR[q], delt, s, &r.mg_iter[q], &r.mg_relmax[q], true);
      cur_sub_ = -1;
      io_last_sub_ = false;
      if (st != ANEL_OK) return st;
      clip_scalars(s);
    }
    st = step_end(delt, s, &r);
    if (st != ANEL_OK) return st;
  }
  ANEL_CUDA_TRY(cudaEventRecord(ev1_, s));
  ANEL_CUDA_TRY(cudaEventSynchronize(ev1_));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ev0_, ev1_);
  r.ms = ms;
  const int st = step_finish(s, launches0, &r);
  if (st != ANEL_OK) return st;
  if (rep) *rep = r;
  return ANEL_OK;
}

int NSSolver::step_cohort(NSSolver* const* ms, int n, int nsteps, MGSolver* bmg, cudaStream_t s,
                          anel_step_report* reps) {
  if (n < 1 || !ms || !bmg || !reps) {
    set_error("step_cohort: n >= 1 members, a batch solver and reports required");
    return ANEL_ERR_ARG;
  }
  for (int b = 0; b < n; ++b) {
    NSSolver* m = ms[b];
    const anel_mg_params& a = m ? m->mg_->params() : bmg->params();
    const anel_mg_params& c = bmg->params();
    const bool same_mg = a.precision == c.precision && a.smoother == c.smoother && a.maxcy == c.maxcy &&
                         a.tolmax == c.tolmax && a.stop == c.stop && a.mode == c.mode &&
                         std::memcmp(a.pre_relax, c.pre_relax, sizeof(a.pre_relax)) == 0 &&
                         std::memcmp(a.post_relax, c.post_relax, sizeof(a.post_relax)) == 0 &&
                         std::memcmp(a.levels, c.levels, sizeof(a.levels)) == 0 &&
                         std::memcmp(a.tbc, c.tbc, sizeof(a.tbc)) == 0 &&
                         std::memcmp(a.vbc, c.vbc, sizeof(a.vbc)) == 0;
    if (!m || m->device_ != bmg->device() || m->nx_ != ms[0]->nx_ || m->ny_ != ms[0]->ny_ ||
        m->nz_ != ms[0]->nz_ || !same_mg || m->mg_->operator_hash() != bmg->operator_hash()) {
      set_error("step_cohort: member %d differs in grid, device, multigrid parameters or operator", b);
      return ANEL_ERR_ARG;
    }
    if (m->io_out_ || m->io_wait_p_) {
      set_error("step_cohort: member %d has a host copy pending", b);
      return ANEL_ERR_ARG;
    }
  }
  ANEL_CUDA_TRY(cudaSetDevice(bmg->device()));
  if (!s) s = bmg->stream();
  std::vector<anel_step_report> r(n);
  std::vector<int64_t> l0(n);
  std::vector<double> delt(n);
  std::vector<double*> phis(n);
  std::vector<const double*> rhss(n);
  std::vector<anel_mg_report> mrep(n);
  for (int b = 0; b < n; ++b) {
    NSSolver* m = ms[b];
    m->acc_mg_ms_ = m->acc_sweep_ms_ = m->acc_diag_ms_ = 0.0;
    m->acc_sweeps_ = 0;
    l0[b] = t_launches;
    phis[b] = m->D_.p;
    rhss[b] = m->D_.psrc;
  }
  ANEL_CUDA_TRY(cudaEventRecord(ms[0]->ev0_, s));
  for (int step = 0; step < nsteps; ++step) {
    // every member's time step with one synchronisation
    for (int b = 0; b < n; ++b) ms[b]->step_begin_issue(s);
    ANEL_CUDA_TRY(cudaStreamSynchronize(s));
    for (int b = 0; b < n; ++b) {
      const int st = ms[b]->step_begin_finish(s, &delt[b]);
      if (st != ANEL_OK) return st;
    }
    for (int q = 0; q < 3; ++q) {
      for (int b = 0; b < n; ++b) {
        NSSolver* m = ms[b];
        if (m->D_.vles && m->nstep_ > m->prm_.les_start) launch_sgs(m->D_, m->zrule(NV_CFLUC), s);
        const double DTR[3] = {1.0 / 3.0 * delt[b], 5.0 / 12.0 * delt[b], 1.0 / 4.0 * delt[b]};
        m->cur_sub_ = q;
        const int st = m->substep_pre(kA1[q], 1.0, kA3[q], DTR[q], delt[b], s, true);
        if (st != ANEL_OK) return st;
      }
      const int sb = bmg->solve_batch(n, phis.data(), rhss.data(), s, mrep.data());
      if (sb != ANEL_OK && sb != ANEL_ERR_NOCONV) return sb;
      for (int b = 0; b < n; ++b) {
        mrep[b].ms /= n;  // the batch's device time, shared out
        const int st = ms[b]->substep_post(mrep[b], s, &r[b].mg_iter[q], &r[b].mg_relmax[q]);
        ms[b]->cur_sub_ = -1;
        if (st != ANEL_OK) return st;
        ms[b]->clip_scalars(s);
      }
    }
    for (int b = 0; b < n; ++b) {
      const int st = ms[b]->step_end(delt[b], s, &r[b]);
      if (st != ANEL_OK) return st;
    }
  }
  ANEL_CUDA_TRY(cudaEventRecord(ms[0]->ev1_, s));
  ANEL_CUDA_TRY(cudaEventSynchronize(ms[0]->ev1_));
  float tms = 0.f;
  cudaEventElapsedTime(&tms, ms[0]->ev0_, ms[0]->ev1_);
  // the divergence of every member's last step (step_end's passes), with
  // one synchronisation
  for (int b = 0; b < n; ++b) ms[b]->divergence_issue(s);
  ANEL_CUDA_TRY(cudaStreamSynchronize(s));
  for (int b = 0; b < n; ++b) {
    NSSolver* m = ms[b];
    anel_step_report& rb = r[b];
    rb.ms = tms;
    rb.mg_ms = m->acc_mg_ms_;
    rb.fine_sweep_ms = m->acc_sweep_ms_;
    rb.fine_sweeps = m->acc_sweeps_;
    rb.diag_ms = m->acc_diag_ms_;
    rb.launches = t_launches - l0[b];
    double dv[2] = {0.0, 0.0};
    if (nsteps > 0) {
      const int st = m->divergence_take(dv);
      if (st != ANEL_OK) return st;
    } else {
      const int st = m->divergence(s, dv);
      if (st != ANEL_OK) return st;
    }
    rb.avg_div = dv[0];
    rb.max_div = dv[1];
    reps[b] = rb;
  }
  return ANEL_OK;
}

int NSSolver::ghost_state(cudaStream_t s) {
  ANEL_CUDA_TRY(cudaSetDevice(device_));
  if (!s) s = stream_;
  fields_changed();
  double* f[6] = {D_.u, D_.v, D_.w, D_.p, D_.rho, D_.s};
  const int vt[6] = {NV_U, NV_V, NV_W, NV_P, NV_RHO, NV_SCAL1};
  for (int q = 0; q < 6; ++q)
    if (f[q]) launch_ghost_field(D_, f[q], zrule(vt[q]), s);
  ANEL_CUDA_TRY(cudaStreamSynchronize(s));
  return ANEL_OK;
}

// --------------------------------------------------- plane statistics
int NSSolver::set_diagnostics(int on, int mode, const int* stretched) {
  if (mode != ANEL_DIAG_LITERAL && mode != ANEL_DIAG_CORRECTED) {
    set_error("diagnostics mode must be ANEL_DIAG_LITERAL or ANEL_DIAG_CORRECTED");
    return ANEL_ERR_ARG;
  }
  const int n[3] = {nx_, ny_, nz_};
  for (int d = 0; d < 3; ++d) {
    const int v = stretched ? stretched[d] : (d == 2);
    if (v && n[d] < 4) {
      set_error("a stretched axis needs at least 4 cells for center_velocity's 5-point window");
      return ANEL_ERR_SIZE;
    }
    diag_str_[d] = v ? 1 : 0;
  }
  diag_mode_ = mode;
  diag_on_ = on != 0;
  return ANEL_OK;
}

int NSSolver::ensure_diag() {
  if (d_diag_) return ANEL_OK;
  ANEL_CUDA_TRY(cudaSetDevice(device_));
  const int X = nx_ + 2, Y = ny_ + 2, Z = nz_ + 2;
  ANEL_CUDA_TRY(cudaMalloc(&d_diag_, 26 * (size_t)Z * sizeof(double)));
  ANEL_CUDA_TRY(cudaMemset(d_diag_, 0, 26 * (size_t)Z * sizeof(double)));
  ANEL_CUDA_TRY(cudaMalloc(&d_dgA_, G_ * sizeof(double)));
  ANEL_CUDA_TRY(cudaMalloc(&d_dgB_, G_ * sizeof(double)));
  ANEL_CUDA_TRY(cudaMalloc(&d_dgpart_, (size_t)plane_part_doubles(D_) * sizeof(double)));
  // dxc[X] dyc[Y] xe[X] xc[X] ye[Y] yc[Y] ze[Z] zc[Z] (m_[d] = xe xc dxe dxc rdxe rdxc)
  std::vector<double> h;
  for (const std::vector<double>* v : {&m_[0][3], &m_[1][3], &m_[0][0], &m_[0][1], &m_[1][0], &m_[1][1],
                                       &m_[2][0], &m_[2][1]})
    h.insert(h.end(), v->begin(), v->end());
  ANEL_CUDA_TRY(cudaMalloc(&d_dgm_, h.size() * sizeof(double)));
  ANEL_CUDA_TRY(cudaMemcpy(d_dgm_, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
  // Area of avgX1X2 (Average.F90:351-356), summed in its order
  double area = 0.0;
  for (int j = 2; j <= ny_ + 1; ++j)
    for (int i = 2; i <= nx_ + 1; ++i) area = area + m_[0][3][i - 1] * m_[1][3][j - 1];
  diag_area_ = area;
  ANEL_CUDA_TRY(cudaEventCreate(&dev0_));
  ANEL_CUDA_TRY(cudaEventCreate(&dev1_));
  (void)X;
  (void)Y;
  return ANEL_OK;
}

int NSSolver::compute_diagnostics(cudaStream_t s) {
  ANEL_CUDA_TRY(cudaSetDevice(device_));
  if (!s) s = stream_;
  const int st = ensure_diag();
  if (st != ANEL_OK) return st;
  const int X = nx_ + 2, Y = ny_ + 2, Z = nz_ + 2;
  double* m = d_diag_ + 16 * (size_t)Z;  // plane averages, see k_diag_update
  const double* dxc = d_dgm_;
  const double* dyc = dxc + X;
  const double* ax_e[3] = {dyc + Y, dyc + Y + 2 * X, dyc + 3 * Y + 2 * X};
  const double* ax_c[3] = {ax_e[0] + X, ax_e[1] + Y, ax_e[2] + Z};
  const double area = diag_area_;
  const bool corr = diag_mode_ == ANEL_DIAG_CORRECTED;
  // u, v, w: centre (then ghost 'u'/'v'/'w'), mean, squared fluctuation
  // (NSsolver.F90:291-358)
  const double* vel[3] = {D_.u, D_.v, D_.w};
  const int vt[3] = {NV_U, NV_V, NV_W};
  const int mean_slot[3] = {0, 1, 4}, sq_slot[3] = {5, 6, 7};
  for (int d = 0; d < 3; ++d) {
    launch_center(D_, vel[d], d_dgA_, d + 1, diag_str_[d], corr, ax_e[d], ax_c[d], s);
    launch_ghost_field(D_, d_dgA_, zrule(vt[d]), s);
    double* mean = m + (size_t)mean_slot[d] * Z;
    launch_plane_avg(D_, d_dgA_, dxc, dyc, area, d_dgpart_, mean, s);
    launch_fluct_sq(D_, d_dgA_, mean, d_dgB_, s);
    launch_ghost_field(D_, d_dgB_, zrule(vt[d]), s);
    launch_plane_avg(D_, d_dgB_, dxc, dyc, area, d_dgpart_, m + (size_t)sq_slot[d] * Z, s);
  }
  // rho and scal1: avgX1X2 ghosts the field itself first (:299-300, 364-393)
  double* sc[2] = {D_.rho, D_.s};
  const int svt[2] = {NV_RHO, NV_SCAL1};
  const int smean[2] = {2, 3}, ssq[2] = {8, 9};
  for (int q = 0; q < 2; ++q) {
    double* mean = m + (size_t)smean[q] * Z;
    double* sq = m + (size_t)ssq[q] * Z;
    if (!sc[q]) {
      ANEL_CUDA_TRY(cudaMemsetAsync(mean, 0, Z * sizeof(double), s));
      ANEL_CUDA_TRY(cudaMemsetAsync(sq, 0, Z * sizeof(double), s));
      continue;
    }
    launch_ghost_field(D_, sc[q], zrule(svt[q]), s);
    launch_plane_avg(D_, sc[q], dxc, dyc, area, d_dgpart_, mean, s);
    launch_fluct_sq(D_, sc[q], mean, d_dgB_, s);
    launch_ghost_field(D_, d_dgB_, zrule(svt[q]), s);
    launch_plane_avg(D_, d_dgB_, dxc, dyc, area, d_dgpart_, sq, s);
  }
  launch_diag_update(Z, time_ - told_, m, d_diag_, s);
  ANEL_CUDA_TRY(cudaGetLastError());
  return ANEL_OK;
}

int NSSolver::get_diagnostics(double* out, int mem) {
  ANEL_CUDA_TRY(cudaSetDevice(device_));
  if (!out) {
    set_error("null output");
    return ANEL_ERR_ARG;
  }
  const size_t bytes = 16 * (size_t)(nz_ + 2) * sizeof(double);
  if (!d_diag_) {
    if (mem == ANEL_MEM_DEVICE) ANEL_CUDA_TRY(cudaMemset(out, 0, bytes));
    else std::memset(out, 0, bytes);
    return ANEL_OK;
  }
  ANEL_CUDA_TRY(cudaStreamSynchronize(stream_));
  ANEL_CUDA_TRY(cudaMemcpy(out, d_diag_, bytes,
                           mem == ANEL_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost));
  return ANEL_OK;
}

int NSSolver::step_host(const anel_fields* in, const anel_fields* out, int nsteps, cudaStream_t s,
                        anel_step_report* rep) {
  ANEL_CUDA_TRY(cudaSetDevice(device_));
  if (!s) s = stream_;
  if (!in || !out || nsteps < 1) {
    set_error("step_host: null fields or nsteps < 1");
    return ANEL_ERR_ARG;
  }
  if (!io_stream_) {
    ANEL_CUDA_TRY(cudaStreamCreateWithFlags(&io_stream_, cudaStreamNonBlocking));
    for (cudaEvent_t& e : io_ev_) ANEL_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  const size_t fb = G_ * sizeof(double);
  double* const* src = reinterpret_cast<double* const*>(in);
  double* const* dst = reinterpret_cast<double* const*>(out);
  // everything but p in on the step's stream (r and densityBG keep their
  // z-profile check of set_fields)
  anel_fields rest = *in;
  rest.p = nullptr;
  int st = set_fields(&rest, ANEL_MEM_HOST, s);
  if (st != ANEL_OK) return st;
  if (in->p) {
    // p in on the copy stream once the others are in, ahead of its first use
    ANEL_CUDA_TRY(cudaEventRecord(io_ev_[3], s));
    ANEL_CUDA_TRY(cudaStreamWaitEvent(io_stream_, io_ev_[3], 0));
    ANEL_CUDA_TRY(cudaMemcpyAsync(D_.p, in->p, fb, cudaMemcpyHostToDevice, io_stream_));
    ANEL_CUDA_TRY(cudaEventRecord(io_ev_[0], io_stream_));
    io_wait_p_ = true;
  }
  io_out_ = out;
  st = step(nsteps, s, rep);
  io_out_ = nullptr;
  if (io_wait_p_) {  // no pressure solve consumed it (cannot happen in a step)
    cudaStreamWaitEvent(s, io_ev_[0], 0);
    io_wait_p_ = false;
  }
  if (st != ANEL_OK) {
    cudaStreamSynchronize(io_stream_);
    return st;
  }
  // the remaining fields out on the step's stream
  for (int q = 0; q < 17; ++q) {
    if (!dst[q] || !d_fields_[q] || q == 3 || q == 4 || q == 5) continue;  // p, rho, scal1: done
    ANEL_CUDA_TRY(cudaMemcpyAsync(dst[q], d_fields_[q], fb, cudaMemcpyDeviceToHost, s));
  }
  ANEL_CUDA_TRY(cudaEventRecord(io_ev_[3], io_stream_));
  ANEL_CUDA_TRY(cudaStreamWaitEvent(s, io_ev_[3], 0));
  ANEL_CUDA_TRY(cudaStreamSynchronize(s));
  (void)src;
  return ANEL_OK;
}

int NSSolver::project(cudaStream_t s, int* iters, double* relmax) {
  ANEL_CUDA_TRY(cudaSetDevice(device_));
  if (!s) s = stream_;
  fields_changed();
  // the velocity ghosts first: with the wall values in place the boundary
  // flux of Psource vanishes and the Neumann problem is compatible
  launch_ghost_field(D_, D_.u, zrule(NV_U), s);
  launch_ghost_field(D_, D_.v, zrule(NV_V), s);
  launch_ghost_field(D_, D_.w, zrule(NV_W), s);
  launch_psource(D_, 1.0, s);
  anel_mg_report rep{};
  const int st = mg_->solve_device(D_.p, D_.psrc, s, &rep);
  if (st != ANEL_OK && st != ANEL_ERR_NOCONV) return st;
  launch_pgrad(D_, 1.0, zrule(NV_U), zrule(NV_V), zrule(NV_W), s);
  ANEL_CUDA_TRY(cudaStreamSynchronize(s));
  if (iters) *iters = rep.iter;
  if (relmax) *relmax = rep.relmax;
  return check_launch("project");
}

// divergence (Routines.F90:54-183) of the current fields into device
// memory: max |div| in d_red_[1], the volume-weighted sums after the fold;
// with_cfl also the CFL maximum in d_red_[2]
int NSSolver::divergence_pass(cudaStream_t s, bool with_cfl) {
  const int64_t nb = divergence_blocks(D_);
  // partial pairs, fold scratch, the two sums
  if (!d_part_)
    ANEL_CUDA_TRY(cudaMalloc(&d_part_, (2 * nb + fold_scratch_doubles() + 2) * sizeof(double)));
  double* sums = d_part_ + 2 * nb + fold_scratch_doubles();
  ANEL_CUDA_TRY(cudaMemsetAsync(d_red_ + 1, 0, (with_cfl ? 2 : 1) * sizeof(unsigned long long), s));
  launch_divergence(D_, d_red_ + 1, d_part_, s, with_cfl ? d_red_ + 2 : nullptr);
  launch_fold_pairs(d_part_, nb, d_part_ + 2 * nb, sums, s);
  return ANEL_OK;
}

void NSSolver::divergence_issue(cudaStream_t s) {
  const int64_t nb = divergence_blocks(D_);
  const double* sums = d_part_ + 2 * nb + fold_scratch_doubles();
  copy_words(d_red_ + 1, h_red_ + 1, 1, s);
  copy_words(sums, h_red_ + 2, 2, s);
}

int NSSolver::divergence_take(double* out) {
  out[0] = h_red_[2] / h_red_[3];
  out[1] = h_red_[1];
  return check_launch("divergence");
}

int NSSolver::divergence_read(cudaStream_t s, double* out) {
  divergence_issue(s);
  ANEL_CUDA_TRY(cudaStreamSynchronize(s));
  return divergence_take(out);
}

int NSSolver::divergence(cudaStream_t s, double* out) {
  ANEL_CUDA_TRY(cudaSetDevice(device_));
  if (!s) s = stream_;
  const int st = divergence_pass(s, false);
  if (st != ANEL_OK) return st;
  div_ready_ = false;  // d_red_[1] and the sums now hold this pass
  return divergence_read(s, out);
}

}  // namespace anel
