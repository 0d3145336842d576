// api.cu -- the extern "C" boundary declared in include/anel.h.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "mg_solver.h"
#include "tune.h"
#include "ns_solver.h"

namespace anel {

std::atomic<int64_t> g_launches{0};
thread_local int64_t t_launches = 0;
static thread_local char t_err[1024] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(t_err, sizeof(t_err), fmt, ap);
  va_end(ap);
}
const char* last_error() { return t_err; }

void set_smem_limit_once(const void* func, int bytes) {
  struct Entry {
    int dev;
    const void* func;
    int bytes;
  };
  static std::mutex mu;
  static std::vector<Entry> done;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  for (auto& d : done)
    if (d.dev == dev && d.func == func) {
      // the attribute is a maximum: raise it when a larger launch comes
      if (bytes > d.bytes) {
        cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        d.bytes = bytes;
      }
      return;
    }
  cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  done.push_back(Entry{dev, func, bytes});
}

__global__ void k_copy_words(const unsigned long long* __restrict__ src, unsigned long long* __restrict__ dst,
                             int64_t n) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
    dst[t] = src[t];
}

void copy_words(const void* src, void* dst, int64_t nwords, cudaStream_t s) {
  int64_t blocks = (nwords + 255) / 256;
  if (blocks > 64) blocks = 64;
  if (blocks < 1) blocks = 1;
  k_copy_words<<<(unsigned)blocks, 256, 0, s>>>(static_cast<const unsigned long long*>(src),
                                               static_cast<unsigned long long*>(dst), nwords);
  count_launch();
}

int check_launch(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("%s: kernel launch failed: %s", what, cudaGetErrorString(e));
    return ANEL_ERR_CUDA;
  }
  return ANEL_OK;
}

}  // namespace anel

struct anel_mg_ctx {
  anel::MGSolver* s;
};

namespace {
std::mutex g_default_mu;
anel::MGSolver* g_default = nullptr;  // the drop-in calls' module state
anel::NSSolver* g_ns = nullptr;       // drop-in stepper
anel_fields g_bound{};                // bound host module arrays
bool g_bound_ok = false;
}  // namespace

extern "C" {

const char* anel_last_error(void) { return anel::last_error(); }
int anel_version(void) { return 100; }
int64_t anel_kernel_launch_count(void) { return anel::g_launches.load(); }

int32_t anel_tuning_report(char* buf, int32_t cap) {
  const std::string r = anel::tune_report();
  if (buf && cap > 0) {
    const size_t n = r.size() < (size_t)(cap - 1) ? r.size() : (size_t)(cap - 1);
    std::memcpy(buf, r.data(), n);
    buf[n] = '\0';
  }
  return (int32_t)r.size();
}

// ------------------------------------------------------------ drop-in MG
int anel_mg_init(const anel_grid_desc* grid, const anel_mg_params* params) {
  std::lock_guard<std::mutex> lk(g_default_mu);
  delete g_default;
  g_default = nullptr;
  int st = ANEL_OK;
  g_default = anel::MGSolver::create(grid, params, 0, &st);
  return st;
}

int anel_mg_set_density(const double* r) {
  std::lock_guard<std::mutex> lk(g_default_mu);
  if (!g_default) {
    anel::set_error("anel_mg_set_density before anel_mg_init");
    return ANEL_ERR_ARG;
  }
  return g_default->set_density_host(r);
}

void anel_mg_solve(double* phif, double* rhsf, int32_t* iter, double* relmax) {
  std::lock_guard<std::mutex> lk(g_default_mu);
  anel_mg_report rep{};
  if (!g_default) {
    anel::set_error("anel_mg_solve before anel_mg_init");
    if (iter) *iter = -1;
    if (relmax) *relmax = -1.0;
    return;
  }
  const int st = g_default->solve_host(phif, rhsf, nullptr, &rep);
  if (st != ANEL_OK && st != ANEL_ERR_NOCONV) {
    if (iter) *iter = -1;
    if (relmax) *relmax = -1.0;
    return;
  }
  if (iter) *iter = rep.iter;
  if (relmax) *relmax = rep.relmax;
}

int anel_mg_finalize(void) {
  std::lock_guard<std::mutex> lk(g_default_mu);
  delete g_default;
  g_default = nullptr;
  return ANEL_OK;
}

// ------------------------------------------------------------ context MG
anel_mg_ctx* anel_mg_create(const anel_grid_desc* grid, const anel_mg_params* params,
                            int32_t device, int32_t* status) {
  int st = ANEL_OK;
  anel::MGSolver* s = anel::MGSolver::create(grid, params, device, &st);
  if (status) *status = st;
  if (!s) return nullptr;
  return new anel_mg_ctx{s};
}

void anel_mg_destroy(anel_mg_ctx* ctx) {
  if (!ctx) return;
  delete ctx->s;
  delete ctx;
}

int anel_mg_ctx_set_density(anel_mg_ctx* ctx, const double* r, int32_t mem) {
  if (!ctx) {
    anel::set_error("null context");
    return ANEL_ERR_ARG;
  }
  return mem == ANEL_MEM_DEVICE ? ctx->s->set_density_device(r, nullptr)
                                : ctx->s->set_density_host(r);
}

int anel_mg_ctx_solve(anel_mg_ctx* ctx, double* phif, const double* rhsf, int32_t mem,
                      void* stream, anel_mg_report* report) {
  if (!ctx) {
    anel::set_error("null context");
    return ANEL_ERR_ARG;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  return mem == ANEL_MEM_DEVICE ? ctx->s->solve_device(phif, rhsf, s, report)
                                : ctx->s->solve_host(phif, rhsf, s, report);
}

int anel_mg_ctx_solve_batch(anel_mg_ctx* ctx, int32_t n, double* const* d_phis, const double* const* d_rhss,
                            void* stream, anel_mg_report* reports) {
  if (!ctx) {
    anel::set_error("null context");
    return ANEL_ERR_ARG;
  }
  return ctx->s->solve_batch(n, d_phis, d_rhss, static_cast<cudaStream_t>(stream), reports);
}

int anel_mg_ctx_set_profiling(anel_mg_ctx* ctx, int32_t on) {
  if (!ctx) return ANEL_ERR_ARG;
  return ctx->s->set_profiling(on != 0);
}

int anel_mg_ctx_levels(const anel_mg_ctx* ctx, int32_t* out, int32_t cap) {
  if (!ctx || !out) return ANEL_ERR_ARG;
  return ctx->s->levels_table(out, cap);
}

int anel_mg_ctx_debug_pass(anel_mg_ctx* ctx, int32_t which, double* d_phi, const double* d_src,
                           void* stream) {
  if (!ctx) return ANEL_ERR_ARG;
  return ctx->s->debug_pass(which, d_phi, d_src, static_cast<cudaStream_t>(stream));
}

// ------------------------------------------------------------ stepper
anel_ns_ctx* anel_ns_create(const anel_grid_desc* grid, const anel_mg_params* mg,
                            const anel_ns_params* ns, int32_t device, int32_t* status) {
  int st = ANEL_OK;
  anel::NSSolver* s = anel::NSSolver::create(grid, mg, ns, device, &st);
  if (status) *status = st;
  if (!s) return nullptr;
  return new anel_ns_ctx{s};
}

void anel_ns_destroy(anel_ns_ctx* ctx) {
  if (!ctx) return;
  delete ctx->s;
  delete ctx;
}

int anel_ns_set_fields(anel_ns_ctx* ctx, const anel_fields* f, int32_t mem) {
  if (!ctx) return ANEL_ERR_ARG;
  return ctx->s->set_fields(f, mem, nullptr);
}

int anel_ns_get_fields(anel_ns_ctx* ctx, const anel_fields* f, int32_t mem) {
  if (!ctx) return ANEL_ERR_ARG;
  return ctx->s->get_fields(f, mem, nullptr);
}

int anel_ns_ctx_substep(anel_ns_ctx* ctx, double a1, double a2, double a3, double dt_rk, double dt,
                        void* stream, int32_t* mg_iter, double* mg_relmax) {
  if (!ctx) return ANEL_ERR_ARG;
  int it = 0;
  double rm = 0.0;
  const int st = ctx->s->substep(a1, a2, a3, dt_rk, dt, static_cast<cudaStream_t>(stream), &it, &rm);
  if (mg_iter) *mg_iter = it;
  if (mg_relmax) *mg_relmax = rm;
  return st;
}

int anel_ns_ctx_step(anel_ns_ctx* ctx, int32_t nsteps, void* stream, anel_step_report* report) {
  if (!ctx || nsteps < 0) return ANEL_ERR_ARG;
  return ctx->s->step(nsteps, static_cast<cudaStream_t>(stream), report);
}

int anel_ns_ctx_step_cohort(anel_ns_ctx* const* ctxs, int32_t n, int32_t nsteps, anel_mg_ctx* batch,
                            void* stream, anel_step_report* reports) {
  if (!ctxs || n < 1 || nsteps < 0 || !reports) {
    anel::set_error("step_cohort: n >= 1 contexts, nsteps >= 0 and reports required");
    return ANEL_ERR_ARG;
  }
  std::vector<anel::NSSolver*> ms(n);
  for (int b = 0; b < n; ++b) {
    if (!ctxs[b]) {
      anel::set_error("step_cohort: null context %d", b);
      return ANEL_ERR_ARG;
    }
    ms[b] = ctxs[b]->s;
  }
  anel::MGSolver* bmg = batch ? batch->s : ms[0]->mg();
  return anel::NSSolver::step_cohort(ms.data(), n, nsteps, bmg, static_cast<cudaStream_t>(stream), reports);
}

int anel_ns_ctx_set_profiling(anel_ns_ctx* ctx, int32_t on) {
  if (!ctx) return ANEL_ERR_ARG;
  return ctx->s->mg()->set_profiling(on != 0);
}

int anel_ns_ctx_set_clock(anel_ns_ctx* ctx, double time, int32_t nstep) {
  if (!ctx) return ANEL_ERR_ARG;
  ctx->s->set_clock(time, nstep);
  return ANEL_OK;
}

int anel_ns_ctx_step_host(anel_ns_ctx* ctx, const anel_fields* in, const anel_fields* out, int32_t nsteps,
                          void* stream, anel_step_report* report) {
  if (!ctx) return ANEL_ERR_ARG;
  return ctx->s->step_host(in, out, nsteps, static_cast<cudaStream_t>(stream), report);
}

int anel_ns_ctx_set_diagnostics(anel_ns_ctx* ctx, int32_t on, int32_t mode, const int32_t* stretched) {
  if (!ctx) return ANEL_ERR_ARG;
  int str[3] = {0, 0, 1};
  if (stretched)
    for (int d = 0; d < 3; ++d) str[d] = stretched[d];
  return ctx->s->set_diagnostics(on, mode, str);
}

int anel_ns_ctx_compute_diagnostics(anel_ns_ctx* ctx, void* stream) {
  if (!ctx) return ANEL_ERR_ARG;
  return ctx->s->compute_diagnostics(static_cast<cudaStream_t>(stream));
}

int anel_ns_ctx_get_diagnostics(anel_ns_ctx* ctx, double* out, int32_t mem) {
  if (!ctx || !out) return ANEL_ERR_ARG;
  if (mem != ANEL_MEM_HOST && mem != ANEL_MEM_DEVICE) return ANEL_ERR_ARG;
  return ctx->s->get_diagnostics(out, mem);
}

int anel_ns_ctx_divergence(anel_ns_ctx* ctx, double* out) {
  if (!ctx || !out) return ANEL_ERR_ARG;
  return ctx->s->divergence(nullptr, out);
}

int anel_ns_ctx_project(anel_ns_ctx* ctx, int32_t* mg_iter, double* mg_relmax) {
  if (!ctx) return ANEL_ERR_ARG;
  int it = 0;
  double rm = 0.0;
  const int st = ctx->s->project(nullptr, &it, &rm);
  if (mg_iter) *mg_iter = it;
  if (mg_relmax) *mg_relmax = rm;
  return st;
}

// drop-in stepper
int anel_ns_init(const anel_grid_desc* grid, const anel_mg_params* mg, const anel_ns_params* ns) {
  std::lock_guard<std::mutex> lk(g_default_mu);
  delete g_ns;
  g_ns = nullptr;
  int st = ANEL_OK;
  g_ns = anel::NSSolver::create(grid, mg, ns, 0, &st);
  return st;
}

int anel_bind_fields(const anel_fields* f) {
  std::lock_guard<std::mutex> lk(g_default_mu);
  if (!f) return ANEL_ERR_ARG;
  g_bound = *f;
  g_bound_ok = true;
  // r and densityBG are copied once here (they change only with the setup)
  if (g_ns && (f->r || f->densityBG)) {
    anel_fields d{};
    d.r = f->r;
    d.densityBG = f->densityBG;
    return g_ns->set_fields(&d, ANEL_MEM_HOST, nullptr);
  }
  return ANEL_OK;
}

void anel_rk_substep(const double* a1, const double* a2, const double* a3, const double* ec,
                     const double* dt_rk, const double* dt, const int32_t* psolve, int32_t* stat) {
  (void)ec;
  (void)psolve;  // rk_ss always solves for the pressure (NSsolver.F90:520-523)
  std::lock_guard<std::mutex> lk(g_default_mu);
  if (!g_ns || !g_bound_ok || !a1 || !a2 || !a3 || !dt_rk || !dt) {
    anel::set_error("anel_rk_substep before anel_ns_init/anel_bind_fields or null argument");
    if (stat) *stat = ANEL_ERR_ARG;
    return;
  }
  anel_fields io = g_bound;
  io.r = nullptr;
  io.densityBG = nullptr;
  int st = g_ns->set_fields(&io, ANEL_MEM_HOST, nullptr);
  if (st == ANEL_OK) st = g_ns->substep(*a1, *a2, *a3, *dt_rk, *dt, nullptr, nullptr, nullptr);
  if (st == ANEL_OK) st = g_ns->get_fields(&io, ANEL_MEM_HOST, nullptr);
  if (stat) *stat = st;
}

int anel_ns_finalize(void) {
  std::lock_guard<std::mutex> lk(g_default_mu);
  delete g_ns;
  g_ns = nullptr;
  g_bound_ok = false;
  return ANEL_OK;
}

}  // extern "C"
