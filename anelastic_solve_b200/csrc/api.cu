// api.cu -- the extern "C" boundary declared in include/anel.h.
#include <cstdarg>
#include <cstdio>
#include <mutex>

#include "mg_solver.h"

namespace anel {

std::atomic<int64_t> g_launches{0};
static thread_local char t_err[1024] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(t_err, sizeof(t_err), fmt, ap);
  va_end(ap);
}
const char* last_error() { return t_err; }

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
}  // namespace

extern "C" {

const char* anel_last_error(void) { return anel::last_error(); }
int anel_version(void) { return 100; }
int64_t anel_kernel_launch_count(void) { return anel::g_launches.load(); }

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

}  // extern "C"
