// ns_solver.h -- host side of the B200 RK3 time stepper.
#pragma once

#include <vector>

#include "mg_solver.h"
#include "ns_launch.h"

namespace anel {

// One shear-layer member: device-resident fields, its multigrid context
// and the sub-step schedule of NSsolver/rk_ss (NSsolver.F90:63-583).
class NSSolver {
 public:
  static NSSolver* create(const anel_grid_desc* g, const anel_mg_params* mg, const anel_ns_params* ns,
                          int device, int* status);
  ~NSSolver();

  int set_fields(const anel_fields* f, int mem, cudaStream_t s);
  int get_fields(const anel_fields* f, int mem, cudaStream_t s);
  int substep(double a1, double a2, double a3, double dt_rk, double dt, cudaStream_t s, int* iters,
              double* relmax, bool q_zero = false);
  int step(int nsteps, cudaStream_t s, anel_step_report* rep);
  // nsteps RK3 steps of n members (contexts of one grid, boundary setup
  // and multigrid parameters; physics, time step and state their own) on
  // stream s, with each sub-step's n pressure solves as one batched solve
  // of bmg (MGSolver::solve_batch; a solver of the members' grid and
  // multigrid parameters).  Each member's fields and report are those of
  // its own step(); reps: n reports.
  static int step_cohort(NSSolver* const* ms, int n, int nsteps, MGSolver* bmg, cudaStream_t s,
                         anel_step_report* reps);
  // nsteps from the host state `in` to the host state `out` (may be the
  // same arrays): the fields are copied in, stepped and copied out, with
  // the copy of p in overlapping sub-step 1 up to its pressure solve and
  // the copies of rho/scal1 and p out overlapping the last sub-step's
  // pressure solve and Pgrad.  Results equal set_fields + step +
  // get_fields.
  int step_host(const anel_fields* in, const anel_fields* out, int nsteps, cudaStream_t s,
                anel_step_report* rep);
  int project(cudaStream_t s, int* iters, double* relmax);
  int divergence(cudaStream_t s, double* out);
  // Re-target a context to a new member with the same grid, models and
  // boundary conditions (serving pool): new physics parameters, clock at
  // step 1, time 0, accumulators and eddy fields zeroed.
  int reset(const anel_ns_params* ns, cudaStream_t s);
  // Seeded shear-layer state on the device (the layout of shear.py's
  // shear_layer_fields): u = tanh(zc) + noise, v, w = noise, rho =
  // -tanh(zc), noise amp*(2U-1) on |zc| < zmax from the Park-Miller
  // sequence of the seed; p, scal1 = 0.
  int init_shear(uint32_t seed, double amp, double zmax, cudaStream_t s);
  void set_clock(double time, int nstep) {
    time_ = time;
    nstep_ = nstep;
  }
  // Plane statistics of the driver's dk/dt block (NSsolver.F90:288-395):
  // with on, step() runs it after every step; compute_diagnostics runs it
  // once on the current fields; get_diagnostics copies the 16 profiles.
  int set_diagnostics(int on, int mode, const int* stretched);
  int compute_diagnostics(cudaStream_t s);
  int get_diagnostics(double* out, int mem);
  MGSolver* mg() { return mg_; }
  cudaStream_t stream() const { return stream_; }
  int64_t cells() const { return (int64_t)nx_ * ny_ * nz_; }
  int64_t ghosted_cells() const { return G_; }
  void sizes(int* nx, int* ny, int* nz) const {
    *nx = nx_;
    *ny = ny_;
    *nz = nz_;
  }
  // ghost() of u, v, w, p, rho and scal1 with their own rules, as after a
  // restart read (Restart.F90:425-430)
  int ghost_state(cudaStream_t s);

 private:
  NSSolver() = default;
  int init(const anel_grid_desc* g, const anel_mg_params* mg, const anel_ns_params* ns, int device);
  int upload_profiles();
  int cn_factors(int slot, double rkdt, cudaStream_t s);
  ZRule zrule(int vtype) const;
  double calcdt(cudaStream_t s, int* st);
  // phases of one RK3 step (step() and step_cohort() run them in order;
  // the pressure solve of each sub-step sits between pre and post)
  int step_begin(cudaStream_t s, double* delt);
  void step_begin_issue(cudaStream_t s);
  int step_begin_finish(cudaStream_t s, double* delt);
  void calcdt_issue(cudaStream_t s);
  double calcdt_take() const;
  int substep_pre(double a1, double a2, double a3, double dt_rk, double dt, cudaStream_t s, bool q_zero);
  int substep_post(const anel_mg_report& rep, cudaStream_t s, int* iters, double* relmax);
  int step_end(double delt, cudaStream_t s, anel_step_report* r);
  int step_finish(cudaStream_t s, int64_t launches0, anel_step_report* r);
  void clip_scalars(cudaStream_t s);
  double pend_dtrk_ = 0.0;  // the sub-step between substep_pre and substep_post
  // step_end's divergence pass also takes the CFL maximum of the fields it
  // leaves (d_red_[2]) and its divergence results stay on the device:
  // cfl_ready_ lets the next calcdt use that maximum, div_ready_ lets
  // step_finish report those results, without another read of u, v, w.
  // Every call that changes u, v or w afterwards clears both.
  bool cfl_ready_ = false, div_ready_ = false;

  void fields_changed() { cfl_ready_ = div_ready_ = false; }
  // pressure initial guess (prm_.pguess): per sub-step index, the member's
  // last two solutions (hist_[q][last_[q]] the newest), nhist_[q] of them
  // valid; cur_sub_ is the sub-step index inside step() (-1 elsewhere)
  double* hist_[3][2] = {{nullptr, nullptr}, {nullptr, nullptr}, {nullptr, nullptr}};
  int last_[3] = {0, 0, 0}, nhist_[3] = {0, 0, 0};
  int cur_sub_ = -1;
  int ensure_hist();
  int divergence_pass(cudaStream_t s, bool with_cfl);
  int divergence_read(cudaStream_t s, double* out);
  void divergence_issue(cudaStream_t s);
  int divergence_take(double* out);
  int les_coeffs(cudaStream_t s);

  anel_ns_params prm_{};
  int device_ = 0;
  cudaStream_t stream_ = nullptr;
  int nx_ = 0, ny_ = 0, nz_ = 0;
  int64_t G_ = 0;
  std::vector<double> m_[3][6];  // fine metrics (xe xc dxe dxc rdxe rdxc)
  std::vector<double> rz_, bgz_;
  double rRe_ = 0, rPr_ = 0, rSc_ = 0, g_orig_ = 0, gnow_ = 0;
  double time_ = 0.0;
  double told_ = 1.0e-16;  // time at the start of the last step (NSsolver.F90:47, 272-273)
  int nstep_ = 1;
  // plane statistics: 16 profiles + 10 plane averages of Z values, two
  // G-sized scratch fields, the metrics they use (dxc dyc xe xc ye yc ze
  // zc) and the plane partial sums; allocated on first use
  bool diag_on_ = false;
  int diag_mode_ = ANEL_DIAG_LITERAL;
  int diag_str_[3] = {0, 0, 0};
  double diag_area_ = 0.0;
  double acc_diag_ms_ = 0.0;
  double* d_diag_ = nullptr;
  double* d_dgA_ = nullptr;
  double* d_dgB_ = nullptr;
  double* d_dgm_ = nullptr;
  double* d_dgpart_ = nullptr;
  cudaEvent_t dev0_ = nullptr, dev1_ = nullptr;
  int ensure_diag();
  // dynamic Smagorinsky models (ns_dsm.cu): scratch fields, metrics
  // (dxc dyc delg, two profiles), plane partial sums and coordinates
  double* d_dyn_ = nullptr;
  double* d_dyn_m_ = nullptr;
  double* dyn_part_ = nullptr;
  double* d_dyn_axes_ = nullptr;
  const double* d_dyn_ax_[6] = {nullptr};
  double dyn_area_ = 0.0;
  bool dyn_ready_ = false;  // dyn_prepare done for the current les_coeffs
  // host-state stepping (step_host): copy stream, events and the hooks
  // the sub-steps read
  cudaStream_t io_stream_ = nullptr;
  cudaEvent_t io_ev_[4] = {nullptr, nullptr, nullptr, nullptr};  // p in, rho out, p out, all in
  bool io_wait_p_ = false;       // the next pressure solve waits for p's copy in
  bool io_last_sub_ = false;     // this sub-step is the last of the call
  const anel_fields* io_out_ = nullptr;
  int ensure_dyn();
  int dyn_prepare(cudaStream_t s);
  // tmp: second scratch field (null: the dynamic models' own)
  void dyn_filter(const double* in, double* out, int vt, int hf, cudaStream_t s, double* tmp = nullptr);
  int smooth_scalars(cudaStream_t s);
  void dyn_ew(int op, double* out, const double* a, const double* b, const double* c, cudaStream_t s);
  int dyn_ratio(double* num, double* den, double* out, cudaStream_t s);
  int dyn_profile(const double* a, double* host, cudaStream_t s);
  int dsm_velocity(cudaStream_t s, double* cs);
  int dsm_scalar(const double* c, cudaStream_t s, double* out);
  MGSolver* mg_ = nullptr;
  NSDev D_{};
  // device allocations
  double* d_fields_[17] = {nullptr};
  double* d_metric_ = nullptr;      // rdxe rdxc rdye rdyc rdze rdzc dze dzc
  double* d_prof_ = nullptr;        // rz bgz
  double* d_les_ = nullptr;         // LES profiles: Csgs CTsgs CSsgs delg^2 (nz+2 each)
  double* d_ic_ = nullptr;          // tanh(zc) and |zc| profiles of init_shear
  double* d_cnb_ = nullptr;         // LES CN: eliminated diagonal per cell
  bool les_any_ = false;            // a subgrid model is on: nuT/kappaT/nappaT exist
  bool les_coeffs_done_ = false;
  double* d_cn_ = nullptr;          // CN factors: 3 slots x 5 vars x 9 arrays x (nz+2)
  double* h_cn_ = nullptr;          // pinned staging of the same
  double cn_rkdt_[3] = {-1, -1, -1};
  int cnvar_ = 0;     // launch variant of the DNS column solve (tune_cn)
  int cnlesvar_ = 0;  // and of the LES column solve
  // the RHS accumulators q_* hold zero ghost cells and the previous step's
  // interior values only (no set_fields, reset or scratch use since the
  // last zeroing): the first sub-step's a1 = 0 form overwrites every
  // interior cell without reading it, so zero_temps can skip them
  bool temps_clean_ = false;
  int tune_cn();
  int cn_next_ = 0;
  unsigned long long* d_red_ = nullptr;
  double* d_part_ = nullptr;
  double* h_red_ = nullptr;
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
  CNFacHost fac(int slot, int vi) const;
  // multigrid totals of the current step() call
  double acc_mg_ms_ = 0.0, acc_sweep_ms_ = 0.0;
  int acc_sweeps_ = 0;
};

}  // namespace anel

// The C-ABI handle of a stepper context.
struct anel_ns_ctx {
  anel::NSSolver* s;
};

namespace anel {
inline NSSolver* ctx_solver(anel_ns_ctx* c) { return c->s; }
}  // namespace anel
