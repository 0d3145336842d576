// mg_solver.h -- host side of the B200 multigrid pressure solver.
#pragma once

#include <memory>
#include <vector>

#include "mg_coarse.h"
#include "mg_col.h"
#include "mg_launch.h"

namespace anel {

// The solver context: what MG_init builds (mg_init.F90:70-351) plus the
// device workspaces.  Not thread-safe; calls are ordered on `stream_`.
class MGSolver {
 public:
  static MGSolver* create(const anel_grid_desc* g, const anel_mg_params* p, int device,
                          int* status);
  ~MGSolver();

  // Density Flow::r on the fine ghosted grid (host pointer).  Must be
  // horizontally uniform, r = r(z), as every density profile of the
  // reference is; otherwise ANEL_ERR_UNSUPPORTED.
  int set_density_host(const double* r);
  int set_density_device(const double* r, cudaStream_t s);

  // mg_solver on device arrays: d_phi inout (ghosted FP64), d_rhs in.
  int solve_device(double* d_phi, const double* d_rhs, cudaStream_t s, anel_mg_report* rep);
  // Same with host arrays (copies in and out through pinned staging).
  int solve_host(double* phi, const double* rhs, cudaStream_t s, anel_mg_report* rep);

  // n independent problems on this solver's grid (same operator), each
  // phis[b] / rhss[b] a device array pair as for solve_device, solved
  // together: every kernel of the mixed z-line cycle runs over all members
  // still iterating (one launch per level step for the whole batch, the
  // defect-correction loop inside one CUDA graph per batch size), each
  // member stopping at its own tolerance test.  Member b's result and
  // report are those of solve_device on it alone.  Needs the column-layout
  // mixed cycle (batch_capable); reps: n reports.
  int solve_batch(int n, double* const* phis, const double* const* rhss, cudaStream_t s,
                  anel_mg_report* reps);
  bool batch_capable() const;
  // room for batches of up to n members (solve_batch grows it on demand)
  int batch_reserve(int n);
  // identifies the operator: a hash of every level's coefficients (equal
  // for solvers of one grid, parameters and density profile)
  uint64_t operator_hash() const { return op_hash_; }

  int debug_pass(int which, double* d_phi, const double* d_src, cudaStream_t s);
  int set_profiling(bool on);
  int levels_table(int32_t* out, int cap) const;

  cudaStream_t stream() const { return stream_; }
  int device() const { return device_; }
  const LevelGeom& fine() const { return geo_[ngrid_]; }
  int ngrid() const { return ngrid_; }
  const anel_mg_params& params() const { return prm_; }
  // Fine-level FP64 descriptor bound to the given arrays.
  DevLevel<double> fine_view(double* phi, const double* src) const;

 private:
  MGSolver() = default;
  int init(const anel_grid_desc* g, const anel_mg_params* p, int device);
  void build_metric_hierarchy();
  int build_coefficients(const std::vector<double>& rz);
  int upload_coefficients();
  void relax64(int l, int iters, cudaStream_t s);
  void cycle64(cudaStream_t s);
  void relax32(int l, int iters, cudaStream_t s);
  void cycle32(cudaStream_t s);
  // correction reset + FP32 V-cycle, replayed from a CUDA graph after the
  // first call (kernel pointers are fixed per solver)
  void run_cycle32(cudaStream_t s);
  cudaGraphExec_t g32x_ = nullptr;
  int64_t g32_launches_ = 0;
  int g32_calls_ = 0;
  bool g32_off_ = false;
  // column layout of the FP32 levels (mg_col.cuh): used by the mixed
  // ZLINE cycle with x/y semi-coarsening when nz = 32*M (M a supported
  // row count) and every level's ghosts are copies the sweeps can write
  bool col_ = false;
  int colM_ = 0;
  float* d_colfac_[ANEL_MAX_LEVELS + 1] = {nullptr};
  int colvar_[ANEL_MAX_LEVELS + 1] = {};  // sweep variant per level (tune_col)
  int* h_err_ = nullptr;  // host-mapped flag: a bounded copy wait of the sweep ran out
  int* d_err_ = nullptr;  // its device address
  int take_kernel_error(const char* what);
  int tune_col();
  // FP64 direct solve of level dirL_ in the column cycle (0: none; the
  // cycle then relaxes down to level 1), and of the fine level for the
  // debug pass that checks it
  int dirL_ = 0;
  DirectHost dir_;
  DirectHost dirfine_;
  int build_direct(int l, DirectHost& D);
  void choose_direct_level();
  ColLevel C32(int l) const;
  int64_t fp32_elems(int l) const;
  // nb = 0: this solver's own FP32 levels; nb >= 1: the first nb members of
  // the batch levels
  void relax_col(int l, int iters, cudaStream_t s, int nb = 0);
  void cycle_col(cudaStream_t s, int nb = 0);
  ColLevel C32b(int l, int nb) const;
  // batch state (solve_batch): capacity, FP32 levels and direct-solve work
  // of bcap_ members, member table, active flags, norms, convergence states
  int bcap_ = 0;
  float* d_bphi32_[ANEL_MAX_LEVELS + 1] = {nullptr};
  float* d_bsrc32_[ANEL_MAX_LEVELS + 1] = {nullptr};
  double* d_bdir_ = nullptr;
  double* d_bpart_ = nullptr;
  double* d_bnorm_ = nullptr;
  MemberIO* d_bmt_ = nullptr;
  MemberIO* h_bmt_ = nullptr;  // pinned staging of the member table
  int* d_bact_ = nullptr;
  void* d_bconv_ = nullptr;
  void* h_bconv_ = nullptr;    // pinned readback of the states
  cudaGraphExec_t bgraph_ = nullptr;
  int bgraph_n_ = 0;
  int64_t bgraph_head_launches_ = 0, bgraph_body_launches_ = 0;
  void batch_free();
  int build_batch_graph(int n, cudaStream_t s);
  int solve_fp64(double* d_phi, const double* d_rhs, cudaStream_t s, anel_mg_report* rep);
  int solve_mixed(double* d_phi, const double* d_rhs, cudaStream_t s, anel_mg_report* rep);
  // the mixed solve as one CUDA graph: the defect-correction loop is a
  // conditional while node whose body (FP32 cycle, correction, FP64
  // residual) ends in a kernel that tests convergence on the device, so a
  // solve needs one host synchronisation instead of one per cycle.  Built
  // per (phi, rhs) pair; 0 = not built, -1 = not available (host loop)
  int solve_mixed_graph(double* d_phi, const double* d_rhs, cudaStream_t s, anel_mg_report* rep);
  int build_solve_graph(double* d_phi, const double* d_rhs, cudaStream_t s);
  cudaGraphExec_t gsolve_ = nullptr;
  const double* gsolve_phi_ = nullptr;
  const double* gsolve_rhs_ = nullptr;
  int gsolve_state_ = 0;
  int64_t gsolve_head_launches_ = 0, gsolve_body_launches_ = 0;
  cudaStream_t side_ = nullptr;   // stream the conditional body is captured on
  void* d_conv_ = nullptr;        // device convergence state of the graph solve
  int coarsen_dirs(int lC) const;
  double true_resid(const double* d_phi, const double* d_rhs, cudaStream_t s, double* fnorm);

  anel_mg_params prm_{};
  uint64_t op_hash_ = 0;
  int device_ = 0;
  cudaStream_t stream_ = nullptr;
  int nx_ = 0, ny_ = 0, nz_ = 0;
  double L_[3] = {0, 0, 0};
  int ngrid_ = 0;
  int nC_[3] = {0, 0, 0};
  LevelGeom geo_[ANEL_MAX_LEVELS + 1];
  int bd_[27] = {0};
  double phibc_[ANEL_MAX_LEVELS + 1][6];
  // fine metrics (n+2 each) and the coarse hierarchy (mg_grids.F90)
  std::vector<double> fm_[3][6];          // xe xc dxe dxc rdxe rdxc
  std::vector<double> hE_[3], hC_[3], hDC_[3], hDE_[3], pA_[3], pB_[3];
  // METRIC mode hierarchy: per level/direction local E, C, DC, DE
  std::vector<double> ag_[ANEL_MAX_LEVELS + 1][3][4];
  void build_agglomerated();
  LevelCoef coef_[ANEL_MAX_LEVELS + 1];
  LevelCoef ljc_[ANEL_MAX_LEVELS + 1];  // LJ line coefficients (pcf_1..6)
  void build_lj_coefficients();
  double* d_ljc64_[ANEL_MAX_LEVELS + 1] = {nullptr};
  float* d_ljc32_[ANEL_MAX_LEVELS + 1] = {nullptr};
  BdryRule rule_[ANEL_MAX_LEVELS + 1];
  BdryRule rule_hom_[ANEL_MAX_LEVELS + 1];  // same with phibc = 0 (error equation)
  bool coef_ready_ = false;
  // device memory
  double* d_phi64_[ANEL_MAX_LEVELS + 1] = {nullptr};
  double* d_src64_[ANEL_MAX_LEVELS + 1] = {nullptr};
  double* d_coef64_[ANEL_MAX_LEVELS + 1] = {nullptr};
  float* d_phi32_[ANEL_MAX_LEVELS + 1] = {nullptr};
  float* d_src32_[ANEL_MAX_LEVELS + 1] = {nullptr};
  float* d_coef32_[ANEL_MAX_LEVELS + 1] = {nullptr};
  // ZLINE: per level eliminated tridiagonal factors ap[Z], bp[Z]
  double* d_zf64_[ANEL_MAX_LEVELS + 1] = {nullptr};
  float* d_zf32_[ANEL_MAX_LEVELS + 1] = {nullptr};
  // partitioned z-line factors of the FP32 cycle (ap, 1/bp, u, v: Z each;
  // then the 2P x 2P interface inverse), null where the level's nz does
  // not split into kZSeg segments of at least two rows
  float* d_zseg32_[ANEL_MAX_LEVELS + 1] = {nullptr};
  // cyclic-reduction multipliers of the FP32 line matrix (see SegFac::cr),
  // on the levels that have partitioned factors and nz <= kCRMaxRows
  float* d_zcr32_[ANEL_MAX_LEVELS + 1] = {nullptr};
  int zcr_steps_[ANEL_MAX_LEVELS + 1] = {};
  // ghost tables of the FP32 levels under the homogeneous rule
  int2* d_gtab32_[ANEL_MAX_LEVELS + 1] = {nullptr};
  // ghost copies done by the partitioned z-line sweep itself (null: the
  // level keeps its boundary pass after each colour); see SegFac
  int* d_img32_[ANEL_MAX_LEVELS + 1] = {nullptr};
  int zcode_[ANEL_MAX_LEVELS + 1][2] = {};
  int build_self_ghosting(int l);
  SegFac<float> segfac32(int l) const;
  int build_zline_factors();
  unsigned long long* d_max_ = nullptr;   // 2 words
  double* d_part_ = nullptr;              // norm partials
  double* d_norm_ = nullptr;              // 2 doubles
  double* d_io_phi_ = nullptr;            // staging for host-pointer solves
  double* d_io_rhs_ = nullptr;
  double* h_pin_ = nullptr;               // pinned small readback (4 doubles)
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
  // profiling of finest-level smoother launches
  bool prof_ = false;
  std::vector<cudaEvent_t> prof_ev_;
  size_t prof_n_ = 0;  // events used in the current solve (pairs)
  void prof_begin(cudaStream_t s);
  void prof_end(cudaStream_t s);
  int prof_collect(anel_mg_report* r);
  DevLevel<double> L64(int l) const;
  DevLevel<float> L32(int l, bool hom) const;
};

}  // namespace anel
