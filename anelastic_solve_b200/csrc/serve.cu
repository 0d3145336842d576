// serve.cu -- continuous-batching serving engine for ensembles of
// independent shear-layer members (many short runs of uneven grid sizes).
// It has no counterpart in the reference, where every run is its own job.
//
// Design:
//   * requests enter a FIFO queue (anel_serve_submit returns at once);
//   * max_active worker threads each drive one cohort: the members of one
//     bucket stepping together.  A worker takes the oldest queued member
//     whose bucket has no cohort running, sets it up (state, initial
//     projection) and, when its multigrid is the column-layout mixed
//     z-line cycle, opens a cohort for its bucket; at every step boundary
//     the cohort admits the bucket's newly queued members (up to
//     kMaxCohort) and retires those that are done, and one step of all
//     members is NSSolver::step_cohort: the members' own kernels, and each
//     sub-step's pressure solves as one batched multigrid solve (every
//     kernel of the cycle over all members, one CUDA graph per batch
//     size).  Other members run alone on their own stream.  Workers of
//     different buckets overlap on the device;
//   * a member is admitted when the device memory it needs fits the HBM
//     budget: an idle context of the same bucket (same grid, models,
//     multigrid and boundary setup) is re-used without allocating;
//     otherwise idle contexts of other buckets are released, least recently
//     used first, until the new context fits;
//   * contexts stay resident between members of their bucket (fields,
//     multigrid hierarchy, factor caches, ghost tables);
//   * standalone pressure solves (ANEL_INIT_POISSON) of one bucket are
//     solved together, up to kMaxCohort right-hand sides per batched solve;
//   * results (status, queue/run/total latency) are collected by
//     anel_serve_poll.
// A member's arithmetic does not depend on what else runs: its kernels
// read and write only its own buffers, and in a batched solve every kernel
// takes each member's work in the one-member order, so its fields are
// bit-identical alone and in the mix.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <vector>

#include "ns_solver.h"

namespace anel {

using Clock = std::chrono::steady_clock;

static double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

static uint64_t fnv1a(const void* p, size_t n, uint64_t h) {
  const unsigned char* c = static_cast<const unsigned char*>(p);
  for (size_t i = 0; i < n; ++i) {
    h ^= c[i];
    h *= 1099511628211ull;
  }
  return h;
}

struct ServeJob {
  int64_t id = 0;
  anel_request req{};
  anel_grid_desc grid{};
  std::vector<double> metric;  // owned copies of the 18 metric arrays
  anel_fields fin{}, fout{};
  bool has_in = false, has_out = false;
  Clock::time_point t_submit;
  std::string key;
  int64_t est_bytes = 0;
};

struct ServeCtx {
  NSSolver* s = nullptr;
  std::string key;
  int64_t bytes = 0;
  Clock::time_point last_used;
};

constexpr int kMaxCohort = 16;  // members per cohort (batched solve size)

// a member being served: its job, context, progress and result
struct Running {
  ServeJob* job = nullptr;
  ServeCtx* ctx = nullptr;
  bool need_new = false;
  int done = 0;
  anel_result res{};
  anel_step_report rep{};
  Clock::time_point t0;
};

class ServeEngine {
 public:
  int init(int device, int64_t budget, int max_active) {
    if (budget <= 0 || max_active < 1) {
      set_error("serve: budget must be positive and max_active >= 1");
      return ANEL_ERR_ARG;
    }
    device_ = device;
    budget_ = budget;
    ANEL_CUDA_TRY(cudaSetDevice(device_));
    for (int t = 0; t < max_active; ++t) threads_.emplace_back([this] { worker(); });
    return ANEL_OK;
  }

  ~ServeEngine() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_work_.notify_all();
    for (auto& t : threads_) t.join();
    cudaSetDevice(device_);
    for (ServeCtx* c : idle_) {
      delete c->s;
      delete c;
    }
    for (ServeJob* j : queue_) delete j;
  }

  int submit(const anel_request* r, int64_t* id) {
    if (!r) {
      set_error("serve: null request");
      return ANEL_ERR_ARG;
    }
    const anel_grid_desc& g = r->grid;
    if (g.nx < 1 || g.ny < 1 || g.nz < 1 || r->nsteps < 0) {
      set_error("serve: bad grid sizes or step count");
      return ANEL_ERR_ARG;
    }
    if (r->init != ANEL_INIT_SHEAR && !(r->init == ANEL_INIT_FIELDS && r->fields_in) &&
        !(r->init == ANEL_INIT_POISSON && r->fields_in && r->fields_in->psrc)) {
      set_error("serve: init must be ANEL_INIT_SHEAR, ANEL_INIT_FIELDS with fields_in, or "
                "ANEL_INIT_POISSON with fields_in->psrc");
      return ANEL_ERR_ARG;
    }
    auto* job = new ServeJob();
    job->req = *r;
    // own copies of the metric arrays (the caller's may go away)
    const int n[3] = {g.nx, g.ny, g.nz};
    const double* src[18] = {g.xe, g.xc, g.dxe, g.dxc, g.rdxe, g.rdxc, g.ye, g.yc, g.dye,
                             g.dyc, g.rdye, g.rdyc, g.ze, g.zc, g.dze, g.dzc, g.rdze, g.rdzc};
    size_t tot = 0;
    for (int a = 0; a < 18; ++a) {
      if (!src[a]) {
        delete job;
        set_error("serve: grid metric array %d is null", a);
        return ANEL_ERR_ARG;
      }
      tot += n[a / 6] + 2;
    }
    job->metric.resize(tot);
    const double** dst[18] = {&job->grid.xe, &job->grid.xc, &job->grid.dxe, &job->grid.dxc,
                              &job->grid.rdxe, &job->grid.rdxc, &job->grid.ye, &job->grid.yc,
                              &job->grid.dye, &job->grid.dyc, &job->grid.rdye, &job->grid.rdyc,
                              &job->grid.ze, &job->grid.zc, &job->grid.dze, &job->grid.dzc,
                              &job->grid.rdze, &job->grid.rdzc};
    job->grid.nx = g.nx;
    job->grid.ny = g.ny;
    job->grid.nz = g.nz;
    job->grid.xL = g.xL;
    job->grid.yL = g.yL;
    job->grid.zL = g.zL;
    size_t off = 0;
    uint64_t h = 1469598103934665603ull;
    for (int a = 0; a < 18; ++a) {
      const size_t len = n[a / 6] + 2;
      std::memcpy(job->metric.data() + off, src[a], len * sizeof(double));
      *dst[a] = job->metric.data() + off;
      h = fnv1a(src[a], len * sizeof(double), h);
      off += len;
    }
    if (r->fields_in) {
      job->fin = *r->fields_in;
      job->has_in = true;
    }
    if (r->fields_out) {
      job->fout = *r->fields_out;
      job->has_out = true;
    }
    // bucket: grid, multigrid setup, models, edge flag, boundary tables and
    // the kind of initial state (a context that took caller fields may
    // carry a non-unit density)
    const anel_ns_params& nk = r->ns;
    h = fnv1a(&r->mg, sizeof(r->mg), h);
    h = fnv1a(nk.tb, sizeof(nk.tb), h);
    h = fnv1a(nk.vb, sizeof(nk.vb), h);
    const int flags[6] = {nk.vmodel, nk.rmodel, nk.smodel, nk.ew, r->init, 0};
    h = fnv1a(flags, sizeof(flags), h);
    // the dynamic models' filter setup is fixed per context
    h = fnv1a(&nk.test_ratio, sizeof(nk.test_ratio), h);
    h = fnv1a(nk.filt, sizeof(nk.filt), h);
    h = fnv1a(nk.stretched, sizeof(nk.stretched), h);
    h = fnv1a(&nk.interp, sizeof(nk.interp), h);
    job->key = std::to_string(g.nx) + "x" + std::to_string(g.ny) + "x" + std::to_string(g.nz) + ":" +
               std::to_string(h);
    // device memory of a context: FP64 fields (14, +3 eddy fields, +2
    // LES-CN scratch), multigrid (FP64 fine pair, FP32 levels) and slack
    const int64_t G = (int64_t)(g.nx + 2) * (g.ny + 2) * (g.nz + 2);
    const bool les_any = nk.vmodel != ANEL_MODEL_DNS || nk.rmodel != ANEL_MODEL_DNS ||
                         nk.smodel != ANEL_MODEL_DNS;
    const bool dyn = nk.vmodel == ANEL_MODEL_DSM || nk.rmodel == ANEL_MODEL_DSM || nk.smodel == ANEL_MODEL_DSM;
    // (+16 scratch fields of the dynamic models)
    const int nf = 14 + (les_any ? 3 : 0) + (nk.vmodel != ANEL_MODEL_DNS ? 2 : 0) + (dyn ? 16 : 0);
    const int64_t mgb = r->mg.precision == ANEL_PREC_MIXED ? 32 : 24;
    job->est_bytes = G * (8 * nf + mgb) + ((int64_t)64 << 20);
    // a Poisson request holds its FP64 phi and right-hand side on the
    // device and one member's FP32 levels in its bucket's batch solver
    if (r->init == ANEL_INIT_POISSON) job->est_bytes = G * (16 + 16) + ((int64_t)1 << 20);
    std::lock_guard<std::mutex> lk(mu_);
    job->id = next_id_++;
    job->t_submit = Clock::now();
    if (id) *id = job->id;
    queue_.push_back(job);
    ++submitted_;
    cv_work_.notify_one();
    return ANEL_OK;
  }

  int poll(anel_result* out, int cap, int* n, int wait_ms) {
    std::unique_lock<std::mutex> lk(mu_);
    if (results_.empty() && wait_ms > 0)
      cv_done_.wait_for(lk, std::chrono::milliseconds(wait_ms), [this] { return !results_.empty(); });
    int k = 0;
    while (k < cap && !results_.empty()) {
      out[k++] = results_.front();
      results_.pop_front();
    }
    if (n) *n = k;
    return ANEL_OK;
  }

  int drain() {
    std::unique_lock<std::mutex> lk(mu_);
    cv_done_.wait(lk, [this] { return queue_.empty() && active_ == 0; });
    return ANEL_OK;
  }

  void stats(anel_serve_stats* st) {
    std::lock_guard<std::mutex> lk(mu_);
    st->submitted = submitted_;
    st->completed = completed_;
    st->failed = failed_;
    st->bytes_in_use = used_;
    st->peak_bytes = peak_;
    st->active = active_;
    st->peak_active = peak_active_;
    st->contexts = contexts_;
    st->queued = (int32_t)queue_.size();
    st->peak_cohort = peak_cohort_;
  }

 private:
  // Admit the head of the queue if it fits (mu_ held).  Returns the job and
  // sets ctx (a re-used idle context) or need_new (budget reserved).
  ServeJob* admit(ServeCtx*& ctx, bool& need_new, const std::string* only = nullptr) {
    // the oldest job of bucket *only, or (only null) the oldest job whose
    // bucket has no cohort running (a running cohort takes its bucket's
    // jobs at its next step boundary)
    auto pick = std::find_if(queue_.begin(), queue_.end(), [&](ServeJob* j) {
      return only ? j->key == *only : cohorts_.count(j->key) == 0;
    });
    if (pick == queue_.end()) return nullptr;
    ServeJob* head = *pick;
    auto it = std::find_if(idle_.begin(), idle_.end(), [&](ServeCtx* c) { return c->key == head->key; });
    if (it != idle_.end()) {
      ctx = *it;
      idle_.erase(it);
      queue_.erase(pick);
      return head;
    }
    while (used_ + head->est_bytes > budget_ && !idle_.empty()) {
      auto lru = std::min_element(idle_.begin(), idle_.end(),
                                  [](ServeCtx* a, ServeCtx* b) { return a->last_used < b->last_used; });
      ServeCtx* c = *lru;
      idle_.erase(lru);
      used_ -= c->bytes;
      --contexts_;
      delete c->s;
      delete c;
    }
    if (used_ + head->est_bytes <= budget_) {
      used_ += head->est_bytes;
      peak_ = std::max(peak_, used_);
      need_new = true;
      queue_.erase(pick);
      return head;
    }
    return nullptr;
  }

  void worker() {
    cudaSetDevice(device_);
    for (;;) {
      Running* r = new Running();
      {
        std::unique_lock<std::mutex> lk(mu_);
        for (;;) {
          if (!queue_.empty()) {
            r->job = admit(r->ctx, r->need_new);
            if (r->job) break;
            if (active_ == 0 && cohorts_.empty()) {
              // does not fit even with the device to itself
              ServeJob* head = queue_.front();
              queue_.pop_front();
              anel_result res{};
              res.id = head->id;
              res.status = ANEL_ERR_NOMEM;
              res.nsteps = head->req.nsteps;
              results_.push_back(res);
              ++failed_;
              delete head;
              cv_done_.notify_all();
              continue;
            }
          } else if (stop_) {
            delete r;
            return;
          }
          cv_work_.wait(lk);
        }
        ++active_;
        peak_active_ = std::max(peak_active_, active_);
      }
      if (r->job->req.init == ANEL_INIT_POISSON) {
        run_poisson(r);
        continue;
      }
      int st = setup(*r);
      if (st == ANEL_OK && r->job->req.nsteps > 0 && r->ctx->s->mg()->batch_capable()) {
        run_cohort(r);
        continue;
      }
      if (st == ANEL_OK && r->job->req.nsteps > 0) {
        st = r->ctx->s->step(r->job->req.nsteps, r->ctx->s->stream(), &r->rep);
        r->done = r->job->req.nsteps;
      }
      finish(r, st);
    }
  }

  // Context (new or re-used), reset, initial state and initial projection
  // of a member, on its own stream.
  int setup(Running& r) {
    ServeJob& job = *r.job;
    r.t0 = Clock::now();
    r.res.id = job.id;
    r.res.queue_ms = ms_between(job.t_submit, r.t0);
    r.res.nsteps = job.req.nsteps;
    r.res.cells = (int64_t)job.grid.nx * job.grid.ny * job.grid.nz;
    int st = ANEL_OK;
    if (r.need_new) {
      NSSolver* s = NSSolver::create(&job.grid, &job.req.mg, &job.req.ns, device_, &st);
      if (!s) return st;
      r.ctx = new ServeCtx{s, job.key, job.est_bytes, r.t0};
      r.need_new = false;
      std::lock_guard<std::mutex> lk(mu_);
      ++contexts_;
    }
    NSSolver* s = r.ctx->s;
    cudaStream_t sm = s->stream();
    st = s->reset(&job.req.ns, sm);
    if (st == ANEL_OK) {
      if (job.req.init == ANEL_INIT_SHEAR) st = s->init_shear(job.req.seed, job.req.amp, 2.0, sm);
      else st = s->set_fields(&job.fin, ANEL_MEM_HOST, sm);
    }
    int it = 0;
    double rm = 0.0;
    if (st == ANEL_OK) st = s->project(sm, &it, &rm);
    if (st == ANEL_ERR_NOCONV) st = ANEL_OK;
    return st;
  }

  // Fields out, result, context back to the idle pool (or freed on error).
  void finish(Running* r, int st) {
    ServeJob& job = *r->job;
    if (st == ANEL_OK && job.has_out) st = r->ctx->s->get_fields(&job.fout, ANEL_MEM_HOST, r->ctx->s->stream());
    const Clock::time_point t1 = Clock::now();
    r->res.status = st;
    r->res.run_ms = ms_between(r->t0, t1);
    r->res.latency_ms = ms_between(job.t_submit, t1);
    r->res.dt_last = r->rep.dt;
    r->res.max_div = r->rep.max_div;
    {
      std::lock_guard<std::mutex> lk(mu_);
      --active_;
      ServeCtx* ctx = r->ctx;
      if (ctx) {
        if (st == ANEL_OK) {
          ctx->last_used = Clock::now();
          idle_.push_back(ctx);
        } else {
          used_ -= ctx->bytes;
          --contexts_;
          delete ctx->s;
          delete ctx;
        }
      } else if (r->need_new) {
        used_ -= job.est_bytes;
      }
      results_.push_back(r->res);
      if (st == ANEL_OK) ++completed_;
      else ++failed_;
      delete r->job;
    }
    delete r;
    cv_work_.notify_all();
    cv_done_.notify_all();
  }

  // Standalone pressure solves of the first request's bucket: every pass
  // takes the bucket's queued requests (up to kMaxCohort, admitted against
  // the budget), copies their right-hand sides and guesses in, solves them
  // as one batched multigrid solve (one at a time where the multigrid is
  // not the column-layout mixed cycle) and copies the solutions out.
  void run_poisson(Running* first) {
    const std::string key = first->job->key;
    int st = ANEL_OK;
    MGSolver* mg = MGSolver::create(&first->job->grid, &first->job->req.mg, device_, &st);
    const int64_t G = (int64_t)(first->job->grid.nx + 2) * (first->job->grid.ny + 2) *
                      (first->job->grid.nz + 2);
    const int64_t mbytes = G * (24 + 16) + ((int64_t)64 << 20);  // the solver's own arrays
    {
      std::lock_guard<std::mutex> lk(mu_);
      cohorts_.insert(key);
      used_ += mbytes;
      peak_ = std::max(peak_, used_);
    }
    cudaStream_t sm = mg ? mg->stream() : nullptr;
    std::vector<double*> dbuf;  // 2 G-sized device arrays per slot (phi, rhs)
    std::vector<Running*> mem{first};
    for (;;) {
      if (!mg || st != ANEL_OK) {
        for (Running* r : mem) finish_poisson(r, st != ANEL_OK ? st : ANEL_ERR_CUDA);
        mem.clear();
      } else {
        // admit the bucket's queued requests
        while ((int)mem.size() < kMaxCohort) {
          Running* r = new Running();
          {
            std::lock_guard<std::mutex> lk(mu_);
            r->job = queue_.empty() ? nullptr : admit(r->ctx, r->need_new, &key);
            if (r->job) {
              ++active_;
              peak_active_ = std::max(peak_active_, active_);
            }
          }
          if (!r->job) {
            delete r;
            break;
          }
          mem.push_back(r);
        }
      }
      if (mem.empty()) {
        std::lock_guard<std::mutex> lk(mu_);
        const bool more = std::any_of(queue_.begin(), queue_.end(), [&](ServeJob* j) { return j->key == key; });
        if (!more || !mg || st != ANEL_OK) {
          cohorts_.erase(key);
          used_ -= mbytes;
          break;
        }
        continue;
      }
      {
        std::lock_guard<std::mutex> lk(mu_);
        peak_cohort_ = std::max(peak_cohort_, (int)mem.size());
      }
      const int n = (int)mem.size();
      int sb = ANEL_OK;
      while ((int)dbuf.size() < 2 * n && sb == ANEL_OK) {
        double* a = nullptr;
        if (cudaMalloc(&a, G * sizeof(double)) != cudaSuccess) {
          cudaGetLastError();
          sb = ANEL_ERR_NOMEM;
        } else {
          dbuf.push_back(a);
        }
      }
      std::vector<double*> phis(n);
      std::vector<const double*> rhss(n);
      std::vector<anel_mg_report> reps(n);
      const size_t fb = G * sizeof(double);
      for (int b = 0; b < n && sb == ANEL_OK; ++b) {
        Running* r = mem[b];
        r->t0 = Clock::now();
        phis[b] = dbuf[2 * b];
        rhss[b] = dbuf[2 * b + 1];
        const anel_fields& in = r->job->fin;
        const cudaError_t e1 = in.p ? cudaMemcpyAsync(phis[b], in.p, fb, cudaMemcpyHostToDevice, sm)
                                    : cudaMemsetAsync(phis[b], 0, fb, sm);
        const cudaError_t e2 = cudaMemcpyAsync(dbuf[2 * b + 1], in.psrc, fb, cudaMemcpyHostToDevice, sm);
        if (e1 != cudaSuccess || e2 != cudaSuccess) sb = ANEL_ERR_CUDA;
      }
      if (sb == ANEL_OK) {
        if (mg->batch_capable()) {
          sb = mg->solve_batch(n, phis.data(), rhss.data(), sm, reps.data());
        } else {
          for (int b = 0; b < n && (sb == ANEL_OK || sb == ANEL_ERR_NOCONV); ++b) {
            const int s1 = mg->solve_device(phis[b], rhss[b], sm, &reps[b]);
            reps[b].status = s1;
            if (s1 != ANEL_OK && s1 != ANEL_ERR_NOCONV) sb = s1;
          }
        }
        if (sb == ANEL_ERR_NOCONV) sb = ANEL_OK;  // the members' own status is in their reports
      }
      for (int b = 0; b < n; ++b) {
        Running* r = mem[b];
        int s1 = sb;
        if (s1 == ANEL_OK) {
          r->res.mg_iter = reps[b].iter;
          r->res.resid = reps[b].resid;
          if (reps[b].status != ANEL_OK) s1 = reps[b].status;
          if (r->job->has_out && r->job->fout.p &&
              cudaMemcpyAsync(r->job->fout.p, phis[b], fb, cudaMemcpyDeviceToHost, sm) != cudaSuccess)
            s1 = ANEL_ERR_CUDA;
        }
        if (sm && cudaStreamSynchronize(sm) != cudaSuccess && s1 == ANEL_OK) s1 = ANEL_ERR_CUDA;
        finish_poisson(r, s1);
      }
      mem.clear();
    }
    if (mg) cudaStreamSynchronize(mg->stream());
    for (double* a : dbuf) cudaFree(a);
    delete mg;
    cv_work_.notify_all();
  }

  // the result of a Poisson request (no stepping context to return)
  void finish_poisson(Running* r, int st) {
    ServeJob& job = *r->job;
    const Clock::time_point t1 = Clock::now();
    if (r->t0 == Clock::time_point()) r->t0 = t1;
    r->res.id = job.id;
    r->res.status = st;
    r->res.cells = (int64_t)job.grid.nx * job.grid.ny * job.grid.nz;
    r->res.queue_ms = ms_between(job.t_submit, r->t0);
    r->res.run_ms = ms_between(r->t0, t1);
    r->res.latency_ms = ms_between(job.t_submit, t1);
    {
      std::lock_guard<std::mutex> lk(mu_);
      --active_;
      if (r->need_new) used_ -= job.est_bytes;
      results_.push_back(r->res);
      if (st == ANEL_OK) ++completed_;
      else ++failed_;
      delete r->job;
    }
    delete r;
    cv_work_.notify_all();
    cv_done_.notify_all();
  }

  // A cohort of the first member's bucket: one step of every member per
  // pass of the loop (NSSolver::step_cohort with the bucket's batch
  // solver), members admitted and retired at step boundaries, until the
  // bucket runs dry.
  void run_cohort(Running* first) {
    const std::string key = first->job->key;
    int st = ANEL_OK;
    MGSolver* bmg = MGSolver::create(&first->job->grid, &first->job->req.mg, device_, &st);
    const int64_t G = (int64_t)(first->job->grid.nx + 2) * (first->job->grid.ny + 2) * (first->job->grid.nz + 2);
    // the batch solver: its own levels plus kMaxCohort members' FP32 levels
    const int64_t bbytes = G * (24 + 16 * (1 + kMaxCohort)) + ((int64_t)64 << 20);
    bool fits = false;
    {
      std::lock_guard<std::mutex> lk(mu_);
      fits = used_ + bbytes <= budget_;
      if (fits) {
        cohorts_.insert(key);
        used_ += bbytes;
        peak_ = std::max(peak_, used_);
      }
    }
    if (fits && bmg && st == ANEL_OK) st = bmg->batch_reserve(kMaxCohort);
    if (!fits || !bmg || st != ANEL_OK) {
      // no room for a batch solver: the member runs alone
      delete bmg;
      if (fits) {
        std::lock_guard<std::mutex> lk(mu_);
        cohorts_.erase(key);
        used_ -= bbytes;
      }
      const int s2 = first->ctx->s->step(first->job->req.nsteps, first->ctx->s->stream(), &first->rep);
      first->done = first->job->req.nsteps;
      finish(first, s2);
      cv_work_.notify_all();
      return;
    }
    std::vector<Running*> mem{first};
    for (;;) {
      // admit the bucket's queued members (each set up on its own stream)
      for (;;) {
        if ((int)mem.size() >= kMaxCohort) break;
        Running* r = new Running();
        {
          std::lock_guard<std::mutex> lk(mu_);
          r->job = queue_.empty() ? nullptr : admit(r->ctx, r->need_new, &key);
          if (r->job) {
            ++active_;
            peak_active_ = std::max(peak_active_, active_);
          }
        }
        if (!r->job) {
          delete r;
          break;
        }
        const int s1 = setup(*r);
        if (s1 != ANEL_OK || r->job->req.nsteps == 0) finish(r, s1);
        else mem.push_back(r);
      }
      if (mem.empty()) {
        std::lock_guard<std::mutex> lk(mu_);
        const bool more = std::any_of(queue_.begin(), queue_.end(), [&](ServeJob* j) { return j->key == key; });
        if (!more) {
          cohorts_.erase(key);
          used_ -= bbytes;
          break;
        }
        continue;
      }
      {
        std::lock_guard<std::mutex> lk(mu_);
        peak_cohort_ = std::max(peak_cohort_, (int)mem.size());
      }
      std::vector<NSSolver*> ms(mem.size());
      std::vector<anel_step_report> reps(mem.size());
      for (size_t b = 0; b < mem.size(); ++b) ms[b] = mem[b]->ctx->s;
      const int sc = NSSolver::step_cohort(ms.data(), (int)ms.size(), 1, bmg, bmg->stream(), reps.data());
      std::vector<Running*> keep;
      for (size_t b = 0; b < mem.size(); ++b) {
        Running* r = mem[b];
        r->rep = reps[b];
        ++r->done;
        if (sc != ANEL_OK) finish(r, sc);
        else if (r->done >= r->job->req.nsteps) finish(r, ANEL_OK);
        else keep.push_back(r);
      }
      mem.swap(keep);
    }
    delete bmg;
    cv_work_.notify_all();
  }

  std::mutex mu_;
  std::condition_variable cv_work_, cv_done_;
  std::deque<ServeJob*> queue_;
  std::vector<ServeCtx*> idle_;
  std::deque<anel_result> results_;
  std::vector<std::thread> threads_;
  int device_ = 0;
  int64_t budget_ = 0, used_ = 0, peak_ = 0;
  int active_ = 0, peak_active_ = 0, contexts_ = 0;
  int64_t submitted_ = 0, completed_ = 0, failed_ = 0, next_id_ = 1;
  bool stop_ = false;
  std::set<std::string> cohorts_;  // buckets with a cohort running
  int peak_cohort_ = 0;
};

}  // namespace anel

struct anel_serve {
  anel::ServeEngine* e;
};

extern "C" {

anel_serve* anel_serve_create(int32_t device, int64_t hbm_budget_bytes, int32_t max_active,
                              int32_t* status) {
  auto* e = new anel::ServeEngine();
  const int st = e->init(device, hbm_budget_bytes, max_active);
  if (status) *status = st;
  if (st != ANEL_OK) {
    delete e;
    return nullptr;
  }
  return new anel_serve{e};
}

int anel_serve_submit(anel_serve* e, const anel_request* req, int64_t* id) {
  if (!e) return ANEL_ERR_ARG;
  return e->e->submit(req, id);
}

int anel_serve_poll(anel_serve* e, anel_result* out, int32_t cap, int32_t* n, int32_t wait_ms) {
  if (!e || (!out && cap > 0)) return ANEL_ERR_ARG;
  int k = 0;
  const int st = e->e->poll(out, cap, &k, wait_ms);
  if (n) *n = k;
  return st;
}

int anel_serve_drain(anel_serve* e) {
  if (!e) return ANEL_ERR_ARG;
  return e->e->drain();
}

int anel_serve_stats_get(anel_serve* e, anel_serve_stats* st) {
  if (!e || !st) return ANEL_ERR_ARG;
  e->e->stats(st);
  return ANEL_OK;
}

void anel_serve_destroy(anel_serve* e) {
  if (!e) return;
  delete e->e;
  delete e;
}

}  // extern "C"
