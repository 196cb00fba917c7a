// Request server: runs of different programs and sizes admitted by device-memory
// budget and stepped side by side (continuous batching).
//
// The reference runs one solver per process (solver_stepping.jl:115-205); the
// serving pattern is new here.  A worker thread owns all GPU work:
//   - admission, in arrival order: the next queued request starts when its
//     estimated device bytes fit the remaining budget and a run slot is free;
//     it gets its own plan and stream;
//   - progress: every running request keeps two chunks of steps (one CUDA
//     graph launch each) queued on its own stream, the next behind the
//     running one, so the chunks of all running requests overlap on the
//     device, no stream waits for this loop to come round, and a request
//     that arrives while others run joins as soon as memory frees up;
//   - completion: the final state is copied to host memory, the plan and its
//     device memory are released, and the time from submission is recorded.
//   - cohorts (tb_server_set_cohort; off by default): RBC requests of one
//     shape (grid, box, walls, stepper, precision) and one dt, with step
//     counts within 25 % of each other, that are queued together are
//     admitted as one run of a stacked plan (the ensemble's fused form: each member's modes are
//     columns of one plan, with its own kappa / nu), stepped by one graph per
//     chunk; each member leaves with its state copied out of its columns when
//     its own step count is reached (the chunks stop at that count), the
//     others step on.
// A request run alone has exactly its arithmetic on its own; in a cohort its
// solves and transforms run in kernels over the stacked columns, which
// changes only the rounding (within 1e-12).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "tb_plan.h"
#include "tb_turb.h"

using namespace tb;

namespace {

// Host threads building admitted requests' plans: half the host's hardware
// threads, 4 to 16 (plan construction is host work that overlaps the steps).
constexpr int kChunksAhead = 2;  // graph launches queued per running request

int setup_threads() {
  const unsigned hw = std::thread::hardware_concurrency();
  return (int)std::max(4u, std::min(16u, hw / 2));
}

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

// One admitted run on the device.
struct Job {
  virtual ~Job() = default;
  virtual cudaStream_t stream() const = 0;
  virtual void launch(double dt, int steps) = 0;
  virtual size_t device_bytes() const = 0;
  virtual int nfields() const = 0;
  virtual size_t field_doubles(int field) const = 0;
  virtual void fetch(int field, double* host) = 0;
  // factors and step graphs built before the first launch
  virtual void prepare(double dt, int chunk) = 0;
};

struct RbcJob : Job {
  tb_plan* P = nullptr;
  ~RbcJob() override {
    if (P) tb_plan_destroy(P);
  }
  cudaStream_t stream() const override { return P->st; }
  void launch(double dt, int steps) override { plan_launch_steps(P, dt, steps, P->st, steps); }
  size_t device_bytes() const override { return plan_device_bytes(P); }
  int nfields() const override { return 3; }  // b, u_x, u_z coefficients
  size_t field_doubles(int) const override { return 2 * P->plane; }
  void fetch(int field, double* host) override {
    TB_CUDA_TRY(cudaMemcpyAsync(host, P->Xp(field), P->plane * sizeof(double2), cudaMemcpyDeviceToHost, P->st));
    TB_CUDA_TRY(cudaStreamSynchronize(P->st));
  }
  void prepare(double dt, int chunk) override { plan_prepare(P, dt, chunk); }
};

// Same-shape RBC requests stacked into one plan (build_plan with B instances).
struct CohortJob : Job {
  std::unique_ptr<tb_plan> P;
  cudaStream_t stream() const override { return P->st; }
  void launch(double dt, int steps) override { plan_launch_steps(P.get(), dt, steps, P->st, steps); }
  size_t device_bytes() const override { return plan_device_bytes(P.get()); }
  int nfields() const override { return 3; }
  size_t field_doubles(int) const override { return (size_t)2 * P->Nz * P->Nkm; }
  // member k's columns of field f, as its own plan would hold them ([Nz][Nkm])
  void fetch_member(int k, int field, double* host) {
    const size_t w = (size_t)P->Nkm * sizeof(double2);
    TB_CUDA_TRY(cudaMemcpy2DAsync(host, w, P->Xp(field) + (size_t)k * P->Nkm, (size_t)P->Nk * sizeof(double2), w,
                                  P->Nz, cudaMemcpyDeviceToHost, P->st));
    TB_CUDA_TRY(cudaStreamSynchronize(P->st));
  }
  void fetch(int field, double* host) override { fetch_member(0, field, host); }
  void prepare(double dt, int chunk) override { plan_prepare(P.get(), dt, chunk); }
};

struct TurbJob : Job {
  tb_turb* T = nullptr;
  ~TurbJob() override {
    if (T) turb_destroy(T);
  }
  cudaStream_t stream() const override { return turb_stream(T); }
  void launch(double dt, int steps) override { turb_launch_steps(T, dt, steps); }
  size_t device_bytes() const override { return turb_device_bytes(T); }
  int nfields() const override { return 1; }  // vorticity coefficients
  size_t field_doubles(int) const override { return turb_field_doubles(T); }
  void fetch(int, double* host) override { turb_fetch(T, host); }
  void prepare(double dt, int) override { turb_prepare(T, dt); }
};

// Device bytes a run of this size will hold (plan, factors, graphs' scratch).
size_t estimate_bytes(const tb_problem_desc& d) {
  if (d.program == TB_PROGRAM_TURB2D) return turb_estimate_bytes(d.Nx, d.Ny, d.timestepper);
  const size_t nk = d.Nx / 2 + 1, plane = (size_t)d.Nz * nk * 16;
  const size_t npad = ((size_t)2 * d.Nz + kTauRowPad - 1) / kTauRowPad * kTauRowPad;
  const size_t groups = (nk + kSolveModes - 1) / kSolveModes;
  const size_t rec = groups * npad * 2 * kSolveModes * (kFwdRec + kBwdRec + kHRec) * 8;
  const size_t work = plane * (4 + 6 + 3 + 4 + 4 * 4 * 2 + 3 * 4 + 1) + (size_t)d.Nz * d.Nz * 8 * 8;
  return rec + work + (16u << 20);
}

struct Request {
  long long id = 0;
  tb_problem_desc desc{};
  double dt = 0;
  int nsteps = 0, left = 0;
  std::vector<double> init;
  double t_submit = 0, t_start = 0, t_ready = 0, t_done = 0;
  int state = TB_REQ_QUEUED;
  std::string error;
  size_t bytes = 0;
  std::unique_ptr<Job> job;
  // chunks in flight on the request's stream: up to kChunksAhead, each
  // followed by an event (ev[head] marks the oldest)
  cudaEvent_t ev[2] = {nullptr, nullptr};
  int inflight = 0, head = 0;
  std::vector<std::vector<double>> result;
  // cohort leader: every member (itself first) and, per member, whether its
  // result has been taken; `hold` stops new chunks until the in-flight ones
  // retire (a member reached its step count)
  std::vector<Request*> cohort;
  std::vector<bool> finished;
  bool hold = false;
  Request* leader = nullptr;  // members other than the leader
  bool solo = false;          // runs alone (its cohort's stacked plan could not be built)
};

// Requests that can share one stacked plan.
bool cohort_fusible(const Request& r) {
  return r.desc.program == TB_PROGRAM_RBC && r.desc.ndim == 2 && !r.solo;
}
// A stacked run steps every column until its longest member is done, so
// members join only with step counts within 25 % of each other.
bool cohort_compatible(const Request& a, const Request& b) {
  const tb_problem_desc &x = a.desc, &y = b.desc;
  const int lo = std::min(a.nsteps, b.nsteps), hi = std::max(a.nsteps, b.nsteps);
  return cohort_fusible(a) && cohort_fusible(b) && a.dt == b.dt && x.Nx == y.Nx && x.Nz == y.Nz && x.Lx == y.Lx &&
         x.Lz == y.Lz && x.timestepper == y.timestepper && x.b_bottom == y.b_bottom && x.b_top == y.b_top &&
         x.precision == y.precision && 4 * hi <= 5 * lo;
}

}  // namespace

struct tb_server {
  tb_context* ctx = nullptr;
  size_t budget = 0;
  int max_running = 1, chunk = 1;
  int cohort_max = 1;  // members of one stacked run (1, the default: every request alone)
  std::mutex mu;
  std::condition_variable cv;
  std::deque<Request*> queue;     // submitted, not admitted
  std::deque<Request*> setupq;    // admitted, waiting for a setup thread
  int setting_up = 0;             // admitted, plan being built
  std::vector<Request*> running;
  std::condition_variable setup_cv;
  std::vector<std::thread> setup_workers;
  // Finished jobs keep their device memory until the budget needs it or the
  // server is idle: cudaFree waits for the whole device, so releasing memory
  // while other requests run would stall them all.
  std::vector<std::unique_ptr<Job>> zombies;
  size_t zombie_bytes = 0;
  std::map<long long, std::unique_ptr<Request>> all;
  long long next_id = 1;
  bool stop = false;
  std::thread worker;
  // statistics
  size_t used = 0, peak = 0;
  int peak_running = 0, peak_cohort = 1;
  long long cohort_requests = 0;
  long long completed = 0, failed = 0, steps_done = 0;
  double first_submit = -1, last_done = 0;
  std::vector<double> tts, waits, setups;

  void loop();
  void setup_loop();
  void admit();
  void progress();
  bool idle_locked() const { return queue.empty() && setupq.empty() && setting_up == 0 && running.empty(); }
  void release_zombies();
  void fail_admitted(Request* r, const std::string& msg);
  void fail_running(Request* r, const std::string& msg);
  void progress_cohort(Request* r);
  void finish_locked(Request* m);
  bool requeue_cohort(Request* r);
};

namespace {

// One stacked plan for the cohort's members: member k's modes are columns
// k Nkm .. (k+1) Nkm - 1; its initial b grid goes through the plan's x FFT and
// forward Chebyshev GEMM straight into its columns (u = 0).
std::unique_ptr<Job> make_cohort_job(tb_context* ctx, const std::vector<Request*>& members) {
  std::vector<tb_problem_desc> descs;
  for (const Request* m : members) descs.push_back(m->desc);
  auto j = std::make_unique<CohortJob>();
  j->P = std::make_unique<tb_plan>();
  build_plan(j->P.get(), ctx, descs.data(), (int)descs.size());
  tb_plan* P = j->P.get();
  if (plan_tau_parts_ok(P, 1)) plan_set_variant(P, 1, 0);  // the one-warp solve, as for single requests
  StreamBuf grid;
  grid.alloc((size_t)P->Nz * P->Nx * sizeof(double), P->st);
  TB_CUDA_TRY(cudaMemsetAsync(P->X.p, 0, P->X.bytes, P->st));
  const int Hp = (P->Hz + 15) / 16 * 16;
  for (size_t k = 0; k < members.size(); ++k) {
    TB_CUDA_TRY(cudaMemcpyAsync(grid.p, members[k]->init.data(), grid.bytes, cudaMemcpyHostToDevice, P->st));
    double2* mixed = P->tmpgrid.as<double2>();  // [Nz][Nkm]
    launch_x_rfft(grid.as<double>(), mixed, P->Nz, P->Nx, P->fpN, P->twN.as<double2>(), P->st);
    double* out = reinterpret_cast<double*>(P->Xp(0) + k * P->Nkm);
    GemmBatch bt{};
    bt.item[0] = GemmItem{P->fE.as<double>(), reinterpret_cast<const double*>(mixed), out, P->Ke, P->Hz, Hp,
                          GEMM_MIRROR, 0};
    bt.item[1] = GemmItem{P->fO.as<double>(), reinterpret_cast<const double*>(mixed), out, P->Ko, P->Hz, Hp,
                          GEMM_MIRROR, 1};
    launch_gemm_f64(bt, P->Ko > 0 ? 2 : 1, 2 * P->Nkm, 2 * P->Nkm, 2 * P->Nk, P->Nz, P->st);
    TB_CUDA_TRY(cudaGetLastError());
    // the staging grid is rewritten for the next member only after these ran
    TB_CUDA_TRY(cudaStreamSynchronize(P->st));
  }
  return j;
}

std::unique_ptr<Job> make_job(tb_context* ctx, const Request& r) {
  if (r.desc.program == TB_PROGRAM_TURB2D) {
    auto j = std::make_unique<TurbJob>();
    j->T = turb_create(ctx, r.desc, r.init.data());
    return j;
  }
  auto j = std::make_unique<RbcJob>();
  tb_status st = tb_plan_create(ctx, &r.desc, &j->P);
  if (st != TB_OK) throw Error{st, tb_last_error(nullptr)};  // this thread's message
  tb_plan* P = j->P;
  // Many requests share the device here, so the tau solves take the one-warp
  // form: its blocks need a fifth of the shared memory of the partitioned
  // form's, so several requests' solves share an SM instead of queueing for
  // whole SMs (the throughput choice the ensemble tuner also makes).
  if (plan_tau_parts_ok(P, 1)) plan_set_variant(P, 1, 0);
  // initial state: b from the grid field, u = 0
  StreamBuf grid, coeff;  // staging released in stream order: no device-wide wait
  grid.alloc(r.init.size() * sizeof(double), P->st);
  coeff.alloc(P->plane * sizeof(double2), P->st);
  TB_CUDA_TRY(cudaMemcpyAsync(grid.p, r.init.data(), grid.bytes, cudaMemcpyHostToDevice, P->st));
  st = tb_transform_forward(P, grid.as<double>(), coeff.as<double>(), 1);
  if (st != TB_OK) throw Error{st, tb_last_error(nullptr)};  // this thread's message
  TB_CUDA_TRY(cudaMemsetAsync(P->X.p, 0, P->X.bytes, P->st));
  TB_CUDA_TRY(cudaMemcpyAsync(P->Xp(0), coeff.p, coeff.bytes, cudaMemcpyDeviceToDevice, P->st));
  TB_CUDA_TRY(cudaStreamSynchronize(P->st));
  return j;
}

}  // namespace

// Admission: in arrival order, while the head's estimated bytes fit the
// remaining budget and a run slot is free; the plan is built by a setup
// thread so that host-side construction overlaps the steps of running requests.
void tb_server::admit() {
  std::lock_guard<std::mutex> lk(mu);
  while (!queue.empty() && (int)running.size() + setting_up + (int)setupq.size() < max_running) {
    Request* h = queue.front();
    if (h->bytes > budget) {  // can never fit
      queue.pop_front();
      h->state = TB_REQ_FAILED;
      h->error = "request needs more device memory than the server budget";
      ++failed;
      cv.notify_all();
      continue;
    }
    if (used + zombie_bytes + h->bytes > budget) {
      if (zombie_bytes == 0 || used + h->bytes > budget) return;  // wait for memory (arrival order)
      release_zombies();  // the finished jobs' memory makes room
      continue;
    }
    queue.pop_front();
    used += h->bytes;
    // cohort: later queued requests of h's shape and dt join it while they fit
    h->cohort.clear();
    if (cohort_max > 1 && cohort_fusible(*h)) {
      h->cohort.push_back(h);
      for (auto it = queue.begin(); it != queue.end() && (int)h->cohort.size() < cohort_max;) {
        Request* c = *it;
        if (cohort_compatible(*h, *c) && used + zombie_bytes + c->bytes <= budget) {
          used += c->bytes;
          c->leader = h;
          h->cohort.push_back(c);
          it = queue.erase(it);
        } else {
          ++it;
        }
      }
      if (h->cohort.size() < 2) h->cohort.clear();
    }
    peak = std::max(peak, used);
    setupq.push_back(h);
    setup_cv.notify_one();
  }
}

// (mu held)
void tb_server::release_zombies() {
  zombies.clear();
  zombie_bytes = 0;
}

void tb_server::setup_loop() {
  cudaSetDevice(ctx->device);
  while (true) {
    Request* r = nullptr;
    {
      std::unique_lock<std::mutex> lk(mu);
      // leave only when stopping with nothing left to admit, build or free
      setup_cv.wait(lk, [&] { return !setupq.empty() || (stop && queue.empty()); });
      if (setupq.empty()) return;
      r = setupq.front();
      setupq.pop_front();
      ++setting_up;
    }
    try {
      r->t_start = now_ms();
      r->job = r->cohort.empty() ? make_job(ctx, *r) : make_cohort_job(ctx, r->cohort);
      r->job->prepare(r->dt, chunk);
      for (auto& e : r->ev) TB_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      r->t_ready = now_ms();
      std::lock_guard<std::mutex> lk(mu);
      --setting_up;
      if (r->cohort.empty()) {
        setups.push_back(r->t_ready - r->t_start);
        r->state = TB_REQ_RUNNING;
      } else {
        r->finished.assign(r->cohort.size(), false);
        r->hold = false;
        peak_cohort = std::max(peak_cohort, (int)r->cohort.size());
        for (Request* m : r->cohort) {
          m->t_start = r->t_start;
          m->t_ready = r->t_ready;
          setups.push_back(r->t_ready - r->t_start);
          m->state = TB_REQ_RUNNING;
        }
      }
      running.push_back(r);
      peak_running = std::max(peak_running, (int)running.size());
    } catch (const Error& e) {
      if (!requeue_cohort(r)) {
        {
          std::lock_guard<std::mutex> lk(mu);
          --setting_up;
        }
        fail_admitted(r, e.msg);
      }
    } catch (const std::exception& e) {
      if (!requeue_cohort(r)) {
        {
          std::lock_guard<std::mutex> lk(mu);
          --setting_up;
        }
        fail_admitted(r, e.what());
      }
    }
  }
}

void tb_server::fail_admitted(Request* r, const std::string& msg) {
  r->job.reset();
  for (auto& e : r->ev) {
    if (e) cudaEventDestroy(e);
    e = nullptr;
  }
  std::lock_guard<std::mutex> lk(mu);
  std::vector<Request*> all_m = r->cohort.empty() ? std::vector<Request*>{r} : r->cohort;
  for (Request* m : all_m) {  // a cohort fails with its stacked plan
    used -= m->bytes;
    m->state = TB_REQ_FAILED;
    m->error = msg;
    ++failed;
  }
  cv.notify_all();
}

// A cohort whose stacked plan could not be built goes back to the head of the
// queue as single requests, so that each one succeeds or fails on its own.
bool tb_server::requeue_cohort(Request* r) {
  if (r->cohort.empty()) return false;
  r->job.reset();
  for (auto& e : r->ev) {
    if (e) cudaEventDestroy(e);
    e = nullptr;
  }
  std::lock_guard<std::mutex> lk(mu);
  --setting_up;
  std::vector<Request*> members = r->cohort;
  r->cohort.clear();
  for (auto it = members.rbegin(); it != members.rend(); ++it) {
    Request* m = *it;
    used -= m->bytes;
    m->solo = true;
    m->leader = nullptr;
    m->state = TB_REQ_QUEUED;
    queue.push_front(m);
  }
  cv.notify_all();
  return true;
}

// (mu held) statistics of a finished request
void tb_server::finish_locked(Request* m) {
  m->t_done = now_ms();
  m->state = TB_REQ_DONE;
  ++completed;
  steps_done += m->nsteps;
  last_done = m->t_done;
  tts.push_back(m->t_done - m->t_submit);
  waits.push_back(m->t_start - m->t_submit);
}

// A cohort's chunks step every member; a chunk never passes the step count
// of a member still running, and when one reaches its count no further chunk
// is queued until the in-flight ones retire and its columns are copied out.
void tb_server::progress_cohort(Request* r) {
  auto* job = static_cast<CohortJob*>(r->job.get());
  while (r->inflight > 0) {
    const cudaError_t e = cudaEventQuery(r->ev[r->head]);
    if (e == cudaErrorNotReady) {
      cudaGetLastError();
      break;
    }
    if (e != cudaSuccess) throw Error{TB_ECUDA, std::string("request stream: ") + cudaGetErrorString(e)};
    r->head ^= 1;
    --r->inflight;
  }
  const size_t n = r->cohort.size();
  if (r->inflight == 0) {
    // members at their count: results out of their columns
    for (size_t k = 0; k < n; ++k) {
      Request* m = r->cohort[k];
      if (r->finished[k] || m->left > 0) continue;
      m->result.resize(job->nfields());
      for (int f = 0; f < job->nfields(); ++f) {
        m->result[f].resize(job->field_doubles(f));
        job->fetch_member((int)k, f, m->result[f].data());
      }
      r->finished[k] = true;
      std::lock_guard<std::mutex> lk(mu);
      finish_locked(m);
      ++cohort_requests;
      cv.notify_all();
    }
    r->hold = false;
  }
  bool active = false;
  int cmin = chunk;
  for (size_t k = 0; k < n; ++k)
    if (r->cohort[k]->left > 0) {
      active = true;
      cmin = std::min(cmin, r->cohort[k]->left);
    }
  while (active && !r->hold && r->inflight < kChunksAhead) {
    job->launch(r->dt, cmin);
    TB_CUDA_TRY(cudaEventRecord(r->ev[(r->head + r->inflight) & 1], job->stream()));
    ++r->inflight;
    active = false;
    int next = chunk;
    for (size_t k = 0; k < n; ++k) {
      Request* m = r->cohort[k];
      if (m->left <= 0) continue;
      m->left -= cmin;
      if (m->left == 0) r->hold = true;  // its result is taken once this chunk retires
      if (m->left > 0) {
        active = true;
        next = std::min(next, m->left);
      }
    }
    cmin = next;
  }
  if (active || r->inflight > 0) return;
  for (size_t k = 0; k < n; ++k)
    if (!r->finished[k]) return;  // results still to take (next round)
  for (auto& e : r->ev) {
    cudaEventDestroy(e);
    e = nullptr;
  }
  std::lock_guard<std::mutex> lk(mu);
  size_t bytes = 0;
  for (Request* m : r->cohort) bytes += m->bytes;
  zombies.push_back(std::move(r->job));
  zombie_bytes += bytes;
  used -= bytes;
  running.erase(std::find(running.begin(), running.end(), r));
  cv.notify_all();
}

void tb_server::progress() {
  std::vector<Request*> act;
  {
    std::lock_guard<std::mutex> lk(mu);
    act = running;
  }
  for (Request* r : act) {
    if (!r->cohort.empty()) {
      try {
        progress_cohort(r);
      } catch (const Error& e) {
        fail_running(r, e.msg);
      } catch (const std::exception& e) {
        fail_running(r, e.what());
      }
      continue;
    }
    try {
      // retire the chunks that have finished, oldest first
      while (r->inflight > 0) {
        const cudaError_t e = cudaEventQuery(r->ev[r->head]);
        if (e == cudaErrorNotReady) {
          cudaGetLastError();
          break;
        }
        if (e != cudaSuccess) throw Error{TB_ECUDA, std::string("request stream: ") + cudaGetErrorString(e)};
        r->head ^= 1;
        --r->inflight;
      }
      // keep the next chunk queued behind the running one, so the stream
      // never waits for this loop to come round
      while (r->left > 0 && r->inflight < kChunksAhead) {
        const int c = std::min(r->left, chunk);
        r->job->launch(r->dt, c);
        TB_CUDA_TRY(cudaEventRecord(r->ev[(r->head + r->inflight) & 1], r->job->stream()));
        r->left -= c;
        ++r->inflight;
      }
      if (r->left > 0 || r->inflight > 0) continue;
      // finished: result to host, device memory back to the pool
      r->result.resize(r->job->nfields());
      for (int f = 0; f < r->job->nfields(); ++f) {
        r->result[f].resize(r->job->field_doubles(f));
        r->job->fetch(f, r->result[f].data());
      }
      for (auto& e : r->ev) {
        cudaEventDestroy(e);
        e = nullptr;
      }
      std::lock_guard<std::mutex> lk(mu);
      zombies.push_back(std::move(r->job));
      zombie_bytes += r->bytes;
      used -= r->bytes;
      r->t_done = now_ms();
      r->state = TB_REQ_DONE;
      running.erase(std::find(running.begin(), running.end(), r));
      ++completed;
      steps_done += r->nsteps;
      last_done = r->t_done;
      tts.push_back(r->t_done - r->t_submit);
      waits.push_back(r->t_start - r->t_submit);
      cv.notify_all();
    } catch (const Error& e) {
      fail_running(r, e.msg);
    } catch (const std::exception& e) {
      fail_running(r, e.what());
    }
  }
}

void tb_server::fail_running(Request* r, const std::string& msg) {
  r->job.reset();
  for (auto& e : r->ev) {
    if (e) cudaEventDestroy(e);
    e = nullptr;
  }
  std::lock_guard<std::mutex> lk(mu);
  running.erase(std::find(running.begin(), running.end(), r));
  std::vector<Request*> all_m = r->cohort.empty() ? std::vector<Request*>{r} : r->cohort;
  for (size_t k = 0; k < all_m.size(); ++k) {
    Request* m = all_m[k];
    used -= m->bytes;
    if (!r->cohort.empty() && r->finished[k]) continue;  // its result was already taken
    m->state = TB_REQ_FAILED;
    m->error = msg;
    ++failed;
  }
  cv.notify_all();
}

void tb_server::loop() {
  cudaSetDevice(ctx->device);
  while (true) {
    {
      std::unique_lock<std::mutex> lk(mu);
      if (idle_locked() && !zombies.empty()) release_zombies();  // nothing runs: free now
      if (stop && idle_locked()) return;
      if (queue.empty() && running.empty()) {
        cv.wait_for(lk, std::chrono::milliseconds(1));
        continue;
      }
    }
    admit();
    progress();
    std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
}

extern "C" {

tb_status tb_server_create(tb_context* ctx, size_t budget_bytes, int max_running, int chunk_steps, tb_server** out) {
  if (!ctx || !out || budget_bytes == 0 || max_running < 1 || chunk_steps < 1) return TB_EINVAL;
  *out = nullptr;
  return guarded(ctx, [&] {
    auto S = std::make_unique<tb_server>();
    S->ctx = ctx;
    S->budget = budget_bytes;
    S->max_running = max_running;
    S->chunk = chunk_steps;
    tb_server* raw = S.get();
    S->worker = std::thread([raw] { raw->loop(); });
    for (int i = 0, n = setup_threads(); i < n; ++i) S->setup_workers.emplace_back([raw] { raw->setup_loop(); });
    *out = S.release();
  });
}

tb_status tb_server_set_cohort(tb_server* S, int max_members) {
  if (!S || max_members < 1 || max_members > 64) return TB_EINVAL;
  std::lock_guard<std::mutex> lk(S->mu);
  S->cohort_max = max_members;
  return TB_OK;
}

tb_status tb_server_submit(tb_server* S, const tb_request* req, long long* id) {
  if (!S || !req || !id || !req->init_grid || req->nsteps < 0 || !(req->dt > 0)) return TB_EINVAL;
  return guarded(S->ctx, [&] {
    const tb_problem_desc& d = req->desc;
    TB_REQUIRE(d.program == TB_PROGRAM_RBC || d.program == TB_PROGRAM_TURB2D, TB_ENOTSUPPORTED, "unknown program");
    auto r = std::make_unique<Request>();
    r->desc = d;
    r->dt = req->dt;
    r->nsteps = r->left = req->nsteps;
    // RBC: real grid (Nz, Nx); TURB2D: complex coefficients (Ny, Nx/2+1)
    const size_t ng = d.program == TB_PROGRAM_TURB2D ? (size_t)2 * d.Ny * (d.Nx / 2 + 1) : (size_t)d.Nx * d.Nz;
    TB_REQUIRE(d.Nx > 0 && (d.program == TB_PROGRAM_TURB2D ? d.Ny > 0 : d.Nz > 0), TB_EINVAL, "bad sizes");
    r->init.assign(req->init_grid, req->init_grid + ng);
    r->bytes = estimate_bytes(d);
    std::lock_guard<std::mutex> lk(S->mu);
    r->id = S->next_id++;
    r->t_submit = now_ms();
    if (S->first_submit < 0) S->first_submit = r->t_submit;
    *id = r->id;
    S->queue.push_back(r.get());
    S->all[r->id] = std::move(r);
    S->cv.notify_all();
  });
}

tb_status tb_server_poll(tb_server* S, long long id, int* state, double* tts_ms) {
  if (!S || !state) return TB_EINVAL;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->all.find(id);
  if (it == S->all.end()) return TB_EINVAL;
  *state = it->second->state;
  if (tts_ms) *tts_ms = it->second->state == TB_REQ_DONE ? it->second->t_done - it->second->t_submit : -1.0;
  if (it->second->state == TB_REQ_FAILED) set_context_error(S->ctx, it->second->error);
  return TB_OK;
}

tb_status tb_server_result(tb_server* S, long long id, int field, double* host_out, size_t* ndoubles) {
  if (!S) return TB_EINVAL;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->all.find(id);
  if (it == S->all.end() || it->second->state != TB_REQ_DONE) return TB_ESTATE;
  const Request& r = *it->second;
  if (field < 0 || field >= (int)r.result.size()) return TB_EINVAL;
  if (ndoubles) *ndoubles = r.result[field].size();
  if (host_out) std::copy(r.result[field].begin(), r.result[field].end(), host_out);
  return TB_OK;
}

tb_status tb_server_wait_all(tb_server* S) {
  if (!S) return TB_EINVAL;
  std::unique_lock<std::mutex> lk(S->mu);
  S->cv.wait(lk, [&] { return S->idle_locked(); });
  return TB_OK;
}

static double percentile(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double pos = q * (v.size() - 1);
  const size_t i = (size_t)pos;
  const double f = pos - i;
  return i + 1 < v.size() ? v[i] * (1 - f) + v[i + 1] * f : v[i];
}

tb_status tb_server_get_stats(tb_server* S, tb_server_stats* out) {
  if (!S || !out) return TB_EINVAL;
  std::lock_guard<std::mutex> lk(S->mu);
  tb_server_stats st{};
  st.submitted = (long long)S->all.size();
  st.completed = S->completed;
  st.failed = S->failed;
  st.running = (long long)S->running.size();
  st.queued = (long long)S->queue.size();
  st.elapsed_ms = S->first_submit >= 0 ? S->last_done - S->first_submit : 0.0;
  st.solves_per_s = st.elapsed_ms > 0 ? S->completed / (st.elapsed_ms / 1e3) : 0.0;
  st.steps_per_s = st.elapsed_ms > 0 ? S->steps_done / (st.elapsed_ms / 1e3) : 0.0;
  st.p50_ms = percentile(S->tts, 0.50);
  st.p99_ms = percentile(S->tts, 0.99);
  double w = 0;
  for (double x : S->waits) w += x;
  st.mean_wait_ms = S->waits.empty() ? 0.0 : w / S->waits.size();
  st.peak_bytes = S->peak;
  st.budget_bytes = S->budget;
  st.peak_running = S->peak_running;
  double su = 0;
  for (double x : S->setups) su += x;
  st.mean_setup_ms = S->setups.empty() ? 0.0 : su / S->setups.size();
  st.peak_cohort = S->peak_cohort;
  st.cohort_requests = S->cohort_requests;
  *out = st;
  return TB_OK;
}

tb_status tb_server_destroy(tb_server* S) {
  if (!S) return TB_EINVAL;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
    S->cv.notify_all();
  }
  if (S->worker.joinable()) S->worker.join();  // drains every admitted request first
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->setup_cv.notify_all();
  }
  for (auto& t : S->setup_workers)
    if (t.joinable()) t.join();
  delete S;
  return TB_OK;
}

}  // extern "C"
