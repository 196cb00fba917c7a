// Ensembles of independent plans stepped together on one GPU.
//
// The reference batches an ensemble's Fourier modes into one factorisation per
// instance and steps instances one after another (mode_batch.jl:23-668,
// step_subproblem_rk_batched.jl:838-1006).  Here every member is a full plan
// whose step is a CUDA graph; a run spreads the members over a small set of
// worker streams so that the graphs of different members execute concurrently
// and fill the SMs that one small instance leaves idle.  Two knobs decide the
// throughput: how many worker streams run at once and how many steps one
// graph launch covers (launch overhead against scheduling granularity).  The
// tuner times candidate settings on the ensemble itself (from a snapshot that
// is restored afterwards) and keeps the fastest.
//
// Fused form: members of one shape (Nx, Nz, domain, walls, stepper, precision)
// that step at the same dt are stacked along the mode axis into one plan
// (build_plan with B instances): every kernel of a step then covers the whole
// group in one launch - the tau solves over all the group's mode groups, the
// transforms over all its columns - under one CUDA graph per group.  A run
// gathers the members' states into the group plan, steps it, and scatters
// the states back (one strided device copy per member each way; SBDF members
// also carry their history, F and M X of the previous step, and fuse only
// when all of a group have the same history depth).  The tuner tries the
// fused form against the per-member form.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "tb_plan.h"

using namespace tb;

struct tb_ensemble {
  struct Group {
    std::vector<int> idx;            // member indices (ascending)
    std::unique_ptr<tb_plan> plan;   // the members stacked along the mode axis
  };
  tb_context* ctx = nullptr;
  std::vector<tb_plan*> members;  // borrowed
  std::vector<double> work;       // relative cost of one step of each member
  int streams = 1;
  int graph_steps = 1;
  bool fused = false;             // step same-shape members as stacked plans
  std::vector<Group> groups;      // built on the first fused run
  bool grouped = false;
  std::vector<cudaStream_t> ws;
  std::vector<cudaEvent_t> done;
  cudaEvent_t start = nullptr;

  ~tb_ensemble() {
    for (auto s : ws) cudaStreamSynchronize(s);
    groups.clear();
    for (auto s : ws) cudaStreamDestroy(s);
    for (auto e : done) cudaEventDestroy(e);
    if (start) cudaEventDestroy(start);
  }
};

namespace {

constexpr int kMaxWorkerStreams = 32;

void ensure_streams(tb_ensemble* E, int n) {
  while ((int)E->ws.size() < n) {
    cudaStream_t s;
    TB_CUDA_TRY(create_work_stream(&s));
    E->ws.push_back(s);
  }
}

bool fusible(const tb_plan* P) {
  return P->ndim == 2 && P->B == 1 && !P->bc_dynamic && P->d.program == TB_PROGRAM_RBC;
}
bool multistep(const tb_plan* P) { return P->d.timestepper == TB_SBDF1 || P->d.timestepper == TB_SBDF2; }

bool same_shape(const tb_plan* a, const tb_plan* b) {
  const tb_problem_desc &x = a->d, &y = b->d;
  return x.Nx == y.Nx && x.Nz == y.Nz && x.Lx == y.Lx && x.Lz == y.Lz && x.timestepper == y.timestepper &&
         x.b_bottom == y.b_bottom && x.b_top == y.b_top && x.precision == y.precision;
}

// Groups of at least two same-shape fusible members, each as a stacked plan.
void build_groups(tb_ensemble* E) {
  if (E->grouped) return;
  const int n = (int)E->members.size();
  std::vector<bool> taken(n, false);
  for (int i = 0; i < n; ++i) {
    if (taken[i] || !fusible(E->members[i])) continue;
    tb_ensemble::Group G;
    for (int j = i; j < n; ++j)
      if (!taken[j] && fusible(E->members[j]) && same_shape(E->members[i], E->members[j])) G.idx.push_back(j);
    if (G.idx.size() < 2) continue;
    std::vector<tb_problem_desc> descs;
    for (int j : G.idx) {
      taken[j] = true;
      descs.push_back(E->members[j]->d);
    }
    G.plan = std::make_unique<tb_plan>();
    build_plan(G.plan.get(), E->ctx, descs.data(), (int)descs.size());
    E->groups.push_back(std::move(G));
  }
  E->grouped = true;
}

// Copy the members' state rows (state planes and tau rows, Nkm modes each)
// into / out of their columns of the group plan; SBDF members also their
// history (F and M X of the previous step, equation planes of Nz rows) and
// history depth.
void move_states(tb_ensemble* E, tb_ensemble::Group& G, cudaStream_t s, bool gather) {
  tb_plan* Q = G.plan.get();
  const size_t w = (size_t)Q->Nkm * sizeof(double2), ldq = (size_t)Q->Nk * sizeof(double2);
  const size_t rows = (size_t)Q->nplanes * Q->Nz + Q->ntau;
  const bool ms = multistep(Q);
  const size_t hrows = (size_t)Q->nplanes * Q->Nz;
  auto move = [&](DevBuf& qb, DevBuf& mb, size_t k, size_t nrows) {
    char* q = static_cast<char*>(qb.p) + k * w;
    if (gather)
      TB_CUDA_TRY(cudaMemcpy2DAsync(q, ldq, mb.p, w, w, nrows, cudaMemcpyDeviceToDevice, s));
    else
      TB_CUDA_TRY(cudaMemcpy2DAsync(mb.p, w, q, ldq, w, nrows, cudaMemcpyDeviceToDevice, s));
  };
  for (size_t k = 0; k < G.idx.size(); ++k) {
    tb_plan* M = E->members[G.idx[k]];
    move(Q->X, M->X, k, rows);
    if (ms && (gather ? M->ms_history : Q->ms_history) > 0) {
      move(Q->Fprev, M->Fprev, k, hrows);
      move(Q->MXprev, M->MXprev, k, hrows);
    }
    if (!gather && ms) M->ms_history = Q->ms_history;
  }
  if (gather && ms) Q->ms_history = E->members[G.idx[0]]->ms_history;
}

// Fused run: each group (members at one dt) as its stacked plan on its own
// worker stream; members left over (other shapes, lone shapes, differing dt)
// step per member on the streams after the groups.
void run_fused(tb_ensemble* E, const double* dt, int nsteps, int streams, int gsteps, float* member_ms,
               float* total_ms) {
  build_groups(E);
  const int n = (int)E->members.size();
  std::vector<int> gi(n, -1);
  std::vector<tb_ensemble::Group*> live;
  for (auto& G : E->groups) {
    bool same_dt = true;
    for (int j : G.idx) {
      same_dt = same_dt && dt[j] == dt[G.idx[0]];
      // multistep members fuse only at one history depth
      same_dt = same_dt && E->members[j]->ms_history == E->members[G.idx[0]]->ms_history;
    }
    if (!same_dt) continue;
    for (int j : G.idx) gi[j] = (int)live.size();
    live.push_back(&G);
  }
  std::vector<int> singles;
  for (int i = 0; i < n; ++i)
    if (gi[i] < 0) singles.push_back(i);
  streams = std::max(1, std::min(std::max(streams, (int)live.size()), kMaxWorkerStreams));
  ensure_streams(E, streams);
  for (tb_plan* P : E->members) TB_CUDA_TRY(cudaStreamSynchronize(P->st));
  std::vector<cudaEvent_t> gdone(live.size());
  for (auto& e : gdone) TB_CUDA_TRY(cudaEventCreateWithFlags(&e, 0));
  TB_CUDA_TRY(cudaEventRecord(E->start, E->ws[0]));
  for (int s = 1; s < streams; ++s) TB_CUDA_TRY(cudaStreamWaitEvent(E->ws[s], E->start, 0));
  for (size_t g = 0; g < live.size(); ++g) {
    cudaStream_t s = E->ws[g % streams];
    tb_plan* Q = live[g]->plan.get();
    move_states(E, *live[g], s, true);
    plan_launch_steps(Q, dt[live[g]->idx[0]], nsteps, s, gsteps);
    move_states(E, *live[g], s, false);
    TB_CUDA_TRY(cudaEventRecord(gdone[g], s));
  }
  // the lone members on the streams after the groups' (round-robin, as run)
  std::vector<int> left(n, nsteps);
  const int s0 = live.empty() ? 0 : (int)(live.size() % streams);
  bool any = !singles.empty();
  while (any) {
    any = false;
    for (size_t k = 0; k < singles.size(); ++k) {
      const int i = singles[k];
      if (left[i] <= 0) continue;
      const int s = (s0 + (int)k) % streams;
      const int chunk = std::min(left[i], gsteps);
      plan_launch_steps(E->members[i], dt[i], chunk, E->ws[s], gsteps);
      left[i] -= chunk;
      if (left[i] == 0) TB_CUDA_TRY(cudaEventRecord(E->done[i], E->ws[s]));
      any = true;
    }
  }
  for (int s = 0; s < streams; ++s) TB_CUDA_TRY(cudaStreamSynchronize(E->ws[s]));
  TB_CUDA_TRY(cudaGetLastError());
  // members' counters follow their group plan's steps
  for (size_t g = 0; g < live.size(); ++g)
    for (int j : live[g]->idx) {
      tb_plan* M = E->members[j];
      M->sim_time += dt[j] * nsteps;
      M->iteration += nsteps;
      M->last_dt = dt[j];
    }
  float tmax = 0.f;
  for (int i = 0; i < n; ++i) {
    float ms = 0.f;
    if (nsteps > 0) TB_CUDA_TRY(cudaEventElapsedTime(&ms, E->start, gi[i] >= 0 ? gdone[gi[i]] : E->done[i]));
    if (member_ms) member_ms[i] = ms;
    tmax = std::max(tmax, ms);
  }
  for (auto& e : gdone) cudaEventDestroy(e);
  if (total_ms) *total_ms = tmax;
}

// One run of every member for nsteps on `streams` worker streams, graphs of
// `gsteps` steps; per-member completion times (ms from the common start).
void run(tb_ensemble* E, const double* dt, int nsteps, int streams, int gsteps, float* member_ms, float* total_ms) {
  if (E->fused) {
    run_fused(E, dt, nsteps, streams, gsteps, member_ms, total_ms);
    return;
  }
  const int n = (int)E->members.size();
  streams = std::max(1, std::min(streams, std::min(n, kMaxWorkerStreams)));
  ensure_streams(E, streams);
  TB_CUDA_TRY(cudaSetDevice(E->ctx->device));
  for (tb_plan* P : E->members) TB_CUDA_TRY(cudaStreamSynchronize(P->st));
  // greedy balance: heaviest member first onto the least-loaded stream
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::sort(order.begin(), order.end(), [&](int a, int b) { return E->work[a] > E->work[b]; });
  std::vector<double> load(streams, 0.0);
  std::vector<std::vector<int>> lanes(streams);
  for (int i : order) {
    const int s = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    load[s] += E->work[i];
    lanes[s].push_back(i);
  }
  TB_CUDA_TRY(cudaEventRecord(E->start, E->ws[0]));
  for (int s = 1; s < streams; ++s) TB_CUDA_TRY(cudaStreamWaitEvent(E->ws[s], E->start, 0));
  // round-robin over the members of each stream, one graph launch at a time,
  // so that the members of a stream progress together
  std::vector<int> left(n, nsteps);
  bool any = true;
  while (any) {
    any = false;
    for (int s = 0; s < streams; ++s)
      for (int i : lanes[s]) {
        if (left[i] <= 0) continue;
        const int chunk = std::min(left[i], gsteps);
        plan_launch_steps(E->members[i], dt[i], chunk, E->ws[s], gsteps);
        left[i] -= chunk;
        if (left[i] == 0) TB_CUDA_TRY(cudaEventRecord(E->done[i], E->ws[s]));
        any = true;
      }
  }
  for (int s = 0; s < streams; ++s) TB_CUDA_TRY(cudaStreamSynchronize(E->ws[s]));
  TB_CUDA_TRY(cudaGetLastError());
  float tmax = 0.f;
  for (int i = 0; i < n; ++i) {
    float ms = 0.f;
    if (nsteps > 0) TB_CUDA_TRY(cudaEventElapsedTime(&ms, E->start, E->done[i]));
    if (member_ms) member_ms[i] = ms;
    tmax = std::max(tmax, ms);
  }
  if (total_ms) *total_ms = tmax;
}

}  // namespace

extern "C" {

tb_status tb_ensemble_create(tb_context* ctx, int n, tb_plan* const* members, tb_ensemble** out) {
  if (!ctx || !out || n < 1 || !members) return TB_EINVAL;
  *out = nullptr;
  return guarded(ctx, [&] {
    auto E = std::make_unique<tb_ensemble>();
    E->ctx = ctx;
    for (int i = 0; i < n; ++i) {
      TB_REQUIRE(members[i] != nullptr, TB_EINVAL, "null ensemble member");
      TB_REQUIRE(members[i]->ctx == ctx, TB_EINVAL, "ensemble members must share the context");
      for (int j = 0; j < i; ++j) TB_REQUIRE(members[j] != members[i], TB_EINVAL, "a plan appears twice in the ensemble");
      E->members.push_back(members[i]);
      // one step moves ~ Nz * Nx log Nx worth of data through the transforms and solves
      const double nx = members[i]->Nx, nz = members[i]->Nz;
      E->work.push_back(nz * nx * std::log2(nx));
    }
    TB_CUDA_TRY(cudaSetDevice(ctx->device));
    E->done.resize(n);
    for (int i = 0; i < n; ++i) TB_CUDA_TRY(cudaEventCreate(&E->done[i]));
    TB_CUDA_TRY(cudaEventCreate(&E->start));
    E->streams = std::min(n, 8);
    E->graph_steps = 1;
    *out = E.release();
  });
}

tb_status tb_ensemble_destroy(tb_ensemble* E) {
  if (!E) return TB_EINVAL;
  cudaSetDevice(E->ctx->device);
  for (auto s : E->ws) cudaStreamSynchronize(s);
  delete E;
  return TB_OK;
}

tb_status tb_ensemble_set_config(tb_ensemble* E, int streams, int graph_steps) {
  if (!E || streams < 1 || graph_steps < 1) return TB_EINVAL;
  E->streams = std::min(streams, kMaxWorkerStreams);
  E->graph_steps = graph_steps;
  return TB_OK;
}

tb_status tb_ensemble_set_form(tb_ensemble* E, int fused) {
  if (!E) return TB_EINVAL;
  E->fused = fused != 0;
  return TB_OK;
}

tb_status tb_ensemble_get_form(const tb_ensemble* E, int* fused, int* groups) {
  if (!E) return TB_EINVAL;
  if (fused) *fused = E->fused ? 1 : 0;
  if (groups) *groups = (int)E->groups.size();
  return TB_OK;
}

tb_status tb_ensemble_config(const tb_ensemble* E, int* streams, int* graph_steps) {
  if (!E) return TB_EINVAL;
  if (streams) *streams = E->streams;
  if (graph_steps) *graph_steps = E->graph_steps;
  return TB_OK;
}

tb_status tb_ensemble_tune(tb_ensemble* E, const double* dt, int trial_steps, int* streams, int* graph_steps) {
  if (!E || !dt || trial_steps < 1) return TB_EINVAL;
  return guarded(E->ctx, [&] {
    const int n = (int)E->members.size();
    std::vector<PlanSnapshot> snaps(n);
    for (int i = 0; i < n; ++i) plan_snapshot(E->members[i], &snaps[i]);
    auto restore = [&] {
      for (int i = 0; i < n; ++i) plan_restore(E->members[i], snaps[i]);
    };
    // tau-solve partitioning of the members: the partitioned solve has the
    // shortest latency for one plan, the one-warp solve the least work when
    // many plans share the GPU; both are tried when every member can run them
    // forms: per member, and fused (same-shape members stacked) when some
    // shape has two or more fusible members
    std::vector<bool> cand_f = {false};
    for (int i = 0; i < n && cand_f.size() == 1; ++i)
      for (int j = i + 1; j < n; ++j)
        if (fusible(E->members[i]) && fusible(E->members[j]) && same_shape(E->members[i], E->members[j])) {
          cand_f.push_back(true);
          break;
        }
    const int cand_s[] = {1, 2, 4, 8, 16, 32};
    const int cand_g[] = {1, 4, 16};
    float best = 1e30f;
    int bs = E->streams, bg = E->graph_steps, bp = E->members[0]->sys[0].tau_parts;
    bool bf = E->fused;
    for (bool fz : cand_f) {
      E->fused = fz;
      if (fz) build_groups(E);
      std::vector<tb_plan*> shaped(E->members.begin(), E->members.end());
      if (fz)
        for (auto& G : E->groups) shaped.push_back(G.plan.get());
      std::vector<int> cand_p;
      for (int pc : {kTauParts8, kTauParts, 1}) {
        bool ok = true;
        for (auto* m : shaped) ok = ok && plan_tau_parts_ok(m, pc);
        if (ok) cand_p.push_back(pc);
      }
      for (int pc : cand_p) {
        for (auto* m : shaped) plan_set_variant(m, pc, 0);
        // warm-up: factors and graphs of every member / group at this dt
        run(E, dt, std::min(trial_steps, 2), std::min(n, 8), 1, nullptr, nullptr);
        restore();
        for (int g : cand_g) {
          if (g > trial_steps) continue;
          for (int s : cand_s) {
            if (s > n || s > kMaxWorkerStreams) continue;
            float tot = 0.f;
            run(E, dt, trial_steps, s, g, nullptr, nullptr);  // captures this graph size
            restore();
            run(E, dt, trial_steps, s, g, nullptr, &tot);
            restore();
            if (tot < best) {
              best = tot;
              bs = s;
              bg = g;
              bp = pc;
              bf = fz;
            }
          }
        }
      }
    }
    E->fused = bf;
    for (auto* m : E->members) plan_set_variant(m, bp, 0);
    if (bf)
      for (auto& G : E->groups) plan_set_variant(G.plan.get(), bp, 0);
    E->streams = bs;
    E->graph_steps = bg;
    // mixed members with a tensor-core form of their transform GEMMs: that
    // form or the SIMT kernel, timed on the chosen configuration (best of two
    // alternating trials each)
    std::vector<tb_plan*> all(E->members.begin(), E->members.end());
    if (bf)
      for (auto& G : E->groups) all.push_back(G.plan.get());
    bool any_tc = false;
    for (auto* m : all) any_tc = any_tc || (m->mixed && (m->tc2img.p != nullptr || m->tc3));
    if (any_tc) {
      auto set_tc = [&](bool on) {
        for (auto* m : all)
          if (m->mixed && m->tc32 != on)
            TB_REQUIRE(tb_plan_set_gemm_path(m, on ? 1 : 0) == TB_OK, TB_ECUDA, "setting a member's GEMM path");
      };
      float tt[2] = {1e30f, 1e30f};
      for (int t = 0; t < 4; ++t) {
        const int tc = t & 1;
        set_tc(tc == 1);
        run(E, dt, trial_steps, bs, bg, nullptr, nullptr);  // captures the graphs of this path
        restore();
        float tot = 0.f;
        run(E, dt, trial_steps, bs, bg, nullptr, &tot);
        restore();
        tt[tc] = std::min(tt[tc], tot);
      }
      set_tc(tt[1] < tt[0]);
    }
    if (streams) *streams = bs;
    if (graph_steps) *graph_steps = bg;
  });
}

tb_status tb_ensemble_run(tb_ensemble* E, const double* dt, int nsteps, float* member_ms, float* total_ms) {
  if (!E || !dt || nsteps < 0) return TB_EINVAL;
  return guarded(E->ctx, [&] {
    for (size_t i = 0; i < E->members.size(); ++i)
      TB_REQUIRE(dt[i] > 0 && std::isfinite(dt[i]), TB_EINVAL, "dt must be positive and finite");
    run(E, dt, nsteps, E->streams, E->graph_steps, member_ms, total_ms);
  });
}

}  // extern "C"
