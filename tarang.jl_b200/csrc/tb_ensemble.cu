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
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "tb_plan.h"

using namespace tb;

struct tb_ensemble {
  tb_context* ctx = nullptr;
  std::vector<tb_plan*> members;  // borrowed
  std::vector<double> work;       // relative cost of one step of each member
  int streams = 1;
  int graph_steps = 1;
  std::vector<cudaStream_t> ws;
  std::vector<cudaEvent_t> done;
  cudaEvent_t start = nullptr;

  ~tb_ensemble() {
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
    TB_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    E->ws.push_back(s);
  }
}

// One run of every member for nsteps on `streams` worker streams, graphs of
// `gsteps` steps; per-member completion times (ms from the common start).
void run(tb_ensemble* E, const double* dt, int nsteps, int streams, int gsteps, float* member_ms, float* total_ms) {
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
    std::vector<int> cand_p;
    for (int pc : {kTauParts, 1}) {
      bool ok = true;
      for (auto* m : E->members) ok = ok && plan_tau_parts_ok(m, pc);
      if (ok) cand_p.push_back(pc);
    }
    const int cand_s[] = {1, 2, 4, 8, 16, 32};
    const int cand_g[] = {1, 4, 16};
    float best = 1e30f;
    int bs = E->streams, bg = E->graph_steps, bp = E->members[0]->sys[0].tau_parts;
    for (int pc : cand_p) {
      for (auto* m : E->members) plan_set_variant(m, pc, 0);
      // warm-up: factors and graphs of every member at this dt
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
          }
        }
      }
    }
    for (auto* m : E->members) plan_set_variant(m, bp, 0);
    E->streams = bs;
    E->graph_steps = bg;
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
