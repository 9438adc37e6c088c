// Served solves: a pool of host workers, each owning a context (its own
// stream and workspaces), takes problems from a FIFO queue and runs whole
// solves concurrently on the device (the batch entry point, which groups the
// integrator iterations of a whole batch, is in stages.cu).  Admission counts
// every worker's device memory: an idle worker's workspaces as they are held
// between solves, a running one's as the larger of those and its problem's
// estimated bytes.  The queue head starts on a free worker when that sum stays
// within the budget (a problem larger than the budget runs alone).  When the
// head does not fit while work is running, idle workers release the
// workspaces they hold (and grow them again on their next solve), so large
// requests do not leave every worker holding their size; workspaces that
// block nothing are kept.  Results do not depend on what else is in flight:
// every kernel reduces in a fixed order.
#include "common.cuh"
#include "solve.cuh"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

namespace mb {
namespace {

using Clock = std::chrono::steady_clock;

struct Job {
  mcnla_b200_problem p;
  int64_t bytes = 0;
  bool done = false;
  Clock::time_point submitted;
  std::string error;        // the worker's error message when the solve failed
};

int64_t round8(int64_t x) { return (x + 7) & ~int64_t(7); }

// Workspaces a blocked worker keeps rather than releases (they cannot matter).
constexpr int64_t kKeepBytes = int64_t(64) << 20;

}  // namespace

int64_t problem_bytes(const mcnla_b200_problem& p) {
  const int64_t m = p.params.nrow, n = p.params.ncol, l = p.params.rank + p.params.over_rank;
  const int64_t L = l * p.params.num_sketch;
  const bool mixed = p.precision == MCNLA_B200_PRECISION_MIXED || p.precision == MCNLA_B200_PRECISION_MIXED3;
  int64_t bytes = (m * L + m * l) * 8 + (mixed ? L * round8(n) * 2 : n * L * 8);  // Q, Qbar, Omega
  int64_t stage = m * L * 8 + 5 * l * l * p.params.num_sketch * 8;              // orthogonalizer
  stage = std::max(stage, L * L * 8 + 8 * L * 3 * l * 8 + 4 * m * 2 * l * 8);   // integrators
  stage = std::max(stage, 4 * l * n * 8 + n * l * 8);                           // formers
  if (mixed) stage = std::max(stage, 3 * l * round8(m) * 2 + 16 * l * n * 8);   // precision former
  bytes += stage + (int64_t(64) << 20);                                         // + split-K partials, small terms
  bytes += int64_t(mb::problem_scratch_bytes(p));                               // FP64 copy or BF16 parts of A, A'
  const bool gramian = p.integrator == MCNLA_B200_ROW_BLOCK_GRAMIAN_KOLMOGOROV_NAGUMO ||
                       p.integrator == MCNLA_B200_ROW_BLOCK_GRAMIAN_WEN_YIN;
  if (mixed && gramian && double(L) * double(L) * double(m) >= kMixedGramianMinFlops) {
    // the BF16 Gramian's scratch: three parts of Qs' and, for the KN integrator, of Bs and of Bc'
    // and the loop's split-K slices
    bytes += 3 * L * round8(m) * 2;
    if (p.integrator == MCNLA_B200_ROW_BLOCK_GRAMIAN_KOLMOGOROV_NAGUMO)
      bytes += 3 * L * round8(L) * 2 + 3 * l * round8(L) * 2 + 16 * L * 3 * l * 8;
  }
  return bytes;
}

}  // namespace mb

struct mcnla_b200_server {
  int device = 0;
  int64_t budget = 0;
  std::vector<std::thread> threads;
  int nworkers = 1;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<int64_t> queue;
  std::unordered_map<int64_t, mb::Job> jobs;
  int64_t next_ticket = 1, in_flight = 0, peak = 0, completed = 0;
  std::vector<int64_t> committed;   // per worker: held workspaces, or max(held, problem bytes) while running
  int64_t committed_total = 0;
  int running = 0;
  bool stop = false;
  std::atomic<int> init_failures{0};

  void worker(int me);
};

void mcnla_b200_server::worker(int me) {
  cudaSetDevice(device);
  cudaStream_t stream = nullptr;
  mcnla_b200_ctx* ctx = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  bool ok = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) == cudaSuccess &&
            mcnla_b200_create(&ctx, device, stream) == MCNLA_B200_OK && cudaEventCreate(&e0) == cudaSuccess &&
            cudaEventCreate(&e1) == cudaSuccess;
  // each worker's persistent kernels take a share of the SMs, so that the
  // workers' integrations (latency-bound chains of small products) run side by side
  if (ok) ctx->coop_cta_limit = std::max(1, ctx->num_sms / nworkers);
  if (!ok) init_failures++;
  mb::SolveScratch scratch;
  int64_t held_floor = 0;   // what this worker still held after its last release (it cannot go lower)
  while (true) {
    int64_t ticket = 0;
    mcnla_b200_problem p;
    int64_t bytes = 0;
    {
      std::unique_lock<std::mutex> lock(mu);
      // the head fits beside what every worker holds; or nothing runs and no other worker holds
      // more than it keeps anyway (the head alone is over the budget)
      auto fits = [&] {
        const int64_t b = jobs[queue.front()].bytes;
        return committed_total - committed[me] + std::max(committed[me], b) <= budget;
      };
      auto alone = [&] {
        return running == 0 && committed_total - committed[me] <= int64_t(nworkers - 1) * mb::kKeepBytes;
      };
      cv_work.wait(lock, [&] {
        if (queue.empty()) return stop;
        return fits() || alone() || committed[me] > std::max(mb::kKeepBytes, held_floor);
      });
      if (queue.empty()) break;
      if (!fits() && !alone()) {
        // this worker's idle workspaces stand in the head's way: release them and wait again
        // (woken by the next completion, or to release again only if it grew past the floor)
        lock.unlock();
        if (ok) {
          mb::solve_scratch_free(ctx, scratch);
          mb::ctx_trim(ctx);
          cudaStreamSynchronize(stream);
        }
        const int64_t held = ok ? mb::ctx_held_bytes(ctx) : 0;
        held_floor = held;
        lock.lock();
        committed_total += held - committed[me];
        committed[me] = held;
        lock.unlock();
        cv_work.notify_all();
        continue;
      }
      ticket = queue.front();
      queue.pop_front();
      p = jobs[ticket].p;
      bytes = jobs[ticket].bytes;
      in_flight += bytes;
      running++;
      const int64_t c = std::max(committed[me], bytes);
      committed_total += c - committed[me];
      committed[me] = c;
      peak = std::max(peak, in_flight);
    }
    int st = MCNLA_B200_ERR_CUDA;
    float ms = 0.f;
    if (ok) {
      cudaEventRecord(e0, stream);
      st = mb::solve_problem(ctx, p, scratch);
      cudaEventRecord(e1, stream);
      if (cudaStreamSynchronize(stream) != cudaSuccess && st == MCNLA_B200_OK) st = MCNLA_B200_ERR_CUDA;
      cudaEventElapsedTime(&ms, e0, e1);
    }
    p.status = st;
    p.seconds = ms * 1e-3;
    std::string err;
    if (st != MCNLA_B200_OK) err = ok ? mb::last_error_text() : "worker initialization failed";
    const int64_t held = ok ? mb::ctx_held_bytes(ctx) + mb::solve_scratch_bytes(scratch) : 0;
    {
      std::lock_guard<std::mutex> lock(mu);
      mb::Job& j = jobs[ticket];
      j.error = err;
      p.latency = std::chrono::duration<double>(mb::Clock::now() - j.submitted).count();
      j.p = p;
      j.done = true;
      in_flight -= bytes;
      running--;
      completed++;
      committed_total += held - committed[me];
      committed[me] = held;
    }
    cv_done.notify_all();
    cv_work.notify_all();
  }
  if (ctx) mb::solve_scratch_free(ctx, scratch);
  if (stream) cudaStreamSynchronize(stream);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (ctx) mcnla_b200_destroy(ctx);
  if (stream) cudaStreamDestroy(stream);
}

extern "C" {

int64_t mcnla_b200_problem_bytes(const mcnla_b200_problem* p) { return p ? mb::problem_bytes(*p) : -1; }

int mcnla_b200_server_create(mcnla_b200_server** out, int device, int workers, int64_t budget_bytes) {
  if (!out || workers < 1 || workers > 256 || budget_bytes <= 0) return MCNLA_B200_ERR_ARG;
  *out = nullptr;
  MB_CHECK_CUDA(cudaSetDevice(device));
  auto* s = new mcnla_b200_server();
  s->device = device;
  s->budget = budget_bytes;
  s->nworkers = workers;
  s->committed.assign(size_t(workers), 0);
  for (int i = 0; i < workers; ++i) s->threads.emplace_back([s, i] { s->worker(i); });
  *out = s;
  return MCNLA_B200_OK;
}

int mcnla_b200_server_submit(mcnla_b200_server* s, const mcnla_b200_problem* problem, int64_t* ticket) {
  if (!s || !problem || !ticket) return MCNLA_B200_ERR_ARG;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->stop) return MCNLA_B200_ERR_ARG;
    const int64_t t = s->next_ticket++;
    mb::Job j;
    j.p = *problem;
    j.p.iteration = 0;
    j.p.status = -1;
    j.p.seconds = 0;
    j.p.latency = 0;
    j.bytes = mb::problem_bytes(*problem);
    j.submitted = mb::Clock::now();
    s->jobs.emplace(t, j);
    s->queue.push_back(t);
    *ticket = t;
  }
  s->cv_work.notify_all();
  return MCNLA_B200_OK;
}

int mcnla_b200_server_wait(mcnla_b200_server* s, int64_t ticket, mcnla_b200_problem* out) {
  if (!s) return MCNLA_B200_ERR_ARG;
  std::unique_lock<std::mutex> lock(s->mu);
  auto it = s->jobs.find(ticket);
  if (it == s->jobs.end()) return MCNLA_B200_ERR_ARG;
  s->cv_done.wait(lock, [&] { return s->jobs[ticket].done; });
  if (out) *out = s->jobs[ticket].p;
  const int st = s->jobs[ticket].p.status;
  if (st != MCNLA_B200_OK) mb::set_last_message("server job: " + s->jobs[ticket].error);
  s->jobs.erase(ticket);
  return st;
}

int mcnla_b200_server_stats(mcnla_b200_server* s, int64_t* in_flight, int64_t* peak, int64_t* completed) {
  if (!s) return MCNLA_B200_ERR_ARG;
  std::lock_guard<std::mutex> lock(s->mu);
  if (in_flight) *in_flight = s->in_flight;
  if (peak) *peak = s->peak;
  if (completed) *completed = s->completed;
  return s->init_failures.load() ? MCNLA_B200_ERR_CUDA : MCNLA_B200_OK;
}

int mcnla_b200_server_destroy(mcnla_b200_server* s) {
  if (!s) return MCNLA_B200_OK;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  for (auto& t : s->threads) t.join();
  delete s;
  return MCNLA_B200_OK;
}

int mcnla_b200_isvd_batched(int device, mcnla_b200_problem* problems, int count, int workers, int64_t budget_bytes) {
  if (count < 0 || (count > 0 && !problems)) return MCNLA_B200_ERR_ARG;
  mcnla_b200_server* s = nullptr;
  MB_CHECK(mcnla_b200_server_create(&s, device, workers, budget_bytes));
  std::vector<int64_t> tickets(static_cast<size_t>(count));
  int first = MCNLA_B200_OK;
  for (int i = 0; i < count; ++i) {
    const int st = mcnla_b200_server_submit(s, &problems[i], &tickets[size_t(i)]);
    if (st != MCNLA_B200_OK) { first = st; tickets[size_t(i)] = 0; }
  }
  for (int i = 0; i < count; ++i) {
    if (!tickets[size_t(i)]) continue;
    const int st = mcnla_b200_server_wait(s, tickets[size_t(i)], &problems[i]);
    if (st != MCNLA_B200_OK && first == MCNLA_B200_OK) first = st;
  }
  int64_t inflight = 0, peak = 0, done = 0;
  const int sst = mcnla_b200_server_stats(s, &inflight, &peak, &done);
  mcnla_b200_server_destroy(s);
  if (first == MCNLA_B200_OK && sst != MCNLA_B200_OK) first = sst;
  return first;
}

int mcnla_b200_isvd_grouped(int device, mcnla_b200_problem* problems, int count, int workers, int64_t budget_bytes) {
  return mb::batched_solve(device, problems, count, workers, budget_bytes);
}

int mcnla_b200_grouped_times(double* seconds, int capacity) {
  if (!seconds && capacity > 0) return -MCNLA_B200_ERR_ARG;
  return mb::batched_times(seconds, capacity);
}

}  // extern "C"
