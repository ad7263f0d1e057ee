// Batched / served proving (see server.h).
#include <algorithm>
#include <chrono>
#include <cstdlib>

#include "server.h"

namespace wl {

namespace {
double steady_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
}  // namespace

// Upper bound of the device memory one proof takes from the stream-ordered pool, by phase,
// from the buffer sizes of prove_air (N = 2^log_n rows, W = 165 columns, 32-byte extension
// values). The witness (W N words) lives throughout, and so do the commitments: the first one
// (2^(n+1+rho) rows of 88 stored columns and its Merkle tree), and in the WHIR rounds the later
// ones (128 columns; the first of them 2^(n+4+rho-d) rows for an RS domain reduction d, each
// next one half as many).
//  * zerocheck: round 0 holds the per-row combination (N values), then either the 52 computed
//    cube inputs per row or the W + 1 folded columns (N / 2^k values each); round 1 holds the
//    folded columns and their halves, with the eq tables.
//  * inner sumcheck: two tables of N values and their halves.
//  * WHIR: g and the weights (2N values each), their halves, the later commitments.
// A margin covers the small tables (eq tables, partial sums, query rows, OOD work) and the
// pool's rounding.
uint64_t proof_footprint_bytes(const Settings& s, int log_n) {
  const uint64_t N = uint64_t(1) << log_n;
  const int rho = s.log_inv_rate, k = s.univariate_skips;
  const uint64_t E = 32;  // bytes per extension value
  const uint64_t wit = uint64_t(AIR_W) * N * 4;
  const uint64_t rows0 = N << (1 + rho);
  const uint64_t c0 = rows0 * 88 * 4 + rows0 * 2 * 32;
  const uint64_t S = N >> k;
  const uint64_t zc0 = E * N + std::max<uint64_t>(4ull * ZC0_NQ * N, uint64_t(AIR_W + 1) * S * E) + E * S;
  const uint64_t zc1 = uint64_t(AIR_W + 1) * S * E * 3 / 2 + E * S * 3 / 2;
  const uint64_t zc = std::max(zc0, zc1);
  const uint64_t inner = E * (S + 3 * N);
  // later commitments: 2^(n+4+rho-d) rows of 128 columns and a tree (d the RS domain
  // reduction of the first round; 2^(n+rho-1) at the defaults), then halving (a geometric
  // series below twice the first)
  const int lr1 = log_n + 4 + rho - s.rs_reduction;
  const uint64_t rows1 = lr1 >= 0 ? uint64_t(1) << lr1 : 1;
  const uint64_t c1 = 2 * (rows1 * 128 * 4 + rows1 * 2 * 32);
  const uint64_t whir = 2 * (2 * N * E) * 3 / 2 + c1 + (2 * N * E) / 8;
  const uint64_t phase = std::max(std::max(zc, inner), whir);
  const uint64_t margin = (uint64_t(64) << 20) + (wit + c0 + phase) / 32;
  return wit + c0 + phase + margin;
}

Server::Server(int device, int workers, uint64_t hbm_budget) : device_(device), budget_(hbm_budget) {
  if (workers < 1) throw std::invalid_argument("a server needs at least one worker");
  for (int i = 0; i < workers; i++) {
    contexts_.push_back(std::make_unique<Context>(device, hbm_budget));
    contexts_.back()->spin_sync = false;  // workers block: the other workers' proofs fill the device
    if (const char* v = std::getenv("WL_WORKER_POLL_US")) contexts_.back()->block_after_us = std::atoi(v);
    contexts_.back()->set_cache_limit(0);  // admission counts running proofs only: no cached buffers
    contexts_.back()->autotune = false;    // concurrent proofs would disturb the timings
    contexts_.back()->grind_lean = true;   // device time, not one search's latency, is what counts
  }
  // The budget is reserved in the stream-ordered pool up front (one allocation, freed at once;
  // the pool keeps it and carves the workers' buffers from it). Growing the pool while proofs
  // run maps new memory under the driver's lock, which stalled every running proof for
  // 0.3-2.5 s each time the concurrency reached a new peak.
  if (hbm_budget) {
    size_t free_b = 0, total_b = 0;
    WL_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t margin = size_t(2) << 30;
    const size_t want = std::min<uint64_t>(hbm_budget, free_b > margin ? free_b - margin : 0);
    cudaStream_t s = contexts_[0]->stream;
    void* p = nullptr;
    if (want && cudaMallocAsync(&p, want, s) == cudaSuccess) {
      WL_CUDA(cudaFreeAsync(p, s));
      WL_CUDA(cudaStreamSynchronize(s));
    } else {
      cudaGetLastError();  // not reserved: the pool grows on demand
    }
  }
  for (int i = 0; i < workers; i++) threads_.emplace_back([this, i] { worker_main(i); });
}

Server::~Server() {
  {
    std::lock_guard<std::mutex> lk(mu_);
    stop_ = true;
  }
  cv_work_.notify_all();
  for (auto& t : threads_) t.join();
}

uint64_t Server::submit(ServeJob job) {
  const uint64_t fp = proof_footprint_bytes(job.settings, job.log_n);
  std::lock_guard<std::mutex> lk(mu_);
  if (budget_ && fp > budget_) throw std::invalid_argument("proof footprint exceeds the HBM budget");
  uint64_t t = next_ticket_++;
  ServeResult r;
  r.state = JOB_QUEUED;
  r.submit_ms = steady_ms();
  r.footprint = fp;
  results_[t] = std::move(r);
  jobs_[t] = std::move(job);
  queue_.push_back(t);
  cv_work_.notify_all();
  return t;
}

JobState Server::poll(uint64_t ticket) {
  std::lock_guard<std::mutex> lk(mu_);
  auto it = results_.find(ticket);
  if (it == results_.end()) throw std::invalid_argument("unknown ticket");
  return it->second.state;
}

ServeResult Server::wait(uint64_t ticket, bool rel) {
  std::unique_lock<std::mutex> lk(mu_);
  if (results_.find(ticket) == results_.end()) throw std::invalid_argument("unknown ticket");
  cv_done_.wait(lk, [&] {
    JobState s = results_[ticket].state;
    return s == JOB_DONE || s == JOB_FAILED;
  });
  ServeResult r = results_[ticket];
  if (rel) results_.erase(ticket);
  return r;
}

void Server::release(uint64_t ticket) {
  std::lock_guard<std::mutex> lk(mu_);
  results_.erase(ticket);
}

void Server::worker_main(int idx) {
  Context& ctx = *contexts_[idx];
  // A worker thread must never throw: a failed device selection fails every job it takes.
  std::string setup_err;
  const cudaError_t se = cudaSetDevice(device_);
  if (se != cudaSuccess) {
    setup_err = std::string("cudaSetDevice: ") + cudaGetErrorString(se);
    cudaGetLastError();
  }
  for (;;) {
    uint64_t ticket = 0;
    ServeJob job;
    uint64_t fp = 0;
    {
      std::unique_lock<std::mutex> lk(mu_);
      // FIFO admission: the head job starts once its footprint fits the remaining budget.
      cv_work_.wait(lk, [&] {
        if (stop_) return true;
        if (queue_.empty()) return false;
        uint64_t need = results_[queue_.front()].footprint;
        return budget_ == 0 || in_use_ + need <= budget_ || running_ == 0;
      });
      if (stop_ && queue_.empty()) return;
      if (stop_ && !queue_.empty()) {
        // drain: keep serving until the queue is empty
      }
      ticket = queue_.front();
      queue_.pop_front();
      job = std::move(jobs_[ticket]);
      jobs_.erase(ticket);
      fp = results_[ticket].footprint;
      in_use_ += fp;
      running_++;
      uint64_t cur = in_use_;
      if (cur > peak_in_use_.load()) peak_in_use_.store(cur);
      if (running_ > peak_running_.load()) peak_running_.store(running_);
      results_[ticket].state = JOB_RUNNING;
      results_[ticket].start_ms = steady_ms();
    }
    std::vector<uint32_t> proof;
    std::string err;
    bool ok = true;
    try {
      if (!setup_err.empty()) throw std::runtime_error(setup_err);
      ProofJob pj;
      pj.settings = job.settings;
      pj.log_n = job.log_n;
      pj.air = air_consts_from(job.constants.data());
      pj.p16 = perm_consts_from<16>(job.constants.data() + N_AIR_CONSTS);
      pj.p24 = perm_consts_from<24>(job.constants.data() + N_AIR_CONSTS + N_P16_CONSTS);
      const size_t n_in = size_t(16) << job.log_n;
      DBuf din(n_in * 4, ctx.stream);
      WL_CUDA(cudaMemcpyAsync(din.as<void>(), job.inputs.data(), n_in * 4, cudaMemcpyHostToDevice, ctx.stream));
      DBuf wit((size_t(AIR_W) << job.log_n) * 4, ctx.stream);
      launch_trace_gen(din.as<uint32_t>(), pj.air, wit.as<uint32_t>(), job.log_n, ctx.stream);
      din.reset();
      proof = prove_air(ctx, pj, wit.as<uint32_t>(), nullptr);
      wit.reset();
      ctx.wait_stream();
    } catch (const std::exception& e) {
      ok = false;
      err = e.what();
      cudaGetLastError();
    }
    {
      std::lock_guard<std::mutex> lk(mu_);
      in_use_ -= fp;
      running_--;
      ServeResult& r = results_[ticket];
      r.end_ms = steady_ms();
      r.state = ok ? JOB_DONE : JOB_FAILED;
      r.proof = std::move(proof);
      r.error = err;
    }
    cv_done_.notify_all();
    cv_work_.notify_all();
  }
}

}  // namespace wl
