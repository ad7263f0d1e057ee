// Batched and served proving: many independent proofs in flight on one GPU.
//
// The reference proves one instance at a time on a rayon pool (src/examples/poseidon2.rs:
// 153-174); this adds the batching and serving patterns around the same prover. A Server
// owns `workers` worker threads, each with its own Context (CUDA stream, twiddles, staging
// buffers), so kernels of different proofs overlap on the device and one proof's host-side
// transcript work hides behind another's kernels. Jobs wait in a FIFO queue; the head job
// is admitted when a worker is idle and its estimated device footprint fits in what is left
// of the HBM budget (continuous batching: a finished proof frees its slot and memory for
// the next arrival at once). Every job carries its own constants, inputs and transcript,
// so a proof is the same whether it runs alone or in a mix.
#pragma once
#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "prover.h"

namespace wl {

struct ServeJob {
  Settings settings;
  int log_n = 0;
  std::vector<uint32_t> constants;  // canonical blob (AIR, Poseidon16, Poseidon24)
  std::vector<uint32_t> inputs;     // canonical, 16 per row, row-major
};

enum JobState { JOB_QUEUED = 0, JOB_RUNNING = 1, JOB_DONE = 2, JOB_FAILED = 3 };

struct ServeResult {
  JobState state = JOB_QUEUED;
  std::vector<uint32_t> proof;
  std::string error;
  double submit_ms = 0, start_ms = 0, end_ms = 0;  // steady-clock timestamps
  uint64_t footprint = 0;
};

// Device bytes one proof of 2^log_n rows may hold at its peak (witness, LDE and Merkle tree
// of the first commitment, zerocheck and inner-sumcheck tables, WHIR tables and later
// commitments), with slack for pool rounding.
uint64_t proof_footprint_bytes(const Settings& s, int log_n);

class Server {
 public:
  Server(int device, int workers, uint64_t hbm_budget);
  ~Server();
  uint64_t submit(ServeJob job);
  JobState poll(uint64_t ticket);
  // Blocks until the job finishes and returns its result; with release, the ticket is
  // forgotten afterwards.
  ServeResult wait(uint64_t ticket, bool release);
  void release(uint64_t ticket);
  int workers() const { return (int)threads_.size(); }
  uint64_t budget() const { return budget_; }
  uint64_t peak_in_use() const { return peak_in_use_.load(); }
  int peak_running() const { return peak_running_.load(); }

 private:
  void worker_main(int idx);
  int device_;
  uint64_t budget_;
  std::vector<std::thread> threads_;
  std::vector<std::unique_ptr<Context>> contexts_;
  std::mutex mu_;
  std::condition_variable cv_work_, cv_done_;
  std::deque<uint64_t> queue_;
  std::unordered_map<uint64_t, ServeJob> jobs_;
  std::unordered_map<uint64_t, ServeResult> results_;
  uint64_t next_ticket_ = 1;
  uint64_t in_use_ = 0;
  int running_ = 0;
  bool stop_ = false;
  std::atomic<uint64_t> peak_in_use_{0};
  std::atomic<int> peak_running_{0};
};

}  // namespace wl
