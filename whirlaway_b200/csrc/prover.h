// The GPU prover: host orchestration of the device kernels in the transcript order of
// AirTable::prove (crates/air/src/prove.rs:49-226).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "host.h"
#include "air_program.h"
#include "kernels.h"

namespace wl {

// Stream-ordered device buffer (pooled by the CUDA async allocator).
class DBuf {
 public:
  DBuf() = default;
  DBuf(size_t bytes, cudaStream_t s);
  ~DBuf();
  DBuf(DBuf&& o) noexcept { *this = std::move(o); }
  DBuf& operator=(DBuf&& o) noexcept;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  template <class T>
  T* as() const { return static_cast<T*>(p_); }
  size_t bytes() const { return bytes_; }
  void reset();

 private:
  void* p_ = nullptr;
  size_t bytes_ = 0;
  cudaStream_t s_ = nullptr;
};

struct Context {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t copy_stream = nullptr;  // host-to-device witness tiles, overlapped with the LDE
  cudaStream_t conv_stream = nullptr;  // Montgomery conversion of the copied tiles
  uint64_t hbm_budget = 0;
  uint2* twiddles = nullptr;  // per-stage Shoup twiddles (launch_twiddles)
  void* pinned = nullptr;        // staging for small device-to-host reads
  size_t pinned_bytes = 0;
  void* pinned_dev = nullptr;    // the same staging as seen by kernels (mapped host memory)
  // Reused device buffer for per-round partial sums (grown on demand, kept by the context).
  void* part_buf = nullptr;
  size_t part_cap = 0;
  ef* partials(size_t n);
  // Second-level partial sums (launch_reduce_wide's output), fixed capacity.
  static constexpr int kWideBlocks = 512;
  // Device counter of bounded pipeline waits that ran out (kernels with mbarrier pipelines);
  // zero on a healthy device, checked after each such kernel's results are read.
  unsigned* pipe_timeouts = nullptr;
  ef* part2 = nullptr;
  // Reduces nb interleaved rows of k partial sums to a few rows in part2 when nb is large
  // (returns part2 and sets nb to its row count), else returns partial unchanged.
  const ef* reduce_wide(const ef* partial, int& nb, int k);
  std::string last_error;
  uint64_t host_syncs = 0;  // stream synchronisations made by the host (diagnostics)
  double host_wait_ms = 0;  // time the host spent in them
  double prof_t0_ms = 0, prof_wait0_ms = 0;  // host clock and host_wait_ms when profiling began
  uint64_t prof_syncs0 = 0;
  Context(int device, uint64_t budget);
  ~Context();
  void to_host(void* dst, const void* src, size_t bytes);
  // Several device-to-host copies behind one wait.
  struct HostCopy {
    void* dst;
    const void* src;
    size_t bytes;
  };
  void to_host_many(const std::vector<HostCopy>& copies);
  void wait_stream();  // host synchronisation with `stream` (counted in host_syncs)
  // How wait_stream waits: true (default) = the host thread polls an event without sleeping,
  // so the OS never has to wake it at the end of a round (blocking waits measured up to
  // ~20 ms of wake-up stalls per proof); false = the thread polls for block_after_us, then
  // sleeps on a blocking-sync event (server workers, which would otherwise occupy one CPU each).
  bool spin_sync = true;
  // When set, the first proof of each table shape tunes the commitment's launch plans (see
  // tuner.h); server workers leave it off and use the plans a tuning context has kept.
  bool autotune = true;
  // Grinding threads: false (default) = about 2^(bits+1), one pass of the grid almost always
  // finds the witness (the shortest search); true = about 2^(bits-2), a few passes but less
  // than half the permutations on average (server workers, whose device time is what counts).
  bool grind_lean = false;
  // When set, prove_air records a per-phase transcript log of each proof into last_dump (JSON).
  bool dump_transcript = false;
  std::string last_dump;
  int block_after_us = 500;
  cudaEvent_t sync_event = nullptr, block_event = nullptr;
  void to_device(void* dst, const void* src, size_t bytes);
  void to_device_impl(void* dst, const void* src, size_t bytes);
  // Freed device buffers of `stream` are kept for reuse by later requests of the same size,
  // up to this many bytes (8 GiB by default; 0 disables the cache).
  void set_cache_limit(size_t bytes);

  // Optional per-kernel-class timing with CUDA events on `stream`.
  bool profile = false;
  std::string profile_only;  // when set, only this kernel class is timed
  struct Pending {
    std::string name;
    cudaEvent_t a, b;
  };
  std::vector<Pending> pending;
  std::vector<cudaEvent_t> event_pool;
  std::map<std::string, std::pair<double, long>> prof_totals;  // name -> (ms, launches)
  cudaEvent_t take_event();
  void prof_flush();  // resolves pending events (synchronises the stream)
};

// Scoped timer of one kernel class (no-op unless ctx.profile).
struct ProfScope {
  Context& c;
  const char* name;
  cudaEvent_t a = nullptr;
  double t_host = 0;  // host time of the scope (the launches), when the thread's HostClock is on
  ProfScope(Context& ctx, const char* n);
  ~ProfScope();
};

struct Timings {
  double commit_ms = 0, zerocheck_ms = 0, inner_ms = 0, whir_ms = 0, total_ms = 0;
};

struct ProofJob {
  Settings settings;
  int log_n = 0;
  AirConsts air;
  kb::P16Consts p16;
  kb::P24Consts p24;
  // An AIR given as a constraint program instead of the built-in Poseidon2 AIR (its witness
  // has prog->W columns; `air` is unused).
  const ProgramAir* prog = nullptr;
};

// Proves with a device-resident, Montgomery-form, column-major witness (165 columns of
// 2^log_n values). Returns the proof in canonical form.
// With `tile_ready`, event t signals that witness columns 16 t .. 16 t + 15 are on the device;
// the first commitment's LDE waits for each tile just before encoding it.
std::vector<uint32_t> prove_air(Context& ctx, const ProofJob& job, const uint32_t* wit_dev, Timings* t,
                                const std::vector<cudaEvent_t>* tile_ready = nullptr);

// Proves from a host witness (canonical, column-major): the witness is copied in tiles of 16
// columns on the context's copy stream while the first commitment encodes the tiles already
// present. Same proof as uploading first.
std::vector<uint32_t> prove_air_host(Context& ctx, const ProofJob& job, const uint32_t* wit_host, Timings* t);

// Standalone zerocheck of eq(r, x) * (a * b - c) with a univariate skip; a, b, c device
// Montgomery arrays of 2^log_n. Returns the proof (canonical) and per-round device times.
std::vector<uint32_t> prove_abc(Context& ctx, const kb::P16Consts& p16, int log_n, int skips, const uint32_t* a,
                                const uint32_t* b, const uint32_t* c, std::vector<float>* round_ms);

// Upper bound of the proof length (u32 words) for an AIR of W columns and constraint degree
// `degree` (the built-in one by default).
size_t proof_len_bound(const Settings& s, int log_n, int W = AIR_W, int degree = 3);

}  // namespace wl
