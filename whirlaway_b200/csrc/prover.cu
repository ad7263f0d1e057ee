// GPU prover orchestration. The order of transcript operations is that of
// AirTable::prove (crates/air/src/prove.rs:49-226), sumcheck::prove / sc_round
// (crates/sumcheck/src/prove.rs:22-254) and the WHIR prover; heavy work runs in the
// kernels of k_commit.cu, k_sumcheck.cu and k_whir.cu, the transcript and the
// small-polynomial arithmetic between rounds run on the host.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>

#include "prover.h"
#include "tuner.h"

namespace wl {

// ------------------------------------------------------------------ memory
// Per-stream cache of freed device buffers, reused for requests of exactly the same size on
// the same stream (stream order makes the reuse safe). Proofs of one size request the same
// buffers every time; without the cache, some of those requests made the stream-ordered
// allocator map new memory, at 0.3-100 ms of host time per request while the device idled.
// Bounded per stream: the oldest entries are freed beyond the limit.
namespace {
struct StreamCache {
  size_t limit = 0, bytes = 0;
  std::deque<std::pair<size_t, void*>> entries;  // oldest first
};
std::mutex g_cache_mu;
std::map<cudaStream_t, StreamCache> g_caches;

bool cache_take(cudaStream_t s, size_t bytes, void** p) {
  std::lock_guard<std::mutex> lk(g_cache_mu);
  auto it = g_caches.find(s);
  if (it == g_caches.end()) return false;
  auto& es = it->second.entries;
  for (auto e = es.rbegin(); e != es.rend(); ++e) {
    if (e->first == bytes) {
      *p = e->second;
      it->second.bytes -= bytes;
      es.erase(std::next(e).base());
      return true;
    }
  }
  return false;
}
bool cache_put(cudaStream_t s, size_t bytes, void* p) {
  std::lock_guard<std::mutex> lk(g_cache_mu);
  auto it = g_caches.find(s);
  if (it == g_caches.end() || bytes > it->second.limit) return false;
  StreamCache& c = it->second;
  c.entries.emplace_back(bytes, p);
  c.bytes += bytes;
  while (c.bytes > c.limit) {
    cudaFreeAsync(c.entries.front().second, s);
    c.bytes -= c.entries.front().first;
    c.entries.pop_front();
  }
  return true;
}
// Frees every cached buffer of stream s (and with remove, stops caching for it).
void cache_flush(cudaStream_t s, bool remove) {
  std::lock_guard<std::mutex> lk(g_cache_mu);
  auto it = g_caches.find(s);
  if (it == g_caches.end()) return;
  for (auto& e : it->second.entries) cudaFreeAsync(e.second, s);
  it->second.entries.clear();
  it->second.bytes = 0;
  if (remove) g_caches.erase(it);
}
}  // namespace

void stream_cache_enable(cudaStream_t s, size_t limit) {
  cache_flush(s, false);
  std::lock_guard<std::mutex> lk(g_cache_mu);
  g_caches[s].limit = limit;
}
void Context::set_cache_limit(size_t bytes) { stream_cache_enable(stream, bytes); }

DBuf::DBuf(size_t bytes, cudaStream_t s) : bytes_(bytes), s_(s) {
  if (bytes) {
    HostClock& hc = host_clock();
    const double t0 = hc.on ? host_now_ms() : 0;
    if (!cache_take(s, bytes, &p_)) {
      cudaError_t e = cudaMallocAsync(&p_, bytes, s);
      if (e == cudaErrorMemoryAllocation) {  // cached buffers of other sizes go back to the pool first
        cudaGetLastError();
        cache_flush(s, false);
        e = cudaMallocAsync(&p_, bytes, s);
      }
      if (e != cudaSuccess) {
        p_ = nullptr;
        bytes_ = 0;
        cudaGetLastError();
        throw CudaError(e, "cudaMallocAsync(" + std::to_string(bytes) + " bytes)");
      }
    }
    if (hc.on) hc.alloc_ms += host_now_ms() - t0, hc.allocs++;
  }
}
DBuf::~DBuf() { reset(); }
void DBuf::reset() {
  if (p_) {
    HostClock& hc = host_clock();
    const double t0 = hc.on ? host_now_ms() : 0;
    if (!cache_put(s_, bytes_, p_)) cudaFreeAsync(p_, s_);
    if (hc.on) hc.alloc_ms += host_now_ms() - t0;
  }
  p_ = nullptr;
  bytes_ = 0;
}
DBuf& DBuf::operator=(DBuf&& o) noexcept {
  if (this != &o) {
    reset();
    p_ = o.p_;
    bytes_ = o.bytes_;
    s_ = o.s_;
    o.p_ = nullptr;
    o.bytes_ = 0;
  }
  return *this;
}

namespace {
constexpr size_t kCacheBytes = size_t(8) << 30;  // device buffer cache per context stream
constexpr size_t kUpBytes = 4 << 20;    // pinned upload ring
constexpr size_t kDownBytes = 4 << 20;  // pinned download staging
thread_local size_t g_up_off = 0;
}  // namespace

Context::Context(int dev, uint64_t budget) : device(dev), hbm_budget(budget) {
  WL_CUDA(cudaSetDevice(dev));
  WL_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  WL_CUDA(cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking));
  int prio_lo = 0, prio_hi = 0;  // conversions first: the encoding of a tile waits for them
  WL_CUDA(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
  WL_CUDA(cudaStreamCreateWithPriority(&conv_stream, cudaStreamNonBlocking, prio_hi));
  stream_cache_enable(stream, kCacheBytes);
  cudaMemPool_t pool;
  WL_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
  uint64_t thr = UINT64_MAX;
  WL_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
  WL_CUDA(cudaMalloc(&twiddles, sizeof(uint2) * TWIDDLE_ENTRIES));
  WL_CUDA(cudaMalloc(&part2, sizeof(ef) * kWideBlocks * 32));
  WL_CUDA(cudaMalloc(&pipe_timeouts, sizeof(unsigned)));
  WL_CUDA(cudaMemsetAsync(pipe_timeouts, 0, sizeof(unsigned), stream));
  launch_twiddles(twiddles, stream);
  pinned_bytes = kUpBytes + kDownBytes;
  WL_CUDA(cudaMallocHost(&pinned, pinned_bytes));
  WL_CUDA(cudaHostGetDevicePointer(&pinned_dev, pinned, 0));
  WL_CUDA(cudaStreamSynchronize(stream));
}
Context::~Context() {
  cudaSetDevice(device);
  cache_flush(stream, true);
  cudaStreamSynchronize(stream);
  for (auto& p : pending) { cudaEventDestroy(p.a); cudaEventDestroy(p.b); }
  for (auto e : event_pool) cudaEventDestroy(e);
  if (sync_event) cudaEventDestroy(sync_event);
  if (block_event) cudaEventDestroy(block_event);
  cudaFree(twiddles);
  if (part_buf) cudaFree(part_buf);
  if (part2) cudaFree(part2);
  if (pipe_timeouts) cudaFree(pipe_timeouts);
  cudaFreeHost(pinned);
  cudaStreamSynchronize(copy_stream);
  cudaStreamDestroy(copy_stream);
  cudaStreamSynchronize(conv_stream);
  cudaStreamDestroy(conv_stream);
  cudaStreamDestroy(stream);
}
cudaEvent_t Context::take_event() {
  if (!event_pool.empty()) {
    cudaEvent_t e = event_pool.back();
    event_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  WL_CUDA(cudaEventCreate(&e));
  return e;
}
void Context::prof_flush() {
  if (pending.empty()) return;
  WL_CUDA(cudaStreamSynchronize(stream));
  for (auto& p : pending) {
    float ms = 0;
    WL_CUDA(cudaEventElapsedTime(&ms, p.a, p.b));
    auto& t = prof_totals[p.name];
    t.first += ms;
    t.second += 1;
    event_pool.push_back(p.a);
    event_pool.push_back(p.b);
  }
  pending.clear();
}
ProfScope::ProfScope(Context& ctx, const char* n) : c(ctx), name(n) {
  if (host_clock().on) t_host = host_now_ms();
  if (!c.profile || (!c.profile_only.empty() && c.profile_only != n)) return;
  a = c.take_event();
  WL_CUDA(cudaEventRecord(a, c.stream));
}
ProfScope::~ProfScope() {
  HostClock& hc = host_clock();
  if (hc.on && t_host > 0) hc.launch_ms += host_now_ms() - t_host, hc.launches++;
  if (!c.profile || !a) return;
  cudaEvent_t b = nullptr;
  try {
    b = c.take_event();
  } catch (...) {
    return;
  }
  cudaEventRecord(b, c.stream);
  c.pending.push_back({name, a, b});
}

void Transcript::host_clock_phase(const char* name) {
  HostClock& hc = host_clock();
  if (hc.on) hc.phase = name;
}

void Context::wait_stream() {
  const auto w0 = std::chrono::steady_clock::now();
  HostClock& hclk = host_clock();
  if (hclk.on) {
    const double t = host_now_ms();
    if (hclk.last_wait_end > 0) hclk.add_busy(t - hclk.last_wait_end);
  }
  if (spin_sync) {
    if (!sync_event) WL_CUDA(cudaEventCreateWithFlags(&sync_event, cudaEventDisableTiming));
    WL_CUDA(cudaEventRecord(sync_event, stream));
    cudaError_t e;
    while ((e = cudaEventQuery(sync_event)) == cudaErrorNotReady) {
    }
    WL_CUDA(e);
  } else {
    // polls for at most block_after_us, then sleeps on an event with blocking sync (a plain
    // stream synchronisation may spin, and many spinning workers starve the host work of the
    // others; sleeping at once costs a wake-up on every short wait)
    if (!block_event) WL_CUDA(cudaEventCreateWithFlags(&block_event, cudaEventDisableTiming | cudaEventBlockingSync));
    WL_CUDA(cudaEventRecord(block_event, stream));
    const auto until = w0 + std::chrono::microseconds(block_after_us);
    cudaError_t e;
    while ((e = cudaEventQuery(block_event)) == cudaErrorNotReady && std::chrono::steady_clock::now() < until) {
    }
    if (e == cudaErrorNotReady) e = cudaEventSynchronize(block_event);
    WL_CUDA(e);
  }
  host_syncs++;
  host_wait_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - w0).count();
  if (hclk.on) hclk.last_wait_end = host_now_ms();
}
const ef* Context::reduce_wide(const ef* partial, int& nb, int k) {
  if (nb <= 2 * kWideBlocks || k > 32) return partial;
  {
    ProfScope _ps(*this, "reduce");
    nb = launch_reduce_wide(partial, nb, k, part2, kWideBlocks, stream);
  }
  return part2;
}
ef* Context::partials(size_t n) {
  if (n > part_cap) {
    if (part_buf) WL_CUDA(cudaFreeAsync(part_buf, stream));
    part_buf = nullptr;
    const size_t cap = std::max<size_t>(n, size_t(1) << 16);
    WL_CUDA(cudaMallocAsync(&part_buf, sizeof(ef) * cap, stream));
    part_cap = cap;
  }
  return static_cast<ef*>(part_buf);
}
void Context::to_host(void* dst, const void* src, size_t bytes) {
  char* down = static_cast<char*>(pinned) + kUpBytes;
  if (bytes <= kDownBytes) {
    WL_CUDA(cudaMemcpyAsync(down, src, bytes, cudaMemcpyDeviceToHost, stream));
    wait_stream();
    memcpy(dst, down, bytes);
  } else {
    WL_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, stream));
    wait_stream();
  }
  g_up_off = 0;  // every earlier upload has completed
}
void Context::to_host_many(const std::vector<HostCopy>& copies) {
  char* down = static_cast<char*>(pinned) + kUpBytes;
  size_t off = 0;
  for (const HostCopy& c : copies) off += (c.bytes + 255) & ~size_t(255);
  if (off > kDownBytes) {  // too large for the staging: one copy (and wait) each
    for (const HostCopy& c : copies) to_host(c.dst, c.src, c.bytes);
    return;
  }
  off = 0;
  for (const HostCopy& c : copies) {
    if (c.bytes) WL_CUDA(cudaMemcpyAsync(down + off, c.src, c.bytes, cudaMemcpyDeviceToHost, stream));
    off += (c.bytes + 255) & ~size_t(255);
  }
  wait_stream();
  off = 0;
  for (const HostCopy& c : copies) {
    if (c.bytes) memcpy(c.dst, down + off, c.bytes);
    off += (c.bytes + 255) & ~size_t(255);
  }
  g_up_off = 0;  // every earlier upload has completed
}
void Context::to_device(void* dst, const void* src, size_t bytes) {
  HostClock& hc = host_clock();
  const double t0 = hc.on ? host_now_ms() : 0;
  to_device_impl(dst, src, bytes);
  if (hc.on) hc.upload_ms += host_now_ms() - t0, hc.uploads++;
}
void Context::to_device_impl(void* dst, const void* src, size_t bytes) {
  if (bytes > kUpBytes) {
    WL_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream));
    wait_stream();
    g_up_off = 0;
    return;
  }
  if (g_up_off + bytes > kUpBytes) {
    wait_stream();
    g_up_off = 0;
  }
  char* up = static_cast<char*>(pinned) + g_up_off;
  memcpy(up, src, bytes);
  WL_CUDA(cudaMemcpyAsync(dst, up, bytes, cudaMemcpyHostToDevice, stream));
  g_up_off += (bytes + 255) & ~size_t(255);
}

namespace {

double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

template <class T>
DBuf upload(Context& ctx, const std::vector<T>& v) {
  DBuf b(v.size() * sizeof(T), ctx.stream);
  if (!v.empty()) ctx.to_device(b.as<void>(), v.data(), v.size() * sizeof(T));
  return b;
}

// The reduction writes its k sums straight into the mapped download staging.
std::vector<ef> reduce_to_host(Context& ctx, const ef* partial, int nblk, int k) {
  if (sizeof(ef) * size_t(k) > kDownBytes) throw std::invalid_argument("reduce_to_host: too many sums");
  char* down = static_cast<char*>(ctx.pinned) + kUpBytes;
  ef* down_dev = reinterpret_cast<ef*>(static_cast<char*>(ctx.pinned_dev) + kUpBytes);
  partial = ctx.reduce_wide(partial, nblk, k);
  { ProfScope _ps(ctx, "reduce"); launch_reduce_partials(partial, nblk, k, down_dev, ctx.stream); }
  ctx.wait_stream();
  g_up_off = 0;  // every earlier upload has completed
  std::vector<ef> h(k);
  memcpy(h.data(), down, sizeof(ef) * k);
  return h;
}

DBuf eq_table_dev(Context& ctx, const std::vector<ef>& pt) {
  DBuf out(sizeof(ef) << pt.size(), ctx.stream);
  if (pt.empty()) {
    std::vector<ef> one{kb::ef_one()};
    ctx.to_device(out.as<void>(), one.data(), sizeof(ef));
    return out;
  }
  DBuf p = upload(ctx, pt);
  { ProfScope _ps(ctx, "eq_table"); launch_eq_table(p.as<ef>(), (int)pt.size(), out.as<ef>(), ctx.stream); }
  return out;
}

DBuf scalar_dev(Context& ctx, const ef& v) { return upload(ctx, std::vector<ef>{v}); }

// Constants of the round-finishing kernels for one proof.
FinishConsts finish_consts(const kb::P16Consts& p16) {
  FinishConsts fc;
  fc.p16 = p16;
  for (int b = 0; b < 2; b++) {
    const auto& basis = lagrange_basis_cached(3 + b);
    for (int i = 0; i < 4; i++)
      for (int k = 0; k < 4; k++) fc.basis[b][i][k] = (i < 3 + b && k < 3 + b) ? basis[i][k] : 0u;
  }
  fc.one = fm(1);
  fc.two = fm(2);
  fc.inv2 = kb::inv_m(fm(2));
  return fc;
}

// A phase of sumcheck rounds whose transcript runs on the device (finish.cuh). The challenger
// state, the claim, the finish constants and (for eq-factor rounds) every round's eq challenge
// and its inverse go to the device in one copy at the start; the host then enqueues every
// round (its sums, the finish, the fold at the sampled challenge) without waiting, and
// finish() reads the state, the appended proof words and the challenges back in one copy,
// leaving the host transcript exactly where the host-driven rounds would have left it.
struct DevPhase {
  Context& ctx;
  Transcript& ts;
  int rounds;
  size_t words_per_round;
  // [DevRound][FinishConsts][eq challenges][their inverses][challenges][proof words], each
  // section 64-byte aligned
  DBuf buf;
  size_t off_fc = 0, off_req = 0, off_rinv = 0, off_ch = 0, off_words = 0, total = 0;
  DevRound* st = nullptr;
  ef* chs = nullptr;
  uint32_t* words = nullptr;
  FinArgs fin{};
  static size_t up64(size_t x) { return (x + 63) & ~size_t(63); }
  DevPhase(Context& c, Transcript& t, int nrounds, size_t wpr, const ef& sum, const ef& mmf, const kb::P16Consts& p16,
           const ef* req = nullptr)
      : ctx(c), ts(t), rounds(nrounds), words_per_round(wpr) {
    const size_t nq = req ? size_t(rounds) : 0;
    off_fc = up64(sizeof(DevRound));
    off_req = up64(off_fc + sizeof(FinishConsts));
    off_rinv = up64(off_req + sizeof(ef) * nq);
    off_ch = up64(off_rinv + sizeof(ef) * nq);
    off_words = up64(off_ch + sizeof(ef) * rounds);
    total = off_words + sizeof(uint32_t) * rounds * words_per_round;
    buf = DBuf(total, ctx.stream);
    char* base = buf.as<char>();
    st = reinterpret_cast<DevRound*>(base);
    chs = reinterpret_cast<ef*>(base + off_ch);
    words = reinterpret_cast<uint32_t*>(base + off_words);
    fin.st = st;
    fin.proof = words;
    fin.ch_out = chs;
    fin.fc = reinterpret_cast<const FinishConsts*>(base + off_fc);
    fin.req = req ? reinterpret_cast<const ef*>(base + off_req) : nullptr;
    fin.rinv = req ? reinterpret_cast<const ef*>(base + off_rinv) : nullptr;
    std::vector<char> h(off_ch, 0);
    DevRound d{};
    memcpy(d.ch.state, ts.ch.state, sizeof(d.ch.state));
    memcpy(d.ch.in, ts.ch.in, sizeof(d.ch.in));
    memcpy(d.ch.out, ts.ch.out, sizeof(d.ch.out));
    d.ch.in_len = ts.ch.in_len;
    d.ch.out_len = ts.ch.out_len;
    d.sum = sum;
    d.mmf = mmf;
    memcpy(h.data(), &d, sizeof(d));
    const FinishConsts fc = finish_consts(p16);
    memcpy(h.data() + off_fc, &fc, sizeof(fc));
    for (size_t q = 0; q < nq; q++) {
      const ef ri = kb::ef_inv(req[q]);
      memcpy(h.data() + off_req + sizeof(ef) * q, &req[q], sizeof(ef));
      memcpy(h.data() + off_rinv + sizeof(ef) * q, &ri, sizeof(ef));
    }
    ctx.to_device(base, h.data(), h.size());
  }
  // The round's finish as its own kernel, after an evaluation kernel that left nb partial rows.
  void finish_round(int kind, const ef* partial, int nb) {
    const ef* red = ctx.reduce_wide(partial, nb, fin_kind_sums(kind));
    ProfScope _ps(ctx, "round_finish");
    launch_round_finish(kind, red, nb, fin, ctx.stream);
  }
  // Returns the challenges; *sum (and *mmf) receive the final claim (and eq weight).
  std::vector<ef> finish(ef* sum, ef* mmf) {
    std::vector<char> h(total);
    ctx.to_host(h.data(), buf.as<void>(), h.size());
    DevRound d;
    memcpy(&d, h.data(), sizeof(d));
    if (d.round != rounds || d.proof_len != rounds * words_per_round)
      throw std::runtime_error("device sumcheck phase: round count mismatch");
    memcpy(ts.ch.state, d.ch.state, sizeof(d.ch.state));
    memcpy(ts.ch.in, d.ch.in, sizeof(d.ch.in));
    memcpy(ts.ch.out, d.ch.out, sizeof(d.ch.out));
    ts.ch.in_len = d.ch.in_len;
    ts.ch.out_len = d.ch.out_len;
    std::vector<ef> ch(rounds);
    memcpy(ch.data(), h.data() + off_ch, sizeof(ef) * rounds);
    const uint32_t* w = reinterpret_cast<const uint32_t*>(h.data() + off_words);
    for (int r = 0; r < rounds; r++) {
      ts.proof.insert(ts.proof.end(), w + r * words_per_round, w + (r + 1) * words_per_round);
      if (ts.log) ts.log->add("challenge", ts.proof.size(), ch[r].c, 8, true);
    }
    if (sum) *sum = d.sum;
    if (mmf) *mmf = d.mmf;
    return ch;
  }
};

// Grinding: the smallest witness (searched on the device in batches), then the host
// challenger replays observe(w) + sample_bits exactly as check_witness does.
void grind(Context& ctx, Transcript& ts, const kb::P16Consts& p16, int bits) {
  if (bits <= 0) return;
  DBuf res(sizeof(uint32_t), ctx.stream);
  // 2^(bits+3) candidates per batch: a witness is missed with probability e^-8 (one more
  // round trip then); the search stops soon after the first witness, so a larger batch costs
  // no device work
  const uint32_t batch = 1u << std::min(24, bits + 3);
  // the first witness lies near 2^bits: 2^(bits+1) threads find it in one pass of the grid
  // almost always; 2^(bits-2) threads take a few passes and stop about 2^bits candidates in
  const uint32_t threads = ctx.grind_lean ? 1u << std::max(8, bits - 2) : 1u << std::min(20, bits + 1);
  for (uint64_t base = 0; base < kb::P; base += batch) {
    uint32_t init = UINT32_MAX;
    ctx.to_device(res.as<void>(), &init, 4);
    { ProfScope _ps(ctx, "grind"); launch_grind(p16, ts.ch.state, ts.ch.in, ts.ch.in_len, bits, (uint32_t)base, batch, threads, res.as<uint32_t>(),
                 ctx.stream); }
    uint32_t r;
    ctx.to_host(&r, res.as<uint32_t>(), 4);
    if (r != UINT32_MAX) {
      uint32_t w = kb::to_mont(r);
      ts.ch.observe(w);
      if (ts.ch.sample_bits(bits) != 0) throw std::runtime_error("grinding witness failed on the host");
      if (ts.log) ts.log->add("grinding", ts.proof.size(), &w, 1, true);
      ts.proof.push_back(w);
      return;
    }
  }
  throw std::runtime_error("grinding: no witness");
}

// ------------------------------------------------------------------ commitments
struct Commitment {
  int num_vars = 0, fold = 0, elem = 1, log_leaves = 0, n_cols = 0;
  DBuf lde, tree;
  uint32_t root[8];
};
size_t level_offset(int LL, int l) { return (size_t(1) << (LL + 1)) - (size_t(1) << (LL + 1 - l)); }

// Runs launch(plan) with the autotuner's plan for (family, key): a forced plan, else the kept
// one, else (on a tuning context) every plan in turn, each timed twice with CUDA events on the
// context's stream, keeping the fastest (all plans write the same result, so the data is
// right whichever ran last); a context that does not tune uses the default plan.
template <class Launch>
void tuned(Context& ctx, int family, uint64_t key, Launch&& launch) {
  int plan = tune_forced(family);
  if (plan < 0) plan = tune_lookup(ctx.device, family, key);
  if (plan >= 0 || !ctx.autotune) {
    launch(plan >= 0 ? plan : tune_default_plan(family));
    return;
  }
  const int n = tune_plan_count(family);
  std::vector<float> ms(n, 1e30f);
  cudaEvent_t a = ctx.take_event(), b = ctx.take_event();
  for (int rep = 0; rep < 2; rep++)
    for (int c = 0; c < n; c++) {
      WL_CUDA(cudaEventRecord(a, ctx.stream));
      launch(c);
      WL_CUDA(cudaEventRecord(b, ctx.stream));
      WL_CUDA(cudaEventSynchronize(b));
      float t = 0;
      WL_CUDA(cudaEventElapsedTime(&t, a, b));
      ms[c] = std::min(ms[c], t);
    }
  ctx.event_pool.push_back(a);
  ctx.event_pool.push_back(b);
  int best = 0;
  for (int c = 1; c < n; c++)
    if (ms[c] < ms[best]) best = c;
  tune_store(ctx.device, family, key, best, ms);
}
// The kept (or forced) plan without tuning: the tile-pipelined commitment cannot re-run its
// launches, it uses what a device-witness proof of the same shape has tuned.
int tuned_plan(Context& ctx, int family, uint64_t key) {
  int plan = tune_forced(family);
  if (plan < 0) plan = tune_lookup(ctx.device, family, key);
  return plan >= 0 ? plan : tune_default_plan(family);
}
uint64_t lde_key(const LdeSource& src) {
  return uint64_t(src.L) | uint64_t(src.rho) << 8 | uint64_t(src.n_cols) << 16 | uint64_t(src.elem) << 32;
}

Commitment commit(Context& ctx, const LdeSource& src, int num_vars, int fold, const kb::P24Consts& p24,
                  const kb::P16Consts& p16, const std::vector<cudaEvent_t>* tile_ready = nullptr) {
  Commitment c;
  c.num_vars = num_vars;
  c.fold = fold;
  c.elem = src.elem;
  c.log_leaves = src.L + src.rho;
  c.n_cols = src.n_cols;
  if ((src.elem << fold) != 128) throw std::invalid_argument("leaf rows must hold 128 base-field values");
  const size_t rows = size_t(1) << c.log_leaves;
  c.lde = DBuf(rows * c.n_cols * sizeof(uint32_t), ctx.stream);
  const int LL = c.log_leaves;
  c.tree = DBuf(((size_t(2) << LL) - 1) * 8 * sizeof(uint32_t), ctx.stream);
  uint32_t* t = c.tree.as<uint32_t>();
  if (tile_ready) {
    // Tile t's source columns arrive behind event t. The leaf sponges run one absorption at
    // a time: chunk ch reads LDE tiles up to 2ch + 1, so it is hashed as soon as those tiles
    // are encoded, and the hashing overlaps the rest of the upload too.
    DBuf cap(sizeof(uint32_t) * 8 * rows, ctx.stream);
    const int ntiles = c.n_cols / 8;
    const int lde_plan = tuned_plan(ctx, TUNE_LDE, lde_key(src));
    const int leaf_plan = tuned_plan(ctx, TUNE_LEAF, lde_key(src));
    int next = 0;
    for (int ch = 0; ch < 8; ch++) {
      for (; next < std::min(ntiles, 2 * ch + 2); next++) {
        if (next < (int)tile_ready->size()) WL_CUDA(cudaStreamWaitEvent(ctx.stream, (*tile_ready)[next], 0));
        ProfScope _ps(ctx, "lde");
        launch_lde(src, c.lde.as<uint32_t>(), ctx.twiddles, ctx.stream, next, next + 1, lde_plan);
      }
      ProfScope _ps(ctx, "merkle_tree");
      launch_leaf_absorb(c.lde.as<uint32_t>(), rows, c.n_cols, c.elem, p24, ch, cap.as<uint32_t>(), t, LL, ctx.stream,
                         leaf_plan);
    }
    for (size_t e = ntiles; e < tile_ready->size(); e++) WL_CUDA(cudaStreamWaitEvent(ctx.stream, (*tile_ready)[e], 0));
    { ProfScope _ps(ctx, "merkle_tree"); launch_merkle_levels(t, LL, p16, ctx.stream, tuned_plan(ctx, TUNE_MERKLE, LL)); }
  } else {
    {
      ProfScope _ps(ctx, "lde");
      tuned(ctx, TUNE_LDE, lde_key(src), [&](int plan) {
        launch_lde(src, c.lde.as<uint32_t>(), ctx.twiddles, ctx.stream, 0, -1, plan);
      });
    }
    ProfScope _ps(ctx, "merkle_tree");
    tuned(ctx, TUNE_LEAF, lde_key(src), [&](int plan) {
      launch_leaf_hash(c.lde.as<uint32_t>(), rows, c.n_cols, c.elem, p24, t, LL, ctx.stream, plan);
    });
    tuned(ctx, TUNE_MERKLE, LL, [&](int plan) { launch_merkle_levels(t, LL, p16, ctx.stream, plan); });
  }
  ctx.to_host(c.root, t + level_offset(LL, LL) * 8, 32);
  for (uint32_t& w : c.root) w = kb::to_mont(w);  // the tree holds canonical digests
  return c;
}

std::vector<uint32_t> sample_queries(Transcript& ts, int log_leaves, int count) {
  std::vector<uint32_t> q(count);
  for (auto& x : q) x = ts.ch.sample_bits(log_leaves);
  std::sort(q.begin(), q.end());
  q.erase(std::unique(q.begin(), q.end()), q.end());
  if (ts.log) ts.log->add("queries", ts.proof.size(), q.data(), q.size(), false);
  return q;
}

// Appends rows (Moebius-transformed over the position bits, as hashed) and
// authentication paths as hints. With mono (the folding monomials of the commitment's fold
// randomness), returns each opened row's folded value (its STIR answer).
std::vector<ef> open(Context& ctx, const Commitment& c, const std::vector<uint32_t>& idx, Transcript& ts,
                     const std::vector<ef>* mono = nullptr) {
  const int LL = c.log_leaves, nq = (int)idx.size();
  std::vector<uint64_t> ridx(idx.begin(), idx.end()), didx;
  for (uint32_t i : idx)
    for (int l = 0; l < LL; l++) didx.push_back(level_offset(LL, l) + ((i >> l) ^ 1u));
  DBuf dr = upload(ctx, ridx), dd = upload(ctx, didx);
  const int log_elem = c.elem == 8 ? 3 : 0;
  DBuf rows(sizeof(uint32_t) * 128 * std::max(nq, 1), ctx.stream);
  DBuf digs(sizeof(uint32_t) * 8 * std::max<size_t>(didx.size(), 1), ctx.stream);
  DBuf dmono = mono ? upload(ctx, *mono) : DBuf();
  DBuf dfold(mono ? sizeof(ef) * std::max(nq, 1) : 0, ctx.stream);
  { ProfScope _ps(ctx, "gather"); launch_gather_lde_rows(c.lde.as<uint32_t>(), LL, dr.as<uint64_t>(), c.n_cols, log_elem, nq, rows.as<uint32_t>(), mono ? dmono.as<ef>() : nullptr, mono ? dfold.as<ef>() : nullptr, ctx.stream); }
  { ProfScope _ps(ctx, "gather"); launch_gather_u32(c.tree.as<uint32_t>(), dd.as<uint64_t>(), 8, (int)didx.size(), digs.as<uint32_t>(), ctx.stream); }
  std::vector<uint32_t> hr(size_t(128) * nq), hd(didx.size() * 8);
  std::vector<ef> folded(mono ? nq : 0);
  if (nq) {
    ctx.to_host_many({{hr.data(), rows.as<uint32_t>(), hr.size() * 4},
                      {hd.data(), digs.as<uint32_t>(), hd.size() * 4},
                      {folded.data(), dfold.as<ef>(), mono ? sizeof(ef) * nq : 0}});
    for (uint32_t& w : hd) w = kb::to_mont(w);  // canonical digests
  }
  for (int q = 0; q < nq; q++) {
    ts.hint(&hr[size_t(q) * 128], 128);  // Moebius-transformed on the device, as hashed
    ts.hint(&hd[size_t(q) * LL * 8], size_t(LL) * 8);
  }
  return folded;
}

}  // namespace

const std::vector<std::vector<uint32_t>>& lagrange_basis_cached(int n) {
  static std::mutex mu;
  static std::map<int, std::vector<std::vector<uint32_t>>> cache;
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(n);
  if (it == cache.end()) it = cache.emplace(n, lagrange_basis(n)).first;
  return it->second;
}

namespace {

// Coefficient-form multilinear evaluation of a (transformed) row at r (row MSB <-> r_1):
// folding the row by v[q] + r_i v[q + h], MSB first, gives sum_p v_p m_p with the monomial
// m_p = prod of r_i over the set bits of p (bit fold-1-i <-> r_i). The monomials depend on r
// only, so one table serves every query of a round (the dot products run in the row gather).
std::vector<ef> fold_monomials(int fold, const std::vector<ef>& r) {
  std::vector<ef> m(size_t(1) << fold);
  m[0] = kb::ef_one();
  for (int b = 0; b < fold; b++) {
    const size_t w = size_t(1) << b;
    for (size_t p = 0; p < w; p++) m[p + w] = kb::ef_mul(m[p], r[fold - 1 - b]);
  }
  return m;
}
void split_vars(int lv, int& lh, int& ll) {
  ll = std::min(10, lv);
  lh = lv - ll;
}

// Factored eq tables of an extension point: hi over pt[0..lh), lo over pt[lh..).
struct EqPair {
  DBuf hi, lo;
};
EqPair eq_pair(Context& ctx, const std::vector<ef>& pt, int lh) {
  EqPair e;
  e.hi = eq_table_dev(ctx, std::vector<ef>(pt.begin(), pt.begin() + lh));
  e.lo = eq_table_dev(ctx, std::vector<ef>(pt.begin() + lh, pt.end()));
  return e;
}

// Adds sum_t coefs[t] * eq(points[t], .) for extension-field points.
void add_eq_ef(Context& ctx, ef* w, int m, const std::vector<std::vector<ef>>& pts, const std::vector<ef>& coefs) {
  int lh, ll;
  split_vars(m, lh, ll);
  const int np = (int)pts.size();
  if (!np) return;
  DBuf hi(sizeof(ef) * (size_t(np) << lh), ctx.stream), lo(sizeof(ef) * (size_t(np) << ll), ctx.stream);
  for (int t = 0; t < np; t++) {
    EqPair e = eq_pair(ctx, pts[t], lh);
    WL_CUDA(cudaMemcpyAsync(hi.as<ef>() + (size_t(t) << lh), e.hi.as<ef>(), sizeof(ef) << lh,
                            cudaMemcpyDeviceToDevice, ctx.stream));
    WL_CUDA(cudaMemcpyAsync(lo.as<ef>() + (size_t(t) << ll), e.lo.as<ef>(), sizeof(ef) << ll,
                            cudaMemcpyDeviceToDevice, ctx.stream));
  }
  DBuf dc = upload(ctx, coefs);
  { ProfScope _ps(ctx, "add_eq"); launch_add_eq_terms_ef(w, lh, ll, np, hi.as<ef>(), lo.as<ef>(), dc.as<ef>(), ctx.stream); }
}

// Adds sum_t coefs[t] * eq(points[t], .) for base-field points (STIR queries).
void add_eq_f(Context& ctx, ef* w, int m, const std::vector<std::vector<uint32_t>>& pts,
              const std::vector<ef>& coefs) {
  int lh, ll;
  split_vars(m, lh, ll);
  const int np = (int)pts.size();
  if (!np) return;
  std::vector<uint32_t> ph, pl;
  for (auto& p : pts) {
    ph.insert(ph.end(), p.begin(), p.begin() + lh);
    pl.insert(pl.end(), p.begin() + lh, p.end());
  }
  DBuf dph = upload(ctx, ph.empty() ? std::vector<uint32_t>{0} : ph), dpl = upload(ctx, pl);
  DBuf hi(sizeof(uint32_t) * (size_t(np) << lh), ctx.stream), lo(sizeof(uint32_t) * (size_t(np) << ll), ctx.stream);
  { ProfScope _ps(ctx, "eq_table"); launch_eq_table_f(dph.as<uint32_t>(), np, lh, hi.as<uint32_t>(), ctx.stream); }
  { ProfScope _ps(ctx, "eq_table"); launch_eq_table_f(dpl.as<uint32_t>(), np, ll, lo.as<uint32_t>(), ctx.stream); }
  DBuf dc = upload(ctx, coefs);
  { ProfScope _ps(ctx, "add_eq"); launch_add_eq_terms_f(w, lh, ll, np, hi.as<uint32_t>(), lo.as<uint32_t>(), dc.as<ef>(), ctx.stream); }
}

// g(pt) for a device extension table g over m variables.
ef mle_eval_dev(Context& ctx, const ef* g, int m, const std::vector<ef>& pt) {
  int lh, ll;
  split_vars(m, lh, ll);
  EqPair e = eq_pair(ctx, pt, lh);
  ef* part = ctx.partials(size_t(1) << lh);
  { ProfScope _ps(ctx, "mle_eval"); launch_mle_eval_ef(g, lh, ll, e.hi.as<ef>(), e.lo.as<ef>(), part, ctx.stream); }
  return reduce_to_host(ctx, part, 1 << lh, 1)[0];
}

// k rounds of the WHIR sumcheck on device tables (g, w), both of size 2^m on entry. Without
// grinding the transcript runs on the device (one host wait for the whole block of rounds).
void whir_sumcheck_dev(Context& ctx, Transcript& ts, DBuf& g, DBuf& w, int& m, ef& sigma, int rounds, int pow_bits,
                       const kb::P16Consts& p16, std::vector<ef>& rnd) {
  if (pow_bits == 0 && rounds > 0) {
    DevPhase ph(ctx, ts, rounds, 24, sigma, kb::ef_one(), p16);
    // round 0 evaluates the tables as they are (the finish its own kernel); round t >= 1 folds
    // at challenge t - 1, evaluates and finishes in one kernel; the last challenge's fold
    // closes the block
    for (int t = 0; t < rounds; t++) {
      const size_t half = size_t(1) << (m - 1 - t);
      if (t == 0) {
        const int nb = whir_sc_blocks(half);
        ef* part = ctx.partials(size_t(3) * nb);
        {
          ProfScope _ps(ctx, "whir_sc_eval");
          launch_whir_sc_eval(g.as<ef>(), w.as<ef>(), half, part, ctx.stream);
        }
        ph.finish_round(FIN_WHIR, part, nb);
      } else {
        ef* part = ctx.partials(size_t(3) * fold_eval_blocks(half));
        DBuf ng(sizeof(ef) * 2 * half, ctx.stream), nw(sizeof(ef) * 2 * half, ctx.stream);
        {
          ProfScope _ps(ctx, "fold_eval");
          launch_pair_fold_eval(3, g.as<ef>(), w.as<ef>(), ph.chs + (t - 1), ng.as<ef>(), nw.as<ef>(), half, part,
                                &ph.fin, ctx.stream);
        }
        g = std::move(ng);
        w = std::move(nw);
      }
    }
    {
      const size_t half = size_t(1) << (m - rounds);
      DBuf ng(sizeof(ef) * half, ctx.stream), nw(sizeof(ef) * half, ctx.stream);
      { ProfScope _ps(ctx, "fold"); launch_fold2_dev(g.as<ef>(), w.as<ef>(), ng.as<ef>(), nw.as<ef>(), half, ph.chs + (rounds - 1), ctx.stream); }
      g = std::move(ng);
      w = std::move(nw);
      m -= rounds;
    }
    const std::vector<ef> r = ph.finish(&sigma, nullptr);
    rnd.insert(rnd.end(), r.begin(), r.end());
    return;
  }
  for (int t = 0; t < rounds; t++) {
    size_t half = size_t(1) << (m - 1);
    int nb = whir_sc_blocks(half);
    ef* part = ctx.partials(size_t(3) * nb);
    { ProfScope _ps(ctx, "whir_sc_eval"); launch_whir_sc_eval(g.as<ef>(), w.as<ef>(), half, part, ctx.stream); }
    std::vector<ef> h = reduce_to_host(ctx, part, nb, 3);
    ts.add_ext(h.data(), 3);
    grind(ctx, ts, p16, pow_bits);
    ef r = ts.sample_ext();
    rnd.push_back(r);
    sigma = quad_eval(h.data(), r);
    DBuf ng(sizeof(ef) * half, ctx.stream), nw(sizeof(ef) * half, ctx.stream);
    { ProfScope _ps(ctx, "fold"); launch_fold2_at(g.as<ef>(), w.as<ef>(), ng.as<ef>(), nw.as<ef>(), half, r, ctx.stream); }
    g = std::move(ng);
    w = std::move(nw);
    m--;
  }
}

// Host sumcheck on small tables (initial WHIR block and the final rounds).
void whir_sumcheck_host(Context& ctx, Transcript& ts, std::vector<std::vector<ef>>& G, std::vector<std::vector<ef>>& E,
                        const std::vector<ef>& coef, ef& sigma, int rounds, int pow_bits, const kb::P16Consts& p16,
                        std::vector<ef>& rnd) {
  for (int t = 0; t < rounds; t++) {
    size_t half = G[0].size() / 2;
    ef h[3] = {kb::ef_zero(), kb::ef_zero(), kb::ef_zero()};
    for (size_t j = 0; j < G.size(); j++) {
      ef s[3] = {kb::ef_zero(), kb::ef_zero(), kb::ef_zero()};
      for (size_t x = 0; x < half; x++) {
        const ef &gl = G[j][x], &gh = G[j][x + half], &el = E[j][x], &eh = E[j][x + half];
        s[0] = kb::ef_add(s[0], kb::ef_mul(gl, el));
        s[1] = kb::ef_add(s[1], kb::ef_mul(gh, eh));
        s[2] = kb::ef_add(s[2], kb::ef_mul(kb::ef_sub(kb::ef_add(gh, gh), gl), kb::ef_sub(kb::ef_add(eh, eh), el)));
      }
      for (int q = 0; q < 3; q++) h[q] = kb::ef_add(h[q], kb::ef_mul(coef[j], s[q]));
    }
    ts.add_ext(h, 3);
    grind(ctx, ts, p16, pow_bits);
    ef r = ts.sample_ext();
    rnd.push_back(r);
    sigma = quad_eval(h, r);
    for (size_t j = 0; j < G.size(); j++) {
      for (size_t x = 0; x < half; x++) {
        G[j][x] = kb::ef_lerp(G[j][x], G[j][x + half], r);
        E[j][x] = kb::ef_lerp(E[j][x], E[j][x + half], r);
      }
      G[j].resize(half);
      E[j].resize(half);
    }
  }
}

std::vector<uint32_t> to_canonical(const std::vector<uint32_t>& v) {
  std::vector<uint32_t> out(v.size());
  for (size_t i = 0; i < v.size(); i++) out[i] = kb::from_mont(v[i]);
  return out;
}

}  // namespace

size_t proof_len_bound(const Settings& s, int log_n, int W, int degree) {
  WhirSchedule w = WhirSchedule::build(log_n + log2_up(size_t(W)), s);
  const int k = s.univariate_skips;
  size_t n = 8 + 8 * w.c[0].ood;                              // root + OOD answers
  n += 8 * size_t((degree + 1) * ((1 << k) - 1) + 1);         // zerocheck round 0
  n += 8 * size_t(degree + 2) * (log_n - k);                  // zerocheck rounds >= 1
  n += 8 * size_t(2 * W) + 8 * (size_t(1) << k);              // inner sums, sub-evaluations
  n += 8 * size_t(3) * log_n;                                 // inner sumcheck
  n += 16;                                                    // grinding witnesses (generous)
  n += 8 * 3 * size_t(w.num_vars);                            // WHIR sumcheck messages
  for (int j = 0; j <= w.num_rounds; j++) {
    const WhirRound& r = w.c[j];
    if (j > 0) n += 8 + 8 * r.ood;
    n += size_t(r.queries) * (128 + 8 * size_t(r.log_leaves())) + 2;
  }
  n += 8 * (size_t(1) << w.final_vars);
  return n;
}

// The zerocheck of an AIR given as a constraint program (air_program.h), round for round as
// crates/sumcheck/src/prove.rs:97-254 runs it on the 2W up/down columns: the sums from the
// interpreter kernels, the round polynomial and challenge on the device transcript (degrees 2
// and 3; the host transcript for round 0, degree 1 and rounds that grind), the fold of all 2W
// columns after every round; the last folds are the up and down evaluations.
// The first P of the W columns are preprocessed (in the zerocheck, not committed): up and down
// receive the witness columns' evaluations only.
void zerocheck_program(Context& ctx, Transcript& ts, const ProofJob& job, const ProgramAir& prog, const uint32_t* wit,
                       const DBuf& d_alphas, const std::vector<ef>& zc, const DBuf& eq0, std::vector<ef>& challenges,
                       std::vector<ef>& up, std::vector<ef>& down) {
  const Settings& s = job.settings;
  const int n = job.log_n, k = s.univariate_skips, W = prog.W, P = prog.P, d = prog.degree, nsk = 1 << k, R = n - k;
  const size_t S = size_t(1) << R;
  cudaStream_t st = ctx.stream;
  if (P > 0 && prog.pre_log_n != n) throw std::invalid_argument("AIR program: preprocessed columns of another height");
  const int n_code = (int)prog.code.size();
  DBuf code = upload(ctx, prog.code);
  std::vector<uint32_t> cv = prog.consts;
  if (cv.empty()) cv.push_back(0);
  DBuf consts = upload(ctx, cv);
  DBuf pre = P > 0 ? upload(ctx, prog.pre) : DBuf(sizeof(uint32_t), st);
  const auto& sel = lagrange_basis_cached(nsk);
  // round 0: the values at z < 2^k vanish; the kernel sums z = 2^k .. d (2^k - 1)
  const int nz = d * (nsk - 1) - nsk + 1;
  std::vector<ef> ys(nsk, kb::ef_zero());
  if (nz > 0) {
    std::vector<uint32_t> lw(size_t(nz) * nsk);
    for (int zi = 0; zi < nz; zi++)
      for (int j = 0; j < nsk; j++) lw[size_t(zi) * nsk + j] = upoly_eval_f(sel[j], fm(nsk + zi));
    DBuf d_lw = upload(ctx, lw);
    const int B = prog_zc_blocks(S);
    ef* part = ctx.partials(size_t(B) * nz);
    {
      ProfScope _ps(ctx, "prog_zc0");
      launch_prog_zc0(wit, pre.as<uint32_t>(), P, n, k, code.as<uint2>(), n_code, consts.as<uint32_t>(), nz,
                      d_lw.as<uint32_t>(), eq0.as<ef>(), d_alphas.as<ef>(), part, st);
    }
    const std::vector<ef> sums = reduce_to_host(ctx, part, B, nz);
    ys.insert(ys.end(), sums.begin(), sums.end());
  }
  std::vector<ef> p = interpolate(lagrange_basis_cached((int)ys.size()), ys);
  std::vector<ef> qv(nsk);
  for (int i = 0; i < nsk; i++) qv[i] = upoly_eval(sel[i], zc[0]);
  p = poly_mul(p, interpolate(sel, qv));
  const int deg0 = (d + 1) * (nsk - 1);
  p.resize(deg0 + 1, kb::ef_zero());
  ts.add_ext(p.data(), p.size());
  const ef r0 = ts.sample_ext();
  challenges.push_back(r0);
  ef sum = poly_eval(p, r0);
  grind(ctx, ts, job.p16, sumcheck_pow_bits(s.security_bits, deg0));
  std::vector<ef> selr(nsk);
  ef mmf = kb::ef_zero();
  for (int i = 0; i < nsk; i++) {
    selr[i] = upoly_eval(sel[i], r0);
    mmf = kb::ef_add(mmf, kb::ef_mul(qv[i], selr[i]));
  }
  DBuf cols(sizeof(ef) * size_t(2 * W) * S, st);
  {
    DBuf d_sel = upload(ctx, selr);
    ProfScope _ps(ctx, "prog_fold0");
    launch_prog_fold0(wit, pre.as<uint32_t>(), P, n, k, W, d_sel.as<ef>(), cols.as<ef>(), st);
  }
  // rounds >= 1: sums at z = 0, 2, .., d; z = 1 from the claim
  DBuf eqr;
  if (R >= 1) {
    eqr = DBuf(sizeof(ef) * (S / 2), st);
    launch_fold_cols(nullptr, nullptr, 0, 0, nullptr, st, eq0.as<ef>(), eqr.as<ef>(), S / 2);
  }
  // Degrees 2 and 3 without grinding: every round's transcript on the device (the finishing
  // kernel of an eq-factor round with d + 1 points), one host wait for the phase.
  const bool on_device = R >= 1 && (d == 2 || d == 3) && sumcheck_pow_bits(s.security_bits, d + 1) == 0;
  if (on_device) {
    const int kind = d == 3 ? FIN_EQSC4 : FIN_EQSC3;
    DevPhase ph(ctx, ts, R, size_t(8) * (d + 2), sum, mmf, job.p16, zc.data() + 1);
    for (int round = 1; round <= R; round++) {
      const int m = R - round + 1;
      const size_t half = size_t(1) << (m - 1);
      const int B = prog_zc_blocks(half);
      ef* part = ctx.partials(size_t(B) * d);
      {
        ProfScope _ps(ctx, "prog_zc_ef");
        launch_prog_zc_ef(cols.as<ef>(), m, W, code.as<uint2>(), n_code, consts.as<uint32_t>(), d, eqr.as<ef>(),
                          d_alphas.as<ef>(), part, st);
      }
      ph.finish_round(kind, part, B);
      DBuf nc(sizeof(ef) * size_t(2 * W) * half, st);
      DBuf eqn(sizeof(ef) * std::max<size_t>(half / 2, 1), st);
      {
        ProfScope _ps(ctx, "fold");
        launch_fold_cols_dev(cols.as<ef>(), nc.as<ef>(), 2 * W, half, ph.chs + (round - 1), st,
                             half >= 2 ? eqr.as<ef>() : nullptr, eqn.as<ef>(), half / 2);
      }
      cols = std::move(nc);
      eqr = std::move(eqn);
    }
    const std::vector<ef> ch = ph.finish(&sum, &mmf);
    challenges.insert(challenges.end(), ch.begin(), ch.end());
  }
  const auto& basis = lagrange_basis_cached(d + 1);
  for (int round = 1; !on_device && round <= R; round++) {
    const int m = R - round + 1;
    const size_t half = size_t(1) << (m - 1);
    const int B = prog_zc_blocks(half);
    ef* part = ctx.partials(size_t(B) * d);
    {
      ProfScope _ps(ctx, "prog_zc_ef");
      launch_prog_zc_ef(cols.as<ef>(), m, W, code.as<uint2>(), n_code, consts.as<uint32_t>(), d, eqr.as<ef>(),
                        d_alphas.as<ef>(), part, st);
    }
    const std::vector<ef> sz = reduce_to_host(ctx, part, B, d);
    const ef& r = zc[round];
    std::vector<ef> e(d + 1);
    e[0] = kb::ef_mul(sz[0], mmf);
    for (int z = 2; z <= d; z++) e[z] = kb::ef_mul(sz[z - 1], mmf);
    e[1] = kb::ef_mul(kb::ef_sub(sum, kb::ef_mul(e[0], kb::ef_sub(kb::ef_one(), r))), kb::ef_inv(r));
    std::vector<ef> q = interpolate(basis, e);
    q = poly_mul(q, {kb::ef_sub(kb::ef_one(), r), kb::ef_sub(kb::ef_add(r, r), kb::ef_one())});
    q.resize(d + 2, kb::ef_zero());
    ts.add_ext(q.data(), q.size());
    const ef c = ts.sample_ext();
    challenges.push_back(c);
    sum = poly_eval(q, c);
    grind(ctx, ts, job.p16, sumcheck_pow_bits(s.security_bits, d + 1));
    mmf = kb::ef_mul(kb::ef_add(kb::ef_mul(kb::ef_sub(kb::ef_one(), r), kb::ef_sub(kb::ef_one(), c)), kb::ef_mul(r, c)),
                     mmf);
    DBuf nc(sizeof(ef) * size_t(2 * W) * half, st);
    DBuf eqn(sizeof(ef) * std::max<size_t>(half / 2, 1), st);
    {
      ProfScope _ps(ctx, "fold");
      launch_fold_cols_at(cols.as<ef>(), nc.as<ef>(), 2 * W, half, c, st, half >= 2 ? eqr.as<ef>() : nullptr,
                          eqn.as<ef>(), half / 2);
    }
    cols = std::move(nc);
    eqr = std::move(eqn);
  }
  std::vector<ef> fin(size_t(2) * W);
  ctx.to_host(fin.data(), cols.as<ef>(), sizeof(ef) * fin.size());
  up.assign(fin.begin() + P, fin.begin() + W);
  down.assign(fin.begin() + W + P, fin.end());
}

std::vector<uint32_t> prove_air(Context& ctx, const ProofJob& job, const uint32_t* wit, Timings* tm,
                                const std::vector<cudaEvent_t>* tile_ready) {
  const Settings& s = job.settings;
  const ProgramAir* prog = job.prog;
  const int n = job.log_n, k = s.univariate_skips, W = prog ? prog->witness_columns() : AIR_W;
  const int NC = prog ? prog->NC : AIR_NC, LOGW = log2_up(size_t(W));
  if (k >= n) throw std::invalid_argument("univariate_skips must be smaller than log_n_rows");
  if (s.fold_first != 7 || s.fold_rest != 4) throw std::invalid_argument("folding factors other than (7, 4)");
  const size_t N = size_t(1) << n, S = N >> k;
  const int m0 = n + LOGW;
  const WhirSchedule ws = WhirSchedule::build(m0, s);
  cudaStream_t st = ctx.stream;
  Transcript ts(&job.p16);
  TranscriptLog tlog;
  if (ctx.dump_transcript) ts.log = &tlog;
  for (uint32_t x : ws.domain_separator()) ts.ch.observe(kb::to_mont(x));
  const double t0 = now_ms();
  ts.phase("commit");

  // ---------------------------------------------------------------- 1) commit
  const size_t t_len = size_t(W) * N;
  const int lu = ws.c[0].fold, lv = m0 - lu;
  int lh_v, ll_v;
  split_vars(lv, lh_v, ll_v);
  LdeSource src0{wit, t_len, 1, lv, ws.c[0].log_inv_rate, 0};
  src0.n_cols = (int)(((t_len + (size_t(1) << lv) - 1) >> lv) + 7) / 8 * 8;
  Commitment c0 = commit(ctx, src0, m0, ws.c[0].fold, job.p24, job.p16, tile_ready);
  ts.add_base(c0.root, 8);
  // Commitment OOD: F_0[u] = sum_v T[u, v] eq(pt_v, v), answer = sum_u eq(pt_u, u) F_0[u].
  std::vector<std::vector<ef>> ood_pts;
  std::vector<ef> ood_vals;
  std::vector<std::vector<ef>> Fu;  // per initial constraint, the 2^lu partial evaluations
  auto partial_eval = [&](const std::vector<ef>& pt) {
    std::vector<ef> pv(pt.begin() + lu, pt.end());
    EqPair e = eq_pair(ctx, pv, lh_v);
    DBuf out(sizeof(ef) * (size_t(1) << lu) * 17, st);  // results + 16 split partials
    const size_t scratch_bytes = mle_partial_scratch_bytes(lu, lh_v, ll_v);
    DBuf scratch(scratch_bytes, st);
    {
      ProfScope _ps(ctx, "whir_partial_eval");
      if (!launch_mle_partial_mma(wit, t_len, lu, lh_v, ll_v, e.hi.as<ef>(), e.lo.as<ef>(), out.as<ef>(), scratch.as<void>(), st))
        launch_mle_partial_base(wit, t_len, lu, lh_v, ll_v, 1, e.hi.as<ef>(), e.lo.as<ef>(), out.as<ef>(), st);
    }
    std::vector<ef> h(size_t(1) << lu);
    ctx.to_host(h.data(), out.as<ef>(), sizeof(ef) * h.size());
    return h;
  };
  for (int q = 0; q < ws.c[0].ood; q++) {
    ef z = ts.sample_ext();
    std::vector<ef> pt = pow_point(z, m0);
    std::vector<ef> f = partial_eval(pt);
    std::vector<ef> eu = eq_table_host(std::vector<ef>(pt.begin(), pt.begin() + lu));
    ef y = kb::ef_zero();
    for (size_t u = 0; u < f.size(); u++) y = kb::ef_add(y, kb::ef_mul(eu[u], f[u]));
    ts.add_ext(&y, 1);
    ood_pts.push_back(pt);
    ood_vals.push_back(y);
    Fu.push_back(f);
  }
  const double t1 = now_ms();

  // ---------------------------------------------------------------- 2) challenges
  ts.phase("batching");
  grind(ctx, ts, job.p16, batching_pow_bits(s.security_bits, log2_up(size_t(NC))));
  ef alpha = ts.sample_ext();
  std::vector<ef> alphas(NC);
  alphas[0] = kb::ef_one();
  for (int i = 1; i < NC; i++) alphas[i] = kb::ef_mul(alphas[i - 1], alpha);
  DBuf d_alphas = upload(ctx, alphas);
  // beta_f = MDS^T alpha_f for the 8 full rounds (constraints 16f.. for the beginning rounds,
  // 84 + 16(f - 4).. for the ending rounds); MDS = circ(2 M4, M4, M4, M4).
  std::vector<ef> betas(8 * 16, kb::ef_zero());
  if (!prog) {
    static const int M4[4][4] = {{2, 3, 1, 1}, {1, 2, 3, 1}, {1, 1, 2, 3}, {3, 1, 1, 2}};
    for (int f = 0; f < 8; f++) {
      const int c0 = f < 4 ? 16 * f : 84 + 16 * (f - 4);
      for (int j = 0; j < 16; j++)
        for (int i = 0; i < 16; i++) {
          const int mij = M4[i % 4][j % 4] * (i / 4 == j / 4 ? 2 : 1);
          betas[16 * f + j] = kb::ef_add(betas[16 * f + j], kb::ef_mul_f(alphas[c0 + i], fm(mij)));
        }
    }
  }
  DBuf d_betas = upload(ctx, betas);
  grind(ctx, ts, job.p16, batching_pow_bits(s.security_bits, n));
  std::vector<ef> zc(n + 1 - k);
  for (auto& x : zc) x = ts.sample_ext();

  // ---------------------------------------------------------------- 3) zerocheck
  ts.phase("zerocheck");
  const int nsk = 1 << k;
  const auto sel = [&] {
    auto b = lagrange_basis_cached(nsk);
    return b;
  }();  // L_i on {0..2^k-1}
  const int nz = 3 * (nsk - 1) - nsk + 1;
  std::vector<ef> zc_tail(zc.begin() + 1, zc.end());
  DBuf eq0 = eq_table_dev(ctx, zc_tail);
  std::vector<ef> challenges;
  std::vector<ef> inner_up(W), inner_down(W);
  if (prog) {
    zerocheck_program(ctx, ts, job, *prog, wit, d_alphas, zc, eq0, challenges, inner_up, inner_down);
  } else {
    ef sum = kb::ef_zero();
    ef mmf = kb::ef_one();
    DBuf cols;
    // the committed-column combination sum_i alpha_i col_(17+i) of every row; folded, it is the
    // last of the W + 1 columns of the rounds >= 1
    DBuf arow(sizeof(ef) * N, st);
    {
      std::vector<uint32_t> lw(size_t(nz) * nsk);
      for (int zi = 0; zi < nz; zi++)
        for (int j = 0; j < nsk; j++) lw[size_t(zi) * nsk + j] = upoly_eval_f(sel[j], fm(nsk + zi));
      DBuf d_lw = upload(ctx, lw);
      const int nb = zc0_blocks(n, k), nbr = zc0_row_blocks(n);
      ef* part = ctx.partials(size_t(nb + nbr) * nz);
      {
        DBuf q(sizeof(uint32_t) * ZC0_NQ * N, st);
        { ProfScope _ps(ctx, "zc0_rows"); launch_zc0_rows(wit, n, k, nz, d_lw.as<uint32_t>(), eq0.as<ef>(), d_alphas.as<ef>(), job.air, q.as<uint32_t>(), part + size_t(nb) * nz, arow.as<ef>(), st); }
        { ProfScope _ps(ctx, "zc0_eval"); launch_zc0_eval(wit, q.as<uint32_t>(), n, k, nz, d_lw.as<uint32_t>(), eq0.as<ef>(), d_alphas.as<ef>(), d_betas.as<ef>(), job.air, part, st); }
      }
      std::vector<ef> sums = reduce_to_host(ctx, part, nb + nbr, nz);
      std::vector<ef> ys(nsk, kb::ef_zero());
      ys.insert(ys.end(), sums.begin(), sums.end());
      std::vector<ef> p = interpolate(lagrange_basis_cached((int)ys.size()), ys);
      std::vector<ef> qv(nsk);
      for (int i = 0; i < nsk; i++) qv[i] = upoly_eval(sel[i], zc[0]);
      p = poly_mul(p, interpolate(sel, qv));
      const int deg = 4 * (nsk - 1);
      p.resize(deg + 1, kb::ef_zero());
      ts.add_ext(p.data(), p.size());
      ef r0 = ts.sample_ext();
      challenges.push_back(r0);
      sum = poly_eval(p, r0);
      grind(ctx, ts, job.p16, sumcheck_pow_bits(s.security_bits, deg));
      std::vector<ef> selr(nsk);
      mmf = kb::ef_zero();
      for (int i = 0; i < nsk; i++) {
        selr[i] = upoly_eval(sel[i], r0);
        mmf = kb::ef_add(mmf, kb::ef_mul(qv[i], selr[i]));
      }
      DBuf d_sel = upload(ctx, selr);
      cols = DBuf(sizeof(ef) * size_t(W + 1) * S, st);
      { ProfScope _ps(ctx, "zc0_fold"); launch_zc0_fold(wit, n, k, d_sel.as<ef>(), cols.as<ef>(), st); }
      { ProfScope _ps(ctx, "zc0_fold"); launch_zc0_fold_ef(arow.as<ef>(), n, k, d_sel.as<ef>(), cols.as<ef>() + size_t(W) * S, st); }
      arow.reset();
    }
    const auto basis4 = lagrange_basis_cached(4);
    // eq table of round r (over zc[1+r..]) = eq table of round r-1 with its leading variable
    // summed out; each fold below carries it along.
    DBuf eqr;
    if (n - k >= 1) {
      eqr = DBuf(sizeof(ef) * (S / 2), st);
      { ProfScope _ps(ctx, "fold"); launch_fold_cols(nullptr, nullptr, 0, 0, nullptr, st, eq0.as<ef>(), eqr.as<ef>(), S / 2); }
    }
    const bool zc_on_device = sumcheck_pow_bits(s.security_bits, 4) == 0;
    if (zc_on_device && n - k >= 1) {
      // every round's transcript on the device: the sums, the finishing kernel (interpolation,
      // absorption, challenge) and the fold at the device-sampled challenge, one host wait
      DevPhase ph(ctx, ts, n - k, 40, sum, mmf, job.p16, zc.data() + 1);
      for (int round = 1; round <= n - k; round++) {
        const int m = n - k - round + 1;
        const size_t half = size_t(1) << (m - 1);
        const int nb = zc_ef_blocks(m);
        ef* part = ctx.partials(size_t(nb) * 3);
        { ProfScope _ps(ctx, zc_eval_is_dense(m) ? "zc_eval_dense" : "zc_eval_ef"); launch_zc_eval_ef(cols.as<ef>(), m, eqr.as<ef>(), d_alphas.as<ef>(), d_betas.as<ef>(), job.air, part, st); }
        ph.finish_round(FIN_EQSC4, part, nb);
        DBuf nc(sizeof(ef) * size_t(W + 1) * half, st);
        DBuf eqn(sizeof(ef) * std::max<size_t>(half / 2, 1), st);
        { ProfScope _ps(ctx, "fold"); launch_fold_cols_dev(cols.as<ef>(), nc.as<ef>(), W + 1, half, ph.chs + (round - 1), st,
                                                      half >= 2 ? eqr.as<ef>() : nullptr, eqn.as<ef>(), half / 2); }
        cols = std::move(nc);
        eqr = std::move(eqn);
      }
      const std::vector<ef> ch = ph.finish(&sum, &mmf);
      challenges.insert(challenges.end(), ch.begin(), ch.end());
    }
    for (int round = 1; !zc_on_device && round <= n - k; round++) {
      const int m = n - k - round + 1;  // variables of the current columns
      const size_t half = size_t(1) << (m - 1);
      const int nb = zc_ef_blocks(m);
      ef* part = ctx.partials(size_t(nb) * 3);
      { ProfScope _ps(ctx, zc_eval_is_dense(m) ? "zc_eval_dense" : "zc_eval_ef"); launch_zc_eval_ef(cols.as<ef>(), m, eqr.as<ef>(), d_alphas.as<ef>(), d_betas.as<ef>(), job.air, part, st); }
      std::vector<ef> s3 = reduce_to_host(ctx, part, nb, 3);
      const ef& r = zc[round];
      ef e0 = kb::ef_mul(s3[0], mmf), e2 = kb::ef_mul(s3[1], mmf), e3 = kb::ef_mul(s3[2], mmf);
      ef e1 = kb::ef_mul(kb::ef_sub(sum, kb::ef_mul(e0, kb::ef_sub(kb::ef_one(), r))), kb::ef_inv(r));
      std::vector<ef> p = interpolate(basis4, {e0, e1, e2, e3});
      p = poly_mul(p, {kb::ef_sub(kb::ef_one(), r), kb::ef_sub(kb::ef_add(r, r), kb::ef_one())});
      ts.add_ext(p.data(), p.size());
      ef c = ts.sample_ext();
      challenges.push_back(c);
      sum = poly_eval(p, c);
      grind(ctx, ts, job.p16, sumcheck_pow_bits(s.security_bits, 4));
      mmf = kb::ef_mul(kb::ef_add(kb::ef_mul(kb::ef_sub(kb::ef_one(), r), kb::ef_sub(kb::ef_one(), c)), kb::ef_mul(r, c)),
                       mmf);
      DBuf nc(sizeof(ef) * size_t(W + 1) * half, st);
      DBuf eqn(sizeof(ef) * std::max<size_t>(half / 2, 1), st);
      { ProfScope _ps(ctx, "fold"); launch_fold_cols_at(cols.as<ef>(), nc.as<ef>(), W + 1, half, c, st,
                                                     half >= 2 ? eqr.as<ef>() : nullptr, eqn.as<ef>(), half / 2); }
      cols = std::move(nc);
      eqr = std::move(eqn);
    }
    // inner sums: every up / down column evaluated at (r_0 over the skipped variables, r_tail)
    // The zerocheck's returned challenges replace the eq challenges from here on
    // (crates/air/src/prove.rs:114 rebinds zerocheck_challenges).
    const std::vector<ef> rtail(challenges.begin() + 1, challenges.end());
    {
      std::vector<ef> selr(nsk);
      for (int i = 0; i < nsk; i++) selr[i] = upoly_eval(sel[i], challenges[0]);
      DBuf d_sel = upload(ctx, selr);
      const int ll_t = std::min(12, n - k), lh_t = n - k - ll_t;
      EqPair et = eq_pair(ctx, rtail, lh_t);
      const size_t plen = size_t(W) * (1 + (size_t(nsk) << lh_t));
      DBuf up(sizeof(ef) * plen, st), down(sizeof(ef) * plen, st);
      DBuf limbs(size_t(64) << ll_t, st);
      {
        ProfScope _ps(ctx, "inner_sums");
        tuned(ctx, TUNE_INNER, uint64_t(n) | uint64_t(k) << 8, [&](int plan) {
          launch_inner_sums(wit, n, k, ll_t, et.hi.as<ef>(), et.lo.as<ef>(), d_sel.as<ef>(), up.as<ef>(), down.as<ef>(),
                            limbs.as<uint8_t>(), st, plan, ctx.pipe_timeouts);
        });
      }
      unsigned timeouts = 0;
      ctx.to_host_many({{inner_up.data(), up.as<ef>(), sizeof(ef) * W}, {inner_down.data(), down.as<ef>(), sizeof(ef) * W},
                        {&timeouts, ctx.pipe_timeouts, sizeof(unsigned)}});
      if (timeouts) throw std::runtime_error("inner sums: a bounded pipeline wait ran out on the device");
    }
    cols.reset();
  }
  const std::vector<ef> rtail(challenges.begin() + 1, challenges.end());
  DBuf eqt = eq_table_dev(ctx, rtail);
  const double t2 = now_ms();

  // ---------------------------------------------------------------- 4) inner sumcheck
  ts.phase("inner_sums");
  ts.add_ext(inner_up.data(), W);
  ts.add_ext(inner_down.data(), W);
  grind(ctx, ts, job.p16, batching_pow_bits(s.security_bits, LOGW));
  std::vector<ef> cbs(LOGW);
  for (auto& x : cbs) x = ts.sample_ext();
  std::vector<ef> eqc = eq_table_host(cbs);
  eqc.resize(W);
  DBuf d_eqc = upload(ctx, eqc);
  DBuf B(sizeof(ef) * N, st);
  if (prog) {
    ProfScope _ps(ctx, "batch_cols");
    launch_batch_cols_generic(wit, n, W, d_eqc.as<ef>(), B.as<ef>(), st);
  } else {
    DBuf limbs(colsum_limb_bytes(W), st);
    ProfScope _ps(ctx, "batch_cols");
    launch_batch_cols_mma(wit, n, d_eqc.as<ef>(), B.as<ef>(), limbs.as<uint8_t>(), st);
  }
  ef alpha2 = ts.sample_ext();
  std::vector<ef> sub(nsk);
  {
    const int nb = sub_eval_blocks(n, k);
    ef* part = ctx.partials(size_t(nb) * nsk * 2);
    { ProfScope _ps(ctx, "sub_evals"); launch_sub_evals(B.as<ef>(), n, k, nullptr, eqt.as<ef>(), part, st); }
    std::vector<ef> ud = reduce_to_host(ctx, part, nb, nsk * 2);
    for (int j = 0; j < nsk; j++) sub[j] = kb::ef_add(ud[2 * j], kb::ef_mul(alpha2, ud[2 * j + 1]));
  }
  ts.add_ext(sub.data(), sub.size());
  std::vector<ef> eps(k);
  for (auto& x : eps) x = ts.sample_ext();
  std::vector<ef> point = eps;
  point.insert(point.end(), rtail.begin(), rtail.end());
  DBuf A(sizeof(ef) * N, st);
  {
    DBuf ep = eq_table_dev(ctx, point);
    DBuf da2 = scalar_dev(ctx, alpha2);
    { ProfScope _ps(ctx, "inner_mle"); launch_inner_mle(ep.as<ef>(), n, da2.as<ef>(), A.as<ef>(), st); }
  }
  ef inner_sum = kb::ef_zero();
  {
    std::vector<ef> ee = eq_table_host(eps);
    for (int j = 0; j < nsk; j++) inner_sum = kb::ef_add(inner_sum, kb::ef_mul(ee[j], sub[j]));
  }
  const auto basis3 = lagrange_basis_cached(3);
  std::vector<ef> inner_ch;
  ts.phase("inner_sumcheck");
  const bool inner_on_device = sumcheck_pow_bits(s.security_bits, 2) == 0;
  if (inner_on_device) {
    DevPhase ph(ctx, ts, n, 24, inner_sum, kb::ef_one(), job.p16);
    // round 0 evaluates A and B as they are (the finish its own kernel); round r >= 1 folds
    // them at challenge r - 1, evaluates and finishes in one kernel; the last challenge's fold
    // leaves the final values
    for (int round = 0; round < n; round++) {
      const size_t half = N >> (round + 1);
      if (round == 0) {
        const int nb = prod_blocks(half);
        ef* part = ctx.partials(size_t(nb) * 2);
        {
          ProfScope _ps(ctx, "prod_eval");
          launch_prod_eval(A.as<ef>(), B.as<ef>(), half, part, st);
        }
        ph.finish_round(FIN_PROD, part, nb);
      } else {
        ef* part = ctx.partials(size_t(2) * fold_eval_blocks(half));
        DBuf na(sizeof(ef) * 2 * half, st), nbuf(sizeof(ef) * 2 * half, st);
        {
          ProfScope _ps(ctx, "fold_eval");
          launch_pair_fold_eval(2, A.as<ef>(), B.as<ef>(), ph.chs + (round - 1), na.as<ef>(), nbuf.as<ef>(), half, part,
                                &ph.fin, st);
        }
        A = std::move(na);
        B = std::move(nbuf);
      }
    }
    {
      DBuf na(sizeof(ef), st), nbuf(sizeof(ef), st);
      { ProfScope _ps(ctx, "fold"); launch_fold2_dev(A.as<ef>(), B.as<ef>(), na.as<ef>(), nbuf.as<ef>(), 1, ph.chs + (n - 1), st); }
      A = std::move(na);
      B = std::move(nbuf);
    }
    inner_ch = ph.finish(&inner_sum, nullptr);
  }
  for (int round = 0; !inner_on_device && round < n; round++) {
    const size_t half = N >> (round + 1);
    const int nb = prod_blocks(half);
    ef* part = ctx.partials(size_t(nb) * 2);
    { ProfScope _ps(ctx, "prod_eval"); launch_prod_eval(A.as<ef>(), B.as<ef>(), half, part, st); }
    std::vector<ef> s02 = reduce_to_host(ctx, part, nb, 2);
    ef s1 = kb::ef_sub(inner_sum, s02[0]);
    std::vector<ef> p = interpolate(basis3, {s02[0], s1, s02[1]});
    ts.add_ext(p.data(), p.size());
    ef c = ts.sample_ext();
    inner_ch.push_back(c);
    inner_sum = poly_eval(p, c);
    grind(ctx, ts, job.p16, sumcheck_pow_bits(s.security_bits, 2));
    DBuf na(sizeof(ef) * half, st), nbuf(sizeof(ef) * half, st);
    { ProfScope _ps(ctx, "fold"); launch_fold2_at(A.as<ef>(), B.as<ef>(), na.as<ef>(), nbuf.as<ef>(), half, c, st); }
    A = std::move(na);
    B = std::move(nbuf);
  }
  ef packed_value;
  ctx.to_host(&packed_value, B.as<ef>(), sizeof(ef));
  A.reset();
  B.reset();
  std::vector<ef> final_point = cbs;
  final_point.insert(final_point.end(), inner_ch.begin(), inner_ch.end());
  const double t3 = now_ms();

  // ---------------------------------------------------------------- 5) WHIR opening
  ts.phase("whir");
  {
    // initial constraints: the commitment OOD points, then the statement
    std::vector<std::vector<ef>> pts = ood_pts;
    pts.push_back(final_point);
    std::vector<ef> vals = ood_vals;
    vals.push_back(packed_value);
    Fu.push_back(partial_eval(final_point));
    ef gamma = ts.sample_ext();
    std::vector<ef> coef(pts.size());
    ef sigma = kb::ef_zero(), cur = kb::ef_one();
    for (size_t j = 0; j < pts.size(); j++) {
      coef[j] = cur;
      sigma = kb::ef_add(sigma, kb::ef_mul(cur, vals[j]));
      cur = kb::ef_mul(cur, gamma);
    }
    // first folding block on the 2^lu partial evaluations
    std::vector<std::vector<ef>> E;
    for (auto& pt : pts) E.push_back(eq_table_host(std::vector<ef>(pt.begin(), pt.begin() + lu)));
    std::vector<std::vector<ef>> G = Fu;
    std::vector<ef> r0;
    whir_sumcheck_host(ctx, ts, G, E, coef, sigma, lu, ws.fold_pow_bits, job.p16, r0);
    // g_1 = T(r0, .), w_1 = sum_j coef_j eq(pt_j^u, r0) eq(pt_j^v, .)
    int m = m0 - lu;
    DBuf g(sizeof(ef) << m, st), w(sizeof(ef) << m, st);
    {
      DBuf er = upload(ctx, eq_table_host(r0));
      DBuf fscratch(whir_fold_T_scratch_bytes(lu), st);
      { ProfScope _ps(ctx, "whir_fold_T"); launch_whir_fold_T(wit, t_len, lu, m, er.as<ef>(), g.as<ef>(), st, fscratch.as<uint32_t>()); }
      WL_CUDA(cudaMemsetAsync(w.as<void>(), 0, sizeof(ef) << m, st));
      std::vector<std::vector<ef>> pv;
      std::vector<ef> cv;
      for (size_t j = 0; j < pts.size(); j++) {
        pv.emplace_back(pts[j].begin() + lu, pts[j].end());
        cv.push_back(kb::ef_mul(coef[j], E[j][0]));
      }
      add_eq_ef(ctx, w.as<ef>(), m, pv, cv);
    }
    std::vector<ef> last_r = r0;
    std::deque<Commitment> commits;  // stable addresses: `prev` points into it
    const Commitment* prev = &c0;
    for (int i = 0; i < ws.num_rounds; i++) {
      const WhirRound& ci = ws.c[i];
      const WhirRound& cn = ws.c[i + 1];
      ts.phase(("whir_round_" + std::to_string(i + 1)).c_str());
      LdeSource src{g.as<uint32_t>(), size_t(8) << m, 8, m - cn.fold, cn.log_inv_rate, 128};
      commits.push_back(commit(ctx, src, m, cn.fold, job.p24, job.p16));
      const Commitment& cd = commits.back();
      ts.add_base(cd.root, 8);
      std::vector<std::vector<ef>> npts_ef;
      std::vector<ef> nvals;
      for (int q = 0; q < cn.ood; q++) {
        ef z = ts.sample_ext();
        std::vector<ef> pt = pow_point(z, m);
        ef y = mle_eval_dev(ctx, g.as<ef>(), m, pt);
        ts.add_ext(&y, 1);
        npts_ef.push_back(pt);
        nvals.push_back(y);
      }
      grind(ctx, ts, job.p16, ci.pow_bits);
      std::vector<uint32_t> q = sample_queries(ts, prev->log_leaves, ci.queries);
      const std::vector<ef> mono = fold_monomials(prev->fold, last_r);
      const std::vector<ef> stir_vals = open(ctx, *prev, q, ts, &mono);
      const uint32_t gen = kb::two_adic_gen_m(prev->log_leaves);
      std::vector<std::vector<uint32_t>> stir_pts;
      for (size_t t = 0; t < q.size(); t++) {
        uint32_t y = kb::pow_m(gen, q[t]);
        std::vector<uint32_t> pt(m);
        for (int b = 0; b < m; b++) { pt[b] = y; y = kb::mul(y, y); }
        stir_pts.push_back(pt);
      }
      ef gm = ts.sample_ext();
      std::vector<ef> coef_ef, coef_f;
      ef cc = kb::ef_one();
      for (size_t t = 0; t < npts_ef.size(); t++) {
        coef_ef.push_back(cc);
        sigma = kb::ef_add(sigma, kb::ef_mul(cc, nvals[t]));
        cc = kb::ef_mul(cc, gm);
      }
      for (size_t t = 0; t < stir_pts.size(); t++) {
        coef_f.push_back(cc);
        sigma = kb::ef_add(sigma, kb::ef_mul(cc, stir_vals[t]));
        cc = kb::ef_mul(cc, gm);
      }
      add_eq_ef(ctx, w.as<ef>(), m, npts_ef, coef_ef);
      add_eq_f(ctx, w.as<ef>(), m, stir_pts, coef_f);
      last_r.clear();
      whir_sumcheck_dev(ctx, ts, g, w, m, sigma, cn.fold, ws.fold_pow_bits, job.p16, last_r);
      prev = &cd;
    }
    // final round
    ts.phase("whir_final");
    std::vector<ef> gf(size_t(1) << m), wf(size_t(1) << m);
    ctx.to_host_many({{gf.data(), g.as<ef>(), sizeof(ef) << m}, {wf.data(), w.as<ef>(), sizeof(ef) << m}});
    ts.add_ext(gf.data(), gf.size());
    const WhirRound& cl = ws.c[ws.num_rounds];
    grind(ctx, ts, job.p16, cl.pow_bits);
    std::vector<uint32_t> q = sample_queries(ts, prev->log_leaves, cl.queries);
    open(ctx, *prev, q, ts);
    std::vector<std::vector<ef>> Gf{gf}, Wf{wf};
    std::vector<ef> fr;
    whir_sumcheck_host(ctx, ts, Gf, Wf, {kb::ef_one()}, sigma, ws.final_vars, ws.fold_pow_bits, job.p16, fr);
  }
  const double t4 = now_ms();
  if (tm) {
    tm->commit_ms = t1 - t0;
    tm->zerocheck_ms = t2 - t1;
    tm->inner_ms = t3 - t2;
    tm->whir_ms = t4 - t3;
    tm->total_ms = t4 - t0;
  }
  if (ts.log) ctx.last_dump = tlog.json(ts.proof.size());
  return to_canonical(ts.proof);
}

std::vector<uint32_t> prove_air_host(Context& ctx, const ProofJob& job, const uint32_t* wit_host, Timings* tm) {
  const size_t N = size_t(1) << job.log_n;
  if (job.prog) {
    // a constraint-program AIR: the whole witness, then the proof
    const size_t words = N * size_t(job.prog->witness_columns());
    DBuf wit(sizeof(uint32_t) * words, ctx.stream);
    WL_CUDA(cudaMemcpyAsync(wit.as<uint32_t>(), wit_host, sizeof(uint32_t) * words, cudaMemcpyHostToDevice,
                            ctx.stream));
    launch_to_mont(wit.as<uint32_t>(), words, ctx.stream);
    return prove_air(ctx, job, wit.as<uint32_t>(), tm);
  }
  DBuf wit(sizeof(uint32_t) * N * AIR_W, ctx.stream);
  // the copy stream must not start before the allocation is usable
  cudaEvent_t alloc_done;
  WL_CUDA(cudaEventCreateWithFlags(&alloc_done, cudaEventDisableTiming));
  WL_CUDA(cudaEventRecord(alloc_done, ctx.stream));
  WL_CUDA(cudaStreamWaitEvent(ctx.copy_stream, alloc_done, 0));
  // The copy stream only copies (back to back, so the copy engine never waits for a kernel);
  // the conversion stream converts each tile to Montgomery form once its copy has landed.
  WL_CUDA(cudaStreamWaitEvent(ctx.conv_stream, alloc_done, 0));
  std::vector<cudaEvent_t> copied, ready;
  auto destroy = [&] {
    for (auto e : copied) cudaEventDestroy(e);
    for (auto e : ready) cudaEventDestroy(e);
    cudaEventDestroy(alloc_done);
  };
  for (int c0 = 0; c0 < AIR_W; c0 += 16) {
    const size_t cols = std::min(16, AIR_W - c0);
    uint32_t* dst = wit.as<uint32_t>() + size_t(c0) * N;
    cudaEvent_t ec, er;
    WL_CUDA(cudaEventCreateWithFlags(&ec, cudaEventDisableTiming));
    copied.push_back(ec);
    WL_CUDA(cudaEventCreateWithFlags(&er, cudaEventDisableTiming));
    ready.push_back(er);
    WL_CUDA(cudaMemcpyAsync(dst, wit_host + size_t(c0) * N, sizeof(uint32_t) * cols * N, cudaMemcpyHostToDevice,
                            ctx.copy_stream));
    WL_CUDA(cudaEventRecord(ec, ctx.copy_stream));
    WL_CUDA(cudaStreamWaitEvent(ctx.conv_stream, ec, 0));
    launch_to_mont(dst, cols * N, ctx.conv_stream);
    WL_CUDA(cudaEventRecord(er, ctx.conv_stream));
  }
  std::vector<uint32_t> proof;
  try {
    proof = prove_air(ctx, job, wit.as<uint32_t>(), tm, &ready);
  } catch (...) {
    cudaStreamSynchronize(ctx.copy_stream);
    cudaStreamSynchronize(ctx.conv_stream);
    destroy();
    throw;
  }
  destroy();
  return proof;
}

// ------------------------------------------------------------------ a*b - c zerocheck
std::vector<uint32_t> prove_abc(Context& ctx, const kb::P16Consts& p16, int n, int k, const uint32_t* a,
                                const uint32_t* b, const uint32_t* c, std::vector<float>* round_ms) {
  if (k < 1 || k > 4 || k >= n) throw std::invalid_argument("skips must be in [1, 4] and below log_n");
  cudaStream_t st = ctx.stream;
  Transcript ts(&p16);
  const int nsk = 1 << k;
  const size_t S = size_t(1) << (n - k);
  std::vector<ef> r(n + 1 - k);
  for (auto& x : r) x = ts.sample_ext();
  auto sel = lagrange_basis_cached(nsk);
  const int nz = 2 * (nsk - 1) - nsk + 1;
  ef sum = kb::ef_zero(), mmf;
  std::vector<ef> ch;
  cudaEvent_t e0, e1;
  WL_CUDA(cudaEventCreate(&e0));
  WL_CUDA(cudaEventCreate(&e1));
  auto tick = [&]() { WL_CUDA(cudaEventRecord(e0, st)); };
  auto tock = [&]() {
    WL_CUDA(cudaEventRecord(e1, st));
    WL_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    WL_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (round_ms) round_ms->push_back(ms);
  };
  DBuf cols;
  DBuf eq0;
  {
    tick();
    std::vector<uint32_t> lw(size_t(nz) * nsk);
    for (int zi = 0; zi < nz; zi++)
      for (int j = 0; j < nsk; j++) lw[size_t(zi) * nsk + j] = upoly_eval_f(sel[j], fm(nsk + zi));
    DBuf d_lw = upload(ctx, lw);
    eq0 = eq_table_dev(ctx, std::vector<ef>(r.begin() + 1, r.end()));
    const int nb = abc0_blocks(n, k);
    ef* part = ctx.partials(size_t(nb) * nz);
    { ProfScope _ps(ctx, "abc0_eval"); launch_abc0_eval(a, b, c, n, k, nz, d_lw.as<uint32_t>(), eq0.as<ef>(), part, st); }
    std::vector<ef> sums = reduce_to_host(ctx, part, nb, nz);
    std::vector<ef> ys(nsk, kb::ef_zero());
    ys.insert(ys.end(), sums.begin(), sums.end());
    std::vector<ef> p = interpolate(lagrange_basis_cached((int)ys.size()), ys);
    std::vector<ef> qv(nsk);
    for (int i = 0; i < nsk; i++) qv[i] = upoly_eval(sel[i], r[0]);
    p = poly_mul(p, interpolate(sel, qv));
    const int deg = 3 * (nsk - 1);
    p.resize(deg + 1, kb::ef_zero());
    ts.add_ext(p.data(), p.size());
    ef c0 = ts.sample_ext();
    ch.push_back(c0);
    sum = poly_eval(p, c0);
    grind(ctx, ts, p16, sumcheck_pow_bits(128, deg));
    std::vector<ef> selr(nsk);
    mmf = kb::ef_zero();
    for (int i = 0; i < nsk; i++) {
      selr[i] = upoly_eval(sel[i], c0);
      mmf = kb::ef_add(mmf, kb::ef_mul(qv[i], selr[i]));
    }
    DBuf d_sel = upload(ctx, selr);
    cols = DBuf(sizeof(ef) * 3 * S, st);
    { ProfScope _ps(ctx, "abc0_fold"); launch_abc0_fold(a, b, c, n, k, d_sel.as<ef>(), cols.as<ef>(), st); }
    tock();
  }
  const auto basis3 = lagrange_basis_cached(3);
  DBuf eqr;  // eq table of the current round, carried by the folds (see prove_air)
  if (n - k >= 1) {
    eqr = DBuf(sizeof(ef) * (S / 2), st);
    { ProfScope _ps(ctx, "fold"); launch_fold_cols(nullptr, nullptr, 0, 0, nullptr, st, eq0.as<ef>(), eqr.as<ef>(), S / 2); }
  }
  if (n - k >= 1 && sumcheck_pow_bits(128, 3) == 0) {
    // rounds >= 1 with the transcript on the device; per-round times from events recorded at
    // the round boundaries, read after the phase
    DevPhase ph(ctx, ts, n - k, 32, sum, mmf, p16, r.data() + 1);
    std::vector<cudaEvent_t> ev(n - k + 1);
    for (auto& e : ev) WL_CUDA(cudaEventCreate(&e));
    WL_CUDA(cudaEventRecord(ev[0], st));
    // round 1 evaluates the round-0 fold as it is; round r >= 2 folds the columns (and sums the
    // eq table's leading variable out) at challenge r - 1 and evaluates in one pass; the last
    // challenge's fold leaves the three final values
    for (int round = 1; round <= n - k; round++) {
      const int m = n - k - round + 1;
      const size_t half = size_t(1) << (m - 1);
      if (round == 1) {
        const int nb = (int)((half + 31) / 32);
        ef* part = ctx.partials(size_t(nb) * 2);
        {
          ProfScope _ps(ctx, "abc_eval_ef");
          launch_abc_eval_ef(cols.as<ef>(), m, eqr.as<ef>(), part, st);
        }
        ph.finish_round(FIN_EQSC3, part, nb);
      } else {
        ef* part = ctx.partials(size_t(2) * fold_eval_blocks(half));
        DBuf nc(sizeof(ef) * 3 * 2 * half, st), eqn(sizeof(ef) * half, st);
        {
          ProfScope _ps(ctx, "fold_eval");
          launch_abc_fold_eval(cols.as<ef>(), ph.chs + (round - 2), eqr.as<ef>(), nc.as<ef>(), eqn.as<ef>(), half, part,
                               &ph.fin, st);
        }
        cols = std::move(nc);
        eqr = std::move(eqn);
      }
      if (round == n - k) {
        DBuf nc(sizeof(ef) * 3, st);
        { ProfScope _ps(ctx, "fold"); launch_fold_cols_dev(cols.as<ef>(), nc.as<ef>(), 3, 1, ph.chs + (round - 1), st); }
        cols = std::move(nc);
      }
      WL_CUDA(cudaEventRecord(ev[round], st));
    }
    ph.finish(&sum, &mmf);
    for (int round = 1; round <= n - k; round++) {
      float ms = 0;
      WL_CUDA(cudaEventElapsedTime(&ms, ev[round - 1], ev[round]));
      if (round_ms) round_ms->push_back(ms);
    }
    for (auto e : ev) cudaEventDestroy(e);
  }
  for (int round = 1; sumcheck_pow_bits(128, 3) != 0 && round <= n - k; round++) {
    tick();
    const int m = n - k - round + 1;
    const size_t half = size_t(1) << (m - 1);
    const int nb = (int)((half + 31) / 32);
    ef* part = ctx.partials(size_t(nb) * 2);
    { ProfScope _ps(ctx, "abc_eval_ef"); launch_abc_eval_ef(cols.as<ef>(), m, eqr.as<ef>(), part, st); }
    std::vector<ef> s2 = reduce_to_host(ctx, part, nb, 2);
    const ef& rr = r[round];
    ef v0 = kb::ef_mul(s2[0], mmf), v2 = kb::ef_mul(s2[1], mmf);
    ef v1 = kb::ef_mul(kb::ef_sub(sum, kb::ef_mul(v0, kb::ef_sub(kb::ef_one(), rr))), kb::ef_inv(rr));
    std::vector<ef> p = interpolate(basis3, {v0, v1, v2});
    p = poly_mul(p, {kb::ef_sub(kb::ef_one(), rr), kb::ef_sub(kb::ef_add(rr, rr), kb::ef_one())});
    ts.add_ext(p.data(), p.size());
    ef cc = ts.sample_ext();
    ch.push_back(cc);
    sum = poly_eval(p, cc);
    grind(ctx, ts, p16, sumcheck_pow_bits(128, 3));
    mmf = kb::ef_mul(kb::ef_add(kb::ef_mul(kb::ef_sub(kb::ef_one(), rr), kb::ef_sub(kb::ef_one(), cc)),
                                kb::ef_mul(rr, cc)),
                     mmf);
    DBuf nc(sizeof(ef) * 3 * half, st);
    DBuf eqn(sizeof(ef) * std::max<size_t>(half / 2, 1), st);
    { ProfScope _ps(ctx, "fold"); launch_fold_cols_at(cols.as<ef>(), nc.as<ef>(), 3, half, cc, st,
                                                   half >= 2 ? eqr.as<ef>() : nullptr, eqn.as<ef>(), half / 2); }
    cols = std::move(nc);
    eqr = std::move(eqn);
    tock();
  }
  ef fin[3];
  ctx.to_host(fin, cols.as<ef>(), sizeof(fin));
  ts.add_ext(fin, 3);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return to_canonical(ts.proof);
}

}  // namespace wl
