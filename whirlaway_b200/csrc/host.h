// Host-side pieces of the prover: the Fiat-Shamir transcript (DuplexChallenger over
// Poseidon2-16 plus the proof buffer of whir-p3's ProverState), small-polynomial helpers
// (Lagrange interpolation on integer nodes, products, evaluation, univariate selectors),
// the WHIR round schedule and the workload generator (rand 0.9 StdRng). All field values
// are Montgomery form unless a name says otherwise.
#pragma once
#include <algorithm>
#include <chrono>
#include <cstdint>
#include <exception>
#include <mutex>
#include <stdexcept>
#include <string>
#include <system_error>
#include <thread>
#include <vector>

#include "air.cuh"
#include "poseidon2.cuh"

namespace wl {

using kb::ef;

// ------------------------------------------------------------------ settings
// AirSettings (crates/air/src/lib.rs:13-41) plus WHIR_POW_BITS (crates/air/src/lib.rs:9).
struct Settings {
  int security_bits = 128;
  int log_inv_rate = 1;
  int fold_first = 7;
  int fold_rest = 4;
  int univariate_skips = 4;
  int rs_reduction = 5;
  int whir_pow_bits = 16;
};

// ------------------------------------------------------------------ host time accounting
// Per-thread totals of the host work between device waits (profiling diagnostics: only
// counted while the thread's context profiles).
struct HostClock {
  bool on = false;
  double perm_ms = 0, alloc_ms = 0, launch_ms = 0, upload_ms = 0;
  long perms = 0, allocs = 0, launches = 0, uploads = 0;
  // host time between device waits, by proof phase (the phase current when the wait begins)
  std::string phase = "setup";
  double last_wait_end = 0;
  std::vector<std::pair<std::string, double>> busy;
  void add_busy(double ms) {
    for (auto& b : busy)
      if (b.first == phase) { b.second += ms; return; }
    busy.emplace_back(phase, ms);
  }
};
inline HostClock& host_clock() {
  thread_local HostClock c;
  return c;
}
inline double host_now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// ------------------------------------------------------------------ transcript
// DuplexChallenger<F, Poseidon16, 16, 8>: observations overwrite the rate part of the
// sponge once eight are buffered; samples pop from the end of the last squeeze.
// Poseidon2-16 on the host (host_perm.cpp): AVX-512 when the CPU has it, else scalar.
void host_p16_permute(uint32_t* s, const kb::P16Consts& c);
// n independent permutations of states laid out one after the other (W words each), sixteen at
// a time with AVX-512 when the CPU has it; the same map as kb::p2_permute<W>.
void host_p24_permute_many(uint32_t* states, size_t n, const kb::P24Consts& c);
void host_p16_permute_many(uint32_t* states, size_t n, const kb::P16Consts& c);

struct HostChallenger {
  const kb::P16Consts* perm = nullptr;
  uint32_t state[16] = {0};
  uint32_t in[8] = {0};
  int in_len = 0;
  uint32_t out[8] = {0};
  int out_len = 0;
  void duplex() {
    for (int i = 0; i < in_len; i++) state[i] = in[i];
    in_len = 0;
    HostClock& hc = host_clock();
    const double t0 = hc.on ? host_now_ms() : 0;
    host_p16_permute(state, *perm);
    if (hc.on) hc.perm_ms += host_now_ms() - t0, hc.perms++;
    for (int i = 0; i < 8; i++) out[i] = state[i];
    out_len = 8;
  }
  void observe(uint32_t x) {
    out_len = 0;
    in[in_len++] = x;
    if (in_len == 8) duplex();
  }
  uint32_t sample() {
    if (in_len || !out_len) duplex();
    return out[--out_len];
  }
  uint32_t sample_bits(int bits) { return kb::from_mont(sample()) & ((1u << bits) - 1); }
};

// Per-phase record of a transcript, for diffing one implementation against another: where
// each phase starts in proof_data, and every challenge, query batch and grinding witness with
// the proof offset at which it was drawn (values canonical).
struct TranscriptLog {
  struct Event {
    std::string kind;   // "phase", "challenge", "queries", "grinding"
    std::string phase;  // the phase it belongs to
    size_t offset = 0;  // words of proof_data before it
    std::vector<uint32_t> values;
  };
  std::vector<Event> events;
  std::string phase;
  void begin(const char* name, size_t offset) {
    phase = name;
    events.push_back({"phase", phase, offset, {}});
  }
  void add(const char* kind, size_t offset, const uint32_t* v, size_t n, bool mont) {
    Event e{kind, phase, offset, {}};
    for (size_t i = 0; i < n; i++) e.values.push_back(mont ? kb::from_mont(v[i]) : v[i]);
    events.push_back(std::move(e));
  }
  std::string json(size_t proof_len) const {
    std::string o = "{\"proof_len\": " + std::to_string(proof_len) + ", \"events\": [";
    for (size_t i = 0; i < events.size(); i++) {
      const Event& e = events[i];
      o += (i ? ", " : "") + std::string("{\"kind\": \"") + e.kind + "\", \"phase\": \"" + e.phase +
           "\", \"offset\": " + std::to_string(e.offset) + ", \"values\": [";
      for (size_t k = 0; k < e.values.size(); k++) o += (k ? ", " : "") + std::to_string(e.values[k]);
      o += "]}";
    }
    return o + "]}";
  }
};

struct Transcript {
  HostChallenger ch;
  std::vector<uint32_t> proof;  // Montgomery form
  TranscriptLog* log = nullptr;
  explicit Transcript(const kb::P16Consts* p) { ch.perm = p; }
  void add_base(const uint32_t* v, size_t n) {
    for (size_t i = 0; i < n; i++) { proof.push_back(v[i]); ch.observe(v[i]); }
  }
  void add_ext(const ef* v, size_t n) {
    for (size_t i = 0; i < n; i++) add_base(v[i].c, 8);
  }
  void hint(const uint32_t* v, size_t n) { proof.insert(proof.end(), v, v + n); }
  ef sample_ext() {
    ef e;
    for (int i = 0; i < 8; i++) e.c[i] = ch.sample();
    if (log) log->add("challenge", proof.size(), e.c, 8, true);
    return e;
  }
  void phase(const char* name) {
    if (log) log->begin(name, proof.size());
    host_clock_phase(name);
  }
  static void host_clock_phase(const char* name);
};

// ------------------------------------------------------------------ small polynomials
inline uint32_t fm(int64_t x) {  // Montgomery form of a small signed integer
  int64_t v = x % int64_t(kb::P);
  if (v < 0) v += kb::P;
  return kb::to_mont(uint32_t(v));
}
inline ef ef_scale(const ef& a, uint32_t f) { return kb::ef_mul_f(a, f); }

// Basis polynomials (coefficients, base field) of Lagrange interpolation on nodes 0..n-1.
inline std::vector<std::vector<uint32_t>> lagrange_basis(int n) {
  std::vector<std::vector<uint32_t>> basis(n);
  for (int i = 0; i < n; i++) {
    std::vector<uint32_t> p{kb::R_MOD_P};
    uint32_t denom = kb::R_MOD_P;
    for (int j = 0; j < n; j++) {
      if (j == i) continue;
      std::vector<uint32_t> q(p.size() + 1, 0);
      uint32_t negj = fm(-j);
      for (size_t a = 0; a < p.size(); a++) {
        q[a] = kb::add(q[a], kb::mul(p[a], negj));
        q[a + 1] = kb::add(q[a + 1], p[a]);
      }
      p.swap(q);
      denom = kb::mul(denom, fm(i - j));
    }
    uint32_t inv = kb::inv_m(denom);
    for (auto& c : p) c = kb::mul(c, inv);
    basis[i] = p;
  }
  return basis;
}
// The same bases, computed once per n and process.
const std::vector<std::vector<uint32_t>>& lagrange_basis_cached(int n);
inline std::vector<ef> interpolate(const std::vector<std::vector<uint32_t>>& basis, const std::vector<ef>& ys) {
  size_t n = ys.size();
  std::vector<ef> out(n, kb::ef_zero());
  for (size_t i = 0; i < n; i++)
    for (size_t k = 0; k < n; k++) out[k] = kb::ef_add(out[k], kb::ef_mul_f(ys[i], basis[i][k]));
  return out;
}
inline std::vector<ef> poly_mul(const std::vector<ef>& a, const std::vector<ef>& b) {
  std::vector<ef> r(a.size() + b.size() - 1, kb::ef_zero());
  for (size_t i = 0; i < a.size(); i++)
    for (size_t j = 0; j < b.size(); j++) r[i + j] = kb::ef_add(r[i + j], kb::ef_mul(a[i], b[j]));
  return r;
}
inline ef poly_eval(const std::vector<ef>& c, const ef& x) {
  ef r = kb::ef_zero();
  for (size_t i = c.size(); i-- > 0;) r = kb::ef_add(kb::ef_mul(r, x), c[i]);
  return r;
}
inline ef upoly_eval(const std::vector<uint32_t>& c, const ef& x) {
  ef r = kb::ef_zero();
  for (size_t i = c.size(); i-- > 0;) r = kb::ef_add_f(kb::ef_mul(r, x), c[i]);
  return r;
}
inline uint32_t upoly_eval_f(const std::vector<uint32_t>& c, uint32_t x) {
  uint32_t r = 0;
  for (size_t i = c.size(); i-- > 0;) r = kb::add(kb::mul(r, x), c[i]);
  return r;
}
// eq table over `pt` (x_1 = most significant bit)
inline std::vector<ef> eq_table_host(const std::vector<ef>& pt) {
  std::vector<ef> t{kb::ef_one()};
  for (const ef& r : pt) {
    std::vector<ef> n(t.size() * 2);
    ef om = kb::ef_sub(kb::ef_one(), r);
    for (size_t j = 0; j < t.size(); j++) {
      n[2 * j] = kb::ef_mul(t[j], om);
      n[2 * j + 1] = kb::ef_mul(t[j], r);
    }
    t.swap(n);
  }
  return t;
}
inline ef eq_eval(const std::vector<ef>& a, const std::vector<ef>& b) {
  ef r = kb::ef_one();
  for (size_t i = 0; i < a.size(); i++) {
    ef t = kb::ef_add(kb::ef_mul(a[i], b[i]), kb::ef_mul(kb::ef_sub(kb::ef_one(), a[i]), kb::ef_sub(kb::ef_one(), b[i])));
    r = kb::ef_mul(r, t);
  }
  return r;
}
inline std::vector<ef> pow_point(const ef& z, int m) {
  std::vector<ef> pt(m);
  ef cur = z;
  for (int i = 0; i < m; i++) { pt[i] = cur; cur = kb::ef_mul(cur, cur); }
  return pt;
}
// h(r) for h given by its values at 0, 1, 2
inline ef quad_eval(const ef h[3], const ef& r) {
  static const uint32_t inv2 = kb::inv_m(fm(2));
  ef rm1 = kb::ef_sub_f(r, fm(1)), rm2 = kb::ef_sub_f(r, fm(2));
  ef a = kb::ef_mul_f(kb::ef_mul(kb::ef_mul(h[0], rm1), rm2), inv2);
  ef b = kb::ef_mul(kb::ef_mul(h[1], r), rm2);
  ef c = kb::ef_mul_f(kb::ef_mul(kb::ef_mul(h[2], r), rm1), inv2);
  return kb::ef_add(kb::ef_sub(a, b), c);
}

inline int log2_up(size_t x) {
  int r = 0;
  while ((size_t(1) << r) < x) r++;
  return r;
}
// SumcheckGrinding::Auto (crates/sumcheck/src/lib.rs:21-31) with EF::bits() = 8 * 31.
inline int sumcheck_pow_bits(int security_bits, int degree) {
  int t = std::max(0, 248 - log2_up(size_t(degree) + 1));
  return std::max(0, security_bits - t);
}
inline int batching_pow_bits(int security_bits, int log_size) {  // crates/air/src/utils.rs:162-212
  return std::max(0, security_bits - std::max(0, 248 - log_size));
}

// ------------------------------------------------------------------ WHIR schedule
// Folding ConstantFromSecondRound(first, rest): commitments C_0..C_R, the first over all
// num_vars variables folded by `first`, the others folded by `rest`; the RS domain shrinks by
// 2^rs_reduction after C_0 and by 2 afterwards. Queries per opening follow the
// capacity-bound count ceil((security - pow) / rate_bits); the remaining gap to the security
// level is closed by grinding. One OOD sample per commitment meets 128 bits with the
// 248-bit extension field.
struct WhirRound {
  int num_vars, fold, log_inv_rate, log_domain, queries, pow_bits, ood;
  int log_leaves() const { return log_domain - fold; }
};
struct WhirSchedule {
  int num_vars = 0, num_rounds = 0, final_vars = 0, security_bits = 128, fold_pow_bits = 0;
  std::vector<WhirRound> c;
  static WhirSchedule build(int m0, const Settings& s) {
    WhirSchedule w;
    w.num_vars = m0;
    w.security_bits = s.security_bits;
    const int k0 = s.fold_first, k = s.fold_rest;
    if (m0 <= k0) throw std::invalid_argument("too few variables for the first folding");
    const int rest = m0 - k0;
    const int kMaxVarsSent = 6;
    if (rest < kMaxVarsSent) {
      w.num_rounds = 0;
      w.final_vars = rest;
    } else {
      w.num_rounds = (rest - kMaxVarsSent + k - 1) / k;
      w.final_vars = rest - w.num_rounds * k;
    }
    const int sec = std::max(0, s.security_bits - s.whir_pow_bits);
    int m = m0, ld = m0 + s.log_inv_rate;
    for (int j = 0; j <= w.num_rounds; j++) {
      WhirRound r;
      r.num_vars = m;
      r.fold = j == 0 ? k0 : k;
      r.log_domain = ld;
      r.log_inv_rate = ld - m;
      r.queries = (sec + r.log_inv_rate - 1) / r.log_inv_rate;
      r.pow_bits = std::max(0, s.security_bits - r.queries * r.log_inv_rate);
      r.ood = ood_samples(s.security_bits, m, r.log_inv_rate);
      if (r.log_leaves() > 24) throw std::invalid_argument("domain exceeds the two-adicity of KoalaBear");
      w.c.push_back(r);
      ld -= j == 0 ? s.rs_reduction : 1;
      m -= r.fold;
    }
    w.fold_pow_bits = std::max(0, s.security_bits - (248 - (m0 + s.log_inv_rate) - 1));
    return w;
  }
  static int ood_samples(int security, int m, int rate) {
    for (int s = 1; s < 64; s++) {
      double err = 2.0 * (m + rate) + double(m) * s;
      if (double(s) * 248 + 1.0 - err >= security) return s;
    }
    throw std::invalid_argument("no OOD sample count reaches the security level");
  }
  std::vector<uint32_t> domain_separator() const {  // canonical words, absorbed first
    std::vector<uint32_t> d{uint32_t(num_vars), uint32_t(num_rounds), uint32_t(final_vars), uint32_t(security_bits),
                            uint32_t(fold_pow_bits)};
    for (const auto& r : c)
      for (int x : {r.num_vars, r.fold, r.log_domain, r.queries, r.pow_bits, r.ood}) d.push_back(uint32_t(x));
    return d;
  }
};

// ------------------------------------------------------------------ workload generator
// rand 0.9 StdRng: ChaCha12 keyed by PCG32 expansion of a u64 seed (rand_core
// seed_from_u64), 64-bit block counter, words consumed in order.
struct StdRng {
  uint32_t key[8];
  uint64_t counter = 0;
  uint32_t buf[16];
  int idx = 16;
  explicit StdRng(uint64_t state) {
    const uint64_t MUL = 6364136223846793005ull, INC = 11634580456548416449ull;
    for (int i = 0; i < 8; i++) {
      state = state * MUL + INC;
      uint32_t xs = uint32_t(((state >> 18) ^ state) >> 27);
      uint32_t rot = uint32_t(state >> 59);
      key[i] = (xs >> rot) | (xs << ((32 - rot) & 31));
    }
  }
  static uint32_t rotl(uint32_t x, int k) { return (x << k) | (x >> (32 - k)); }
  void refill() {
    uint32_t s[16] = {0x61707865, 0x3320646e, 0x79622d32, 0x6b206574};
    for (int i = 0; i < 8; i++) s[4 + i] = key[i];
    s[12] = uint32_t(counter);
    s[13] = uint32_t(counter >> 32);
    s[14] = s[15] = 0;
    uint32_t x[16];
    for (int i = 0; i < 16; i++) x[i] = s[i];
    auto qr = [&](int a, int b, int c, int d) {
      x[a] += x[b]; x[d] ^= x[a]; x[d] = rotl(x[d], 16);
      x[c] += x[d]; x[b] ^= x[c]; x[b] = rotl(x[b], 12);
      x[a] += x[b]; x[d] ^= x[a]; x[d] = rotl(x[d], 8);
      x[c] += x[d]; x[b] ^= x[c]; x[b] = rotl(x[b], 7);
    };
    for (int r = 0; r < 12; r += 2) {
      qr(0, 4, 8, 12); qr(1, 5, 9, 13); qr(2, 6, 10, 14); qr(3, 7, 11, 15);
      qr(0, 5, 10, 15); qr(1, 6, 11, 12); qr(2, 7, 8, 13); qr(3, 4, 9, 14);
    }
    for (int i = 0; i < 16; i++) buf[i] = x[i] + s[i];
    counter++;
    idx = 0;
  }
  uint32_t next_u32() {
    if (idx == 16) refill();
    return buf[idx++];
  }
  // Plonky3 MontyField31 StandardUniform: a 31-bit word below p taken as a Montgomery
  // representative; returns the canonical value.
  uint32_t random_f() {
    for (;;) {
      uint32_t u = next_u32() >> 1;
      if (u < kb::P) return kb::from_mont(u);
    }
  }
};

constexpr int N_AIR_CONSTS = 2 * 4 * 16 + 20;
constexpr int N_P16_CONSTS = 8 * 16 + 20;
constexpr int N_P24_CONSTS = 8 * 24 + 23;
constexpr int N_CONSTS = N_AIR_CONSTS + N_P16_CONSTS + N_P24_CONSTS;

// Constants blob (canonical): AIR round constants (beginning, partial, ending), then
// Poseidon16 (initial, terminal, internal), then Poseidon24 (same order).
inline AirConsts air_consts_from(const uint32_t* c) {
  AirConsts a;
  int i = 0;
  for (int r = 0; r < 4; r++)
    for (int j = 0; j < 16; j++) a.begin[r][j] = kb::to_mont(c[i++]);
  for (int r = 0; r < 20; r++) a.partial[r] = kb::to_mont(c[i++]);
  for (int r = 0; r < 4; r++)
    for (int j = 0; j < 16; j++) a.end[r][j] = kb::to_mont(c[i++]);
  return a;
}
template <int W>
inline kb::P2Consts<W> perm_consts_from(const uint32_t* c) {
  kb::P2Consts<W> p;
  int i = 0;
  for (int k = 0; k < 4 * W; k++) p.ext_init[k] = kb::to_mont(c[i++]);
  for (int k = 0; k < 4 * W; k++) p.ext_term[k] = kb::to_mont(c[i++]);
  for (int k = 0; k < kb::P2Consts<W>::RP; k++) p.internal[k] = kb::to_mont(c[i++]);
  return p;
}


// Runs `work` on the calling thread and on up to T - 1 more host threads, then joins them.
// A thread that cannot be started (the process is at its thread limit) leaves the work to the
// threads already running; an exception thrown by `work` on any thread is rethrown here after
// every thread has been joined, so nothing terminates the process.
template <class Work>
void run_on_threads(size_t T, Work&& work) {
  std::exception_ptr first;
  std::mutex mu;
  auto guarded = [&] {
    try {
      work();
    } catch (...) {
      std::lock_guard<std::mutex> lk(mu);
      if (!first) first = std::current_exception();
    }
  };
  std::vector<std::thread> pool;
  try {
    for (size_t t = 1; t < T; t++) pool.emplace_back(guarded);
  } catch (const std::system_error&) {
  }
  guarded();
  for (auto& th : pool) th.join();
  if (first) std::rethrow_exception(first);
}

}  // namespace wl
