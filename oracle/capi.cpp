// CPU oracle (test infrastructure): flat C entry points for the test-suite and
// the benchmark's CPU-baseline leg. All field values are canonical u32.
#include <omp.h>

#include <chrono>
#include <cstring>
#include <exception>
#include <stdexcept>

#include "oracle.h"

using namespace wlo;

namespace {
Settings settings_from(const int32_t* s) {
  Settings st;
  if (s) {
    st.security_bits = s[0];
    st.log_inv_rate = s[1];
    st.fold_first = s[2];
    st.fold_rest = s[3];
    st.univariate_skips = s[4];
    st.rs_reduction = s[5];
    st.whir_pow_bits = s[6];
  }
  return st;
}
AirConstants air_from(const uint32_t* c) {
  AirConstants a;
  int i = 0;
  for (int r = 0; r < HALF_FULL; r++)
    for (int j = 0; j < 16; j++) a.begin[r][j] = F(c[i++]);
  for (int r = 0; r < PARTIAL; r++) a.partial[r] = F(c[i++]);
  for (int r = 0; r < HALF_FULL; r++)
    for (int j = 0; j < 16; j++) a.end[r][j] = F(c[i++]);
  return a;
}
Poseidon2 perm_from(int width, const uint32_t* c) {
  Poseidon2 p;
  p.width = width;
  p.rounds_f = 8;
  p.rounds_p = width == 16 ? 20 : 23;
  int i = 0;
  for (int k = 0; k < 4 * width; k++) p.ext_init.push_back(F(c[i++]));
  for (int k = 0; k < 4 * width; k++) p.ext_term.push_back(F(c[i++]));
  for (int k = 0; k < p.rounds_p; k++) p.internal.push_back(F(c[i++]));
  p.diag = internal_diag(width);
  return p;
}
// constants blob: AIR (148) | P16 (148) | P24 (215)
constexpr int AIR_NC = 2 * 4 * 16 + 20, P16_NC = 8 * 16 + 20, P24_NC = 8 * 24 + 23;
// A constraint program from flat arrays: ops holds (op, a, b) per instruction.
// The first n_pre columns are preprocessed: pre holds them (n_pre columns of 2^log_n values).
ProgramAirSpec program_from(int W, int n_constraints, int degree, int n_ops, const int32_t* ops, int n_consts,
                            const uint32_t* consts, int n_pre, const uint32_t* pre, int log_n) {
  ProgramAirSpec p;
  p.W = W;
  p.NC = n_constraints;
  p.deg = degree;
  p.P = n_pre;
  for (int i = 0; i < n_ops; i++) p.code.push_back({ops[3 * i], ops[3 * i + 1], ops[3 * i + 2]});
  for (int i = 0; i < n_consts; i++) p.consts.push_back(F(consts[i]));
  if (n_pre < 0 || n_pre >= W) throw std::runtime_error("AIR program: bad preprocessed column count");
  for (size_t i = 0; i < (size_t(n_pre) << log_n); i++) p.pre.push_back(F(pre[i]));
  p.check();
  return p;
}
}  // namespace

extern "C" {

int wlo_constants_size() { return AIR_NC + P16_NC + P24_NC; }

// Workload of src/examples/poseidon2.rs:104-151: one StdRng stream gives the AIR
// round constants, then the 16*2^log_n inputs (row-major), then the Poseidon16 and
// Poseidon24 constants. `input_seed` < 0 keeps that single stream; otherwise the
// constants come from the seed-0 stream with the inputs skipped and the inputs
// come from StdRng::seed_from_u64(input_seed).
int wlo_workload(int log_n, int64_t input_seed, uint32_t* constants, uint32_t* inputs) {
  try {
    StdRng rng(0);
    size_t n = size_t(16) << log_n;
    int ci = 0;
    for (int i = 0; i < AIR_NC; i++) constants[ci++] = rng.random_f().v;
    if (input_seed < 0) {
      for (size_t i = 0; i < n; i++) inputs[i] = rng.random_f().v;
    } else {
      StdRng r2((uint64_t)input_seed);
      for (size_t i = 0; i < n; i++) inputs[i] = r2.random_f().v;
    }
    for (int i = 0; i < P16_NC + P24_NC; i++) constants[ci++] = rng.random_f().v;
    return 0;
  } catch (...) {
    return -1;
  }
}

int wlo_trace(int log_n, const uint32_t* constants, const uint32_t* inputs, uint32_t* witness_colmajor) {
  AirConstants a = air_from(constants);
  size_t N = size_t(1) << log_n;
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < (int64_t)N; r++) {
    F in[16], row[AIR_COLS];
    for (int i = 0; i < 16; i++) in[i] = F(inputs[r * 16 + i]);
    air_trace_row(a, in, row);
    for (int c = 0; c < AIR_COLS; c++) witness_colmajor[size_t(c) * N + r] = row[c].v;
  }
  return 0;
}

int wlo_air_cols() { return AIR_COLS; }

int wlo_prove(const int32_t* settings, const uint32_t* constants, int log_n, const uint32_t* witness, uint32_t* proof,
              size_t* proof_len, double* timings) {
  try {
    Settings s = settings_from(settings);
    AirConstants a = air_from(constants);
    Hashes h{perm_from(16, constants + AIR_NC), perm_from(24, constants + AIR_NC + P16_NC)};
    size_t N = size_t(1) << log_n;
    std::vector<F> w(size_t(AIR_COLS) * N);
    for (size_t i = 0; i < w.size(); i++) w[i] = F::raw(witness[i]);
    ProveTimings t;
    std::vector<F> pr = prove_air(s, a, h, log_n, w, &t);
    if (timings) { timings[0] = t.commit; timings[1] = t.zerocheck; timings[2] = t.inner; timings[3] = t.whir; }
    if (*proof_len < pr.size()) { *proof_len = pr.size(); return -2; }
    for (size_t i = 0; i < pr.size(); i++) proof[i] = pr[i].v;
    *proof_len = pr.size();
    return 0;
  } catch (const std::exception&) {
    return -1;
  }
}

int wlo_verify(const int32_t* settings, const uint32_t* constants, int log_n, const uint32_t* proof, size_t proof_len) {
  try {
    Settings s = settings_from(settings);
    AirConstants a = air_from(constants);
    Hashes h{perm_from(16, constants + AIR_NC), perm_from(24, constants + AIR_NC + P16_NC)};
    std::vector<F> pr(proof_len);
    for (size_t i = 0; i < proof_len; i++) pr[i] = F::raw(proof[i] % P);
    return verify_air(s, a, h, log_n, pr);
  } catch (const std::exception&) {
    return 100;
  }
}

// An AIR given as a constraint program (hash_consts: P16 (148) | P24 (215)); its first n_pre
// columns are preprocessed (pre: n_pre columns of 2^log_n values); witness: the other W - n_pre
// columns of 2^log_n values, column-major.
int wlo_prove_program(const int32_t* settings, const uint32_t* hash_consts, int W, int n_constraints, int degree,
                      int n_ops, const int32_t* ops, int n_consts, const uint32_t* consts, int n_pre,
                      const uint32_t* pre, int log_n, const uint32_t* witness, uint32_t* proof, size_t* proof_len) {
  try {
    Settings s = settings_from(settings);
    ProgramAirSpec air = program_from(W, n_constraints, degree, n_ops, ops, n_consts, consts, n_pre, pre, log_n);
    Hashes h{perm_from(16, hash_consts), perm_from(24, hash_consts + P16_NC)};
    size_t N = size_t(1) << log_n;
    std::vector<F> w(size_t(W - n_pre) * N);
    for (size_t i = 0; i < w.size(); i++) w[i] = F::raw(witness[i]);
    std::vector<F> pr = prove_air_spec(s, air, h, log_n, w);
    if (*proof_len < pr.size()) { *proof_len = pr.size(); return -2; }
    for (size_t i = 0; i < pr.size(); i++) proof[i] = pr[i].v;
    *proof_len = pr.size();
    return 0;
  } catch (const std::exception&) {
    return -1;
  }
}

int wlo_verify_program(const int32_t* settings, const uint32_t* hash_consts, int W, int n_constraints, int degree,
                       int n_ops, const int32_t* ops, int n_consts, const uint32_t* consts, int n_pre,
                       const uint32_t* pre, int log_n, const uint32_t* proof, size_t proof_len) {
  try {
    Settings s = settings_from(settings);
    ProgramAirSpec air = program_from(W, n_constraints, degree, n_ops, ops, n_consts, consts, n_pre, pre, log_n);
    Hashes h{perm_from(16, hash_consts), perm_from(24, hash_consts + P16_NC)};
    std::vector<F> pr(proof_len);
    for (size_t i = 0; i < proof_len; i++) pr[i] = F::raw(proof[i] % P);
    return verify_air_spec(s, air, h, log_n, pr);
  } catch (const std::exception&) {
    return 100;
  }
}

int wlo_prove_abc(const uint32_t* p16c, int log_n, int skips, const uint32_t* a, const uint32_t* b, const uint32_t* c,
                  uint32_t* proof, size_t* proof_len) {
  try {
    Poseidon2 p16 = perm_from(16, p16c);
    size_t N = size_t(1) << log_n;
    std::vector<F> va(N), vb(N), vc(N);
    for (size_t i = 0; i < N; i++) { va[i] = F::raw(a[i]); vb[i] = F::raw(b[i]); vc[i] = F::raw(c[i]); }
    std::vector<F> pr = prove_abc(p16, log_n, skips, va, vb, vc);
    if (*proof_len < pr.size()) { *proof_len = pr.size(); return -2; }
    for (size_t i = 0; i < pr.size(); i++) proof[i] = pr[i].v;
    *proof_len = pr.size();
    return 0;
  } catch (const std::exception&) {
    return -1;
  }
}

int wlo_verify_abc(const uint32_t* p16c, int log_n, int skips, const uint32_t* proof, size_t proof_len) {
  try {
    Poseidon2 p16 = perm_from(16, p16c);
    std::vector<F> pr(proof_len);
    for (size_t i = 0; i < proof_len; i++) pr[i] = F::raw(proof[i] % P);
    return verify_abc(p16, log_n, skips, pr);
  } catch (const std::exception&) {
    return 100;
  }
}

// --- primitives for known-answer and self-consistency tests
void wlo_chacha_block(const uint32_t* key, uint64_t counter, int rounds, uint32_t* out) {
  chacha_block(key, counter, 0, rounds, out);
}
void wlo_stdrng_u32(uint64_t seed, uint32_t* out, size_t n) {
  StdRng r(seed);
  for (size_t i = 0; i < n; i++) out[i] = r.next_u32();
}
void wlo_poseidon2(int width, const uint32_t* consts, uint32_t* state) {
  Poseidon2 p = perm_from(width, consts);
  F s[24];
  for (int i = 0; i < width; i++) s[i] = F(state[i]);
  p.permute(s);
  for (int i = 0; i < width; i++) state[i] = s[i].v;
}
void wlo_ef_mul(const uint32_t* a, const uint32_t* b, uint32_t* out) {
  EF x, y;
  for (int i = 0; i < 8; i++) { x.c[i] = F(a[i]); y.c[i] = F(b[i]); }
  EF z = x * y;
  for (int i = 0; i < 8; i++) out[i] = z.c[i].v;
}
void wlo_ef_inv(const uint32_t* a, uint32_t* out) {
  EF x;
  for (int i = 0; i < 8; i++) x.c[i] = F(a[i]);
  EF z = efinv(x);
  for (int i = 0; i < 8; i++) out[i] = z.c[i].v;
}
void wlo_ntt(const uint32_t* coeffs, size_t n_coeffs, int log_size, uint32_t* out) {
  std::vector<F> c(n_coeffs);
  for (size_t i = 0; i < n_coeffs; i++) c[i] = F(coeffs[i]);
  auto e = ntt_eval(c, log_size);
  for (size_t i = 0; i < e.size(); i++) out[i] = e[i].v;
}
int wlo_whir_config(int num_vars, const int32_t* settings, int32_t* out, int max_rounds) {
  try {
    WhirConfig cfg = WhirConfig::build(num_vars, settings_from(settings));
    if ((int)cfg.c.size() > max_rounds) return -2;
    out[0] = cfg.num_rounds;
    out[1] = cfg.final_vars;
    out[2] = cfg.fold_pow_bits;
    for (size_t j = 0; j < cfg.c.size(); j++) {
      const WhirRound& r = cfg.c[j];
      int32_t* o = out + 3 + 7 * j;
      o[0] = r.num_vars; o[1] = r.fold; o[2] = r.log_inv_rate; o[3] = r.log_domain;
      o[4] = r.queries; o[5] = r.pow_bits; o[6] = r.ood;
    }
    return 0;
  } catch (const std::exception&) {
    return -1;
  }
}
void wlo_set_threads(int n) { omp_set_num_threads(n); }
int wlo_max_threads() { return omp_get_max_threads(); }

}  // extern "C"
