// CPU oracle for the Whirlaway Poseidon2-AIR prover path.
//
// TEST INFRASTRUCTURE ONLY. This is a plain, independent CPU restatement of the
// reference prover (crates/air, crates/sumcheck, crates/utils and the whir-p3 /
// Plonky3 pieces they call). Only the test-suite, the smoke check and the
// benchmark's CPU-baseline leg may load it; the product library never links it.
//
// Style is deliberately different from the product: field elements are kept in
// canonical form and multiplied with 64-bit `%`, the NTT is a textbook radix-2
// loop, Poseidon2 is written straight from the round structure. Agreement with
// the CUDA path is therefore evidence, not a tautology.
//
// Parity status: the reference's arithmetic lives in un-vendored crates
// (Plonky3 rev d0c4a36, whir-p3 rev 9caef91, rand 0.9.1 / rand_chacha 0.9.0) and
// the reference holds no golden vectors for this path, so byte identity with the
// Rust prover is UNPINNED. ChaCha (the StdRng core) is pinned against an
// independent ChaCha20 implementation; everything else is pinned by the
// self-consistency properties the tests check (verifier acceptance, sumcheck
// invariants, NTT/DFT agreement, field identities).
#pragma once
#include <array>
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace wlo {

constexpr uint32_t P = 0x7f000001u;  // KoalaBear: 2^31 - 2^24 + 1

struct F {
  uint32_t v = 0;
  F() = default;
  explicit F(uint64_t x) : v(uint32_t(x % P)) {}
  static F raw(uint32_t x) { F f; f.v = x; return f; }
  friend F operator+(F a, F b) { uint32_t s = a.v + b.v; return raw(s >= P ? s - P : s); }
  friend F operator-(F a, F b) { return raw(a.v >= b.v ? a.v - b.v : a.v + P - b.v); }
  friend F operator*(F a, F b) { return raw(uint32_t((uint64_t)a.v * b.v % P)); }
  F operator-() const { return raw(v ? P - v : 0); }
  F& operator+=(F o) { return *this = *this + o; }
  F& operator-=(F o) { return *this = *this - o; }
  F& operator*=(F o) { return *this = *this * o; }
  bool operator==(F o) const { return v == o.v; }
  bool operator!=(F o) const { return v != o.v; }
};
F fpow(F a, uint64_t e);
F finv(F a);
F two_adic_generator(int log_size);  // generator of the subgroup of order 2^log_size

// Degree-8 binomial extension F[X]/(X^8 - 3), coefficients lowest degree first.
constexpr uint32_t EXT_W = 3;
constexpr int EXT_D = 8;
struct EF {
  F c[8];
  EF() = default;
  explicit EF(F a) { c[0] = a; }
  static EF from_u32(uint32_t x) { return EF(F(x)); }
  friend EF operator+(const EF& a, const EF& b) { EF r; for (int i = 0; i < 8; i++) r.c[i] = a.c[i] + b.c[i]; return r; }
  friend EF operator-(const EF& a, const EF& b) { EF r; for (int i = 0; i < 8; i++) r.c[i] = a.c[i] - b.c[i]; return r; }
  friend EF operator*(const EF& a, F b) { EF r; for (int i = 0; i < 8; i++) r.c[i] = a.c[i] * b; return r; }
  friend EF operator*(F b, const EF& a) { return a * b; }
  friend EF operator+(const EF& a, F b) { EF r = a; r.c[0] += b; return r; }
  friend EF operator-(const EF& a, F b) { EF r = a; r.c[0] -= b; return r; }
  friend EF operator*(const EF& a, const EF& b);
  EF operator-() const { EF r; for (int i = 0; i < 8; i++) r.c[i] = -c[i]; return r; }
  EF& operator+=(const EF& o) { return *this = *this + o; }
  EF& operator-=(const EF& o) { return *this = *this - o; }
  EF& operator*=(const EF& o) { return *this = *this * o; }
  bool operator==(const EF& o) const { for (int i = 0; i < 8; i++) if (c[i] != o.c[i]) return false; return true; }
  bool operator!=(const EF& o) const { return !(*this == o); }
  bool is_zero() const { return *this == EF(); }
};
EF efinv(const EF& a);
inline EF ef_one() { return EF(F(1)); }
inline EF cube(const EF& x) { return x * x * x; }
inline F cube(F x) { return x * x * x; }

// ---------------------------------------------------------------- randomness
// rand 0.9 StdRng = ChaCha12, seeded from a u64 through PCG32 (rand_core).
struct StdRng {
  uint32_t key[8];
  uint64_t counter = 0;
  uint32_t buf[16];
  int idx = 16;
  explicit StdRng(uint64_t seed);
  uint32_t next_u32();
  F random_f();  // Plonky3 MontyField31 StandardUniform: rejection-sampled 31-bit Montgomery word
};
void chacha_block(const uint32_t key[8], uint64_t counter, uint64_t stream, int rounds, uint32_t out[16]);

// ---------------------------------------------------------------- Poseidon2
struct Poseidon2 {
  int width = 16, rounds_f = 8, rounds_p = 20;
  std::vector<F> ext_init;   // (rounds_f/2) * width
  std::vector<F> ext_term;   // (rounds_f/2) * width
  std::vector<F> internal;   // rounds_p
  std::vector<F> diag;       // internal matrix is J + diag
  static Poseidon2 from_rng(int width, StdRng& rng);
  void permute(F* state) const;
};
std::vector<F> internal_diag(int width);
void mds_light(F* s, int width);
template <class T> void mds_light_t(T* s, int width);
template <class T> void internal_layer_t(T* s, int width, const std::vector<F>& diag);

// PaddingFreeSponge<P24, 24, 16, 8> and TruncatedPermutation<P16, 2, 8, 16>.
using Digest = std::array<F, 8>;
Digest sponge_hash(const Poseidon2& p24, const F* in, size_t len);
Digest compress(const Poseidon2& p16, const Digest& l, const Digest& r);

// ---------------------------------------------------------------- transcript
// DuplexChallenger<F, P16, 16, 8> plus the proof_data buffer of ProverState.
struct Challenger {
  const Poseidon2* perm;
  F state[16];
  std::vector<F> in_buf, out_buf;
  explicit Challenger(const Poseidon2* p) : perm(p) {}
  void duplex();
  void observe(F x);
  F sample();
  uint32_t sample_bits(int bits);
  bool check_witness(int bits, F w) const;
};

struct Transcript {
  Challenger ch;
  std::vector<F> proof;
  size_t cursor = 0;  // verifier read cursor
  explicit Transcript(const Poseidon2* p16) : ch(p16) {}
  // prover side
  void add_base(const F* v, size_t n);
  void add_ext(const EF* v, size_t n);
  void hint(const F* v, size_t n);
  EF sample_ext();
  void grind(int bits);
  // verifier side; return false on a short proof
  bool next_base(F* v, size_t n);
  bool next_ext(EF* v, size_t n);
  bool next_hint(F* v, size_t n);
  bool check_grind(int bits);
};

// ---------------------------------------------------------------- polynomials
std::vector<EF> eval_eq(const std::vector<EF>& point);                 // x_1 = MSB
EF eq_poly(const std::vector<EF>& a, const std::vector<EF>& b);
EF mle_evaluate(const std::vector<EF>& evals, const std::vector<EF>& point);
std::vector<EF> poly_lagrange(const std::vector<std::pair<F, EF>>& pts);  // coefficients
std::vector<EF> poly_mul(const std::vector<EF>& a, const std::vector<EF>& b);
EF poly_eval(const std::vector<EF>& coeffs, const EF& x);
EF poly_eval_f(const std::vector<EF>& coeffs, F x);
std::vector<std::vector<F>> univariate_selectors(int skips);  // coefficients of L_i on {0..2^skips-1}
F upoly_eval(const std::vector<F>& c, F x);
EF upoly_eval(const std::vector<F>& c, const EF& x);
int log2_up(size_t x);

// ---------------------------------------------------------------- AIR
constexpr int P2_WIDTH = 16, HALF_FULL = 4, PARTIAL = 20;
constexpr int AIR_COLS = 1 + P2_WIDTH + HALF_FULL * P2_WIDTH + PARTIAL + HALF_FULL * P2_WIDTH;  // 165
constexpr int AIR_CONSTRAINTS = 2 * HALF_FULL * P2_WIDTH + PARTIAL;                           // 148
struct AirConstants {
  F begin[HALF_FULL][P2_WIDTH];
  F partial[PARTIAL];
  F end[HALF_FULL][P2_WIDTH];
  static AirConstants from_rng(StdRng& rng);
};
// Row-major trace row generation (one permutation per row) -> column-major trace.
void air_trace_row(const AirConstants& c, const F* input16, F* row);
EF air_eval_base(const AirConstants& c, const F* up, const std::vector<EF>& alphas);
EF air_eval_ext(const AirConstants& c, const EF* up, const std::vector<EF>& alphas);

// ---------------------------------------------------------------- AIRs in general
// What the AIR prover and verifier need of an AIR (crates/air/src/table.rs:15-60: width,
// constraint count, constraint degree; the constraints as p3-air's ConstraintFolder sees
// them): the batched value sum_i alphas[i] C_i over a point holding the up values of the W
// columns followed by their down values (crates/air/src/utils.rs:140-160).
struct AirSpec {
  virtual ~AirSpec() = default;
  virtual int columns() const = 0;
  // Preprocessed columns (crates/air/src/table.rs:19,59-70): the first preprocessed() of the
  // columns are fixed by the AIR (preprocessed_column(c): 2^log_n values); they take part in the
  // zerocheck but are not committed, and the verifier evaluates them itself.
  virtual int preprocessed() const { return 0; }
  virtual const F* preprocessed_column(int c, size_t N) const { return nullptr; }
  virtual int constraints() const = 0;
  virtual int degree() const = 0;
  virtual EF eval_base(const F* ud, const std::vector<EF>& alphas) const = 0;
  virtual EF eval_ext(const EF* ud, const std::vector<EF>& alphas) const = 0;
};
// The Poseidon2-KoalaBear width-16 AIR above (reads the up values only).
struct Poseidon2AirSpec : AirSpec {
  const AirConstants& c;
  explicit Poseidon2AirSpec(const AirConstants& k) : c(k) {}
  int columns() const override { return AIR_COLS; }
  int constraints() const override { return AIR_CONSTRAINTS; }
  int degree() const override { return 3; }
  EF eval_base(const F* ud, const std::vector<EF>& a) const override { return air_eval_base(c, ud, a); }
  EF eval_ext(const EF* ud, const std::vector<EF>& a) const override { return air_eval_ext(c, ud, a); }
};
// An AIR given as a constraint program: instruction i computes value v_i from
//   UP c / DOWN c (column c's up / down value), CONST j (consts[j]),
//   ADD / SUB / MUL a b (v_a op v_b, a and b < i), EMIT a (the next constraint is v_a; v_i = v_a).
// The constraints are the EMITs in program order.
enum AirOpCode { AIR_OP_UP = 0, AIR_OP_DOWN = 1, AIR_OP_CONST = 2, AIR_OP_ADD = 3, AIR_OP_SUB = 4, AIR_OP_MUL = 5,
                 AIR_OP_EMIT = 6 };
struct AirInstr {
  int op, a, b;
};
struct ProgramAirSpec : AirSpec {
  int W = 0, NC = 0, deg = 0, P = 0;
  std::vector<AirInstr> code;
  std::vector<F> consts;
  std::vector<F> pre;  // P columns of 2^log_n values
  int columns() const override { return W; }
  int preprocessed() const override { return P; }
  const F* preprocessed_column(int c, size_t N) const override {
    if (pre.size() != size_t(P) * N) throw std::runtime_error("AIR program: preprocessed columns of the wrong height");
    return pre.data() + size_t(c) * N;
  }
  int constraints() const override { return NC; }
  int degree() const override { return deg; }
  EF eval_base(const F* ud, const std::vector<EF>& a) const override;
  EF eval_ext(const EF* ud, const std::vector<EF>& a) const override;
  // Throws unless every operand refers to an earlier value, a column < W or a constant, and
  // the EMITs number NC.
  void check() const;
};

// ---------------------------------------------------------------- settings
struct Settings {
  int security_bits = 128;
  int log_inv_rate = 1;
  int fold_first = 7;
  int fold_rest = 4;
  int univariate_skips = 4;
  int rs_reduction = 5;
  int whir_pow_bits = 16;
};

struct WhirRound {   // one commitment C_j
  int num_vars;      // m_j
  int fold;          // k_j
  int log_inv_rate;  // rho_j
  int log_domain;    // m_j + rho_j
  int queries;       // STIR queries opened on C_j
  int pow_bits;      // grinding before those queries
  int ood;           // OOD samples taken right after committing C_j
};
struct WhirConfig {
  int num_vars = 0;
  int num_rounds = 0;       // commitments after the first
  int final_vars = 0;
  int security_bits = 128;
  int fold_pow_bits = 0;    // grinding inside the WHIR sumcheck rounds
  std::vector<WhirRound> c;  // num_rounds + 1 commitments
  static WhirConfig build(int num_vars, const Settings& s);
  std::vector<F> domain_separator() const;
};
int sumcheck_pow_bits(int security_bits, int degree);

// ---------------------------------------------------------------- WHIR
struct CommitData {
  int num_vars, fold, log_leaves, elem;  // elem = 1 (F) or 8 (EF)
  std::vector<F> leaves;                 // 2^log_leaves rows x (2^fold * elem)
  std::vector<std::vector<Digest>> tree; // tree[0] = leaf digests ... tree.back() = {root}
  size_t row_len() const { return size_t(elem) << fold; }
};
CommitData whir_encode_commit(const std::vector<F>& coeff_evals_flat, int num_vars, int fold, int log_domain, int elem,
                              const Poseidon2& p24, const Poseidon2& p16);
void mobius_inplace(std::vector<EF>& v);
void mobius_inplace_f(std::vector<F>& v);
std::vector<F> ntt_eval(const std::vector<F>& coeffs, int log_size);  // evaluate at w^r, r < 2^log_size
EF fold_leaf(const F* row, int fold, int elem, const std::vector<EF>& r);
std::vector<EF> pow_point(const EF& z, int num_vars);

struct Hashes {
  Poseidon2 p16, p24;
};

// ---------------------------------------------------------------- provers
struct ProveTimings { double commit = 0, zerocheck = 0, inner = 0, whir = 0; };
std::vector<F> prove_air(const Settings& s, const AirConstants& air, const Hashes& h, int log_n,
                         const std::vector<F>& witness_colmajor, ProveTimings* t = nullptr);
std::vector<F> prove_air_spec(const Settings& s, const AirSpec& air, const Hashes& h, int log_n,
                              const std::vector<F>& witness_colmajor, ProveTimings* t = nullptr);
enum VerifyStatus { V_OK = 0, V_INVALID_PCS_COMMITMENT = 1, V_INVALID_PCS_OPENING = 2, V_FS = 3,
                    V_SUMCHECK = 4, V_BOUNDARY = 5, V_SUM_MISMATCH = 6 };
int verify_air(const Settings& s, const AirConstants& air, const Hashes& h, int log_n, const std::vector<F>& proof);
int verify_air_spec(const Settings& s, const AirSpec& air, const Hashes& h, int log_n, const std::vector<F>& proof);

// Standalone zerocheck of eq(r,x) * (a*b - c) (a, b, c base-field multilinears).
std::vector<F> prove_abc(const Poseidon2& p16, int log_n, int skips, const std::vector<F>& a,
                         const std::vector<F>& b, const std::vector<F>& c);
int verify_abc(const Poseidon2& p16, int log_n, int skips, const std::vector<F>& proof,
               std::vector<EF>* final_point = nullptr, EF* final_value = nullptr);

}  // namespace wlo
