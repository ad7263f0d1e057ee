// CPU oracle (test infrastructure): the Poseidon2-KoalaBear width-16 AIR.
//
// Restates p3-poseidon2-air (Plonky3 rev d0c4a36, not vendored) as configured in
// src/examples/poseidon2.rs:21-36 of the reference: S-box x^3, no S-box registers,
// 4 + 4 full rounds, 20 partial rounds. Column layout (165 columns):
//   [export, inputs(16), 4 x full-round post(16), 20 x partial post_sbox(1), 4 x full-round post(16)]
// Constraint order: one per full-round output (16 per round) and one per partial
// round, in permutation order: 148 constraints, all of degree 3. The AIR reads the
// local row only (no transition constraints), so the "down" half of the zerocheck
// point is not used by the constraint polynomial.
#include <stdexcept>

#include "oracle.h"

namespace wlo {

// RoundConstants::from_rng: beginning rounds, partial rounds, ending rounds.
AirConstants AirConstants::from_rng(StdRng& rng) {
  AirConstants c;
  for (int r = 0; r < HALF_FULL; r++)
    for (int i = 0; i < P2_WIDTH; i++) c.begin[r][i] = rng.random_f();
  for (int r = 0; r < PARTIAL; r++) c.partial[r] = rng.random_f();
  for (int r = 0; r < HALF_FULL; r++)
    for (int i = 0; i < P2_WIDTH; i++) c.end[r][i] = rng.random_f();
  return c;
}

void air_trace_row(const AirConstants& c, const F* input, F* row) {
  static const std::vector<F> diag = internal_diag(16);
  F s[16];
  row[0] = F(1);  // export flag
  for (int i = 0; i < 16; i++) { s[i] = input[i]; row[1 + i] = input[i]; }
  int col = 17;
  mds_light(s, 16);
  for (int r = 0; r < HALF_FULL; r++) {
    for (int i = 0; i < 16; i++) s[i] = cube(s[i] + c.begin[r][i]);
    mds_light(s, 16);
    for (int i = 0; i < 16; i++) row[col++] = s[i];
  }
  for (int r = 0; r < PARTIAL; r++) {
    s[0] = cube(s[0] + c.partial[r]);
    row[col++] = s[0];
    internal_layer_t<F>(s, 16, diag);
  }
  for (int r = 0; r < HALF_FULL; r++) {
    for (int i = 0; i < 16; i++) s[i] = cube(s[i] + c.end[r][i]);
    mds_light(s, 16);
    for (int i = 0; i < 16; i++) row[col++] = s[i];
  }
}

// Sum_i alpha^i * h_i(up), the ConstraintFolder accumulator.
template <class T>
static EF air_eval_t(const AirConstants& c, const T* up, const std::vector<EF>& alphas) {
  static const std::vector<F> diag = internal_diag(16);
  T s[16];
  for (int i = 0; i < 16; i++) s[i] = up[1 + i];
  int col = 17, ci = 0;
  EF acc;
  mds_light_t<T>(s, 16);
  for (int r = 0; r < HALF_FULL; r++) {
    for (int i = 0; i < 16; i++) s[i] = cube(s[i] + c.begin[r][i]);
    mds_light_t<T>(s, 16);
    for (int i = 0; i < 16; i++) {
      acc += alphas[ci++] * (s[i] - up[col]);
      s[i] = up[col++];
    }
  }
  for (int r = 0; r < PARTIAL; r++) {
    s[0] = cube(s[0] + c.partial[r]);
    acc += alphas[ci++] * (s[0] - up[col]);
    s[0] = up[col++];
    internal_layer_t<T>(s, 16, diag);
  }
  for (int r = 0; r < HALF_FULL; r++) {
    for (int i = 0; i < 16; i++) s[i] = cube(s[i] + c.end[r][i]);
    mds_light_t<T>(s, 16);
    for (int i = 0; i < 16; i++) {
      acc += alphas[ci++] * (s[i] - up[col]);
      s[i] = up[col++];
    }
  }
  return acc;
}

EF air_eval_base(const AirConstants& c, const F* up, const std::vector<EF>& alphas) {
  return air_eval_t<F>(c, up, alphas);
}
EF air_eval_ext(const AirConstants& c, const EF* up, const std::vector<EF>& alphas) {
  return air_eval_t<EF>(c, up, alphas);
}

// ---------------------------------------------------------------- constraint programs
template <class T>
static EF program_eval_t(const ProgramAirSpec& p, const T* ud, const std::vector<EF>& alphas) {
  std::vector<T> v(p.code.size());
  EF acc;
  int ci = 0;
  for (size_t i = 0; i < p.code.size(); i++) {
    const AirInstr& in = p.code[i];
    switch (in.op) {
      case AIR_OP_UP: v[i] = ud[in.a]; break;
      case AIR_OP_DOWN: v[i] = ud[p.W + in.a]; break;
      case AIR_OP_CONST: v[i] = T(p.consts[in.a]); break;
      case AIR_OP_ADD: v[i] = v[in.a] + v[in.b]; break;
      case AIR_OP_SUB: v[i] = v[in.a] - v[in.b]; break;
      case AIR_OP_MUL: v[i] = v[in.a] * v[in.b]; break;
      default:  // AIR_OP_EMIT
        acc += alphas[ci++] * v[in.a];
        v[i] = v[in.a];
        break;
    }
  }
  return acc;
}
EF ProgramAirSpec::eval_base(const F* ud, const std::vector<EF>& a) const { return program_eval_t<F>(*this, ud, a); }
EF ProgramAirSpec::eval_ext(const EF* ud, const std::vector<EF>& a) const { return program_eval_t<EF>(*this, ud, a); }
void ProgramAirSpec::check() const {
  if (W < 1 || NC < 1 || deg < 1 || deg > 3) throw std::runtime_error("AIR program: bad width, count or degree");
  int emits = 0;
  for (size_t i = 0; i < code.size(); i++) {
    const AirInstr& in = code[i];
    const bool two = in.op == AIR_OP_ADD || in.op == AIR_OP_SUB || in.op == AIR_OP_MUL;
    if (in.op == AIR_OP_UP || in.op == AIR_OP_DOWN) {
      if (in.a < 0 || in.a >= W) throw std::runtime_error("AIR program: column out of range");
    } else if (in.op == AIR_OP_CONST) {
      if (in.a < 0 || in.a >= (int)consts.size()) throw std::runtime_error("AIR program: constant out of range");
    } else if (two || in.op == AIR_OP_EMIT) {
      if (in.a < 0 || in.a >= (int)i || (two && (in.b < 0 || in.b >= (int)i)))
        throw std::runtime_error("AIR program: operand is not an earlier value");
      emits += in.op == AIR_OP_EMIT;
    } else {
      throw std::runtime_error("AIR program: unknown instruction");
    }
  }
  if (emits != NC) throw std::runtime_error("AIR program: constraint count mismatch");
}

}  // namespace wlo
