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

}  // namespace wlo
