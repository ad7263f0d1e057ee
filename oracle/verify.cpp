// CPU oracle (test infrastructure): the verifier. Follows
//   crates/air/src/verify.rs:55-249      (AirTable::verify)
//   crates/sumcheck/src/verify.rs:23-113 (verify, verify_with_univariate_skip)
//   crates/air/src/utils.rs:12-138       (matrix_up_lde, matrix_down_lde, next_mle)
// and the WHIR verifier in whir.cpp. Error codes mirror AirVerifError.
#include <stdexcept>

#include "oracle.h"

namespace wlo {

bool whir_parse_commitment(const WhirConfig& cfg, Transcript& ts, Digest& root,
                           std::vector<std::pair<std::vector<EF>, EF>>& ood);
bool whir_verify(const WhirConfig& cfg, Transcript& ts, const Digest& root0,
                 const std::vector<std::pair<std::vector<EF>, EF>>& ood, const std::vector<EF>& point,
                 const EF& value, const Hashes& h);

struct ScClaim {
  EF sum;
  std::vector<EF> point;
  EF value;
};

// verify_core: returns 0, V_FS (short proof / bad grinding) or V_SUMCHECK
static int verify_core(Transcript& ts, const std::vector<int>& degs, const std::vector<int>& set_sizes, int security,
                       ScClaim& out) {
  EF target;
  for (size_t r = 0; r < degs.size(); r++) {
    std::vector<EF> coeffs(degs[r] + 1);
    if (!ts.next_ext(coeffs.data(), coeffs.size())) return V_FS;
    EF s;
    for (int x = 0; x < set_sizes[r]; x++) s += poly_eval_f(coeffs, F(x));
    if (r == 0) out.sum = s;
    else if (s != target) return V_SUMCHECK;
    EF ch = ts.sample_ext();
    if (!ts.check_grind(sumcheck_pow_bits(security, degs[r]))) return V_FS;
    target = poly_eval(coeffs, ch);
    out.point.push_back(ch);
  }
  out.value = target;
  return 0;
}

static EF matrix_up_lde(const std::vector<EF>& pt) {
  size_t n = pt.size() / 2;
  std::vector<EF> s1(pt.begin(), pt.begin() + n), s2(pt.begin() + n, pt.end());
  EF prod = ef_one();
  for (size_t i = 0; i + 1 < pt.size(); i++) prod = prod * pt[i];
  return eq_poly(s1, s2) + prod * (ef_one() - pt.back() * F(2));
}
static EF next_mle(const std::vector<EF>& pt) {
  size_t n = pt.size() / 2;
  const EF* x = pt.data();
  const EF* y = pt.data() + n;
  EF total;
  for (size_t k = 0; k < n; k++) {
    EF eq_hi = ef_one();
    for (size_t i = k + 1; i < n; i++)
      eq_hi = eq_hi * (x[n - 1 - i] * y[n - 1 - i] + (ef_one() - x[n - 1 - i]) * (ef_one() - y[n - 1 - i]));
    EF carry = (ef_one() - x[n - 1 - k]) * y[n - 1 - k];
    EF low = ef_one();
    for (size_t i = 0; i < k; i++) low = low * (x[n - 1 - i] * (ef_one() - y[n - 1 - i]));
    total += eq_hi * carry * low;
  }
  return total;
}
static EF matrix_down_lde(const std::vector<EF>& pt) {
  EF prod = ef_one();
  for (auto& x : pt) prod = prod * x;
  return next_mle(pt) + prod;
}

int verify_air(const Settings& s, const AirConstants& air, const Hashes& h, int log_n, const std::vector<F>& proof) {
  return verify_air_spec(s, Poseidon2AirSpec(air), h, log_n, proof);
}

int verify_air_spec(const Settings& s, const AirSpec& air, const Hashes& h, int log_n, const std::vector<F>& proof) {
  const int W = air.columns(), NC = air.constraints(), P = air.preprocessed(), Ww = W - P, n = log_n,
            k = s.univariate_skips;
  const int logW = log2_up(Ww);
  WhirConfig cfg = WhirConfig::build(n + logW, s);
  Transcript ts(&h.p16);
  ts.proof = proof;
  for (F x : cfg.domain_separator()) ts.ch.observe(x);
  Digest root;
  std::vector<std::pair<std::vector<EF>, EF>> ood;
  if (!whir_parse_commitment(cfg, ts, root, ood)) return V_INVALID_PCS_COMMITMENT;
  if (!ts.check_grind(std::max(0, s.security_bits - std::max(0, 31 * EXT_D - log2_up(NC))))) return V_FS;
  EF alpha = ts.sample_ext();
  if (!ts.check_grind(std::max(0, s.security_bits - std::max(0, 31 * EXT_D - n)))) return V_FS;
  std::vector<EF> zc(n - k + 1);
  for (auto& x : zc) x = ts.sample_ext();

  // verify_with_univariate_skip(degree = constraint_degree + 1)
  const int d1 = air.degree() + 1;
  std::vector<int> degs{d1 * ((1 << k) - 1)}, sets{1 << k};
  for (int i = 0; i < n - k; i++) { degs.push_back(d1); sets.push_back(2); }
  ScClaim outer;
  if (int e = verify_core(ts, degs, sets, s.security_bits, outer)) return e;
  if (!outer.sum.is_zero()) return V_SUM_MISMATCH;

  std::vector<EF> wup(Ww), wdown(Ww);
  if (!ts.next_ext(wup.data(), Ww) || !ts.next_ext(wdown.data(), Ww)) return V_FS;
  auto sel = univariate_selectors(k);
  std::vector<EF> outer_sel(1 << k), zc_sel(1 << k);
  for (int i = 0; i < (1 << k); i++) {
    outer_sel[i] = upoly_eval(sel[i], outer.point[0]);
    zc_sel[i] = upoly_eval(sel[i], zc[0]);
  }
  // the preprocessed columns' up / down versions folded over the skipped variables at the
  // outer challenge and evaluated at its tail (crates/air/src/verify.rs:119-135)
  std::vector<EF> global(2 * W);
  const size_t N = size_t(1) << n, S = N >> k;
  const std::vector<EF> otail(outer.point.begin() + 1, outer.point.end());
  for (int c = 0; c < P; c++) {
    const F* col = air.preprocessed_column(c, N);
    for (int half = 0; half < 2; half++) {
      std::vector<EF> f(S);
      for (size_t x = 0; x < S; x++) {
        EF acc;
        for (int j = 0; j < (1 << k); j++) {
          const size_t r = size_t(j) * S + x;
          const size_t src = half == 0 ? (r == N - 1 ? N - 2 : r) : (r == N - 1 ? r : r + 1);
          acc += outer_sel[j] * col[src];
        }
        f[x] = acc;
      }
      global[half * W + c] = mle_evaluate(f, otail);
    }
  }
  for (int c = 0; c < Ww; c++) { global[P + c] = wup[c]; global[W + P + c] = wdown[c]; }
  std::vector<EF> alphas(NC);
  alphas[0] = ef_one();
  for (int i = 1; i < NC; i++) alphas[i] = alphas[i - 1] * alpha;
  EF constraint_eval = air.eval_ext(global.data(), alphas);
  EF dot;
  for (int i = 0; i < (1 << k); i++) dot += zc_sel[i] * outer_sel[i];
  std::vector<EF> zc_tail(zc.begin() + 1, zc.end()), outer_tail(outer.point.begin() + 1, outer.point.end());
  if (dot * eq_poly(zc_tail, outer_tail) * constraint_eval != outer.value) return V_SUM_MISMATCH;

  if (!ts.check_grind(std::max(0, s.security_bits - std::max(0, 31 * EXT_D - log2_up(Ww))))) return V_FS;
  std::vector<EF> cbs(logW);
  for (auto& x : cbs) x = ts.sample_ext();
  EF alpha2 = ts.sample_ext();
  std::vector<EF> sub(size_t(1) << k);
  if (!ts.next_ext(sub.data(), sub.size())) return V_FS;
  std::vector<EF> eqc = eval_eq(cbs);
  EF lhs, su, sd;
  for (int i = 0; i < (1 << k); i++) lhs += sub[i] * outer_sel[i];
  for (int c = 0; c < Ww; c++) { su += wup[c] * eqc[c]; sd += wdown[c] * eqc[c]; }
  if (lhs != su + sd * alpha2) return V_SUM_MISMATCH;
  std::vector<EF> eps(k);
  for (auto& x : eps) x = ts.sample_ext();

  std::vector<int> d2(n, 2), s2(n, 2);
  ScClaim inner;
  if (int e = verify_core(ts, d2, s2, s.security_bits, inner)) return e;
  if (inner.sum != mle_evaluate(sub, eps)) return V_SUM_MISMATCH;

  std::vector<EF> lde_pt = eps;
  lde_pt.insert(lde_pt.end(), outer_tail.begin(), outer_tail.end());
  lde_pt.insert(lde_pt.end(), inner.point.begin(), inner.point.end());
  EF up = matrix_up_lde(lde_pt), down = matrix_down_lde(lde_pt);
  EF denom = up + alpha2 * down;
  if (denom.is_zero()) return V_SUM_MISMATCH;
  EF expected = inner.value * efinv(denom);
  std::vector<EF> final_point = cbs;
  final_point.insert(final_point.end(), inner.point.begin(), inner.point.end());
  if (!whir_verify(cfg, ts, root, ood, final_point, expected, h)) return V_INVALID_PCS_OPENING;
  if (ts.cursor != ts.proof.size()) return V_FS;
  return V_OK;
}

int verify_abc(const Poseidon2& p16, int log_n, int skips, const std::vector<F>& proof, std::vector<EF>* fp, EF* fv) {
  Transcript ts(&p16);
  ts.proof = proof;
  std::vector<EF> r(log_n + 1 - skips);
  for (auto& x : r) x = ts.sample_ext();
  std::vector<int> degs{3 * ((1 << skips) - 1)}, sets{1 << skips};
  for (int i = 0; i < log_n - skips; i++) { degs.push_back(3); sets.push_back(2); }
  ScClaim cl;
  if (int e = verify_core(ts, degs, sets, 128, cl)) return e;
  if (!cl.sum.is_zero()) return V_SUM_MISMATCH;
  EF abc[3];
  if (!ts.next_ext(abc, 3)) return V_FS;
  auto sel = univariate_selectors(skips);
  EF dot;
  for (int i = 0; i < (1 << skips); i++) dot += upoly_eval(sel[i], r[0]) * upoly_eval(sel[i], cl.point[0]);
  std::vector<EF> rt(r.begin() + 1, r.end()), ct(cl.point.begin() + 1, cl.point.end());
  if (dot * eq_poly(rt, ct) * (abc[0] * abc[1] - abc[2]) != cl.value) return V_SUM_MISMATCH;
  if (ts.cursor != ts.proof.size()) return V_FS;
  if (fp) *fp = cl.point;
  if (fv) *fv = cl.value;
  return V_OK;
}

}  // namespace wlo
