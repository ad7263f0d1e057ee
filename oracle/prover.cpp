// CPU oracle (test infrastructure): sumcheck prover with univariate skip and the
// AIR prover. Follows, step for step:
//   crates/sumcheck/src/prove.rs:22-93   (prove)
//   crates/sumcheck/src/prove.rs:97-254  (sc_round)
//   crates/sumcheck/src/prove.rs:256-335 (compute_over_hypercube)
//   crates/utils/src/multilinear.rs      (folds, linear combination, packing)
//   crates/air/src/prove.rs:49-226       (AirTable::prove)
//   crates/air/src/uni_skip_utils.rs     (matrix_up_folded / matrix_down_folded)
// Round polynomials are always sent with exactly degree+1 coefficients (the
// verifier reads that many), padding with zeros if the top coefficients vanish.
#include <omp.h>

#include <chrono>
#include <functional>
#include <stdexcept>

#include "oracle.h"

namespace wlo {

CommitData whir_commit_base(const WhirConfig& cfg, const std::vector<F>& evals, Transcript& ts, const Hashes& h,
                            std::vector<std::pair<std::vector<EF>, EF>>& ood);
void whir_prove(const WhirConfig& cfg, Transcript& ts, const std::vector<F>& evals, const CommitData& cd0,
                const std::vector<std::pair<std::vector<EF>, EF>>& ood, const std::vector<EF>& point, const EF& value,
                const Hashes& h);

struct Computation {
  virtual ~Computation() = default;
  virtual EF eval_f(const F* pt) const = 0;
  virtual EF eval_e(const EF* pt) const = 0;
};

template <class NF> static EF comp_eval(const Computation& c, const NF* pt);
template <> EF comp_eval<F>(const Computation& c, const F* pt) { return c.eval_f(pt); }
template <> EF comp_eval<EF>(const Computation& c, const EF* pt) { return c.eval_e(pt); }

template <class NF> static EF to_ef(const NF& x);
template <> EF to_ef<F>(const F& x) { return EF(x); }
template <> EF to_ef<EF>(const EF& x) { return x; }

using Cols = std::vector<std::vector<EF>>;

// compute_over_hypercube: sum_x comp(point(x)) * eq(x)
template <class NF>
static EF over_hypercube(const std::vector<std::vector<NF>>& pols, const Computation& comp, const std::vector<EF>* eq) {
  size_t n = pols[0].size(), w = pols.size();
  EF total;
#pragma omp parallel
  {
    EF acc;
    std::vector<NF> pt(w);
#pragma omp for schedule(static) nowait
    for (int64_t x = 0; x < (int64_t)n; x++) {
      for (size_t c = 0; c < w; c++) pt[c] = pols[c][x];
      EF r = comp_eval<NF>(comp, pt.data());
      acc += eq ? r * (*eq)[x] : r;
    }
#pragma omp critical
    total += acc;
  }
  return total;
}

template <class NF>
static std::vector<std::vector<NF>> fold_small(const std::vector<std::vector<NF>>& m, const std::vector<F>& s) {
  std::vector<std::vector<NF>> out(m.size());
#pragma omp parallel for schedule(dynamic)
  for (int64_t c = 0; c < (int64_t)m.size(); c++) {
    size_t ns = m[c].size() / s.size();
    out[c].resize(ns);
    for (size_t i = 0; i < ns; i++) {
      NF acc{};
      for (size_t j = 0; j < s.size(); j++) acc = acc + m[c][i + j * ns] * s[j];
      out[c][i] = acc;
    }
  }
  return out;
}

template <class NF>
static Cols fold_large(const std::vector<std::vector<NF>>& m, const std::vector<EF>& s) {
  Cols out(m.size());
#pragma omp parallel for schedule(dynamic)
  for (int64_t c = 0; c < (int64_t)m.size(); c++) {
    size_t ns = m[c].size() / s.size();
    out[c].resize(ns);
    for (size_t i = 0; i < ns; i++) {
      EF acc;
      for (size_t j = 0; j < s.size(); j++) acc += s[j] * to_ef<NF>(m[c][i + j * ns]);
      out[c][i] = acc;
    }
  }
  return out;
}

struct ScState {
  EF sum;
  bool has_mmf = false;
  EF mmf;
  std::vector<EF> challenges;
};

template <class NF>
static Cols sc_round(int skips, const std::vector<std::vector<NF>>& mls, const Computation& comp,
                     const std::vector<EF>* eq_factor, bool is_zerocheck, Transcript& ts, int comp_degree,
                     int security_bits, int round, ScState& st) {
  std::vector<EF> eq_mle;
  if (eq_factor) eq_mle = eval_eq(std::vector<EF>(eq_factor->begin() + 1 + round, eq_factor->end()));
  std::vector<std::vector<F>> sel;
  if (skips != 1) sel = univariate_selectors(skips);
  const int n_sk = 1 << skips;
  std::vector<std::pair<F, EF>> p_evals;
  int start = 0;
  if (is_zerocheck) {
    for (int i = 0; i < n_sk; i++) p_evals.push_back({F(i), EF()});
    start = n_sk;
  }
  for (int z = start; z <= comp_degree * (n_sk - 1); z++) {
    EF sum_z;
    if (z == n_sk - 1) {
      if (eq_factor) {
        const EF& r = (*eq_factor)[round];
        if (skips == 1) {
          sum_z = (st.sum - p_evals[0].second * (ef_one() - r)) * efinv(r);
        } else {
          EF acc;
          for (int i = 0; i < n_sk - 1; i++) acc += p_evals[i].second * upoly_eval(sel[i], r);
          sum_z = (st.sum - acc) * efinv(upoly_eval(sel[n_sk - 1], r));
        }
      } else {
        EF acc;
        for (auto& pe : p_evals) acc += pe.second;
        sum_z = st.sum - acc;
      }
    } else {
      std::vector<std::vector<NF>> folded;
      if (skips == 1 && z == 0) {
        folded.resize(mls.size());
        for (size_t c = 0; c < mls.size(); c++)
          folded[c].assign(mls[c].begin(), mls[c].begin() + mls[c].size() / 2);
      } else {
        std::vector<F> s;
        if (skips == 1) s = {F(1) - F(z), F(z)};
        else for (int i = 0; i < n_sk; i++) s.push_back(upoly_eval(sel[i], F(z)));
        folded = fold_small<NF>(mls, s);
      }
      sum_z = over_hypercube<NF>(folded, comp, eq_factor ? &eq_mle : nullptr);
      if (st.has_mmf) sum_z = sum_z * st.mmf;
    }
    p_evals.push_back({F(z), sum_z});
  }
  std::vector<EF> p = poly_lagrange(p_evals);
  if (eq_factor) {
    const EF& r = (*eq_factor)[round];
    if (skips == 1) {
      p = poly_mul(p, {ef_one() - r, r + r - ef_one()});
    } else {
      std::vector<std::pair<F, EF>> pts;
      for (int i = 0; i < n_sk; i++) pts.push_back({F(i), upoly_eval(sel[i], r)});
      p = poly_mul(p, poly_lagrange(pts));
    }
  }
  int deg = (comp_degree + (eq_factor ? 1 : 0)) * (n_sk - 1);
  p.resize(deg + 1);
  ts.add_ext(p.data(), p.size());
  EF ch = ts.sample_ext();
  st.challenges.push_back(ch);
  st.sum = poly_eval(p, ch);
  ts.grind(sumcheck_pow_bits(security_bits, deg));
  if (eq_factor) {
    const EF& r = (*eq_factor)[round];
    EF f;
    if (skips == 1) {
      f = (ef_one() - r) * (ef_one() - ch) + r * ch;
    } else {
      for (int i = 0; i < n_sk; i++) f += upoly_eval(sel[i], r) * upoly_eval(sel[i], ch);
    }
    st.mmf = st.has_mmf ? f * st.mmf : f;
    st.has_mmf = true;
  }
  std::vector<EF> fs;
  if (skips == 1) fs = {ef_one() - ch, ch};
  else for (int i = 0; i < n_sk; i++) fs.push_back(upoly_eval(sel[i], ch));
  return fold_large<NF>(mls, fs);
}

template <class NF>
static Cols sumcheck_prove(int skips, const std::vector<std::vector<NF>>& mls, const Computation& comp, int degree,
                           const std::vector<EF>* eq_factor, bool is_zerofier, Transcript& ts, EF sum, int n_rounds,
                           int security_bits, ScState& st) {
  st.sum = sum;
  Cols folded = sc_round<NF>(skips, mls, comp, eq_factor, is_zerofier, ts, degree, security_bits, 0, st);
  for (int i = 1; i < n_rounds; i++)
    folded = sc_round<EF>(1, folded, comp, eq_factor, false, ts, degree, security_bits, i, st);
  return folded;
}

// ------------------------------------------------------------ computations
struct AirComputation : Computation {
  const AirSpec& air;
  const std::vector<EF>& alphas;
  AirComputation(const AirSpec& a, const std::vector<EF>& al) : air(a), alphas(al) {}
  EF eval_f(const F* pt) const override { return air.eval_base(pt, alphas); }
  EF eval_e(const EF* pt) const override { return air.eval_ext(pt, alphas); }
};
struct ProductComputation : Computation {  // InnerSumcheckCircuit (crates/air/src/prove.rs:229-235)
  EF eval_f(const F* pt) const override { return EF(pt[0] * pt[1]); }
  EF eval_e(const EF* pt) const override { return pt[0] * pt[1]; }
};
struct AbcComputation : Computation {  // a*b - c
  EF eval_f(const F* pt) const override { return EF(pt[0] * pt[1] - pt[2]); }
  EF eval_e(const EF* pt) const override { return pt[0] * pt[1] - pt[2]; }
};

// uni_skip_utils.rs:5-34
static std::vector<EF> matrix_up_folded(const std::vector<EF>& pt) {
  size_t n = pt.size();
  std::vector<EF> f = eval_eq(pt);
  EF prod = ef_one();
  for (auto& x : pt) prod = prod * x;
  f[(size_t(1) << n) - 1] -= prod;
  f[(size_t(1) << n) - 2] += prod;
  return f;
}
static std::vector<EF> matrix_down_folded(const std::vector<EF>& pt) {
  size_t n = pt.size();
  std::vector<EF> f(size_t(1) << n);
  for (size_t k = 0; k < n; k++) {
    EF prod = ef_one() - pt[n - k - 1];
    for (size_t j = n - k; j < n; j++) prod = prod * pt[j];
    std::vector<EF> e = eval_eq(std::vector<EF>(pt.begin(), pt.begin() + (n - k - 1)));
    for (size_t i = 0; i < e.size(); i++) f[(i << (k + 1)) + (size_t(1) << k)] += e[i] * prod;
  }
  EF all = ef_one();
  for (auto& x : pt) all = all * x;
  f[(size_t(1) << n) - 1] += all;
  return f;
}

static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

std::vector<F> prove_air(const Settings& s, const AirConstants& air, const Hashes& h, int log_n,
                         const std::vector<F>& witness, ProveTimings* tm) {
  return prove_air_spec(s, Poseidon2AirSpec(air), h, log_n, witness, tm);
}

std::vector<F> prove_air_spec(const Settings& s, const AirSpec& air, const Hashes& h, int log_n,
                              const std::vector<F>& witness, ProveTimings* tm) {
  // W: all columns (the preprocessed ones first); Ww: the witness columns, the committed ones
  const int W = air.columns(), NC = air.constraints(), P = air.preprocessed(), Ww = W - P, n = log_n,
            k = s.univariate_skips;
  if (k >= n) throw std::runtime_error("univariate_skips must be < log_n_rows");
  const size_t N = size_t(1) << n;
  if (Ww < 1 || witness.size() != size_t(Ww) * N) throw std::runtime_error("witness size mismatch");
  const int logW = log2_up(Ww);
  WhirConfig cfg = WhirConfig::build(n + logW, s);
  Transcript ts(&h.p16);
  for (F x : cfg.domain_separator()) ts.ch.observe(x);
  double t0 = now_s();

  // 1) commit to the packed witness (packed_multilinear: column index = high variables)
  std::vector<F> packed(N << logW);
  std::copy(witness.begin(), witness.end(), packed.begin());
  std::vector<std::pair<std::vector<EF>, EF>> ood;
  CommitData cd0 = whir_commit_base(cfg, packed, ts, h, ood);
  double t1 = now_s();

  // 2) batching scalars and zerocheck challenges
  ts.grind(std::max(0, s.security_bits - std::max(0, 31 * EXT_D - log2_up(NC))));
  EF alpha = ts.sample_ext();
  std::vector<EF> alphas(NC);
  alphas[0] = ef_one();
  for (int i = 1; i < NC; i++) alphas[i] = alphas[i - 1] * alpha;
  ts.grind(std::max(0, s.security_bits - std::max(0, 31 * EXT_D - n)));
  std::vector<EF> zc(n + 1 - k);
  for (auto& x : zc) x = ts.sample_ext();

  // 3) zerocheck over the up/down columns (crates/air/src/utils.rs:140-160)
  std::vector<std::vector<F>> ud(2 * W);
  for (int c = 0; c < W; c++) {
    const F* col = c < P ? air.preprocessed_column(c, N) : &witness[size_t(c - P) * N];
    ud[c].assign(col, col + N);
    ud[c][N - 1] = ud[c][N - 2];
    ud[W + c].assign(col + 1, col + N);
    F last = ud[W + c].back();
    ud[W + c].push_back(last);
  }
  AirComputation comp(air, alphas);
  ScState st;
  Cols fin = sumcheck_prove<F>(k, ud, comp, air.degree(), &zc, true, ts, EF(), n - k + 1, s.security_bits, st);
  std::vector<EF> zc_ch = st.challenges;
  double t2 = now_s();

  // 4) inner sums and the inner sumcheck
  std::vector<EF> up(Ww), down(Ww);
  for (int c = 0; c < Ww; c++) { up[c] = fin[P + c][0]; down[c] = fin[W + P + c][0]; }
  ts.add_ext(up.data(), Ww);
  ts.add_ext(down.data(), Ww);
  ts.grind(std::max(0, s.security_bits - std::max(0, 31 * EXT_D - logW)));
  std::vector<EF> cbs(logW);
  for (auto& x : cbs) x = ts.sample_ext();
  std::vector<EF> eqc = eval_eq(cbs);
  std::vector<EF> batched(N);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)N; i++) {
    EF acc;
    for (int c = 0; c < Ww; c++) acc += eqc[c] * witness[size_t(c) * N + i];
    batched[i] = acc;
  }
  EF alpha2 = ts.sample_ext();
  std::vector<EF> mixed(N);
  for (size_t i = 0; i < N; i++) {
    EF u = i == N - 1 ? batched[N - 2] : batched[i];
    EF d = i == N - 1 ? batched[N - 1] : batched[i + 1];
    mixed[i] = u + alpha2 * d;
  }
  // EvaluationsList::fold(zc[1..]): bind the last n-k variables
  std::vector<EF> tail(zc_ch.begin() + 1, zc_ch.end());
  std::vector<EF> sub(size_t(1) << k);
  {
    size_t chunk = N >> k;
    for (size_t j = 0; j < sub.size(); j++)
      sub[j] = mle_evaluate(std::vector<EF>(mixed.begin() + j * chunk, mixed.begin() + (j + 1) * chunk), tail);
  }
  ts.add_ext(sub.data(), sub.size());
  std::vector<EF> eps(k);
  for (auto& x : eps) x = ts.sample_ext();
  std::vector<EF> point = eps;
  point.insert(point.end(), tail.begin(), tail.end());
  std::vector<EF> mu = matrix_up_folded(point), md = matrix_down_folded(point);
  std::vector<std::vector<EF>> mles(2);
  mles[0].resize(N);
  for (size_t i = 0; i < N; i++) mles[0][i] = mu[i] + alpha2 * md[i];
  mles[1] = batched;
  EF inner_sum = mle_evaluate(mixed, point);
  ProductComputation prod;
  ScState st2;
  Cols fin2 = sumcheck_prove<EF>(1, mles, prod, 2, nullptr, false, ts, inner_sum, n, s.security_bits, st2);
  std::vector<EF> final_point = cbs;
  final_point.insert(final_point.end(), st2.challenges.begin(), st2.challenges.end());
  EF packed_value = fin2[1][0];
  double t3 = now_s();

  // 5) WHIR opening of the packed witness at final_point
  whir_prove(cfg, ts, packed, cd0, ood, final_point, packed_value, h);
  double t4 = now_s();
  if (tm) { tm->commit = t1 - t0; tm->zerocheck = t2 - t1; tm->inner = t3 - t2; tm->whir = t4 - t3; }
  return ts.proof;
}

// ------------------------------------------------------------ a*b - c zerocheck
std::vector<F> prove_abc(const Poseidon2& p16, int log_n, int skips, const std::vector<F>& a, const std::vector<F>& b,
                         const std::vector<F>& c) {
  Transcript ts(&p16);
  std::vector<EF> r(log_n + 1 - skips);
  for (auto& x : r) x = ts.sample_ext();
  std::vector<std::vector<F>> m{a, b, c};
  AbcComputation comp;
  ScState st;
  Cols fin = sumcheck_prove<F>(skips, m, comp, 2, &r, true, ts, EF(), log_n - skips + 1, 128, st);
  EF finals[3] = {fin[0][0], fin[1][0], fin[2][0]};
  ts.add_ext(finals, 3);
  return ts.proof;
}

}  // namespace wlo
