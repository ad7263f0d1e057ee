// CPU oracle (test infrastructure): WHIR configuration, Reed-Solomon encoding,
// Merkle commitment and the WHIR prover rounds.
//
// whir-p3 (rev 9caef91) is not vendored, so this follows the WHIR paper
// (eprint 2024/1586) with the call shapes of crates/air/src/prove.rs:74-91,216-225
// and table.rs:113-139 (ConstantFromSecondRound(7, 4) folding, rate 1/2, initial RS
// domain reduction 2^5, 16 PoW bits, CapacityBound soundness). Every choice that
// the missing crate would have fixed is explicit here:
//  * codeword layout: commitment C_j of an m-variable multilinear g with folding k
//    is a 2^(D-k) x 2^k matrix, D = m + rho. Row r holds H_p(w^r) for p < 2^k, where
//    H_p(Y) = sum_b' C[p || b'] * Y^(sum_i b'_i 2^(i-1)) and C is the monomial
//    coefficient table of g (Moebius transform of the evaluation table, x_1 = MSB),
//    w generates the subgroup of order 2^(D-k). Folding a row at r_1..r_k is the
//    coefficient-form multilinear evaluation of the row (p's MSB <-> r_1) and gives
//    the folded polynomial's univariate embedding at w^r;
//  * leaves: one row per leaf, hashed by PaddingFreeSponge<P24,24,16,8> over the row's
//    base-field coordinates (EF rows flattened coefficient by coefficient);
//    2-to-1 compression TruncatedPermutation<P16,2,8,16>;
//  * sumcheck messages: evaluations h(0), h(1), h(2);
//  * the queried rows and their authentication paths are appended to the proof as
//    hints (not absorbed by the challenger); query indices are sampled as
//    `sample() & mask`, then sorted and de-duplicated;
//  * combination randomness gamma weighs a round's constraints by 1, gamma, gamma^2...
#include <omp.h>

#include <algorithm>
#include <stdexcept>

#include "oracle.h"

namespace wlo {

static int ood_samples(int security, int num_vars, int log_inv_rate) {
  const int field_bits = 31 * EXT_D;
  for (int s = 1; s < 64; s++) {
    double list_bits = num_vars + log_inv_rate;
    double err = 2.0 * list_bits + double(num_vars) * s;
    if (double(s) * field_bits + 1.0 - err >= security) return s;
  }
  throw std::runtime_error("no OOD sample count reaches the security level");
}

WhirConfig WhirConfig::build(int m0, const Settings& s) {
  WhirConfig cfg;
  cfg.num_vars = m0;
  cfg.security_bits = s.security_bits;
  int k0 = s.fold_first, k = s.fold_rest;
  if (m0 <= k0) throw std::runtime_error("too few variables for the first folding");
  int rest = m0 - k0;
  const int MAX_VARS_SENT = 6;
  if (rest < MAX_VARS_SENT) {
    cfg.num_rounds = 0;
    cfg.final_vars = rest;
  } else {
    cfg.num_rounds = (rest - MAX_VARS_SENT + k - 1) / k;
    cfg.final_vars = rest - cfg.num_rounds * k;
  }
  int protocol_security = std::max(0, s.security_bits - s.whir_pow_bits);
  int m = m0, log_domain = m0 + s.log_inv_rate;
  for (int j = 0; j <= cfg.num_rounds; j++) {
    WhirRound r;
    r.num_vars = m;
    r.fold = j == 0 ? k0 : k;
    r.log_domain = log_domain;
    r.log_inv_rate = log_domain - m;
    r.queries = (protocol_security + r.log_inv_rate - 1) / r.log_inv_rate;
    r.pow_bits = std::max(0, s.security_bits - r.queries * r.log_inv_rate);
    r.ood = ood_samples(s.security_bits, m, r.log_inv_rate);
    if (r.log_domain - r.fold > 24) throw std::runtime_error("domain exceeds the two-adicity of KoalaBear");
    cfg.c.push_back(r);
    log_domain -= j == 0 ? s.rs_reduction : 1;
    m -= r.fold;
  }
  const int field_bits = 31 * EXT_D;
  cfg.fold_pow_bits = std::max(0, s.security_bits - (field_bits - (m0 + s.log_inv_rate) - 1));
  return cfg;
}

std::vector<F> WhirConfig::domain_separator() const {
  std::vector<F> d{F(num_vars), F(num_rounds), F(final_vars), F(security_bits), F(fold_pow_bits)};
  for (const auto& r : c)
    for (int x : {r.num_vars, r.fold, r.log_domain, r.queries, r.pow_bits, r.ood}) d.push_back(F(x));
  return d;
}

// ------------------------------------------------------------ encoding
void mobius_inplace_f(std::vector<F>& v) {
  for (size_t h = 1; h < v.size(); h <<= 1)
    for (size_t i = 0; i < v.size(); i += 2 * h)
      for (size_t j = i; j < i + h; j++) v[j + h] -= v[j];
}
void mobius_inplace(std::vector<EF>& v) {
  for (size_t h = 1; h < v.size(); h <<= 1)
    for (size_t i = 0; i < v.size(); i += 2 * h)
      for (size_t j = i; j < i + h; j++) v[j + h] -= v[j];
}

static uint32_t bitrev(uint32_t x, int bits) {
  uint32_t r = 0;
  for (int i = 0; i < bits; i++) r |= ((x >> i) & 1u) << (bits - 1 - i);
  return r;
}

std::vector<F> ntt_eval(const std::vector<F>& coeffs, int log_size) {
  size_t n = size_t(1) << log_size;
  if (coeffs.size() > n) throw std::runtime_error("ntt: too many coefficients");
  std::vector<F> a(n);
  for (size_t i = 0; i < coeffs.size(); i++) a[bitrev(uint32_t(i), log_size)] = coeffs[i];
  for (int s = 1; s <= log_size; s++) {
    size_t len = size_t(1) << s, half = len >> 1;
    F wlen = two_adic_generator(s);
    for (size_t i = 0; i < n; i += len) {
      F w(1);
      for (size_t j = 0; j < half; j++) {
        F u = a[i + j], v = a[i + j + half] * w;
        a[i + j] = u + v;
        a[i + j + half] = u - v;
        w *= wlen;
      }
    }
  }
  return a;
}

CommitData whir_encode_commit(const std::vector<F>& flat, int m, int k, int log_domain, int elem,
                              const Poseidon2& p24, const Poseidon2& p16) {
  CommitData cd;
  cd.num_vars = m;
  cd.fold = k;
  cd.elem = elem;
  cd.log_leaves = log_domain - k;
  const int L = m - k;
  const size_t rows = size_t(1) << cd.log_leaves, width = size_t(1) << k, rl = cd.row_len();
  if (flat.size() != (size_t(elem) << m)) throw std::runtime_error("encode: size mismatch");
  cd.leaves.assign(rows * rl, F());
  for (int e = 0; e < elem; e++) {
    std::vector<F> v(size_t(1) << m);
    for (size_t i = 0; i < v.size(); i++) v[i] = flat[i * elem + e];
    mobius_inplace_f(v);
#pragma omp parallel for schedule(dynamic)
    for (int64_t p = 0; p < (int64_t)width; p++) {
      std::vector<F> a(size_t(1) << L);
      for (size_t j = 0; j < a.size(); j++) a[j] = v[(size_t(p) << L) + bitrev(uint32_t(j), L)];
      std::vector<F> ev = ntt_eval(a, cd.log_leaves);
      for (size_t r = 0; r < rows; r++) cd.leaves[r * rl + size_t(p) * elem + e] = ev[r];
    }
  }
  cd.tree.emplace_back(rows);
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < (int64_t)rows; r++) cd.tree[0][r] = sponge_hash(p24, &cd.leaves[r * rl], rl);
  while (cd.tree.back().size() > 1) {
    const auto& lv = cd.tree.back();
    std::vector<Digest> up(lv.size() / 2);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)up.size(); i++) up[i] = compress(p16, lv[2 * i], lv[2 * i + 1]);
    cd.tree.push_back(std::move(up));
  }
  return cd;
}

EF fold_leaf(const F* row, int k, int elem, const std::vector<EF>& r) {
  std::vector<EF> v(size_t(1) << k);
  for (size_t p = 0; p < v.size(); p++)
    for (int e = 0; e < elem; e++) v[p].c[e] = row[p * elem + e];
  for (int i = 0; i < k; i++) {
    size_t h = v.size() / 2;
    for (size_t q = 0; q < h; q++) v[q] = v[q] + r[i] * v[q + h];
    v.resize(h);
  }
  return v[0];
}

std::vector<EF> pow_point(const EF& z, int m) {
  std::vector<EF> pt(m);
  EF cur = z;
  for (int i = 0; i < m; i++) { pt[i] = cur; cur = cur * cur; }
  return pt;
}

// ------------------------------------------------------------ WHIR sumcheck
static EF quad_eval(const EF h[3], const EF& r) {
  // Lagrange on {0,1,2}: h0 (r-1)(r-2)/2 - h1 r(r-2) + h2 r(r-1)/2
  static const F inv2 = finv(F(2));
  EF rm1 = r - F(1), rm2 = r - F(2);
  return (h[0] * rm1 * rm2) * inv2 - h[1] * r * rm2 + (h[2] * r * rm1) * inv2;
}

static void whir_sumcheck(std::vector<EF>& g, std::vector<EF>& w, EF& sigma, int rounds, int pow_bits, Transcript& ts,
                          std::vector<EF>& rand_out) {
  for (int t = 0; t < rounds; t++) {
    size_t h = g.size() / 2;
    EF s0, s1, s2;
#pragma omp parallel
    {
      EF a0, a1, a2;
#pragma omp for schedule(static) nowait
      for (int64_t i = 0; i < (int64_t)h; i++) {
        a0 += g[i] * w[i];
        a1 += g[i + h] * w[i + h];
        a2 += (g[i + h] + g[i + h] - g[i]) * (w[i + h] + w[i + h] - w[i]);
      }
#pragma omp critical
      { s0 += a0; s1 += a1; s2 += a2; }
    }
    EF hv[3] = {s0, s1, s2};
    ts.add_ext(hv, 3);
    ts.grind(pow_bits);
    EF r = ts.sample_ext();
    rand_out.push_back(r);
    sigma = quad_eval(hv, r);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)h; i++) {
      g[i] = g[i] + r * (g[i + h] - g[i]);
      w[i] = w[i] + r * (w[i + h] - w[i]);
    }
    g.resize(h);
    w.resize(h);
  }
}

static std::vector<uint32_t> sample_queries(Transcript& ts, int log_leaves, int count) {
  std::vector<uint32_t> q(count);
  for (auto& x : q) x = ts.ch.sample_bits(log_leaves);
  std::sort(q.begin(), q.end());
  q.erase(std::unique(q.begin(), q.end()), q.end());
  return q;
}

static void open_queries(const CommitData& cd, const std::vector<uint32_t>& idx, Transcript& ts) {
  for (uint32_t i : idx) {
    ts.hint(&cd.leaves[size_t(i) * cd.row_len()], cd.row_len());
    uint32_t pos = i;
    for (int l = 0; l < cd.log_leaves; l++) {
      ts.hint(cd.tree[l][pos ^ 1].data(), 8);
      pos >>= 1;
    }
  }
}

// Adds sum_t gamma^t eq(pt_t, .) to w and sum_t gamma^t v_t to sigma.
static void add_constraints(std::vector<EF>& w, EF& sigma, const EF& gamma,
                            const std::vector<std::pair<std::vector<EF>, EF>>& cons) {
  EF coef = ef_one();
  for (const auto& c : cons) {
    std::vector<EF> e = eval_eq(c.first);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)w.size(); i++) w[i] += coef * e[i];
    sigma += coef * c.second;
    coef = coef * gamma;
  }
}

static EF mle_evaluate_f(const std::vector<F>& evals, const std::vector<EF>& point) {
  size_t h = evals.size() / 2;
  std::vector<EF> cur(h);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)h; i++) cur[i] = EF(evals[i]) + point[0] * EF(evals[i + h] - evals[i]);
  std::vector<EF> rest(point.begin() + 1, point.end());
  return mle_evaluate(cur, rest);
}

CommitData whir_commit_base(const WhirConfig& cfg, const std::vector<F>& evals, Transcript& ts, const Hashes& h,
                            std::vector<std::pair<std::vector<EF>, EF>>& ood) {
  const WhirRound& c0 = cfg.c[0];
  CommitData cd = whir_encode_commit(evals, c0.num_vars, c0.fold, c0.log_domain, 1, h.p24, h.p16);
  ts.add_base(cd.tree.back()[0].data(), 8);
  for (int s = 0; s < c0.ood; s++) {
    EF z = ts.sample_ext();
    std::vector<EF> pt = pow_point(z, c0.num_vars);
    EF y = mle_evaluate_f(evals, pt);
    ts.add_ext(&y, 1);
    ood.push_back({pt, y});
  }
  return cd;
}

void whir_prove(const WhirConfig& cfg, Transcript& ts, const std::vector<F>& evals, const CommitData& cd0,
                const std::vector<std::pair<std::vector<EF>, EF>>& ood, const std::vector<EF>& point, const EF& value,
                const Hashes& h) {
  std::vector<std::pair<std::vector<EF>, EF>> cons = ood;
  cons.push_back({point, value});
  std::vector<EF> g(evals.size()), w(evals.size());
  for (size_t i = 0; i < evals.size(); i++) g[i] = EF(evals[i]);
  EF sigma;
  EF gamma = ts.sample_ext();
  add_constraints(w, sigma, gamma, cons);
  std::vector<EF> rnd;
  whir_sumcheck(g, w, sigma, cfg.c[0].fold, cfg.fold_pow_bits, ts, rnd);
  std::vector<EF> last_r = rnd;
  const CommitData* prev = &cd0;
  std::vector<CommitData> commits;
  commits.reserve(cfg.num_rounds);
  for (int i = 0; i < cfg.num_rounds; i++) {
    const WhirRound& ci = cfg.c[i];
    const WhirRound& cn = cfg.c[i + 1];
    std::vector<F> flat(g.size() * 8);
    for (size_t x = 0; x < g.size(); x++)
      for (int e = 0; e < 8; e++) flat[x * 8 + e] = g[x].c[e];
    commits.push_back(whir_encode_commit(flat, cn.num_vars, cn.fold, cn.log_domain, 8, h.p24, h.p16));
    const CommitData& cd = commits.back();
    ts.add_base(cd.tree.back()[0].data(), 8);
    std::vector<std::pair<std::vector<EF>, EF>> nc;
    for (int s = 0; s < cn.ood; s++) {
      EF z = ts.sample_ext();
      std::vector<EF> pt = pow_point(z, cn.num_vars);
      EF y = mle_evaluate(g, pt);
      ts.add_ext(&y, 1);
      nc.push_back({pt, y});
    }
    ts.grind(ci.pow_bits);
    std::vector<uint32_t> q = sample_queries(ts, prev->log_leaves, ci.queries);
    open_queries(*prev, q, ts);
    F gen = two_adic_generator(prev->log_leaves);
    for (uint32_t idx : q) {
      EF y(fpow(gen, idx));
      EF v = fold_leaf(&prev->leaves[size_t(idx) * prev->row_len()], prev->fold, prev->elem, last_r);
      nc.push_back({pow_point(y, cn.num_vars), v});
    }
    EF gm = ts.sample_ext();
    add_constraints(w, sigma, gm, nc);
    last_r.clear();
    whir_sumcheck(g, w, sigma, cn.fold, cfg.fold_pow_bits, ts, last_r);
    prev = &cd;
  }
  // final round: send the remaining polynomial, open the last commitment, finish the sumcheck
  ts.add_ext(g.data(), g.size());
  const WhirRound& cl = cfg.c[cfg.num_rounds];
  ts.grind(cl.pow_bits);
  std::vector<uint32_t> q = sample_queries(ts, prev->log_leaves, cl.queries);
  open_queries(*prev, q, ts);
  std::vector<EF> fr;
  whir_sumcheck(g, w, sigma, cfg.final_vars, cfg.fold_pow_bits, ts, fr);
}

// ------------------------------------------------------------ WHIR verifier
struct ConstraintGroup {
  int first_round;  // index into the list of folding-randomness blocks
  std::vector<std::pair<std::vector<EF>, EF>> cons;  // points and coefficients
};

static bool verify_path(const Hashes& h, const F* row, size_t rl, uint32_t idx, const F* path, int depth,
                        const Digest& root) {
  Digest cur = sponge_hash(h.p24, row, rl);
  for (int l = 0; l < depth; l++) {
    Digest sib;
    for (int e = 0; e < 8; e++) sib[e] = path[l * 8 + e];
    cur = ((idx >> l) & 1) ? compress(h.p16, sib, cur) : compress(h.p16, cur, sib);
  }
  return cur == root;
}

static bool whir_sumcheck_verify(Transcript& ts, EF& sigma, int rounds, int pow_bits, std::vector<EF>& rnd) {
  for (int t = 0; t < rounds; t++) {
    EF hv[3];
    if (!ts.next_ext(hv, 3)) return false;
    if (hv[0] + hv[1] != sigma) return false;
    if (!ts.check_grind(pow_bits)) return false;
    EF r = ts.sample_ext();
    rnd.push_back(r);
    sigma = quad_eval(hv, r);
  }
  return true;
}

bool whir_parse_commitment(const WhirConfig& cfg, Transcript& ts, Digest& root,
                           std::vector<std::pair<std::vector<EF>, EF>>& ood) {
  if (!ts.next_base(root.data(), 8)) return false;
  for (int s = 0; s < cfg.c[0].ood; s++) {
    EF z = ts.sample_ext();
    EF y;
    if (!ts.next_ext(&y, 1)) return false;
    ood.push_back({pow_point(z, cfg.num_vars), y});
  }
  return true;
}

bool whir_verify(const WhirConfig& cfg, Transcript& ts, const Digest& root0,
                 const std::vector<std::pair<std::vector<EF>, EF>>& ood, const std::vector<EF>& point,
                 const EF& value, const Hashes& h) {
  std::vector<std::vector<EF>> blocks;  // folding randomness per sumcheck block
  std::vector<ConstraintGroup> groups;
  EF sigma;
  {
    EF gamma = ts.sample_ext();
    ConstraintGroup g0{0, {}};
    EF coef = ef_one();
    auto all = ood;
    all.push_back({point, value});
    for (auto& c : all) {
      g0.cons.push_back({c.first, coef});
      sigma += coef * c.second;
      coef = coef * gamma;
    }
    groups.push_back(g0);
  }
  std::vector<EF> r;
  if (!whir_sumcheck_verify(ts, sigma, cfg.c[0].fold, cfg.fold_pow_bits, r)) return false;
  blocks.push_back(r);
  Digest prev_root = root0;
  for (int i = 0; i < cfg.num_rounds; i++) {
    const WhirRound& ci = cfg.c[i];
    const WhirRound& cn = cfg.c[i + 1];
    Digest root;
    if (!ts.next_base(root.data(), 8)) return false;
    std::vector<std::pair<std::vector<EF>, EF>> nc;
    for (int s = 0; s < cn.ood; s++) {
      EF z = ts.sample_ext();
      EF y;
      if (!ts.next_ext(&y, 1)) return false;
      nc.push_back({pow_point(z, cn.num_vars), y});
    }
    if (!ts.check_grind(ci.pow_bits)) return false;
    int log_leaves = ci.log_domain - ci.fold;
    std::vector<uint32_t> q = sample_queries(ts, log_leaves, ci.queries);
    int elem = i == 0 ? 1 : 8;
    size_t rl = size_t(elem) << ci.fold;
    F gen = two_adic_generator(log_leaves);
    for (uint32_t idx : q) {
      std::vector<F> row(rl), path(size_t(8) * log_leaves);
      if (!ts.next_hint(row.data(), rl) || !ts.next_hint(path.data(), path.size())) return false;
      if (!verify_path(h, row.data(), rl, idx, path.data(), log_leaves, prev_root)) return false;
      nc.push_back({pow_point(EF(fpow(gen, idx)), cn.num_vars), fold_leaf(row.data(), ci.fold, elem, blocks.back())});
    }
    EF gm = ts.sample_ext();
    ConstraintGroup grp{i + 1, {}};
    EF coef = ef_one();
    for (auto& c : nc) {
      grp.cons.push_back({c.first, coef});
      sigma += coef * c.second;
      coef = coef * gm;
    }
    groups.push_back(grp);
    std::vector<EF> rr;
    if (!whir_sumcheck_verify(ts, sigma, cn.fold, cfg.fold_pow_bits, rr)) return false;
    blocks.push_back(rr);
    prev_root = root;
  }
  // final round
  std::vector<EF> gfin(size_t(1) << cfg.final_vars);
  if (!ts.next_ext(gfin.data(), gfin.size())) return false;
  const WhirRound& cl = cfg.c[cfg.num_rounds];
  if (!ts.check_grind(cl.pow_bits)) return false;
  {
    int log_leaves = cl.log_domain - cl.fold;
    std::vector<uint32_t> q = sample_queries(ts, log_leaves, cl.queries);
    int elem = cfg.num_rounds == 0 ? 1 : 8;
    size_t rl = size_t(elem) << cl.fold;
    F gen = two_adic_generator(log_leaves);
    for (uint32_t idx : q) {
      std::vector<F> row(rl), path(size_t(8) * log_leaves);
      if (!ts.next_hint(row.data(), rl) || !ts.next_hint(path.data(), path.size())) return false;
      if (!verify_path(h, row.data(), rl, idx, path.data(), log_leaves, prev_root)) return false;
      EF folded = fold_leaf(row.data(), cl.fold, elem, blocks.back());
      if (folded != mle_evaluate(gfin, pow_point(EF(fpow(gen, idx)), cfg.final_vars))) return false;
    }
  }
  std::vector<EF> rf;
  if (!whir_sumcheck_verify(ts, sigma, cfg.final_vars, cfg.fold_pow_bits, rf)) return false;
  blocks.push_back(rf);
  // sigma must equal g_final(rf) * W(all folding randomness)
  EF wsum;
  for (const auto& grp : groups) {
    std::vector<EF> pt;
    for (size_t b = grp.first_round; b < blocks.size(); b++) pt.insert(pt.end(), blocks[b].begin(), blocks[b].end());
    for (const auto& c : grp.cons) wsum += c.second * eq_poly(c.first, pt);
  }
  return sigma == mle_evaluate(gfin, rf) * wsum;
}

}  // namespace wlo
