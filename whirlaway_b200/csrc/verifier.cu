// Host-side verifiers (no device, no context):
//  * the AIR proof: AirTable::verify (crates/air/src/verify.rs:55-249), with the sumcheck
//    verifiers sumcheck::verify / verify_with_univariate_skip (crates/sumcheck/src/verify.rs:
//    23-113), the shift-matrix evaluations matrix_up_lde / matrix_down_lde / next_mle
//    (crates/air/src/utils.rs:12-138) and whir-p3's WHIR verifier (commitment parsing, OOD
//    answers, STIR queries with Merkle paths, folding sumchecks, final polynomial), reading the
//    transcript in the order prove_air (prover.cu) writes it;
//  * the a*b - c zerocheck proof of prove_abc (the sumcheck microbenchmark).
// Outcomes follow AirVerifError (crates/air/src/verify.rs:26-34): anything that fails inside a
// sumcheck (short proof, grinding, a round sum) is a sumcheck error, anything inside the WHIR
// opening an opening error.
#include <algorithm>
#include <thread>
#include <atomic>
#include <string>
#include <vector>

#include "verifier.h"

namespace wl {
namespace {

using kb::ef;

// proof_data as the verifier's VerifierState reads it: messages go through the challenger,
// hints (Merkle rows and paths) do not. Words arrive canonical and are used in Montgomery form.
struct ProofReader {
  HostChallenger ch;
  const uint32_t* words;
  size_t len, pos = 0;
  TranscriptLog* log = nullptr;
  ProofReader(const kb::P16Consts* p16, const uint32_t* w, size_t n, TranscriptLog* lg = nullptr)
      : words(w), len(n), log(lg) {
    ch.perm = p16;
  }
  void phase(const char* name) {
    if (log) log->begin(name, pos);
  }
  bool base(uint32_t* v, size_t n) {
    if (len - pos < n) return false;
    for (size_t i = 0; i < n; i++) {
      v[i] = kb::to_mont(words[pos++]);
      ch.observe(v[i]);
    }
    return true;
  }
  bool ext(ef* v, size_t n) {
    for (size_t i = 0; i < n; i++)
      if (!base(v[i].c, 8)) return false;
    return true;
  }
  bool hint(uint32_t* v, size_t n) {
    if (len - pos < n) return false;
    for (size_t i = 0; i < n; i++) v[i] = kb::to_mont(words[pos++]);
    return true;
  }
  ef sample() {
    ef e;
    for (int i = 0; i < 8; i++) e.c[i] = ch.sample();
    if (log) log->add("challenge", pos, e.c, 8, true);
    return e;
  }
  // check_pow_grinding: the witness is observed, then `bits` sampled bits must be zero (no
  // witness at all for 0 bits)
  bool pow(int bits) {
    if (bits <= 0) return true;
    const size_t at = pos;
    uint32_t w;
    if (!base(&w, 1)) return false;
    if (log) log->add("grinding", at, &w, 1, true);
    return ch.sample_bits(bits) == 0;
  }
};

ef ef_int(int64_t x) { return kb::ef_from(fm(x)); }

// Sumcheck rounds: round r sends deg[r] + 1 coefficients whose sum over {0..set[r]-1} is the
// first round's claim or the previous round's target; then a challenge, then grinding.
struct Claim {
  ef sum;
  std::vector<ef> point;
  ef value;
};
bool sumcheck_rounds(ProofReader& rd, const std::vector<int>& deg, const std::vector<int>& set, int security,
                     Claim& out) {
  ef target = kb::ef_zero();
  for (size_t r = 0; r < deg.size(); r++) {
    std::vector<ef> c(deg[r] + 1);
    if (!rd.ext(c.data(), c.size())) return false;
    ef s = kb::ef_zero();
    for (int x = 0; x < set[r]; x++) s = kb::ef_add(s, poly_eval(c, ef_int(x)));
    if (r == 0) out.sum = s;
    else if (!kb::ef_eq(s, target)) return false;
    const ef ch = rd.sample();
    if (!rd.pow(sumcheck_pow_bits(security, deg[r]))) return false;
    target = poly_eval(c, ch);
    out.point.push_back(ch);
  }
  out.value = target;
  return true;
}

ef mle_eval(const std::vector<ef>& table, const std::vector<ef>& pt) {
  const std::vector<ef> e = eq_table_host(pt);
  ef r = kb::ef_zero();
  for (size_t i = 0; i < table.size(); i++) r = kb::ef_add(r, kb::ef_mul(e[i], table[i]));
  return r;
}

// Shift matrices as multilinears in (row bits, column bits), both big-endian. UP is the
// identity with its last row repeating the one above; DOWN maps row x to x + 1 with its last
// row repeating itself.
ef ef_product(const std::vector<ef>& v, size_t n) {
  ef p = kb::ef_one();
  for (size_t i = 0; i < n; i++) p = kb::ef_mul(p, v[i]);
  return p;
}
ef matrix_up(const std::vector<ef>& pt) {
  const size_t n = pt.size() / 2;
  const std::vector<ef> x(pt.begin(), pt.begin() + n), y(pt.begin() + n, pt.end());
  const ef last = pt.back();
  return kb::ef_add(eq_eval(x, y), kb::ef_mul(ef_product(pt, pt.size() - 1), kb::ef_sub(kb::ef_one(), kb::ef_add(last, last))));
}
// successor(x, y) = sum over the carry position k of [bits above k equal] [x_k = 0, y_k = 1]
// [bits below k: x = 1, y = 0], accumulated from the least significant bit in one pass:
// acc_k = acc_(k-1) e_k + c_k o_0 ... o_(k-1).
ef successor(const std::vector<ef>& pt) {
  const size_t n = pt.size() / 2;
  const ef one = kb::ef_one();
  ef acc = kb::ef_zero(), low = one;
  for (size_t k = 0; k < n; k++) {
    const ef& x = pt[n - 1 - k];
    const ef& y = pt[2 * n - 1 - k];
    const ef ox = kb::ef_sub(one, x), oy = kb::ef_sub(one, y);
    const ef e = kb::ef_add(kb::ef_mul(x, y), kb::ef_mul(ox, oy));
    acc = kb::ef_add(kb::ef_mul(acc, e), kb::ef_mul(kb::ef_mul(ox, y), low));
    low = kb::ef_mul(low, kb::ef_mul(x, oy));
  }
  return acc;
}
ef matrix_down(const std::vector<ef>& pt) { return kb::ef_add(successor(pt), ef_product(pt, pt.size())); }

// ---------------------------------------------------------------- WHIR
using Digest = std::array<uint32_t, 8>;
// Merkle checks of queries [i0, i1) of a round: the leaf sponges (PaddingFreeSponge over
// Poseidon2-24, rate 16, zero capacity, of each 128-value row) and then, level by level, the
// 2-to-1 compressions (the first 8 words of Poseidon2-16(left || right)) of every query at once,
// as batches of independent permutations (sixteen per vector with AVX-512). ok[i] = 1 when the
// path of query i ends at the root.
void merkle_check_range(const uint32_t* rows, const uint32_t* paths, const uint32_t* q, size_t i0, size_t i1, int ll,
                        const Digest& root, const kb::P24Consts& p24, const kb::P16Consts& p16, char* ok) {
  const size_t m = i1 - i0, rl = 128, pl = size_t(8) * ll;
  std::vector<uint32_t> st(m * 24, 0u);
  for (int c = 0; c < 8; c++) {
    for (size_t j = 0; j < m; j++)
      for (int i = 0; i < 16; i++) st[j * 24 + i] = rows[(i0 + j) * rl + 16 * c + i];
    host_p24_permute_many(st.data(), m, p24);
  }
  std::vector<uint32_t> cur(m * 8), s16(m * 16);
  for (size_t j = 0; j < m; j++)
    for (int e = 0; e < 8; e++) cur[j * 8 + e] = st[j * 24 + e];
  for (int l = 0; l < ll; l++) {
    for (size_t j = 0; j < m; j++) {
      const uint32_t* sib = paths + (i0 + j) * pl + size_t(l) * 8;
      const bool right = (q[i0 + j] >> l) & 1;  // the current node is the right child
      for (int e = 0; e < 8; e++) {
        s16[j * 16 + e] = right ? sib[e] : cur[j * 8 + e];
        s16[j * 16 + 8 + e] = right ? cur[j * 8 + e] : sib[e];
      }
    }
    host_p16_permute_many(s16.data(), m, p16);
    for (size_t j = 0; j < m; j++)
      for (int e = 0; e < 8; e++) cur[j * 8 + e] = s16[j * 16 + e];
  }
  for (size_t j = 0; j < m; j++) ok[i0 + j] = std::equal(root.begin(), root.end(), cur.begin() + j * 8) ? 1 : 0;
}

struct Constraint {
  std::vector<ef> point;
  ef coef;
};
struct Group {
  size_t first_block;  // the folding blocks its points span, from this one to the end
  std::vector<Constraint> cons;
};

class WhirVerifier {
 public:
  WhirVerifier(const WhirSchedule& ws, const kb::P16Consts& p16, const kb::P24Consts& p24, ProofReader& rd,
               int threads, std::vector<MerkleOpening>* defer)
      : ws_(ws), p16_(p16), p24_(p24), rd_(rd), threads_(threads), defer_(defer) {}

  // Commitment: the root, then one answer per OOD sample z at the point (z, z^2, z^4, ...).
  bool parse_commitment(Digest& root, std::vector<std::vector<ef>>& pts, std::vector<ef>& vals) {
    root0_off_ = rd_.pos;
    if (!rd_.base(root.data(), 8)) return false;
    for (int q = 0; q < ws_.c[0].ood; q++) {
      const ef z = rd_.sample();
      ef y;
      if (!rd_.ext(&y, 1)) return false;
      pts.push_back(pow_point(z, ws_.num_vars));
      vals.push_back(y);
    }
    return true;
  }

  bool verify(const Digest& root0, std::vector<std::vector<ef>> pts, std::vector<ef> vals) {
    rd_.phase("whir");
    ef sigma = kb::ef_zero();
    add_group(0, pts, vals, rd_.sample(), sigma);
    if (!fold_block(ws_.c[0].fold, sigma)) return false;
    Digest prev_root = root0;
    size_t prev_root_off = root0_off_;
    for (int i = 0; i < ws_.num_rounds; i++) {
      const WhirRound& ci = ws_.c[i];
      const WhirRound& cn = ws_.c[i + 1];
      rd_.phase(("whir_round_" + std::to_string(i + 1)).c_str());
      Digest root;
      const size_t root_off = rd_.pos;
      if (!rd_.base(root.data(), 8)) return false;
      std::vector<std::vector<ef>> npts;
      std::vector<ef> nvals;
      for (int q = 0; q < cn.ood; q++) {
        const ef z = rd_.sample();
        ef y;
        if (!rd_.ext(&y, 1)) return false;
        npts.push_back(pow_point(z, cn.num_vars));
        nvals.push_back(y);
      }
      if (!rd_.pow(ci.pow_bits)) return false;
      // STIR queries on the previous commitment: the folded value of each opened row
      std::vector<uint32_t> q;
      std::vector<ef> folded;
      if (!open(ci, i == 0 ? 1 : 8, prev_root, prev_root_off, q, folded)) return false;
      const uint32_t gen = kb::two_adic_gen_m(ci.log_leaves());
      for (size_t t = 0; t < q.size(); t++) {
        npts.push_back(pow_point(kb::ef_from(kb::pow_m(gen, q[t])), cn.num_vars));
        nvals.push_back(folded[t]);
      }
      add_group(blocks_.size(), npts, nvals, rd_.sample(), sigma);
      if (!fold_block(cn.fold, sigma)) return false;
      prev_root = root;
      prev_root_off = root_off;
    }
    // final polynomial, its queries, the last sumcheck
    rd_.phase("whir_final");
    std::vector<ef> gfin(size_t(1) << ws_.final_vars);
    if (!rd_.ext(gfin.data(), gfin.size())) return false;
    const WhirRound& cl = ws_.c[ws_.num_rounds];
    if (!rd_.pow(cl.pow_bits)) return false;
    std::vector<uint32_t> q;
    std::vector<ef> folded;
    if (!open(cl, ws_.num_rounds == 0 ? 1 : 8, prev_root, prev_root_off, q, folded)) return false;
    const uint32_t gen = kb::two_adic_gen_m(cl.log_leaves());
    for (size_t t = 0; t < q.size(); t++)
      if (!kb::ef_eq(folded[t], mle_eval(gfin, pow_point(kb::ef_from(kb::pow_m(gen, q[t])), ws_.final_vars))))
        return false;
    if (!fold_block(ws_.final_vars, sigma)) return false;
    // sigma = g_final(r_final) * sum over all constraints of coef * eq(point, folding randomness)
    ef wsum = kb::ef_zero();
    for (const Group& g : groups_) {
      std::vector<ef> r;
      for (size_t b = g.first_block; b < blocks_.size(); b++) r.insert(r.end(), blocks_[b].begin(), blocks_[b].end());
      for (const Constraint& c : g.cons) wsum = kb::ef_add(wsum, kb::ef_mul(c.coef, eq_eval(c.point, r)));
    }
    return kb::ef_eq(sigma, kb::ef_mul(mle_eval(gfin, blocks_.back()), wsum));
  }

 private:
  // Constraints batched by powers of the round's combination randomness.
  void add_group(size_t first_block, const std::vector<std::vector<ef>>& pts, const std::vector<ef>& vals,
                 const ef& gamma, ef& sigma) {
    Group g{first_block, {}};
    ef cur = kb::ef_one();
    for (size_t j = 0; j < pts.size(); j++) {
      g.cons.push_back({pts[j], cur});
      sigma = kb::ef_add(sigma, kb::ef_mul(cur, vals[j]));
      cur = kb::ef_mul(cur, gamma);
    }
    groups_.push_back(std::move(g));
  }
  // `rounds` quadratic sumcheck rounds (values at 0, 1, 2), each with the folding grinding.
  bool fold_block(int rounds, ef& sigma) {
    std::vector<ef> r;
    for (int t = 0; t < rounds; t++) {
      ef h[3];
      if (!rd_.ext(h, 3)) return false;
      if (!kb::ef_eq(kb::ef_add(h[0], h[1]), sigma)) return false;
      if (!rd_.pow(ws_.fold_pow_bits)) return false;
      const ef c = rd_.sample();
      r.push_back(c);
      sigma = quad_eval(h, c);
    }
    blocks_.push_back(std::move(r));
    return true;
  }
  // Samples the queries of round `rc` on the commitment with `root`, checks each opened row
  // (128 values, Moebius-transformed as hashed) against it and folds it with the last block's
  // randomness (coefficient form, the row's most significant position bit first).
  // With a deferral list, the paths are not hashed here: each opening (offsets of its row, path
  // and root in proof_data) is appended to the list for a batched check, and the rows are
  // folded as if their paths held.
  bool open(const WhirRound& rc, int elem, const Digest& root, size_t root_off, std::vector<uint32_t>& q,
            std::vector<ef>& folded) {
    const int ll = rc.log_leaves();
    q.resize(rc.queries);
    for (auto& x : q) x = rd_.ch.sample_bits(ll);
    std::sort(q.begin(), q.end());
    q.erase(std::unique(q.begin(), q.end()), q.end());
    if (rd_.log) rd_.log->add("queries", rd_.pos, q.data(), q.size(), false);
    // the hints are read in order; the paths are then checked and the rows folded in parallel
    // (each query is independent: one leaf sponge, ll compressions, one fold)
    const size_t nq = q.size(), rl = 128, pl = size_t(8) * ll;
    std::vector<uint32_t> rows(nq * rl), paths(nq * pl);
    for (size_t i = 0; i < nq; i++) {
      const size_t row_off = rd_.pos;
      if (!rd_.hint(&rows[i * rl], rl)) return false;
      const size_t path_off = rd_.pos;
      if (!rd_.hint(&paths[i * pl], pl)) return false;
      if (defer_) defer_->push_back({row_off, path_off, root_off, q[i], ll});
    }
    const std::vector<ef>& r = blocks_.back();
    folded.assign(nq, kb::ef_zero());
    std::vector<char> good(nq, 0);
    // The fold v[p] <- v[p] + r_j v[p + h] (top variable first) of a row is sum_p row[p] m[p]
    // with m[p] the product of r_j over the bits j of p (bit k-1-j for r_j): one table per
    // round, then an extension x base product per value for base-field rows.
    const int k = rc.fold;
    std::vector<ef> m(size_t(1) << k, kb::ef_one());
    for (int j = 0; j < k; j++) {
      const size_t bit = size_t(1) << (k - 1 - j);
      for (size_t p = 0; p < m.size(); p++)
        if (p & bit) m[p] = kb::ef_mul(m[p], r[j]);
    }
    // queries in chunks of 32: the chunk's Merkle paths as batched permutations, then its folds
    constexpr size_t CHUNK = 32;
    auto check = [&](size_t i0, size_t i1) {
      if (defer_) {
        for (size_t i = i0; i < i1; i++) good[i] = 1;
      } else {
        merkle_check_range(rows.data(), paths.data(), q.data(), i0, i1, ll, root, p24_, p16_, good.data());
      }
      for (size_t i = i0; i < i1; i++) {
        if (!good[i]) continue;
        const uint32_t* row = &rows[i * rl];
        ef acc = kb::ef_zero();
        for (size_t p = 0; p < m.size(); p++) {
          if (elem == 1) {
            acc = kb::ef_add(acc, kb::ef_mul_f(m[p], row[p]));
          } else {
            ef v = kb::ef_zero();
            for (int e = 0; e < elem; e++) v.c[e] = row[p * elem + e];
            acc = kb::ef_add(acc, kb::ef_mul(m[p], v));
          }
        }
        folded[i] = acc;
      }
    };
    const size_t nchunks = (nq + CHUNK - 1) / CHUNK;
    const unsigned hw = std::thread::hardware_concurrency();
    const size_t cap = threads_ > 0 ? size_t(threads_) : std::min<size_t>(hw ? hw : 1, 16);
    const size_t T = std::min<size_t>(cap, nchunks);
    std::atomic<size_t> next{0};
    auto work = [&] {
      for (size_t c = next++; c < nchunks; c = next++) check(c * CHUNK, std::min(nq, (c + 1) * CHUNK));
    };
    if (T <= 1) {
      work();
    } else {
      run_on_threads(T, work);
    }
    for (size_t i = 0; i < nq; i++)
      if (!good[i]) return false;
    return true;
  }

  const WhirSchedule& ws_;
  const kb::P16Consts& p16_;
  const kb::P24Consts& p24_;
  ProofReader& rd_;
  int threads_;                          // host threads for the query checks (0: up to 16)
  std::vector<MerkleOpening>* defer_;    // when set, openings are listed instead of checked
  size_t root0_off_ = 0;
  std::vector<std::vector<ef>> blocks_;  // folding randomness of each sumcheck block
  std::vector<Group> groups_;
};

}  // namespace

int verify_air_proof(const Settings& s, const AirConsts& air, const kb::P16Consts& p16, const kb::P24Consts& p24,
                     int n, const uint32_t* proof, size_t proof_len, TranscriptLog* log, int threads,
                     std::vector<MerkleOpening>* defer, const ProgramAir* prog) {
  // W: the witness (committed) columns; the program's first P columns are preprocessed
  const int k = s.univariate_skips, W = prog ? prog->witness_columns() : AIR_W, nsk = 1 << k;
  const int NC = prog ? prog->NC : AIR_NC, LOGW = log2_up(size_t(W)), d1 = (prog ? prog->degree : 3) + 1;
  const int P = prog ? prog->P : 0;
  if (P > 0 && prog->pre_log_n != n) return VERIFY_FS;
  const WhirSchedule ws = WhirSchedule::build(n + LOGW, s);
  ProofReader rd(&p16, proof, proof_len, log);
  for (uint32_t x : ws.domain_separator()) rd.ch.observe(kb::to_mont(x));
  rd.phase("commit");
  WhirVerifier whir(ws, p16, p24, rd, threads, defer);
  Digest root;
  std::vector<std::vector<ef>> ood_pts;
  std::vector<ef> ood_vals;
  if (!whir.parse_commitment(root, ood_pts, ood_vals)) return VERIFY_PCS_COMMITMENT;

  rd.phase("batching");
  if (!rd.pow(batching_pow_bits(s.security_bits, log2_up(size_t(NC))))) return VERIFY_FS;
  const ef alpha = rd.sample();
  if (!rd.pow(batching_pow_bits(s.security_bits, n))) return VERIFY_FS;
  std::vector<ef> zc(n - k + 1);
  for (auto& x : zc) x = rd.sample();

  // zerocheck with univariate skip: degree (constraint degree + 1) per variable
  std::vector<int> deg{d1 * (nsk - 1)}, set{nsk};
  for (int i = 0; i < n - k; i++) deg.push_back(d1), set.push_back(2);
  Claim outer;
  rd.phase("zerocheck");
  if (!sumcheck_rounds(rd, deg, set, s.security_bits, outer)) return VERIFY_SUMCHECK;
  if (!kb::ef_is_zero(outer.sum)) return VERIFY_SUM_MISMATCH;

  std::vector<ef> up(W), down(W);
  rd.phase("inner_sums");
  if (!rd.ext(up.data(), W) || !rd.ext(down.data(), W)) return VERIFY_FS;
  const auto& sel = lagrange_basis_cached(nsk);
  std::vector<ef> outer_sel(nsk);
  ef sel_dot = kb::ef_zero();
  for (int i = 0; i < nsk; i++) {
    outer_sel[i] = upoly_eval(sel[i], outer.point[0]);
    sel_dot = kb::ef_add(sel_dot, kb::ef_mul(upoly_eval(sel[i], zc[0]), outer_sel[i]));
  }
  std::vector<ef> alphas(NC);
  alphas[0] = kb::ef_one();
  for (int i = 1; i < NC; i++) alphas[i] = kb::ef_mul(alphas[i - 1], alpha);
  ef constraints;
  if (prog) {
    // the preprocessed columns' up / down versions folded over the skipped variables at the
    // outer challenge and evaluated at its tail (crates/air/src/verify.rs:119-135)
    const size_t N = size_t(1) << n, S = N >> k;
    const std::vector<ef> otail(outer.point.begin() + 1, outer.point.end());
    std::vector<ef> gup(P + W), gdown(P + W);
    for (int c = 0; c < P; c++) {
      const uint32_t* col = prog->pre.data() + size_t(c) * N;
      for (int half = 0; half < 2; half++) {
        std::vector<ef> f(S);
        for (size_t x = 0; x < S; x++) {
          ef acc = kb::ef_zero();
          for (int j = 0; j < nsk; j++) {
            const size_t r = size_t(j) * S + x;
            const size_t src = half == 0 ? (r == N - 1 ? N - 2 : r) : (r == N - 1 ? r : r + 1);
            acc = kb::ef_add(acc, kb::ef_mul_f(outer_sel[j], col[src]));
          }
          f[x] = acc;
        }
        (half == 0 ? gup : gdown)[c] = mle_eval(f, otail);
      }
    }
    for (int c = 0; c < W; c++) gup[P + c] = up[c], gdown[P + c] = down[c];
    constraints = prog->eval_ef(gup.data(), gdown.data(), alphas.data());
  } else {
    constraints = air_eval_ef(air, alphas.data(), [&](int c) { return up[c]; });
  }
  const std::vector<ef> zc_tail(zc.begin() + 1, zc.end()), outer_tail(outer.point.begin() + 1, outer.point.end());
  if (!kb::ef_eq(kb::ef_mul(kb::ef_mul(sel_dot, eq_eval(zc_tail, outer_tail)), constraints), outer.value))
    return VERIFY_SUM_MISMATCH;

  // column batching and the up/down combination
  if (!rd.pow(batching_pow_bits(s.security_bits, log2_up(W)))) return VERIFY_FS;
  std::vector<ef> cbs(LOGW);
  for (auto& x : cbs) x = rd.sample();
  const ef alpha2 = rd.sample();
  std::vector<ef> sub(nsk);
  if (!rd.ext(sub.data(), sub.size())) return VERIFY_FS;
  const std::vector<ef> eqc = eq_table_host(cbs);
  ef lhs = kb::ef_zero(), su = kb::ef_zero(), sd = kb::ef_zero();
  for (int i = 0; i < nsk; i++) lhs = kb::ef_add(lhs, kb::ef_mul(sub[i], outer_sel[i]));
  for (int c = 0; c < W; c++) {
    su = kb::ef_add(su, kb::ef_mul(up[c], eqc[c]));
    sd = kb::ef_add(sd, kb::ef_mul(down[c], eqc[c]));
  }
  if (!kb::ef_eq(lhs, kb::ef_add(su, kb::ef_mul(sd, alpha2)))) return VERIFY_SUM_MISMATCH;
  std::vector<ef> eps(k);
  for (auto& x : eps) x = rd.sample();

  // inner product sumcheck over the n row variables, degree 2
  Claim inner;
  rd.phase("inner_sumcheck");
  if (!sumcheck_rounds(rd, std::vector<int>(n, 2), std::vector<int>(n, 2), s.security_bits, inner))
    return VERIFY_SUMCHECK;
  if (!kb::ef_eq(inner.sum, mle_eval(sub, eps))) return VERIFY_SUM_MISMATCH;
  std::vector<ef> lde_pt = eps;
  lde_pt.insert(lde_pt.end(), outer_tail.begin(), outer_tail.end());
  lde_pt.insert(lde_pt.end(), inner.point.begin(), inner.point.end());
  const ef denom = kb::ef_add(matrix_up(lde_pt), kb::ef_mul(alpha2, matrix_down(lde_pt)));
  if (kb::ef_is_zero(denom)) return VERIFY_SUM_MISMATCH;
  const ef expected = kb::ef_mul(inner.value, kb::ef_inv(denom));

  // the WHIR opening of the packed witness at (column batching point, inner point)
  std::vector<ef> final_point = cbs;
  final_point.insert(final_point.end(), inner.point.begin(), inner.point.end());
  ood_pts.push_back(final_point);
  ood_vals.push_back(expected);
  if (!whir.verify(root, ood_pts, ood_vals)) return VERIFY_PCS_OPENING;
  if (rd.pos != rd.len) return VERIFY_FS;  // trailing words
  return VERIFY_OK;
}

int verify_abc_proof(const kb::P16Consts& p16, int n, int k, const uint32_t* proof, size_t proof_len) {
  const int nsk = 1 << k;
  ProofReader rd(&p16, proof, proof_len);
  std::vector<ef> r(n + 1 - k);
  for (auto& x : r) x = rd.sample();
  std::vector<int> deg{3 * (nsk - 1)}, set{nsk};
  for (int i = 0; i < n - k; i++) deg.push_back(3), set.push_back(2);
  Claim cl;
  if (!sumcheck_rounds(rd, deg, set, 128, cl)) return VERIFY_SUMCHECK;
  if (!kb::ef_is_zero(cl.sum)) return VERIFY_SUM_MISMATCH;
  ef fin[3];
  if (!rd.ext(fin, 3)) return VERIFY_FS;
  const auto& sel = lagrange_basis_cached(nsk);
  ef sel_dot = kb::ef_zero();
  for (int i = 0; i < nsk; i++)
    sel_dot = kb::ef_add(sel_dot, kb::ef_mul(upoly_eval(sel[i], r[0]), upoly_eval(sel[i], cl.point[0])));
  const std::vector<ef> rt(r.begin() + 1, r.end()), ct(cl.point.begin() + 1, cl.point.end());
  const ef abc = kb::ef_sub(kb::ef_mul(fin[0], fin[1]), fin[2]);
  if (!kb::ef_eq(kb::ef_mul(kb::ef_mul(sel_dot, eq_eval(rt, ct)), abc), cl.value)) return VERIFY_SUM_MISMATCH;
  if (rd.pos != rd.len) return VERIFY_FS;
  return VERIFY_OK;
}

}  // namespace wl
