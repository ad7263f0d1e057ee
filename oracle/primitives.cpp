// CPU oracle (test infrastructure): field, extension field, StdRng, Poseidon2,
// sponge / compression, duplex challenger, transcript and polynomial helpers.
// See oracle.h for the scope and the parity status.
#include <omp.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <stdexcept>

#include "oracle.h"

namespace wlo {

// ============================================================== field
F fpow(F a, uint64_t e) {
  F r(1);
  while (e) {
    if (e & 1) r *= a;
    a *= a;
    e >>= 1;
  }
  return r;
}
F finv(F a) {
  if (a.v == 0) throw std::runtime_error("inverse of zero");
  return fpow(a, P - 2);
}
// KoalaBear's multiplicative group is generated by 3 and p - 1 = 2^24 * 127, so
// 3^(127 * 2^(24 - k)) generates the subgroup of order 2^k.
F two_adic_generator(int log_size) {
  if (log_size < 0 || log_size > 24) throw std::runtime_error("two-adicity exceeded");
  return fpow(F(3), uint64_t(127) << (24 - log_size));
}

EF operator*(const EF& a, const EF& b) {
  uint64_t acc[15] = {0};
  for (int i = 0; i < 8; i++)
    for (int j = 0; j < 8; j++) acc[i + j] += (a.c[i] * b.c[j]).v;
  EF r;
  for (int i = 0; i < 8; i++) {
    uint64_t hi = i + 8 < 15 ? acc[i + 8] % P : 0;
    r.c[i] = F(acc[i] + EXT_W * hi);
  }
  return r;
}

// a^(p^8 - 2) by square-and-multiply over the 248-bit exponent.
EF efinv(const EF& a) {
  if (a.is_zero()) throw std::runtime_error("inverse of zero (EF)");
  uint32_t e[9] = {1, 0, 0, 0, 0, 0, 0, 0, 0};  // little-endian limbs of p^8
  for (int k = 0; k < 8; k++) {
    uint64_t carry = 0;
    for (int i = 0; i < 9; i++) {
      uint64_t t = (uint64_t)e[i] * P + carry;
      e[i] = uint32_t(t);
      carry = t >> 32;
    }
  }
  // subtract 2
  uint64_t borrow = 2;
  for (int i = 0; i < 9 && borrow; i++) {
    uint64_t cur = e[i];
    if (cur >= borrow) { e[i] = uint32_t(cur - borrow); borrow = 0; }
    else { e[i] = uint32_t(cur + (1ull << 32) - borrow); borrow = 1; }
  }
  EF r = ef_one(), base = a;
  for (int i = 0; i < 9; i++)
    for (int b = 0; b < 32; b++) {
      if ((e[i] >> b) & 1) r = r * base;
      base = base * base;
    }
  return r;
}

// ============================================================== ChaCha / StdRng
static inline uint32_t rotl(uint32_t x, int k) { return (x << k) | (x >> (32 - k)); }
#define QR(a, b, c, d)           \
  a += b; d ^= a; d = rotl(d, 16); \
  c += d; b ^= c; b = rotl(b, 12); \
  a += b; d ^= a; d = rotl(d, 8);  \
  c += d; b ^= c; b = rotl(b, 7);

void chacha_block(const uint32_t key[8], uint64_t counter, uint64_t stream, int rounds, uint32_t out[16]) {
  uint32_t s[16] = {0x61707865, 0x3320646e, 0x79622d32, 0x6b206574};
  for (int i = 0; i < 8; i++) s[4 + i] = key[i];
  s[12] = uint32_t(counter);
  s[13] = uint32_t(counter >> 32);
  s[14] = uint32_t(stream);
  s[15] = uint32_t(stream >> 32);
  uint32_t x[16];
  memcpy(x, s, sizeof x);
  for (int r = 0; r < rounds; r += 2) {
    QR(x[0], x[4], x[8], x[12]);
    QR(x[1], x[5], x[9], x[13]);
    QR(x[2], x[6], x[10], x[14]);
    QR(x[3], x[7], x[11], x[15]);
    QR(x[0], x[5], x[10], x[15]);
    QR(x[1], x[6], x[11], x[12]);
    QR(x[2], x[7], x[8], x[13]);
    QR(x[3], x[4], x[9], x[14]);
  }
  for (int i = 0; i < 16; i++) out[i] = x[i] + s[i];
}

// rand_core 0.9 SeedableRng::seed_from_u64: PCG32 fills the 32-byte seed.
StdRng::StdRng(uint64_t state) {
  const uint64_t MUL = 6364136223846793005ull, INC = 11634580456548416449ull;
  for (int i = 0; i < 8; i++) {
    state = state * MUL + INC;
    uint32_t xorshifted = uint32_t(((state >> 18) ^ state) >> 27);
    uint32_t rot = uint32_t(state >> 59);
    key[i] = (xorshifted >> rot) | (xorshifted << ((32 - rot) & 31));
  }
}
uint32_t StdRng::next_u32() {
  if (idx == 16) {
    chacha_block(key, counter++, 0, 12, buf);
    idx = 0;
  }
  return buf[idx++];
}
F StdRng::random_f() {
  // The sampled 31-bit word is a Montgomery representative (R = 2^32).
  static const F rinv = finv(F(uint64_t(1) << 32));
  for (;;) {
    uint32_t u = next_u32() >> 1;
    if (u < P) return F(u) * rinv;
  }
}

// ============================================================== Poseidon2
std::vector<F> internal_diag(int width) {
  auto h = [](int k) { return finv(fpow(F(2), k)); };
  F two(2), three(3), four(4), one(1);
  if (width == 16)
    return {-two, one, two, h(1), three, four, -h(1), -three, -four, h(8), h(3), h(24), -h(8), -h(3), -h(4), -h(24)};
  if (width == 24)
    return {-two, one,   two,   h(1),  three, four,  -h(1), -three, -four, h(8),  h(2),  h(3),
            h(4), h(5),  h(6),  h(24), -h(8), -h(3), -h(4), -h(5),  -h(6), -h(7), -h(9), -h(24)};
  throw std::runtime_error("unsupported Poseidon2 width");
}

template <class T>
void mds_light_t(T* s, int width) {
  // circ(2*M4, M4, ..., M4) with M4 = [[2,3,1,1],[1,2,3,1],[1,1,2,3],[3,1,1,2]]
  for (int c = 0; c < width; c += 4) {
    T x0 = s[c], x1 = s[c + 1], x2 = s[c + 2], x3 = s[c + 3];
    T t01 = x0 + x1, t23 = x2 + x3, t0123 = t01 + t23;
    T t01123 = t0123 + x1, t01233 = t0123 + x3;
    s[c + 3] = t01233 + x0 + x0;
    s[c + 1] = t01123 + x2 + x2;
    s[c + 0] = t01123 + t01;
    s[c + 2] = t01233 + t23;
  }
  T sums[4];
  for (int k = 0; k < 4; k++) {
    sums[k] = s[k];
    for (int j = 4 + k; j < width; j += 4) sums[k] = sums[k] + s[j];
  }
  for (int i = 0; i < width; i++) s[i] = s[i] + sums[i % 4];
}
template void mds_light_t<F>(F*, int);
template void mds_light_t<EF>(EF*, int);
void mds_light(F* s, int width) { mds_light_t<F>(s, width); }

template <class T>
void internal_layer_t(T* s, int width, const std::vector<F>& diag) {
  T sum = s[0];
  for (int i = 1; i < width; i++) sum = sum + s[i];
  for (int i = 0; i < width; i++) s[i] = s[i] * diag[i] + sum;
}
template void internal_layer_t<F>(F*, int, const std::vector<F>&);
template void internal_layer_t<EF>(EF*, int, const std::vector<F>&);

Poseidon2 Poseidon2::from_rng(int width, StdRng& rng) {
  Poseidon2 p;
  p.width = width;
  p.rounds_f = 8;
  p.rounds_p = width == 16 ? 20 : 23;
  int hf = p.rounds_f / 2;
  for (int i = 0; i < hf * width; i++) p.ext_init.push_back(rng.random_f());
  for (int i = 0; i < hf * width; i++) p.ext_term.push_back(rng.random_f());
  for (int i = 0; i < p.rounds_p; i++) p.internal.push_back(rng.random_f());
  p.diag = internal_diag(width);
  return p;
}

void Poseidon2::permute(F* s) const {
  int hf = rounds_f / 2;
  mds_light(s, width);
  for (int r = 0; r < hf; r++) {
    for (int i = 0; i < width; i++) s[i] = cube(s[i] + ext_init[r * width + i]);
    mds_light(s, width);
  }
  for (int r = 0; r < rounds_p; r++) {
    s[0] = cube(s[0] + internal[r]);
    internal_layer_t<F>(s, width, diag);
  }
  for (int r = 0; r < hf; r++) {
    for (int i = 0; i < width; i++) s[i] = cube(s[i] + ext_term[r * width + i]);
    mds_light(s, width);
  }
}

Digest sponge_hash(const Poseidon2& p24, const F* in, size_t len) {
  F st[24];
  size_t pos = 0;
  for (;;) {
    bool done = false;
    for (int i = 0; i < 16; i++) {
      if (pos < len) {
        st[i] = in[pos++];
      } else {
        if (i != 0) p24.permute(st);
        done = true;
        break;
      }
    }
    if (done) break;
    p24.permute(st);
  }
  Digest d;
  for (int i = 0; i < 8; i++) d[i] = st[i];
  return d;
}

Digest compress(const Poseidon2& p16, const Digest& l, const Digest& r) {
  F st[16];
  for (int i = 0; i < 8; i++) { st[i] = l[i]; st[8 + i] = r[i]; }
  p16.permute(st);
  Digest d;
  for (int i = 0; i < 8; i++) d[i] = st[i];
  return d;
}

// ============================================================== challenger
void Challenger::duplex() {
  for (size_t i = 0; i < in_buf.size(); i++) state[i] = in_buf[i];
  in_buf.clear();
  perm->permute(state);
  out_buf.assign(state, state + 8);
}
void Challenger::observe(F x) {
  out_buf.clear();
  in_buf.push_back(x);
  if (in_buf.size() == 8) duplex();
}
F Challenger::sample() {
  if (!in_buf.empty() || out_buf.empty()) duplex();
  F r = out_buf.back();
  out_buf.pop_back();
  return r;
}
uint32_t Challenger::sample_bits(int bits) { return sample().v & ((1u << bits) - 1); }
bool Challenger::check_witness(int bits, F w) const {
  Challenger c = *this;
  c.observe(w);
  return c.sample_bits(bits) == 0;
}

void Transcript::add_base(const F* v, size_t n) {
  for (size_t i = 0; i < n; i++) { proof.push_back(v[i]); ch.observe(v[i]); }
}
void Transcript::add_ext(const EF* v, size_t n) {
  for (size_t i = 0; i < n; i++) add_base(v[i].c, 8);
}
void Transcript::hint(const F* v, size_t n) { proof.insert(proof.end(), v, v + n); }
EF Transcript::sample_ext() {
  EF e;
  for (int i = 0; i < 8; i++) e.c[i] = ch.sample();
  return e;
}
// The smallest witness is taken so that the proof is deterministic.
void Transcript::grind(int bits) {
  if (bits == 0) return;
  const uint32_t block = 1u << 14;
  for (uint32_t base = 0; base < P; base += block) {
    uint32_t best = UINT32_MAX;
    uint32_t hi = std::min<uint64_t>(uint64_t(base) + block, P);
#pragma omp parallel for reduction(min : best) schedule(static)
    for (int64_t w = base; w < (int64_t)hi; w++)
      if (ch.check_witness(bits, F::raw(uint32_t(w))) && uint32_t(w) < best) best = uint32_t(w);
    if (best != UINT32_MAX) {
      ch.observe(F::raw(best));
      ch.sample_bits(bits);
      proof.push_back(F::raw(best));
      return;
    }
  }
  throw std::runtime_error("grinding failed");
}
bool Transcript::next_base(F* v, size_t n) {
  if (cursor + n > proof.size()) return false;
  for (size_t i = 0; i < n; i++) { v[i] = proof[cursor + i]; ch.observe(v[i]); }
  cursor += n;
  return true;
}
bool Transcript::next_ext(EF* v, size_t n) {
  for (size_t i = 0; i < n; i++)
    if (!next_base(v[i].c, 8)) return false;
  return true;
}
bool Transcript::next_hint(F* v, size_t n) {
  if (cursor + n > proof.size()) return false;
  for (size_t i = 0; i < n; i++) v[i] = proof[cursor + i];
  cursor += n;
  return true;
}
bool Transcript::check_grind(int bits) {
  if (bits == 0) return true;
  if (cursor + 1 > proof.size()) return false;
  F w = proof[cursor++];
  ch.observe(w);
  return ch.sample_bits(bits) == 0;
}

// ============================================================== polynomials
int log2_up(size_t x) {
  int r = 0;
  while ((size_t(1) << r) < x) r++;
  return r;
}

std::vector<EF> eval_eq(const std::vector<EF>& point) {
  std::vector<EF> t(1, ef_one());
  for (const EF& r : point) {
    std::vector<EF> n(t.size() * 2);
    EF one_minus = ef_one() - r;
    for (size_t j = 0; j < t.size(); j++) {
      n[2 * j] = t[j] * one_minus;
      n[2 * j + 1] = t[j] * r;
    }
    t.swap(n);
  }
  return t;
}

EF eq_poly(const std::vector<EF>& a, const std::vector<EF>& b) {
  if (a.size() != b.size()) throw std::runtime_error("eq_poly size mismatch");
  EF r = ef_one();
  for (size_t i = 0; i < a.size(); i++) r = r * (a[i] * b[i] + (ef_one() - a[i]) * (ef_one() - b[i]));
  return r;
}

EF mle_evaluate(const std::vector<EF>& evals, const std::vector<EF>& point) {
  std::vector<EF> cur = evals;
  for (const EF& r : point) {
    size_t h = cur.size() / 2;
    for (size_t i = 0; i < h; i++) cur[i] = cur[i] + r * (cur[i + h] - cur[i]);
    cur.resize(h);
  }
  return cur.at(0);
}

static std::vector<F> poly_mul_f(const std::vector<F>& a, const std::vector<F>& b) {
  std::vector<F> r(a.size() + b.size() - 1);
  for (size_t i = 0; i < a.size(); i++)
    for (size_t j = 0; j < b.size(); j++) r[i + j] += a[i] * b[j];
  return r;
}

std::vector<EF> poly_lagrange(const std::vector<std::pair<F, EF>>& pts) {
  size_t n = pts.size();
  std::vector<EF> out(n);
  for (size_t i = 0; i < n; i++) {
    std::vector<F> basis{F(1)};
    F denom(1);
    for (size_t j = 0; j < n; j++) {
      if (j == i) continue;
      basis = poly_mul_f(basis, {-pts[j].first, F(1)});
      denom *= pts[i].first - pts[j].first;
    }
    EF scale = pts[i].second * finv(denom);
    for (size_t k = 0; k < n; k++) out[k] += scale * basis[k];
  }
  return out;
}

std::vector<EF> poly_mul(const std::vector<EF>& a, const std::vector<EF>& b) {
  std::vector<EF> r(a.size() + b.size() - 1);
  for (size_t i = 0; i < a.size(); i++)
    for (size_t j = 0; j < b.size(); j++) r[i + j] += a[i] * b[j];
  return r;
}

EF poly_eval(const std::vector<EF>& c, const EF& x) {
  EF r;
  for (size_t i = c.size(); i-- > 0;) r = r * x + c[i];
  return r;
}
EF poly_eval_f(const std::vector<EF>& c, F x) {
  EF r;
  for (size_t i = c.size(); i-- > 0;) r = r * x + c[i];
  return r;
}
F upoly_eval(const std::vector<F>& c, F x) {
  F r;
  for (size_t i = c.size(); i-- > 0;) r = r * x + c[i];
  return r;
}
EF upoly_eval(const std::vector<F>& c, const EF& x) {
  EF r;
  for (size_t i = c.size(); i-- > 0;) r = r * x + c[i];
  return r;
}

std::vector<std::vector<F>> univariate_selectors(int skips) {
  int n = 1 << skips;
  std::vector<std::vector<F>> sel(n);
  for (int i = 0; i < n; i++) {
    std::vector<std::pair<F, EF>> pts;
    for (int j = 0; j < n; j++) pts.push_back({F(j), EF(F(i == j ? 1 : 0))});
    auto c = poly_lagrange(pts);
    for (auto& e : c) sel[i].push_back(e.c[0]);
  }
  return sel;
}

int sumcheck_pow_bits(int security_bits, int degree) {
  int ef_bits = 31 * EXT_D;
  int t = ef_bits - log2_up(size_t(degree) + 1);
  if (t < 0) t = 0;
  return security_bits > t ? security_bits - t : 0;
}

}  // namespace wlo
