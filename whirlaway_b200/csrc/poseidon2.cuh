// Poseidon2 over KoalaBear for widths 16 and 24 (S-box x^3, 8 full rounds, 20 / 23
// partial rounds), host and device. Replaces Plonky3's Poseidon2KoalaBear<16/24>
// (reference: src/examples/poseidon2.rs:22-26,148-151) and the linear layers of
// GenericPoseidon2LinearLayersKoalaBear used by the AIR.
//
// External layer: circ(2*M4, M4, ..., M4), M4 = [[2,3,1,1],[1,2,3,1],[1,1,2,3],[3,1,1,2]].
// Internal layer: J + diag(V) (state_i <- V_i * state_i + sum(state)).
// Round constants are runtime data (drawn from the workload's StdRng stream) and are
// kept in Montgomery form.
#pragma once
#include <cmath>
#include <cstring>

#include "kb.cuh"

namespace kb {

namespace detail {
constexpr uint64_t cpow(uint64_t a, uint64_t e) {
  uint64_t r = 1;
  a %= P;
  while (e) {
    if (e & 1) r = r * a % P;
    a = a * a % P;
    e >>= 1;
  }
  return r;
}
constexpr uint32_t cm(int64_t x) {  // Montgomery form of a signed small constant
  uint64_t v = uint64_t(((x % int64_t(P)) + int64_t(P)) % int64_t(P));
  return uint32_t((v << 32) % P);
}
constexpr uint32_t cm_inv2(int k, bool negative) {  // Montgomery form of +-1/2^k
  uint64_t v = cpow(cpow(2, k), P - 2);
  if (negative) v = (P - v) % P;
  return uint32_t((v << 32) % P);
}
}  // namespace detail

// Internal-layer diagonals V (Montgomery form); the internal matrix is J + diag(V).
//   width 16: [-2, 1, 2, 1/2, 3, 4, -1/2, -3, -4, 1/2^8, 1/8, 1/2^24, -1/2^8, -1/8, -1/16, -1/2^24]
//   width 24: [-2, 1, 2, 1/2, 3, 4, -1/2, -3, -4, 1/2^8, 1/4, 1/8, 1/16, 1/32, 1/64, 1/2^24,
//              -1/2^8, -1/8, -1/16, -1/32, -1/64, -1/2^7, -1/2^9, -1/2^24]
template <int W>
KB_HD constexpr uint32_t p2_diag(int i) {
  using detail::cm;
  using detail::cm_inv2;
  switch (i) {
    case 0: return cm(-2);
    case 1: return cm(1);
    case 2: return cm(2);
    case 3: return cm_inv2(1, false);
    case 4: return cm(3);
    case 5: return cm(4);
    case 6: return cm_inv2(1, true);
    case 7: return cm(-3);
    case 8: return cm(-4);
    case 9: return cm_inv2(8, false);
    default: break;
  }
  if (W == 16) {
    switch (i) {
      case 10: return cm_inv2(3, false);
      case 11: return cm_inv2(24, false);
      case 12: return cm_inv2(8, true);
      case 13: return cm_inv2(3, true);
      case 14: return cm_inv2(4, true);
      default: return cm_inv2(24, true);
    }
  }
  switch (i) {
    case 10: return cm_inv2(2, false);
    case 11: return cm_inv2(3, false);
    case 12: return cm_inv2(4, false);
    case 13: return cm_inv2(5, false);
    case 14: return cm_inv2(6, false);
    case 15: return cm_inv2(24, false);
    case 16: return cm_inv2(8, true);
    case 17: return cm_inv2(3, true);
    case 18: return cm_inv2(4, true);
    case 19: return cm_inv2(5, true);
    case 20: return cm_inv2(6, true);
    case 21: return cm_inv2(7, true);
    case 22: return cm_inv2(9, true);
    default: return cm_inv2(24, true);
  }
}

// Sign of the diagonal entry V_i.
template <int W>
KB_HD constexpr bool p2_diag_neg(int i) {
  if (i == 0 || i == 6 || i == 7 || i == 8) return true;
  return W == 16 ? i >= 12 : i >= 16;
}

// |V_i| * x using doublings, halvings and shifted reductions instead of a general product.
template <int W>
KB_HD uint32_t p2_diag_mag(int i, uint32_t x) {
  switch (i) {
    case 0: return dbl(x);
    case 1: return x;
    case 2: return dbl(x);
    case 3: return halve(x);
    case 4: return add(dbl(x), x);
    case 5: return dbl(dbl(x));
    case 6: return halve(x);
    case 7: return add(dbl(x), x);
    case 8: return dbl(dbl(x));
    case 9: return mul_inv_pow2(x, 8);
    default: break;
  }
  if (W == 16) {
    switch (i) {
      case 10: return mul_inv_pow2(x, 3);
      case 11: return mul_inv_pow2(x, 24);
      case 12: return mul_inv_pow2(x, 8);
      case 13: return mul_inv_pow2(x, 3);
      case 14: return mul_inv_pow2(x, 4);
      default: return mul_inv_pow2(x, 24);
    }
  }
  switch (i) {
    case 10: return mul_inv_pow2(x, 2);
    case 11: return mul_inv_pow2(x, 3);
    case 12: return mul_inv_pow2(x, 4);
    case 13: return mul_inv_pow2(x, 5);
    case 14: return mul_inv_pow2(x, 6);
    case 15: return mul_inv_pow2(x, 24);
    case 16: return mul_inv_pow2(x, 8);
    case 17: return mul_inv_pow2(x, 3);
    case 18: return mul_inv_pow2(x, 4);
    case 19: return mul_inv_pow2(x, 5);
    case 20: return mul_inv_pow2(x, 6);
    case 21: return mul_inv_pow2(x, 7);
    case 22: return mul_inv_pow2(x, 9);
    default: return mul_inv_pow2(x, 24);
  }
}

// V_i * x; equal to mul(x, p2_diag<W>(i)).
template <int W>
KB_HD uint32_t p2_diag_mul(int i, uint32_t x) {
  const uint32_t m = p2_diag_mag<W>(i, x);
  return p2_diag_neg<W>(i) ? neg(m) : m;
}

// V_i * x + sum, subtracting |V_i| x for the negative entries (no separate negation).
template <int W>
KB_HD uint32_t p2_diag_mul_add(int i, uint32_t x, uint32_t sum) {
  const uint32_t m = p2_diag_mag<W>(i, x);
  return p2_diag_neg<W>(i) ? sub(sum, m) : add(m, sum);
}

template <int W>
struct P2Consts {
  static constexpr int RP = W == 16 ? 20 : 23;
  uint32_t ext_init[4 * W];
  uint32_t ext_term[4 * W];
  uint32_t internal[RP];
};
using P16Consts = P2Consts<16>;
using P24Consts = P2Consts<24>;

// Pairwise (depth log2 N) sum; the modular additions do not reassociate on their own.
template <int N>
KB_HD uint32_t tree_sum(const uint32_t* v) {
  if constexpr (N == 1) {
    return v[0];
  } else {
    return add(tree_sum<N / 2>(v), tree_sum<N - N / 2>(v + N / 2));
  }
}

template <int W>
KB_HD void mds_light(uint32_t* s) {
#pragma unroll
  for (int c = 0; c < W; c += 4) {
    uint32_t x0 = s[c], x1 = s[c + 1], x2 = s[c + 2], x3 = s[c + 3];
    uint32_t t01 = add(x0, x1), t23 = add(x2, x3), t0123 = add(t01, t23);
    uint32_t t01123 = add(t0123, x1), t01233 = add(t0123, x3);
    s[c + 3] = add(t01233, dbl(x0));
    s[c + 1] = add(t01123, dbl(x2));
    s[c + 0] = add(t01123, t01);
    s[c + 2] = add(t01233, t23);
  }
  uint32_t sums[4];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    uint32_t v[W / 4];
#pragma unroll
    for (int j = 0; j < W / 4; j++) v[j] = s[4 * j + k];
    sums[k] = tree_sum<W / 4>(v);
  }
#pragma unroll
  for (int i = 0; i < W; i++) s[i] = add(s[i], sums[i & 3]);
}

// (v[0] + ... + v[N-1] + x0) mod p for values < p: pairs are added without carry (each pair
// is below 2^32), the pair sums in 64 bits (below 2^36), then the total is folded with
// 2^32 = 2^25 - 2 and 2^31 = 2^24 - 1 (mod p) to below 2p and reduced once.
template <int N>
KB_HD uint32_t sum_mod(const uint32_t* v, uint32_t x0) {
  uint64_t a = x0;
#pragma unroll
  for (int i = 0; i + 1 < N; i += 2) a += uint32_t(v[i] + v[i + 1]);
  if (N & 1) a += v[N - 1];
  const uint64_t b = uint64_t(uint32_t(a)) + uint64_t(uint32_t(a >> 32)) * ((1u << 25) - 2);  // < 2^33
  const uint32_t c = (uint32_t(b) & 0x7fffffffu) + uint32_t(b >> 31) * ((1u << 24) - 1);        // < 2p
  return umin(c, c - P);
}

// Internal layer applied to the state with s[0] replaced by x0 (the S-box output of a
// partial round); the sum of the other lanes does not wait for the S-box.
template <int W>
KB_HD void internal_layer_with0(uint32_t* s, uint32_t x0) {
  const uint32_t sum = sum_mod<W - 1>(s + 1, x0);
  s[0] = p2_diag_mul_add<W>(0, x0, sum);
#pragma unroll
  for (int i = 1; i < W; i++) s[i] = p2_diag_mul_add<W>(i, s[i], sum);
}
template <int W>
KB_HD void internal_layer(uint32_t* s) {
  internal_layer_with0<W>(s, s[0]);
}

template <int W>
KB_HD void p2_permute(uint32_t* s, const P2Consts<W>& c) {
  mds_light<W>(s);
#pragma unroll 1
  for (int r = 0; r < 4; r++) {
#pragma unroll
    for (int i = 0; i < W; i++) s[i] = cube(add(s[i], c.ext_init[r * W + i]));
    mds_light<W>(s);
  }
#pragma unroll 1
  for (int r = 0; r < P2Consts<W>::RP; r++) internal_layer_with0<W>(s, cube(add(s[0], c.internal[r])));
#pragma unroll 1
  for (int r = 0; r < 4; r++) {
#pragma unroll
    for (int i = 0; i < W; i++) s[i] = cube(add(s[i], c.ext_term[r * W + i]));
    mds_light<W>(s);
  }
}

// ---------------------------------------------------------------- canonical-domain S-box
// The Merkle hashes run in the canonical (non-Montgomery) domain with an S-box whose two
// products take their quotients by p from the fp64 pipe, which the integer kernels leave
// idle, instead of two Montgomery reductions (four high-word integer products) on the
// integer multiply pipe. For a product t = a b with |a|, |b| < 2^32 and |t| < 2^64, the
// fp64 product fl(a b) is within 2^11 of t and fl(1/p) within 2^-84 of 1/p, so
// fl(a b) fl(1/p) is within 2^-19 of t / p; one fused multiply-add that also adds
// 1.5 * 2^52 rounds it to an integer held in the low mantissa bits: q = floor(t / p) or one
// more. t - q p, formed exactly in 32-bit arithmetic (only its low word is needed), lies in
// [-p, p). The linear layers are the same in either domain.
constexpr double FQ_INV_P = 1.0 / 2130706433.0;
constexpr double FQ_ROUND = 6755399441055744.0;  // 1.5 * 2^52

// u as an fp64 value (exact).
KB_HD double fq_from_u32(uint32_t u) {
#ifdef __CUDA_ARCH__
  return __hiloint2double(0x43300000, int(u)) - 4503599627370496.0;  // (2^52 + u) - 2^52
#else
  return double(u);
#endif
}
// r read as a signed 32-bit value, as an fp64 value (exact).
KB_HD double fq_from_i32(uint32_t r) {
#ifdef __CUDA_ARCH__
  return __hiloint2double(0x43300000, int(r ^ 0x80000000u)) - 4503601774854144.0;  // - (2^52 + 2^31)
#else
  return double(int32_t(r));
#endif
}
// Low word of the rounded quotient prod / p (|prod / p| < 2^51).
KB_HD uint32_t fq_quot(double prod) {
#ifdef __CUDA_ARCH__
  return uint32_t(__double2loint(fma(prod, FQ_INV_P, FQ_ROUND)));
#else
  const double y = std::fma(prod, FQ_INV_P, FQ_ROUND);
  uint64_t bits;
  std::memcpy(&bits, &y, sizeof bits);
  return uint32_t(bits);
#endif
}
// u^3 mod p for u < 2p (an unreduced sum of two canonical values), canonical.
KB_HD uint32_t cube_fq(uint32_t u) {
  const double du = fq_from_u32(u);
  const uint32_t r = u * u - fq_quot(du * du) * P;               // u^2 mod p, in [-p, p)
  const uint32_t r3 = r * u - fq_quot(fq_from_i32(r) * du) * P;  // |r u| < 2 p^2
  return umin(r3, r3 + P);
}

// k of the diagonal entries +-2^-k (entries 9.., both widths).
template <int W>
KB_HD constexpr int p2_diag_k(int i) {
  constexpr int k16[16] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 8, 3, 24, 8, 3, 4, 24};
  constexpr int k24[24] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 8, 2, 3, 4, 5, 6, 24, 8, 3, 4, 5, 6, 7, 9, 24};
  return W == 16 ? k16[i] : k24[i];
}

// Internal layer with lazily reduced words. Words 0..8 (multipliers -2, 1, 2, 1/2, 3, 4, -1/2,
// -3, -4, applied by doublings and halvings) are canonical on entry and exit. Words 9.. (the
// multipliers +-2^-k, 2 <= k <= 24) may enter with any value below 2^32 and leave below 2^32:
// x 2^-k = (x >> k) - (x mod 2^k)(p - 1)/2^k (mod p) holds for every x, and its canonical
// form is umin(r, r + p) because r < 2^(32-k) <= p. The sum is reduced once, from 64 bits.
//  * positive, k >= 8: hi + sum + p - lo c in (0, 2p + 2^24), no reduction at all;
//  * positive, k < 8: r + sum in [0, 2p);  negative: sum + p - r in (0, 2p).
template <int W>
KB_HD void internal_layer_lazy_with0(uint32_t* s, uint32_t x0) {
  // canonical words pair up without carry (each pair below 2p < 2^32)
  uint64_t a = uint64_t(x0 + s[1]) + uint32_t(s[2] + s[3]) + uint32_t(s[4] + s[5]) + uint32_t(s[6] + s[7]) + s[8];
#pragma unroll
  for (int i = 9; i < W; i++) a += s[i];  // below 2^37
  const uint64_t b = uint64_t(uint32_t(a)) + uint64_t(uint32_t(a >> 32)) * ((1u << 25) - 2);  // < 2^33
  uint32_t sum = (uint32_t(b) & 0x7fffffffu) + uint32_t(b >> 31) * ((1u << 24) - 1);         // < 2p
  sum = umin(sum, sum - P);
  s[0] = p2_diag_mul_add<W>(0, x0, sum);
#pragma unroll
  for (int i = 1; i < 9; i++) s[i] = p2_diag_mul_add<W>(i, s[i], sum);
#pragma unroll
  for (int i = 9; i < W; i++) {
    const int k = p2_diag_k<W>(i);
    const uint32_t x = s[i], hi = x >> k, lo = x & ((1u << k) - 1), cst = (P - 1) >> k;
    if (!p2_diag_neg<W>(i) && k >= 8) {
      s[i] = hi + sum + P - lo * cst;
    } else {
      uint32_t r = hi - lo * cst;
      r = umin(r, r + P);
      s[i] = p2_diag_neg<W>(i) ? sum + P - r : sum + r;
    }
  }
}
// Canonical form of the lazy words after the last internal round (below 2p + 2^24).
template <int W>
KB_HD void internal_lazy_finish(uint32_t* s) {
#pragma unroll
  for (int i = 9; i < W; i++) {
    uint32_t x = umin(s[i], s[i] - P);
    if (!p2_diag_neg<W>(i) && p2_diag_k<W>(i) >= 8) x = umin(x, x - P);
    s[i] = x;
  }
}

// Canonical round constants (the canonical-domain S-box and lane kernels).
template <int W>
inline P2Consts<W> p2_consts_canonical(const P2Consts<W>& m) {
  P2Consts<W> c;
  for (int i = 0; i < 4 * W; i++) c.ext_init[i] = from_mont(m.ext_init[i]), c.ext_term[i] = from_mont(m.ext_term[i]);
  for (int i = 0; i < P2Consts<W>::RP; i++) c.internal[i] = from_mont(m.internal[i]);
  return c;
}

// ---------------------------------------------------------------- fp64 full rounds
// The full rounds can hold the state as fp64 values that are exact integers. The external
// linear layer is then nine additions per four words plus the column sums, with no reduction:
// its rows sum to 49, so inputs below 2^32 in magnitude give outputs below 2^38, far inside
// the 53-bit mantissa. The S-box takes such a value z unreduced: fl(z^2) is within 2^23 of z^2
// (z^2 < 2^76), so fq_quot(z * z) = round(z^2 / p) up to an error below 2^-7 and z^2 - q p
// lies in (-p, p); it is formed from low words, z mod 2^32 being the low word of
// z + 1.5 * 2^52. The second product r z (|r| < p) likewise. The cube is left as a signed
// residue in (-p, p), which the next linear layer takes as it is. The partial rounds run on
// 32-bit words with the canonical-domain S-box and the lazy internal layer (which multiplies
// by 2^-k, which fp64 cannot hold exactly). Round constants are fp64 copies of the canonical
// ones.
template <int W>
struct P2ConstsFd {
  static constexpr int RP = P2Consts<W>::RP;
  double ext_init[4 * W];
  double ext_term[4 * W];
  uint32_t internal[RP];
};
template <int W>
inline P2ConstsFd<W> p2_consts_fd(const P2Consts<W>& m) {
  P2ConstsFd<W> c;
  for (int i = 0; i < 4 * W; i++) c.ext_init[i] = double(from_mont(m.ext_init[i])), c.ext_term[i] = double(from_mont(m.ext_term[i]));
  for (int i = 0; i < P2Consts<W>::RP; i++) c.internal[i] = from_mont(m.internal[i]);
  return c;
}

// z mod 2^32 for an integer-valued z with |z| < 2^51.
KB_HD uint32_t fd_low(double z) {
#ifdef __CUDA_ARCH__
  return uint32_t(__double2loint(z + FQ_ROUND));
#else
  const double y = z + FQ_ROUND;
  uint64_t bits;
  std::memcpy(&bits, &y, sizeof bits);
  return uint32_t(bits);
#endif
}
// z^3 mod p as a signed residue in (-p, p), for an integer-valued z with |z| < 2^38.
KB_HD double sbox_fd(double z) {
  const uint32_t zi = fd_low(z);
  const uint32_t r2 = zi * zi - fq_quot(z * z) * P;  // z^2 mod p in (-p, p)
  const double r2d = fq_from_i32(r2);
  const uint32_t r3 = r2 * zi - fq_quot(r2d * z) * P;  // z^3 mod p in (-p, p)
  return fq_from_i32(r3);
}
// The canonical residue of an integer-valued z with |z| < 2^38: z - round(z / p) p lies in
// [-p/2, p/2], and umin maps its negative values to r + p.
KB_HD uint32_t fd_canonical(double z) {
  const uint32_t r = fd_low(z) - fq_quot(z) * P;
  return umin(r, r + P);
}

template <int W>
KB_HD void mds_light_fd(double* s) {
#pragma unroll
  for (int c = 0; c < W; c += 4) {
    const double x0 = s[c], x1 = s[c + 1], x2 = s[c + 2], x3 = s[c + 3];
    const double t01 = x0 + x1, t23 = x2 + x3, t0123 = t01 + t23;
    const double t01123 = t0123 + x1, t01233 = t0123 + x3;
    s[c + 3] = t01233 + 2.0 * x0;
    s[c + 1] = t01123 + 2.0 * x2;
    s[c + 0] = t01123 + t01;
    s[c + 2] = t01233 + t23;
  }
  double sums[4];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    double a = s[k] + s[4 + k];
#pragma unroll
    for (int j = 2; j < W / 4; j++) a += s[4 * j + k];
    sums[k] = a;
  }
#pragma unroll
  for (int i = 0; i < W; i++) s[i] += sums[i & 3];
}

// The permutation on canonical values (the map p2_permute computes on Montgomery forms),
// full rounds in fp64.
template <int W>
KB_HD void p2_permute_fd(uint32_t* s, const P2ConstsFd<W>& c) {
  double d[W];
#pragma unroll
  for (int i = 0; i < W; i++) d[i] = fq_from_u32(s[i]);
  mds_light_fd<W>(d);
#pragma unroll 1
  for (int r = 0; r < 4; r++) {
#pragma unroll
    for (int i = 0; i < W; i++) d[i] = sbox_fd(d[i] + c.ext_init[r * W + i]);
    mds_light_fd<W>(d);
  }
#pragma unroll
  for (int i = 0; i < W; i++) s[i] = fd_canonical(d[i]);
#pragma unroll 1
  for (int r = 0; r < P2ConstsFd<W>::RP; r++) internal_layer_lazy_with0<W>(s, cube_fq(s[0] + c.internal[r]));
  // words 9.. leave the lazy layer below 2p + 2^24 < 2^32: exact as fp64 without reduction
#pragma unroll
  for (int i = 0; i < W; i++) d[i] = fq_from_u32(s[i]);
#pragma unroll 1
  for (int r = 0; r < 4; r++) {
#pragma unroll
    for (int i = 0; i < W; i++) d[i] = sbox_fd(d[i] + c.ext_term[r * W + i]);
    mds_light_fd<W>(d);
  }
#pragma unroll
  for (int i = 0; i < W; i++) s[i] = fd_canonical(d[i]);
}

// Extension-field versions of the linear layers (constraint evaluation over EF).
KB_HD void mds_light_ef16(ef* s) {
#pragma unroll
  for (int c = 0; c < 16; c += 4) {
    ef x0 = s[c], x1 = s[c + 1], x2 = s[c + 2], x3 = s[c + 3];
    ef t01 = ef_add(x0, x1), t23 = ef_add(x2, x3), t0123 = ef_add(t01, t23);
    ef t01123 = ef_add(t0123, x1), t01233 = ef_add(t0123, x3);
    s[c + 3] = ef_add(t01233, ef_add(x0, x0));
    s[c + 1] = ef_add(t01123, ef_add(x2, x2));
    s[c + 0] = ef_add(t01123, t01);
    s[c + 2] = ef_add(t01233, t23);
  }
#pragma unroll
  for (int k = 0; k < 4; k++) {
    ef sk = ef_add(ef_add(s[k], s[4 + k]), ef_add(s[8 + k], s[12 + k]));
#pragma unroll
    for (int j = k; j < 16; j += 4) s[j] = ef_add(s[j], sk);
  }
}
KB_HD void internal_layer_ef16(ef* s) {
  ef sum = s[0];
#pragma unroll
  for (int i = 1; i < 16; i++) sum = ef_add(sum, s[i]);
#pragma unroll
  for (int i = 0; i < 16; i++) s[i] = ef_add(ef_mul_f(s[i], p2_diag<16>(i)), sum);
}

}  // namespace kb
