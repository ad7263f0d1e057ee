// KoalaBear (p = 2^31 - 2^24 + 1) and its degree-8 binomial extension F[X]/(X^8 - 3),
// for host and device. Replaces Plonky3's p3-koala-bear / p3-monty-31 arithmetic and
// BinomialExtensionField<KoalaBear, 8> (reference: src/examples/poseidon2.rs:30-31).
//
// Device values are 32-bit Montgomery representatives (R = 2^32). Sums of products are
// accumulated lazily in 64 bits: four products of values < p stay below 4p^2 < 2^64 and
// are folded with a single Montgomery reduction, which roughly halves the instruction
// count of an extension-field product against one reduction per product.
#pragma once
#ifdef __CUDACC_RTC__
// runtime compilation (the generated constraint kernels): no host headers
typedef unsigned int uint32_t;
typedef unsigned long long uint64_t;
typedef int int32_t;
typedef long long int64_t;
typedef unsigned char uint8_t;
#else
#include <cstdint>
#endif

#ifdef __CUDACC__
#define KB_HD __host__ __device__ __forceinline__
#else
#define KB_HD inline
#endif

namespace kb {

constexpr uint32_t P = 0x7f000001u;
constexpr uint32_t PINV = 0x81000001u;  // p^-1 mod 2^32
constexpr uint32_t R_MOD_P = 0x01fffffeu;   // Montgomery form of 1
constexpr uint32_t R2_MOD_P = 0x17f7efe4u;  // 2^64 mod p
constexpr uint32_t FROB_GAMMA = 0x6832fe4au;  // 3^((p-1)/8), canonical

KB_HD uint32_t umulhi(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
  return __umulhi(a, b);
#else
  return uint32_t((uint64_t(a) * b) >> 32);
#endif
}

KB_HD uint32_t umin(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
  return ::min(a, b);
#else
  return a < b ? a : b;
#endif
}
// For a, b < p: a + b - p wraps above a + b exactly when a + b < p, so the unsigned
// minimum selects the reduced sum (and likewise for the difference).
KB_HD uint32_t add(uint32_t a, uint32_t b) {
  uint32_t r = a + b;
  return umin(r, r - P);
}
KB_HD uint32_t sub(uint32_t a, uint32_t b) {
  uint32_t r = a - b;
  return umin(r, r + P);
}
KB_HD uint32_t neg(uint32_t a) { return a ? P - a : 0; }
KB_HD uint32_t dbl(uint32_t a) { return add(a, a); }

// Montgomery product: a * b * 2^-32 mod p, inputs and output in [0, p).
KB_HD uint32_t mul(uint32_t a, uint32_t b) {
  uint32_t lo = a * b, hi = umulhi(a, b);
  uint32_t m = lo * PINV;
  uint32_t mh = umulhi(m, P);
  uint32_t r = hi - mh;
  return hi < mh ? r + P : r;  // measured faster than the unsigned-min form for products
}

// Montgomery reduction of a lazily accumulated sum t < 4p^2 (at most four products).
KB_HD uint32_t redc(uint64_t t) {
  uint32_t lo = uint32_t(t), hi = uint32_t(t >> 32);
  uint32_t m = lo * PINV;
  uint32_t mh = umulhi(m, P);
  uint32_t r = hi - mh;  // in (-p, 2p): 3p > 2^32, so the sign needs the comparison
  r = hi < mh ? r + P : r;
  return umin(r, r - P);
}
// x * 2^-k for 1 <= k <= 24, x < p (linear, so Montgomery form is preserved). With
// x = hi 2^k + lo and 2^24 | p - 1, 2^-k = -(p - 1) / 2^k (mod p), so the product is
// hi - lo (p - 1) / 2^k, which lies in (-(p - 1), 2^(31 - k)): one low-word multiply and a
// sign fix, no high-word product.
KB_HD uint32_t mul_inv_pow2(uint32_t x, int k) {
  const uint32_t r = (x >> k) - (x & ((1u << k) - 1)) * ((P - 1) >> k);
  return umin(r, r + P);
}
KB_HD uint32_t halve(uint32_t x) { return (x & 1) ? (x >> 1) + ((P + 1) >> 1) : (x >> 1); }
KB_HD uint64_t wmul(uint32_t a, uint32_t b) { return uint64_t(a) * b; }

KB_HD uint32_t to_mont(uint32_t x) { return mul(x % P, R2_MOD_P); }
KB_HD uint32_t from_mont(uint32_t x) { return mul(x, 1u); }
// Montgomery product left in (0, 2p) instead of [0, p): hi - mh lies in (-p, p/2) for
// a, b < p, so adding p replaces the sign fix. Only for feeding another product.
KB_HD uint32_t mul_lazy(uint32_t a, uint32_t b) {
  uint32_t lo = a * b, hi = umulhi(a, b);
  uint32_t m = lo * PINV;
  uint32_t mh = umulhi(m, P);
  return hi - mh + P;
}
// x^3 for x < p: (x^2 in (0, 2p)) * x < 2 p^2 keeps the second product's hi word below p.
KB_HD uint32_t cube(uint32_t x) { return mul(mul_lazy(x, x), x); }

inline uint32_t pow_m(uint32_t a, uint64_t e) {  // Montgomery in, Montgomery out
  uint32_t r = R_MOD_P;
  while (e) {
    if (e & 1) r = mul(r, a);
    a = mul(a, a);
    e >>= 1;
  }
  return r;
}
inline uint32_t inv_m(uint32_t a) { return pow_m(a, P - 2); }
// Montgomery form of the generator of the subgroup of order 2^log_size
// (3 generates F_p^*, and p - 1 = 2^24 * 127).
inline uint32_t two_adic_gen_m(int log_size) { return pow_m(to_mont(3), uint64_t(127) << (24 - log_size)); }

// ------------------------------------------------------------------ extension
struct ef {
  uint32_t c[8];
};

KB_HD ef ef_zero() {
  ef r;
#pragma unroll
  for (int i = 0; i < 8; i++) r.c[i] = 0;
  return r;
}
KB_HD ef ef_from(uint32_t a) {
  ef r = ef_zero();
  r.c[0] = a;
  return r;
}
KB_HD ef ef_one() { return ef_from(R_MOD_P); }
KB_HD ef ef_add(const ef& a, const ef& b) {
  ef r;
#pragma unroll
  for (int i = 0; i < 8; i++) r.c[i] = add(a.c[i], b.c[i]);
  return r;
}
KB_HD ef ef_sub(const ef& a, const ef& b) {
  ef r;
#pragma unroll
  for (int i = 0; i < 8; i++) r.c[i] = sub(a.c[i], b.c[i]);
  return r;
}
KB_HD ef ef_add_f(const ef& a, uint32_t b) {
  ef r = a;
  r.c[0] = add(r.c[0], b);
  return r;
}
KB_HD ef ef_sub_f(const ef& a, uint32_t b) {
  ef r = a;
  r.c[0] = sub(r.c[0], b);
  return r;
}
KB_HD ef ef_mul_f(const ef& a, uint32_t b) {
  ef r;
#pragma unroll
  for (int i = 0; i < 8; i++) r.c[i] = mul(a.c[i], b);
  return r;
}
KB_HD bool ef_eq(const ef& a, const ef& b) {
  bool e = true;
#pragma unroll
  for (int i = 0; i < 8; i++) e = e && a.c[i] == b.c[i];
  return e;
}
KB_HD bool ef_is_zero(const ef& a) { return ef_eq(a, ef_zero()); }

// Schoolbook product with X^8 = 3: coefficient k is the 8-term dot product of a with
// (b_k, ..., b_0, 3 b_7, ..., 3 b_{k+1}), reduced in two lazy halves of four terms.
KB_HD ef ef_mul(const ef& a, const ef& b) {
  uint32_t b3[8];
#pragma unroll
  for (int j = 0; j < 8; j++) b3[j] = add(dbl(b.c[j]), b.c[j]);
  ef r;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    uint64_t s0 = 0, s1 = 0;
#pragma unroll
    for (int t = 0; t < 4; t++) s0 += wmul(a.c[t], t <= k ? b.c[k - t] : b3[k + 8 - t]);
#pragma unroll
    for (int t = 4; t < 8; t++) s1 += wmul(a.c[t], t <= k ? b.c[k - t] : b3[k + 8 - t]);
    r.c[k] = add(redc(s0), redc(s1));
  }
  return r;
}
// Square with the 36 distinct products: coefficient k sums a_i a_j over i <= j with
// i + j = k (cross terms by 2 a_i) and, times 3, over i + j = k + 8 (cross terms by 6 a_i);
// the doubled and tripled operands are formed once. At most five products per coefficient,
// folded with 2^32 = 2^25 - 2 (mod p) after the fourth, then one Montgomery reduction.
KB_HD ef ef_sqr(const ef& a) {
  uint32_t d[8], t[8], s[8];
#pragma unroll
  for (int i = 0; i < 8; i++) {
    d[i] = dbl(a.c[i]);
    t[i] = add(d[i], a.c[i]);
    s[i] = dbl(t[i]);
  }
  ef r;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    uint64_t acc = 0;
    int n = 0;
#pragma unroll
    for (int i = 0; i <= k / 2; i++) {
      acc += wmul(i == k - i ? a.c[i] : d[i], a.c[k - i]);
      if (++n == 4) acc = uint64_t(uint32_t(acc >> 32)) * ((1u << 25) - 2) + uint32_t(acc);
    }
#pragma unroll
    for (int i = k + 1; i <= (k + 8) / 2; i++) {
      acc += wmul(i == k + 8 - i ? t[i] : s[i], a.c[k + 8 - i]);
      if (++n == 4) acc = uint64_t(uint32_t(acc >> 32)) * ((1u << 25) - 2) + uint32_t(acc);
    }
    r.c[k] = redc(acc);
  }
  return r;
}
KB_HD ef ef_cube(const ef& a) { return ef_mul(ef_sqr(a), a); }

// a + r * (b - a)
KB_HD ef ef_lerp(const ef& a, const ef& b, const ef& r) { return ef_add(a, ef_mul(r, ef_sub(b, a))); }

// Frobenius power a^(p^i): coefficient j picks up gamma^(i*j), gamma = 3^((p-1)/8).
inline ef ef_frobenius(const ef& a, int i) {
  uint32_t g = pow_m(to_mont(FROB_GAMMA), uint64_t(i));
  ef r;
  uint32_t gj = R_MOD_P;
  for (int j = 0; j < 8; j++) {
    r.c[j] = mul(a.c[j], gj);
    gj = mul(gj, g);
  }
  return r;
}
// a^-1 = (a^p * a^p^2 * ... * a^p^7) / N(a), with the norm N(a) in the base field.
inline ef ef_inv(const ef& a) {
  ef prod = ef_frobenius(a, 1);
  for (int i = 2; i < 8; i++) prod = ef_mul(prod, ef_frobenius(a, i));
  ef norm = ef_mul(prod, a);
  return ef_mul_f(prod, inv_m(norm.c[0]));
}

}  // namespace kb
