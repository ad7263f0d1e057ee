// Host Poseidon2-16 for the transcript's duplex challenger. Every sumcheck round observes a
// few extension elements and samples a challenge, so a proof runs several hundred of these
// permutations on the host between device round trips. With AVX-512 the 16-word state is
// one vector register: the S-boxes and the diagonal scaling are vector Montgomery products
// (32x32->64-bit multiplies on the even and odd lanes), the 4x4 external blocks are
// in-lane shuffles and the internal layer's sum is a horizontal add. The result is the same
// permutation as kb::p2_permute<16> (checked bit for bit in the tests); without AVX-512
// the scalar version runs.
// For the verifier's Merkle checks (many independent leaf sponges and compressions), batches
// of Poseidon2-24 / Poseidon2-16 run sixteen at a time with one instance per lane.
#include <immintrin.h>

#include <cstdint>

#include "poseidon2.cuh"

namespace wl {

namespace {

#define WL_AVX512 __attribute__((target("avx512f,avx512bw,avx512dq,avx512vl")))

struct V {
  __m512i p, pinv;
};

WL_AVX512 inline __m512i vadd(const V& k, __m512i a, __m512i b) {
  const __m512i s = _mm512_add_epi32(a, b);
  return _mm512_min_epu32(s, _mm512_sub_epi32(s, k.p));
}

// Montgomery product of 16 lanes (inputs below p): for each 64-bit product t, m = t * PINV mod
// 2^32 and t - m p is divisible by 2^32; its upper half lies in (-p, p), made canonical by
// the unsigned-min of r and r + p.
WL_AVX512 inline __m512i vmul(const V& k, __m512i a, __m512i b) {
  const __m512i te = _mm512_mul_epu32(a, b);
  const __m512i to = _mm512_mul_epu32(_mm512_srli_epi64(a, 32), _mm512_srli_epi64(b, 32));
  const __m512i me = _mm512_mul_epu32(te, k.pinv);
  const __m512i mo = _mm512_mul_epu32(to, k.pinv);
  const __m512i de = _mm512_sub_epi64(te, _mm512_mul_epu32(me, k.p));
  const __m512i dor = _mm512_sub_epi64(to, _mm512_mul_epu32(mo, k.p));
  const __m512i r = _mm512_mask_blend_epi32(0xAAAA, _mm512_srli_epi64(de, 32), dor);
  return _mm512_min_epu32(r, _mm512_add_epi32(r, k.p));
}

WL_AVX512 inline __m512i vcube(const V& k, __m512i x) { return vmul(k, vmul(k, x, x), x); }

// circ(2 M4, M4, M4, M4): lane i of a 4-word chunk gets 2 x_i + 3 x_(i+1) + x_(i+2) + x_(i+3),
// then every lane adds the sum over the four chunks at its position.
WL_AVX512 inline __m512i vmds(const V& k, __m512i a) {
  const __m512i b = _mm512_shuffle_epi32(a, (_MM_PERM_ENUM)0x39);
  const __m512i c = _mm512_shuffle_epi32(a, (_MM_PERM_ENUM)0x4E);
  const __m512i d = _mm512_shuffle_epi32(a, (_MM_PERM_ENUM)0x93);
  const __m512i y = vadd(k, vadd(k, vadd(k, a, b), vadd(k, c, d)), vadd(k, a, vadd(k, b, b)));
  __m512i t = vadd(k, y, _mm512_shuffle_i32x4(y, y, 0xB1));
  t = vadd(k, t, _mm512_shuffle_i32x4(t, t, 0x4E));
  return vadd(k, y, t);
}

WL_AVX512 void permute16_avx512(uint32_t* s, const kb::P16Consts& c) {
  V k;
  k.p = _mm512_set1_epi32((int)kb::P);
  k.pinv = _mm512_set1_epi32((int)kb::PINV);
  alignas(64) uint32_t diag[16];
  for (int i = 0; i < 16; i++) diag[i] = kb::p2_diag<16>(i);
  const __m512i dg = _mm512_load_si512(diag);
  __m512i x = _mm512_loadu_si512(s);
  x = vmds(k, x);
  for (int r = 0; r < 4; r++) x = vmds(k, vcube(k, vadd(k, x, _mm512_loadu_si512(c.ext_init + 16 * r))));
  // Partial rounds: word 0 stays in a scalar register through its S-box, while the sum of
  // words 1..15 (which does not wait for it) is formed from the vector; lane 0 of the vector
  // is refreshed once at the end.
  uint32_t x0 = (uint32_t)_mm_cvtsi128_si32(_mm512_castsi512_si128(x));
  const uint32_t d0 = kb::p2_diag<16>(0);
  for (int r = 0; r < 20; r++) {
    const __m512i rest = _mm512_maskz_mov_epi32(0xFFFE, x);
    const __m512i lo = _mm512_cvtepu32_epi64(_mm512_castsi512_si256(rest));
    const __m512i hi = _mm512_cvtepu32_epi64(_mm512_extracti64x4_epi64(rest, 1));
    const uint64_t tot = (uint64_t)_mm512_reduce_add_epi64(_mm512_add_epi64(lo, hi));  // < 2^35
    uint32_t s15 = uint32_t(tot & 0x7fffffffu) + uint32_t(tot >> 31) * ((1u << 24) - 1);  // < 2p
    s15 = kb::umin(s15, s15 - kb::P);
    const uint32_t xs = kb::cube(kb::add(x0, c.internal[r]));
    const uint32_t sum = kb::add(s15, xs);
    x0 = kb::add(kb::mul(xs, d0), sum);
    x = vadd(k, vmul(k, x, dg), _mm512_set1_epi32((int)sum));
  }
  x = _mm512_mask_set1_epi32(x, 1, (int)x0);
  for (int r = 0; r < 4; r++) x = vmds(k, vcube(k, vadd(k, x, _mm512_loadu_si512(c.ext_term + 16 * r))));
  _mm512_storeu_si512(s, x);
}

// ---- sixteen independent permutations: lane j of every vector is instance j, vector i holds
// word i of the sixteen states (the Merkle checks of the verifier hash many rows and paths).
template <int W>
WL_AVX512 inline void vmds_x16(const V& k, __m512i* x) {
  for (int c = 0; c < W; c += 4) {
    const __m512i x0 = x[c], x1 = x[c + 1], x2 = x[c + 2], x3 = x[c + 3];
    const __m512i t01 = vadd(k, x0, x1), t23 = vadd(k, x2, x3), t0123 = vadd(k, t01, t23);
    const __m512i t01123 = vadd(k, t0123, x1), t01233 = vadd(k, t0123, x3);
    x[c + 3] = vadd(k, t01233, vadd(k, x0, x0));
    x[c + 1] = vadd(k, t01123, vadd(k, x2, x2));
    x[c + 0] = vadd(k, t01123, t01);
    x[c + 2] = vadd(k, t01233, t23);
  }
  __m512i sums[4];
  for (int j = 0; j < 4; j++) {
    __m512i a = x[j];
    for (int c = 4 + j; c < W; c += 4) a = vadd(k, a, x[c]);
    sums[j] = a;
  }
  for (int i = 0; i < W; i++) x[i] = vadd(k, x[i], sums[i & 3]);
}

template <int W>
WL_AVX512 void permute_x16(__m512i* x, const kb::P2Consts<W>& c) {
  V k;
  k.p = _mm512_set1_epi32((int)kb::P);
  k.pinv = _mm512_set1_epi32((int)kb::PINV);
  vmds_x16<W>(k, x);
  for (int r = 0; r < 4; r++) {
    for (int i = 0; i < W; i++) x[i] = vcube(k, vadd(k, x[i], _mm512_set1_epi32((int)c.ext_init[r * W + i])));
    vmds_x16<W>(k, x);
  }
  for (int r = 0; r < kb::P2Consts<W>::RP; r++) {
    x[0] = vcube(k, vadd(k, x[0], _mm512_set1_epi32((int)c.internal[r])));
    __m512i sum = x[0];
    for (int i = 1; i < W; i++) sum = vadd(k, sum, x[i]);
    for (int i = 0; i < W; i++) x[i] = vadd(k, vmul(k, x[i], _mm512_set1_epi32((int)kb::p2_diag<W>(i))), sum);
  }
  for (int r = 0; r < 4; r++) {
    for (int i = 0; i < W; i++) x[i] = vcube(k, vadd(k, x[i], _mm512_set1_epi32((int)c.ext_term[r * W + i])));
    vmds_x16<W>(k, x);
  }
}

// n states of W words each (contiguous), in groups of sixteen (the last group padded).
template <int W>
WL_AVX512 void permute_many_avx512(uint32_t* states, size_t n, const kb::P2Consts<W>& c) {
  alignas(64) uint32_t t[W][16];
  __m512i x[W];
  for (size_t g = 0; g < n; g += 16) {
    const size_t m = n - g < 16 ? n - g : 16;
    for (size_t j = 0; j < 16; j++)
      for (int i = 0; i < W; i++) t[i][j] = j < m ? states[(g + j) * W + i] : 0u;
    for (int i = 0; i < W; i++) x[i] = _mm512_load_si512(t[i]);
    permute_x16<W>(x, c);
    for (int i = 0; i < W; i++) _mm512_store_si512(t[i], x[i]);
    for (size_t j = 0; j < m; j++)
      for (int i = 0; i < W; i++) states[(g + j) * W + i] = t[i][j];
  }
}

bool have_avx512() {
  static const bool ok = __builtin_cpu_supports("avx512f") && __builtin_cpu_supports("avx512bw") &&
                         __builtin_cpu_supports("avx512dq") && __builtin_cpu_supports("avx512vl");
  return ok;
}

}  // namespace

void host_p16_permute(uint32_t* s, const kb::P16Consts& c) {
  if (have_avx512()) {
    permute16_avx512(s, c);
  } else {
    kb::p2_permute<16>(s, c);
  }
}

// The portable version, for comparisons.
void host_p16_permute_scalar(uint32_t* s, const kb::P16Consts& c) { kb::p2_permute<16>(s, c); }

void host_p24_permute_many(uint32_t* states, size_t n, const kb::P24Consts& c) {
  if (have_avx512()) {
    permute_many_avx512<24>(states, n, c);
  } else {
    for (size_t i = 0; i < n; i++) kb::p2_permute<24>(states + 24 * i, c);
  }
}
void host_p16_permute_many(uint32_t* states, size_t n, const kb::P16Consts& c) {
  if (have_avx512()) {
    permute_many_avx512<16>(states, n, c);
  } else {
    for (size_t i = 0; i < n; i++) kb::p2_permute<16>(states + 16 * i, c);
  }
}

}  // namespace wl
