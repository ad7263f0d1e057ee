// Host-side check of the product's field arithmetic (whirlaway_b200/csrc/kb.cuh and
// poseidon2.cuh compile for the host too): Montgomery products, lazy reductions, the
// unsigned-min additions, the shortcut multiplications of the Poseidon2 internal layer and the
// canonical-domain S-box with fp64 quotients,
// each against a plain modular reference. Built and run by tests/test_boundary.py.
#include <cstdio>
#include <random>
#include <vector>
#include <type_traits>
#include "poseidon2.cuh"
namespace wl {
void host_p16_permute(uint32_t* s, const kb::P16Consts& c);
void host_p24_permute_many(uint32_t* states, size_t n, const kb::P24Consts& c);
void host_p16_permute_many(uint32_t* states, size_t n, const kb::P16Consts& c);
}
using namespace kb;
int main() {
  std::mt19937_64 g(1);
  long b1=0,b2=0,b3=0,b4=0,b5=0,b6=0;
  for (int it = 0; it < 100000; it++) {
    uint32_t x = g() % P, y = g() % P;
    if (add(x, y) != (uint32_t)(((uint64_t)x + y) % P)) b1++;
    if (sub(x, y) != (uint32_t)(((uint64_t)x + P - y) % P)) b2++;
    uint32_t xm = to_mont(x), ym = to_mont(y);
    if (from_mont(mul(xm, ym)) != (uint32_t)((uint64_t)x * y % P)) b3++;
    for (int i = 0; i < 16; i++) if (p2_diag_mul<16>(i, xm) != mul(xm, p2_diag<16>(i))) { if(b4<5) printf("w16 i=%d x=%u got %u want %u\n", i, xm, p2_diag_mul<16>(i, xm), mul(xm, p2_diag<16>(i))); b4++; }
    if (halve(xm) != mul(xm, inv_m(to_mont(2)))) b5++;
  }
  for (int it = 0; it < 100000; it++) {
    uint64_t acc = 0; uint32_t ref = 0;
    for (int k = 0; k < 4; k++) { uint32_t a = g() % P, b = g() % P; acc += wmul(a, b); ref = add(ref, mul(a, b)); }
    if (redc(acc) != ref) b6++;
  }
  for (int it = 0; it < 2000; it++) {
    uint32_t x = g() % P, xm = to_mont(x);
    for (int i = 0; i < 24; i++) if (p2_diag_mul<24>(i, xm) != mul(xm, p2_diag<24>(i))) b4++;
  }
  // extension-field square (distinct products only) against the general product
  for (int it = 0; it < 200000; it++) {
    ef a;
    for (int i = 0; i < 8; i++) a.c[i] = (it % 4 == 0) ? P - 1 - uint32_t(g() % 3) : uint32_t(g() % P);
    if (!ef_eq(ef_sqr(a), ef_mul(a, a))) b3++;
  }
  // x * 2^-k at the ends of the range and with all low bits set
  for (int k = 1; k <= 24; k++) {
    const uint32_t inv = detail::cm_inv2(k, false);
    const uint32_t lowk = (1u << k) - 1;
    const uint32_t edge[] = {0u, 1u, P - 1, P - 2, lowk, P - 1 - lowk, (P - 1) & ~lowk, ((P - 1) & ~lowk) - 1};
    for (uint32_t x : edge) if (mul_inv_pow2(x, k) != mul(x, inv)) b4++;
    for (int it = 0; it < 20000; it++) {
      const uint32_t x = g() % P;
      if (mul_inv_pow2(x, k) != mul(x, inv)) b4++;
    }
  }
  // cube (lazy inner square), the lazily reduced sums and whole permutations against plain
  // modular arithmetic
  long b7 = 0, b8 = 0;
  for (int it = 0; it < 100000; it++) {
    uint32_t v[23];
    uint64_t ref = 0;
    const bool top = it & 1;  // values at the top of the range
    for (int i = 0; i < 23; i++) v[i] = top ? P - 1 - uint32_t(g() % 7) : uint32_t(g() % P), ref += v[i];
    uint32_t x0 = top ? P - 1 : uint32_t(g() % P);
    if (sum_mod<23>(v, x0) != uint32_t((ref + x0) % P)) b7++;
    if (sum_mod<15>(v, x0) != uint32_t((ref - v[15] - v[16] - v[17] - v[18] - v[19] - v[20] - v[21] - v[22] + x0) % P)) b7++;
  }
  auto pm = [](uint64_t a, uint64_t b) { return uint32_t(a * b % P); };
  for (int it = 0; it < 100000; it++) {
    uint32_t x = g() % P;
    if (from_mont(cube(to_mont(x))) != pm(pm(x, x), x)) b7++;
  }
  // canonical-domain S-box with fp64 quotients, on unreduced inputs below 2p
  {
    const uint32_t edge[] = {0u, 1u, 2u, P - 2, P - 1, P, P + 1, 2 * P - 2, 2 * P - 1, 46341u, 65535u, 65536u,
                             1u << 30, (1u << 31) - 1, 1u << 31, 0xfe000000u, 0xfe000001u};
    for (uint32_t u : edge) if (cube_fq(u) != pm(pm(u % P, u % P), u % P)) b7++;
    for (int it = 0; it < 2000000; it++) {
      const uint32_t u = uint32_t(g() % (2ull * P));
      if (cube_fq(u) != pm(pm(u % P, u % P), u % P)) b7++;
    }
  }
  // internal layer with lazily reduced words 9.. (any value below 2^32) against the canonical one
  {
    auto lazy_check = [&](auto wtag) {
      constexpr int W = decltype(wtag)::value;
      for (int it = 0; it < 200000; it++) {
        uint32_t s[W], r[W];
        const uint32_t x0 = (it % 7 == 0) ? P - 1 : uint32_t(g() % P);
        for (int i = 0; i < W; i++) {
          if (i < 9) s[i] = (it % 5 == 0) ? P - 1 - uint32_t(g() % 3) : uint32_t(g() % P);
          else s[i] = (it % 3 == 0) ? 0xffffffffu - uint32_t(g() % 5) : uint32_t(g());
          r[i] = s[i] % P;
        }
        internal_layer_lazy_with0<W>(s, x0);
        internal_layer_with0<W>(r, x0);
        for (int i = 0; i < W; i++) {
          if (i < 9 && s[i] >= P) { b4++; break; }
          if (s[i] % P != r[i]) { b4++; break; }
        }
        internal_lazy_finish<W>(s);
        for (int i = 0; i < W; i++) if (s[i] != r[i]) { b4++; break; }
      }
    };
    lazy_check(std::integral_constant<int, 16>{});
    lazy_check(std::integral_constant<int, 24>{});
  }
  for (int w = 0; w < 2; w++) {
    const int W = w ? 24 : 16, RP = w ? 23 : 20;
    for (int it = 0; it < 300; it++) {
      P16Consts c16;
      P24Consts c24;
      uint32_t* ei = w ? c24.ext_init : c16.ext_init;
      uint32_t* et = w ? c24.ext_term : c16.ext_term;
      uint32_t* in = w ? c24.internal : c16.internal;
      for (int i = 0; i < 4 * W; i++) ei[i] = to_mont(g() % P), et[i] = to_mont(g() % P);
      for (int i = 0; i < RP; i++) in[i] = to_mont(g() % P);
      uint32_t s[24], r[24];
      for (int i = 0; i < W; i++) s[i] = g() % P, r[i] = s[i];
      // reference on canonical values: diag entries and constants through from_mont
      auto mds = [&](uint32_t* v) {
        uint32_t t[24];
        for (int c = 0; c < W; c += 4)
          for (int i = 0; i < 4; i++) {
            static const int M4[4][4] = {{2, 3, 1, 1}, {1, 2, 3, 1}, {1, 1, 2, 3}, {3, 1, 1, 2}};
            uint64_t a = 0;
            for (int j = 0; j < 4; j++) a += uint64_t(M4[i][j]) * v[c + j];
            t[c + i] = uint32_t(a % P);
          }
        for (int i = 0; i < W; i++) {
          uint64_t a = t[i];
          for (int c = 0; c < W; c += 4) a += t[c + (i & 3)];
          v[i] = uint32_t(a % P);
        }
      };
      auto cub = [&](uint32_t x) { return pm(pm(x, x), x); };
      mds(r);
      for (int rd = 0; rd < 4; rd++) {
        for (int i = 0; i < W; i++) r[i] = cub(uint32_t((uint64_t(r[i]) + from_mont(ei[rd * W + i])) % P));
        mds(r);
      }
      for (int rd = 0; rd < RP; rd++) {
        r[0] = cub(uint32_t((uint64_t(r[0]) + from_mont(in[rd])) % P));
        uint64_t sum = 0;
        for (int i = 0; i < W; i++) sum += r[i];
        for (int i = 0; i < W; i++) {
          const uint32_t d = from_mont(w ? p2_diag<24>(i) : p2_diag<16>(i));
          r[i] = uint32_t((uint64_t(pm(d, r[i])) + sum) % P);
        }
      }
      for (int rd = 0; rd < 4; rd++) {
        for (int i = 0; i < W; i++) r[i] = cub(uint32_t((uint64_t(r[i]) + from_mont(et[rd * W + i])) % P));
        mds(r);
      }
      uint32_t sc[24];  // the canonical-domain permutation of the Merkle hashes (full rounds in fp64)
      for (int i = 0; i < W; i++) sc[i] = s[i];
      if (w) p2_permute_fd<24>(sc, p2_consts_fd(c24)); else p2_permute_fd<16>(sc, p2_consts_fd(c16));
      for (int i = 0; i < W; i++) if (sc[i] != r[i]) { b8++; break; }
      for (int i = 0; i < W; i++) s[i] = to_mont(s[i]);
      uint32_t sv[16];
      for (int i = 0; i < 16; i++) sv[i] = s[i];
      if (w) p2_permute<24>(s, c24); else p2_permute<16>(s, c16);
      for (int i = 0; i < W; i++) if (from_mont(s[i]) != r[i]) { b8++; break; }
      if (!w) {  // the transcript's host permutation (vector when the CPU has AVX-512)
        wl::host_p16_permute(sv, c16);
        for (int i = 0; i < 16; i++) if (sv[i] != s[i]) { b8++; break; }
      }
    }
  }
  // batches of independent permutations (sixteen per vector, lane = instance; ragged last
  // group) against one at a time
  for (int w = 0; w < 2; w++) {
    const int W = w ? 24 : 16;
    P16Consts c16;
    P24Consts c24;
    uint32_t* ei = w ? c24.ext_init : c16.ext_init;
    uint32_t* et = w ? c24.ext_term : c16.ext_term;
    uint32_t* in = w ? c24.internal : c16.internal;
    for (int i = 0; i < 4 * W; i++) ei[i] = to_mont(g() % P), et[i] = to_mont(g() % P);
    for (int i = 0; i < (w ? 23 : 20); i++) in[i] = to_mont(g() % P);
    for (size_t n : {size_t(1), size_t(15), size_t(16), size_t(17), size_t(40)}) {
      std::vector<uint32_t> many(n * W), one(n * W);
      for (size_t i = 0; i < n * W; i++) many[i] = one[i] = (i % 7 == 3) ? P - 1 : uint32_t(g() % P);
      if (w) wl::host_p24_permute_many(many.data(), n, c24); else wl::host_p16_permute_many(many.data(), n, c16);
      for (size_t j = 0; j < n; j++) {
        if (w) p2_permute<24>(one.data() + 24 * j, c24); else p2_permute<16>(one.data() + 16 * j, c16);
      }
      if (many != one) b8++;
    }
  }
  // the fp64 S-box and canonical reduction over the whole input range of the fp64 full rounds:
  // signed integers below 49 * 2^32 + p in magnitude, at the ends and at random
  {
    const int64_t zmax = 49 * (int64_t(1) << 32) + P;
    auto cube_ref = [&](int64_t z) {
      const uint32_t u = uint32_t(((z % int64_t(P)) + int64_t(P)) % int64_t(P));
      return pm(pm(u, u), u);
    };
    auto check = [&](int64_t z) {
      const double zd = double(z);
      const double c = sbox_fd(zd);
      const int64_t ci = int64_t(c);
      if (double(ci) != c || ci <= -int64_t(P) || ci >= int64_t(P) ||
          uint32_t(((ci % int64_t(P)) + int64_t(P)) % int64_t(P)) != cube_ref(z)) b7++;
      if (fd_canonical(zd) != uint32_t(((z % int64_t(P)) + int64_t(P)) % int64_t(P))) b7++;
    };
    for (int64_t e : {int64_t(0), int64_t(1), int64_t(P) - 1, int64_t(P), int64_t(P) + 1, zmax - 1, int64_t(1) << 32})
      check(e), check(-e);
    for (int64_t k = -60; k <= 60; k++) check(k * int64_t(P)), check(k * int64_t(P) + 1), check(k * int64_t(P) - 1),
        check(k * int64_t(P) + (int64_t(P) >> 1)), check(k * int64_t(P) - (int64_t(P) >> 1));
    for (int it = 0; it < 1000000; it++) check(int64_t(g() % uint64_t(2 * zmax - 1)) - (zmax - 1));
  }
  printf("add %ld sub %ld mul %ld diag %ld halve %ld redc %ld cube %ld permute %ld\n", b1,b2,b3,b4,b5,b6,b7,b8);
  return (b1 + b2 + b3 + b4 + b5 + b6 + b7 + b8) ? 1 : 0;
}
