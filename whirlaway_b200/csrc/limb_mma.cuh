// Exact modular dot products on the tensor cores through byte limbs: shared helpers of the
// kernels that evaluate extension x base sums as u8 matrix products (k_sumcheck.cu,
// k_whir.cu). With x = sum_a 2^(8a) x_a and w = sum_b 2^(8b) w_b (bytes), sum_k w_k x_k =
// sum_(a,b) 2^(8(a+b)) sum_k w_(k,b) x_(k,a); each inner sum is accumulated in s32 by
// mma.m16n8k32 (at most 2^12 byte products per accumulator, below 2^28).
#pragma once
#include "common.cuh"
#include "poseidon2.cuh"

namespace wl {

#ifdef __CUDACC__
__device__ __forceinline__ void mma_u8_16832(int (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k32.row.col.s32.u8.u8.s32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+r"(c[0]), "+r"(c[1]), "+r"(c[2]), "+r"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
// Byte a of four consecutive values, packed (limb a of a k-quad of the A fragment).
__device__ __forceinline__ void byte_transpose4(const uint4 q, uint32_t (&r)[4]) {
  const uint32_t p01l = __byte_perm(q.x, q.y, 0x5140), p01h = __byte_perm(q.x, q.y, 0x7362);
  const uint32_t p23l = __byte_perm(q.z, q.w, 0x5140), p23h = __byte_perm(q.z, q.w, 0x7362);
  r[0] = __byte_perm(p01l, p23l, 0x5410);
  r[1] = __byte_perm(p01l, p23l, 0x7632);
  r[2] = __byte_perm(p01h, p23h, 0x5410);
  r[3] = __byte_perm(p01h, p23h, 0x7632);
}

// Sum over the limb pairs of one accumulator position held by this lane: acc[a][b][q] for
// the 16 pairs (a, b), combined by diagonal a + b = d (below 4 * 2^12 * 255^2 < 2^31),
// weighted by 2^(8d) mod p and reduced once (the sum stays below 4 p^2). Montgomery inputs
// give the Montgomery product.
__device__ __forceinline__ uint32_t limb_recombine_lane(const int (&acc)[4][4][4], int q) {
  constexpr uint32_t W8[7] = {uint32_t(kb::detail::cpow(2, 0)),  uint32_t(kb::detail::cpow(2, 8)),
                              uint32_t(kb::detail::cpow(2, 16)), uint32_t(kb::detail::cpow(2, 24)),
                              uint32_t(kb::detail::cpow(2, 32)), uint32_t(kb::detail::cpow(2, 40)),
                              uint32_t(kb::detail::cpow(2, 48))};  // 2^(8d) mod p
  uint64_t v = 0;
#pragma unroll
  for (int d = 0; d < 7; d++) {
    uint32_t dd = 0;
#pragma unroll
    for (int a = 0; a < 4; a++)
      if (d - a >= 0 && d - a < 4) dd += uint32_t(acc[a][d - a][q]);
    v += kb::wmul(dd, W8[d]);
  }
  return kb::redc(v);
}
#endif

}  // namespace wl
