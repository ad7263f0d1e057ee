// The Poseidon2-KoalaBear width-16 AIR (p3-poseidon2-air as configured in the reference's
// src/examples/poseidon2.rs:21-36: S-box degree 3, no S-box registers, 4 + 4 full rounds,
// 20 partial rounds), for trace generation and constraint evaluation on the device.
//
// Column layout (165 columns, the trace matrix of one permutation per row):
//   0          export flag
//   1..16      inputs
//   17..80     4 beginning full rounds x 16 post-round states
//   81..100    20 partial rounds x post-S-box state[0]
//   101..164   4 ending full rounds x 16 post-round states
// Constraints (148, degree 3): each full-round output and each partial-round S-box
// output equals its committed column. The constraint polynomial reads the local row
// only, so only the "up" columns of a zerocheck point are used.
#pragma once
#include "poseidon2.cuh"

namespace wl {

constexpr int AIR_W = 165;
constexpr int AIR_NC = 148;
constexpr int AIR_LOG_W = 8;  // log2_up(165)

struct AirConsts {  // Montgomery form
  uint32_t begin[4][16];
  uint32_t partial[20];
  uint32_t end[4][16];
};

// Trace row: fills out[c * stride] for the 165 columns.
__host__ __device__ __forceinline__ void air_trace_row(const AirConsts& K, const uint32_t* in16, uint32_t* out,
                                                       size_t stride) {
  uint32_t s[16];
  out[0] = kb::R_MOD_P;
#pragma unroll
  for (int i = 0; i < 16; i++) {
    s[i] = in16[i];
    out[size_t(1 + i) * stride] = s[i];
  }
  kb::mds_light<16>(s);
  int col = 17;
#pragma unroll 1
  for (int r = 0; r < 4; r++) {
#pragma unroll
    for (int i = 0; i < 16; i++) s[i] = kb::cube(kb::add(s[i], K.begin[r][i]));
    kb::mds_light<16>(s);
#pragma unroll
    for (int i = 0; i < 16; i++) out[size_t(col + i) * stride] = s[i];
    col += 16;
  }
#pragma unroll 1
  for (int r = 0; r < 20; r++) {
    const uint32_t x0 = kb::cube(kb::add(s[0], K.partial[r]));
    out[size_t(col++) * stride] = x0;
    kb::internal_layer_with0<16>(s, x0);
  }
#pragma unroll 1
  for (int r = 0; r < 4; r++) {
#pragma unroll
    for (int i = 0; i < 16; i++) s[i] = kb::cube(kb::add(s[i], K.end[r][i]));
    kb::mds_light<16>(s);
#pragma unroll
    for (int i = 0; i < 16; i++) out[size_t(col + i) * stride] = s[i];
    col += 16;
  }
}

// Base-field constraint evaluation. `get(c)` returns column c of the point, `acc(h, i)`
// receives constraint i's value h; `flush()` is called after every 4 constraints.
template <class Get, class Acc, class Flush>
__device__ __forceinline__ void air_eval_f(const AirConsts& K, Get&& get, Acc&& acc, Flush&& flush) {
  uint32_t s[16];
#pragma unroll
  for (int i = 0; i < 16; i++) s[i] = get(1 + i);
  kb::mds_light<16>(s);
  int col = 17;
#pragma unroll 1
  for (int r = 0; r < 4; r++) {
#pragma unroll
    for (int i = 0; i < 16; i++) s[i] = kb::cube(kb::add(s[i], K.begin[r][i]));
    kb::mds_light<16>(s);
#pragma unroll
    for (int i = 0; i < 16; i++) {
      uint32_t p = get(col + i);
      acc(kb::sub(s[i], p), r * 16 + i);
      s[i] = p;
      if ((i & 3) == 3) flush();
    }
    col += 16;
  }
#pragma unroll 1
  for (int r4 = 0; r4 < 20; r4 += 4) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const uint32_t x0 = kb::cube(kb::add(s[0], K.partial[r4 + q]));
      const uint32_t p = get(col++);
      acc(kb::sub(x0, p), 64 + r4 + q);
      kb::internal_layer_with0<16>(s, p);
    }
    flush();
  }
#pragma unroll 1
  for (int r = 0; r < 4; r++) {
#pragma unroll
    for (int i = 0; i < 16; i++) s[i] = kb::cube(kb::add(s[i], K.end[r][i]));
    kb::mds_light<16>(s);
#pragma unroll
    for (int i = 0; i < 16; i++) {
      uint32_t p = get(col + i);
      acc(kb::sub(s[i], p), 84 + r * 16 + i);
      s[i] = p;
      if ((i & 3) == 3) flush();
    }
    col += 16;
  }
}

// Extension-field constraint evaluation: returns sum_i alpha^i * h_i (device kernels and the
// host verifier).
template <class Get>
__host__ __device__ __forceinline__ kb::ef air_eval_ef(const AirConsts& K, const kb::ef* alphas, Get&& get) {
  using namespace kb;
  ef s[16];
#pragma unroll
  for (int i = 0; i < 16; i++) s[i] = get(1 + i);
  mds_light_ef16(s);
  ef acc = ef_zero();
  int col = 17;
#pragma unroll 1
  for (int r = 0; r < 4; r++) {
#pragma unroll
    for (int i = 0; i < 16; i++) s[i] = ef_cube(ef_add_f(s[i], K.begin[r][i]));
    mds_light_ef16(s);
#pragma unroll
    for (int i = 0; i < 16; i++) {
      ef p = get(col + i);
      acc = ef_add(acc, ef_mul(alphas[r * 16 + i], ef_sub(s[i], p)));
      s[i] = p;
    }
    col += 16;
  }
#pragma unroll 1
  for (int r = 0; r < 20; r++) {
    s[0] = ef_cube(ef_add_f(s[0], K.partial[r]));
    ef p = get(col++);
    acc = ef_add(acc, ef_mul(alphas[64 + r], ef_sub(s[0], p)));
    s[0] = p;
    internal_layer_ef16(s);
  }
#pragma unroll 1
  for (int r = 0; r < 4; r++) {
#pragma unroll
    for (int i = 0; i < 16; i++) s[i] = ef_cube(ef_add_f(s[i], K.end[r][i]));
    mds_light_ef16(s);
#pragma unroll
    for (int i = 0; i < 16; i++) {
      ef p = get(col + i);
      acc = ef_add(acc, ef_mul(alphas[84 + r * 16 + i], ef_sub(s[i], p)));
      s[i] = p;
    }
    col += 16;
  }
  return acc;
}

}  // namespace wl
