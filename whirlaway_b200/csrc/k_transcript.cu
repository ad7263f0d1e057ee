// Device-side Fiat-Shamir for the sumcheck rounds.
//
// A sumcheck round ends with a few extension-field sums (the round polynomial at a handful of
// points), which the prover interpolates, writes to the proof, absorbs into the
// DuplexChallenger<F, Poseidon16, 16, 8> and answers with a sampled challenge that the next
// fold uses (crates/sumcheck/src/prove.rs:190-222 for the zerocheck and product sumchecks;
// the WHIR folding sumcheck sends its three values directly). Done on the host, every round is
// a device-to-host round trip during which the device idles. Here one single-block kernel per
// round reduces the partial sums, finishes the round exactly as the host would (same
// challenger semantics as HostChallenger: observations fill the rate and duplex at eight,
// samples pop from the end of the last squeeze) and leaves the challenge in device memory for
// the fold, so the host enqueues a whole phase of rounds without waiting and reads the
// appended proof words, the challenges and the challenger state back once at its end.
#include <algorithm>

#include "kernels.h"

namespace wl {

namespace {

constexpr int FIN_THREADS = 384;  // up to three sums, 128 threads each

// Poseidon2-16 in Montgomery form for one warp whose 32 lanes all hold the same state (the
// transcript runs redundantly on every lane of warp 0, so every lane has every value). The
// full rounds spread the state over 16 lanes (lane i, and its mirror i + 16, holds word i):
// the S-boxes run side by side and the external layer is three in-chunk shuffles and two
// cross-chunk shuffle sums. The partial rounds run on the whole state in every lane (only word
// 0 takes the S-box, the other words' updates are independent of each other). The field values
// are those of kb::p2_permute<16>: the same linear maps and S-box, evaluated in another order.
__device__ __forceinline__ uint32_t m4_lanes(uint32_t a, int i) {
  const int base = i & ~3;
  const uint32_t b = __shfl_sync(0xffffffffu, a, base | ((i + 1) & 3), 16);
  const uint32_t c = __shfl_sync(0xffffffffu, a, base | ((i + 2) & 3), 16);
  const uint32_t d = __shfl_sync(0xffffffffu, a, base | ((i + 3) & 3), 16);
  // row i of circ(2, 3, 1, 1) within the chunk: 2a + 3b + c + d
  const uint32_t y = kb::add(kb::add(kb::add(a, b), kb::add(c, d)), kb::add(a, kb::dbl(b)));
  uint32_t t = kb::add(y, __shfl_xor_sync(0xffffffffu, y, 4, 16));
  t = kb::add(t, __shfl_xor_sync(0xffffffffu, t, 8, 16));
  return kb::add(y, t);
}
__device__ __forceinline__ uint32_t lane_word(const uint32_t (&s)[16], int i) {
  uint32_t v = s[0];
#pragma unroll
  for (int j = 1; j < 16; j++) v = i == j ? s[j] : v;
  return v;
}
// This lane's full-round constants (word i of each full round), loaded once per kernel: indexed
// by the lane they would be divergent constant-cache loads inside the permutation.
struct LaneRc {
  uint32_t init[4], term[4];
};
__device__ __forceinline__ LaneRc lane_rc(const kb::P16Consts& c) {
  const int i = threadIdx.x & 15;
  LaneRc l;
#pragma unroll
  for (int r = 0; r < 4; r++) l.init[r] = c.ext_init[r * 16 + i], l.term[r] = c.ext_term[r * 16 + i];
  return l;
}
__device__ __forceinline__ void p16_warp(uint32_t (&s)[16], const kb::P16Consts& c, const LaneRc& lr) {
  const int i = threadIdx.x & 15;
  uint32_t v = m4_lanes(lane_word(s, i), i);
#pragma unroll
  for (int r = 0; r < 4; r++) v = m4_lanes(kb::cube(kb::add(v, lr.init[r])), i);
#pragma unroll
  for (int j = 0; j < 16; j++) s[j] = __shfl_sync(0xffffffffu, v, j, 16);
#pragma unroll 4
  for (int r = 0; r < kb::P16Consts::RP; r++) kb::internal_layer_with0<16>(s, kb::cube(kb::add(s[0], c.internal[r])));
  v = lane_word(s, i);
#pragma unroll
  for (int r = 0; r < 4; r++) v = m4_lanes(kb::cube(kb::add(v, lr.term[r])), i);
#pragma unroll
  for (int j = 0; j < 16; j++) s[j] = __shfl_sync(0xffffffffu, v, j, 16);
}

// The challenger stays in registers: its buffers are indexed only through unrolled selects
// (a dynamic index would put the whole state in local memory). Every lane of the calling warp
// takes part, with the same values.
__device__ __forceinline__ void dch_duplex(DevChallenger& c, const kb::P16Consts& p, const LaneRc& lr) {
  uint32_t s[16];
#pragma unroll
  for (int i = 0; i < 16; i++) s[i] = (i < 8 && i < c.in_len) ? c.in[i] : c.state[i];
  c.in_len = 0;
  p16_warp(s, p, lr);
#pragma unroll
  for (int i = 0; i < 16; i++) c.state[i] = s[i];
#pragma unroll
  for (int i = 0; i < 8; i++) c.out[i] = s[i];
  c.out_len = 8;
}
__device__ __forceinline__ void dch_observe(DevChallenger& c, uint32_t x, const kb::P16Consts& p, const LaneRc& lr) {
  c.out_len = 0;
#pragma unroll
  for (int j = 0; j < 8; j++) c.in[j] = j == c.in_len ? x : c.in[j];
  if (++c.in_len == 8) dch_duplex(c, p, lr);
}
__device__ __forceinline__ uint32_t dch_sample(DevChallenger& c, const kb::P16Consts& p, const LaneRc& lr) {
  if (c.in_len || !c.out_len) dch_duplex(c, p, lr);
  --c.out_len;
  uint32_t v = c.out[0];
#pragma unroll
  for (int j = 1; j < 8; j++) v = j == c.out_len ? c.out[j] : v;
  return v;
}
// Writes v to the proof and absorbs it (Transcript::add_ext).
__device__ __forceinline__ void dts_add_ext(DevRound& st, uint32_t* proof, const ef& v, const kb::P16Consts& p,
                                            const LaneRc& lr) {
#pragma unroll
  for (int i = 0; i < 8; i++) {
    if ((threadIdx.x & 31) == 0) proof[st.proof_len] = v.c[i];
    st.proof_len++;
    dch_observe(st.ch, v.c[i], p, lr);
  }
}
__device__ __forceinline__ ef dts_sample_ext(DevRound& st, const kb::P16Consts& p, const LaneRc& lr) {
  ef e;
#pragma unroll
  for (int i = 0; i < 8; i++) e.c[i] = dch_sample(st.ch, p, lr);
  return e;
}

// Sums of `nsum` interleaved partials (partial[b * nsum + z]) into red[z]; every thread of the
// block takes part, the result is valid after the final barrier.
__device__ void reduce_sums(const ef* __restrict__ partial, int nb, int nsum, ef* red, ef* scratch) {
  const int z = threadIdx.x >> 7, t = threadIdx.x & 127;
  ef acc = kb::ef_zero();
  if (z < nsum) {
    int b = t;
    for (; b + 384 < nb; b += 512) {  // four loads in flight
      const ef v0 = partial[size_t(b) * nsum + z], v1 = partial[size_t(b + 128) * nsum + z];
      const ef v2 = partial[size_t(b + 256) * nsum + z], v3 = partial[size_t(b + 384) * nsum + z];
      acc = kb::ef_add(acc, kb::ef_add(kb::ef_add(v0, v1), kb::ef_add(v2, v3)));
    }
    for (; b < nb; b += 128) acc = kb::ef_add(acc, partial[size_t(b) * nsum + z]);
  }
  acc = warp_reduce_ef(acc);
  if ((threadIdx.x & 31) == 0) scratch[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (t == 0 && z < nsum) {
    ef s = scratch[z * 4];
    for (int w = 1; w < 4; w++) s = kb::ef_add(s, scratch[z * 4 + w]);
    red[z] = s;
  }
  __syncthreads();
}

template <int N>
__device__ __forceinline__ ef poly_eval_dev(const ef (&c)[N], const ef& x) {
  ef r = kb::ef_zero();
#pragma unroll
  for (int i = N - 1; i >= 0; i--) r = kb::ef_add(kb::ef_mul(r, x), c[i]);
  return r;
}
// c[k] of a small register array without a dynamic index.
template <int N>
__device__ __forceinline__ ef pick(const ef (&c)[N], int k) {
  ef r = c[0];
#pragma unroll
  for (int i = 1; i < N; i++)
#pragma unroll
    for (int w = 0; w < 8; w++) r.c[w] = i == k ? c[i].c[w] : r.c[w];
  return r;
}

// Round of a sumcheck with an eq factor (the zerocheck's rounds >= 1 and those of the a*b - c
// zerocheck): the computed sums are at z = 0, 2, .., NPTS - 1 (NPTS - 1 of them), weighted by
// the factor mmf of the variables already folded; the value at 1 follows from the claim,
// e1 = (sum - e0 (1 - r)) / r. The round polynomial is the interpolation on 0..NPTS-1 times the
// eq factor of the current variable, (1 - r) + (2r - 1) X: NPTS + 1 coefficients.
template <int NPTS>
__global__ void __launch_bounds__(FIN_THREADS, 1) k_eqsc_round_finish(const ef* __restrict__ partial, int nb, ef r,
                                                                   ef rinv, const __grid_constant__ FinishConsts fc,
                                                                   DevRound* __restrict__ stp,
                                                                   uint32_t* __restrict__ proof,
                                                                   ef* __restrict__ ch_out) {
  __shared__ ef red[3], scratch[12];
  reduce_sums(partial, nb, NPTS - 1, red, scratch);
  if (threadIdx.x >= 32) return;  // warp 0 finishes the round, every lane the same values
  const LaneRc lr = lane_rc(fc.p16);
  DevRound st = *stp;
  ef e[NPTS];
  e[0] = kb::ef_mul(red[0], st.mmf);
#pragma unroll
  for (int i = 2; i < NPTS; i++) e[i] = kb::ef_mul(red[i - 1], st.mmf);
  const ef one = kb::ef_one();
  const ef omr = kb::ef_sub(one, r);
  e[1] = kb::ef_mul(kb::ef_sub(st.sum, kb::ef_mul(e[0], omr)), rinv);
  ef q[NPTS];
#pragma unroll
  for (int k = 0; k < NPTS; k++) q[k] = kb::ef_zero();
#pragma unroll
  for (int i = 0; i < NPTS; i++)
#pragma unroll
    for (int k = 0; k < NPTS; k++) q[k] = kb::ef_add(q[k], kb::ef_mul_f(e[i], fc.basis[NPTS - 3][i][k]));
  const ef lin = kb::ef_sub(kb::ef_add(r, r), one);  // (1 - r) + lin X
  ef p[NPTS + 1];
#pragma unroll
  for (int k = 0; k <= NPTS; k++) p[k] = kb::ef_zero();
#pragma unroll
  for (int k = 0; k < NPTS; k++) {
    p[k] = kb::ef_add(p[k], kb::ef_mul(q[k], omr));
    p[k + 1] = kb::ef_add(p[k + 1], kb::ef_mul(q[k], lin));
  }
#pragma unroll 1
  for (int k = 0; k <= NPTS; k++) dts_add_ext(st, proof, pick(p, k), fc.p16, lr);
  const ef c = dts_sample_ext(st, fc.p16, lr);
  st.sum = poly_eval_dev(p, c);
  st.mmf = kb::ef_mul(kb::ef_add(kb::ef_mul(omr, kb::ef_sub(one, c)), kb::ef_mul(r, c)), st.mmf);
  if (threadIdx.x == 0) {
    ch_out[st.round] = c;
    st.round++;
    *stp = st;
  }
}

// Round of the product sumcheck (the inner sumcheck): sums at 0 and 2, the value at 1 from the
// claim; the round polynomial (3 coefficients) interpolates 0, 1, 2.
__global__ void __launch_bounds__(FIN_THREADS, 1) k_prod_round_finish(const ef* __restrict__ partial, int nb,
                                                                   const __grid_constant__ FinishConsts fc,
                                                                   DevRound* __restrict__ stp,
                                                                   uint32_t* __restrict__ proof,
                                                                   ef* __restrict__ ch_out) {
  __shared__ ef red[3], scratch[12];
  reduce_sums(partial, nb, 2, red, scratch);
  if (threadIdx.x >= 32) return;  // warp 0 finishes the round, every lane the same values
  const LaneRc lr = lane_rc(fc.p16);
  DevRound st = *stp;
  const ef y[3] = {red[0], kb::ef_sub(st.sum, red[0]), red[1]};
  ef p[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    p[k] = kb::ef_zero();
#pragma unroll
    for (int i = 0; i < 3; i++) p[k] = kb::ef_add(p[k], kb::ef_mul_f(y[i], fc.basis[0][i][k]));
  }
#pragma unroll 1
  for (int k = 0; k < 3; k++) dts_add_ext(st, proof, pick(p, k), fc.p16, lr);
  const ef c = dts_sample_ext(st, fc.p16, lr);
  st.sum = poly_eval_dev(p, c);
  if (threadIdx.x == 0) {
    ch_out[st.round] = c;
    st.round++;
    *stp = st;
  }
}

// Round of the WHIR folding sumcheck: the three values h(0), h(1), h(2) go to the proof as
// they are; the next claim is h(r) by quadratic interpolation on 0, 1, 2.
__global__ void __launch_bounds__(FIN_THREADS, 1) k_whir_round_finish(const ef* __restrict__ partial, int nb,
                                                                   const __grid_constant__ FinishConsts fc,
                                                                   DevRound* __restrict__ stp,
                                                                   uint32_t* __restrict__ proof,
                                                                   ef* __restrict__ ch_out) {
  __shared__ ef red[3], scratch[12];
  reduce_sums(partial, nb, 3, red, scratch);
  if (threadIdx.x >= 32) return;  // warp 0 finishes the round, every lane the same values
  const LaneRc lr = lane_rc(fc.p16);
  DevRound st = *stp;
  const ef h[3] = {red[0], red[1], red[2]};
#pragma unroll 1
  for (int k = 0; k < 3; k++) dts_add_ext(st, proof, pick(h, k), fc.p16, lr);
  const ef r = dts_sample_ext(st, fc.p16, lr);
  // h(r) = h0 (r-1)(r-2)/2 - h1 r (r-2) + h2 r (r-1)/2
  const ef rm1 = kb::ef_sub_f(r, fc.one), rm2 = kb::ef_sub_f(r, fc.two);
  const ef a = kb::ef_mul_f(kb::ef_mul(kb::ef_mul(red[0], rm1), rm2), fc.inv2);
  const ef b = kb::ef_mul(kb::ef_mul(red[1], r), rm2);
  const ef c = kb::ef_mul_f(kb::ef_mul(kb::ef_mul(red[2], r), rm1), fc.inv2);
  st.sum = kb::ef_add(kb::ef_sub(a, b), c);
  if (threadIdx.x == 0) {
    ch_out[st.round] = r;
    st.round++;
    *stp = st;
  }
}

// First level of the reduction of nb interleaved rows of k partial sums (partial[row * k + z]):
// block b sums a contiguous range of rows into out[b * k + z]. Thread t takes sum z = t % k on
// rows t / k, t / k + tpz, ... (tpz = 256 / k threads per sum), so a warp reads consecutive
// extension elements.
constexpr int WIDE_THREADS = 256;
__global__ void __launch_bounds__(WIDE_THREADS) k_reduce_wide(const ef* __restrict__ partial, int nb, int k,
                                                              ef* __restrict__ out) {
  __shared__ ef red[WIDE_THREADS];
  const int tpz = WIDE_THREADS / k, t = threadIdx.x;
  const int per = (nb + gridDim.x - 1) / gridDim.x;
  const int r0 = blockIdx.x * per, r1 = min(nb, r0 + per);
  ef acc = kb::ef_zero();
  if (t < tpz * k) {
    const int z = t % k;
    for (int r = r0 + t / k; r < r1; r += tpz) acc = kb::ef_add(acc, partial[size_t(r) * k + z]);
  }
  red[t] = acc;
  __syncthreads();
  if (t < k) {
    ef s = kb::ef_zero();
    for (int i = 0; i < tpz; i++) s = kb::ef_add(s, red[i * k + t]);
    out[size_t(blockIdx.x) * k + t] = s;
  }
}

}  // namespace

int launch_reduce_wide(const ef* partial, int nb, int k, ef* out, int max_blocks, cudaStream_t s) {
  if (k < 1 || k > 32) throw std::invalid_argument("wide reduction of 1..32 sums");
  const int blocks = std::max(1, std::min(max_blocks, (nb + 63) / 64));
  k_reduce_wide<<<blocks, WIDE_THREADS, 0, s>>>(partial, nb, k, out);
  WL_LAUNCH_CHECK();
  return blocks;
}

void launch_eqsc_round_finish(int npts, const ef* partial, int nb, const ef& r, const ef& rinv,
                              const FinishConsts& fc, DevRound* st, uint32_t* proof, ef* ch_out, cudaStream_t s) {
  if (npts == 4)
    k_eqsc_round_finish<4><<<1, FIN_THREADS, 0, s>>>(partial, nb, r, rinv, fc, st, proof, ch_out);
  else if (npts == 3)
    k_eqsc_round_finish<3><<<1, FIN_THREADS, 0, s>>>(partial, nb, r, rinv, fc, st, proof, ch_out);
  else
    throw std::invalid_argument("eq-factor sumcheck rounds of 3 or 4 points");
  WL_LAUNCH_CHECK();
}
void launch_prod_round_finish(const ef* partial, int nb, const FinishConsts& fc, DevRound* st, uint32_t* proof,
                              ef* ch_out, cudaStream_t s) {
  k_prod_round_finish<<<1, FIN_THREADS, 0, s>>>(partial, nb, fc, st, proof, ch_out);
  WL_LAUNCH_CHECK();
}
void launch_whir_round_finish(const ef* partial, int nb, const FinishConsts& fc, DevRound* st, uint32_t* proof,
                              ef* ch_out, cudaStream_t s) {
  k_whir_round_finish<<<1, FIN_THREADS, 0, s>>>(partial, nb, fc, st, proof, ch_out);
  WL_LAUNCH_CHECK();
}

}  // namespace wl
