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
constexpr unsigned FULL = 0xffffffffu;

// A round's finish runs as one warp over little code: a finishing kernel executes each of its
// instructions only a few times, so straight-line code would spend most of its time fetching
// instructions. The permutation, the absorption and the extension-field products are rolled
// loops; the challenger lives in shared memory (lane 0 updates its buffers, lanes 0-15 the
// state), and every lane of warp 0 computes the same round values.
struct FinShared {
  DevChallenger ch;
  uint32_t rc[8][16];  // full-round constants: rounds 0-3 initial, 4-7 terminal
  uint32_t sample[8];
  ef red[3], scratch[12];
};

// a * b in F[X]/(X^8 - 3): kb::ef_mul behind a call, so that every product of a finish runs
// the same few hundred instructions from the instruction cache.
__device__ __noinline__ ef fin_mul(const ef a, const ef b) { return kb::ef_mul(a, b); }

__device__ __forceinline__ uint32_t m4_lanes(uint32_t a, int i) {
  const int base = i & ~3;
  const uint32_t b = __shfl_sync(FULL, a, base | ((i + 1) & 3), 16);
  const uint32_t c = __shfl_sync(FULL, a, base | ((i + 2) & 3), 16);
  const uint32_t d = __shfl_sync(FULL, a, base | ((i + 3) & 3), 16);
  // row i of circ(2, 3, 1, 1) within the chunk: 2a + 3b + c + d; then the sums over the chunks
  const uint32_t y = kb::add(kb::add(kb::add(a, b), kb::add(c, d)), kb::add(a, kb::dbl(b)));
  uint32_t t = kb::add(y, __shfl_xor_sync(FULL, y, 4, 16));
  t = kb::add(t, __shfl_xor_sync(FULL, t, 8, 16));
  return kb::add(y, t);
}

// Duplexing: Poseidon2-16 (Montgomery form, the values of kb::p2_permute<16>) of the state with
// the pending inputs written over its first words. Full rounds across 16 lanes (lane i and its
// mirror i + 16 hold word i), partial rounds on the whole state in every lane.
__device__ __noinline__ void fin_duplex(FinShared& fs, const kb::P16Consts& c) {
  const int lane = threadIdx.x & 31, i = lane & 15;
  uint32_t v = (i < 8 && i < fs.ch.in_len) ? fs.ch.in[i] : fs.ch.state[i];
  v = m4_lanes(v, i);
#pragma unroll 1
  for (int r = 0; r < 4; r++) v = m4_lanes(kb::cube(kb::add(v, fs.rc[r][i])), i);
  uint32_t s[16];
#pragma unroll
  for (int j = 0; j < 16; j++) s[j] = __shfl_sync(FULL, v, j, 16);
#pragma unroll 1
  for (int r = 0; r < kb::P16Consts::RP; r++) kb::internal_layer_with0<16>(s, kb::cube(kb::add(s[0], c.internal[r])));
  v = s[0];
#pragma unroll
  for (int j = 1; j < 16; j++) v = i == j ? s[j] : v;
#pragma unroll 1
  for (int r = 4; r < 8; r++) v = m4_lanes(kb::cube(kb::add(v, fs.rc[r][i])), i);
  __syncwarp();
  if (lane < 16) {
    fs.ch.state[i] = v;
    if (i < 8) fs.ch.out[i] = v;
  }
  if (lane == 0) {
    fs.ch.in_len = 0;
    fs.ch.out_len = 8;
  }
  __syncwarp();
}
// Transcript::add_ext: the value goes to the proof (word offset *plen) and into the challenger.
__device__ __noinline__ void fin_add_ext(FinShared& fs, const ef v, uint32_t* proof, uint32_t* plen,
                                         const kb::P16Consts& c) {
  const int lane = threadIdx.x & 31;
#pragma unroll 1
  for (int w = 0; w < 8; w++) {
    uint32_t x = v.c[0];
#pragma unroll
    for (int u = 1; u < 8; u++) x = w == u ? v.c[u] : x;
    if (lane == 0) {
      proof[*plen + w] = x;
      fs.ch.out_len = 0;
      fs.ch.in[fs.ch.in_len] = x;
      fs.ch.in_len++;
    }
    __syncwarp();
    if (fs.ch.in_len == 8) fin_duplex(fs, c);
  }
  *plen += 8;
}
__device__ __noinline__ ef fin_sample_ext(FinShared& fs, const kb::P16Consts& c) {
  const int lane = threadIdx.x & 31;
#pragma unroll 1
  for (int k = 0; k < 8; k++) {
    if (fs.ch.in_len || !fs.ch.out_len) fin_duplex(fs, c);
    if (lane == 0) {
      fs.ch.out_len--;
      fs.sample[k] = fs.ch.out[fs.ch.out_len];
    }
    __syncwarp();
  }
  ef e;
#pragma unroll
  for (int k = 0; k < 8; k++) e.c[k] = fs.sample[k];
  __syncwarp();
  return e;
}

// Block prologue of every finishing kernel: the challenger and the full-round constants into
// shared memory, and the `nsum` sums of nb interleaved partial rows (partial[row * nsum + z])
// into fs.red. Returns false for the threads that take no part in the finish (warps >= 1).
__device__ bool fin_begin(FinShared& fs, const DevRound* stp, const kb::P16Consts& c, const ef* __restrict__ partial,
                          int nb, int nsum) {
  const int tid = threadIdx.x;
  if (tid < 128) fs.rc[tid >> 4][tid & 15] = (tid >> 4) < 4 ? c.ext_init[tid] : c.ext_term[tid - 64];
  if (tid == 0) fs.ch = stp->ch;
  const int z = tid >> 7, t = tid & 127;
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
  if ((tid & 31) == 0) fs.scratch[tid >> 5] = acc;
  __syncthreads();
  if (t == 0 && z < nsum) {
    ef s = fs.scratch[z * 4];
    for (int w = 1; w < 4; w++) s = kb::ef_add(s, fs.scratch[z * 4 + w]);
    fs.red[z] = s;
  }
  __syncthreads();
  return tid < 32;
}
// Block epilogue: the round's challenge and the updated state (lane 0).
__device__ void fin_end(const FinShared& fs, DevRound* stp, DevRound& st, const ef& chal, ef* ch_out) {
  if ((threadIdx.x & 31) == 0) {
    st.ch = fs.ch;
    ch_out[st.round] = chal;
    st.round++;
    *stp = st;
  }
}
__device__ ef fin_poly_eval(const ef* p, int n, const ef& x) {
  ef r = kb::ef_zero();
#pragma unroll 1
  for (int i = n - 1; i >= 0; i--) r = kb::ef_add(fin_mul(r, x), p[i]);
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
  __shared__ FinShared fs;
  __shared__ ef e[NPTS], p[NPTS + 1];
  if (!fin_begin(fs, stp, fc.p16, partial, nb, NPTS - 1)) return;
  const int lane = threadIdx.x;
  DevRound st = *stp;
  const ef one = kb::ef_one();
  const ef omr = kb::ef_sub(one, r);
  if (lane == 0) {
    e[0] = fin_mul(fs.red[0], st.mmf);
    for (int i = 2; i < NPTS; i++) e[i] = fin_mul(fs.red[i - 1], st.mmf);
    e[1] = fin_mul(kb::ef_sub(st.sum, fin_mul(e[0], omr)), rinv);
    const ef lin = kb::ef_sub(kb::ef_add(r, r), one);  // (1 - r) + lin X
    for (int k = 0; k <= NPTS; k++) p[k] = kb::ef_zero();
    for (int k = 0; k < NPTS; k++) {
      ef q = kb::ef_zero();
      for (int i = 0; i < NPTS; i++) q = kb::ef_add(q, kb::ef_mul_f(e[i], fc.basis[NPTS - 3][i][k]));
      p[k] = kb::ef_add(p[k], fin_mul(q, omr));
      p[k + 1] = kb::ef_add(p[k + 1], fin_mul(q, lin));
    }
  }
  __syncwarp();
  uint32_t plen = st.proof_len;
#pragma unroll 1
  for (int k = 0; k <= NPTS; k++) fin_add_ext(fs, p[k], proof, &plen, fc.p16);
  const ef c = fin_sample_ext(fs, fc.p16);
  st.proof_len = plen;
  if (lane == 0) {
    st.sum = fin_poly_eval(p, NPTS + 1, c);
    st.mmf = fin_mul(kb::ef_add(fin_mul(omr, kb::ef_sub(one, c)), fin_mul(r, c)), st.mmf);
  }
  fin_end(fs, stp, st, c, ch_out);
}

// Round of the product sumcheck (the inner sumcheck): sums at 0 and 2, the value at 1 from the
// claim; the round polynomial (3 coefficients) interpolates 0, 1, 2.
__global__ void __launch_bounds__(FIN_THREADS, 1) k_prod_round_finish(const ef* __restrict__ partial, int nb,
                                                                      const __grid_constant__ FinishConsts fc,
                                                                      DevRound* __restrict__ stp,
                                                                      uint32_t* __restrict__ proof,
                                                                      ef* __restrict__ ch_out) {
  __shared__ FinShared fs;
  __shared__ ef p[3];
  if (!fin_begin(fs, stp, fc.p16, partial, nb, 2)) return;
  const int lane = threadIdx.x;
  DevRound st = *stp;
  if (lane == 0) {
    const ef y[3] = {fs.red[0], kb::ef_sub(st.sum, fs.red[0]), fs.red[1]};
    for (int k = 0; k < 3; k++) {
      ef v = kb::ef_zero();
      for (int i = 0; i < 3; i++) v = kb::ef_add(v, kb::ef_mul_f(y[i], fc.basis[0][i][k]));
      p[k] = v;
    }
  }
  __syncwarp();
  uint32_t plen = st.proof_len;
#pragma unroll 1
  for (int k = 0; k < 3; k++) fin_add_ext(fs, p[k], proof, &plen, fc.p16);
  const ef c = fin_sample_ext(fs, fc.p16);
  st.proof_len = plen;
  if (lane == 0) st.sum = fin_poly_eval(p, 3, c);
  fin_end(fs, stp, st, c, ch_out);
}

// Round of the WHIR folding sumcheck: the three values h(0), h(1), h(2) go to the proof as
// they are; the next claim is h(r) by quadratic interpolation on 0, 1, 2.
__global__ void __launch_bounds__(FIN_THREADS, 1) k_whir_round_finish(const ef* __restrict__ partial, int nb,
                                                                      const __grid_constant__ FinishConsts fc,
                                                                      DevRound* __restrict__ stp,
                                                                      uint32_t* __restrict__ proof,
                                                                      ef* __restrict__ ch_out) {
  __shared__ FinShared fs;
  if (!fin_begin(fs, stp, fc.p16, partial, nb, 3)) return;
  DevRound st = *stp;
  uint32_t plen = st.proof_len;
#pragma unroll 1
  for (int k = 0; k < 3; k++) fin_add_ext(fs, fs.red[k], proof, &plen, fc.p16);
  const ef r = fin_sample_ext(fs, fc.p16);
  st.proof_len = plen;
  if (threadIdx.x == 0) {
    // h(r) = h0 (r-1)(r-2)/2 - h1 r (r-2) + h2 r (r-1)/2
    const ef rm1 = kb::ef_sub_f(r, fc.one), rm2 = kb::ef_sub_f(r, fc.two);
    const ef a = kb::ef_mul_f(fin_mul(fin_mul(fs.red[0], rm1), rm2), fc.inv2);
    const ef b = fin_mul(fin_mul(fs.red[1], r), rm2);
    const ef c = kb::ef_mul_f(fin_mul(fin_mul(fs.red[2], r), rm1), fc.inv2);
    st.sum = kb::ef_add(kb::ef_sub(a, b), c);
  }
  fin_end(fs, stp, st, r, ch_out);
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
