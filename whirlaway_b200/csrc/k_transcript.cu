// Device-side Fiat-Shamir for the sumcheck rounds.
//
// A sumcheck round ends with a few extension-field sums (the round polynomial at a handful of
// points), which the prover interpolates, writes to the proof, absorbs into the
// DuplexChallenger<F, Poseidon16, 16, 8> and answers with a sampled challenge that the next
// fold uses (crates/sumcheck/src/prove.rs:190-222 for the zerocheck and product sumchecks;
// the WHIR folding sumcheck sends its three values directly). Done on the host, every round is
// a device-to-host round trip during which the device idles. Here the round is finished on the
// device exactly as the host would (same challenger semantics as HostChallenger: observations
// fill the rate and duplex at eight, samples pop from the end of the last squeeze) and the
// challenge stays in device memory for the fold, so the host enqueues a whole phase of rounds
// without waiting and reads the appended proof words, the challenges and the challenger state
// back once at its end. The finish itself (finish.cuh) runs either in the last block of the
// kernel that computed the round's sums (the fused fold-and-evaluate kernels) or, after the
// other evaluation kernels, in the single-block kernel below.
#include <algorithm>

#include "finish.cuh"
#include "kernels.h"

namespace wl {

namespace {

// One round's finish as its own kernel: the block reduces the partial rows, warp 0 finishes.
__global__ void __launch_bounds__(FIN_MAX_THREADS, 1) k_round_finish(int kind, const ef* __restrict__ partial, int nb,
                                                                     const FinArgs a) {
  fin_load(kind, a);
  fin_reduce_rows(partial, nb, fin_kind_sums_dev(kind));
  __syncthreads();
  if (threadIdx.x < 32) fin_round(kind, a);
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

int fin_kind_sums(int kind) { return kind == FIN_EQSC4 || kind == FIN_WHIR ? 3 : 2; }

int launch_reduce_wide(const ef* partial, int nb, int k, ef* out, int max_blocks, cudaStream_t s) {
  if (k < 1 || k > 32) throw std::invalid_argument("wide reduction of 1..32 sums");
  const int blocks = std::max(1, std::min(max_blocks, (nb + 63) / 64));
  k_reduce_wide<<<blocks, WIDE_THREADS, 0, s>>>(partial, nb, k, out);
  WL_LAUNCH_CHECK();
  return blocks;
}

void launch_round_finish(int kind, const ef* partial, int nb, const FinArgs& a, cudaStream_t s) {
  if (kind < FIN_EQSC4 || kind > FIN_WHIR) throw std::invalid_argument("round finish: unknown round kind");
  if ((kind == FIN_EQSC4 || kind == FIN_EQSC3) && (!a.req || !a.rinv))
    throw std::invalid_argument("round finish: eq-factor rounds need their eq challenges");
  k_round_finish<<<1, FIN_MAX_THREADS, 0, s>>>(kind, partial, nb, a);
  WL_LAUNCH_CHECK();
}

}  // namespace wl
