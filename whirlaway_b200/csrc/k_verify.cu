// Batched Merkle-path checks for the verifier (the GPU part of wl_verify_batch_device). The
// host replays each proof's transcript with its Merkle openings deferred (verify_air_proof
// with a deferral list); the openings of all proofs are then checked here, one thread per
// opening: the leaf sponge over the opened row (PaddingFreeSponge over Poseidon2-24, rate 16,
// 8 absorptions), then one 2-to-1 compression (Poseidon2-16) per level of its path, and the
// comparison with the root. The words are the proofs' canonical proof_data, so the
// permutations run in the canonical domain (p2_permute_fd), as the prover's trees are built.
#include "kernels.h"

namespace wl {

namespace {

constexpr int VERIFY_THREADS = 128;

__global__ void __launch_bounds__(VERIFY_THREADS) k_check_openings(const uint32_t* __restrict__ words,
                                                                   const OpeningCheck* __restrict__ ops, int n,
                                                                   const __grid_constant__ kb::P2ConstsFd<24> c24,
                                                                   const __grid_constant__ kb::P2ConstsFd<16> c16,
                                                                   uint8_t* __restrict__ ok) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const OpeningCheck op = ops[i];
  uint32_t s[24];
#pragma unroll
  for (int j = 0; j < 24; j++) s[j] = 0;
#pragma unroll 1
  for (int ch = 0; ch < 8; ch++) {
#pragma unroll
    for (int j = 0; j < 16; j++) s[j] = words[op.row + 16 * ch + j];
    kb::p2_permute_fd<24>(s, c24);
  }
  uint32_t cur[8];
#pragma unroll
  for (int j = 0; j < 8; j++) cur[j] = s[j];
#pragma unroll 1
  for (int l = 0; l < op.ll; l++) {
    const uint32_t* sib = words + op.path + size_t(l) * 8;
    uint32_t t[16];
    const bool right = (op.q >> l) & 1;
#pragma unroll
    for (int j = 0; j < 8; j++) {
      t[j] = right ? sib[j] : cur[j];
      t[8 + j] = right ? cur[j] : sib[j];
    }
    kb::p2_permute_fd<16>(t, c16);
#pragma unroll
    for (int j = 0; j < 8; j++) cur[j] = t[j];
  }
  bool same = true;
#pragma unroll
  for (int j = 0; j < 8; j++) same = same && cur[j] == words[op.root + j];
  ok[i] = same ? 1 : 0;
}

}  // namespace

void launch_check_openings(const uint32_t* words, const OpeningCheck* ops, int n, const kb::P24Consts& p24,
                           const kb::P16Consts& p16, uint8_t* ok, cudaStream_t s) {
  if (n <= 0) return;
  const kb::P2ConstsFd<24> c24 = kb::p2_consts_fd(p24);
  const kb::P2ConstsFd<16> c16 = kb::p2_consts_fd(p16);
  k_check_openings<<<(n + VERIFY_THREADS - 1) / VERIFY_THREADS, VERIFY_THREADS, 0, s>>>(words, ops, n, c24, c16, ok);
  WL_LAUNCH_CHECK();
}

}  // namespace wl
