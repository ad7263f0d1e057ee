// Throughput probes: the integer-pipe ceilings the kernels are measured against. Both run
// from registers only (no memory traffic besides one store per thread): independent chains
// of Montgomery products, and back-to-back Poseidon2-24 permutations (the canonical-domain
// form the Merkle leaves use).
#include "prover.h"

namespace wl {

namespace {
constexpr int PROBE_CHAINS = 8;

__global__ void k_probe_modmul(uint32_t seed, int iters, uint32_t* out) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t a[PROBE_CHAINS], b[PROBE_CHAINS];
#pragma unroll
  for (int i = 0; i < PROBE_CHAINS; i++) {
    a[i] = (seed * 2654435761u + tid * 97u + i * 131u) % kb::P;
    b[i] = (seed + tid + i * 7919u) % kb::P | 1u;
  }
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int i = 0; i < PROBE_CHAINS; i++) a[i] = kb::mul(a[i], b[i]);
  }
  uint32_t x = 0;
#pragma unroll
  for (int i = 0; i < PROBE_CHAINS; i++) x ^= a[i];
  out[tid] = x;
}

__global__ void k_probe_p24(const __grid_constant__ kb::P24Consts c, int iters, uint32_t* out) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t s[24];
#pragma unroll
  for (int i = 0; i < 24; i++) s[i] = (tid * 24u + i) % kb::P;
  for (int it = 0; it < iters; it++) kb::p2_permute_fq<24>(s, c);
  uint32_t x = 0;
#pragma unroll
  for (int i = 0; i < 24; i++) x ^= s[i];
  out[tid] = x;
}

int sm_count(int device) {
  int n = 0;
  WL_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device));
  return n;
}

template <class Launch>
double time_best(Context& ctx, Launch&& launch, int reps) {
  cudaEvent_t a = ctx.take_event(), b = ctx.take_event();
  launch();  // warm-up
  double best = 1e30;
  for (int r = 0; r < reps; r++) {
    WL_CUDA(cudaEventRecord(a, ctx.stream));
    launch();
    WL_CUDA(cudaEventRecord(b, ctx.stream));
    WL_CUDA(cudaEventSynchronize(b));
    float ms = 0;
    WL_CUDA(cudaEventElapsedTime(&ms, a, b));
    best = std::min(best, double(ms));
  }
  ctx.event_pool.push_back(a);
  ctx.event_pool.push_back(b);
  return best;
}
}  // namespace

double bench_modmul_per_s(Context& ctx) {
  const int blocks = sm_count(ctx.device) * 8, threads = 256, iters = 4096;
  DBuf out(sizeof(uint32_t) * blocks * threads, ctx.stream);
  double ms = time_best(ctx, [&] {
    k_probe_modmul<<<blocks, threads, 0, ctx.stream>>>(12345u, iters, out.as<uint32_t>());
    WL_LAUNCH_CHECK();
  }, 5);
  return double(blocks) * threads * iters * PROBE_CHAINS / (ms * 1e-3);
}

double bench_p24_per_s(Context& ctx, const kb::P24Consts& c) {
  const int blocks = sm_count(ctx.device) * 8, threads = 128, iters = 32;
  DBuf out(sizeof(uint32_t) * blocks * threads, ctx.stream);
  const kb::P24Consts cc = kb::p2_consts_canonical(c);
  double ms = time_best(ctx, [&] {
    k_probe_p24<<<blocks, threads, 0, ctx.stream>>>(cc, iters, out.as<uint32_t>());
    WL_LAUNCH_CHECK();
  }, 5);
  return double(blocks) * threads * iters / (ms * 1e-3);
}

}  // namespace wl
