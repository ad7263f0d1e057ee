// Integer-pipe throughput probes, built as their own library (libwl_probe.so) for the
// benchmark; the prover library does not contain them. All run from registers only (no memory
// traffic besides one store per thread). The raw 32-bit multiply probes (mul.lo, mul.hi) give
// the hardware ceiling the modular arithmetic is measured against: a Montgomery product takes
// two of each. Independent chains of Montgomery products and back-to-back Poseidon2-24
// permutations (the canonical-domain form the Merkle leaves use) are diagnostics beside it.
#include <cuda_runtime.h>

#include <algorithm>

#include "../host.h"

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

// Raw 32-bit multiply throughput (mul.lo or mul.hi), eight independent chains per thread.
template <bool HI>
__global__ void k_probe_mul(uint32_t seed, int iters, uint32_t* out) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t a[PROBE_CHAINS];
  const uint32_t b = (seed ^ tid) | 0x80000001u;
#pragma unroll
  for (int i = 0; i < PROBE_CHAINS; i++) a[i] = seed * 2654435761u + tid * 97u + i * 131u;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int i = 0; i < PROBE_CHAINS; i++) {
      if (HI)
        asm volatile("mul.hi.u32 %0, %0, %1;" : "+r"(a[i]) : "r"(b));
      else
        asm volatile("mul.lo.u32 %0, %0, %1;" : "+r"(a[i]) : "r"(b));
    }
  }
  uint32_t x = 0;
#pragma unroll
  for (int i = 0; i < PROBE_CHAINS; i++) x ^= a[i];
  out[tid] = x;
}

__global__ void k_probe_p24(const __grid_constant__ kb::P2ConstsFd<24> c, int iters, uint32_t* out) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t s[24];
#pragma unroll
  for (int i = 0; i < 24; i++) s[i] = (tid * 24u + i) % kb::P;
  for (int it = 0; it < iters; it++) kb::p2_permute_fd<24>(s, c);
  uint32_t x = 0;
#pragma unroll
  for (int i = 0; i < 24; i++) x ^= s[i];
  out[tid] = x;
}

// Best of `reps` timed launches (after one untimed launch), in milliseconds.
template <class Launch>
float time_best(cudaStream_t s, Launch&& launch, int reps, cudaError_t& err) {
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  launch();
  float best = 1e30f;
  for (int r = 0; r < reps; r++) {
    cudaEventRecord(a, s);
    launch();
    cudaEventRecord(b, s);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    best = std::min(best, ms);
  }
  err = cudaGetLastError();
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return best;
}

}  // namespace

// Montgomery products per second and Poseidon2-24 permutations per second on `device`;
// `constants` is a workload constants blob (its Poseidon24 part is used). 0 on success, else
// the CUDA error code.
extern "C" int wlp_int_peaks(int device, const uint32_t* constants, double* modmul_per_s, double* p24_per_s) {
  cudaError_t err = cudaSetDevice(device);
  if (err != cudaSuccess) return int(err);
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaStream_t s;
  if ((err = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) != cudaSuccess) return int(err);
  const int blocks = sms * 8;
  uint32_t* out = nullptr;
  if ((err = cudaMalloc(&out, sizeof(uint32_t) * blocks * 256)) != cudaSuccess) {
    cudaStreamDestroy(s);
    return int(err);
  }
  {
    const int threads = 256, iters = 4096;
    const float ms = time_best(s, [&] { k_probe_modmul<<<blocks, threads, 0, s>>>(12345u, iters, out); }, 5, err);
    if (modmul_per_s) *modmul_per_s = double(blocks) * threads * iters * PROBE_CHAINS / (ms * 1e-3);
  }
  if (err == cudaSuccess) {
    const int threads = 128, iters = 32;
    const kb::P2ConstsFd<24> cc =
        kb::p2_consts_fd(wl::perm_consts_from<24>(constants + wl::N_AIR_CONSTS + wl::N_P16_CONSTS));
    const float ms = time_best(s, [&] { k_probe_p24<<<blocks, threads, 0, s>>>(cc, iters, out); }, 5, err);
    if (p24_per_s) *p24_per_s = double(blocks) * threads * iters / (ms * 1e-3);
  }
  cudaFree(out);
  cudaStreamDestroy(s);
  return int(err);
}

// Raw 32-bit integer multiplies per second on `device` (mul.lo and mul.hi, each from
// independent register chains): the hardware's integer multiply throughput, with no modular
// arithmetic around it. 0 on success, else the CUDA error code.
extern "C" int wlp_mul_peaks(int device, double* mul_lo_per_s, double* mul_hi_per_s) {
  cudaError_t err = cudaSetDevice(device);
  if (err != cudaSuccess) return int(err);
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaStream_t s;
  if ((err = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) != cudaSuccess) return int(err);
  const int blocks = sms * 8, threads = 256, iters = 8192;
  uint32_t* out = nullptr;
  if ((err = cudaMalloc(&out, sizeof(uint32_t) * blocks * threads)) != cudaSuccess) {
    cudaStreamDestroy(s);
    return int(err);
  }
  const double n = double(blocks) * threads * iters * PROBE_CHAINS;
  float ms = time_best(s, [&] { k_probe_mul<false><<<blocks, threads, 0, s>>>(7u, iters, out); }, 5, err);
  if (mul_lo_per_s) *mul_lo_per_s = n / (ms * 1e-3);
  if (err == cudaSuccess) {
    ms = time_best(s, [&] { k_probe_mul<true><<<blocks, threads, 0, s>>>(7u, iters, out); }, 5, err);
    if (mul_hi_per_s) *mul_hi_per_s = n / (ms * 1e-3);
  }
  cudaFree(out);
  cudaStreamDestroy(s);
  return int(err);
}
