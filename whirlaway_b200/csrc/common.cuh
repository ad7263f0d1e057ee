// Shared device helpers: error checks, extension-field reductions, lazy accumulators.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

#include "kb.cuh"

namespace wl {

struct CudaError : std::runtime_error {
  cudaError_t code;
  CudaError(cudaError_t c, const std::string& where)
      : std::runtime_error(where + ": " + cudaGetErrorString(c)), code(c) {}
};

#define WL_CUDA(expr)                                                        \
  do {                                                                       \
    cudaError_t e_ = (expr);                                                 \
    if (e_ != cudaSuccess) throw ::wl::CudaError(e_, std::string(#expr)); \
  } while (0)
// Every kernel launch in the library is followed by WL_LAUNCH_CHECK, which also counts it.
inline std::atomic<uint64_t>& launch_counter() {
  static std::atomic<uint64_t> n{0};
  return n;
}
#define WL_LAUNCH_CHECK()                      \
  do {                                         \
    ::wl::launch_counter().fetch_add(1);       \
    WL_CUDA(cudaGetLastError());               \
  } while (0)

using kb::ef;

#ifdef __CUDACC__
__device__ __forceinline__ ef shfl_down_ef(const ef& v, int d) {
  ef r;
#pragma unroll
  for (int i = 0; i < 8; i++) r.c[i] = __shfl_down_sync(0xffffffffu, v.c[i], d);
  return r;
}
__device__ __forceinline__ ef warp_reduce_ef(ef v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v = kb::ef_add(v, shfl_down_ef(v, d));
  return v;
}
// Sum over the whole block (blockDim.x * blockDim.y * blockDim.z <= 1024); the result
// is valid in thread 0. `scratch` holds 32 ef.
__device__ __forceinline__ ef block_reduce_ef(ef v, ef* scratch) {
  int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  int nthreads = blockDim.x * blockDim.y * blockDim.z;
  v = warp_reduce_ef(v);
  int lane = tid & 31, warp = tid >> 5;
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  if (warp == 0) {
    int nw = (nthreads + 31) >> 5;
    v = lane < nw ? scratch[lane] : kb::ef_zero();
    v = warp_reduce_ef(v);
  }
  return v;
}

// Lazy extension-field multiply-accumulate by base-field scalars. Each coordinate is a 64-bit
// running sum; flush() folds it with 2^32 = 2^25 - 2 (mod p) into hi * (2^25 - 2) + lo, one
// wide multiply-add, leaving it below 2^57 + 2^32, so that at most four more products (each
// below p^2, 4 p^2 = 2^64 - 2^58 + ...) keep it below 2^64. value() folds once more and
// makes the single Montgomery reduction (its input is below 4 p^2).
struct EfMacF {
  static constexpr uint32_t C32 = (1u << 25) - 2;  // 2^32 mod p
  uint64_t s[8];
  __device__ __forceinline__ void init() {
#pragma unroll
    for (int i = 0; i < 8; i++) s[i] = 0;
  }
  // starts from v (Montgomery form): v * 2^32 reduces to v, and is stored folded
  __device__ __forceinline__ void init_with(const ef& v) {
#pragma unroll
    for (int i = 0; i < 8; i++) s[i] = uint64_t(v.c[i]) * C32;
  }
  __device__ __forceinline__ void mac(const ef& a, uint32_t f) {
#pragma unroll
    for (int i = 0; i < 8; i++) s[i] += kb::wmul(a.c[i], f);
  }
  __device__ __forceinline__ void flush() {
#pragma unroll
    for (int i = 0; i < 8; i++) s[i] = uint64_t(uint32_t(s[i] >> 32)) * C32 + uint32_t(s[i]);
  }
  __device__ __forceinline__ ef value() {
    flush();
    ef r;
#pragma unroll
    for (int i = 0; i < 8; i++) r.c[i] = kb::redc(s[i]);
    return r;
  }
};

// Lazy extension x extension multiply-accumulate: acc += a * b in F[X]/(X^8 - 3). Coefficient
// k of a * b is sum_t a_t * b'_(k-t), b'_i = b_i for i >= 0 and 3 b_(i+8) for the wrapped
// terms; its 8 products go into the 64-bit running sum in two groups of four, each followed
// by the fold of EfMacF (so the sum stays below 2^64), and value() reduces once. Against a
// full product and an addition this saves the 16 reductions of every term.
struct EfMacE {
  uint64_t s[8];
  __device__ __forceinline__ void init() {
#pragma unroll
    for (int i = 0; i < 8; i++) s[i] = 0;
  }
  __device__ __forceinline__ static uint64_t fold(uint64_t v) {
    return uint64_t(uint32_t(v >> 32)) * EfMacF::C32 + uint32_t(v);
  }
  __device__ __forceinline__ void mac(const ef& a, const ef& b) {
    uint32_t b3[8];
#pragma unroll
    for (int j = 0; j < 8; j++) b3[j] = kb::add(kb::dbl(b.c[j]), b.c[j]);
#pragma unroll
    for (int k = 0; k < 8; k++) {
      uint64_t v = s[k];
#pragma unroll
      for (int t = 0; t < 4; t++) v += kb::wmul(a.c[t], t <= k ? b.c[k - t] : b3[k + 8 - t]);
      v = fold(v);
#pragma unroll
      for (int t = 4; t < 8; t++) v += kb::wmul(a.c[t], t <= k ? b.c[k - t] : b3[k + 8 - t]);
      s[k] = fold(v);
    }
  }
  __device__ __forceinline__ ef value() const {
    ef r;
#pragma unroll
    for (int i = 0; i < 8; i++) r.c[i] = kb::redc(fold(s[i]));
    return r;
  }
};
#endif

}  // namespace wl
