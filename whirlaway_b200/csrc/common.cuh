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

// Lazy extension-field multiply-accumulate by base-field scalars: at most four products
// per coordinate are summed in 64 bits before a Montgomery reduction.
struct EfMacF {
  uint64_t s[8];
  ef acc;
  __device__ __forceinline__ void init() {
#pragma unroll
    for (int i = 0; i < 8; i++) s[i] = 0;
    acc = kb::ef_zero();
  }
  __device__ __forceinline__ void mac(const ef& a, uint32_t f) {
#pragma unroll
    for (int i = 0; i < 8; i++) s[i] += kb::wmul(a.c[i], f);
  }
  __device__ __forceinline__ void flush() {
#pragma unroll
    for (int i = 0; i < 8; i++) {
      acc.c[i] = kb::add(acc.c[i], kb::redc(s[i]));
      s[i] = 0;
    }
  }
};
#endif

}  // namespace wl
