// Zerocheck kernels for AIRs given as constraint programs (air_program.h): an interpreter over a
// per-thread register file of PROG_MAX_REGS values, one thread per row of the current cube,
// blockIdx.y the evaluation point. The program's instructions are read by every thread of a
// warp at once (one broadcast load each); the register file lives in local memory. An
// operand that is a constant comes as an immediate (MULC, ADDC): over the extension a product
// by a base-field element instead of a full extension product.
//
// Round 0 (univariate skip over the top k variables) reads the witness: column c's value at
// point z and row x of the subcube is sum_j L_j(z) col[j S + x] over the 2^k rows of its coset,
// of the column's up version (row N - 1 repeats row N - 2) or its down version (row i reads row
// i + 1, row N - 1 itself), as crates/air/src/utils.rs:140-160 builds them. Rounds >= 1 read the
// 2W folded extension columns (up versions, then down versions); the value at z is
// lo + z (hi - lo). Every row's batched constraint sum_i alpha^i C_i is weighted by the eq
// table and summed per block.
#include <algorithm>

#include "air_program.h"
#include "kernels.h"

namespace wl {

namespace {

using kb::ef_add;
using kb::ef_mul;
using kb::ef_mul_f;
using kb::ef_sub;
using kb::ef_zero;

constexpr int PROG_THREADS = 128;

__device__ __forceinline__ void prog_decode(uint2 in, int& op, int& dst, uint32_t& a, int& b) {
  op = int(in.x & 0xffu);
  dst = int((in.x >> 8) & 0xffu);
  a = in.x >> 16;
  b = int(in.y);
}

__global__ void __launch_bounds__(PROG_THREADS) k_prog_zc0(const uint32_t* __restrict__ wit,
                                                           const uint32_t* __restrict__ pre, int P, int log_n, int k,
                                                           const uint2* __restrict__ code, int n_code,
                                                           const uint32_t* __restrict__ consts,
                                                           const uint32_t* __restrict__ lw, const ef* __restrict__ eq,
                                                           const ef* __restrict__ alphas, ef* __restrict__ partial) {
  __shared__ ef scratch[32];
  __shared__ uint32_t w_s[16];
  const int zi = blockIdx.y, nsk = 1 << k;
  if (threadIdx.x < nsk) w_s[threadIdx.x] = lw[zi * nsk + threadIdx.x];
  __syncthreads();
  const size_t N = size_t(1) << log_n, S = N >> k;
  uint32_t reg[PROG_MAX_REGS];
  ef tot = ef_zero();
  for (size_t x = size_t(blockIdx.x) * blockDim.x + threadIdx.x; x < S; x += size_t(gridDim.x) * blockDim.x) {
    ef acc = ef_zero();
    int ci = 0;
    for (int i = 0; i < n_code; i++) {
      int op, dst, b;
      uint32_t a;
      prog_decode(__ldg(code + i), op, dst, a, b);
      if (op == PROG_UP || op == PROG_DOWN) {
        const uint32_t* col = int(a) < P ? pre + size_t(a) * N : wit + size_t(int(a) - P) * N;
        uint64_t g[4] = {0, 0, 0, 0};  // at most four products of values below p per group
        for (int j = 0; j < nsk; j++) {
          const size_t r = size_t(j) * S + x;
          const size_t src = op == PROG_UP ? (r == N - 1 ? N - 2 : r) : (r == N - 1 ? r : r + 1);
          g[j & 3] += kb::wmul(w_s[j], __ldg(col + src));
        }
        reg[dst] = kb::add(kb::add(kb::redc(g[0]), kb::redc(g[1])), kb::add(kb::redc(g[2]), kb::redc(g[3])));
      } else if (op == PROG_CONST) {
        reg[dst] = __ldg(consts + a);
      } else if (op == PROG_ADD) {
        const uint32_t u = reg[a], v = reg[b];
        reg[dst] = kb::add(u, v);
      } else if (op == PROG_SUB) {
        const uint32_t u = reg[a], v = reg[b];
        reg[dst] = kb::sub(u, v);
      } else if (op == PROG_MUL) {
        const uint32_t u = reg[a], v = reg[b];
        reg[dst] = kb::mul(u, v);
      } else if (op == PROG_MULC) {
        reg[dst] = kb::mul(reg[a], uint32_t(b));
      } else if (op == PROG_ADDC) {
        reg[dst] = kb::add(reg[a], uint32_t(b));
      } else {  // PROG_EMIT
        acc = ef_add(acc, ef_mul_f(alphas[ci++], reg[a]));
      }
    }
    tot = ef_add(tot, ef_mul(acc, eq[x]));
  }
  tot = block_reduce_ef(tot, scratch);
  if (threadIdx.x == 0) partial[size_t(blockIdx.x) * gridDim.y + zi] = tot;
}

// The 2W up/down columns folded over the skipped variables: out[c * S + x] =
// sum_j sel[j] ud_c[j S + x] (c < W: up versions, c >= W: down versions). Columns below P are
// the preprocessed ones (pre), the others the witness's (wit, column c - P).
__global__ void k_prog_fold0(const uint32_t* __restrict__ wit, const uint32_t* __restrict__ pre, int P, int log_n,
                             int k, int W, const ef* __restrict__ sel, ef* __restrict__ out) {
  __shared__ ef s_s[16];
  const int nsk = 1 << k;
  if (threadIdx.x < nsk) s_s[threadIdx.x] = sel[threadIdx.x];
  __syncthreads();
  const size_t N = size_t(1) << log_n, S = N >> k;
  const int c = blockIdx.y;
  const bool up = c < W;
  const int cc = up ? c : c - W;
  const uint32_t* col = cc < P ? pre + size_t(cc) * N : wit + size_t(cc - P) * N;
  for (size_t x = size_t(blockIdx.x) * blockDim.x + threadIdx.x; x < S; x += size_t(gridDim.x) * blockDim.x) {
    ef acc = ef_zero();
    for (int j = 0; j < nsk; j++) {
      const size_t r = size_t(j) * S + x;
      const size_t src = up ? (r == N - 1 ? N - 2 : r) : (r == N - 1 ? r : r + 1);
      acc = ef_add(acc, ef_mul_f(s_s[j], __ldg(col + src)));
    }
    out[size_t(c) * S + x] = acc;
  }
}

__global__ void __launch_bounds__(PROG_THREADS) k_prog_zc_ef(const ef* __restrict__ cols, int m, int W,
                                                             const uint2* __restrict__ code, int n_code,
                                                             const uint32_t* __restrict__ consts,
                                                             const ef* __restrict__ eq, const ef* __restrict__ alphas,
                                                             ef* __restrict__ partial) {
  __shared__ ef scratch[32];
  const int zi = blockIdx.y, z = zi == 0 ? 0 : zi + 1;  // points 0, 2, 3, ..
  const uint32_t zf = kb::to_mont(uint32_t(z));
  const size_t L = size_t(1) << m, half = L >> 1;
  ef reg[PROG_MAX_REGS];
  ef tot = ef_zero();
  for (size_t x = size_t(blockIdx.x) * blockDim.x + threadIdx.x; x < half; x += size_t(gridDim.x) * blockDim.x) {
    ef acc = ef_zero();
    int ci = 0;
    for (int i = 0; i < n_code; i++) {
      int op, dst, b;
      uint32_t a;
      prog_decode(__ldg(code + i), op, dst, a, b);
      if (op == PROG_UP || op == PROG_DOWN) {
        const ef* col = cols + size_t(op == PROG_UP ? a : a + W) * L;
        const ef lo = col[x];
        reg[dst] = z == 0 ? lo : ef_add(lo, ef_mul_f(ef_sub(col[x + half], lo), zf));
      } else if (op == PROG_CONST) {
        ef v = ef_zero();
        v.c[0] = __ldg(consts + a);
        reg[dst] = v;
      } else if (op == PROG_ADD) {
        const ef u = reg[a], v = reg[b];
        reg[dst] = ef_add(u, v);
      } else if (op == PROG_SUB) {
        const ef u = reg[a], v = reg[b];
        reg[dst] = ef_sub(u, v);
      } else if (op == PROG_MUL) {
        const ef u = reg[a], v = reg[b];
        reg[dst] = ef_mul(u, v);
      } else if (op == PROG_MULC) {
        reg[dst] = ef_mul_f(reg[a], uint32_t(b));
      } else if (op == PROG_ADDC) {
        ef v = reg[a];
        v.c[0] = kb::add(v.c[0], uint32_t(b));
        reg[dst] = v;
      } else {  // PROG_EMIT
        acc = ef_add(acc, ef_mul(alphas[ci++], reg[a]));
      }
    }
    tot = ef_add(tot, ef_mul(acc, eq[x]));
  }
  tot = block_reduce_ef(tot, scratch);
  if (threadIdx.x == 0) partial[size_t(blockIdx.x) * gridDim.y + zi] = tot;
}

// The batched column of the inner phase over W columns: out[i] = sum_c eqc[c] wit[c N + i].
__global__ void k_batch_cols_generic(const uint32_t* __restrict__ wit, int log_n, int W, const ef* __restrict__ eqc,
                                     ef* __restrict__ out) {
  const size_t N = size_t(1) << log_n;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N; i += size_t(gridDim.x) * blockDim.x) {
    ef acc = ef_zero();
    for (int c = 0; c < W; c++) acc = ef_add(acc, ef_mul_f(eqc[c], __ldg(wit + size_t(c) * N + i)));
    out[i] = acc;
  }
}

int prog_sm_count() {
  int dev = 0, n = 0;
  WL_CUDA(cudaGetDevice(&dev));
  WL_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
  return n;
}

}  // namespace

int prog_zc_blocks(size_t rows) {
  return (int)std::max<size_t>(1, std::min<size_t>((rows + PROG_THREADS - 1) / PROG_THREADS, size_t(prog_sm_count()) * 4));
}

void launch_prog_zc0(const uint32_t* wit, const uint32_t* pre, int P, int log_n, int k, const uint2* code, int n_code,
                     const uint32_t* consts, int nz, const uint32_t* lw, const ef* eq, const ef* alphas, ef* partial,
                     cudaStream_t s) {
  if (k < 1 || k > 4 || k >= log_n) throw std::invalid_argument("program zerocheck: 1 <= skips <= 4, below log_n");
  if (nz < 1) return;
  const dim3 grid(prog_zc_blocks(size_t(1) << (log_n - k)), nz);
  k_prog_zc0<<<grid, PROG_THREADS, 0, s>>>(wit, pre, P, log_n, k, code, n_code, consts, lw, eq, alphas, partial);
  WL_LAUNCH_CHECK();
}

void launch_prog_fold0(const uint32_t* wit, const uint32_t* pre, int P, int log_n, int k, int W, const ef* sel, ef* out,
                       cudaStream_t s) {
  const size_t S = size_t(1) << (log_n - k);
  const dim3 grid((unsigned)std::max<size_t>(1, std::min<size_t>((S + 255) / 256, 1024)), 2 * W);
  k_prog_fold0<<<grid, 256, 0, s>>>(wit, pre, P, log_n, k, W, sel, out);
  WL_LAUNCH_CHECK();
}

void launch_prog_zc_ef(const ef* cols, int m, int W, const uint2* code, int n_code, const uint32_t* consts, int npts,
                       const ef* eq, const ef* alphas, ef* partial, cudaStream_t s) {
  if (m < 1) throw std::invalid_argument("program zerocheck: a round needs at least one variable");
  const dim3 grid(prog_zc_blocks(size_t(1) << (m - 1)), npts);
  k_prog_zc_ef<<<grid, PROG_THREADS, 0, s>>>(cols, m, W, code, n_code, consts, eq, alphas, partial);
  WL_LAUNCH_CHECK();
}

void launch_batch_cols_generic(const uint32_t* wit, int log_n, int W, const ef* eqc, ef* out, cudaStream_t s) {
  const size_t N = size_t(1) << log_n;
  const unsigned blocks = (unsigned)std::max<size_t>(1, std::min<size_t>((N + 255) / 256, size_t(prog_sm_count()) * 8));
  k_batch_cols_generic<<<blocks, 256, 0, s>>>(wit, log_n, W, eqc, out);
  WL_LAUNCH_CHECK();
}

}  // namespace wl
