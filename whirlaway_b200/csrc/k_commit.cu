// Reed-Solomon encoding, Merkle hashing and grinding kernels (the work of whir-p3's
// CommitmentWriter::commit and EvalsDft, reached from crates/air/src/prove.rs:82-91,
// and of the DuplexChallenger grinding behind pow_grinding).
//
// LDE. For one commitment every column of the codeword matrix is the evaluation, on the
// subgroup of order 2^(L+rho), of a polynomial whose monomial coefficients are the Moebius
// transform of a 2^L-long slice of the evaluation table, read in bit-reversed exponent
// order. A radix-2 decimation-in-time NTT takes exactly that bit-reversed input, so the
// Moebius step of the variable at stage t is fused into stage t's butterfly (v <- v - u
// before u +- w v). Zero padding for the rate makes the first rho stages plain copies, so
// the first pass replicates each input value 2^rho times and starts at stage rho + 1.
// Stages run in shared-memory passes of up to 2^11 points over tiles of 8 columns; the
// second pass works in place on the output, whose rows are the Merkle leaves.
#include <algorithm>

#include "kernels.h"

namespace wl {

namespace {
constexpr int CT = 8;         // columns per tile
constexpr int MAXB = 11;      // log2 points per shared-memory pass
constexpr int NTT_THREADS = 512;

// Shared-memory tile: CT columns of 2^B points, column-major with one word of padding.
__device__ __forceinline__ uint32_t sidx(uint32_t col, uint32_t i, int B) { return col * ((1u << B) + 1) + i; }

// One fused Moebius + DIT stage on local bit tl. The twiddle exponent of a pair is its
// global index modulo 2^(t-1): lo_global plus the local bits below tl shifted by lo_bits.
__device__ __forceinline__ void butterfly_stage(uint32_t* sm, int B, int tl, int t, uint32_t lo_global, int lo_bits,
                                                const uint32_t* __restrict__ tw) {
  const uint32_t hl = 1u << tl;
  const uint32_t npairs = 1u << (B - 1);
  for (uint32_t bf = threadIdx.x; bf < (uint32_t)CT * npairs; bf += blockDim.x) {
    uint32_t col = bf / npairs, m = bf % npairs;
    uint32_t a = ((m >> tl) << (tl + 1)) | (m & (hl - 1));
    uint32_t twi = lo_global + ((m & (hl - 1)) << lo_bits);
    uint32_t w = tw[twi << (24 - t)];
    uint32_t ia = sidx(col, a, B), ib = sidx(col, a + hl, B);
    uint32_t u = sm[ia], v = sm[ib];
    v = kb::sub(v, u);
    uint32_t wv = kb::mul(w, v);
    sm[ia] = kb::add(u, wv);
    sm[ib] = kb::sub(u, wv);
  }
}

// First pass: points i of block blk (2^B of them) read source entry s = i >> rho, which
// realises the zero-padded stages 1..rho as copies; then stages rho+1..B.
__global__ void k_ntt_first(LdeSource in, int B, uint32_t* __restrict__ out, const uint32_t* __restrict__ tw) {
  extern __shared__ uint32_t sm[];
  const int tile = blockIdx.y;
  const size_t i0 = size_t(blockIdx.x) << B;
  const uint32_t npts = 1u << B;
  const size_t col_block = size_t(in.elem) << in.L;
  for (uint32_t idx = threadIdx.x; idx < (uint32_t)CT * npts; idx += blockDim.x) {
    uint32_t col, il;
    if (in.elem == 1) { il = idx % npts; col = idx / npts; }
    else { col = idx % CT; il = idx / CT; }
    uint32_t gcol = tile * CT + col;
    size_t s = (i0 + il) >> in.rho;
    size_t addr = (gcol / in.elem) * col_block + (gcol % in.elem) + s * in.elem;
    sm[sidx(col, il, B)] = (gcol < (uint32_t)in.n_cols && addr < in.src_len) ? in.src[addr] : 0u;
  }
  __syncthreads();
  for (int t = in.rho + 1; t <= B; t++) {
    butterfly_stage(sm, B, t - 1, t, 0, 0, tw);
    __syncthreads();
  }
  for (uint32_t idx = threadIdx.x; idx < (uint32_t)CT * npts; idx += blockDim.x) {
    uint32_t col = idx % CT, il = idx / CT;
    uint32_t gcol = tile * CT + col;
    if (gcol < (uint32_t)in.n_cols) out[(i0 + il) * in.n_cols + gcol] = sm[sidx(col, il, B)];
  }
}

// Later pass, in place: points i = lo + (j << B0) + (hi << (B0 + Bp)), stages B0+1..B0+Bp
// (stages up to rho are copies and are skipped).
__global__ void k_ntt_mid(uint32_t* __restrict__ data, int n_cols, int B0, int Bp, int rho,
                          const uint32_t* __restrict__ tw) {
  extern __shared__ uint32_t sm[];
  const int tile = blockIdx.y;
  const size_t g = blockIdx.x;
  const uint32_t lo = uint32_t(g & ((size_t(1) << B0) - 1));
  const size_t hi = g >> B0;
  auto row_of = [&](uint32_t j) -> size_t { return lo + (size_t(j) << B0) + (hi << (B0 + Bp)); };
  const uint32_t npts = 1u << Bp;
  for (uint32_t idx = threadIdx.x; idx < (uint32_t)CT * npts; idx += blockDim.x) {
    uint32_t col = idx % CT, j = idx / CT;
    uint32_t gcol = tile * CT + col;
    sm[sidx(col, j, Bp)] = gcol < (uint32_t)n_cols ? data[row_of(j) * n_cols + gcol] : 0u;
  }
  __syncthreads();
  for (int tl = 0; tl < Bp; tl++) {
    int t = B0 + 1 + tl;
    if (t <= rho) continue;
    butterfly_stage(sm, Bp, tl, t, lo, B0, tw);
    __syncthreads();
  }
  for (uint32_t idx = threadIdx.x; idx < (uint32_t)CT * npts; idx += blockDim.x) {
    uint32_t col = idx % CT, j = idx / CT;
    uint32_t gcol = tile * CT + col;
    if (gcol < (uint32_t)n_cols) data[row_of(j) * n_cols + gcol] = sm[sidx(col, j, Bp)];
  }
}

__device__ uint32_t pow_dev(uint32_t a, uint32_t e) {
  uint32_t r = kb::R_MOD_P;
  while (e) {
    if (e & 1) r = kb::mul(r, a);
    a = kb::mul(a, a);
    e >>= 1;
  }
  return r;
}
__global__ void k_twiddles(uint32_t* tw, uint32_t w24) {
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < (1u << 23)) tw[j] = pow_dev(w24, j);
}

constexpr int LEAF_ROWS = 64;
constexpr int LEAF_PAD = 129;

__global__ void k_leaf_hash(const uint32_t* __restrict__ lde, size_t rows, int n_cols, int log_elem,
                            const __grid_constant__ kb::P24Consts c, uint32_t* __restrict__ dig) {
  __shared__ uint32_t sm[LEAF_ROWS * LEAF_PAD];
  const size_t row0 = size_t(blockIdx.x) * LEAF_ROWS;
  for (uint32_t idx = threadIdx.x; idx < LEAF_ROWS * 128; idx += blockDim.x) {
    uint32_t r = idx / 128, col = idx % 128;
    size_t row = row0 + r;
    sm[r * LEAF_PAD + col] = (col < (uint32_t)n_cols && row < rows) ? lde[row * n_cols + col] : 0u;
  }
  __syncthreads();
  const int t = threadIdx.x;
  if (t >= LEAF_ROWS || row0 + t >= rows) return;
  uint32_t* r = sm + t * LEAF_PAD;
  for (int b = log_elem; b < 7; b++) {
    int h = 1 << b;
    for (int i = 0; i < 128; i++)
      if (!(i & h)) r[i + h] = kb::sub(r[i + h], r[i]);
  }
  uint32_t st[24];
#pragma unroll
  for (int i = 0; i < 24; i++) st[i] = 0;
#pragma unroll 1
  for (int ch = 0; ch < 8; ch++) {
#pragma unroll
    for (int i = 0; i < 16; i++) st[i] = r[ch * 16 + i];
    kb::p2_permute<24>(st, c);
  }
  uint32_t* o = dig + (row0 + t) * 8;
#pragma unroll
  for (int i = 0; i < 8; i++) o[i] = st[i];
}

__global__ void k_merkle_level(const uint32_t* __restrict__ child, uint32_t* __restrict__ parent, size_t n,
                               const __grid_constant__ kb::P16Consts c) {
  size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t st[16];
  const uint4* src = reinterpret_cast<const uint4*>(child + i * 16);
#pragma unroll
  for (int q = 0; q < 4; q++) {
    uint4 v = src[q];
    st[4 * q] = v.x; st[4 * q + 1] = v.y; st[4 * q + 2] = v.z; st[4 * q + 3] = v.w;
  }
  kb::p2_permute<16>(st, c);
  uint4* dst = reinterpret_cast<uint4*>(parent + i * 8);
  dst[0] = make_uint4(st[0], st[1], st[2], st[3]);
  dst[1] = make_uint4(st[4], st[5], st[6], st[7]);
}

__global__ void k_gather(const uint32_t* __restrict__ src, const uint64_t* __restrict__ idx, int width, int n,
                         uint32_t* __restrict__ out) {
  int q = blockIdx.x;
  if (q >= n) return;
  for (int w = threadIdx.x; w < width; w += blockDim.x) out[size_t(q) * width + w] = src[idx[q] * width + w];
}

struct GrindState {
  uint32_t st[16];
  uint32_t in[8];
};

__global__ void k_grind(const __grid_constant__ kb::P16Consts c, const __grid_constant__ GrindState g, int inlen,
                        int bits, uint32_t base, uint32_t count, uint32_t* result) {
  uint32_t off = blockIdx.x * blockDim.x + threadIdx.x;
  if (off >= count) return;
  uint32_t w = base + off;
  if (w >= kb::P) return;
  uint32_t st[16];
#pragma unroll
  for (int i = 0; i < 16; i++) st[i] = g.st[i];
  for (int i = 0; i < inlen; i++) st[i] = g.in[i];
  uint32_t wm = kb::to_mont(w);
#pragma unroll
  for (int i = 0; i < 8; i++)
    if (i == inlen) st[i] = wm;
  kb::p2_permute<16>(st, c);
  uint32_t v = kb::from_mont(st[7]);
  if ((v & ((1u << bits) - 1)) == 0) atomicMin(result, w);
}

__global__ void k_to_mont(uint32_t* x, size_t n) {
  size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) x[i] = kb::to_mont(x[i]);
}

__global__ void k_trace_gen(const uint32_t* __restrict__ inputs, const __grid_constant__ AirConsts K,
                            uint32_t* __restrict__ wit, int log_n) {
  size_t row = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  size_t N = size_t(1) << log_n;
  if (row >= N) return;
  uint32_t in[16];
#pragma unroll
  for (int i = 0; i < 16; i++) in[i] = kb::to_mont(inputs[row * 16 + i]);
  air_trace_row(K, in, wit + row, N);
}
}  // namespace

void launch_to_mont(uint32_t* x, size_t n, cudaStream_t s) {
  if (!n) return;
  k_to_mont<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(x, n);
  WL_LAUNCH_CHECK();
}

void launch_trace_gen(const uint32_t* inputs, const AirConsts& K, uint32_t* wit, int log_n, cudaStream_t s) {
  size_t N = size_t(1) << log_n;
  k_trace_gen<<<(unsigned)((N + 127) / 128), 128, 0, s>>>(inputs, K, wit, log_n);
  WL_LAUNCH_CHECK();
}

void launch_twiddles(uint32_t* tw, cudaStream_t s) {
  k_twiddles<<<(1u << 23) / 256, 256, 0, s>>>(tw, kb::two_adic_gen_m(24));
  WL_LAUNCH_CHECK();
}

void launch_lde(const LdeSource& in, uint32_t* tmp, uint32_t* out, const uint32_t* tw, cudaStream_t s) {
  (void)tmp;
  const int T = in.L + in.rho;
  if (T > 2 * MAXB || T > 24) throw std::runtime_error("LDE size beyond two shared-memory passes");
  const int tiles = (in.n_cols + CT - 1) / CT;
  const int B0 = T <= MAXB ? T : (T + 1) / 2;
  const size_t smem_max = size_t(CT) * ((1u << MAXB) + 1) * 4;
  static bool attr_set = false;
  if (!attr_set) {
    WL_CUDA(cudaFuncSetAttribute(k_ntt_first, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_max));
    WL_CUDA(cudaFuncSetAttribute(k_ntt_mid, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_max));
    attr_set = true;
  }
  dim3 g1((unsigned)(size_t(1) << (T - B0)), tiles);
  k_ntt_first<<<g1, NTT_THREADS, size_t(CT) * ((1u << B0) + 1) * 4, s>>>(in, B0, out, tw);
  WL_LAUNCH_CHECK();
  if (B0 < T) {
    const int Bp = T - B0;
    dim3 g2((unsigned)(size_t(1) << (T - Bp)), tiles);
    k_ntt_mid<<<g2, NTT_THREADS, size_t(CT) * ((1u << Bp) + 1) * 4, s>>>(out, in.n_cols, B0, Bp, in.rho, tw);
    WL_LAUNCH_CHECK();
  }
}

void launch_leaf_hash(const uint32_t* lde, size_t rows, int n_cols, int elem, const kb::P24Consts& p24,
                      uint32_t* digests, cudaStream_t s) {
  int log_elem = elem == 8 ? 3 : 0;
  k_leaf_hash<<<(unsigned)((rows + LEAF_ROWS - 1) / LEAF_ROWS), 128, 0, s>>>(lde, rows, n_cols, log_elem, p24,
                                                                            digests);
  WL_LAUNCH_CHECK();
}

void launch_merkle_level(const uint32_t* child, uint32_t* parent, size_t n, const kb::P16Consts& p16,
                         cudaStream_t s) {
  k_merkle_level<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(child, parent, n, p16);
  WL_LAUNCH_CHECK();
}

void launch_gather_u32(const uint32_t* src, const uint64_t* idx, int width, int n, uint32_t* out, cudaStream_t s) {
  if (!n) return;
  k_gather<<<n, 128, 0, s>>>(src, idx, width, n, out);
  WL_LAUNCH_CHECK();
}

void launch_grind(const kb::P16Consts& p16, const uint32_t* state16, const uint32_t* inbuf, int inlen, int bits,
                  uint32_t base, uint32_t count, uint32_t* result, cudaStream_t s) {
  GrindState g;
  for (int i = 0; i < 16; i++) g.st[i] = state16[i];
  for (int i = 0; i < 8; i++) g.in[i] = i < inlen ? inbuf[i] : 0;
  k_grind<<<(count + 255) / 256, 256, 0, s>>>(p16, g, inlen, bits, base, count, result);
  WL_LAUNCH_CHECK();
}

}  // namespace wl
