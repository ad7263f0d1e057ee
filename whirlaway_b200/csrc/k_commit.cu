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

// Per-block twiddle table: for local bit tl (global stage t = tl + 1 + lo_bits) the 2^tl
// factors w_{2^t}^(lo_global + (m << lo_bits)), m < 2^tl, at offset 2^tl - 1, each as the
// pair (canonical w, floor(w * 2^32 / p)) for Shoup multiplication.
__device__ __forceinline__ void load_twiddles(uint2* tab, int B, int tl0, uint32_t lo_global, int lo_bits,
                                              const uint2* __restrict__ tw) {
  for (uint32_t e = threadIdx.x; e < (1u << B) - 1; e += blockDim.x) {
    const int tl = 31 - __clz(e + 1);  // e + 1 in [2^tl, 2^(tl+1))
    if (tl < tl0) continue;
    const uint32_t m = e + 1 - (1u << tl);
    const int t = tl + 1 + lo_bits;
    tab[e] = tw[(lo_global + (m << lo_bits)) << (24 - t)];
  }
}

// x * w mod p for x < 2^32 and a canonical constant w with ws = floor(w 2^32 / p) (Shoup):
// the quotient estimate is off by at most one, so x w - q p lies in [0, 2p). Montgomery form
// of x is preserved (the product is linear in x).
__device__ __forceinline__ uint32_t mul_shoup(uint32_t x, uint2 w) {
  const uint32_t q = __umulhi(x, w.y);
  const uint32_t r = x * w.x - q * kb::P;
  return kb::umin(r, r - kb::P);
}

// Fused Moebius + DIT butterfly on (u, v): d = w (v - u), (u, v) <- (u + d, u - d).
__device__ __forceinline__ void bfly(uint32_t& u, uint32_t& v, uint2 w) {
  const uint32_t d = mul_shoup(v + kb::P - u, w);
  v = kb::sub(u, d);
  u = kb::add(u, d);
}

// Stages on local bits [tl0, tl1) of the 2^B points of CT columns in shared memory: two
// bits per shared-memory round trip (radix 4), a final single bit if the count is odd.
__device__ __forceinline__ void run_stages(uint32_t* sm, const uint2* tab, int B, int tl0, int tl1) {
  const uint32_t npts = 1u << B;
  int tl = tl0;
  for (; tl + 1 < tl1; tl += 2) {
    const uint32_t h = 1u << tl;
    const uint32_t ngroups = npts >> 2;  // 2^(B-2): shifts, not divisions
    for (uint32_t g = threadIdx.x; g < (uint32_t)CT * ngroups; g += blockDim.x) {
      const uint32_t col = g >> (B - 2), q = g & (ngroups - 1);
      const uint32_t r = q & (h - 1);
      const uint32_t a = ((q >> tl) << (tl + 2)) | r;
      uint32_t* base = sm + sidx(col, a, B);
      uint32_t x0 = base[0], x1 = base[h], x2 = base[2 * h], x3 = base[3 * h];
      const uint2 w1 = tab[h - 1 + r];
      bfly(x0, x1, w1);
      bfly(x2, x3, w1);
      bfly(x0, x2, tab[2 * h - 1 + r]);
      bfly(x1, x3, tab[2 * h - 1 + h + r]);
      base[0] = x0;
      base[h] = x1;
      base[2 * h] = x2;
      base[3 * h] = x3;
    }
    __syncthreads();
  }
  if (tl < tl1) {
    const uint32_t h = 1u << tl;
    const uint32_t npairs = npts >> 1;
    for (uint32_t g = threadIdx.x; g < (uint32_t)CT * npairs; g += blockDim.x) {
      const uint32_t col = g >> (B - 1), m = g & (npairs - 1);
      const uint32_t r = m & (h - 1);
      const uint32_t a = ((m >> tl) << (tl + 1)) | r;
      uint32_t* base = sm + sidx(col, a, B);
      uint32_t x0 = base[0], x1 = base[h];
      bfly(x0, x1, tab[h - 1 + r]);
      base[0] = x0;
      base[h] = x1;
    }
    __syncthreads();
  }
}

// First pass: points i of block blk (2^B of them) read source entry s = i >> rho, which
// realises the zero-padded stages 1..rho as copies; then stages rho+1..B.
__global__ void k_ntt_first(LdeSource in, int B, uint32_t* __restrict__ out, const uint2* __restrict__ tw) {
  extern __shared__ __align__(16) uint32_t sm[];
  uint2* tab = reinterpret_cast<uint2*>(sm + ((CT * ((1u << B) + 1) + 1) & ~1u));
  const int tile = blockIdx.y;
  const size_t i0 = size_t(blockIdx.x) << B;
  const uint32_t npts = 1u << B;
  const size_t col_block = size_t(in.elem) << in.L;
  load_twiddles(tab, B, in.rho, 0, 0, tw);
  for (uint32_t idx = threadIdx.x; idx < (uint32_t)CT * npts; idx += blockDim.x) {
    uint32_t col, il;
    if (in.elem == 1) { il = idx & (npts - 1); col = idx >> B; }
    else { col = idx % CT; il = idx / CT; }
    uint32_t gcol = tile * CT + col;
    size_t s = (i0 + il) >> in.rho;
    const int le = in.elem == 8 ? 3 : 0;  // log2(elem)
    size_t addr = size_t(gcol >> le) * col_block + (gcol & (in.elem - 1)) + (s << le);
    sm[sidx(col, il, B)] = (gcol < (uint32_t)in.n_cols && addr < in.src_len) ? in.src[addr] : 0u;
  }
  __syncthreads();
  if (in.rho < B) run_stages(sm, tab, B, in.rho, B);
  for (uint32_t idx = threadIdx.x; idx < (uint32_t)CT * npts; idx += blockDim.x) {
    uint32_t col = idx % CT, il = idx / CT;
    uint32_t gcol = tile * CT + col;
    if (gcol < (uint32_t)in.n_cols) out[(i0 + il) * in.n_cols + gcol] = sm[sidx(col, il, B)];
  }
}

// Later pass, in place: points i = lo + (j << B0) + (hi << (B0 + Bp)), stages B0+1..B0+Bp
// (stages up to rho are copies and are skipped).
__global__ void k_ntt_mid(uint32_t* __restrict__ data, int n_cols, int B0, int Bp, int rho,
                          const uint2* __restrict__ tw) {
  extern __shared__ __align__(16) uint32_t sm[];
  uint2* tab = reinterpret_cast<uint2*>(sm + ((CT * ((1u << Bp) + 1) + 1) & ~1u));
  const int tile = blockIdx.y;
  const size_t g = blockIdx.x;
  const uint32_t lo = uint32_t(g & ((size_t(1) << B0) - 1));
  const size_t hi = g >> B0;
  auto row_of = [&](uint32_t j) -> size_t { return lo + (size_t(j) << B0) + (hi << (B0 + Bp)); };
  const int tl0 = rho > B0 ? rho - B0 : 0;
  load_twiddles(tab, Bp, tl0, lo, B0, tw);
  const uint32_t npts = 1u << Bp;
  for (uint32_t idx = threadIdx.x; idx < (uint32_t)CT * npts; idx += blockDim.x) {
    uint32_t col = idx % CT, j = idx / CT;
    uint32_t gcol = tile * CT + col;
    sm[sidx(col, j, Bp)] = gcol < (uint32_t)n_cols ? data[row_of(j) * n_cols + gcol] : 0u;
  }
  __syncthreads();
  if (tl0 < Bp) run_stages(sm, tab, Bp, tl0, Bp);
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
__global__ void k_twiddles(uint2* tw, uint32_t w24) {
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < (1u << 23)) {
    const uint32_t w = kb::from_mont(pow_dev(w24, j));
    tw[j] = make_uint2(w, uint32_t((uint64_t(w) << 32) / kb::P));
  }
}

constexpr int LEAF_ROWS = 128;
constexpr int SUBTREE_LEVELS = 7;  // levels folded per pass (2^7 digests per block)

// Tree layout: level l (2^(LL-l) digests of 8 words) starts at digest offset
// 2^(LL+1) - 2^(LL+1-l).
__device__ __forceinline__ size_t tree_off(int LL, int l) {
  return (size_t(1) << (LL + 1)) - (size_t(1) << (LL + 1 - l));
}

// `d` holds cnt digests of level l0 whose first global index is `first`; compresses
// `levels` levels in shared memory and writes every new level to the tree.
__device__ __forceinline__ void subtree_reduce(uint32_t (*d)[8], int cnt, int levels, uint32_t* __restrict__ tree,
                                               int LL, int l0, size_t first, const kb::P16Consts& c) {
  for (int lev = 1; lev <= levels; lev++) {
    const int m = cnt >> lev;
    const int t = threadIdx.x;
    uint32_t st[16];
    const bool act = t < m;
    if (act) {
#pragma unroll
      for (int i = 0; i < 8; i++) {
        st[i] = d[2 * t][i];
        st[8 + i] = d[2 * t + 1][i];
      }
      kb::p2_permute<16>(st, c);
    }
    __syncthreads();
    if (act) {
      uint32_t* o = tree + (tree_off(LL, l0 + lev) + (first >> lev) + t) * 8;
#pragma unroll
      for (int i = 0; i < 8; i++) {
        d[t][i] = st[i];
        o[i] = st[i];
      }
    }
    __syncthreads();
  }
}

// Adds (sign +1) or subtracts (sign -1) the 16 row entries of chunk `ch` (columns
// 16 ch .. 16 ch + 15, zero at and beyond n_cols) into x, or loads them (sign 0).
__device__ __forceinline__ void leaf_chunk(const uint32_t* __restrict__ row, int n_cols, bool vec4, int ch, int sign,
                                           uint32_t* x) {
  const int c0 = ch * 16;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    uint32_t v[4];
    const int c = c0 + 4 * q;
    if (vec4) {
      if (c < n_cols) {
        const uint4 u = __ldg(reinterpret_cast<const uint4*>(row + c));
        v[0] = u.x, v[1] = u.y, v[2] = u.z, v[3] = u.w;
      } else {
        v[0] = v[1] = v[2] = v[3] = 0u;
      }
    } else {
#pragma unroll
      for (int e = 0; e < 4; e++) v[e] = c + e < n_cols ? __ldg(row + c + e) : 0u;
    }
#pragma unroll
    for (int e = 0; e < 4; e++) {
      uint32_t& d = x[4 * q + e];
      d = sign == 0 ? v[e] : (sign > 0 ? kb::add(d, v[e]) : kb::sub(d, v[e]));
    }
  }
}

// Leaf digests of 128 rows per block, then the first levels of the tree above them.
// Each thread hashes one row of 128 entries with the width-24 sponge (16 entries per
// absorption), after the Moebius transform over the position bits [log_elem, 7) of the
// column index: entry j becomes sum over i <= j (bitwise on those bits, equal elsewhere)
// of (-1)^popcount(i ^ j) row[i]. Bits 4..6 select the 16-entry chunk, so chunk ch is the
// signed sum of the chunks below it, and bits below 4 are transformed inside the chunk;
// rows are read straight from global memory (no shared-memory staging, so occupancy
// is bounded by registers).
__global__ void __launch_bounds__(LEAF_ROWS) k_leaf_hash(const uint32_t* __restrict__ lde, size_t rows, int n_cols,
                                                         int log_elem, const __grid_constant__ kb::P24Consts c,
                                                         const __grid_constant__ kb::P16Consts c16,
                                                         uint32_t* __restrict__ tree, int LL, int levels) {
  __shared__ uint32_t d[LEAF_ROWS][8];
  const size_t row0 = size_t(blockIdx.x) * LEAF_ROWS;
  const int nrows = (rows - row0) < size_t(LEAF_ROWS) ? int(rows - row0) : LEAF_ROWS;
  const int t = threadIdx.x;
  uint32_t st[24];
  if (t < nrows) {
    const uint32_t* row = lde + (row0 + t) * size_t(n_cols);
    const bool vec4 = (n_cols & 3) == 0;
    const int cmask = log_elem <= 4 ? 7 : (7 << (log_elem - 4)) & 7;  // chunk bits in the transform
#pragma unroll
    for (int i = 0; i < 24; i++) st[i] = 0;
#pragma unroll 1
    for (int ch = 0; ch < 8; ch++) {
      leaf_chunk(row, n_cols, vec4, ch, 0, st);
      const int m = ch & cmask;
      if (m) {
        // every proper subset of m, with the sign of the bits it drops
        for (int sub = (m - 1) & m;; sub = (sub - 1) & m) {
          const int sign = (__popc(m ^ sub) & 1) ? -1 : 1;
          leaf_chunk(row, n_cols, vec4, (ch & ~m) | sub, sign, st);
          if (!sub) break;
        }
      }
#pragma unroll
      for (int b = 0; b < 4; b++) {
        if (b < log_elem) continue;
        const int h = 1 << b;
#pragma unroll
        for (int i = 0; i < 16; i++)
          if (!(i & h)) st[i + h] = kb::sub(st[i + h], st[i]);
      }
      kb::p2_permute<24>(st, c);
    }
    uint32_t* o = tree + (row0 + t) * 8;
#pragma unroll
    for (int i = 0; i < 8; i++) {
      o[i] = st[i];
      d[t][i] = st[i];
    }
  }
  __syncthreads();
  subtree_reduce(d, nrows, levels, tree, LL, 0, row0, c16);
}

// Levels l0+1 .. l0+levels from 2^levels level-l0 digests per block.
__global__ void k_merkle_subtree(uint32_t* __restrict__ tree, int LL, int l0, int levels,
                                 const __grid_constant__ kb::P16Consts c) {
  __shared__ uint32_t d[1 << SUBTREE_LEVELS][8];
  const int cnt = 1 << levels;
  const size_t first = size_t(blockIdx.x) * cnt;
  const uint32_t* src = tree + (tree_off(LL, l0) + first) * 8;
  for (int i = threadIdx.x; i < cnt * 8; i += blockDim.x) d[i / 8][i % 8] = src[i];
  __syncthreads();
  subtree_reduce(d, cnt, levels, tree, LL, l0, first, c);
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

void launch_twiddles(uint2* tw, cudaStream_t s) {
  k_twiddles<<<(1u << 23) / 256, 256, 0, s>>>(tw, kb::two_adic_gen_m(24));
  WL_LAUNCH_CHECK();
}

void launch_lde(const LdeSource& in, uint32_t* tmp, uint32_t* out, const uint2* tw, cudaStream_t s) {
  (void)tmp;
  const int T = in.L + in.rho;
  if (T > 2 * MAXB || T > 24) throw std::runtime_error("LDE size beyond two shared-memory passes");
  const int tiles = (in.n_cols + CT - 1) / CT;
  const int B0 = T <= MAXB ? T : (T + 1) / 2;
  auto smem_for = [](int B) { return (((size_t(CT) * ((1u << B) + 1) + 1) & ~size_t(1)) + 2 * (size_t(1) << B)) * 4; };
  const size_t smem_max = smem_for(MAXB);
  WL_CUDA(cudaFuncSetAttribute(k_ntt_first, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_max));
  WL_CUDA(cudaFuncSetAttribute(k_ntt_mid, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_max));
  dim3 g1((unsigned)(size_t(1) << (T - B0)), tiles);
  k_ntt_first<<<g1, NTT_THREADS, smem_for(B0), s>>>(in, B0, out, tw);
  WL_LAUNCH_CHECK();
  if (B0 < T) {
    const int Bp = T - B0;
    dim3 g2((unsigned)(size_t(1) << (T - Bp)), tiles);
    k_ntt_mid<<<g2, NTT_THREADS, smem_for(Bp), s>>>(out, in.n_cols, B0, Bp, in.rho, tw);
    WL_LAUNCH_CHECK();
  }
}

void launch_merkle_tree(const uint32_t* lde, size_t rows, int n_cols, int elem, const kb::P24Consts& p24,
                        const kb::P16Consts& p16, uint32_t* tree, int LL, cudaStream_t s) {
  const int log_elem = elem == 8 ? 3 : 0;
  const int first_levels = LL < SUBTREE_LEVELS ? LL : SUBTREE_LEVELS;
  k_leaf_hash<<<(unsigned)((rows + LEAF_ROWS - 1) / LEAF_ROWS), LEAF_ROWS, 0, s>>>(lde, rows, n_cols, log_elem, p24,
                                                                                     p16, tree, LL, first_levels);
  WL_LAUNCH_CHECK();
  for (int l0 = first_levels; l0 < LL; l0 += SUBTREE_LEVELS) {
    const int lv = (LL - l0) < SUBTREE_LEVELS ? (LL - l0) : SUBTREE_LEVELS;
    const unsigned blocks = 1u << (LL - l0 - lv);
    k_merkle_subtree<<<blocks, 1 << (lv - 1), 0, s>>>(tree, LL, l0, lv, p16);
    WL_LAUNCH_CHECK();
  }
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
