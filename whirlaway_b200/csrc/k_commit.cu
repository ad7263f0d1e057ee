// Reed-Solomon encoding, Merkle hashing and grinding kernels (the work of whir-p3's
// CommitmentWriter::commit and EvalsDft, reached from crates/air/src/prove.rs:82-91,
// and of the DuplexChallenger grinding behind pow_grinding).
//
// LDE. For one commitment every column of the codeword matrix is the evaluation, on the
// subgroup of order 2^T (T = L + rho), of a polynomial whose monomial coefficients are the
// Moebius transform of a 2^L-long slice of the evaluation table, read in bit-reversed
// exponent order. A radix-2 decimation-in-time NTT takes exactly that bit-reversed input,
// so the Moebius step of the variable at stage t is fused into stage t's butterfly
// (v <- v - u before u +- w v). Zero padding for the rate makes stages 1..rho plain
// copies: after them point i holds source entry i >> rho, so the work is stages
// rho+1..T, split into passes of at most 8 stages.
//
// LDE layout in HBM (tile-major): columns in tiles of 8, word (tile, row, c) at
// (tile * 2^T + row) * 8 + c, so 4 consecutive rows of a tile are one 128-byte line.
// A pass over stages Bs+1..Bs+Bp works on lines of 2^Bp points i = lo + (j << Bs) +
// (hi << (Bs + Bp)); a warp's 32 lanes are 8 columns x 4 (lo, hi) pairs of adjacent
// rows, so every global access of a warp is one or two whole lines. Each thread keeps
// 2^rb points of its line in registers for rb <= 4 stages, and a pass is two such
// register rounds with one shared-memory exchange between them.
#include <algorithm>
#include <map>
#include <mutex>

#include "kernels.h"

namespace wl {

namespace {
constexpr int NTT_WARPS = 8;
constexpr int NTT_MAX_BP = 8;  // stages per pass

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

// Where a round reads its points from and writes them to.
enum NttIo { IO_SRC = 0, IO_GLOBAL = 1, IO_SMEM = 2 };

// Per-lane addressing of a pass: point j of this lane's line lives at base[j << step] for
// each of the three places a round reads or writes.
struct NttLane {
  const uint32_t* src;      // commitment source at j = 0 (nullptr: column beyond n_cols)
  const uint32_t* src_end;  // one past the source (entries beyond it read as zero)
  int src_step;             // log2(elem)
  uint32_t* data;           // LDE word of row j = 0, this lane's column
  int data_step;            // Bs + 3 (rows are 8 words apart within a tile)
  uint32_t* X;              // exchange buffer [2^Bp][32], this lane's column
  int Bp;
};

// One register round: stages b0..b0+RB-1 (local numbering, b0 = B0) on the groups of 2^RB
// points j = base + (k << b0) handled by this warp, in a pass of BP stages (both compile-time,
// so the shared-memory and twiddle offsets below are immediates). `tws` is this lane's twiddle table: entry
// 2^tl - 1 + r is the factor of local stage tl for j mod 2^tl = r. Addresses are formed
// once per group (a base pointer and a stride); the source range is checked once per group.
template <int RB, int B0, int BP, int IN, int OUT>
__device__ __forceinline__ void ntt_round(const NttLane& ln, const uint2* tws, int warp, bool active) {
  constexpr int R = 1 << RB, b0 = B0;
  constexpr uint32_t groups = 1u << (BP - RB);
  for (uint32_t g = warp; g < groups; g += NTT_WARPS) {
    const uint32_t base = (g & ((1u << b0) - 1)) | ((g >> b0) << (b0 + RB));
    if (!active) continue;
    uint32_t x[R];
    if constexpr (IN == IO_SRC) {
      const uint32_t* p0 = ln.src + (size_t(base) << ln.src_step);
      const size_t stride = size_t(1) << (b0 + ln.src_step);
      if (ln.src && p0 + (R - 1) * stride < ln.src_end) {
#pragma unroll
        for (int k = 0; k < R; k++) x[k] = __ldg(p0 + k * stride);
      } else {
#pragma unroll
        for (int k = 0; k < R; k++) x[k] = (ln.src && p0 + k * stride < ln.src_end) ? __ldg(p0 + k * stride) : 0u;
      }
    } else if constexpr (IN == IO_GLOBAL) {
      const uint32_t* p0 = ln.data + (size_t(base) << ln.data_step);
      const size_t stride = size_t(1) << (b0 + ln.data_step);
#pragma unroll
      for (int k = 0; k < R; k++) x[k] = p0[k * stride];
    } else {
      const uint32_t* p0 = ln.X + (base << 5);
#pragma unroll
      for (int k = 0; k < R; k++) x[k] = p0[(uint32_t(k) << b0) << 5];
    }
    const uint32_t blo = base & ((1u << b0) - 1);
#pragma unroll
    for (int st = 0; st < RB; st++) {
      const int tl = b0 + st;
      const uint2* tt = tws + (1u << tl) - 1 + blo;
      uint2 w[R > 1 ? R / 2 : 1];
#pragma unroll
      for (int m = 0; m < (1 << st); m++) w[m] = tt[uint32_t(m) << b0];
#pragma unroll
      for (int k = 0; k < R; k++) {
        if (k & (1 << st)) continue;
        bfly(x[k], x[k + (1 << st)], w[k & ((1 << st) - 1)]);
      }
    }
    if constexpr (OUT == IO_GLOBAL) {
      uint32_t* p0 = ln.data + (size_t(base) << ln.data_step);
      const size_t stride = size_t(1) << (b0 + ln.data_step);
#pragma unroll
      for (int k = 0; k < R; k++) p0[k * stride] = x[k];
    } else {
      uint32_t* p0 = ln.X + (base << 5);
#pragma unroll
      for (int k = 0; k < R; k++) p0[(uint32_t(k) << b0) << 5] = x[k];
    }
  }
}

// The two register rounds of a pass of BP stages (ceil(BP/2) then floor(BP/2) stages, one
// shared-memory exchange between them); the first reads from IN, the last writes the codeword.
template <int BP, int IN>
__device__ __forceinline__ void ntt_rounds(const NttLane& ln, const uint2* tws, int warp, bool active) {
  constexpr int RB1 = (BP + 1) / 2, RB2 = BP - RB1;
  if constexpr (RB2 == 0) {
    ntt_round<RB1, 0, BP, IN, IO_GLOBAL>(ln, tws, warp, active);
  } else {
    ntt_round<RB1, 0, BP, IN, IO_SMEM>(ln, tws, warp, active);
    __syncthreads();
    ntt_round<RB2, RB1, BP, IO_SMEM, IO_GLOBAL>(ln, tws, warp, active);
  }
}

// One pass over stages Bs+1..Bs+Bp (global numbering) for the lines of one tile.
// blockIdx.x = (hi group << (Bs - lr_log)) | lo group; 2^lr_log lo values and 2^hg_log hi
// values per block. The first pass (FROM_SRC, Bs = rho) reads the commitment source.
template <bool FROM_SRC, int BP>
__global__ void __launch_bounds__(NTT_WARPS * 32) k_ntt_pass(LdeSource in, uint32_t* __restrict__ data, int T,
                                                            int Bs, int lr_log, int hg_log,
                                                            const uint2* __restrict__ tw, int tile0) {
  constexpr int Bp = BP;
  const int tile = tile0 + blockIdx.y;
  extern __shared__ __align__(16) uint32_t sm[];
  const uint32_t npts = 1u << Bp, ntw = npts - 1;
  const int LR = 1 << lr_log;
  uint2* TW = reinterpret_cast<uint2*>(sm + (size_t(npts) << 5));  // [LR][2^Bp - 1]
  const uint32_t lg = blockIdx.x & ((1u << (Bs - lr_log)) - 1);
  const size_t hg = blockIdx.x >> (Bs - lr_log);
  for (uint32_t idx = threadIdx.x; idx < (ntw << lr_log); idx += blockDim.x) {
    const uint32_t l = idx & (LR - 1), e = idx >> lr_log;
    const int tl = 31 - __clz(e + 1);  // e + 1 in [2^tl, 2^(tl+1))
    const uint32_t r = e + 1 - (1u << tl);
    const int t = Bs + tl + 1;
    TW[l * ntw + e] = tw[((size_t(1) << (t - 1)) - 1) + (lg << lr_log) + l + (size_t(r) << Bs)];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int c = lane & 7, l = (lane >> 3) & (LR - 1), h2 = lane >> (3 + lr_log);
  const bool active = h2 < (1 << hg_log);
  NttLane ln;
  const int le = in.elem == 8 ? 3 : 0;
  const uint32_t gcol = tile * 8 + c;
  const size_t hi = (hg << hg_log) + h2;
  const size_t row0 = (size_t(tile) << T) + (lg << lr_log) + l + (hi << (Bs + Bp));
  ln.src = nullptr;
  ln.src_end = in.src + in.src_len;
  if (FROM_SRC && gcol < (uint32_t)in.n_cols)
    ln.src = in.src + size_t(gcol >> le) * (size_t(in.elem) << in.L) + (gcol & ((1u << le) - 1)) +
             ((hi << Bp) << le);
  ln.src_step = le;
  ln.data = data + (row0 << 3) + c;
  ln.data_step = Bs + 3;
  ln.X = sm + lane;
  ln.Bp = Bp;
  const uint2* tws = TW + l * ntw;
  ntt_rounds<BP, FROM_SRC ? IO_SRC : IO_GLOBAL>(ln, tws, warp, active);
}

__device__ __forceinline__ void cp_async16(uint32_t* smem, const uint32_t* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit16() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait16() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// Passes after the first (Bs >= 2, so a block's 4 lo values are 4 consecutive rows and point
// j of a line is one contiguous 128-byte piece of the tile: 4 rows x 8 columns). Persistent
// blocks walk a contiguous range of lines (lo group outermost, then tile, then hi) and copy
// the next line into the second of two shared-memory buffers with cp.async while the current
// one is transformed: the first register round reads and writes shared memory in place, the
// second writes the codeword. Twiddles are reloaded when the lo group changes.
constexpr int NTT_ASYNC_BLOCKS_PER_SM = 4;
template <int BP>
__global__ void __launch_bounds__(NTT_WARPS * 32, NTT_ASYNC_BLOCKS_PER_SM)
    k_ntt_pass_async(uint32_t* __restrict__ data, int T, int Bs, const uint2* __restrict__ tw, int tile0, int tiles,
                     uint32_t nlines, uint32_t per_block) {
  constexpr int Bp = BP;
  extern __shared__ __align__(16) uint32_t sm[];
  const uint32_t npts = 1u << Bp, ntw = npts - 1;
  uint2* TW = reinterpret_cast<uint2*>(sm + (npts << 6));  // [4][2^Bp - 1]
  const uint32_t nhi = 1u << (T - Bs - Bp);
  const uint32_t first = blockIdx.x * per_block;
  const uint32_t last = first + per_block < nlines ? first + per_block : nlines;
  if (first >= last) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int c = lane & 7, l = lane >> 3;
  auto coords = [&](uint32_t id, uint32_t& lg, int& tile, uint32_t& hi) {
    hi = id % nhi;
    const uint32_t r = id / nhi;
    tile = tile0 + int(r % uint32_t(tiles));
    lg = r / uint32_t(tiles);
  };
  auto row_base = [&](uint32_t lg, int tile, uint32_t hi) {
    return (size_t(tile) << T) + (size_t(lg) << 2) + (size_t(hi) << (Bs + Bp));
  };
  auto prefetch = [&](uint32_t id, uint32_t* X) {
    uint32_t lg, hi;
    int tile;
    coords(id, lg, tile, hi);
    const uint32_t* g = data + (row_base(lg, tile, hi) << 3);
    for (uint32_t idx = threadIdx.x; idx < (npts << 3); idx += blockDim.x) {
      const uint32_t j = idx >> 3, q = idx & 7;
      cp_async16(X + (j << 5) + 4 * q, g + ((size_t(j) << Bs) << 3) + 4 * q);
    }
    cp_async_commit16();
  };
  uint32_t cur_lg = ~0u;
  prefetch(first, sm);
  for (uint32_t id = first, it = 0; id < last; id++, it++) {
    uint32_t* X = sm + ((it & 1) << (Bp + 5));
    if (id + 1 < last) {
      prefetch(id + 1, sm + (((it + 1) & 1) << (Bp + 5)));
      cp_async_wait16<1>();
    } else {
      cp_async_wait16<0>();
    }
    __syncthreads();  // line id is in X for every thread
    uint32_t lg, hi;
    int tile;
    coords(id, lg, tile, hi);
    if (lg != cur_lg) {
      for (uint32_t idx = threadIdx.x; idx < (ntw << 2); idx += blockDim.x) {
        const uint32_t ll = idx & 3, e = idx >> 2;
        const int tl = 31 - __clz(e + 1);  // e + 1 in [2^tl, 2^(tl+1))
        const uint32_t r = e + 1 - (1u << tl);
        const int t = Bs + tl + 1;
        TW[ll * ntw + e] = tw[((size_t(1) << (t - 1)) - 1) + (size_t(lg) << 2) + ll + (size_t(r) << Bs)];
      }
      cur_lg = lg;
      __syncthreads();
    }
    NttLane ln;
    ln.src = nullptr;
    ln.src_end = nullptr;
    ln.src_step = 0;
    ln.data = data + ((row_base(lg, tile, hi) + l) << 3) + c;
    ln.data_step = Bs + 3;
    ln.X = X + lane;
    ln.Bp = Bp;
    const uint2* tws = TW + l * ntw;
    ntt_rounds<BP, IO_SMEM>(ln, tws, warp, true);
    __syncthreads();  // X is free for the prefetch two lines ahead
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
// Per-stage twiddles: stage t (1..24) holds w_{2^t}^x for x < 2^(t-1) at offset
// 2^(t-1) - 1, each as (canonical w, floor(w 2^32 / p)) for Shoup multiplication.
__global__ void k_twiddles(uint2* tw, uint32_t w24) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < (1u << 24) - 1) {
    const int t = 32 - __clz(j + 1);
    const uint32_t x = j + 1 - (1u << (t - 1));
    const uint32_t w = kb::from_mont(pow_dev(w24, x << (24 - t)));
    tw[j] = make_uint2(w, uint32_t((uint64_t(w) << 32) / kb::P));
  }
}

// Leaf rows per block: 64, 128 (default) or 256, the autotuner's pick (LEAF_PLANS).
constexpr int TOP_LEVELS = 7;  // the last levels (<= 2^7 digests) run in one block
constexpr int FLAT_LEVEL_MIN_LOG = 13;  // levels of at least 2^13 digests get their own launch

// Tree layout: level l (2^(LL-l) digests of 8 words) starts at digest offset
// 2^(LL+1) - 2^(LL+1-l).
__device__ __forceinline__ size_t tree_off(int LL, int l) {
  return (size_t(1) << (LL + 1)) - (size_t(1) << (LL + 1 - l));
}

// Adds (sign +1) or subtracts (sign -1) the 16 entries of chunk `ch` (columns 16 ch ..
// 16 ch + 15, zero at and beyond n_cols) of LDE row `row` into x, or loads them (sign 0).
// The LDE is tile-major with 2^T rows (n_cols a multiple of 8).
__device__ __forceinline__ void leaf_chunk(const uint32_t* __restrict__ lde, int T, size_t row, int n_cols, int ch,
                                           int sign, uint32_t* x) {
  const int c0 = ch * 16;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    uint32_t v[4];
    const int c = c0 + 4 * q;
    if (c < n_cols) {
      const uint4 u = __ldg(reinterpret_cast<const uint4*>(lde + (((size_t(c >> 3) << T) + row) << 3) + (c & 7)));
      v[0] = u.x, v[1] = u.y, v[2] = u.z, v[3] = u.w;
    } else {
      v[0] = v[1] = v[2] = v[3] = 0u;
    }
#pragma unroll
    for (int e = 0; e < 4; e++) {
      uint32_t& d = x[4 * q + e];
      d = sign == 0 ? v[e] : (sign > 0 ? kb::add(d, v[e]) : kb::sub(d, v[e]));
    }
  }
}

// The tree holds canonical digests: the permutations run in the canonical domain (see
// p2_permute_fd), the absorbed LDE entries are converted from Montgomery form, and the host
// converts the root and the opened digests back.
//
// Absorbs chunk ch of LDE row `row` into the sponge state st (the chunk overwrites the rate
// st[0..15]; st[16..23] is the capacity): the Moebius transform over the position bits
// [log_elem, 7) of the column index makes entry j the sum over i <= j (bitwise on those bits,
// equal elsewhere) of (-1)^popcount(i ^ j) row[i]. Bits 4..6 select the 16-entry chunk, so
// chunk ch is the signed sum of the chunks below it, and bits below 4 are transformed inside
// the chunk. Then the permutation.
__device__ __forceinline__ void leaf_absorb(const uint32_t* __restrict__ lde, int T, size_t row, int n_cols,
                                            int log_elem, int ch, const kb::P2ConstsFd<24>& c, uint32_t* st) {
  const int cmask = log_elem <= 4 ? 7 : (7 << (log_elem - 4)) & 7;  // chunk bits in the transform
  leaf_chunk(lde, T, row, n_cols, ch, 0, st);
  const int m = ch & cmask;
  if (m) {
    // every proper subset of m, with the sign of the bits it drops
    for (int sub = (m - 1) & m;; sub = (sub - 1) & m) {
      const int sign = (__popc(m ^ sub) & 1) ? -1 : 1;
      leaf_chunk(lde, T, row, n_cols, (ch & ~m) | sub, sign, st);
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
#pragma unroll
  for (int i = 0; i < 16; i++) st[i] = kb::from_mont(st[i]);
  kb::p2_permute_fd<24>(st, c);
}

// Leaf digests (level 0 of the tree), one row per thread: each thread hashes one row of 128
// entries with the width-24 sponge (16 entries per absorption, 8 absorptions). Rows are read
// straight from the tile-major LDE (no shared-memory staging, so occupancy is bounded by
// registers).
template <int ROWS>
__global__ void __launch_bounds__(ROWS) k_leaf_hash(const uint32_t* __restrict__ lde, int T, int n_cols,
                                                    int log_elem, const __grid_constant__ kb::P2ConstsFd<24> c,
                                                    uint32_t* __restrict__ tree) {
  const size_t row0 = size_t(blockIdx.x) * ROWS;
  const size_t rows = size_t(1) << T;
  const int nrows = (rows - row0) < size_t(ROWS) ? int(rows - row0) : ROWS;
  const int t = threadIdx.x;
  uint32_t st[24];
  if (t < nrows) {
    const size_t row = row0 + t;
#pragma unroll
    for (int i = 0; i < 24; i++) st[i] = 0;
#pragma unroll 1
    for (int ch = 0; ch < 8; ch++) leaf_absorb(lde, T, row, n_cols, log_elem, ch, c, st);
    uint4* o = reinterpret_cast<uint4*>(tree + (row0 + t) * 8);
    o[0] = make_uint4(st[0], st[1], st[2], st[3]);
    o[1] = make_uint4(st[4], st[5], st[6], st[7]);
  }
}

// One absorption (chunk ch) for every row, the capacity carried between launches in cap
// (8 words per row): the sponge of k_leaf_hash split by chunk, so that chunk ch can be hashed
// as soon as the LDE tiles it reads exist. The last chunk writes the digests.
template <int ROWS>
__global__ void __launch_bounds__(ROWS) k_leaf_absorb(const uint32_t* __restrict__ lde, int T, int n_cols,
                                                      int log_elem, const __grid_constant__ kb::P2ConstsFd<24> c,
                                                      int ch, uint32_t* __restrict__ cap,
                                                      uint32_t* __restrict__ tree) {
  const size_t row = size_t(blockIdx.x) * ROWS + threadIdx.x;
  if (row >= (size_t(1) << T)) return;
  uint32_t st[24];
  if (ch == 0) {
#pragma unroll
    for (int i = 16; i < 24; i++) st[i] = 0;
  } else {
    const uint4* in = reinterpret_cast<const uint4*>(cap + row * 8);
    const uint4 a = in[0], b = in[1];
    st[16] = a.x, st[17] = a.y, st[18] = a.z, st[19] = a.w, st[20] = b.x, st[21] = b.y, st[22] = b.z, st[23] = b.w;
  }
  leaf_absorb(lde, T, row, n_cols, log_elem, ch, c, st);
  uint4* o = reinterpret_cast<uint4*>(ch == 7 ? tree + row * 8 : cap + row * 8);
  if (ch == 7) {
    o[0] = make_uint4(st[0], st[1], st[2], st[3]);
    o[1] = make_uint4(st[4], st[5], st[6], st[7]);
  } else {
    o[0] = make_uint4(st[16], st[17], st[18], st[19]);
    o[1] = make_uint4(st[20], st[21], st[22], st[23]);
  }
}

// Level l of the tree from level l - 1, one 2-to-1 compression per thread.
__global__ void k_merkle_level(uint32_t* __restrict__ tree, int LL, int l, const __grid_constant__ kb::P2ConstsFd<16> c) {
  const size_t m = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (m >= (size_t(1) << (LL - l))) return;
  const uint4* src = reinterpret_cast<const uint4*>(tree + (tree_off(LL, l - 1) + 2 * m) * 8);
  uint32_t st[16];
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const uint4 u = src[q];
    st[4 * q] = u.x, st[4 * q + 1] = u.y, st[4 * q + 2] = u.z, st[4 * q + 3] = u.w;
  }
  kb::p2_permute_fd<16>(st, c);
  uint4* o = reinterpret_cast<uint4*>(tree + (tree_off(LL, l) + m) * 8);
  o[0] = make_uint4(st[0], st[1], st[2], st[3]);
  o[1] = make_uint4(st[4], st[5], st[6], st[7]);
}

// Poseidon2-16 (canonical domain, canonical constants; the internal diagonal is applied by
// Montgomery products with its Montgomery form, which is the same linear map) with the state
// spread over the 16 lanes of a half-warp (lane i holds word i),
// for the narrow top of a Merkle tree where one thread per permutation leaves the device
// idle and a single permutation's latency is the cost. Every lane of the warp calls it.
// External layer: lane i's M4 row is 2 x_i + 3 x_(i+1) + x_(i+2) + x_(i+3) within its chunk
// of 4, then the sum over the 4 chunks at the same position. Internal layer: lane 0 takes the
// S-box, the sum is a 16-lane reduction, and each lane scales by its own diagonal entry.
__device__ __forceinline__ uint32_t mds16_lanes(uint32_t a, int i) {
  const int base = i & ~3;
  const uint32_t b = __shfl_sync(0xffffffffu, a, base | ((i + 1) & 3), 16);
  const uint32_t c = __shfl_sync(0xffffffffu, a, base | ((i + 2) & 3), 16);
  const uint32_t d = __shfl_sync(0xffffffffu, a, base | ((i + 3) & 3), 16);
  const uint32_t y = kb::add(kb::add(kb::add(a, b), kb::add(c, d)), kb::add(a, kb::dbl(b)));
  uint32_t t = kb::add(y, __shfl_xor_sync(0xffffffffu, y, 4, 16));
  t = kb::add(t, __shfl_xor_sync(0xffffffffu, t, 8, 16));
  return kb::add(y, t);
}
// rc_s: the full-round constants in shared memory (initial rounds at 0, terminal at 64): each
// lane reads its own word, which from the constant bank would serialise across the warp.
__device__ __forceinline__ void stage_p16_full_rounds(uint32_t* rc_s, const kb::P16Consts& c) {
  for (int q = threadIdx.x; q < 128; q += blockDim.x) rc_s[q] = q < 64 ? c.ext_init[q] : c.ext_term[q - 64];
}
__device__ uint32_t p2_permute16_lanes(uint32_t v, const uint32_t* rc_s, const kb::P16Consts& c) {
  const int i = threadIdx.x & 15;
  const uint32_t dg = kb::p2_diag<16>(i);
  v = mds16_lanes(v, i);
#pragma unroll 1
  for (int r = 0; r < 4; r++) v = mds16_lanes(kb::cube_fq(v + rc_s[r * 16 + i]), i);
#pragma unroll 1
  for (int r = 0; r < 20; r++) {
    if (i == 0) v = kb::cube_fq(v + c.internal[r]);
    uint32_t sum = v;
#pragma unroll
    for (int d = 8; d > 0; d >>= 1) sum = kb::add(sum, __shfl_xor_sync(0xffffffffu, sum, d, 16));
    v = kb::add(kb::mul(v, dg), sum);
  }
#pragma unroll 1
  for (int r = 0; r < 4; r++) v = mds16_lanes(kb::cube_fq(v + rc_s[64 + r * 16 + i]), i);
  return v;
}

// One level l of the tree, 16 lanes per compression (grid covers 16 * 2^(LL-l) threads).
__global__ void k_merkle_level_lanes(uint32_t* __restrict__ tree, int LL, int l, const __grid_constant__ kb::P16Consts c) {
  __shared__ uint32_t rc_s[128];
  stage_p16_full_rounds(rc_s, c);
  __syncthreads();
  const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const size_t m = t >> 4;
  const int i = threadIdx.x & 15;
  const size_t cnt = size_t(1) << (LL - l);
  const bool act = m < cnt;
  const size_t warp_first = (t & ~size_t(31)) >> 4;
  if (warp_first >= cnt) return;  // whole warp idle (uniform per warp)
  uint32_t v = act ? tree[(tree_off(LL, l - 1) + 2 * m) * 8 + i] : 0u;
  v = p2_permute16_lanes(v, rc_s, c);
  if (act && i < 8) tree[(tree_off(LL, l) + m) * 8 + i] = v;
}

// Levels l0+1 .. LL in one block of 1024 threads (at most 64 compressions per level).
__global__ void __launch_bounds__(1024) k_merkle_top(uint32_t* __restrict__ tree, int LL, int l0,
                                                     const __grid_constant__ kb::P16Consts c) {
  __shared__ uint32_t rc_s[128];
  stage_p16_full_rounds(rc_s, c);
  __syncthreads();
  const int g = threadIdx.x >> 4, i = threadIdx.x & 15;
  for (int l = l0 + 1; l <= LL; l++) {
    const int cnt = 1 << (LL - l);
    if ((threadIdx.x >> 5) * 2 < cnt) {  // warps holding at least one live compression
      const bool act = g < cnt;
      uint32_t v = act ? tree[(tree_off(LL, l - 1) + 2 * size_t(g)) * 8 + i] : 0u;
      v = p2_permute16_lanes(v, rc_s, c);
      if (act && i < 8) tree[(tree_off(LL, l) + g) * 8 + i] = v;
    }
    __syncthreads();
  }
}

// Rows idx[q] of the tile-major LDE (2^T rows, n_cols columns) into out[q * n_cols + col].
// Row idx[q] of the tile-major LDE (128 threads, one per position; positions >= n_cols are
// zero), Moebius-transformed over the position bits [log_elem, 7) as the leaf hash absorbs it:
// for each bit b, v[i | 2^b] -= v[i]. Writes out[q * 128 + i]. With mono, also the row's
// folded value folded[q] = sum_p v_p mono[p] over its 128 >> log_elem elements (base-field
// values, or extension elements of 8 consecutive words).
__global__ void __launch_bounds__(128) k_gather_lde(const uint32_t* __restrict__ lde, int T,
                                                    const uint64_t* __restrict__ idx, int n_cols, int log_elem,
                                                    int n, uint32_t* __restrict__ out, const kb::ef* __restrict__ mono,
                                                    kb::ef* __restrict__ folded) {
  __shared__ uint32_t v[128];
  __shared__ kb::ef scratch[32];
  const int q = blockIdx.x, i = threadIdx.x;
  if (q >= n) return;  // whole block
  v[i] = i < n_cols ? lde[(((size_t(i >> 3) << T) + idx[q]) << 3) + (i & 7)] : 0u;
  __syncthreads();
  for (int b = log_elem; b < 7; b++) {
    const uint32_t lo = v[i & ~(1 << b)];
    __syncthreads();
    if (i & (1 << b)) v[i] = kb::sub(v[i], lo);
    __syncthreads();
  }
  out[size_t(q) * 128 + i] = v[i];
  if (mono) {
    kb::ef c = kb::ef_zero();
    if (log_elem == 0) {
      c = kb::ef_mul_f(mono[i], v[i]);
    } else if (i < (128 >> log_elem)) {
      kb::ef e = kb::ef_zero();
      for (int k = 0; k < (1 << log_elem); k++) e.c[k] = v[(i << log_elem) + k];
      c = kb::ef_mul(e, mono[i]);
    }
    c = block_reduce_ef(c, scratch);
    if (i == 0) folded[q] = c;
  }
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

// Grinding: the smallest w in [base, base + count), below p, for which the challenger (state
// st, input buffer in[0..inlen)) samples `bits` zero bits after observing w. The words are
// canonical, the permutation runs in the canonical domain. Thread t tries base + t, then
// base + t + G, ... (G threads in the grid) and stops at the first candidate above a witness
// already found: every candidate below the smallest witness is tried, so the result does not
// depend on the order in which the threads run, and the search ends soon after the first hit
// instead of covering the whole batch.
__global__ void __launch_bounds__(256) k_grind(const __grid_constant__ kb::P2ConstsFd<16> c,
                                               const __grid_constant__ GrindState g, int inlen, int bits,
                                               uint32_t base, uint32_t count, uint32_t* result) {
  const uint32_t G = gridDim.x * blockDim.x;
  const uint32_t mask = (1u << bits) - 1;
  for (uint32_t off = blockIdx.x * blockDim.x + threadIdx.x; off < count; off += G) {
    const uint32_t w = base + off;
    if (w >= kb::P) return;
    if (*reinterpret_cast<volatile const uint32_t*>(result) < w) return;  // a smaller witness is known
    uint32_t st[16];
#pragma unroll
    for (int i = 0; i < 16; i++) st[i] = g.st[i];
    for (int i = 0; i < inlen; i++) st[i] = g.in[i];
#pragma unroll
    for (int i = 0; i < 8; i++)
      if (i == inlen) st[i] = w;
    kb::p2_permute_fd<16>(st, c);
    if ((st[7] & mask) == 0) atomicMin(result, w);
  }
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
  k_twiddles<<<(1u << 24) / 256, 256, 0, s>>>(tw, kb::two_adic_gen_m(24));
  WL_LAUNCH_CHECK();
}

namespace {
int ntt_sm_count() {
  int dev = 0, n = 0;
  WL_CUDA(cudaGetDevice(&dev));
  WL_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
  return n;
}
// Opts the double-buffered pass into more than 48 KB of dynamic shared memory (once per
// device and size).
template <int BP>
void ntt_async_smem_limit(size_t bytes) {
  if (bytes <= 48 * 1024) return;
  static std::mutex mu;
  static std::map<int, size_t> done;
  int dev = 0;
  WL_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if (done[dev] >= bytes) return;
  WL_CUDA(cudaFuncSetAttribute(k_ntt_pass_async<BP>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
  done[dev] = bytes;
}
// Launches one pass of BP stages: the first (from the commitment source), a later one-shot
// pass, or the double-buffered persistent pass.
enum NttPassKind { NTT_FIRST, NTT_LATER, NTT_ASYNC };
struct NttPassArgs {
  LdeSource in;
  uint32_t* out;
  int T, Bs, lr_log, hg_log, tile0, tiles;
  const uint2* tw;
  dim3 grid;
  size_t smem;
  uint32_t nlines, per;
};
template <int BP>
void ntt_pass_launch(NttPassKind kind, const NttPassArgs& a, cudaStream_t s) {
  if (kind == NTT_FIRST) {
    k_ntt_pass<true, BP><<<a.grid, NTT_WARPS * 32, a.smem, s>>>(a.in, a.out, a.T, a.Bs, a.lr_log, a.hg_log, a.tw,
                                                                 a.tile0);
  } else if (kind == NTT_LATER) {
    k_ntt_pass<false, BP><<<a.grid, NTT_WARPS * 32, a.smem, s>>>(a.in, a.out, a.T, a.Bs, a.lr_log, a.hg_log, a.tw,
                                                                  a.tile0);
  } else {
    ntt_async_smem_limit<BP>(a.smem);
    k_ntt_pass_async<BP><<<a.grid, NTT_WARPS * 32, a.smem, s>>>(a.out, a.T, a.Bs, a.tw, a.tile0, a.tiles, a.nlines,
                                                                 a.per);
  }
}
void ntt_pass_dispatch(int Bp, NttPassKind kind, const NttPassArgs& a, cudaStream_t s) {
  switch (Bp) {
    case 1: ntt_pass_launch<1>(kind, a, s); break;
    case 2: ntt_pass_launch<2>(kind, a, s); break;
    case 3: ntt_pass_launch<3>(kind, a, s); break;
    case 4: ntt_pass_launch<4>(kind, a, s); break;
    case 5: ntt_pass_launch<5>(kind, a, s); break;
    case 6: ntt_pass_launch<6>(kind, a, s); break;
    case 7: ntt_pass_launch<7>(kind, a, s); break;
    case 8: ntt_pass_launch<8>(kind, a, s); break;
    default: throw std::runtime_error("NTT pass of 1..8 stages");
  }
}
}  // namespace

void launch_lde(const LdeSource& in, uint32_t* out, const uint2* tw, cudaStream_t s, int tile_begin, int tile_end,
                int plan) {
  const int T = in.L + in.rho;
  if (T > 24) throw std::runtime_error("LDE beyond the two-adic subgroup of order 2^24");
  if (in.n_cols % 8 || in.n_cols <= 0) throw std::runtime_error("LDE column count must be a multiple of 8");
  if (tile_end < 0) tile_end = in.n_cols / 8;
  if (tile_begin < 0 || tile_begin >= tile_end || tile_end > in.n_cols / 8) throw std::runtime_error("LDE tile range");
  if (plan < 0 || plan >= LDE_PLANS) plan = LDE_PLAN_DEFAULT;
  const int tiles = tile_end - tile_begin;
  // plan: the fewest passes of at most NTT_MAX_BP stages (plans 0-2) or one pass more (3-5),
  // with 2, 3 or 4 persistent blocks per SM for the double-buffered passes
  const int np = (in.L <= NTT_MAX_BP ? 1 : (in.L + NTT_MAX_BP - 1) / NTT_MAX_BP) + (plan >= 3 && in.L >= 2 ? 1 : 0);
  const uint32_t async_per_sm = 2 + uint32_t(plan % 3);
  int Bs = in.rho, left = in.L;
  for (int p = 0; p < np; p++) {
    const int Bp = (left + (np - p) - 1) / (np - p);
    const int lr_log = Bs < 2 ? Bs : 2;
    const int hi_bits = T - Bs - Bp;
    const int hg_log = (2 - lr_log) < hi_bits ? (2 - lr_log) : hi_bits;
    const unsigned gx = 1u << ((Bs - lr_log) + (hi_bits - hg_log));
    const size_t smem = ((size_t(32) << Bp) + (size_t(2) << lr_log) * ((1u << Bp) - 1)) * 4;
    const uint32_t nlines = gx * uint32_t(tiles);
    const size_t smem2 = ((size_t(64) << Bp) + size_t(8) * ((1u << Bp) - 1)) * 4;
    const uint32_t per_sm = std::min<uint32_t>(async_per_sm, uint32_t((227 * 1024) / (smem2 + 1024)));
    const uint32_t nblk = uint32_t(ntt_sm_count()) * std::max<uint32_t>(per_sm, 1);
    NttPassArgs a{in, out, T, Bs, lr_log, hg_log, tile_begin, tiles, tw, dim3(gx, tiles), smem, nlines, 0};
    if (p == 0) {
      ntt_pass_dispatch(Bp, NTT_FIRST, a, s);
    } else if (lr_log == 2 && hg_log == 0 && nlines >= 4 * nblk) {
      // enough lines for every block to pipeline several: the double-buffered kernel
      a.per = (nlines + nblk - 1) / nblk;
      a.grid = dim3((nlines + a.per - 1) / a.per);
      a.smem = smem2;
      ntt_pass_dispatch(Bp, NTT_ASYNC, a, s);
    } else {
      ntt_pass_dispatch(Bp, NTT_LATER, a, s);
    }
    WL_LAUNCH_CHECK();
    Bs += Bp;
    left -= Bp;
  }
}

void launch_merkle_tree(const uint32_t* lde, size_t rows, int n_cols, int elem, const kb::P24Consts& p24,
                        const kb::P16Consts& p16, uint32_t* tree, int LL, cudaStream_t s) {
  const int log_elem = elem == 8 ? 3 : 0;
  if (rows != (size_t(1) << LL) || n_cols % 8) throw std::runtime_error("Merkle leaves: 2^LL rows, columns in tiles of 8");
  (void)log_elem;
  launch_leaf_hash(lde, rows, n_cols, elem, p24, tree, LL, s, LEAF_PLAN_DEFAULT);
  launch_merkle_levels(tree, LL, p16, s);
}

void launch_leaf_hash(const uint32_t* lde, size_t rows, int n_cols, int elem, const kb::P24Consts& p24,
                      uint32_t* tree, int LL, cudaStream_t s, int rows_choice) {
  const int log_elem = elem == 8 ? 3 : 0;
  if (rows != (size_t(1) << LL) || n_cols % 8) throw std::runtime_error("Merkle leaves: 2^LL rows, columns in tiles of 8");
  const kb::P2ConstsFd<24> p24c = kb::p2_consts_fd(p24);
  switch (rows_choice) {
    case 0: k_leaf_hash<64><<<(unsigned)((rows + 63) / 64), 64, 0, s>>>(lde, LL, n_cols, log_elem, p24c, tree); break;
    case 2: k_leaf_hash<256><<<(unsigned)((rows + 255) / 256), 256, 0, s>>>(lde, LL, n_cols, log_elem, p24c, tree); break;
    default: k_leaf_hash<128><<<(unsigned)((rows + 127) / 128), 128, 0, s>>>(lde, LL, n_cols, log_elem, p24c, tree); break;
  }
  WL_LAUNCH_CHECK();
}

void launch_leaf_absorb(const uint32_t* lde, size_t rows, int n_cols, int elem, const kb::P24Consts& p24, int ch,
                        uint32_t* cap, uint32_t* tree, int LL, cudaStream_t s, int rows_choice) {
  const int log_elem = elem == 8 ? 3 : 0;
  if (rows != (size_t(1) << LL) || n_cols % 8) throw std::runtime_error("Merkle leaves: 2^LL rows, columns in tiles of 8");
  if (ch < 0 || ch > 7) throw std::invalid_argument("leaf chunk out of range");
  const kb::P2ConstsFd<24> p24c = kb::p2_consts_fd(p24);
  switch (rows_choice) {
    case 0: k_leaf_absorb<64><<<(unsigned)((rows + 63) / 64), 64, 0, s>>>(lde, LL, n_cols, log_elem, p24c, ch, cap, tree); break;
    case 2: k_leaf_absorb<256><<<(unsigned)((rows + 255) / 256), 256, 0, s>>>(lde, LL, n_cols, log_elem, p24c, ch, cap, tree); break;
    default: k_leaf_absorb<128><<<(unsigned)((rows + 127) / 128), 128, 0, s>>>(lde, LL, n_cols, log_elem, p24c, ch, cap, tree); break;
  }
  WL_LAUNCH_CHECK();
}

void launch_merkle_levels(uint32_t* tree, int LL, const kb::P16Consts& p16, cudaStream_t s, int plan) {
  const kb::P16Consts p16c = kb::p2_consts_canonical(p16);
  const kb::P2ConstsFd<16> p16d = kb::p2_consts_fd(p16);
  // Wide levels: one launch each, one compression per thread. Narrower levels: 16 lanes per
  // compression. The last levels (at most 128 digests) in one block. The plan sets the width
  // from which a level runs one compression per thread: 2^11, 2^13 (default) or 2^15 digests.
  const int flat_min = plan == 0 ? 11 : plan == 2 ? 15 : FLAT_LEVEL_MIN_LOG;
  int l0 = 0;
  while (l0 < LL && LL - l0 - 1 >= flat_min) {
    const size_t cnt = size_t(1) << (LL - l0 - 1);
    k_merkle_level<<<(unsigned)((cnt + 127) / 128), 128, 0, s>>>(tree, LL, l0 + 1, p16d);
    WL_LAUNCH_CHECK();
    l0++;
  }
  while (l0 < LL && LL - l0 > TOP_LEVELS) {
    const size_t threads = size_t(16) << (LL - l0 - 1);
    k_merkle_level_lanes<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(tree, LL, l0 + 1, p16c);
    WL_LAUNCH_CHECK();
    l0++;
  }
  if (l0 < LL) {
    k_merkle_top<<<1, 1024, 0, s>>>(tree, LL, l0, p16c);
    WL_LAUNCH_CHECK();
  }
}

void launch_gather_lde_rows(const uint32_t* lde, int T, const uint64_t* idx, int n_cols, int log_elem, int n,
                            uint32_t* out, const ef* mono, ef* folded, cudaStream_t s) {
  if (n_cols > 128 || log_elem < 0 || log_elem > 7) throw std::invalid_argument("gather: rows of at most 128 values");
  if (!n) return;
  k_gather_lde<<<n, 128, 0, s>>>(lde, T, idx, n_cols, log_elem, n, out, mono, folded);
  WL_LAUNCH_CHECK();
}

void launch_gather_u32(const uint32_t* src, const uint64_t* idx, int width, int n, uint32_t* out, cudaStream_t s) {
  if (!n) return;
  k_gather<<<n, 128, 0, s>>>(src, idx, width, n, out);
  WL_LAUNCH_CHECK();
}

void launch_grind(const kb::P16Consts& p16, const uint32_t* state16, const uint32_t* inbuf, int inlen, int bits,
                  uint32_t base, uint32_t count, uint32_t threads, uint32_t* result, cudaStream_t s) {
  if (bits < 1 || bits > 31 || inlen < 0 || inlen > 7) throw std::invalid_argument("grinding: bits 1..31, inlen 0..7");
  GrindState g;
  for (int i = 0; i < 16; i++) g.st[i] = kb::from_mont(state16[i]);
  for (int i = 0; i < 8; i++) g.in[i] = i < inlen ? kb::from_mont(inbuf[i]) : 0;
  threads = std::max<uint32_t>(256, std::min<uint32_t>(count, threads));
  k_grind<<<(threads + 255) / 256, 256, 0, s>>>(kb::p2_consts_fd(p16), g, inlen, bits, base, count, result);
  WL_LAUNCH_CHECK();
}

}  // namespace wl
