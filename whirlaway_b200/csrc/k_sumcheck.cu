// Sumcheck kernels: the AIR zerocheck (univariate-skip first round over the base field,
// later rounds over the extension field), the folds between rounds, the inner-phase
// helpers and the standalone a*b - c zerocheck. They compute the sums of
// crates/sumcheck/src/prove.rs:97-335 (sc_round / compute_over_hypercube) and the folds of
// crates/utils/src/multilinear.rs; the transcript work between rounds stays on the host.
//
// Column conventions: the witness is column-major (column c at wit + c * 2^n, Montgomery).
// "up" columns replace the last row by the one before it and "down" columns shift by one
// row and repeat the last (crates/air/src/utils.rs:140-160); neither is materialised.
// Folded columns are extension-field arrays, column c at cols + c * len.
#include <algorithm>
#include "finish.cuh"
#include "kernels.h"
#include "limb_mma.cuh"

namespace wl {

namespace {
using namespace kb;

__device__ __forceinline__ size_t up_row(size_t i, size_t N) { return i == N - 1 ? N - 2 : i; }
__device__ __forceinline__ size_t down_row(size_t i, size_t N) { return i == N - 1 ? N - 1 : i + 1; }

// ------------------------------------------------------------------ eq tables
// out[x] = prod_i (x_i ? r_i : 1 - r_i), x_1 = most significant bit of x.
// eq(pt, x) for x < 2^nvars, x's leading bit pairing with pt[0]. A block writes 2^EQ_BLK_BITS
// consecutive entries: x = (block << nbits) + (a << nb) + b, eq = H * A[a] * B[b], where A and
// B are tables over the block's two groups of low variables (<= 16 entries each, built in
// shared memory) and H is the product over the block's high variables (a product tree).
constexpr int EQ_MAX_VARS = 32;
constexpr int EQ_BLK_BITS = 8;
constexpr int EQ_THREADS = 1 << EQ_BLK_BITS;
__global__ void __launch_bounds__(EQ_THREADS) k_eq_table(const ef* __restrict__ pt, int nvars, ef* __restrict__ out) {
  __shared__ ef r1[EQ_MAX_VARS], r0[EQ_MAX_VARS], fac[EQ_MAX_VARS], A[16], B[16];
  const int nbits = nvars < EQ_BLK_BITS ? nvars : EQ_BLK_BITS;
  const int nhi = nvars - nbits, na = nbits / 2, nb = nbits - na;
  const int tid = threadIdx.x;
  for (int i = tid; i < nvars; i += blockDim.x) {
    const ef r = pt[i];
    r1[i] = r;
    r0[i] = ef_sub(ef_one(), r);
  }
  __syncthreads();
  const size_t xhi = blockIdx.x;
  if (tid < nhi) fac[tid] = ((xhi >> (nhi - 1 - tid)) & 1) ? r1[tid] : r0[tid];
  if (tid >= 64 && tid - 64 < (1 << na)) {
    const int a = tid - 64;
    ef v = ef_one();
    for (int i = 0; i < na; i++) v = ef_mul(v, ((a >> (na - 1 - i)) & 1) ? r1[nhi + i] : r0[nhi + i]);
    A[a] = v;
  }
  if (tid >= 96 && tid - 96 < (1 << nb)) {
    const int b = tid - 96;
    ef v = ef_one();
    for (int i = 0; i < nb; i++) v = ef_mul(v, ((b >> (nb - 1 - i)) & 1) ? r1[nhi + na + i] : r0[nhi + na + i]);
    B[b] = v;
  }
  __syncthreads();
  for (int len = nhi; len > 1;) {
    const int m = (len + 1) >> 1;
    if (tid < len - m) fac[tid] = ef_mul(fac[tid], fac[tid + m]);
    __syncthreads();
    len = m;
  }
  if (tid < (1 << nbits)) {
    const ef h = nhi ? fac[0] : ef_one();
    out[(xhi << nbits) + tid] = ef_mul(ef_mul(h, A[tid >> nb]), B[tid & ((1 << nb) - 1)]);
  }
}

__global__ void k_eq_table_f(const uint32_t* __restrict__ pts, int npts, int nvars, uint32_t* __restrict__ out) {
  size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  size_t n = size_t(npts) << nvars;
  if (i >= n) return;
  size_t p = i >> nvars;
  uint32_t x = uint32_t(i & ((size_t(1) << nvars) - 1));
  uint32_t v = R_MOD_P;
  for (int k = 0; k < nvars; k++) {
    uint32_t r = pts[p * nvars + k];
    bool bit = (x >> (nvars - 1 - k)) & 1;
    v = mul(v, bit ? r : sub(R_MOD_P, r));
  }
  out[i] = v;
}

__global__ void k_reduce_partials(const ef* __restrict__ partial, int nblk, int k, ef* __restrict__ out) {
  __shared__ ef scratch[32];
  const int j = blockIdx.x;
  ef acc = ef_zero();
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) acc = ef_add(acc, partial[size_t(b) * k + j]);
  acc = block_reduce_ef(acc, scratch);
  if (threadIdx.x == 0) out[j] = acc;
}

// ------------------------------------------------------------------ AIR zerocheck
constexpr int ZC0_X = 32;
constexpr int ZC0_STAGES = 2;   // input groups in flight
constexpr int ZC0_GROUP = 8;    // inputs per staged group (one block barrier per group)
constexpr int ZC0_PAD = 20;     // words per x in a staged column tile (16 values + padding)

__device__ __forceinline__ void cp_async4(uint32_t* smem, const uint32_t* gmem) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// The batched constraint sum_i alpha_i C_i is rewritten as
//   sum_i gamma_i cube(u_i) - sum_i alpha_i col_(17+i),
// since constraint i is (a linear map of an S-box layer) minus its committed column 17 + i:
// the full rounds' linear map moves onto the weights (gamma = MDS^T alpha, the host's betas)
// and the partial rounds' weight is alpha itself. Each cube input u_i is an affine function
// of the row: a committed column plus a round constant (the inputs of beginning and ending
// rounds 1..3), or, for the 52 others, MDS of the inputs (beginning round 0), the partial
// chain's state word 0 (the 20 partial rounds) and the state after the chain (ending round
// 0). The extension to a point z is linear and keeps constants (the Lagrange weights sum to
// one), so k_zc0_rows computes those 52 inputs once per row, and the committed-column term,
// which is linear, once per row as well (weighted by L_j(z) after its sum over x); per
// point z only the 148 cube inputs are extended, cubed and weighted.

// Source of cube input i: computed input q[qcol] (round constant included), or committed
// column 1 + i (qcol < 0) plus the round constant zc0_rc.
__device__ __forceinline__ int zc0_qcol(int i) {
  if (i < 16) return i;             // beginning round 0
  if (i < 64) return -1;            // beginning rounds 1..3: columns 17..64
  if (i < 100) return i - 48;       // partial rounds (q 16..35), ending round 0 (q 36..51)
  return -1;                        // ending rounds 1..3: columns 101..148
}
__device__ __forceinline__ uint32_t zc0_rc(const AirConsts& K, int i) {
  if (i >= 16 && i < 64) return K.begin[(i - 16) / 16 + 1][i & 15];
  if (i >= 100) return K.end[(i - 100) / 16 + 1][(i - 100) & 15];
  return 0u;
}

// One thread per row r = j S + x, reading the row's up row. Writes q[c * N + r]:
//   c < 16       MDS(inputs)_c + rc_begin[0][c]
//   16 <= c < 36 state word 0 before partial round c - 16, plus its round constant
//   36 <= c < 52 state after the 20 partial rounds, plus rc_end[0]
// and the committed-column term -L_j(z) sum_r eq[x] sum_i alpha_i col_(17+i) of the block's
// rows as partial[blockIdx.x * nz + z]; arow[r] = sum_i alpha_i col_(17+i) (the later rounds
// carry its fold as one more column).
constexpr int ZC0R_THREADS = 256;
__global__ void __launch_bounds__(ZC0R_THREADS) k_zc0_rows(const uint32_t* __restrict__ wit, int log_n, int k,
                                                           int nz, const uint32_t* __restrict__ lw,
                                                           const ef* __restrict__ eq,
                                                           const ef* __restrict__ alphas_g,
                                                           const __grid_constant__ AirConsts K,
                                                           uint32_t* __restrict__ q, ef* __restrict__ partial,
                                                           ef* __restrict__ arow) {
  __shared__ ef alphas[AIR_NC];
  __shared__ ef scratch[32];
  __shared__ ef total;
  for (int i = threadIdx.x; i < AIR_NC; i += blockDim.x) alphas[i] = alphas_g[i];
  __syncthreads();
  const int lS = log_n - k;
  const size_t N = size_t(1) << log_n;
  const size_t rb = size_t(blockIdx.x) * ZC0R_THREADS;
  const size_t r = rb + threadIdx.x;
  ef c = ef_zero();
  if (r < N) {
    const uint32_t* row = wit + up_row(r, N);
    EfMacF m;
    m.init();
#pragma unroll 1
    for (int i = 0; i < AIR_NC; i += 4) {
      uint32_t v[4];
#pragma unroll
      for (int e = 0; e < 4; e++) v[e] = __ldg(row + size_t(17 + i + e) * N);
#pragma unroll
      for (int e = 0; e < 4; e++) m.mac(alphas[i + e], v[e]);
      m.flush();
    }
    uint32_t s[16];
#pragma unroll
    for (int t = 0; t < 16; t++) s[t] = __ldg(row + size_t(1 + t) * N);
    mds_light<16>(s);
    uint32_t* qr = q + r;
#pragma unroll
    for (int t = 0; t < 16; t++) qr[size_t(t) * N] = add(s[t], K.begin[0][t]);
#pragma unroll
    for (int t = 0; t < 16; t++) s[t] = __ldg(row + size_t(65 + t) * N);
#pragma unroll 1
    for (int pr = 0; pr < 20; pr++) {
      qr[size_t(16 + pr) * N] = add(s[0], K.partial[pr]);
      internal_layer_with0<16>(s, __ldg(row + size_t(81 + pr) * N));
    }
#pragma unroll
    for (int t = 0; t < 16; t++) qr[size_t(36 + t) * N] = add(s[t], K.end[0][t]);
    const ef a = m.value();
    arow[r] = a;
    c = ef_mul(a, eq[r & ((size_t(1) << lS) - 1)]);
  }
  const size_t last = (rb + ZC0R_THREADS <= N ? rb + ZC0R_THREADS : N) - 1;
  const int nsk = 1 << k;
  if ((rb >> lS) == (last >> lS)) {  // one skip index j in the block: reduce, then weight
    const ef tot = block_reduce_ef(c, scratch);
    if (threadIdx.x == 0) total = tot;
    __syncthreads();
    const int j = int(rb >> lS);
    for (int z = threadIdx.x; z < nz; z += blockDim.x)
      partial[size_t(blockIdx.x) * nz + z] = ef_sub(ef_zero(), ef_mul_f(total, lw[size_t(z) * nsk + j]));
  } else {  // small tables: weight per row, reduce per point
    const int j = r < N ? int(r >> lS) : 0;
    for (int z = 0; z < nz; z++) {
      const ef v = block_reduce_ef(ef_mul_f(c, lw[size_t(z) * nsk + j]), scratch);
      if (threadIdx.x == 0) partial[size_t(blockIdx.x) * nz + z] = ef_sub(ef_zero(), v);
    }
  }
}

// The 148 cube inputs of every row x are extended from their values at rows j S + x, j < 2^k,
// to the points z by the Lagrange weights L_j(z), cubed, weighted by gamma and summed, weighted
// by eq[x]. The extension runs on the tensor cores: sum_j L_j(z) v_j(x) is an exact modular
// dot product over j, computed as a byte-limb integer matrix product whose rows are x, whose
// reduction index is (j, a) for the 16 points j and the 4 bytes a of v_j(x), and whose
// columns are (z, b) for the 4 bytes b of M(j, z, a) = the Montgomery form of L_j(z) 2^(8a).
// The reduction index needs no byte shuffling: the staged words [x][j] are the A operand as
// they lie (byte a of word j is k = 4j + a). With acc_b = sum_(j,a) v_(j,a) M_b(j, z, a) below
// 2^22, v = sum_b acc_b 2^(8b) < 2^46 is congruent to (sum_j v_j L_j(z)) R^2, so one Montgomery
// reduction (with the round constant in the high word) gives the cube input in Montgomery form.
// A block holds 32 x (two 16-row tiles) and the z-octets of all points; warp (tile, octet)
// issues 4 n8 tiles (b = 0..3) per k32 step, so each lane ends with all limbs of 4 (x, z)
// sums, and the B fragments (16 words per lane) depend on z only. The 16 x 32 values of each
// input are staged in shared memory by a cp.async pipeline, ZC0_GROUP inputs per stage; the
// weights of j >= 2^k are zero, so unstaged entries contribute nothing.
constexpr int ZC0M_WARPS = 8;  // 2 x-tiles x 4 z-octets (30 points)
__global__ void __launch_bounds__(ZC0M_WARPS * 32, 2) k_zc0_eval_mma(const uint32_t* __restrict__ wit,
                                                                    const uint32_t* __restrict__ q, int log_n,
                                                                    int k, int nz, const uint32_t* __restrict__ lw,
                                                                    const ef* __restrict__ eq,
                                                                    const ef* __restrict__ alphas_g,
                                                                    const ef* __restrict__ betas_g,
                                                                    const __grid_constant__ AirConsts K,
                                                                    ef* __restrict__ partial) {
  __shared__ ef gam[AIR_NC];
  __shared__ uint32_t rcs[AIR_NC];
  __shared__ __align__(16) uint32_t tile[ZC0_STAGES][ZC0_GROUP][ZC0_X * ZC0_PAD];
  __shared__ ef red[4][8];  // per z-octet and point: the sum over the second x-tile
  constexpr int NT = ZC0M_WARPS * 32;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3, mt = warp & 1, zo = warp >> 1;
  for (int i = tid; i < AIR_NC; i += NT) {
    gam[i] = i < 64 ? betas_g[i] : (i < 84 ? alphas_g[i] : betas_g[i - 20]);
    rcs[i] = zc0_rc(K, i);
  }
  const int nsk = 1 << k;
  const size_t N = size_t(1) << log_n;
  const size_t S = N >> k;
  const size_t x0 = size_t(blockIdx.x) * ZC0_X;
  const bool zwarp = zo * 8 < nz;  // warps of octets past the last point only stage

  // B fragments: bf[b][kk][h] packs, in byte a, byte b of M(j, z, a) for j = 8 kk + 4 h + t
  // and z = 8 zo + g (the lane's B column)
  uint32_t bf[4][2][2];
  {
    const int z = zo * 8 + g;
#pragma unroll
    for (int kk = 0; kk < 2; kk++)
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int j = 8 * kk + 4 * h + t;
        const uint32_t L = (z < nz && j < nsk) ? lw[z * nsk + j] : 0u;
        uint32_t m[4];
#pragma unroll
        for (int a = 0; a < 4; a++) m[a] = kb::mul(L, uint32_t(kb::detail::cpow(2, 8 * a + 32)));
#pragma unroll
        for (int b = 0; b < 4; b++)
          bf[b][kk][h] = ((m[0] >> (8 * b)) & 0xffu) | (((m[1] >> (8 * b)) & 0xffu) << 8) |
                         (((m[2] >> (8 * b)) & 0xffu) << 16) | (((m[3] >> (8 * b)) & 0xffu) << 24);
      }
  }

  // staged entries of this thread: e = tid, tid + NT of the 16 x 32 (j, x) grid; source row
  // j S + x (the up row for committed columns differs only at row N - 1)
  constexpr int NE = (16 * ZC0_X + NT - 1) / NT;
  uint32_t srow[NE], sdst[NE];
  bool sval[NE], slast[NE];
#pragma unroll
  for (int e = 0; e < NE; e++) {
    const int idx = tid + e * NT;
    const int j = idx / ZC0_X, xl = idx % ZC0_X;
    size_t xx = x0 + xl;
    if (xx >= S) xx = 0;
    sval[e] = idx < 16 * ZC0_X && j < nsk;
    srow[e] = uint32_t(size_t(j) * S + xx);
    slast[e] = size_t(j) * S + xx == N - 1;
    sdst[e] = uint32_t(xl * ZC0_PAD + j);
  }
  auto issue = [&](int grp) {
#pragma unroll
    for (int cc = 0; cc < ZC0_GROUP; cc++) {
      const int i = ZC0_GROUP * grp + cc;
      if (i < AIR_NC) {
        const int qc = zc0_qcol(i);
        const uint32_t* col = qc >= 0 ? q + size_t(qc) * N : wit + size_t(1 + i) * N;
        uint32_t* dst = tile[grp % ZC0_STAGES][cc];
#pragma unroll
        for (int e = 0; e < NE; e++)
          if (sval[e]) cp_async4(dst + sdst[e], col + (srow[e] - uint32_t(slast[e] && qc < 0)));
      }
    }
    cp_async_commit();
  };
  for (int grp = 0; grp < ZC0_STAGES - 1; grp++) issue(grp);
  EfMacF m[4];  // (x, z) = (g, 2t), (g, 2t + 1), (g + 8, 2t), (g + 8, 2t + 1) of the warp's tile
#pragma unroll
  for (int o = 0; o < 4; o++) m[o].init();
  constexpr int NG = (AIR_NC + ZC0_GROUP - 1) / ZC0_GROUP;
  static_assert(ZC0_GROUP % 4 == 0 && AIR_NC % 4 == 0, "flushes after every 4 products");
#pragma unroll 1
  for (int grp = 0; grp < NG; grp++) {
    cp_async_wait<ZC0_STAGES - 2>();
    __syncthreads();  // group grp landed for every thread; the slot of group grp - 1 is free
    issue(grp + ZC0_STAGES - 1);
    if (zwarp) {
#pragma unroll 2
      for (int cc = 0; cc < ZC0_GROUP; cc++) {
        const int i = ZC0_GROUP * grp + cc;
        if (i >= AIR_NC) break;  // the last group is partial
        const uint32_t* r0 = tile[grp % ZC0_STAGES][cc] + (16 * mt + g) * ZC0_PAD;
        const uint32_t* r1 = r0 + 8 * ZC0_PAD;
        int acc[4][4];
#pragma unroll
        for (int b = 0; b < 4; b++)
#pragma unroll
          for (int o = 0; o < 4; o++) acc[b][o] = 0;
#pragma unroll
        for (int kk = 0; kk < 2; kk++) {
          const uint32_t af[4] = {r0[8 * kk + t], r1[8 * kk + t], r0[8 * kk + t + 4], r1[8 * kk + t + 4]};
#pragma unroll
          for (int b = 0; b < 4; b++) mma_u8_16832(acc[b], af, bf[b][kk][0], bf[b][kk][1]);
        }
        const uint64_t rc_hi = uint64_t(rcs[i]) << 32;
        const ef& gm = gam[i];
#pragma unroll
        for (int o = 0; o < 4; o++) {
          const uint32_t lo = uint32_t(acc[0][o]) + (uint32_t(acc[1][o]) << 8);  // < 2^31
          const uint32_t hi = uint32_t(acc[2][o]) + (uint32_t(acc[3][o]) << 8);  // < 2^31
          const uint32_t u = kb::redc(uint64_t(lo) + (uint64_t(hi) << 16) + rc_hi);
          m[o].mac(gm, kb::cube(u));
        }
        if ((cc & 3) == 3) {
#pragma unroll
          for (int o = 0; o < 4; o++) m[o].flush();
        }
      }
    }
  }
  cp_async_wait<0>();
  // weight by eq[x], sum over the 16 x of the tile (lanes of equal t), then over the two tiles
  ef sz[2];
#pragma unroll
  for (int c = 0; c < 2; c++) {
    ef acc = ef_zero();
#pragma unroll
    for (int hh = 0; hh < 2; hh++) {
      const size_t x = x0 + 16 * mt + g + 8 * hh;
      const ef v = m[2 * hh + c].value();
      if (zwarp && x < S) acc = ef_add(acc, ef_mul(v, eq[x]));
    }
#pragma unroll
    for (int d = 4; d < 32; d <<= 1) {
      ef o;
#pragma unroll
      for (int w = 0; w < 8; w++) o.c[w] = __shfl_xor_sync(0xffffffffu, acc.c[w], d);
      acc = ef_add(acc, o);
    }
    sz[c] = acc;
  }
  if (mt == 1 && g == 0) {
    red[zo][2 * t] = sz[0];
    red[zo][2 * t + 1] = sz[1];
  }
  __syncthreads();
  if (mt == 0 && g == 0) {
#pragma unroll
    for (int c = 0; c < 2; c++) {
      const int z = zo * 8 + 2 * t + c;
      if (z < nz) partial[size_t(blockIdx.x) * nz + z] = ef_add(sz[c], red[zo][2 * t + c]);
    }
  }
}

// out[c * S + x] = sum_j sel[j] * up_c[j * S + x] for every column c, on the tensor cores as
// in k_zc0_eval_mma: rows x, reduction index (j, a) over the 16 points and the 4 bytes of
// up_c[j S + x] (the staged [x][j] words as they lie), columns (n, b) for the 8 coefficients n
// of sel[j] and the 4 bytes b of the Montgomery form of sel[j]_n 2^(8a). Each lane ends with
// all limbs of coefficients 2t, 2t + 1 of rows g, g + 8; one Montgomery reduction each. A
// block holds 32 x and walks the columns in staged groups of ZC0_GROUP; warp (tile, slot)
// takes columns slot and slot + 4 of each group. The up row of row N - 1 is N - 2.
__global__ void __launch_bounds__(ZC0M_WARPS * 32) k_zc0_fold_mma(const uint32_t* __restrict__ wit, int log_n,
                                                                 int k, const ef* __restrict__ sel,
                                                                 ef* __restrict__ out) {
  __shared__ __align__(16) uint32_t tile[ZC0_STAGES][ZC0_GROUP][ZC0_X * ZC0_PAD];
  constexpr int NT = ZC0M_WARPS * 32;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3, mt = warp & 1, slot = warp >> 1;
  const int nsk = 1 << k;
  const size_t N = size_t(1) << log_n;
  const size_t S = N >> k;
  const size_t x0 = size_t(blockIdx.x) * ZC0_X;
  // B fragments: bf[b][kk][h] packs, in byte a, byte b of the Montgomery form of
  // sel[j]_n 2^(8a) for j = 8 kk + 4 h + t and coefficient n = g (the lane's B column)
  uint32_t bf[4][2][2];
#pragma unroll
  for (int kk = 0; kk < 2; kk++)
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int j = 8 * kk + 4 * h + t;
      const uint32_t v = j < nsk ? sel[j].c[g] : 0u;
      uint32_t m[4];
#pragma unroll
      for (int a = 0; a < 4; a++) m[a] = kb::mul(v, uint32_t(kb::detail::cpow(2, 8 * a + 32)));
#pragma unroll
      for (int b = 0; b < 4; b++)
        bf[b][kk][h] = ((m[0] >> (8 * b)) & 0xffu) | (((m[1] >> (8 * b)) & 0xffu) << 8) |
                       (((m[2] >> (8 * b)) & 0xffu) << 16) | (((m[3] >> (8 * b)) & 0xffu) << 24);
    }
  constexpr int NE = (16 * ZC0_X + NT - 1) / NT;
  uint32_t srow[NE], sdst[NE];
  bool sval[NE];
#pragma unroll
  for (int e = 0; e < NE; e++) {
    const int idx = tid + e * NT;
    const int j = idx / ZC0_X, xl = idx % ZC0_X;
    size_t xx = x0 + xl;
    if (xx >= S) xx = 0;
    sval[e] = idx < 16 * ZC0_X && j < nsk;
    const size_t row = size_t(j) * S + xx;
    srow[e] = uint32_t(row == N - 1 ? N - 2 : row);
    sdst[e] = uint32_t(xl * ZC0_PAD + j);
  }
  auto issue = [&](int grp) {
#pragma unroll
    for (int cc = 0; cc < ZC0_GROUP; cc++) {
      const int c = ZC0_GROUP * grp + cc;
      if (c < AIR_W) {
        const uint32_t* col = wit + size_t(c) * N;
        uint32_t* dst = tile[grp % ZC0_STAGES][cc];
#pragma unroll
        for (int e = 0; e < NE; e++)
          if (sval[e]) cp_async4(dst + sdst[e], col + srow[e]);
      }
    }
    cp_async_commit();
  };
  for (int grp = 0; grp < ZC0_STAGES - 1; grp++) issue(grp);
  constexpr int NG = (AIR_W + ZC0_GROUP - 1) / ZC0_GROUP;
  const size_t xa = x0 + 16 * mt + g, xb = xa + 8;
#pragma unroll 1
  for (int grp = 0; grp < NG; grp++) {
    cp_async_wait<ZC0_STAGES - 2>();
    __syncthreads();  // group grp landed for every thread; the slot of group grp - 1 is free
    issue(grp + ZC0_STAGES - 1);
#pragma unroll
    for (int r = 0; r < 2; r++) {
      const int cc = slot + 4 * r;
      const int c = ZC0_GROUP * grp + cc;
      if (c >= AIR_W) break;
      const uint32_t* r0 = tile[grp % ZC0_STAGES][cc] + (16 * mt + g) * ZC0_PAD;
      const uint32_t* r1 = r0 + 8 * ZC0_PAD;
      int acc[4][4];
#pragma unroll
      for (int b = 0; b < 4; b++)
#pragma unroll
        for (int o = 0; o < 4; o++) acc[b][o] = 0;
#pragma unroll
      for (int kk = 0; kk < 2; kk++) {
        const uint32_t af[4] = {r0[8 * kk + t], r1[8 * kk + t], r0[8 * kk + t + 4], r1[8 * kk + t + 4]};
#pragma unroll
        for (int b = 0; b < 4; b++) mma_u8_16832(acc[b], af, bf[b][kk][0], bf[b][kk][1]);
      }
      uint32_t res[4];
#pragma unroll
      for (int o = 0; o < 4; o++) {
        const uint32_t lo = uint32_t(acc[0][o]) + (uint32_t(acc[1][o]) << 8);  // < 2^31
        const uint32_t hi = uint32_t(acc[2][o]) + (uint32_t(acc[3][o]) << 8);  // < 2^31
        res[o] = kb::redc(uint64_t(lo) + (uint64_t(hi) << 16));
      }
      if (xa < S) reinterpret_cast<uint2*>(out + size_t(c) * S + xa)[t] = make_uint2(res[0], res[1]);
      if (xb < S) reinterpret_cast<uint2*>(out + size_t(c) * S + xb)[t] = make_uint2(res[2], res[3]);
    }
  }
  cp_async_wait<0>();
}

// out[x] = sum_j sel[j] * a[j * S + x] for an extension-field table a that is already read at
// up rows (the committed-column combination of k_zc0_rows).
__global__ void k_zc0_fold_ef(const ef* __restrict__ a, int log_n, int k, const ef* __restrict__ sel,
                              ef* __restrict__ out) {
  const size_t N = size_t(1) << log_n, S = N >> k;
  const size_t x = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (x >= S) return;
  EfMacE m;
  m.init();
  for (int j = 0; j < (1 << k); j++) m.mac(sel[j], a[size_t(j) * S + x]);
  out[x] = m.value();
}

// ------------------------------------------------------------------ zerocheck rounds >= 1
// One block per (x, z), x < 2^(m-1), z in {0, 2, 3}: the 148 batched constraints at the
// point whose columns are lo + z (hi - lo) (lo, hi = the column at x and 2^(m-1) + x).
//  * Warps 0-3: thread (seg, j), seg < 7, j < 16, one full-round constraint without state.
//    For full round f with weights alpha_(c0+i), sum_i alpha_(c0+i) (MDS(cubes)_i - post_i)
//    = sum_j beta_(f,j) cube_j - sum_i alpha_(c0+i) post_i with beta_f = MDS^T alpha (from
//    the host); each round's input is committed: the previous round's post columns, or
//    MDS(inputs) for the first round. seg 0..3 = beginning rounds, 4..6 = ending rounds 1..3.
//  * Warp 4: the 20 partial rounds and ending round 0, whose input is the state after the
//    partial rounds. Lane i < 16 holds state word i; the internal layer's sum is a shuffle
//    reduction over the 16 lanes. The state continues from the committed partial post p_r,
//    so the S-box of round r is off the chain: lane r keeps state word 0 of round r and the
//    20 S-box constraints are evaluated in parallel after the loop.
constexpr int ZCE_THREADS = 160;

__device__ __forceinline__ void m4_ef(ef& x0, ef& x1, ef& x2, ef& x3) {
  ef t01 = ef_add(x0, x1), t23 = ef_add(x2, x3), t0123 = ef_add(t01, t23);
  ef t01123 = ef_add(t0123, x1), t01233 = ef_add(t0123, x3);
  ef y3 = ef_add(t01233, ef_add(x0, x0));
  ef y1 = ef_add(t01123, ef_add(x2, x2));
  ef y0 = ef_add(t01123, t01);
  ef y2 = ef_add(t01233, t23);
  x0 = y0;
  x1 = y1;
  x2 = y2;
  x3 = y3;
}

__device__ __forceinline__ ef shfl_xor_ef(const ef& v, int d) {
  ef r;
#pragma unroll
  for (int i = 0; i < 8; i++) r.c[i] = __shfl_xor_sync(0xffffffffu, v.c[i], d);
  return r;
}
__device__ __forceinline__ ef shfl_idx_ef(const ef& v, int src) {
  ef r;
#pragma unroll
  for (int i = 0; i < 8; i++) r.c[i] = __shfl_sync(0xffffffffu, v.c[i], src);
  return r;
}

__global__ void __launch_bounds__(ZCE_THREADS) k_zc_ef(const ef* __restrict__ cols, int m, const ef* __restrict__ eq,
                                                      const ef* __restrict__ alphas, const ef* __restrict__ betas,
                                                      const __grid_constant__ AirConsts K, ef* __restrict__ partial) {
  const size_t len = size_t(1) << m, half = len >> 1;
  const size_t x = blockIdx.x / 3;
  const int zi = blockIdx.x - int(x) * 3;
  auto get = [&](int c) -> ef {
    const ef lo = cols[size_t(c) * len + x];
    if (zi == 0) return lo;
    const ef hi = cols[size_t(c) * len + half + x];
    ef d = ef_sub(hi, lo);
    ef v = ef_add(hi, d);               // z = 2: 2 hi - lo
    return zi == 1 ? v : ef_add(v, d);  // z = 3: 3 hi - 2 lo
  };
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  ef acc = ef_zero();
  if (warp < 4) {
    if (tid < 112) {
      const int seg = tid >> 4, j = tid & 15;
      const int f = seg < 4 ? seg : seg + 1;
      const uint32_t rc = seg < 4 ? K.begin[seg][j] : K.end[seg - 3][j];
      const int post = seg < 4 ? 17 + 16 * seg : 101 + 16 * (seg - 3);
      ef in;
      if (seg == 0) {
        // MDS(inputs)_j: the M4 output of chunk j / 4 plus the sum over chunks of position j % 4
        const int q0 = j >> 2, k0 = j & 3;
        ef S = ef_zero(), own = ef_zero();
#pragma unroll 1
        for (int q = 0; q < 4; q++) {
          ef y[4] = {get(1 + 4 * q), get(2 + 4 * q), get(3 + 4 * q), get(4 + 4 * q)};
          m4_ef(y[0], y[1], y[2], y[3]);
          const ef yk = k0 == 0 ? y[0] : k0 == 1 ? y[1] : k0 == 2 ? y[2] : y[3];
          S = ef_add(S, yk);
          if (q == q0) own = yk;
        }
        in = ef_add(own, S);
      } else {
        in = get(post - 16 + j);
      }
      acc = ef_mul(betas[16 * f + j], ef_cube(ef_add_f(in, rc)));
    }
  } else {
    const int i = lane & 15;
    ef st = get(65 + i);                          // state after beginning round 3
    const ef pr = lane < 20 ? get(81 + lane) : ef_zero();  // partial posts
    const uint32_t dg = p2_diag<16>(i);
    ef s0r = ef_zero();  // lane r: state word 0 at partial round r
#pragma unroll 1
    for (int r = 0; r < 20; r++) {
      const ef w0 = shfl_idx_ef(st, 0);
      if (lane == r) s0r = w0;
      const ef p = shfl_idx_ef(pr, r);
      ef sp = i == 0 ? p : st;
      ef sum = sp;
#pragma unroll
      for (int d = 8; d > 0; d >>= 1) sum = ef_add(sum, shfl_xor_ef(sum, d));
      st = ef_add(ef_mul_f(sp, dg), sum);
    }
    if (lane < 20) {
      const ef x0 = ef_cube(ef_add_f(s0r, K.partial[lane]));
      acc = ef_mul(alphas[64 + lane], x0);
    }
    if (lane < 16) {
      acc = ef_add(acc, ef_mul(betas[16 * 4 + i], ef_cube(ef_add_f(st, K.end[0][i]))));
    }
  }
  acc = warp_reduce_ef(acc);
  __shared__ ef wsum[ZCE_THREADS / 32];
  if (lane == 0) wsum[warp] = acc;
  __syncthreads();
  if (tid == 0) {
    ef tot = wsum[0];
#pragma unroll
    for (int w = 1; w < ZCE_THREADS / 32; w++) tot = ef_add(tot, wsum[w]);
    // the committed-post terms of all 148 constraints: the carried column
    partial[blockIdx.x] = ef_mul(ef_sub(tot, get(AIR_W)), eq[x]);
  }
}

// Dense forms of k_zc_ef for large rounds, in two kernels so that each keeps few
// registers; both weight each point by eq[x] and write one partial sum per block and z
// (blockIdx.y), first the full-round kernel's blocks, then the partial-round kernel's.
//  * k_zc_full_dense: 16 lanes per point (2 points per warp); lane j evaluates constraint j
//    of the 7 stateless full rounds. Beginning round 0 takes MDS(inputs): the lane's M4
//    output plus the sum over the point's 4 chunks (two shuffles).
//  * k_zc_partial_dense: 8 lanes per point (4 per warp); lane sub holds state words 2 sub,
//    2 sub + 1 through the 20 partial rounds (the internal layer's sum is a local add plus
//    three shuffles), keeps state word 0 of rounds r = sub (mod 8) for their S-box
//    constraints, evaluated after the chain, and evaluates its two words of ending round 0.
constexpr int ZCD_WARPS = 4;
constexpr int ZCD_FULL_PTS = ZCD_WARPS * 2;     // points per block
constexpr int ZCD_PARTIAL_PTS = ZCD_WARPS * 4;

template <int PTS>
__device__ __forceinline__ void zcd_block_store(ef v, ef* __restrict__ partial, size_t blk, int zi) {
  __shared__ ef wsum[ZCD_WARPS];
  v = warp_reduce_ef(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) wsum[warp] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    ef t = wsum[0];
#pragma unroll
    for (int w = 1; w < ZCD_WARPS; w++) t = ef_add(t, wsum[w]);
    partial[blk * 3 + zi] = t;
  }
}

#define ZCD_GET                                                            \
  auto get = [&](int c) -> ef {                                             \
    const ef lo = cols[size_t(c) * len + xs];                               \
    if (zi == 0) return lo;                                                 \
    const ef hi = cols[size_t(c) * len + half + xs];                        \
    ef d = ef_sub(hi, lo);                                                  \
    ef v = ef_add(hi, d);                                                   \
    return zi == 1 ? v : ef_add(v, d);                                      \
  }

__global__ void __launch_bounds__(ZCD_WARPS * 32) k_zc_full_dense(const ef* __restrict__ cols, int m,
                                                                 const ef* __restrict__ eq,
                                                                 const ef* __restrict__ alphas,
                                                                 const ef* __restrict__ betas,
                                                                 const __grid_constant__ AirConsts K,
                                                                 ef* __restrict__ partial) {
  const size_t len = size_t(1) << m, half = len >> 1;
  const int lane = threadIdx.x & 31, zi = blockIdx.y;
  const int j = lane & 15;
  const size_t x = size_t(blockIdx.x) * ZCD_FULL_PTS + (threadIdx.x >> 4);
  const bool valid = x < half;
  const size_t xs = valid ? x : 0;
  ZCD_GET;
  ef in;
  {
    const int q = j >> 2;
    ef y0 = get(1 + 4 * q), y1 = get(2 + 4 * q), y2 = get(3 + 4 * q), y3 = get(4 + 4 * q);
    m4_ef(y0, y1, y2, y3);
    const int k0 = j & 3;
    const ef y = k0 == 0 ? y0 : k0 == 1 ? y1 : k0 == 2 ? y2 : y3;
    ef t = ef_add(y, shfl_xor_ef(y, 4));
    t = ef_add(t, shfl_xor_ef(t, 8));
    in = ef_add(y, t);
  }
  EfMacE pos;  // beta * cube terms
  pos.init();
  // A round's input is the previous round's post, which this lane already holds, except for
  // ending round 1 (segment 4), whose input is ending round 0's post. The next segment's
  // post (and that one input) are loaded a segment ahead.
  auto post_of = [](int seg) { return seg < 4 ? 17 + 16 * seg : 101 + 16 * (seg - 3); };
  ef pv = get(post_of(0) + j);
  ef in4 = ef_zero();
#pragma unroll 1
  for (int seg = 0; seg < 7; seg++) {
    const int f = seg < 4 ? seg : seg + 1;
    const uint32_t rc = seg < 4 ? K.begin[seg][j] : K.end[seg - 3][j];
    const ef pv_next = seg < 5 ? get(post_of(seg + 1) + j) : ef_zero();
    if (seg == 3) in4 = get(101 + j);
    pos.mac(betas[16 * f + j], ef_cube(ef_add_f(in, rc)));
    in = seg == 3 ? in4 : pv;
    pv = pv_next;
  }
  // the committed-post terms of all 148 constraints are the carried column sum_i alpha_i
  // col_(17+i), subtracted once per point
  const ef acc = j == 0 ? ef_sub(pos.value(), get(AIR_W)) : pos.value();
  // fold the point's 16 lanes, weight by eq, then the block sum
  ef pt = acc;
#pragma unroll
  for (int d = 8; d > 0; d >>= 1) pt = ef_add(pt, shfl_xor_ef(pt, d));
  const ef res = (j == 0 && valid) ? ef_mul(pt, eq[xs]) : ef_zero();
  zcd_block_store<ZCD_FULL_PTS>(res, partial, blockIdx.x, zi);
}

__global__ void __launch_bounds__(ZCD_WARPS * 32) k_zc_partial_dense(const ef* __restrict__ cols, int m,
                                                                    const ef* __restrict__ eq,
                                                                    const ef* __restrict__ alphas,
                                                                    const ef* __restrict__ betas,
                                                                    const __grid_constant__ AirConsts K,
                                                                    ef* __restrict__ partial) {
  const size_t len = size_t(1) << m, half = len >> 1;
  const int lane = threadIdx.x & 31, zi = blockIdx.y;
  const int sub = lane & 7, gbase = lane & ~7;
  const size_t x = size_t(blockIdx.x) * ZCD_PARTIAL_PTS + (threadIdx.x >> 3);
  const bool valid = x < half;
  const size_t xs = valid ? x : 0;
  ZCD_GET;
  ef st[2];
  uint32_t dg[2];
#pragma unroll
  for (int kk = 0; kk < 2; kk++) {
    st[kk] = get(65 + 2 * sub + kk);
    dg[kk] = p2_diag<16>(2 * sub + kk);
  }
  // rounds in groups of 8 (a rolled loop keeps the code small): in group t, lane sub holds
  // the partial post p_(8t+sub), records state word 0 of round 8t + sub, and evaluates that
  // round's S-box constraint once the group is done
  EfMacE pos;  // S-box / cube terms (the committed-post terms are in k_zc_full_dense)
  pos.init();
  ef p_cur = get(81 + sub);
#pragma unroll 1
  for (int t = 0; t < 3; t++) {
    ef s0_cur = ef_zero();
#pragma unroll
    for (int o = 0; o < 8; o++) {
      if (8 * t + o >= 20) break;
      const ef w0 = shfl_idx_ef(st[0], gbase);
      if (sub == o) s0_cur = w0;
      const ef p = shfl_idx_ef(p_cur, gbase | o);
      if (sub == 0) st[0] = p;
      ef sum = ef_add(st[0], st[1]);
      sum = ef_add(sum, shfl_xor_ef(sum, 1));
      sum = ef_add(sum, shfl_xor_ef(sum, 2));
      sum = ef_add(sum, shfl_xor_ef(sum, 4));
#pragma unroll
      for (int kk = 0; kk < 2; kk++) st[kk] = ef_add(ef_mul_f(st[kk], dg[kk]), sum);
    }
    const int r = 8 * t + sub;
    if (r < 20) {
      pos.mac(alphas[64 + r], ef_cube(ef_add_f(s0_cur, K.partial[r])));
    }
    if (t < 2) p_cur = (r + 8 < 20) ? get(81 + r + 8) : ef_zero();
  }
#pragma unroll
  for (int kk = 0; kk < 2; kk++) {
    const int j = 2 * sub + kk;
    pos.mac(betas[16 * 4 + j], ef_cube(ef_add_f(st[kk], K.end[0][j])));
  }
  ef pt = pos.value();
#pragma unroll
  for (int d = 4; d > 0; d >>= 1) pt = ef_add(pt, shfl_xor_ef(pt, d));
  const ef res = (sub == 0 && valid) ? ef_mul(pt, eq[xs]) : ef_zero();
  zcd_block_store<ZCD_PARTIAL_PTS>(res, partial, blockIdx.x, zi);
}

// Folds every column at the challenge (*r, or rv when r is null) and, in the extra column
// slot, sums the next round's eq table out of the current one.
__global__ void k_fold_cols(const ef* __restrict__ in, ef* __restrict__ out, size_t half, int ncols,
                            const ef* __restrict__ r, ef rv, const ef* __restrict__ eq_in, ef* __restrict__ eq_out,
                            size_t eq_half) {
  const size_t x = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (c == ncols) {
    if (x < eq_half) eq_out[x] = ef_add(eq_in[x], eq_in[x + eq_half]);
    return;
  }
  if (x >= half) return;
  const ef* src = in + size_t(c) * 2 * half;
  out[size_t(c) * half + x] = ef_lerp(src[x], src[half + x], r ? *r : rv);
}

// lo + r (hi - lo) for the 16 values of a warp's tile on the tensor cores (byte-limb value
// form): r d = sum_e d_e (X^e r), so the product is a matrix product with rows = values,
// reduction index = (coefficient e of d, byte a), columns = (n, b) for the 8 coefficients n and
// 4 bytes b of the Montgomery form of (X^e r)_n 2^(8a) (the lane's B fragments, fold_frag).
// One k32 step: four mma per 16 values; acc_b < 32 255^2, one reduction per coefficient.
__device__ __forceinline__ void fold_frag(const ef& r, int g, int t, uint32_t (&bf)[4][2]) {
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int e = t + 4 * h;
    // (X^e r)_g = r_(g - e), times 3 where X^8 = 3 wraps it
    const uint32_t w = g >= e ? r.c[g - e] : kb::add(kb::dbl(r.c[g - e + 8]), r.c[g - e + 8]);
    uint32_t m[4];
#pragma unroll
    for (int a = 0; a < 4; a++) m[a] = kb::mul(w, uint32_t(kb::detail::cpow(2, 8 * a + 32)));
#pragma unroll
    for (int b = 0; b < 4; b++)
      bf[b][h] = ((m[0] >> (8 * b)) & 0xffu) | (((m[1] >> (8 * b)) & 0xffu) << 8) |
                 (((m[2] >> (8 * b)) & 0xffu) << 16) | (((m[3] >> (8 * b)) & 0xffu) << 24);
  }
}
__device__ __forceinline__ void lerp16_mma(const ef* __restrict__ lo, const ef* __restrict__ hi, ef* __restrict__ out,
                                           uint32_t nv, const uint32_t (&bf)[4][2], int g, int t) {
  const uint32_t* l32 = reinterpret_cast<const uint32_t*>(lo);
  const uint32_t* h32 = reinterpret_cast<const uint32_t*>(hi);
  const bool va = uint32_t(g) < nv, vb = uint32_t(g + 8) < nv;
  auto dw = [&](int row, int e, bool v) -> uint32_t { return v ? kb::sub(h32[row * 8 + e], l32[row * 8 + e]) : 0u; };
  const uint32_t af[4] = {dw(g, t, va), dw(g + 8, t, vb), dw(g, t + 4, va), dw(g + 8, t + 4, vb)};
  int acc[4][4];
#pragma unroll
  for (int b = 0; b < 4; b++) {
#pragma unroll
    for (int o = 0; o < 4; o++) acc[b][o] = 0;
    mma_u8_16832(acc[b], af, bf[b][0], bf[b][1]);
  }
  auto prod = [&](int o) {
    return kb::redc(uint64_t(uint32_t(acc[0][o])) + (uint64_t(uint32_t(acc[1][o])) << 8) +
                    (uint64_t(uint32_t(acc[2][o])) << 16) + (uint64_t(uint32_t(acc[3][o])) << 24));
  };
  // lane (g, t) holds coefficients 2t, 2t + 1 of rows g and g + 8
  if (va) {
    const uint2 l = reinterpret_cast<const uint2*>(lo + g)[t];
    reinterpret_cast<uint2*>(out + g)[t] = make_uint2(kb::add(l.x, prod(0)), kb::add(l.y, prod(1)));
  }
  if (vb) {
    const uint2 l = reinterpret_cast<const uint2*>(lo + g + 8)[t];
    reinterpret_cast<uint2*>(out + g + 8)[t] = make_uint2(kb::add(l.x, prod(2)), kb::add(l.y, prod(3)));
  }
}
// k_fold_cols with the challenge by value, 16 values per warp on the tensor cores; the extra
// column slot (blockIdx.y == ncols) sums the next eq table as k_fold_cols does.
// The challenge comes by value (rv) or, when rptr is set, from device memory (a challenge
// sampled on the device by the round-finishing kernel).
__global__ void __launch_bounds__(256) k_fold_cols_mma(const ef* __restrict__ in, ef* __restrict__ out, size_t half,
                                                      int ncols, ef rv, const ef* __restrict__ rptr,
                                                      const ef* __restrict__ eq_in, ef* __restrict__ eq_out,
                                                      size_t eq_half) {
  const int c = blockIdx.y;
  if (c == ncols) {
    const size_t x = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (x < eq_half) eq_out[x] = ef_add(eq_in[x], eq_in[x + eq_half]);
    return;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  const size_t x0 = (size_t(blockIdx.x) * 8 + warp) * 16;
  if (x0 >= half) return;  // whole warp
  uint32_t bf[4][2];
  fold_frag(rptr ? *rptr : rv, g, t, bf);
  const ef* src = in + size_t(c) * 2 * half;
  const uint32_t nv = half - x0 < 16 ? uint32_t(half - x0) : 16u;
  lerp16_mma(src + x0, src + half + x0, out + size_t(c) * half + x0, nv, bf, g, t);
}
// lo + r (hi - lo) for two tables with the challenge by value: blockIdx.y selects (a, oa) or (b, ob).
__global__ void __launch_bounds__(256) k_fold2_mma(const ef* __restrict__ a, const ef* __restrict__ b,
                                                  ef* __restrict__ oa, ef* __restrict__ ob, size_t half, ef rv,
                                                  const ef* __restrict__ rptr) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  const size_t x0 = (size_t(blockIdx.x) * 8 + warp) * 16;
  if (x0 >= half) return;  // whole warp
  uint32_t bf[4][2];
  fold_frag(rptr ? *rptr : rv, g, t, bf);
  const ef* src = blockIdx.y ? b : a;
  ef* dst = blockIdx.y ? ob : oa;
  const uint32_t nv = half - x0 < 16 ? uint32_t(half - x0) : 16u;
  lerp16_mma(src + x0, src + half + x0, dst + x0, nv, bf, g, t);
}

// Per (column c, j < 2^k, x_hi): eq_hi[x_hi] * sum_{x_lo} eq_lo[x_lo] * up_c[j S + x] (and the
// same for down), x = x_hi 2^ll + x_lo, with eq(tail, x) = eq_hi(x_hi) eq_lo(x_lo) factored so
// every warp reads the same small eq_lo table. One warp per x_hi; 2^ll is a multiple of 32
// or smaller than 32. Outputs pu/pd[(c * 2^k + j) * nhi + x_hi].
constexpr int IS_WARPS = 8;
__global__ void __launch_bounds__(IS_WARPS * 32) k_inner_sums(const uint32_t* __restrict__ wit, int log_n, int k,
                                                              int ll, const ef* __restrict__ eq_hi,
                                                              const ef* __restrict__ eq_lo, ef* __restrict__ pu,
                                                              ef* __restrict__ pd) {
  // columns c0 and c0 + 1 (when it exists) share each eq_lo load
  const size_t N = size_t(1) << log_n, S = N >> k;
  const int c0 = 2 * blockIdx.x, j = blockIdx.y;
  const bool two = c0 + 1 < AIR_W;
  const uint32_t nhi = 1u << (log_n - k - ll);
  const uint32_t xh = blockIdx.z * IS_WARPS + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (xh >= nhi) return;
  const uint32_t nlo = 1u << ll;
  const uint32_t* col0 = wit + size_t(c0) * N + size_t(j) * S + (size_t(xh) << ll);
  const uint32_t* col1 = two ? col0 + N : col0;
  const bool last = j == gridDim.y - 1 && xh == nhi - 1;  // holds the wrapped row N - 1
  EfMacF u0, d0, u1, d1;
  u0.init();
  d0.init();
  u1.init();
  d1.init();
  uint32_t xl = lane;
  for (; xl + 96 < nlo; xl += 128) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const uint32_t x = xl + 32 * q;
      const ef e = eq_lo[x];
      const bool wrap = last && x == nlo - 1;
      const uint32_t xu = wrap ? x - 1 : x, xd = wrap ? x : x + 1;
      u0.mac(e, col0[xu]);
      d0.mac(e, col0[xd]);
      u1.mac(e, col1[xu]);
      d1.mac(e, col1[xd]);
    }
    u0.flush();
    d0.flush();
    u1.flush();
    d1.flush();
  }
  for (; xl < nlo; xl += 32) {
    const ef e = eq_lo[xl];
    const bool wrap = last && xl == nlo - 1;
    const uint32_t xu = wrap ? xl - 1 : xl, xd = wrap ? xl : xl + 1;
    u0.mac(e, col0[xu]);
    d0.mac(e, col0[xd]);
    u1.mac(e, col1[xu]);
    d1.mac(e, col1[xd]);
    u0.flush();
    d0.flush();
    u1.flush();
    d1.flush();
  }
  const ef su0 = warp_reduce_ef(u0.value()), sd0 = warp_reduce_ef(d0.value());
  const ef su1 = warp_reduce_ef(u1.value()), sd1 = warp_reduce_ef(d1.value());
  if (lane == 0) {
    const ef h = eq_hi[xh];
    size_t o = (size_t(c0) * gridDim.y + j) * nhi + xh;
    pu[o] = ef_mul(su0, h);
    pd[o] = ef_mul(sd0, h);
    if (two) {
      o = (size_t(c0 + 1) * gridDim.y + j) * nhi + xh;
      pu[o] = ef_mul(su1, h);
      pd[o] = ef_mul(sd1, h);
    }
  }
}

// ---- inner sums on the tensor cores
// A sum of products of 31-bit values is exact in integer matrix products over byte limbs:
// with x = sum_a 2^(8a) x_a and e = sum_b 2^(8b) e_b (bytes), sum_k x e = sum_(a,b) 2^(8(a+b))
// sum_k x_a e_b, and each inner sum of 4096 byte products stays below 2^28. The witness
// segments of 2^ll rows are the rows of A (u32 values, split into 4 byte matrices in
// registers), the eq_lo weights the columns of B: 16 columns, the 8 coefficients of eq_lo[x]
// (up sums) and of eq_lo[x - 1] (down sums, shifted by one row), as 4 byte matrices
// prepared once (k_eq_limbs). Each m16n8k32 u8 product adds 16 x 8 x 32 byte products into
// s32 accumulators; warp b of a block holds the 4 x 2 tiles of B limb b for a 16-row tile.
// The limb products are recombined by diagonal (a + b = d, below 2^30), weighted by
// 2^(8d) mod p (7 wide products, below 4 p^2) and reduced once: the Montgomery values give
// the Montgomery product. The row boundary terms (the down sum's element past the segment,
// the wrapped last row) are added on the CUDA cores.
// limbs[(b * 16 + n) * nlo + x] = byte b of column n of B at row x: n < 8 coefficient n of
// eq_lo[x], n >= 8 coefficient n - 8 of eq_lo[x - 1] (zero at x = 0).
__global__ void k_eq_limbs(const ef* __restrict__ eq_lo, int nlo, uint8_t* __restrict__ limbs) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= 16 * nlo) return;
  const int n = idx / nlo, x = idx - n * nlo;
  uint32_t v = 0;
  if (n < 8) v = eq_lo[x].c[n];
  else if (x > 0) v = eq_lo[x - 1].c[n - 8];
#pragma unroll
  for (int b = 0; b < 4; b++) limbs[(size_t(b) * 16 + n) * nlo + x] = uint8_t(v >> (8 * b));
}
constexpr int ISM_WARPS = 4;  // one per B limb
constexpr int ISM_STAGES = 4;  // chunks of 32 values in flight per tile
constexpr int ISM_ROW = 48;    // words per staged row (32 + 16: conflict-free 16-byte fragment reads)
constexpr int CS_WARPS = 4;   // warps of the kernels whose warps own whole tiles

// Sum over the limb pairs of column value (row, col), from the per-pair accumulators
// cs[a][b][row][col]: diagonals a + b = d (below 4 * 2^12 * 255^2 < 2^31) weighted by
// 2^(8d) mod p, then one Montgomery reduction (the sum stays below 4 p^2).
template <int C>
__device__ __forceinline__ uint32_t limb_recombine(const int (&cs)[4][4][16][C], int row, int col) {
  constexpr uint32_t W8[7] = {uint32_t(kb::detail::cpow(2, 0)),  uint32_t(kb::detail::cpow(2, 8)),
                              uint32_t(kb::detail::cpow(2, 16)), uint32_t(kb::detail::cpow(2, 24)),
                              uint32_t(kb::detail::cpow(2, 32)), uint32_t(kb::detail::cpow(2, 40)),
                              uint32_t(kb::detail::cpow(2, 48))};  // 2^(8d) mod p
  uint64_t v = 0;
#pragma unroll
  for (int d = 0; d < 7; d++) {
    uint32_t dd = 0;
#pragma unroll
    for (int a = 0; a < 4; a++)
      if (d - a >= 0 && d - a < 4) dd += uint32_t(cs[a][d - a][row][col]);
    v += kb::wmul(dd, W8[d]);
  }
  return kb::redc(v);
}
template <int NT, int C>
__device__ __forceinline__ void limb_store(int (&cs)[4][4][16][C], const int (&acc)[4][NT][4], int b, int g, int t) {
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int nt = 0; nt < NT; nt++) {
      cs[a][b][g][nt * 8 + 2 * t] = acc[a][nt][0];
      cs[a][b][g][nt * 8 + 2 * t + 1] = acc[a][nt][1];
      cs[a][b][g + 8][nt * 8 + 2 * t] = acc[a][nt][2];
      cs[a][b][g + 8][nt * 8 + 2 * t + 1] = acc[a][nt][3];
    }
}

__global__ void __launch_bounds__(ISM_WARPS * 32) k_inner_sums_mma(const uint32_t* __restrict__ wit, int log_n, int k,
                                                                  int ll, const ef* __restrict__ eq_hi,
                                                                  const ef* __restrict__ eq_lo,
                                                                  const uint8_t* __restrict__ limbs,
                                                                  ef* __restrict__ pu, ef* __restrict__ pd) {
  __shared__ int cs[4][4][16][17];  // [a][b][row][col], padded
  __shared__ ef up_s[16], dn_s[16];
  __shared__ __align__(16) uint32_t ism_a[ISM_STAGES][16][ISM_ROW];
  const size_t N = size_t(1) << log_n, S = N >> k;
  const uint32_t nsk = 1u << k, nhi = 1u << (log_n - k - ll), nlo = 1u << ll;
  const uint32_t M = uint32_t(AIR_W) * nsk * nhi;
  const uint32_t m0 = blockIdx.x * 16;
  const int lane = threadIdx.x & 31, b = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  auto row_base = [&](uint32_t m) -> size_t {
    const uint32_t xh = m % nhi, cj = m / nhi, j = cj % nsk, c = cj / nsk;
    return size_t(c) * N + size_t(j) * S + (size_t(xh) << ll);
  };
  // The tile's 16 segments stream through shared memory in chunks of 32 values (one 16-byte
  // cp.async per thread and chunk, ISM_STAGES chunks in flight), so the four warps (one per
  // limb of B) read each value from HBM once; rows past M are zero-filled.
  {
    const int crow = threadIdx.x >> 3, cpiece = threadIdx.x & 7;  // 16 rows x 8 pieces
    const uint32_t mr = m0 + crow;
    const bool cval = mr < M;
    const uint32_t* csrc = wit + (cval ? row_base(mr) : 0) + 4 * cpiece;
    const unsigned cdst0 = (unsigned)__cvta_generic_to_shared(&ism_a[0][crow][4 * cpiece]);
    const unsigned cstage = sizeof(ism_a[0]);
    const uint32_t nch = nlo >> 5;
    auto issue = [&](uint32_t c) {
      if (c < nch) {
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(cdst0 + (c % ISM_STAGES) * cstage),
                     "l"(csrc + 32 * c), "r"(cval ? 16 : 0));
      }
      asm volatile("cp.async.commit_group;\n" ::);
    };
    for (int c = 0; c < ISM_STAGES - 1; c++) issue(c);
    int acc[4][2][4];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int nt = 0; nt < 2; nt++)
#pragma unroll
        for (int q = 0; q < 4; q++) acc[a][nt][q] = 0;
    const uint32_t* lb = reinterpret_cast<const uint32_t*>(limbs + size_t(b) * 16 * nlo);
    const uint32_t lstride = nlo >> 2;
#pragma unroll 1
    for (uint32_t c = 0; c < nch; c++) {
      asm volatile("cp.async.wait_group %0;\n" ::"n"(ISM_STAGES - 2));
      __syncthreads();  // chunk c landed for every thread; the slot of chunk c - 1 is free
      issue(c + ISM_STAGES - 1);
      const uint32_t(&X)[16][ISM_ROW] = ism_a[c % ISM_STAGES];
      const uint4 q0 = *reinterpret_cast<const uint4*>(&X[g][4 * t]);
      const uint4 q1 = *reinterpret_cast<const uint4*>(&X[g + 8][4 * t]);
      const uint4 q2 = *reinterpret_cast<const uint4*>(&X[g][16 + 4 * t]);
      const uint4 q3 = *reinterpret_cast<const uint4*>(&X[g + 8][16 + 4 * t]);
      uint32_t l0[4], l1[4], l2[4], l3[4];
      byte_transpose4(q0, l0);
      byte_transpose4(q1, l1);
      byte_transpose4(q2, l2);
      byte_transpose4(q3, l3);
      uint32_t bf[2][2];
#pragma unroll
      for (int nt = 0; nt < 2; nt++) {
        const uint32_t* col = lb + size_t(nt * 8 + g) * lstride + (c << 3) + t;
        bf[nt][0] = __ldg(col);
        bf[nt][1] = __ldg(col + 4);
      }
#pragma unroll
      for (int a = 0; a < 4; a++) {
        const uint32_t af[4] = {l0[a], l1[a], l2[a], l3[a]};
#pragma unroll
        for (int nt = 0; nt < 2; nt++) mma_u8_16832(acc[a][nt], af, bf[nt][0], bf[nt][1]);
      }
    }
    asm volatile("cp.async.wait_group 0;\n" ::);
    limb_store<2>(cs, acc, b, g, t);
  }
  __syncthreads();
  // recombination: 256 (row, column) values, two per thread
  for (int e = threadIdx.x; e < 256; e += ISM_WARPS * 32) {
    const int row = e >> 4, col = e & 15;
    const uint32_t r = limb_recombine(cs, row, col);
    if (col < 8) up_s[row].c[col] = r;
    else dn_s[row].c[col - 8] = r;
  }
  __syncthreads();
  if (threadIdx.x < 16) {
    const uint32_t m = m0 + threadIdx.x;
    if (m < M) {
      const uint32_t xh = m % nhi, cj = m / nhi, j = cj % nsk, c = cj / nsk;
      const size_t base = size_t(c) * N + size_t(j) * S + (size_t(xh) << ll);
      const uint32_t* col = wit + size_t(c) * N;
      const bool last = j == nsk - 1 && xh == nhi - 1;  // the segment holding row N - 1
      const ef el = eq_lo[nlo - 1];
      ef up = up_s[threadIdx.x], dn = dn_s[threadIdx.x];
      if (last) {
        // up row of N - 1 is N - 2; down row of N - 1 is N - 1
        up = ef_add(up, ef_mul_f(el, kb::sub(col[N - 2], col[N - 1])));
        dn = ef_add(dn, ef_mul_f(el, col[N - 1]));
      } else {
        dn = ef_add(dn, ef_mul_f(el, wit[base + nlo]));
      }
      const ef h = eq_hi[xh];
      pu[m] = ef_mul(up, h);
      pd[m] = ef_mul(dn, h);
    }
  }
}

// The same inner sums with the tile staged by the bulk-copy (TMA) engine: one thread issues,
// per chunk, one cp.async.bulk of 128 bytes for each of the 16 segments, completing on the
// chunk's mbarrier (expected bytes set by the same thread); all threads wait on the mbarrier's
// phase before reading the chunk. ISB_STAGES chunks are in flight. Every wait is bounded: a
// wait that runs out counts a pipeline timeout (the host checks the counter after the inner
// sums and fails the proof) and the kernel stops consuming. Rows past M copy segment m0's data
// (their results are never stored). The B fragments of the next chunk are loaded from L2
// while the current chunk is multiplied.
constexpr int ISB_STAGES = 6;
constexpr uint32_t PIPE_WAIT_LIMIT = 1u << 20;  // try_wait rounds (each a bounded hardware wait)

__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
  for (uint32_t i = 0; i < PIPE_WAIT_LIMIT; i++) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__global__ void __launch_bounds__(ISM_WARPS * 32) k_inner_sums_bulk(const uint32_t* __restrict__ wit, int log_n, int k,
                                                                   int ll, const ef* __restrict__ eq_hi,
                                                                   const ef* __restrict__ eq_lo,
                                                                   const uint8_t* __restrict__ limbs,
                                                                   ef* __restrict__ pu, ef* __restrict__ pd,
                                                                   unsigned* __restrict__ timeouts) {
  __shared__ int cs[4][4][16][17];  // [a][b][row][col], padded
  __shared__ ef up_s[16], dn_s[16];
  __shared__ __align__(128) uint32_t isb_a[ISB_STAGES][16][ISM_ROW];
  __shared__ __align__(8) uint64_t bars[ISB_STAGES];
  __shared__ int stop;
  const size_t N = size_t(1) << log_n, S = N >> k;
  const uint32_t nsk = 1u << k, nhi = 1u << (log_n - k - ll), nlo = 1u << ll;
  const uint32_t M = uint32_t(AIR_W) * nsk * nhi;
  const uint32_t m0 = blockIdx.x * 16;
  const int lane = threadIdx.x & 31, b = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  auto row_base = [&](uint32_t m) -> size_t {
    const uint32_t xh = m % nhi, cj = m / nhi, j = cj % nsk, c = cj / nsk;
    return size_t(c) * N + size_t(j) * S + (size_t(xh) << ll);
  };
  const uint32_t nch = nlo >> 5;
  const unsigned bar0 = (unsigned)__cvta_generic_to_shared(&bars[0]);
  const unsigned dst0 = (unsigned)__cvta_generic_to_shared(&isb_a[0][0][0]);
  if (threadIdx.x == 0) {
    stop = 0;
    for (int st = 0; st < ISB_STAGES; st++)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar0 + 8 * st));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  // issued by thread 0 only: chunk c into slot c % ISB_STAGES
  auto issue = [&](uint32_t c) {
    if (c >= nch) return;
    const uint32_t slot = c % ISB_STAGES;
    const unsigned bar = bar0 + 8 * slot;
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");  // earlier reads of the slot come first
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(16u * 128u) : "memory");
    for (int row = 0; row < 16; row++) {
      const uint32_t m = m0 + row < M ? m0 + row : m0;
      const uint32_t* src = wit + row_base(m) + 32 * size_t(c);
      const unsigned dst = dst0 + ((slot * 16 + row) * ISM_ROW) * 4;
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], 128, [%2];\n" ::"r"(dst),
          "l"(src), "r"(bar)
          : "memory");
    }
  };
  if (threadIdx.x == 0)
    for (int c = 0; c < ISB_STAGES - 1; c++) issue(c);
  int acc[4][2][4];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int nt = 0; nt < 2; nt++)
#pragma unroll
      for (int q = 0; q < 4; q++) acc[a][nt][q] = 0;
  const uint32_t* lb = reinterpret_cast<const uint32_t*>(limbs + size_t(b) * 16 * nlo);
  const uint32_t lstride = nlo >> 2;
  uint32_t bf[2][2], bfn[2][2];
  auto load_b = [&](uint32_t c, uint32_t (&f)[2][2]) {
#pragma unroll
    for (int nt = 0; nt < 2; nt++) {
      const uint32_t* col = lb + size_t(nt * 8 + g) * lstride + (c << 3) + t;
      f[nt][0] = __ldg(col);
      f[nt][1] = __ldg(col + 4);
    }
  };
  load_b(0, bf);
  uint32_t consumed = 0;
#pragma unroll 1
  for (uint32_t c = 0; c < nch; c++) {
    if (!mbar_wait_bounded(bar0 + 8 * (c % ISB_STAGES), (c / ISB_STAGES) & 1)) {
      atomicAdd(timeouts, 1u);
      stop = 1;
    }
    __syncthreads();  // chunk c landed; every thread is done with the slot of chunk c - 1
    if (stop) break;
    if (threadIdx.x == 0) issue(c + ISB_STAGES - 1);
    if (c + 1 < nch) load_b(c + 1, bfn);
    const uint32_t(&X)[16][ISM_ROW] = isb_a[c % ISB_STAGES];
    const uint4 q0 = *reinterpret_cast<const uint4*>(&X[g][4 * t]);
    const uint4 q1 = *reinterpret_cast<const uint4*>(&X[g + 8][4 * t]);
    const uint4 q2 = *reinterpret_cast<const uint4*>(&X[g][16 + 4 * t]);
    const uint4 q3 = *reinterpret_cast<const uint4*>(&X[g + 8][16 + 4 * t]);
    uint32_t l0[4], l1[4], l2[4], l3[4];
    byte_transpose4(q0, l0);
    byte_transpose4(q1, l1);
    byte_transpose4(q2, l2);
    byte_transpose4(q3, l3);
#pragma unroll
    for (int a = 0; a < 4; a++) {
      const uint32_t af[4] = {l0[a], l1[a], l2[a], l3[a]};
#pragma unroll
      for (int nt = 0; nt < 2; nt++) mma_u8_16832(acc[a][nt], af, bf[nt][0], bf[nt][1]);
    }
#pragma unroll
    for (int nt = 0; nt < 2; nt++) bf[nt][0] = bfn[nt][0], bf[nt][1] = bfn[nt][1];
    consumed = c + 1;
  }
  if (consumed < nch) {
    // a wait ran out: let the copies already issued land (bounded) before the block exits
    const uint32_t issued = min(nch, consumed + ISB_STAGES - 1);
    for (uint32_t c = consumed; c < issued; c++) mbar_wait_bounded(bar0 + 8 * (c % ISB_STAGES), (c / ISB_STAGES) & 1);
    return;
  }
  limb_store<2>(cs, acc, b, g, t);
  __syncthreads();
  for (int e = threadIdx.x; e < 256; e += ISM_WARPS * 32) {
    const int row = e >> 4, col = e & 15;
    const uint32_t r = limb_recombine(cs, row, col);
    if (col < 8) up_s[row].c[col] = r;
    else dn_s[row].c[col - 8] = r;
  }
  __syncthreads();
  if (threadIdx.x < 16) {
    const uint32_t m = m0 + threadIdx.x;
    if (m < M) {
      const uint32_t xh = m % nhi, cj = m / nhi, j = cj % nsk, c = cj / nsk;
      const size_t base = size_t(c) * N + size_t(j) * S + (size_t(xh) << ll);
      const uint32_t* col = wit + size_t(c) * N;
      const bool last = j == nsk - 1 && xh == nhi - 1;  // the segment holding row N - 1
      const ef el = eq_lo[nlo - 1];
      ef up = up_s[threadIdx.x], dn = dn_s[threadIdx.x];
      if (last) {
        up = ef_add(up, ef_mul_f(el, kb::sub(col[N - 2], col[N - 1])));
        dn = ef_add(dn, ef_mul_f(el, col[N - 1]));
      } else {
        dn = ef_add(dn, ef_mul_f(el, wit[base + nlo]));
      }
      const ef h = eq_hi[xh];
      pu[m] = ef_mul(up, h);
      pd[m] = ef_mul(dn, h);
    }
  }
}

// WHIR partial evaluation on the tensor cores: rows m = (u, v_hi) are the segments
// T[m 2^ll .. m 2^ll + 2^ll) of the packed table (zero past t_len), B the 8 coefficients of
// lo (limbs[(b * 8 + n) * nlo + x]). Each warp owns a 16-row tile (16 consecutive v_hi of one
// u) and all 4 x 4 limb pairs, so every segment value is loaded and split into limbs once;
// its rows' dot products times hi[v_hi], summed, are partial[(v_hi / 16) * 2^lu + u].
__global__ void __launch_bounds__(CS_WARPS * 32) k_mle_partial_mma(const uint32_t* __restrict__ T, size_t t_len,
                                                                  int lu, int lh, int ll,
                                                                  const ef* __restrict__ hi,
                                                                  const uint8_t* __restrict__ limbs,
                                                                  ef* __restrict__ partial) {
  __shared__ int cs_all[CS_WARPS][4][4][16][9];
  __shared__ ef rows_all[CS_WARPS][16];
  const uint32_t nhi = 1u << lh, nlo = 1u << ll;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  int(&cs)[4][4][16][9] = cs_all[warp];
  const uint32_t m0 = (blockIdx.x * CS_WARPS + warp) * 16;  // 16 rows of one u (16 divides nhi)
  if (m0 >= (1u << (lu + lh))) return;  // whole warp (no block barrier below)
  const size_t ba = size_t(m0 + g) << ll, bb = size_t(m0 + g + 8) << ll;
  const bool va = ba < t_len, vb = bb < t_len;  // t_len is a multiple of 2^ll
  const uint32_t* pa = T + (va ? ba : 0) + 4 * t;
  const uint32_t* pb = T + (vb ? bb : 0) + 4 * t;
  const uint32_t* lw = reinterpret_cast<const uint32_t*>(limbs);
  const uint32_t lstride = nlo >> 2;
  int acc[4][4][4];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++)
#pragma unroll
      for (int q = 0; q < 4; q++) acc[a][b][q] = 0;
  const uint4 zero4 = make_uint4(0, 0, 0, 0);
  // the next step's values are requested before this step's products (two steps in flight)
  uint4 n0 = va ? __ldg(reinterpret_cast<const uint4*>(pa)) : zero4;
  uint4 n1 = vb ? __ldg(reinterpret_cast<const uint4*>(pb)) : zero4;
  uint4 n2 = va ? __ldg(reinterpret_cast<const uint4*>(pa + 16)) : zero4;
  uint4 n3 = vb ? __ldg(reinterpret_cast<const uint4*>(pb + 16)) : zero4;
#pragma unroll 1
  for (uint32_t k0 = 0; k0 < nlo; k0 += 32) {
    const uint4 q0 = n0, q1 = n1, q2 = n2, q3 = n3;
    if (k0 + 32 < nlo) {
      n0 = va ? __ldg(reinterpret_cast<const uint4*>(pa + k0 + 32)) : zero4;
      n1 = vb ? __ldg(reinterpret_cast<const uint4*>(pb + k0 + 32)) : zero4;
      n2 = va ? __ldg(reinterpret_cast<const uint4*>(pa + k0 + 48)) : zero4;
      n3 = vb ? __ldg(reinterpret_cast<const uint4*>(pb + k0 + 48)) : zero4;
    }
    uint32_t l0[4], l1[4], l2[4], l3[4];
    byte_transpose4(q0, l0);
    byte_transpose4(q1, l1);
    byte_transpose4(q2, l2);
    byte_transpose4(q3, l3);
#pragma unroll
    for (int b = 0; b < 4; b++) {
      const uint32_t* col = lw + size_t(b * 8 + g) * lstride + (k0 >> 2) + t;
      const uint32_t b0 = __ldg(col), b1 = __ldg(col + 4);
#pragma unroll
      for (int a = 0; a < 4; a++) {
        const uint32_t af[4] = {l0[a], l1[a], l2[a], l3[a]};
        mma_u8_16832(acc[a][b], af, b0, b1);
      }
    }
  }
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) {
      cs[a][b][g][2 * t] = acc[a][b][0];
      cs[a][b][g][2 * t + 1] = acc[a][b][1];
      cs[a][b][g + 8][2 * t] = acc[a][b][2];
      cs[a][b][g + 8][2 * t + 1] = acc[a][b][3];
    }
  __syncwarp();
#pragma unroll
  for (int e = lane; e < 128; e += 32) rows_all[warp][e >> 3].c[e & 7] = limb_recombine(cs, e >> 3, e & 7);
  __syncwarp();
  const uint32_t u = m0 >> lh, vh0 = m0 & (nhi - 1);
  ef v = lane < 16 ? ef_mul(rows_all[warp][lane], hi[vh0 + lane]) : ef_zero();
  v = warp_reduce_ef(v);
  if (lane == 0) partial[size_t(vh0 >> 4) * (size_t(1) << lu) + u] = v;
}
// limbs[(b * 8 + n) * nlo + x] = byte b of coefficient n of lo[x].
__global__ void k_lo_limbs(const ef* __restrict__ lo, int nlo, uint8_t* __restrict__ limbs) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= 8 * nlo) return;
  const int n = idx / nlo, x = idx - n * nlo;
  const uint32_t v = lo[x].c[n];
#pragma unroll
  for (int b = 0; b < 4; b++) limbs[(size_t(b) * 8 + n) * nlo + x] = uint8_t(v >> (8 * b));
}

// Weighted column sums on the tensor cores: out[m] = sum_(k < K) w[k] A[m][k] for extension
// weights w and base-field A, by byte-limb matrix products (as the inner sums) with the rows
// m on the M side and the short K (<= 192) in chunks of 32. A[m][k] sits at
// src[k * kstride + m] (consecutive rows are consecutive words, so every load of a warp reads
// whole sectors). Used for the batched column (the witness columns, kstride N). The same form
// was measured slower than the CUDA-core kernels for the WHIR table g (K = 128) and for the
// round-0 fold (K = 2^k <= 16, padded to 32): their loads dominate, and the CUDA-core
// kernels read two rows per load.
// Each warp owns a 16-row tile and all 4 x 4 limb pairs; limbs[(b * 8 + n) * Kp + k] holds
// byte b of coefficient n of w[k] (zero for k >= K).
__global__ void __launch_bounds__(CS_WARPS * 32) k_colsum_mma(const uint32_t* __restrict__ src, size_t M, int K,
                                                             int Kp, size_t kstride,
                                                             const uint8_t* __restrict__ limbs, ef* __restrict__ out) {
  __shared__ int cs_all[CS_WARPS][4][4][16][9];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  int(&cs)[4][4][16][9] = cs_all[warp];
  const size_t m0 = (size_t(blockIdx.x) * CS_WARPS + warp) * 16;
  if (m0 >= M) return;  // whole warp (no block barrier below)
  const size_t ra = m0 + g, rb = m0 + g + 8;
  const bool va = ra < M, vb = rb < M;
  auto load = [&](size_t m, bool vm, int kk) -> uint32_t {
    return (vm && kk < K) ? __ldg(src + size_t(kk) * kstride + m) : 0u;
  };
  int acc[4][4][4];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++)
#pragma unroll
      for (int q = 0; q < 4; q++) acc[a][b][q] = 0;
  const uint32_t* lw = reinterpret_cast<const uint32_t*>(limbs);
  const int lstride = Kp >> 2;
  // the next step's values are requested before this step's products (two steps in flight)
  auto load_step = [&](int k0, uint4 (&q)[4]) {
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int kb0 = k0 + 16 * h + 4 * t;
      q[2 * h] = make_uint4(load(ra, va, kb0), load(ra, va, kb0 + 1), load(ra, va, kb0 + 2), load(ra, va, kb0 + 3));
      q[2 * h + 1] =
          make_uint4(load(rb, vb, kb0), load(rb, vb, kb0 + 1), load(rb, vb, kb0 + 2), load(rb, vb, kb0 + 3));
    }
  };
  uint4 nq[4];
  load_step(0, nq);
#pragma unroll 1
  for (int k0 = 0; k0 < Kp; k0 += 32) {
    uint4 q[4];
#pragma unroll
    for (int i = 0; i < 4; i++) q[i] = nq[i];
    if (k0 + 32 < Kp) load_step(k0 + 32, nq);
    uint32_t l[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++) byte_transpose4(q[i], l[i]);
#pragma unroll
    for (int b = 0; b < 4; b++) {
      const uint32_t* col = lw + size_t(b * 8 + g) * lstride + (k0 >> 2) + t;
      const uint32_t b0 = __ldg(col), b1 = __ldg(col + 4);
#pragma unroll
      for (int a = 0; a < 4; a++) {
        const uint32_t af[4] = {l[0][a], l[1][a], l[2][a], l[3][a]};
        mma_u8_16832(acc[a][b], af, b0, b1);
      }
    }
  }
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) {
      cs[a][b][g][2 * t] = acc[a][b][0];
      cs[a][b][g][2 * t + 1] = acc[a][b][1];
      cs[a][b][g + 8][2 * t] = acc[a][b][2];
      cs[a][b][g + 8][2 * t + 1] = acc[a][b][3];
    }
  __syncwarp();
  uint32_t* o = reinterpret_cast<uint32_t*>(out);
#pragma unroll
  for (int e = lane; e < 128; e += 32) {
    const int row = e >> 3, col = e & 7;
    if (m0 + row < M) o[(m0 + row) * 8 + col] = limb_recombine(cs, row, col);
  }
}
// limbs[(b * 8 + n) * Kp + k] = byte b of coefficient n of w[k] (zero for k >= K).
__global__ void k_w_limbs(const ef* __restrict__ w, int K, int Kp, uint8_t* __restrict__ limbs) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= 8 * Kp) return;
  const int n = idx / Kp, x = idx - n * Kp;
  const uint32_t v = x < K ? w[x].c[n] : 0u;
#pragma unroll
  for (int b = 0; b < 4; b++) limbs[(size_t(b) * 8 + n) * Kp + x] = uint8_t(v >> (8 * b));
}

// out[c] = sum_j sel[j] * sum_h partial[(c * nsk + j) * nh + h]; one warp per column.
__global__ void k_combine_sel(const ef* __restrict__ partial, const ef* __restrict__ sel, int nsk, int nh, int ncols,
                              ef* __restrict__ out) {
  const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (c >= ncols) return;
  ef acc = ef_zero();
  for (int idx = lane; idx < nsk * nh; idx += 32)
    acc = ef_add(acc, ef_mul(sel[idx / nh], partial[size_t(c) * nsk * nh + idx]));
  acc = warp_reduce_ef(acc);
  if (lane == 0) out[c] = acc;
}

// ------------------------------------------------------------------ inner phase
// out[row] = sum_c eqc[c] * wit[c][row]; two adjacent rows per thread (8-byte loads).
__global__ void k_batch_cols(const uint32_t* __restrict__ wit, int log_n, const ef* __restrict__ eqc_g,
                             ef* __restrict__ out) {
  __shared__ ef eqc[AIR_W + 3];
  for (int i = threadIdx.x; i < AIR_W + 3; i += blockDim.x) eqc[i] = i < AIR_W ? eqc_g[i] : ef_zero();
  __syncthreads();
  const size_t N = size_t(1) << log_n;
  const size_t row = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) * 2;
  if (row >= N) return;
  EfMacF m0, m1;
  m0.init();
  m1.init();
#pragma unroll 2
  for (int c = 0; c < AIR_W; c += 4) {
    uint2 v[4];
#pragma unroll
    for (int q = 0; q < 4; q++)
      v[q] = c + q < AIR_W ? __ldg(reinterpret_cast<const uint2*>(wit + size_t(c + q) * N + row)) : make_uint2(0, 0);
#pragma unroll
    for (int q = 0; q < 4; q++) {
      m0.mac(eqc[c + q], v[q].x);
      m1.mac(eqc[c + q], v[q].y);
    }
    m0.flush();
    m1.flush();
  }
  out[row] = m0.value();
  out[row + 1] = m1.value();
}

constexpr int SUB_THREADS = 256, SUB_PER_THREAD = 16;

// partial[(chunk * 2^k + j) * 2 + {0,1}] = sum_x eqt[x] * B[up/down(j S + x)] over the chunk's x
__global__ void k_sub_evals(const ef* __restrict__ B, int log_n, int k, const ef* __restrict__ eqt,
                            ef* __restrict__ partial) {
  __shared__ ef scratch[32];
  const size_t N = size_t(1) << log_n, S = N >> k;
  const int j = blockIdx.y;
  const size_t chunk = blockIdx.x;
  ef u = ef_zero(), d = ef_zero();
  for (int q = 0; q < SUB_PER_THREAD; q++) {
    size_t x = (chunk * SUB_PER_THREAD + q) * SUB_THREADS + threadIdx.x;
    if (x < S) {
      size_t i = size_t(j) * S + x;
      const ef e = eqt[x];
      u = ef_add(u, ef_mul(e, B[up_row(i, N)]));
      d = ef_add(d, ef_mul(e, B[down_row(i, N)]));
    }
  }
  u = block_reduce_ef(u, scratch);
  d = block_reduce_ef(d, scratch);
  if (threadIdx.x == 0) {
    size_t o = (chunk * gridDim.y + j) * 2;
    partial[o] = u;
    partial[o + 1] = d;
  }
}

// A[y] = up-shift matrix row + alpha2 * down-shift matrix row, folded at the point whose
// eq table is e (crates/air/src/uni_skip_utils.rs:5-34).
__global__ void k_inner_mle(const ef* __restrict__ e, int log_n, const ef* __restrict__ alpha2, ef* __restrict__ out) {
  const size_t N = size_t(1) << log_n;
  const size_t y = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (y >= N) return;
  const ef last = e[N - 1];
  ef mu = e[y];
  if (y == N - 2) mu = ef_add(mu, last);
  if (y == N - 1) mu = ef_zero();
  ef md = y >= 1 ? e[y - 1] : ef_zero();
  if (y == N - 1) md = ef_add(md, last);
  out[y] = ef_add(mu, ef_mul(*alpha2, md));
}

constexpr int PROD_THREADS = 256;
// points per thread: 8 for large tables, fewer for small ones so that latency, not a
// serial loop, bounds the small rounds
int prod_per_thread(size_t half) { return half >= (size_t(1) << 19) ? 8 : half >= (size_t(1) << 16) ? 2 : 1; }

__global__ void k_prod_eval(const ef* __restrict__ a, const ef* __restrict__ b, size_t half, int per,
                            ef* __restrict__ partial) {
  __shared__ ef scratch[32];
  ef s0 = ef_zero(), s2 = ef_zero();
  for (int q = 0; q < per; q++) {
    size_t x = (size_t(blockIdx.x) * per + q) * PROD_THREADS + threadIdx.x;
    if (x < half) {
      ef al = a[x], ah = a[x + half], bl = b[x], bh = b[x + half];
      s0 = ef_add(s0, ef_mul(al, bl));
      ef a2 = ef_sub(ef_add(ah, ah), al), b2 = ef_sub(ef_add(bh, bh), bl);
      s2 = ef_add(s2, ef_mul(a2, b2));
    }
  }
  s0 = block_reduce_ef(s0, scratch);
  s2 = block_reduce_ef(s2, scratch);
  if (threadIdx.x == 0) {
    partial[size_t(blockIdx.x) * 2] = s0;
    partial[size_t(blockIdx.x) * 2 + 1] = s2;
  }
}


// ------------------------------------------------------------------ fold fused with the next round
// The fold of the previous round at its challenge (lo + r (hi - lo), the challenge read from
// device memory where the round-finishing kernel left it) fused with this round's sums, so
// every table is read once per round: thread x of this round (x < h, the tables' new length
// being 2h) reads old entries x, x + h, x + 2h, x + 3h, writes the two folded entries x and
// x + h, and accumulates the round polynomial's values. Grid-stride; one partial per block.
constexpr int FE_THREADS = FIN_MAX_THREADS;
__device__ __forceinline__ ef fe_lerp(const ef* t, size_t i, size_t L, const ef& r) {
  const ef lo = t[i];
  return ef_add(lo, ef_mul(r, ef_sub(t[i + L], lo)));
}
// Product sumcheck (NS = 2: values at 0 and 2; the inner sumcheck) and WHIR folding sumcheck
// (NS = 3: values at 0, 1, 2) on the pair of tables (a, b).
template <int NS>
__global__ void __launch_bounds__(FE_THREADS) k_pair_fold_eval(const ef* __restrict__ a, const ef* __restrict__ b,
                                                               const ef* __restrict__ rptr, ef* __restrict__ na,
                                                               ef* __restrict__ nb, size_t h,
                                                               ef* __restrict__ partial, const FinArgs fin) {
  __shared__ ef scratch[32];
  const ef r = *rptr;
  const size_t L = 2 * h;
  ef s0 = ef_zero(), s1 = ef_zero(), s2 = ef_zero();
  for (size_t x = size_t(blockIdx.x) * blockDim.x + threadIdx.x; x < h; x += size_t(gridDim.x) * blockDim.x) {
    const ef al = fe_lerp(a, x, L, r), ah = fe_lerp(a, x + h, L, r);
    const ef bl = fe_lerp(b, x, L, r), bh = fe_lerp(b, x + h, L, r);
    na[x] = al;
    na[x + h] = ah;
    nb[x] = bl;
    nb[x + h] = bh;
    s0 = ef_add(s0, ef_mul(al, bl));
    if (NS == 3) s1 = ef_add(s1, ef_mul(ah, bh));
    s2 = ef_add(s2, ef_mul(ef_sub(ef_add(ah, ah), al), ef_sub(ef_add(bh, bh), bl)));
  }
  s0 = block_reduce_ef(s0, scratch);
  if (threadIdx.x == 0) partial[size_t(blockIdx.x) * NS] = s0;
  __syncthreads();
  if (NS == 3) {
    s1 = block_reduce_ef(s1, scratch);
    if (threadIdx.x == 0) partial[size_t(blockIdx.x) * NS + 1] = s1;
    __syncthreads();
  }
  s2 = block_reduce_ef(s2, scratch);
  if (threadIdx.x == 0) partial[size_t(blockIdx.x) * NS + NS - 1] = s2;
  if (fin.st) fin_last_block(NS == 2 ? FIN_PROD : FIN_WHIR, fin, partial, NS);
}
// The a*b - c zerocheck's rounds >= 2: three columns (column q of old length 4h at q 4h, of new
// length 2h at q 2h) and the eq table (old length 2h, the leading variable summed out into the
// new table of length h); values at z = 0 and 2 of (A B - C) eq.
__global__ void __launch_bounds__(FE_THREADS) k_abc_fold_eval(const ef* __restrict__ cols, const ef* __restrict__ rptr,
                                                              const ef* __restrict__ eq_prev, ef* __restrict__ nc,
                                                              ef* __restrict__ eq_new, size_t h,
                                                              ef* __restrict__ partial, const FinArgs fin) {
  __shared__ ef scratch[32];
  const ef r = *rptr;
  const size_t L = 2 * h;
  ef s0 = ef_zero(), s2 = ef_zero();
  for (size_t x = size_t(blockIdx.x) * blockDim.x + threadIdx.x; x < h; x += size_t(gridDim.x) * blockDim.x) {
    ef lo[3], t[3];
#pragma unroll
    for (int q = 0; q < 3; q++) {
      const ef* col = cols + size_t(q) * 2 * L;
      lo[q] = fe_lerp(col, x, L, r);
      const ef hi = fe_lerp(col, x + h, L, r);
      nc[size_t(q) * L + x] = lo[q];
      nc[size_t(q) * L + x + h] = hi;
      t[q] = ef_sub(ef_add(hi, hi), lo[q]);
    }
    const ef e = ef_add(eq_prev[x], eq_prev[x + h]);
    eq_new[x] = e;
    s0 = ef_add(s0, ef_mul(ef_sub(ef_mul(lo[0], lo[1]), lo[2]), e));
    s2 = ef_add(s2, ef_mul(ef_sub(ef_mul(t[0], t[1]), t[2]), e));
  }
  s0 = block_reduce_ef(s0, scratch);
  if (threadIdx.x == 0) partial[size_t(blockIdx.x) * 2] = s0;
  __syncthreads();
  s2 = block_reduce_ef(s2, scratch);
  if (threadIdx.x == 0) partial[size_t(blockIdx.x) * 2 + 1] = s2;
  if (fin.st) fin_last_block(FIN_EQSC3, fin, partial, 2);
}

// ------------------------------------------------------------------ a*b - c

// Round 0 of the a*b - c zerocheck: for every point z of the skipped variables' extension and
// every x, v_z(x) = A_z(x) B_z(x) - C_z(x) with A_z(x) = sum_j L_j(z) a[j S + x] (and B, C the
// same), weighted by eq(x). Grid-stride over x, one thread per x at a time, all nz points per
// thread: each value is read once (a, b, c and eq(x) coalesced), the points' products stay in
// registers, and each thread keeps nz extension accumulators that one block reduction sums at
// the end (one partial per block and point).
constexpr int ABC_X = 32;
constexpr int ABC0_THREADS = 256;
constexpr int ABC0_MAX_Z = 7;  // 2 (2^k - 1) - 2^k + 1 points for k <= 3
__global__ void __launch_bounds__(ABC0_THREADS, 2) k_abc0_eval(const uint32_t* __restrict__ a,
                                                           const uint32_t* __restrict__ b,
                                                           const uint32_t* __restrict__ c, int log_n, int k, int nz,
                                                           const uint32_t* __restrict__ lw,
                                                           const ef* __restrict__ eq, ef* __restrict__ partial) {
  __shared__ uint32_t w_s[ABC0_MAX_Z * 8];
  __shared__ ef scratch[32];
  const int nsk = 1 << k;
  for (int i = threadIdx.x; i < nz * nsk; i += blockDim.x) w_s[i] = lw[i];
  __syncthreads();
  const size_t N = size_t(1) << log_n, S = N >> k;
  ef acc[ABC0_MAX_Z];
#pragma unroll
  for (int z = 0; z < ABC0_MAX_Z; z++) acc[z] = ef_zero();
  for (size_t x = size_t(blockIdx.x) * blockDim.x + threadIdx.x; x < S; x += size_t(gridDim.x) * blockDim.x) {
    uint32_t va[8], vb[8], vc[8];
#pragma unroll
    for (int j = 0; j < 8; j++)
      if (j < nsk) va[j] = a[size_t(j) * S + x], vb[j] = b[size_t(j) * S + x], vc[j] = c[size_t(j) * S + x];
    const ef e = eq[x];
#pragma unroll
    for (int z = 0; z < ABC0_MAX_Z; z++) {
      if (z >= nz) break;
      const uint32_t* wz = w_s + z * nsk;
      uint64_t sa = 0, sb = 0, sc = 0, ta = 0, tb = 0, tc = 0;
#pragma unroll
      for (int j = 0; j < 8; j++) {
        if (j >= nsk) break;
        if (j < 4) sa += wmul(wz[j], va[j]), sb += wmul(wz[j], vb[j]), sc += wmul(wz[j], vc[j]);
        else ta += wmul(wz[j], va[j]), tb += wmul(wz[j], vb[j]), tc += wmul(wz[j], vc[j]);
      }
      const uint32_t A = add(redc(sa), redc(ta)), B = add(redc(sb), redc(tb)), C = add(redc(sc), redc(tc));
      acc[z] = ef_add(acc[z], ef_mul_f(e, sub(mul(A, B), C)));
    }
  }
#pragma unroll
  for (int z = 0; z < ABC0_MAX_Z; z++) {
    if (z >= nz) break;
    const ef t = block_reduce_ef(acc[z], scratch);
    if (threadIdx.x == 0) partial[size_t(blockIdx.x) * nz + z] = t;
    __syncthreads();  // scratch is reused by the next point
  }
}

// One thread per (x, point) with the block spanning the points: the form for 4 skipped
// variables (15 points, too many to keep per thread).
__global__ void k_abc0_eval_points(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b,
                            const uint32_t* __restrict__ c, int log_n, int k, int nz, const uint32_t* __restrict__ lw,
                            const ef* __restrict__ eq, ef* __restrict__ partial) {
  __shared__ uint32_t w_s[32 * 16];
  const int nsk = 1 << k;
  const int tid = threadIdx.y * ABC_X + threadIdx.x;
  for (int i = tid; i < nz * nsk; i += ABC_X * blockDim.y) w_s[i] = lw[i];
  __syncthreads();
  const size_t N = size_t(1) << log_n, S = N >> k;
  const size_t x = size_t(blockIdx.x) * ABC_X + threadIdx.x;
  const int zi = threadIdx.y;
  ef res = ef_zero();
  if (x < S && zi < nz) {
    const uint32_t* wz = w_s + zi * nsk;
    uint64_t sa[4] = {0, 0, 0, 0}, sb[4] = {0, 0, 0, 0}, sc[4] = {0, 0, 0, 0};
    for (int j = 0; j < nsk; j++) {
      size_t i = size_t(j) * S + x;
      sa[j & 3] += wmul(wz[j], a[i]);
      sb[j & 3] += wmul(wz[j], b[i]);
      sc[j & 3] += wmul(wz[j], c[i]);
    }
    auto fin = [](uint64_t* s) { return add(add(redc(s[0]), redc(s[1])), add(redc(s[2]), redc(s[3]))); };
    uint32_t v = sub(mul(fin(sa), fin(sb)), fin(sc));
    res = ef_mul_f(eq[x], v);
  }
  res = warp_reduce_ef(res);
  if (threadIdx.x == 0 && zi < nz) partial[size_t(blockIdx.x) * nz + zi] = res;
}

__global__ void k_abc0_fold(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b,
                            const uint32_t* __restrict__ c, int log_n, int k, const ef* __restrict__ sel_g,
                            ef* __restrict__ out) {
  __shared__ ef sel[16];
  const int nsk = 1 << k;
  if (threadIdx.x < nsk) sel[threadIdx.x] = sel_g[threadIdx.x];
  __syncthreads();
  const size_t N = size_t(1) << log_n, S = N >> k;
  const size_t x = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (x >= S) return;
  const uint32_t* src = blockIdx.y == 0 ? a : blockIdx.y == 1 ? b : c;
  EfMacF m;
  m.init();
  for (int j = 0; j < nsk; j++) {
    m.mac(sel[j], src[size_t(j) * S + x]);
    if ((j & 3) == 3 || j == nsk - 1) m.flush();
  }
  out[size_t(blockIdx.y) * S + x] = m.value();
}

__global__ void k_abc_eval_ef(const ef* __restrict__ cols, int m, const ef* __restrict__ eq, ef* __restrict__ partial) {
  const size_t len = size_t(1) << m, half = len >> 1;
  const size_t x = size_t(blockIdx.x) * 32 + threadIdx.x;
  const int zi = threadIdx.y;  // z = 0 or 2
  ef res = ef_zero();
  if (x < half) {
    ef v[3];
    for (int q = 0; q < 3; q++) {
      ef lo = cols[q * len + x], hi = cols[q * len + half + x];
      v[q] = zi == 0 ? lo : ef_sub(ef_add(hi, hi), lo);
    }
    res = ef_mul(ef_sub(ef_mul(v[0], v[1]), v[2]), eq[x]);
  }
  res = warp_reduce_ef(res);
  if (threadIdx.x == 0) partial[size_t(blockIdx.x) * 2 + zi] = res;
}
}  // namespace

// ------------------------------------------------------------------ launchers
void launch_eq_table(const ef* point, int nvars, ef* out, cudaStream_t s) {
  if (nvars > EQ_MAX_VARS) throw std::invalid_argument("eq table: too many variables");
  const int nbits = nvars < EQ_BLK_BITS ? nvars : EQ_BLK_BITS;
  k_eq_table<<<(unsigned)(size_t(1) << (nvars - nbits)), EQ_THREADS, 0, s>>>(point, nvars, out);
  WL_LAUNCH_CHECK();
}
void launch_eq_table_f(const uint32_t* pts, int npts, int nvars, uint32_t* out, cudaStream_t s) {
  size_t n = size_t(npts) << nvars;
  if (!n) return;
  k_eq_table_f<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(pts, npts, nvars, out);
  WL_LAUNCH_CHECK();
}
void launch_reduce_partials(const ef* partial, int nblk, int k, ef* out, cudaStream_t s) {
  k_reduce_partials<<<k, 256, 0, s>>>(partial, nblk, k, out);
  WL_LAUNCH_CHECK();
}

int zc0_blocks(int log_n, int k) {
  size_t S = size_t(1) << (log_n - k);
  return (int)((S + ZC0_X - 1) / ZC0_X);
}
int zc0_row_blocks(int log_n) { return (int)(((size_t(1) << log_n) + ZC0R_THREADS - 1) / ZC0R_THREADS); }
void launch_zc0_rows(const uint32_t* wit, int log_n, int k, int nz, const uint32_t* lw, const ef* eq,
                     const ef* alphas, const AirConsts& K, uint32_t* q, ef* partial, ef* arow, cudaStream_t s) {
  k_zc0_rows<<<zc0_row_blocks(log_n), ZC0R_THREADS, 0, s>>>(wit, log_n, k, nz, lw, eq, alphas, K, q, partial,
                                                            arow);
  WL_LAUNCH_CHECK();
}
void launch_zc0_fold_ef(const ef* a, int log_n, int k, const ef* sel, ef* out, cudaStream_t s) {
  const size_t S = size_t(1) << (log_n - k);
  k_zc0_fold_ef<<<(unsigned)((S + 255) / 256), 256, 0, s>>>(a, log_n, k, sel, out);
  WL_LAUNCH_CHECK();
}
void launch_zc0_eval(const uint32_t* wit, const uint32_t* q, int log_n, int k, int nz, const uint32_t* lw,
                     const ef* eq, const ef* alphas, const ef* betas, const AirConsts& K, ef* partial,
                     cudaStream_t s) {
  if (nz > 32) throw std::invalid_argument("zc0_eval: at most 32 points");
  k_zc0_eval_mma<<<zc0_blocks(log_n, k), ZC0M_WARPS * 32, 0, s>>>(wit, q, log_n, k, nz, lw, eq, alphas, betas, K,
                                                                  partial);
  WL_LAUNCH_CHECK();
}
void launch_zc0_fold(const uint32_t* wit, int log_n, int k, const ef* sel, ef* out, cudaStream_t s) {
  size_t S = size_t(1) << (log_n - k);
  if (S < 2) throw std::invalid_argument("zc0_fold: at least 2 points per skip block");
  k_zc0_fold_mma<<<zc0_blocks(log_n, k), ZC0M_WARPS * 32, 0, s>>>(wit, log_n, k, sel, out);
  WL_LAUNCH_CHECK();
}
// Rounds with at least ZC_DENSE_MIN_HALF points per z use the dense kernels.
constexpr size_t ZC_DENSE_MIN_HALF = size_t(1) << 10;
bool zc_eval_is_dense(int m) { return (size_t(1) << (m - 1)) >= ZC_DENSE_MIN_HALF; }
int zc_ef_blocks(int m) {  // partial sums per z
  const size_t half = size_t(1) << (m - 1);
  if (half < ZC_DENSE_MIN_HALF) return (int)half;
  return (int)((half + ZCD_FULL_PTS - 1) / ZCD_FULL_PTS + (half + ZCD_PARTIAL_PTS - 1) / ZCD_PARTIAL_PTS);
}
void launch_zc_eval_ef(const ef* cols, int m, const ef* eq, const ef* alphas, const ef* betas, const AirConsts& K,
                       ef* partial, cudaStream_t s) {
  const size_t half = size_t(1) << (m - 1);
  if (half >= ZC_DENSE_MIN_HALF) {
    const unsigned bf = (unsigned)((half + ZCD_FULL_PTS - 1) / ZCD_FULL_PTS);
    const unsigned bp = (unsigned)((half + ZCD_PARTIAL_PTS - 1) / ZCD_PARTIAL_PTS);
    k_zc_full_dense<<<dim3(bf, 3), ZCD_WARPS * 32, 0, s>>>(cols, m, eq, alphas, betas, K, partial);
    WL_LAUNCH_CHECK();
    k_zc_partial_dense<<<dim3(bp, 3), ZCD_WARPS * 32, 0, s>>>(cols, m, eq, alphas, betas, K,
                                                              partial + size_t(bf) * 3);
  } else {
    k_zc_ef<<<(unsigned)(half * 3), ZCE_THREADS, 0, s>>>(cols, m, eq, alphas, betas, K, partial);
  }
  WL_LAUNCH_CHECK();
}
void launch_fold_cols(const ef* in, ef* out, int ncols, size_t half, const ef* r, cudaStream_t s, const ef* eq_in,
                      ef* eq_out, size_t eq_half) {
  const size_t width = eq_in && eq_half > half ? eq_half : half;
  dim3 grid((unsigned)((width + 255) / 256), ncols + (eq_in ? 1 : 0));
  k_fold_cols<<<grid, 256, 0, s>>>(in, out, half, ncols, r, ef_zero(), eq_in, eq_out, eq_half);
  WL_LAUNCH_CHECK();
}
void launch_fold_cols_at(const ef* in, ef* out, int ncols, size_t half, const ef& r, cudaStream_t s, const ef* eq_in,
                         ef* eq_out, size_t eq_half) {
  // 128 values per block for the columns, 256 for the eq table
  const size_t bx = std::max((half + 127) / 128, eq_in ? (eq_half + 255) / 256 : size_t(0));
  dim3 grid((unsigned)std::max<size_t>(bx, 1), ncols + (eq_in ? 1 : 0));
  k_fold_cols_mma<<<grid, 256, 0, s>>>(in, out, half, ncols, r, nullptr, eq_in, eq_out, eq_half);
  WL_LAUNCH_CHECK();
}
void launch_fold_cols_dev(const ef* in, ef* out, int ncols, size_t half, const ef* r_dev, cudaStream_t s,
                          const ef* eq_in, ef* eq_out, size_t eq_half) {
  const size_t bx = std::max((half + 127) / 128, eq_in ? (eq_half + 255) / 256 : size_t(0));
  dim3 grid((unsigned)std::max<size_t>(bx, 1), ncols + (eq_in ? 1 : 0));
  k_fold_cols_mma<<<grid, 256, 0, s>>>(in, out, half, ncols, ef_zero(), r_dev, eq_in, eq_out, eq_half);
  WL_LAUNCH_CHECK();
}
void launch_inner_sums(const uint32_t* wit, int log_n, int k, int ll, const ef* eq_hi, const ef* eq_lo,
                       const ef* sel, ef* out_up, ef* out_down, uint8_t* limbs, cudaStream_t s, int plan,
                       unsigned* timeouts) {
  // out_up / out_down hold AIR_W results followed by AIR_W * 2^k * 2^(log_n - k - ll) partials.
  const int nsk = 1 << k;
  const int nh = 1 << (log_n - k - ll);
  ef* pu = out_up + AIR_W;
  ef* pd = out_down + AIR_W;
  if (limbs && ll >= INNER_MMA_MIN_LL && ll <= 12) {  // 2^12 byte products per s32 sum
    const int nlo = 1 << ll;
    k_eq_limbs<<<(16 * nlo + 255) / 256, 256, 0, s>>>(eq_lo, nlo, limbs);
    WL_LAUNCH_CHECK();
    const uint32_t M = uint32_t(AIR_W) * nsk * nh;
    if (plan == 1 && timeouts)
      k_inner_sums_bulk<<<(M + 15) / 16, ISM_WARPS * 32, 0, s>>>(wit, log_n, k, ll, eq_hi, eq_lo, limbs, pu, pd,
                                                                 timeouts);
    else
      k_inner_sums_mma<<<(M + 15) / 16, ISM_WARPS * 32, 0, s>>>(wit, log_n, k, ll, eq_hi, eq_lo, limbs, pu, pd);
  } else {
    k_inner_sums<<<dim3((AIR_W + 1) / 2, nsk, (nh + IS_WARPS - 1) / IS_WARPS), IS_WARPS * 32, 0, s>>>(
        wit, log_n, k, ll, eq_hi, eq_lo, pu, pd);
  }
  WL_LAUNCH_CHECK();
  k_combine_sel<<<(AIR_W + 7) / 8, 256, 0, s>>>(pu, sel, nsk, nh, AIR_W, out_up);
  WL_LAUNCH_CHECK();
  k_combine_sel<<<(AIR_W + 7) / 8, 256, 0, s>>>(pd, sel, nsk, nh, AIR_W, out_down);
  WL_LAUNCH_CHECK();
}
size_t colsum_limb_bytes(int K) { return K > 192 ? 0 : size_t(32) * ((K + 31) / 32 * 32); }
void launch_batch_cols_mma(const uint32_t* wit, int log_n, const ef* eqc, ef* out, uint8_t* limbs, cudaStream_t s) {
  const size_t N = size_t(1) << log_n;
  const int K = AIR_W, Kp = (K + 31) / 32 * 32;
  k_w_limbs<<<(8 * Kp + 255) / 256, 256, 0, s>>>(eqc, K, Kp, limbs);
  WL_LAUNCH_CHECK();
  const size_t tiles = (N + 15) / 16;
  k_colsum_mma<<<(unsigned)((tiles + CS_WARPS - 1) / CS_WARPS), CS_WARPS * 32, 0, s>>>(wit, N, K, Kp, N, limbs, out);
  WL_LAUNCH_CHECK();
}
size_t mle_partial_scratch_bytes(int lu, int lh, int ll) {
  if (ll < INNER_MMA_MIN_LL || ll > 12 || lh < 4) return 0;
  return (sizeof(ef) << (lu + lh - 4)) + (size_t(32) << ll);
}
bool launch_mle_partial_mma(const uint32_t* T, size_t t_len, int lu, int lh, int ll, const ef* hi, const ef* lo,
                            ef* out, void* scratch, cudaStream_t s) {
  if (!scratch || !mle_partial_scratch_bytes(lu, lh, ll) || t_len % (size_t(1) << ll)) return false;
  ef* partial = static_cast<ef*>(scratch);
  uint8_t* limbs = reinterpret_cast<uint8_t*>(partial + (size_t(1) << (lu + lh - 4)));
  const int nlo = 1 << ll;
  k_lo_limbs<<<(8 * nlo + 255) / 256, 256, 0, s>>>(lo, nlo, limbs);
  WL_LAUNCH_CHECK();
  const uint32_t tiles = 1u << (lu + lh - 4);
  k_mle_partial_mma<<<(tiles + CS_WARPS - 1) / CS_WARPS, CS_WARPS * 32, 0, s>>>(T, t_len, lu, lh, ll, hi, limbs,
                                                                               partial);
  WL_LAUNCH_CHECK();
  launch_reduce_partials(partial, 1 << (lh - 4), 1 << lu, out, s);
  return true;
}
void launch_batch_cols(const uint32_t* wit, int log_n, const ef* eqc, ef* out, cudaStream_t s) {
  if (log_n < 1) throw std::invalid_argument("batch_cols: at least 2 rows");
  size_t N = size_t(1) << log_n;
  k_batch_cols<<<(unsigned)((N / 2 + 255) / 256), 256, 0, s>>>(wit, log_n, eqc, out);
  WL_LAUNCH_CHECK();
}
int sub_eval_blocks(int log_n, int k) {
  size_t S = size_t(1) << (log_n - k);
  size_t per = size_t(SUB_THREADS) * SUB_PER_THREAD;
  return (int)((S + per - 1) / per);
}
void launch_sub_evals(const ef* B, int log_n, int k, const ef* alpha2, const ef* eqt, ef* partial, cudaStream_t s) {
  (void)alpha2;
  dim3 grid(sub_eval_blocks(log_n, k), 1u << k);
  k_sub_evals<<<grid, SUB_THREADS, 0, s>>>(B, log_n, k, eqt, partial);
  WL_LAUNCH_CHECK();
}
void launch_inner_mle(const ef* e, int log_n, const ef* alpha2, ef* out, cudaStream_t s) {
  size_t N = size_t(1) << log_n;
  k_inner_mle<<<(unsigned)((N + 255) / 256), 256, 0, s>>>(e, log_n, alpha2, out);
  WL_LAUNCH_CHECK();
}
int prod_blocks(size_t half) {
  size_t per = size_t(PROD_THREADS) * prod_per_thread(half);
  return (int)((half + per - 1) / per);
}
void launch_prod_eval(const ef* a, const ef* b, size_t half, ef* partial, cudaStream_t s) {
  k_prod_eval<<<prod_blocks(half), PROD_THREADS, 0, s>>>(a, b, half, prod_per_thread(half), partial);
  WL_LAUNCH_CHECK();
}
void launch_fold2_at(const ef* a, const ef* b, ef* oa, ef* ob, size_t half, const ef& r, cudaStream_t s) {
  k_fold2_mma<<<dim3((unsigned)((half + 127) / 128), 2), 256, 0, s>>>(a, b, oa, ob, half, r, nullptr);
  WL_LAUNCH_CHECK();
}
void launch_fold2_dev(const ef* a, const ef* b, ef* oa, ef* ob, size_t half, const ef* r_dev, cudaStream_t s) {
  k_fold2_mma<<<dim3((unsigned)((half + 127) / 128), 2), 256, 0, s>>>(a, b, oa, ob, half, ef_zero(), r_dev);
  WL_LAUNCH_CHECK();
}

int fold_eval_blocks(size_t h) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return (int)std::max<size_t>(1, std::min<size_t>((h + FE_THREADS - 1) / FE_THREADS, size_t(sms) * 4));
}
void launch_pair_fold_eval(int nsums, const ef* a, const ef* b, const ef* r_dev, ef* na, ef* nb, size_t h,
                           ef* partial, const FinArgs* fin, cudaStream_t s) {
  const int g = fold_eval_blocks(h);
  const FinArgs f = fin ? *fin : FinArgs{};
  if (nsums == 2)
    k_pair_fold_eval<2><<<g, FE_THREADS, 0, s>>>(a, b, r_dev, na, nb, h, partial, f);
  else if (nsums == 3)
    k_pair_fold_eval<3><<<g, FE_THREADS, 0, s>>>(a, b, r_dev, na, nb, h, partial, f);
  else
    throw std::invalid_argument("fold-evaluate: 2 or 3 sums");
  WL_LAUNCH_CHECK();
}
void launch_abc_fold_eval(const ef* cols, const ef* r_dev, const ef* eq_prev, ef* nc, ef* eq_new, size_t h, ef* partial,
                          const FinArgs* fin, cudaStream_t s) {
  const FinArgs f = fin ? *fin : FinArgs{};
  if (fin && (!f.req || !f.rinv)) throw std::invalid_argument("fold-evaluate: eq-factor rounds need their eq challenges");
  k_abc_fold_eval<<<fold_eval_blocks(h), FE_THREADS, 0, s>>>(cols, r_dev, eq_prev, nc, eq_new, h, partial, f);
  WL_LAUNCH_CHECK();
}

int abc0_blocks(int log_n, int k) {
  const size_t S = size_t(1) << (log_n - k);
  if (k > 3) return (int)((S + ABC_X - 1) / ABC_X);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return (int)std::max<size_t>(1, std::min<size_t>((S + ABC0_THREADS - 1) / ABC0_THREADS, size_t(sms) * 2));
}
void launch_abc0_eval(const uint32_t* a, const uint32_t* b, const uint32_t* c, int log_n, int k, int nz,
                      const uint32_t* lw, const ef* eq, ef* partial, cudaStream_t s) {
  if (k > 3) {
    if (nz > 32 || k > 4) throw std::runtime_error("abc round 0: too many points");
    k_abc0_eval_points<<<abc0_blocks(log_n, k), dim3(ABC_X, nz), 0, s>>>(a, b, c, log_n, k, nz, lw, eq, partial);
  } else {
    if (nz > ABC0_MAX_Z) throw std::runtime_error("abc round 0: too many points");
    k_abc0_eval<<<abc0_blocks(log_n, k), ABC0_THREADS, 0, s>>>(a, b, c, log_n, k, nz, lw, eq, partial);
  }
  WL_LAUNCH_CHECK();
}
void launch_abc0_fold(const uint32_t* a, const uint32_t* b, const uint32_t* c, int log_n, int k, const ef* sel,
                      ef* out, cudaStream_t s) {
  size_t S = size_t(1) << (log_n - k);
  k_abc0_fold<<<dim3((unsigned)((S + 255) / 256), 3), 256, 0, s>>>(a, b, c, log_n, k, sel, out);
  WL_LAUNCH_CHECK();
}
void launch_abc_eval_ef(const ef* cols, int m, const ef* eq, ef* partial, cudaStream_t s) {
  size_t half = size_t(1) << (m - 1);
  k_abc_eval_ef<<<(unsigned)((half + 31) / 32), dim3(32, 2), 0, s>>>(cols, m, eq, partial);
  WL_LAUNCH_CHECK();
}

}  // namespace wl
