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
#include "kernels.h"

namespace wl {

namespace {
using namespace kb;

__device__ __forceinline__ size_t up_row(size_t i, size_t N) { return i == N - 1 ? N - 2 : i; }
__device__ __forceinline__ size_t down_row(size_t i, size_t N) { return i == N - 1 ? N - 1 : i + 1; }

// ------------------------------------------------------------------ eq tables
// out[x] = prod_i (x_i ? r_i : 1 - r_i), x_1 = most significant bit of x.
__global__ void k_eq_table(const ef* __restrict__ pt, int nvars, ef* __restrict__ out) {
  __shared__ ef hi_val;
  const int nlo = nvars < 10 ? nvars : 10;
  const int nhi = nvars - nlo;
  const size_t xhi = blockIdx.x;
  if (threadIdx.x == 0) {
    ef h = ef_one();
    for (int i = 0; i < nhi; i++) {
      bool bit = (xhi >> (nhi - 1 - i)) & 1;
      h = ef_mul(h, bit ? pt[i] : ef_sub(ef_one(), pt[i]));
    }
    hi_val = h;
  }
  __syncthreads();
  const uint32_t xlo = threadIdx.x;
  if (xlo >= (1u << nlo)) return;
  ef v = hi_val;
  for (int i = 0; i < nlo; i++) {
    bool bit = (xlo >> (nlo - 1 - i)) & 1;
    const ef& r = pt[nhi + i];
    v = ef_mul(v, bit ? r : ef_sub(ef_one(), r));
  }
  out[(xhi << nlo) + xlo] = v;
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
constexpr int ZC0_X = 32, ZC0_Z = 15;
constexpr int ZC0_STAGES = 4;   // columns in flight
constexpr int ZC0_PAD = 20;     // words per x in a staged column tile (16 values + padding)

__device__ __forceinline__ void cp_async4(uint32_t* smem, const uint32_t* gmem) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// Thread (x, z): the up columns are extended from their values at j * 2^(n-k) + x, j < 2^k,
// to the point z by the Lagrange weights L_j(z); the batched constraint over those values is
// weighted by eq[x]. A warp holds 32 consecutive x for one z. The 2^k x 32 values of each
// column are staged in shared memory by a cp.async pipeline (the constraint reads columns
// 1..164 in increasing order, each exactly once), so the extension reads shared memory only.
__global__ void __launch_bounds__(ZC0_X * ZC0_Z, 1) k_zc0_eval(const uint32_t* __restrict__ wit, int log_n, int k,
                                                               int nz, const uint32_t* __restrict__ lw,
                                                               const ef* __restrict__ eq,
                                                               const ef* __restrict__ alphas_g,
                                                               const __grid_constant__ AirConsts K,
                                                               ef* __restrict__ partial) {
  __shared__ ef alphas[AIR_NC];
  __shared__ __align__(16) uint32_t tile[ZC0_STAGES][ZC0_X * ZC0_PAD];
  const int tid = threadIdx.y * ZC0_X + threadIdx.x;
  constexpr int NT = ZC0_X * ZC0_Z;
  for (int i = tid; i < AIR_NC; i += NT) alphas[i] = alphas_g[i];
  const int zi = blockIdx.y * ZC0_Z + threadIdx.y;
  const int nsk = 1 << k;
  const size_t N = size_t(1) << log_n;
  const size_t S = N >> k;
  const size_t x0 = size_t(blockIdx.x) * ZC0_X;
  const size_t x = x0 + threadIdx.x;
  uint32_t w[16];
#pragma unroll
  for (int j = 0; j < 16; j++) w[j] = (zi < nz && j < nsk) ? lw[zi * nsk + j] : 0u;

  // producer: column c's tile -> slot, tile[slot][xl * PAD + j] = up_c[j * S + x0 + xl]
  auto issue = [&](int c) {
    if (c < AIR_W) {
      uint32_t* dst = tile[c % ZC0_STAGES];
      const uint32_t* col = wit + size_t(c) * N;
      for (int idx = tid; idx < 16 * ZC0_X; idx += NT) {
        const int j = idx / ZC0_X, xl = idx % ZC0_X;
        if (j < nsk) {
          size_t xx = x0 + xl;
          if (xx >= S) xx = 0;
          cp_async4(dst + xl * ZC0_PAD + j, col + up_row(size_t(j) * S + xx, N));
        }
      }
    }
    cp_async_commit();
  };
  for (int c = 1; c < 1 + ZC0_STAGES - 1; c++) issue(c);
  int next = ZC0_STAGES;  // next column to prefetch
  auto get = [&](int c) -> uint32_t {
    cp_async_wait<ZC0_STAGES - 2>();
    __syncthreads();
    issue(next++);
    const uint4* row = reinterpret_cast<const uint4*>(tile[c % ZC0_STAGES] + threadIdx.x * ZC0_PAD);
    uint64_t s0 = 0, s1 = 0, s2 = 0, s3 = 0;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      if (4 * q < nsk) {
        uint4 v = row[q];
        s0 += wmul(w[4 * q], v.x);
        s1 += wmul(w[4 * q + 1], v.y);
        s2 += wmul(w[4 * q + 2], v.z);
        s3 += wmul(w[4 * q + 3], v.w);
      }
    }
    return add(add(redc(s0), redc(s1)), add(redc(s2), redc(s3)));
  };
  __syncthreads();  // alphas
  EfMacF m;
  m.init();
  air_eval_f(
      K, get, [&](uint32_t h, int i) { m.mac(alphas[i], h); }, [&]() { m.flush(); });
  cp_async_wait<0>();
  const bool active = zi < nz && x < S;
  ef res = active ? ef_mul(m.acc, eq[x]) : ef_zero();
  res = warp_reduce_ef(res);
  if (threadIdx.x == 0 && zi < nz) partial[size_t(blockIdx.x) * nz + zi] = res;
}

// out[c * S + x] = sum_j sel[j] * up_c[j * S + x]  (the 2^k loads are issued before the
// products, sel is zero-padded to 16)
__global__ void k_zc0_fold(const uint32_t* __restrict__ wit, int log_n, int k, const ef* __restrict__ sel_g,
                           ef* __restrict__ out) {
  __shared__ ef sel[16];
  const int nsk = 1 << k;
  if (threadIdx.x < 16) sel[threadIdx.x] = threadIdx.x < (unsigned)nsk ? sel_g[threadIdx.x] : ef_zero();
  __syncthreads();
  const size_t N = size_t(1) << log_n, S = N >> k;
  const size_t x = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (x >= S) return;
  const uint32_t* col = wit + size_t(c) * N;
  uint32_t v[16];
#pragma unroll
  for (int j = 0; j < 16; j++) v[j] = j < nsk ? col[up_row(size_t(j) * S + x, N)] : 0u;
  EfMacF m;
  m.init();
#pragma unroll
  for (int j = 0; j < 16; j++) {
    m.mac(sel[j], v[j]);
    if ((j & 3) == 3) m.flush();
  }
  out[size_t(c) * S + x] = m.acc;
}

constexpr int ZCE_T = 128;  // (x, z) points per block

// The 16 extension-field state words of each thread live in shared memory as two planes
// of uint4 (coordinates 0-3 and 4-7), so that a warp's 128-bit accesses are conflict-free.
struct SmemState {
  uint4* p0;
  uint4* p1;
  int t;
  __device__ __forceinline__ ef get(int i) const {
    uint4 a = p0[i * ZCE_T + t], b = p1[i * ZCE_T + t];
    return ef{{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w}};
  }
  __device__ __forceinline__ void set(int i, const ef& v) const {
    p0[i * ZCE_T + t] = make_uint4(v.c[0], v.c[1], v.c[2], v.c[3]);
    p1[i * ZCE_T + t] = make_uint4(v.c[4], v.c[5], v.c[6], v.c[7]);
  }
};

__device__ __forceinline__ ef ef_diag16(int i, const ef& a) {
  ef r;
#pragma unroll
  for (int k = 0; k < 8; k++) r.c[k] = p2_diag_mul<16>(i, a.c[k]);
  return r;
}

__device__ void mds_light_smem(const SmemState& S) {
#pragma unroll 1
  for (int c = 0; c < 16; c += 4) {
    ef x0 = S.get(c), x1 = S.get(c + 1), x2 = S.get(c + 2), x3 = S.get(c + 3);
    ef t01 = ef_add(x0, x1), t23 = ef_add(x2, x3), t0123 = ef_add(t01, t23);
    ef t01123 = ef_add(t0123, x1), t01233 = ef_add(t0123, x3);
    S.set(c + 3, ef_add(t01233, ef_add(x0, x0)));
    S.set(c + 1, ef_add(t01123, ef_add(x2, x2)));
    S.set(c, ef_add(t01123, t01));
    S.set(c + 2, ef_add(t01233, t23));
  }
#pragma unroll 1
  for (int k = 0; k < 4; k++) {
    ef a = S.get(k), b = S.get(4 + k), c = S.get(8 + k), d = S.get(12 + k);
    ef sk = ef_add(ef_add(a, b), ef_add(c, d));
    S.set(k, ef_add(a, sk));
    S.set(4 + k, ef_add(b, sk));
    S.set(8 + k, ef_add(c, sk));
    S.set(12 + k, ef_add(d, sk));
  }
}

// Internal layer with lane 0 replaced by x0.
__device__ void internal_layer_smem_with0(const SmemState& S, const ef& x0) {
  ef sum = x0;
#pragma unroll 1
  for (int i = 1; i < 16; i++) sum = ef_add(sum, S.get(i));
  S.set(0, ef_add(ef_diag16(0, x0), sum));
#pragma unroll 1
  for (int i = 1; i < 16; i++) S.set(i, ef_add(ef_diag16(i, S.get(i)), sum));
}

constexpr int ZCE_FULL_SEGS = 7;  // full rounds evaluated without state
constexpr int ZCE_SEGMENTS = ZCE_FULL_SEGS + 1;

// 4x4 block M4 = [[2,3,1,1],[1,2,3,1],[1,1,2,3],[3,1,1,2]] applied to a chunk.
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

// Rounds >= 1, full rounds without state. For full round f with constraint weights
// alpha_(c0 + i), sum_i alpha_(c0+i) (MDS(cubes)_i - post_i) = sum_j beta_(f,j) cube_j -
// sum_i alpha_(c0+i) post_i, beta_f = MDS^T alpha (computed once on the host), and each
// full round's input is committed: the previous round's post columns, or MDS(inputs) for
// the first round (streamed: column sums of the M4 outputs, then chunk by chunk).
// Block (x range, z, segment); segments 0..3 are the beginning rounds, 4..6 the ending
// rounds 1..3. z = 0, 2, 3 for blockIdx.y = 0, 1, 2.
__global__ void __launch_bounds__(ZCE_T, 4) k_zc_full_ef(const ef* __restrict__ cols, int m, const ef* __restrict__ eq,
                                                     const ef* __restrict__ alphas, const ef* __restrict__ betas,
                                                     const __grid_constant__ AirConsts K, ef* __restrict__ partial) {
  const size_t len = size_t(1) << m, half = len >> 1;
  const size_t x = size_t(blockIdx.x) * ZCE_T + threadIdx.x;
  const int zi = blockIdx.y, seg = blockIdx.z;
  const size_t xs = x < half ? x : 0;
  auto get = [&](int c) -> ef {
    const ef lo = cols[size_t(c) * len + xs];
    if (zi == 0) return lo;
    const ef hi = cols[size_t(c) * len + half + xs];
    ef d = ef_sub(hi, lo);
    ef v = ef_add(hi, d);               // z = 2: 2 hi - lo
    return zi == 1 ? v : ef_add(v, d);  // z = 3: 3 hi - 2 lo
  };
  const int f = seg < 4 ? seg : seg + 1;  // full-round index 0..7 (4 = first ending round, not here)
  const uint32_t* rc = seg < 4 ? K.begin[seg] : K.end[seg - 3];
  const int post = seg < 4 ? 17 + 16 * seg : 101 + 16 * (seg - 3);
  const int c0 = seg < 4 ? 16 * seg : 84 + 16 * (seg - 3);
  const ef* beta = betas + 16 * f;
  ef acc = ef_zero();
  if (seg == 0) {
    ef S[4] = {ef_zero(), ef_zero(), ef_zero(), ef_zero()};
#pragma unroll 1
    for (int q = 0; q < 4; q++) {
      ef y0 = get(1 + 4 * q), y1 = get(2 + 4 * q), y2 = get(3 + 4 * q), y3 = get(4 + 4 * q);
      m4_ef(y0, y1, y2, y3);
      S[0] = ef_add(S[0], y0);
      S[1] = ef_add(S[1], y1);
      S[2] = ef_add(S[2], y2);
      S[3] = ef_add(S[3], y3);
    }
#pragma unroll 1
    for (int q = 0; q < 4; q++) {
      ef y[4] = {get(1 + 4 * q), get(2 + 4 * q), get(3 + 4 * q), get(4 + 4 * q)};
      m4_ef(y[0], y[1], y[2], y[3]);
#pragma unroll
      for (int kk = 0; kk < 4; kk++) {
        const int j = 4 * q + kk;
        const ef in = ef_add(y[kk], S[kk]);
        acc = ef_add(acc, ef_mul(beta[j], ef_cube(ef_add_f(in, rc[j]))));
      }
    }
  } else {
    const int src = post - 16;
#pragma unroll 1
    for (int j = 0; j < 16; j++) acc = ef_add(acc, ef_mul(beta[j], ef_cube(ef_add_f(get(src + j), rc[j]))));
  }
#pragma unroll 1
  for (int i = 0; i < 16; i++) acc = ef_sub(acc, ef_mul(alphas[c0 + i], get(post + i)));
  ef res = x < half ? ef_mul(acc, eq[x]) : ef_zero();
  res = warp_reduce_ef(res);
  __shared__ ef wsum[ZCE_T / 32];
  if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = res;
  __syncthreads();
  if (threadIdx.x == 0) {
    ef tot = wsum[0];
    for (int w = 1; w < ZCE_T / 32; w++) tot = ef_add(tot, wsum[w]);
    partial[(size_t(blockIdx.x) * ZCE_FULL_SEGS + seg) * 3 + zi] = tot;
  }
}

// Rounds >= 1, the partial rounds and the first ending round, which starts from the state
// after the partial rounds: the 16-word state lives in shared memory, loops stay rolled.
__global__ void __launch_bounds__(ZCE_T) k_zc_partial_ef(const ef* __restrict__ cols, int m, const ef* __restrict__ eq,
                                                        const ef* __restrict__ alphas_g,
                                                        const ef* __restrict__ betas,
                                                        const __grid_constant__ AirConsts K,
                                                        ef* __restrict__ partial) {
  extern __shared__ __align__(16) unsigned char smraw[];
  ef* alphas = reinterpret_cast<ef*>(smraw);
  uint4* planes = reinterpret_cast<uint4*>(smraw + sizeof(ef) * AIR_NC);
  for (int i = threadIdx.x; i < AIR_NC; i += ZCE_T) alphas[i] = alphas_g[i];
  const SmemState S{planes, planes + 16 * ZCE_T, (int)threadIdx.x};
  __syncthreads();
  const size_t len = size_t(1) << m, half = len >> 1;
  const size_t x = size_t(blockIdx.x) * ZCE_T + threadIdx.x;
  const int zi = blockIdx.y;
  const size_t xs = x < half ? x : 0;
  auto get = [&](int c) -> ef {
    const ef lo = cols[size_t(c) * len + xs];
    if (zi == 0) return lo;
    const ef hi = cols[size_t(c) * len + half + xs];
    ef d = ef_sub(hi, lo);
    ef v = ef_add(hi, d);
    return zi == 1 ? v : ef_add(v, d);
  };
  ef acc = ef_zero();
#pragma unroll 1
  for (int i = 0; i < 16; i++) S.set(i, get(65 + i));
#pragma unroll 1
  for (int r = 0; r < 20; r++) {
    const ef x0 = ef_cube(ef_add_f(S.get(0), K.partial[r]));
    const ef p = get(81 + r);
    acc = ef_add(acc, ef_mul(alphas[64 + r], ef_sub(x0, p)));
    internal_layer_smem_with0(S, p);
  }
  const ef* beta = betas + 16 * 4;
#pragma unroll 1
  for (int j = 0; j < 16; j++) acc = ef_add(acc, ef_mul(beta[j], ef_cube(ef_add_f(S.get(j), K.end[0][j]))));
#pragma unroll 1
  for (int i = 0; i < 16; i++) acc = ef_sub(acc, ef_mul(alphas[84 + i], get(101 + i)));
  ef res = x < half ? ef_mul(acc, eq[x]) : ef_zero();
  res = warp_reduce_ef(res);
  __shared__ ef wsum[ZCE_T / 32];
  if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = res;
  __syncthreads();
  if (threadIdx.x == 0) {
    ef tot = wsum[0];
    for (int w = 1; w < ZCE_T / 32; w++) tot = ef_add(tot, wsum[w]);
    partial[size_t(blockIdx.x) * 3 + zi] = tot;
  }
}

__global__ void k_fold_cols(const ef* __restrict__ in, ef* __restrict__ out, size_t half, int ncols,
                            const ef* __restrict__ r, const ef* __restrict__ eq_in, ef* __restrict__ eq_out,
                            size_t eq_half) {
  const size_t x = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (c == ncols) {
    if (x < eq_half) eq_out[x] = ef_add(eq_in[x], eq_in[x + eq_half]);
    return;
  }
  if (x >= half) return;
  const ef* src = in + size_t(c) * 2 * half;
  out[size_t(c) * half + x] = ef_lerp(src[x], src[half + x], *r);
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
  const size_t N = size_t(1) << log_n, S = N >> k;
  const int c = blockIdx.x, j = blockIdx.y;
  const uint32_t nhi = 1u << (log_n - k - ll);
  const uint32_t xh = blockIdx.z * IS_WARPS + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (xh >= nhi) return;
  const uint32_t nlo = 1u << ll;
  const uint32_t* col = wit + size_t(c) * N + size_t(j) * S + (size_t(xh) << ll);
  const bool last = j == gridDim.y - 1 && xh == nhi - 1;  // holds the wrapped row N - 1
  EfMacF mu, md;
  mu.init();
  md.init();
  uint32_t xl = lane;
  for (; xl + 96 < nlo; xl += 128) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const uint32_t x = xl + 32 * q;
      const ef e = eq_lo[x];
      const bool wrap = last && x == nlo - 1;
      mu.mac(e, col[wrap ? x - 1 : x]);
      md.mac(e, col[wrap ? x : x + 1]);
    }
    mu.flush();
    md.flush();
  }
  for (; xl < nlo; xl += 32) {
    const ef e = eq_lo[xl];
    const bool wrap = last && xl == nlo - 1;
    mu.mac(e, col[wrap ? xl - 1 : xl]);
    md.mac(e, col[wrap ? xl : xl + 1]);
    mu.flush();
    md.flush();
  }
  const ef su = warp_reduce_ef(mu.acc), sd = warp_reduce_ef(md.acc);
  if (lane == 0) {
    const size_t o = (size_t(c) * gridDim.y + j) * nhi + xh;
    pu[o] = ef_mul(su, eq_hi[xh]);
    pd[o] = ef_mul(sd, eq_hi[xh]);
  }
}

// out[c] = sum_j sel[j] * sum_h partial[(c * nsk + j) * nh + h]
__global__ void k_combine_sel(const ef* __restrict__ partial, const ef* __restrict__ sel, int nsk, int nh, int ncols,
                              ef* __restrict__ out) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncols) return;
  ef acc = ef_zero();
  for (int j = 0; j < nsk; j++) {
    ef s = ef_zero();
    for (int h = 0; h < nh; h++) s = ef_add(s, partial[(size_t(c) * nsk + j) * nh + h]);
    acc = ef_add(acc, ef_mul(sel[j], s));
  }
  out[c] = acc;
}

// ------------------------------------------------------------------ inner phase
__global__ void k_batch_cols(const uint32_t* __restrict__ wit, int log_n, const ef* __restrict__ eqc_g,
                             ef* __restrict__ out) {
  __shared__ ef eqc[AIR_W + 3];
  for (int i = threadIdx.x; i < AIR_W + 3; i += blockDim.x) eqc[i] = i < AIR_W ? eqc_g[i] : ef_zero();
  __syncthreads();
  const size_t N = size_t(1) << log_n;
  const size_t row = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (row >= N) return;
  EfMacF m;
  m.init();
#pragma unroll 2
  for (int c = 0; c < AIR_W; c += 4) {
    uint32_t v[4];
#pragma unroll
    for (int q = 0; q < 4; q++) v[q] = c + q < AIR_W ? wit[size_t(c + q) * N + row] : 0u;
#pragma unroll
    for (int q = 0; q < 4; q++) m.mac(eqc[c + q], v[q]);
    m.flush();
  }
  out[row] = m.acc;
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

constexpr int PROD_THREADS = 256, PROD_PER_THREAD = 8;

__global__ void k_prod_eval(const ef* __restrict__ a, const ef* __restrict__ b, size_t half, ef* __restrict__ partial) {
  __shared__ ef scratch[32];
  ef s0 = ef_zero(), s2 = ef_zero();
  for (int q = 0; q < PROD_PER_THREAD; q++) {
    size_t x = (size_t(blockIdx.x) * PROD_PER_THREAD + q) * PROD_THREADS + threadIdx.x;
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

__global__ void k_fold2(const ef* __restrict__ a, const ef* __restrict__ b, ef* __restrict__ oa, ef* __restrict__ ob,
                        size_t half, const ef* __restrict__ r) {
  const size_t x = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (x >= half) return;
  const ef rr = *r;
  oa[x] = ef_lerp(a[x], a[x + half], rr);
  ob[x] = ef_lerp(b[x], b[x + half], rr);
}

// ------------------------------------------------------------------ a*b - c
constexpr int ABC_X = 32;

__global__ void k_abc0_eval(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b,
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
  out[size_t(blockIdx.y) * S + x] = m.acc;
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
  int nlo = nvars < 10 ? nvars : 10;
  k_eq_table<<<(unsigned)(size_t(1) << (nvars - nlo)), 1u << nlo, 0, s>>>(point, nvars, out);
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
void launch_zc0_eval(const uint32_t* wit, int log_n, int k, int nz, const uint32_t* lw, const ef* eq,
                     const ef* alphas, const AirConsts& K, ef* partial, cudaStream_t s) {
  dim3 grid(zc0_blocks(log_n, k), (nz + ZC0_Z - 1) / ZC0_Z), block(ZC0_X, ZC0_Z);
  k_zc0_eval<<<grid, block, 0, s>>>(wit, log_n, k, nz, lw, eq, alphas, K, partial);
  WL_LAUNCH_CHECK();
}
void launch_zc0_fold(const uint32_t* wit, int log_n, int k, const ef* sel, ef* out, cudaStream_t s) {
  size_t S = size_t(1) << (log_n - k);
  dim3 grid((unsigned)((S + 255) / 256), AIR_W);
  k_zc0_fold<<<grid, 256, 0, s>>>(wit, log_n, k, sel, out);
  WL_LAUNCH_CHECK();
}
int zc_ef_blocks(int m) {  // partial sums per z: (x blocks) x (7 full-round segments + 1)
  size_t half = size_t(1) << (m - 1);
  return (int)((half + ZCE_T - 1) / ZCE_T) * ZCE_SEGMENTS;
}
void launch_zc_eval_ef(const ef* cols, int m, const ef* eq, const ef* alphas, const ef* betas, const AirConsts& K,
                       ef* partial, cudaStream_t s) {
  const unsigned xb = (unsigned)(zc_ef_blocks(m) / ZCE_SEGMENTS);
  k_zc_full_ef<<<dim3(xb, 3, ZCE_FULL_SEGS), ZCE_T, 0, s>>>(cols, m, eq, alphas, betas, K, partial);
  WL_LAUNCH_CHECK();
  const size_t smem = sizeof(ef) * AIR_NC + sizeof(uint4) * 2 * 16 * ZCE_T;
  WL_CUDA(cudaFuncSetAttribute(k_zc_partial_ef, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_zc_partial_ef<<<dim3(xb, 3), ZCE_T, smem, s>>>(cols, m, eq, alphas, betas, K,
                                                   partial + size_t(xb) * ZCE_FULL_SEGS * 3);
  WL_LAUNCH_CHECK();
}
void launch_fold_cols(const ef* in, ef* out, int ncols, size_t half, const ef* r, cudaStream_t s, const ef* eq_in,
                      ef* eq_out, size_t eq_half) {
  const size_t width = eq_in && eq_half > half ? eq_half : half;
  dim3 grid((unsigned)((width + 255) / 256), ncols + (eq_in ? 1 : 0));
  k_fold_cols<<<grid, 256, 0, s>>>(in, out, half, ncols, r, eq_in, eq_out, eq_half);
  WL_LAUNCH_CHECK();
}
void launch_inner_sums(const uint32_t* wit, int log_n, int k, int ll, const ef* eq_hi, const ef* eq_lo,
                       const ef* sel, ef* out_up, ef* out_down, cudaStream_t s) {
  // out_up / out_down hold AIR_W results followed by AIR_W * 2^k * 2^(log_n - k - ll) partials.
  const int nsk = 1 << k;
  const int nh = 1 << (log_n - k - ll);
  ef* pu = out_up + AIR_W;
  ef* pd = out_down + AIR_W;
  k_inner_sums<<<dim3(AIR_W, nsk, (nh + IS_WARPS - 1) / IS_WARPS), IS_WARPS * 32, 0, s>>>(wit, log_n, k, ll, eq_hi,
                                                                                         eq_lo, pu, pd);
  WL_LAUNCH_CHECK();
  k_combine_sel<<<(AIR_W + 127) / 128, 128, 0, s>>>(pu, sel, nsk, nh, AIR_W, out_up);
  WL_LAUNCH_CHECK();
  k_combine_sel<<<(AIR_W + 127) / 128, 128, 0, s>>>(pd, sel, nsk, nh, AIR_W, out_down);
  WL_LAUNCH_CHECK();
}
void launch_batch_cols(const uint32_t* wit, int log_n, const ef* eqc, ef* out, cudaStream_t s) {
  size_t N = size_t(1) << log_n;
  k_batch_cols<<<(unsigned)((N + 255) / 256), 256, 0, s>>>(wit, log_n, eqc, out);
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
  size_t per = size_t(PROD_THREADS) * PROD_PER_THREAD;
  return (int)((half + per - 1) / per);
}
void launch_prod_eval(const ef* a, const ef* b, size_t half, ef* partial, cudaStream_t s) {
  k_prod_eval<<<prod_blocks(half), PROD_THREADS, 0, s>>>(a, b, half, partial);
  WL_LAUNCH_CHECK();
}
void launch_fold2(const ef* a, const ef* b, ef* oa, ef* ob, size_t half, const ef* r, cudaStream_t s) {
  k_fold2<<<(unsigned)((half + 255) / 256), 256, 0, s>>>(a, b, oa, ob, half, r);
  WL_LAUNCH_CHECK();
}

int abc0_blocks(int log_n, int k) {
  size_t S = size_t(1) << (log_n - k);
  return (int)((S + ABC_X - 1) / ABC_X);
}
void launch_abc0_eval(const uint32_t* a, const uint32_t* b, const uint32_t* c, int log_n, int k, int nz,
                      const uint32_t* lw, const ef* eq, ef* partial, cudaStream_t s) {
  if (nz > 32 || k > 4) throw std::runtime_error("abc round 0: too many points");
  k_abc0_eval<<<abc0_blocks(log_n, k), dim3(ABC_X, nz), 0, s>>>(a, b, c, log_n, k, nz, lw, eq, partial);
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
