// WHIR kernels (the bulk work of whir-p3's Prover::prove, reached from
// crates/air/src/prove.rs:216-225): partial evaluations of the committed base-field table
// for the initial constraints, the fold of that table after the first sumcheck block,
// accumulation of equality-weight terms for OOD / STIR constraints, the weighted sumcheck
// rounds and OOD answers of extension-field polynomials.
//
// Equality polynomials over m variables are factored as eq(pt, v) = hi(v_hi) * lo(v_lo)
// with v_lo the low ll bits, so a table of 2^m entries costs 2^lh + 2^ll to build.
#include <algorithm>

#include "kernels.h"
#include "limb_mma.cuh"

namespace wl {

namespace {
using namespace kb;

constexpr int MPB_SPLIT = 16;  // v_hi groups per column block

// out[(j * 2^lu + u) * MPB_SPLIT + g] = sum over v_hi in group g, v_lo of
//   T[u * 2^lv + v] * hi_j[v_hi] * lo_j[v_lo]
template <int J>
__global__ void k_mle_partial_base(const uint32_t* __restrict__ T, size_t t_len, int lu, int lh, int ll,
                                   const ef* __restrict__ hi, const ef* __restrict__ lo, ef* __restrict__ out) {
  __shared__ ef scratch[32];
  __shared__ ef hs[J][128];  // this block's slice of the hi tables
  const int u = blockIdx.x, g = blockIdx.y;
  const size_t lv = size_t(lh + ll);
  const size_t base = size_t(u) << lv;
  const uint32_t nlo = 1u << ll;
  const uint32_t nhi = 1u << lh;
  const uint32_t per = (nhi + MPB_SPLIT - 1) / MPB_SPLIT;
  const uint32_t h0 = g * per, h1 = min(nhi, h0 + per);
  if (per <= 128) {
    for (uint32_t i = threadIdx.x; i < per; i += blockDim.x)
      for (int j = 0; j < J; j++) hs[j][i] = h0 + i < h1 ? hi[size_t(j) * nhi + h0 + i] : ef_zero();
  }
  __syncthreads();
  auto hget = [&](int j, uint32_t vh) -> ef { return per <= 128 ? hs[j][vh - h0] : hi[size_t(j) * nhi + vh]; };
  ef res[J];
  for (int j = 0; j < J; j++) res[j] = ef_zero();
  if (base < t_len) {
    for (uint32_t vlo = threadIdx.x; vlo < nlo; vlo += blockDim.x) {
      EfMacF m[J];
      for (int j = 0; j < J; j++) m[j].init();
      uint32_t vh = h0;
      const bool inside = base + (size_t(h1) << ll) <= t_len;  // no entry of this block is past the table
      for (; vh + 4 <= h1; vh += 4) {  // four loads in flight per thread
        uint32_t t[4];
        if (inside) {
#pragma unroll
          for (int q = 0; q < 4; q++) t[q] = __ldg(T + base + (size_t(vh + q) << ll) + vlo);
        } else {
#pragma unroll
          for (int q = 0; q < 4; q++) {
            size_t idx = base + (size_t(vh + q) << ll) + vlo;
            t[q] = idx < t_len ? T[idx] : 0u;
          }
        }
        if (per <= 128) {
#pragma unroll
          for (int q = 0; q < 4; q++)
#pragma unroll
            for (int j = 0; j < J; j++) m[j].mac(hs[j][vh + q - h0], t[q]);
        } else {
#pragma unroll
          for (int q = 0; q < 4; q++)
#pragma unroll
            for (int j = 0; j < J; j++) m[j].mac(hi[size_t(j) * nhi + vh + q], t[q]);
        }
#pragma unroll
        for (int j = 0; j < J; j++) m[j].flush();
      }
      for (; vh < h1; vh++) {
        size_t idx = base + (size_t(vh) << ll) + vlo;
        uint32_t t = idx < t_len ? T[idx] : 0u;
#pragma unroll
        for (int j = 0; j < J; j++) {
          m[j].mac(hget(j, vh), t);
          m[j].flush();
        }
      }
#pragma unroll
      for (int j = 0; j < J; j++) {
        m[j].flush();
        res[j] = ef_add(res[j], ef_mul(m[j].value(), lo[size_t(j) * nlo + vlo]));
      }
    }
  }
  for (int j = 0; j < J; j++) {
    ef r = block_reduce_ef(res[j], scratch);
    if (threadIdx.x == 0) out[((size_t(j) << lu) + u) * MPB_SPLIT + g] = r;
  }
}

__global__ void k_sum_split(const ef* __restrict__ in, size_t n, ef* __restrict__ out) {
  size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  ef acc = ef_zero();
  for (int g = 0; g < MPB_SPLIT; g++) acc = ef_add(acc, in[i * MPB_SPLIT + g]);
  out[i] = acc;
}

// out[v] = sum_u eqr[u] * T[u * 2^lv + v]; two adjacent v per thread (8-byte loads).
// The same fold on the tensor cores (byte-limb form whose reduction index carries the value's
// limbs): rows v, reduction index (u, a) over the nonzero rows u < U of T and the 4 bytes a of
// T[u, v], columns (n, b) for the 8 coefficients n and the 4 bytes b of M(u, n, a) = the
// Montgomery form of eqr[u]_n 2^(8a). The B fragments come from a table built once per launch
// (k_fold_T_limbs, bfrag[((kk * 4 + b) * 2 + h) * 32 + lane]); A fragments are loaded straight
// from T (lanes of equal t read 8 consecutive v: whole 32-byte sectors). Each warp owns 16 rows
// and all 4 n8 tiles; acc_b < 4U 255^2 < 2^25, sum_b acc_b 2^(8b) < 2^50, one Montgomery
// reduction per coefficient.
constexpr int FT_WARPS = 4;
__global__ void k_fold_T_limbs(const ef* __restrict__ eqr, int U, int Up, uint32_t* __restrict__ bfrag) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;  // (kk, b, h, lane)
  if (idx >= Up / 8 * 256) return;
  const int lane = idx & 31, h = (idx >> 5) & 1, b = (idx >> 6) & 3, kk = idx >> 8;
  const int g = lane >> 2, t = lane & 3;
  const int u = 8 * kk + 4 * h + t;
  const uint32_t w = u < U ? eqr[u].c[g] : 0u;
  uint32_t word = 0;
#pragma unroll
  for (int a = 0; a < 4; a++) {
    const uint32_t m = mul(w, uint32_t(detail::cpow(2, 8 * a + 32)));
    word |= ((m >> (8 * b)) & 0xffu) << (8 * a);
  }
  bfrag[idx] = word;
}
__global__ void __launch_bounds__(FT_WARPS * 32) k_whir_fold_T_mma(const uint32_t* __restrict__ T, size_t t_len,
                                                                   int lv, int U, int Up,
                                                                   const uint32_t* __restrict__ bfrag,
                                                                   ef* __restrict__ out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const size_t nv = size_t(1) << lv;
  const size_t v0 = (size_t(blockIdx.x) * FT_WARPS + warp) * 16;
  if (v0 >= nv) return;  // whole warp
  const size_t va = v0 + g, vb = va + 8;
  auto ld = [&](int u, size_t v) -> uint32_t {
    const size_t i = (size_t(u) << lv) + v;
    return (u < U && v < nv && i < t_len) ? __ldg(T + i) : 0u;
  };
  int acc[4][4];
#pragma unroll
  for (int b = 0; b < 4; b++)
#pragma unroll
    for (int o = 0; o < 4; o++) acc[b][o] = 0;
#pragma unroll 1
  for (int kk = 0; kk < Up / 8; kk++) {
    const int u0 = 8 * kk + t;
    const uint32_t af[4] = {ld(u0, va), ld(u0, vb), ld(u0 + 4, va), ld(u0 + 4, vb)};
    const uint32_t* bp = bfrag + size_t(kk) * 256 + lane;
#pragma unroll
    for (int b = 0; b < 4; b++) mma_u8_16832(acc[b], af, __ldg(bp + (2 * b) * 32), __ldg(bp + (2 * b + 1) * 32));
  }
  uint32_t r[4];
#pragma unroll
  for (int o = 0; o < 4; o++)
    r[o] = redc(uint64_t(uint32_t(acc[0][o])) + (uint64_t(uint32_t(acc[1][o])) << 8) +
                (uint64_t(uint32_t(acc[2][o])) << 16) + (uint64_t(uint32_t(acc[3][o])) << 24));
  // lane (g, t) holds coefficients 2t, 2t + 1 of rows va and vb
  if (va < nv) reinterpret_cast<uint2*>(out + va)[t] = make_uint2(r[0], r[1]);
  if (vb < nv) reinterpret_cast<uint2*>(out + vb)[t] = make_uint2(r[2], r[3]);
}

__global__ void k_whir_fold_T(const uint32_t* __restrict__ T, size_t t_len, int lu, int lv,
                              const ef* __restrict__ eqr_g, ef* __restrict__ out) {
  extern __shared__ ef eqr[];
  const int nu = 1 << lu;
  for (int i = threadIdx.x; i < nu; i += blockDim.x) eqr[i] = eqr_g[i];
  __syncthreads();
  const size_t v = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) * 2;
  if (v >= (size_t(1) << lv)) return;
  EfMacF m0, m1;
  m0.init();
  m1.init();
  const size_t row = size_t(1) << lv;
  for (int u0 = 0; u0 < nu; u0 += 4) {
    const size_t base = (size_t(u0) << lv) + v;
    if (base >= t_len) break;  // the rest of the packed table is zero
    uint2 t[4];
    ef e[4];
    if (u0 + 3 < nu && base + 3 * row + 1 < t_len) {  // the whole group is in range
#pragma unroll
      for (int q = 0; q < 4; q++) {
        t[q] = __ldg(reinterpret_cast<const uint2*>(T + base + q * row));
        e[q] = eqr[u0 + q];
      }
    } else {
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const size_t idx = base + q * row;
        const bool in_u = u0 + q < nu;
        t[q] = make_uint2(in_u && idx < t_len ? T[idx] : 0u, in_u && idx + 1 < t_len ? T[idx + 1] : 0u);
        e[q] = in_u ? eqr[u0 + q] : ef_zero();
      }
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
      m0.mac(e[q], t[q].x);
      m1.mac(e[q], t[q].y);
    }
    m0.flush();
    m1.flush();
  }
  out[v] = m0.value();
  out[v + 1] = m1.value();
}

// w[v] += sum_t coefs[t] * hi_t[v_hi] * lo_t[v_lo]   (base-field points). When a block's
// entries share v_hi (2^ll >= blockDim), a_t = coefs[t] * hi_t[v_hi] is formed once per block
// and each entry accumulates a_t * lo_t[v_lo]; otherwise each term multiplies hi and lo.
__global__ void k_add_eq_terms_f(ef* __restrict__ w, int lh, int ll, int npts, const uint32_t* __restrict__ hi,
                                 const uint32_t* __restrict__ lo, const ef* __restrict__ coefs_g) {
  extern __shared__ ef coefs[];
  const size_t nhi = size_t(1) << lh, nlo = size_t(1) << ll;
  const bool shared_hi = nlo >= blockDim.x;
  const size_t vh_blk = (size_t(blockIdx.x) * blockDim.x) >> ll;
  for (int i = threadIdx.x; i < npts; i += blockDim.x)
    coefs[i] = shared_hi ? ef_mul_f(coefs_g[i], hi[i * nhi + vh_blk]) : coefs_g[i];
  __syncthreads();
  const size_t v = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= (size_t(1) << (lh + ll))) return;
  const size_t vh = v >> ll, vl = v & (nlo - 1);
  EfMacF m;
  m.init_with(w[v]);
  int cnt = 0;
  for (int t = 0; t < npts; t++) {
    const uint32_t l = lo[t * nlo + vl];
    m.mac(coefs[t], shared_hi ? l : mul(hi[t * nhi + vh], l));
    if (++cnt == 4) { m.flush(); cnt = 0; }
  }
  w[v] = m.value();
}

// The same on the tensor cores (byte-limb matrix products): the block's rows share v_hi,
// so B[t][n] = coefficient n of coefs[t] hi_t[v_hi] (its limbs in shared memory,
// bs[(b * 8 + n) * Kp + t]); each warp's 16 rows v_lo read lo_t[v_lo] (consecutive rows are
// consecutive words) and own all 16 limb pairs, so every accumulator position is recombined
// by the lane that holds it.
constexpr int AEQ_WARPS = 8;
constexpr int AEQ_MAX_K = 1024;
__global__ void __launch_bounds__(AEQ_WARPS * 32) k_add_eq_terms_f_mma(ef* __restrict__ w, int lh, int ll, int npts,
                                                                      int Kp, const uint32_t* __restrict__ hi,
                                                                      const uint32_t* __restrict__ lo,
                                                                      const ef* __restrict__ coefs) {
  extern __shared__ __align__(16) uint8_t bs[];
  const uint32_t nhi = 1u << lh, nlo = 1u << ll;
  const uint32_t rows = nlo < AEQ_WARPS * 16 ? nlo : AEQ_WARPS * 16;  // one 16-row tile per warp
  const uint32_t per_vh = nlo / rows;
  const uint32_t vh = blockIdx.x / per_vh, xl0 = (blockIdx.x % per_vh) * rows;
  for (int idx = threadIdx.x; idx < 8 * Kp; idx += blockDim.x) {
    const int n = idx / Kp, t = idx - n * Kp;
    const uint32_t v = t < npts ? mul(coefs[t].c[n], hi[size_t(t) * nhi + vh]) : 0u;
#pragma unroll
    for (int b = 0; b < 4; b++) bs[(b * 8 + n) * Kp + t] = uint8_t(v >> (8 * b));
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  for (uint32_t x0 = xl0 + uint32_t(warp) * 16; x0 < xl0 + rows; x0 += AEQ_WARPS * 16) {  // no barrier in here
    const uint32_t xa = x0 + g, xb = xa + 8;
    int acc[4][4][4];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 4; b++)
#pragma unroll
        for (int q = 0; q < 4; q++) acc[a][b][q] = 0;
    auto ld = [&](int k, uint32_t x) -> uint32_t { return k < npts ? __ldg(lo + size_t(k) * nlo + x) : 0u; };
    // the next step's values are requested before this step's products (two steps in flight)
    auto load_step = [&](int k0, uint4 (&q)[4]) {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int kb0 = k0 + 16 * h + 4 * t;
        q[2 * h] = make_uint4(ld(kb0, xa), ld(kb0 + 1, xa), ld(kb0 + 2, xa), ld(kb0 + 3, xa));
        q[2 * h + 1] = make_uint4(ld(kb0, xb), ld(kb0 + 1, xb), ld(kb0 + 2, xb), ld(kb0 + 3, xb));
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
        const uint32_t* col = reinterpret_cast<const uint32_t*>(bs + (b * 8 + g) * Kp + k0) + t;
        const uint32_t b0 = col[0], b1 = col[4];
#pragma unroll
        for (int a = 0; a < 4; a++) {
          const uint32_t af[4] = {l[0][a], l[1][a], l[2][a], l[3][a]};
          mma_u8_16832(acc[a][b], af, b0, b1);
        }
      }
    }
    // lane (g, t) holds coefficients 2t, 2t + 1 of rows xa (q = 0, 1) and xb (q = 2, 3)
    uint2* pa = reinterpret_cast<uint2*>(w + (size_t(vh) << ll) + xa) + t;
    uint2* pb = reinterpret_cast<uint2*>(w + (size_t(vh) << ll) + xb) + t;
    const uint2 oa = *pa, ob = *pb;
    *pa = make_uint2(add(oa.x, limb_recombine_lane(acc, 0)), add(oa.y, limb_recombine_lane(acc, 1)));
    *pb = make_uint2(add(ob.x, limb_recombine_lane(acc, 2)), add(ob.y, limb_recombine_lane(acc, 3)));
  }
}

// w[v] += sum_t coefs[t] * hi_t[v_hi] * lo_t[v_lo]   (extension-field points)
__global__ void k_add_eq_terms_ef(ef* __restrict__ w, int lh, int ll, int npts, const ef* __restrict__ hi,
                                  const ef* __restrict__ lo, const ef* __restrict__ coefs) {
  const size_t v = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= (size_t(1) << (lh + ll))) return;
  const size_t vh = v >> ll, vl = v & ((size_t(1) << ll) - 1);
  const size_t nhi = size_t(1) << lh, nlo = size_t(1) << ll;
  ef acc = w[v];
  for (int t = 0; t < npts; t++) acc = ef_add(acc, ef_mul(ef_mul(coefs[t], hi[t * nhi + vh]), lo[t * nlo + vl]));
  w[v] = acc;
}

constexpr int WSC_THREADS = 256;
// points per thread: 8 for large tables, fewer for small ones (latency-bound rounds)
int wsc_per_thread(size_t half) { return half >= (size_t(1) << 19) ? 8 : half >= (size_t(1) << 16) ? 2 : 1; }

__global__ void k_whir_sc_eval(const ef* __restrict__ g, const ef* __restrict__ w, size_t half, int per,
                               ef* __restrict__ partial) {
  __shared__ ef scratch[32];
  ef s0 = ef_zero(), s1 = ef_zero(), s2 = ef_zero();
  for (int q = 0; q < per; q++) {
    size_t x = (size_t(blockIdx.x) * per + q) * WSC_THREADS + threadIdx.x;
    if (x < half) {
      ef gl = g[x], gh = g[x + half], wl_ = w[x], wh = w[x + half];
      s0 = ef_add(s0, ef_mul(gl, wl_));
      s1 = ef_add(s1, ef_mul(gh, wh));
      s2 = ef_add(s2, ef_mul(ef_sub(ef_add(gh, gh), gl), ef_sub(ef_add(wh, wh), wl_)));
    }
  }
  s0 = block_reduce_ef(s0, scratch);
  s1 = block_reduce_ef(s1, scratch);
  s2 = block_reduce_ef(s2, scratch);
  if (threadIdx.x == 0) {
    partial[size_t(blockIdx.x) * 3] = s0;
    partial[size_t(blockIdx.x) * 3 + 1] = s1;
    partial[size_t(blockIdx.x) * 3 + 2] = s2;
  }
}

// partial[v_hi] = hi[v_hi] * sum_{v_lo} g[v] * lo[v_lo]  (one block per v_hi)
__global__ void k_mle_eval_ef(const ef* __restrict__ g, int lh, int ll, const ef* __restrict__ hi,
                              const ef* __restrict__ lo, ef* __restrict__ partial) {
  __shared__ ef scratch[32];
  const size_t vh = blockIdx.x;
  const size_t nlo = size_t(1) << ll;
  ef acc = ef_zero();
  for (size_t vl = threadIdx.x; vl < nlo; vl += blockDim.x) acc = ef_add(acc, ef_mul(g[(vh << ll) + vl], lo[vl]));
  acc = block_reduce_ef(acc, scratch);
  if (threadIdx.x == 0) partial[vh] = ef_mul(acc, hi[vh]);
}
}  // namespace

void launch_mle_partial_base(const uint32_t* T, size_t t_len, int lu, int lh, int ll, int J, const ef* hi,
                             const ef* lo, ef* out, cudaStream_t s) {
  // `out` must hold J * 2^lu * (MPB_SPLIT + 1) elements; the split partials go past the
  // first J * 2^lu results.
  ef* tmp = out + (size_t(J) << lu);
  dim3 grid(1u << lu, MPB_SPLIT);
  int threads = (1 << ll) < 256 ? (1 << ll) : 256;
  if (threads < 32) threads = 32;
  if (J == 1) k_mle_partial_base<1><<<grid, threads, 0, s>>>(T, t_len, lu, lh, ll, hi, lo, tmp);
  else if (J == 2) k_mle_partial_base<2><<<grid, threads, 0, s>>>(T, t_len, lu, lh, ll, hi, lo, tmp);
  else throw std::runtime_error("mle_partial_base: J must be 1 or 2");
  WL_LAUNCH_CHECK();
  size_t n = size_t(J) << lu;
  k_sum_split<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(tmp, n, out);
  WL_LAUNCH_CHECK();
}

size_t whir_fold_T_scratch_bytes(int lu) { return size_t(4) * (((size_t(1) << lu) + 7) / 8) * 256; }
void launch_whir_fold_T(const uint32_t* T, size_t t_len, int lu, int lv, const ef* eqr, ef* out, cudaStream_t s,
                        uint32_t* scratch) {
  size_t n = size_t(1) << lv;
  if (lv < 1) throw std::invalid_argument("whir_fold_T: at least 2 entries");
  if (scratch && lv >= 4) {
    const size_t rows_nz = (t_len + n - 1) >> lv;  // rows u of T with a nonzero entry
    const int U = int(std::min<size_t>(size_t(1) << lu, rows_nz)), Up = (U + 7) / 8 * 8;
    if (U > 0) {
      k_fold_T_limbs<<<(Up / 8 * 256 + 255) / 256, 256, 0, s>>>(eqr, U, Up, scratch);
      WL_LAUNCH_CHECK();
      const size_t tiles = n / 16;
      k_whir_fold_T_mma<<<(unsigned)((tiles + FT_WARPS - 1) / FT_WARPS), FT_WARPS * 32, 0, s>>>(T, t_len, lv, U, Up,
                                                                                              scratch, out);
      WL_LAUNCH_CHECK();
      return;
    }
  }
  k_whir_fold_T<<<(unsigned)((n / 2 + 255) / 256), 256, sizeof(ef) << lu, s>>>(T, t_len, lu, lv, eqr, out);
  WL_LAUNCH_CHECK();
}

void launch_add_eq_terms_f(ef* w, int lh, int ll, int npts, const uint32_t* hi, const uint32_t* lo, const ef* coefs,
                           cudaStream_t s) {
  if (!npts) return;
  size_t n = size_t(1) << (lh + ll);
  const int Kp = (npts + 31) / 32 * 32;
  if (ll >= 4 && Kp <= AEQ_MAX_K) {
    const uint32_t rows = (1u << ll) < AEQ_WARPS * 16 ? (1u << ll) : AEQ_WARPS * 16;
    k_add_eq_terms_f_mma<<<(unsigned)(n / rows), AEQ_WARPS * 32, size_t(32) * Kp, s>>>(w, lh, ll, npts, Kp, hi, lo,
                                                                                       coefs);
    WL_LAUNCH_CHECK();
    return;
  }
  k_add_eq_terms_f<<<(unsigned)((n + 255) / 256), 256, sizeof(ef) * npts, s>>>(w, lh, ll, npts, hi, lo, coefs);
  WL_LAUNCH_CHECK();
}
void launch_add_eq_terms_ef(ef* w, int lh, int ll, int npts, const ef* hi, const ef* lo, const ef* coefs,
                            cudaStream_t s) {
  if (!npts) return;
  size_t n = size_t(1) << (lh + ll);
  k_add_eq_terms_ef<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(w, lh, ll, npts, hi, lo, coefs);
  WL_LAUNCH_CHECK();
}
int whir_sc_blocks(size_t half) {
  size_t per = size_t(WSC_THREADS) * wsc_per_thread(half);
  return (int)((half + per - 1) / per);
}
void launch_whir_sc_eval(const ef* g, const ef* w, size_t half, ef* partial, cudaStream_t s) {
  k_whir_sc_eval<<<whir_sc_blocks(half), WSC_THREADS, 0, s>>>(g, w, half, wsc_per_thread(half), partial);
  WL_LAUNCH_CHECK();
}
int mle_ef_blocks(int lh) { return 1 << lh; }
void launch_mle_eval_ef(const ef* g, int lh, int ll, const ef* hi, const ef* lo, ef* partial, cudaStream_t s) {
  int threads = (1 << ll) < 256 ? (1 << ll) : 256;
  if (threads < 32) threads = 32;
  k_mle_eval_ef<<<1u << lh, threads, 0, s>>>(g, lh, ll, hi, lo, partial);
  WL_LAUNCH_CHECK();
}

}  // namespace wl
