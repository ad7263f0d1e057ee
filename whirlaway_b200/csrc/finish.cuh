// Device-side finish of a sumcheck round: the transcript step that follows the round's sums
// (interpolation, absorption into the challenger, the sampled challenge, the next claim). Used
// by the single-block finishing kernels (k_transcript.cu) and by the fold-and-evaluate kernels
// whose last block finishes the round itself (k_sumcheck.cu).
//
// Warp 0 of the block runs a finish with its values spread over the lanes rather than
// repeated in one: the challenger's 16-word state has word i in lanes i and i + 16, an
// extension-field value has coordinate k in lanes k, k + 8, k + 16 and k + 24. A
// Poseidon2-16 permutation then takes about a quarter of the cycles of the one-thread form
// (each partial round's state sum is two warp reductions instead of fifteen modular
// additions and sixteen diagonal products per lane), and an extension-field product about a
// third (each lane forms one coordinate's eight-term dot product).
#pragma once
#include "kernels.h"

namespace wl {
namespace {

constexpr unsigned FIN_FULL = 0xffffffffu;

// Shared-memory part of a finish: the permutation's constants and the round's reduced sums.
// One instance per block (fin_sm), so that the finish code addresses it as shared memory.
struct FinSmem {
  uint32_t rc[8][16];                             // full-round constants: rounds 0-3 initial, 4-7 terminal
  uint32_t ci[kb::P16Consts::RP];                 // partial-round constants
  uint32_t diag[16];                              // internal-layer diagonal V_i (Montgomery form)
  uint32_t basis[2][4][4], one, two, inv2;        // FinishConsts' interpolation constants
  DevRound st;                                    // the phase state on entry
  ef r, rinv;                                     // eq-factor rounds: the round's eq challenge and inverse
  ef red[4];                                      // the round's sums, reduced over the partial rows
  ef tmp[FIN_MAX_THREADS / 32];                   // per-warp partial sums of the reduction
};
__shared__ FinSmem fin_sm;

// The challenger, spread over warp 0: state word (lane & 15), pending input (lane & 7),
// squeezed output (lane & 7); the lengths are the same in every lane.
struct FinCh {
  uint32_t st, in, out;
  int in_len, out_len;
};

__device__ __forceinline__ int fin_lane() { return threadIdx.x & 31; }

// Everything the finish reads, into fin_sm, by every thread of the block at once (the loads
// are independent, so their latencies overlap; warp 0 then reads shared memory only). A block
// barrier must follow before warp 0 uses fin_sm.
__device__ __forceinline__ void fin_load(int kind, const FinArgs& a) {
  constexpr int RP = kb::P16Consts::RP;
  constexpr int NST = int(sizeof(DevRound) / 4);
  constexpr int A = 128, B = A + RP, C = B + 16, D = C + 32, E = D + NST, F = E + 16;
  const FinishConsts* __restrict__ fc = a.fc;
  const bool eq = kind == FIN_EQSC4 || kind == FIN_EQSC3;
  for (int t = threadIdx.x; t < F; t += blockDim.x) {
    if (t < A) {
      fin_sm.rc[t >> 4][t & 15] = (t >> 4) < 4 ? fc->p16.ext_init[t] : fc->p16.ext_term[t - 64];
    } else if (t < B) {
      fin_sm.ci[t - A] = fc->p16.internal[t - A];
    } else if (t < C) {
      fin_sm.diag[t - B] = kb::p2_diag<16>(t - B);
    } else if (t < D) {
      (&fin_sm.basis[0][0][0])[t - C] = (&fc->basis[0][0][0])[t - C];
    } else if (t < E) {
      reinterpret_cast<uint32_t*>(&fin_sm.st)[t - D] = reinterpret_cast<const uint32_t*>(a.st)[t - D];
    } else if (eq) {
      const int q = t - E, round = a.st->round;
      if (q < 8)
        fin_sm.r.c[q] = a.req[round].c[q];
      else
        fin_sm.rinv.c[q - 8] = a.rinv[round].c[q - 8];
    }
  }
  if (threadIdx.x == 0) {
    fin_sm.one = fc->one;
    fin_sm.two = fc->two;
    fin_sm.inv2 = fc->inv2;
  }
}

__device__ __forceinline__ FinCh fin_ch_load(const DevChallenger& c) {
  const int l = fin_lane();
  FinCh f;
  f.st = c.state[l & 15];
  f.in = c.in[l & 7];
  f.out = c.out[l & 7];
  f.in_len = c.in_len;
  f.out_len = c.out_len;
  return f;
}
__device__ __forceinline__ void fin_ch_store(DevChallenger& c, const FinCh& f) {
  const int l = fin_lane();
  if (l < 16) c.state[l] = f.st;
  if (l < 8) {
    c.in[l] = f.in;
    c.out[l] = f.out;
  }
  if (l == 0) {
    c.in_len = f.in_len;
    c.out_len = f.out_len;
  }
}

// External layer across the 16 lanes of a half-warp: row i of circ(2, 3, 1, 1) within the
// 4-word chunk, plus the sum of that position over the four chunks (gathered in one step).
__device__ __forceinline__ uint32_t fin_m4(uint32_t a, int i) {
  const int base = i & ~3;
  const uint32_t b = __shfl_sync(FIN_FULL, a, base | ((i + 1) & 3), 16);
  const uint32_t c = __shfl_sync(FIN_FULL, a, base | ((i + 2) & 3), 16);
  const uint32_t d = __shfl_sync(FIN_FULL, a, base | ((i + 3) & 3), 16);
  const uint32_t y = kb::add(kb::add(kb::add(a, b), kb::add(c, d)), kb::add(a, kb::dbl(b)));
  const uint32_t y4 = __shfl_xor_sync(FIN_FULL, y, 4, 16), y8 = __shfl_xor_sync(FIN_FULL, y, 8, 16);
  const uint32_t y12 = __shfl_xor_sync(FIN_FULL, y, 12, 16);
  return kb::add(kb::add(kb::add(y, y4), kb::add(y8, y12)), y);
}

// Poseidon2-16 (Montgomery form; the values of kb::p2_permute<16>) of the state whose word
// (lane & 15) is v. Partial rounds: word 0 is carried in every lane (a), the other words in
// their lanes, kept below 2p between rounds (the diagonal product accepts them and the sum
// below stays in range); the sum of words 1..15 is two warp reductions of their 16-bit halves
// (each total below 2^20), recombined with 2^31 = 2^24 - 1 (mod p) to below 2p, and does not
// wait for the S-box. Measured on the B200 in one warp: 5.2 K cycles per permutation, against
// 23 K with the whole state in every lane and 7.3 K for a form whose partial rounds carry
// only the S-box chain (more instructions per round than the warp hides).
__device__ __noinline__ uint32_t fin_perm(uint32_t v) {
  const int lane = fin_lane(), i = lane & 15;
  const uint32_t d = fin_sm.diag[i];
  v = fin_m4(v, i);
#pragma unroll 1
  for (int r = 0; r < 4; r++) v = fin_m4(kb::cube(kb::add(v, fin_sm.rc[r][i])), i);
  uint32_t a = __shfl_sync(FIN_FULL, v, 0);
  const bool contrib = lane >= 1 && lane < 16;
#pragma unroll 1
  for (int r = 0; r < kb::P16Consts::RP; r++) {
    const uint32_t x0 = kb::cube(kb::add(a, fin_sm.ci[r]));
    const uint32_t w = contrib ? v : 0u;
    const uint32_t lo = __reduce_add_sync(FIN_FULL, w & 0xffffu), hi = __reduce_add_sync(FIN_FULL, w >> 16);
    uint32_t t = ((hi & 0x7fffu) << 16) + (hi >> 15) * 0xffffffu + lo;  // below 2^31 + 2^29 + 2^20 < 2p
    t = kb::umin(t, t - kb::P);
    const uint32_t S = kb::add(t, x0);
    a = kb::sub(S, kb::dbl(x0));  // V_0 = -2
    v = kb::mul(v, d) + S;        // below 2p
  }
  v = i == 0 ? a : kb::umin(v, v - kb::P);
#pragma unroll 1
  for (int r = 4; r < 8; r++) v = fin_m4(kb::cube(kb::add(v, fin_sm.rc[r][i])), i);
  return v;
}

// Duplexing: the pending inputs overwrite the first in_len words of the state, which is
// permuted; the rate part becomes the output.
__device__ __forceinline__ void fin_duplex(FinCh& c) {
  const int lane = fin_lane(), i = lane & 15;
  c.st = fin_perm((i < 8 && i < c.in_len) ? c.in : c.st);
  c.out = __shfl_sync(FIN_FULL, c.st, lane & 7);
  c.in_len = 0;
  c.out_len = 8;
}

// Transcript::add_ext of the value x (coordinate lane & 7): the eight words go to
// proof[plen..] and into the challenger, one observation each. With L words already pending,
// the first 8 - L fill the rate and duplex, the other L are left pending (and the output is
// then empty, as any observation leaves it).
__device__ __forceinline__ void fin_observe_ext(FinCh& c, uint32_t x, uint32_t* __restrict__ proof, uint32_t plen) {
  const int lane = fin_lane(), k = lane & 7;
  if (lane < 8) proof[plen + lane] = x;
  const int L = c.in_len;
  const uint32_t first = __shfl_sync(FIN_FULL, x, (k - L) & 7);  // lane k >= L: word k - L
  c.in = k >= L ? first : c.in;
  c.in_len = 8;
  fin_duplex(c);
  if (L) {
    const uint32_t second = __shfl_sync(FIN_FULL, x, (k + 8 - L) & 7);  // lane k < L: word k + 8 - L
    c.in = k < L ? second : c.in;
    c.in_len = L;
    c.out_len = 0;
  }
}

// Transcript::sample_ext: eight samples, each popped from the end of the output (duplexing
// first when inputs are pending or the output is empty); sample k is coordinate k.
__device__ __forceinline__ uint32_t fin_sample_ext(FinCh& c) {
  const int k = fin_lane() & 7;
  if (c.in_len || !c.out_len) fin_duplex(c);
  const int O = c.out_len;
  const uint32_t a = __shfl_sync(FIN_FULL, c.out, (O - 1 - k) & 7);  // sample k < O: out[O - 1 - k]
  if (O == 8) {
    c.out_len = 0;
    return a;
  }
  fin_duplex(c);  // the output ran out after O samples
  const uint32_t b = __shfl_sync(FIN_FULL, c.out, (7 - (k - O)) & 7);  // sample k >= O: out[7 - (k - O)]
  c.out_len = O;
  return k < O ? a : b;
}

// Extension-field product in F[X]/(X^8 - 3), coordinate (lane & 7) of a * b within each group
// of eight lanes: the dot product of a with (b_k, ..., b_0, 3 b_7, ..., 3 b_{k+1}) in two lazy
// halves of four terms. Inlined: as a call it measured twice the cycles (the call saves and
// restores the caller's live registers).
__device__ __forceinline__ uint32_t fin_mul(uint32_t a, uint32_t b) {
  const int lane = fin_lane(), k = lane & 7, g = lane & 24;
  const uint32_t b3 = kb::add(kb::dbl(b), b);
  uint64_t s0 = 0, s1 = 0;
#pragma unroll
  for (int t = 0; t < 8; t++) {
    const uint32_t at = __shfl_sync(FIN_FULL, a, g | t);
    const uint32_t x = __shfl_sync(FIN_FULL, b, g | ((k - t) & 7)), x3 = __shfl_sync(FIN_FULL, b3, g | ((k - t) & 7));
    const uint32_t bb = t <= k ? x : x3;
    if (t < 4)
      s0 += kb::wmul(at, bb);
    else
      s1 += kb::wmul(at, bb);
  }
  return kb::add(kb::redc(s0), kb::redc(s1));
}
// The base-field constant c as an extension coordinate: c at coordinate 0, zero elsewhere.
__device__ __forceinline__ uint32_t fin_base(uint32_t c) { return (fin_lane() & 7) == 0 ? c : 0u; }
// Coordinate (lane & 7) of an extension element in shared memory.
__device__ __forceinline__ uint32_t fin_coord(const ef& e) { return e.c[fin_lane() & 7]; }

// An extension element written by another block, read past L1.
__device__ __forceinline__ ef fin_ldcg(const ef* p) {
  const uint4* q = reinterpret_cast<const uint4*>(p);
  const uint4 u = __ldcg(q), v = __ldcg(q + 1);
  ef e;
  e.c[0] = u.x, e.c[1] = u.y, e.c[2] = u.z, e.c[3] = u.w;
  e.c[4] = v.x, e.c[5] = v.y, e.c[6] = v.z, e.c[7] = v.w;
  return e;
}
// Sum over `nb` rows of `nsum` interleaved extension sums (partial[row * nsum + z], written by
// other blocks of this grid or an earlier one) into fin_sm.red[z]. Every thread of the block
// calls it (blockDim.x a multiple of 32, at least 32 nsum); warp w sums rows of sum w % nsum,
// then warp 0 adds the warps' totals; fin_sm.red is valid in warp 0 on return.
__device__ void fin_reduce_rows(const ef* __restrict__ partial, int nb, int nsum) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int z = w % nsum, wz = w / nsum, nwz = (nw - 1 - z) / nsum + 1;  // warps wz of the nwz on sum z
  ef acc = kb::ef_zero();
#pragma unroll 4
  for (int row = wz * 32 + lane; row < nb; row += nwz * 32) acc = kb::ef_add(acc, fin_ldcg(partial + size_t(row) * nsum + z));
  acc = warp_reduce_ef(acc);
  if (lane == 0) fin_sm.tmp[w] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    const int zz = lane >> 3, k = lane & 7;
    if (zz < nsum) {
      uint32_t s = 0;
      for (int u = zz; u < nw; u += nsum) s = kb::add(s, fin_sm.tmp[u].c[k]);
      fin_sm.red[zz].c[k] = s;
    }
    __syncwarp();
  }
}

// The round's finish proper (warp 0, every lane). The state st (challenger, claim, eq weight,
// proof length, round) is read from and written back to a.st; the round polynomial goes to
// a.proof, the challenge to a.ch_out[round].
//
// Round of a sumcheck with an eq factor (the AIR zerocheck's rounds >= 1: NPTS = 4; the
// a*b - c zerocheck: NPTS = 3): the sums are at z = 0, 2, .., NPTS - 1, weighted by the eq
// factor mmf of the variables already folded; the value at 1 follows from the claim,
// e1 = (sum - e0 (1 - r)) / r, with r the eq challenge of the current variable. The round
// polynomial is the interpolation on 0..NPTS-1 times (1 - r) + (2r - 1) X: NPTS + 1
// coefficients.
template <int NPTS>
__device__ __noinline__ void fin_round_eqsc(const FinArgs& a) {
  const int lane = fin_lane();
  DevRound* stp = a.st;
  const int round = fin_sm.st.round;
  uint32_t plen = fin_sm.st.proof_len;
  FinCh c = fin_ch_load(fin_sm.st.ch);
  const uint32_t sum = fin_coord(fin_sm.st.sum), mmf = fin_coord(fin_sm.st.mmf);
  const uint32_t r = fin_coord(fin_sm.r), rinv = fin_coord(fin_sm.rinv);
  const uint32_t one = fin_base(kb::R_MOD_P);
  const uint32_t omr = kb::sub(one, r), lin = kb::sub(kb::add(r, r), one);
  uint32_t e[NPTS];
  e[0] = fin_mul(fin_sm.red[0].c[lane & 7], mmf);
#pragma unroll
  for (int i = 2; i < NPTS; i++) e[i] = fin_mul(fin_sm.red[i - 1].c[lane & 7], mmf);
  e[1] = fin_mul(kb::sub(sum, fin_mul(e[0], omr)), rinv);
  uint32_t q[NPTS];
#pragma unroll
  for (int k = 0; k < NPTS; k++) {
    q[k] = 0;
#pragma unroll
    for (int i = 0; i < NPTS; i++) q[k] = kb::add(q[k], kb::mul(e[i], fin_sm.basis[NPTS - 3][i][k]));
  }
  uint32_t p[NPTS + 1];
#pragma unroll
  for (int k = 0; k <= NPTS; k++) {
    uint32_t v = k < NPTS ? fin_mul(q[k], omr) : 0u;
    if (k > 0) v = kb::add(v, fin_mul(q[k - 1], lin));
    p[k] = v;
  }
#pragma unroll
  for (int k = 0; k <= NPTS; k++) {
    fin_observe_ext(c, p[k], a.proof, plen);
    plen += 8;
  }
  const uint32_t ch = fin_sample_ext(c);
  uint32_t s = p[NPTS];
#pragma unroll
  for (int k = NPTS - 1; k >= 0; k--) s = kb::add(fin_mul(s, ch), p[k]);
  const uint32_t m2 = fin_mul(kb::add(fin_mul(omr, kb::sub(one, ch)), fin_mul(r, ch)), mmf);
  __syncwarp();
  fin_ch_store(stp->ch, c);
  if (lane < 8) {
    stp->sum.c[lane] = s;
    stp->mmf.c[lane] = m2;
    a.ch_out[round].c[lane] = ch;
  }
  if (lane == 0) {
    stp->proof_len = plen;
    stp->round = round + 1;
  }
}

// Round of the product sumcheck (the inner sumcheck): sums at 0 and 2, the value at 1 from the
// claim; the round polynomial (3 coefficients) interpolates 0, 1, 2.
__device__ __noinline__ void fin_round_prod(const FinArgs& a) {
  const int lane = fin_lane();
  DevRound* stp = a.st;
  const int round = fin_sm.st.round;
  uint32_t plen = fin_sm.st.proof_len;
  FinCh c = fin_ch_load(fin_sm.st.ch);
  const uint32_t y0 = fin_sm.red[0].c[lane & 7], y2 = fin_sm.red[1].c[lane & 7];
  const uint32_t y1 = kb::sub(fin_coord(fin_sm.st.sum), y0);
  uint32_t p[3];
#pragma unroll
  for (int k = 0; k < 3; k++)
    p[k] = kb::add(kb::add(kb::mul(y0, fin_sm.basis[0][0][k]), kb::mul(y1, fin_sm.basis[0][1][k])),
                   kb::mul(y2, fin_sm.basis[0][2][k]));
#pragma unroll
  for (int k = 0; k < 3; k++) {
    fin_observe_ext(c, p[k], a.proof, plen);
    plen += 8;
  }
  const uint32_t ch = fin_sample_ext(c);
  const uint32_t s = kb::add(fin_mul(kb::add(fin_mul(p[2], ch), p[1]), ch), p[0]);
  __syncwarp();
  fin_ch_store(stp->ch, c);
  if (lane < 8) {
    stp->sum.c[lane] = s;
    a.ch_out[round].c[lane] = ch;
  }
  if (lane == 0) {
    stp->proof_len = plen;
    stp->round = round + 1;
  }
}

// Round of the WHIR folding sumcheck: h(0), h(1), h(2) go to the proof as they are; the next
// claim is h(r) by quadratic interpolation on 0, 1, 2:
// h(r) = h0 (r-1)(r-2)/2 - h1 r (r-2) + h2 r (r-1)/2.
__device__ __noinline__ void fin_round_whir(const FinArgs& a) {
  const int lane = fin_lane();
  DevRound* stp = a.st;
  const int round = fin_sm.st.round;
  uint32_t plen = fin_sm.st.proof_len;
  FinCh c = fin_ch_load(fin_sm.st.ch);
  uint32_t h[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    h[k] = fin_sm.red[k].c[lane & 7];
    fin_observe_ext(c, h[k], a.proof, plen);
    plen += 8;
  }
  const uint32_t r = fin_sample_ext(c);
  const uint32_t rm1 = kb::sub(r, fin_base(fin_sm.one)), rm2 = kb::sub(r, fin_base(fin_sm.two));
  const uint32_t t0 = kb::mul(fin_mul(fin_mul(h[0], rm1), rm2), fin_sm.inv2);
  const uint32_t t1 = fin_mul(fin_mul(h[1], r), rm2);
  const uint32_t t2 = kb::mul(fin_mul(fin_mul(h[2], r), rm1), fin_sm.inv2);
  const uint32_t s = kb::add(kb::sub(t0, t1), t2);
  __syncwarp();
  fin_ch_store(stp->ch, c);
  if (lane < 8) {
    stp->sum.c[lane] = s;
    a.ch_out[round].c[lane] = r;
  }
  if (lane == 0) {
    stp->proof_len = plen;
    stp->round = round + 1;
  }
}

__device__ __forceinline__ int fin_kind_sums_dev(int kind) { return kind == FIN_EQSC4 || kind == FIN_WHIR ? 3 : 2; }

// Dispatch on the round kind (warp 0 only).
__device__ __forceinline__ void fin_round(int kind, const FinArgs& a) {
  if (kind == FIN_EQSC4)
    fin_round_eqsc<4>(a);
  else if (kind == FIN_EQSC3)
    fin_round_eqsc<3>(a);
  else if (kind == FIN_PROD)
    fin_round_prod(a);
  else
    fin_round_whir(a);
}

// Epilogue of a kernel whose blocks each wrote one row of `nsum` partial sums (thread 0 of the
// block, before the call): the block that arrives last reduces all gridDim.x rows and finishes
// the round. Every thread of every block calls it, after its own stores.
__device__ __forceinline__ void fin_last_block(int kind, const FinArgs& a, const ef* __restrict__ partial, int nsum) {
  __shared__ int last;
  __syncthreads();  // thread 0 has written this block's row
  if (threadIdx.x == 0) {
    __threadfence();  // the row before the count
    last = atomicAdd(&a.st->arrived, 1u) == gridDim.x - 1;
    if (last) __threadfence();  // every other row is visible to this block's reads
  }
  __syncthreads();
  if (!last) return;
  fin_load(kind, a);
  fin_reduce_rows(partial, gridDim.x, nsum);
  __syncthreads();
  if (threadIdx.x < 32) {
    fin_round(kind, a);
    if (threadIdx.x == 0) a.st->arrived = 0;  // for the next round's grid
  }
}

}  // namespace
}  // namespace wl
