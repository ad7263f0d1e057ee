// Host-side launchers for the device kernels. All buffers are device pointers, all
// field values Montgomery form, extension elements `kb::ef` (8 u32, lowest degree first).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "air.cuh"
#include "common.cuh"

namespace wl {

// --------------------------------------------------------------- elementwise / trace
void launch_to_mont(uint32_t* x, size_t n, cudaStream_t s);
void launch_trace_gen(const uint32_t* inputs_canonical, const AirConsts& K, uint32_t* wit, int log_n, cudaStream_t s);

// --------------------------------------------------------------- Reed-Solomon + Merkle
// Source of a commitment: an m-variable multilinear given by its evaluation table.
// Column `col` (< n_cols) of the codeword matrix reads src[(col / elem) * (elem << L) +
// (col % elem) + s * elem] for s < 2^L (L = m - fold), zero beyond `src_len`.
struct LdeSource {
  const uint32_t* src;
  size_t src_len;
  int elem;      // 1: base field, 8: extension field (coordinates are separate columns)
  int L;         // log2 of the column length before the rate expansion
  int rho;       // log2 of the rate expansion
  int n_cols;    // stored columns per row (leading columns; the rest are zero)
};
// Codeword matrix of 2^(L + rho) rows and n_cols (a multiple of 8) columns, tile-major:
// word (tile, row, c) at (tile * 2^(L+rho) + row) * 8 + c.
// Tiles [tile_begin, tile_end) of 8 columns only (default: all); tiles are independent.
// plan (0 .. LDE_PLANS - 1, chosen by the autotuner): the pass split and the persistent
// passes' blocks per SM; every plan writes the same codeword.
constexpr int LDE_PLANS = 6, LDE_PLAN_DEFAULT = 2;
void launch_lde(const LdeSource& in, uint32_t* out, const uint2* twiddles, cudaStream_t s, int tile_begin = 0,
                int tile_end = -1, int plan = LDE_PLAN_DEFAULT);
// Per-stage twiddle table (2^24 - 1 entries): stage t = 1..24 holds (w canonical,
// floor(w 2^32 / p)) for w = w_{2^t}^x, x < 2^(t-1), at offset 2^(t-1) - 1.
constexpr size_t TWIDDLE_ENTRIES = (size_t(1) << 24) - 1;
void launch_twiddles(uint2* tw, cudaStream_t s);
// Merkle tree over the rows of a tile-major LDE matrix (rows of 128 values, the first
// `n_cols` stored): leaf digests (each row Moebius-transformed over the bits [log2(elem), 7) of the
// column index, then PaddingFreeSponge over Poseidon2-24) and 2-to-1 compressions
// (Poseidon2-16), written level by level into `tree` (level l at digest offset
// 2^(LL+1) - 2^(LL+1-l), LL = log2(rows)).
void launch_merkle_tree(const uint32_t* lde, size_t rows, int n_cols, int elem, const kb::P24Consts& p24,
                        const kb::P16Consts& p16, uint32_t* tree, int LL, cudaStream_t s);
// The same leaves one absorption at a time: chunk ch (0..7) reads LDE tiles 2ch and 2ch + 1
// (and, through the Moebius transform, those of the chunks below it); the 8 capacity words of
// every row are carried in cap (8 * rows words) and chunk 7 writes the digests. Then
// launch_merkle_levels builds the compressions.
// rows_choice / plan: the autotuner's pick (leaf rows per block 64, 128 (default) or 256; the
// level width from which compressions run one per thread 2^11, 2^13 (default) or 2^15).
constexpr int LEAF_PLANS = 3, LEAF_PLAN_DEFAULT = 1, MERKLE_PLANS = 3, MERKLE_PLAN_DEFAULT = 1;
void launch_leaf_absorb(const uint32_t* lde, size_t rows, int n_cols, int elem, const kb::P24Consts& p24, int ch,
                        uint32_t* cap, uint32_t* tree, int LL, cudaStream_t s, int rows_choice = LEAF_PLAN_DEFAULT);
// Level 0 of the tree (the leaf digests) only.
void launch_leaf_hash(const uint32_t* lde, size_t rows, int n_cols, int elem, const kb::P24Consts& p24,
                      uint32_t* tree, int LL, cudaStream_t s, int rows_choice = LEAF_PLAN_DEFAULT);
void launch_merkle_levels(uint32_t* tree, int LL, const kb::P16Consts& p16, cudaStream_t s,
                          int plan = MERKLE_PLAN_DEFAULT);
// Gathers rows idx[q] of a tile-major LDE matrix (2^T rows, n_cols <= 128 stored columns) as
// the leaves hash them: 128 values per row (zero beyond n_cols), Moebius-transformed over the
// position bits [log_elem, 7), into out[q * 128 + i]. With mono (128 >> log_elem entries),
// also folded[q] = sum_p row_p mono[p] over the row's base-field values (log_elem 0) or
// extension elements (log_elem 3).
void launch_gather_lde_rows(const uint32_t* lde, int T, const uint64_t* idx, int n_cols, int log_elem, int n,
                            uint32_t* out, const ef* mono, ef* folded, cudaStream_t s);
// Gathers rows of a row-major u32 matrix of the given width (Merkle digests: width 8).
void launch_gather_u32(const uint32_t* src, const uint64_t* idx, int width, int n, uint32_t* out, cudaStream_t s);

// --------------------------------------------------------------- PoW
// Smallest w in [base, base + count) with from_mont(sample) & mask == 0 after observing w.
// The smallest witness in [base, base + count) into *result (UINT32_MAX if none), searched by
// `threads` threads in increasing order with an early stop (any thread count gives the same
// result).
void launch_grind(const kb::P16Consts& p16, const uint32_t* state16, const uint32_t* inbuf, int inlen, int bits,
                  uint32_t base, uint32_t count, uint32_t threads, uint32_t* result, cudaStream_t s);

// --------------------------------------------------------------- eq tables / reductions
void launch_eq_table(const ef* point, int nvars, ef* out, cudaStream_t s);
void launch_eq_table_f(const uint32_t* points, int npts, int nvars, uint32_t* out, cudaStream_t s);
void launch_reduce_partials(const ef* partial, int nblk, int k, ef* out, cudaStream_t s);

// --------------------------------------------------------------- AIR zerocheck
// Round 0 with univariate skip over the top k variables: for the nz points z_0.. given by
// their Lagrange weights lw[z * 2^k + j], the eq-weighted batched constraint over the up
// columns, as partial sums partial[blk * nz + z] of two kernels. launch_zc0_rows writes the
// ZC0_NQ computed cube inputs of every row to q (ZC0_NQ * 2^log_n words) and its
// zc0_row_blocks partial sums (the committed-column term); launch_zc0_eval reads q and writes
// zc0_blocks partial sums (the S-box term). The point sums are the sums over both.
constexpr int ZC0_NQ = 52;
int zc0_blocks(int log_n, int k);
int zc0_row_blocks(int log_n);
void launch_zc0_rows(const uint32_t* wit, int log_n, int k, int nz, const uint32_t* lw, const ef* eq,
                     const ef* alphas, const AirConsts& K, uint32_t* q, ef* partial, ef* arow, cudaStream_t s);
// Round-0 fold of the committed-column combination arow (2^log_n EF, one per row): out[x] =
// sum_j sel[j] arow[j 2^(log_n-k) + x]. The rounds >= 1 carry it as column AIR_W of their
// folded columns: the committed-post terms of every constraint, summed once per point.
void launch_zc0_fold_ef(const ef* arow, int log_n, int k, const ef* sel, ef* out, cudaStream_t s);
void launch_zc0_eval(const uint32_t* wit, const uint32_t* q, int log_n, int k, int nz, const uint32_t* lw,
                     const ef* eq, const ef* alphas, const ef* betas, const AirConsts& K, ef* partial,
                     cudaStream_t s);
void launch_zc0_fold(const uint32_t* wit, int log_n, int k, const ef* sel, ef* out, cudaStream_t s);
int zc_ef_blocks(int m);
// True when the round over m variables runs on the dense kernels (k_zc_full_dense,
// k_zc_partial_dense) rather than one block per point (k_zc_ef).
bool zc_eval_is_dense(int m);
// cols: AIR_W + 1 folded columns (the last one the committed-column combination).
// betas: the 8 full rounds' 16 weights beta_f = MDS^T (alpha_(c0(f)+i))_i, f = 0..7.
void launch_zc_eval_ef(const ef* cols, int m, const ef* eq, const ef* alphas, const ef* betas, const AirConsts& K,
                       ef* partial, cudaStream_t s);
// Folds every column at r; with eq_in, also writes the next round's eq table
// eq_out[x] = eq_in[x] + eq_in[x + eq_half].
void launch_fold_cols(const ef* in, ef* out, int ncols, size_t half, const ef* r, cudaStream_t s,
                      const ef* eq_in = nullptr, ef* eq_out = nullptr, size_t eq_half = 0);
// The same with the challenge passed by value (no device copy of it).
void launch_fold_cols_at(const ef* in, ef* out, int ncols, size_t half, const ef& r, cudaStream_t s,
                         const ef* eq_in = nullptr, ef* eq_out = nullptr, size_t eq_half = 0);
// The same with the challenge in device memory (sampled by a round-finishing kernel).
void launch_fold_cols_dev(const ef* in, ef* out, int ncols, size_t half, const ef* r_dev, cudaStream_t s,
                          const ef* eq_in = nullptr, ef* eq_out = nullptr, size_t eq_half = 0);
// Up/down evaluations of every column at (r0; tail), with eq(tail, .) factored as
// eq_hi (2^(log_n-k-ll) entries) x eq_lo (2^ll entries). out_up / out_down must hold
// AIR_W * (1 + 2^k * 2^(log_n-k-ll)) elements; the first AIR_W are the results.
// With limbs (64 * 2^ll bytes of scratch) and ll >= INNER_MMA_MIN_LL, the segment sums run
// as byte-limb integer matrix products on the tensor cores.
constexpr int INNER_MMA_MIN_LL = 5;
// plan 0 stages the witness tiles with cp.async per thread, plan 1 with bulk copies (the TMA
// engine) completing on mbarriers; plan 1 needs `timeouts`, a device counter of pipeline waits
// that ran out (each wait is bounded; the caller fails the proof when it is not zero).
constexpr int INNER_PLANS = 2;
void launch_inner_sums(const uint32_t* wit, int log_n, int k, int ll, const ef* eq_hi, const ef* eq_lo,
                       const ef* sel, ef* out_up, ef* out_down, uint8_t* limbs, cudaStream_t s, int plan = 0,
                       unsigned* timeouts = nullptr);

// --------------------------------------------------------------- inner phase
void launch_batch_cols(const uint32_t* wit, int log_n, const ef* eqc, ef* out, cudaStream_t s);
int sub_eval_blocks(int log_n, int k);
void launch_sub_evals(const ef* batched, int log_n, int k, const ef* alpha2, const ef* eqt, ef* partial,
                      cudaStream_t s);
void launch_inner_mle(const ef* eqp, int log_n, const ef* alpha2, ef* out, cudaStream_t s);
int prod_blocks(size_t half);
void launch_prod_eval(const ef* a, const ef* b, size_t half, ef* partial, cudaStream_t s);
// Folds the tables a and b at the challenge r (lo + r (hi - lo)).
void launch_fold2_at(const ef* a, const ef* b, ef* oa, ef* ob, size_t half, const ef& r, cudaStream_t s);
void launch_fold2_dev(const ef* a, const ef* b, ef* oa, ef* ob, size_t half, const ef* r_dev, cudaStream_t s);

// --------------------------------------------------------------- fold fused with the next round
// The previous round's fold at its device challenge r_dev fused with this round's sums (each
// table read once per round). Pair form: tables a, b of length 4h fold into na, nb of length
// 2h, and block partials of sum_x na_lo nb_lo (and na_hi nb_hi with 3 sums) and of
// (2 na_hi - na_lo)(2 nb_hi - nb_lo) over x < h go to partial[blk * nsums + z]. The a*b - c
// form folds three columns (4h -> 2h) and the eq table (2h -> h: the leading variable summed
// out) and sums (A B - C) eq at z = 0 and 2. fold_eval_blocks(h) partial rows.
int fold_eval_blocks(size_t h);
// With fin non-null the kernel's last block also finishes the round (kind FIN_PROD for 2 sums,
// FIN_WHIR for 3, FIN_EQSC3 for the a*b - c form).
struct FinArgs;
void launch_pair_fold_eval(int nsums, const ef* a, const ef* b, const ef* r_dev, ef* na, ef* nb, size_t h,
                           ef* partial, const FinArgs* fin, cudaStream_t s);
void launch_abc_fold_eval(const ef* cols, const ef* r_dev, const ef* eq_prev, ef* nc, ef* eq_new, size_t h, ef* partial,
                          const FinArgs* fin, cudaStream_t s);

// --------------------------------------------------------------- a*b - c zerocheck
void launch_abc0_eval(const uint32_t* a, const uint32_t* b, const uint32_t* c, int log_n, int k, int nz,
                      const uint32_t* lw, const ef* eq, ef* partial, cudaStream_t s);
int abc0_blocks(int log_n, int k);
void launch_abc0_fold(const uint32_t* a, const uint32_t* b, const uint32_t* c, int log_n, int k, const ef* sel,
                      ef* out, cudaStream_t s);
void launch_abc_eval_ef(const ef* cols, int m, const ef* eq, ef* partial, cudaStream_t s);

// --------------------------------------------------------------- WHIR
// F_j[u] = sum_v T[u * 2^lv + v] * eq(pt_j, v) for J points given as factored tables
// hi_j (2^lh entries) x lo_j (2^ll entries), lv = lh + ll; T is the zero-padded packed
// witness of `t_len` values. out[j * 2^lu + u].
void launch_mle_partial_base(const uint32_t* T, size_t t_len, int lu, int lh, int ll, int J, const ef* hi,
                             const ef* lo, ef* out, cudaStream_t s);
// The same for one point on the tensor cores (byte-limb matrix products, as for the inner
// sums), writing out[u] for u < 2^lu. Needs mle_partial_scratch_bytes (0: not available for
// these sizes) of scratch; returns false, launching nothing, when it does not apply.
size_t mle_partial_scratch_bytes(int lu, int lh, int ll);
// The batched column (launch_batch_cols) on the tensor cores (byte-limb matrix products),
// with colsum_limb_bytes(AIR_W) bytes of scratch for the limbs of the weights.
size_t colsum_limb_bytes(int K);
void launch_batch_cols_mma(const uint32_t* wit, int log_n, const ef* eqc, ef* out, uint8_t* limbs, cudaStream_t s);
bool launch_mle_partial_mma(const uint32_t* T, size_t t_len, int lu, int lh, int ll, const ef* hi, const ef* lo,
                            ef* out, void* scratch, cudaStream_t s);
// out[v] = sum_u eqr[u] T[u 2^lv + v] (zero past t_len); with scratch
// (whir_fold_T_scratch_bytes(lu)) on the tensor cores.
size_t whir_fold_T_scratch_bytes(int lu);
void launch_whir_fold_T(const uint32_t* T, size_t t_len, int lu, int lv, const ef* eqr, ef* out, cudaStream_t s,
                        uint32_t* scratch = nullptr);
void launch_add_eq_terms_f(ef* w, int lh, int ll, int npts, const uint32_t* hi, const uint32_t* lo, const ef* coefs,
                           cudaStream_t s);
void launch_add_eq_terms_ef(ef* w, int lh, int ll, int npts, const ef* hi, const ef* lo, const ef* coefs,
                            cudaStream_t s);
int whir_sc_blocks(size_t half);
void launch_whir_sc_eval(const ef* g, const ef* w, size_t half, ef* partial, cudaStream_t s);
int mle_ef_blocks(int lh);
void launch_mle_eval_ef(const ef* g, int lh, int ll, const ef* hi, const ef* lo, ef* partial, cudaStream_t s);

// --------------------------------------------------------------- device-side transcript
// The DuplexChallenger<F, Poseidon16, 16, 8> state (Montgomery form), as HostChallenger holds it.
struct DevChallenger {
  uint32_t state[16];
  uint32_t in[8];
  uint32_t out[8];
  int32_t in_len, out_len;
};
// State of a phase of sumcheck rounds run on the device: the challenger, the current claim,
// the zerocheck's eq weight of the folded variables, the proof words appended so far, the
// number of rounds finished (index of the next challenge) and the count of blocks of the
// current round's kernel that have written their partial sums (the last one finishes the round).
struct DevRound {
  DevChallenger ch;
  ef sum;
  ef mmf;
  uint32_t proof_len;
  int32_t round;
  uint32_t arrived;
};
// Constants of the round finish: Poseidon2-16 (Montgomery), the Lagrange bases on the nodes
// 0..2 and 0..3 (basis[0][i][k], basis[1][i][k]: coefficient k of basis polynomial i) and the
// Montgomery forms of 1, 2 and 1/2.
struct FinishConsts {
  kb::P16Consts p16;
  uint32_t basis[2][4][4];
  uint32_t one, two, inv2;
};
// Round kinds: eq-factor rounds with 4 computed points (the AIR zerocheck's rounds >= 1) or 3
// (the a*b - c zerocheck), the product sumcheck (inner sumcheck), the WHIR folding sumcheck.
enum FinKind { FIN_EQSC4 = 0, FIN_EQSC3 = 1, FIN_PROD = 2, FIN_WHIR = 3 };
// Where a round's finish reads and writes, all in device memory: the phase state, the proof
// words (appended at st->proof_len), the challenges (ch_out[st->round]), the constants and, for
// the eq-factor rounds, every round's eq challenge r and its inverse (indexed by st->round).
struct FinArgs {
  DevRound* st;
  uint32_t* proof;
  ef* ch_out;
  const FinishConsts* fc;
  const ef* req;
  const ef* rinv;
};
constexpr int FIN_MAX_THREADS = 256;  // block size of every kernel that finishes a round
// First level of a reduction of nb interleaved rows of k <= 32 partial sums
// (partial[row * k + z]) into at most max_blocks rows in out (coalesced reads, many blocks);
// returns the number of rows written. The finishing kernel (and the host reads) then sum those.
int launch_reduce_wide(const ef* partial, int nb, int k, ef* out, int max_blocks, cudaStream_t s);
// One round's finish on the device (one block): reduces `nb` interleaved rows of the round's
// sums (3 for FIN_EQSC4 and FIN_WHIR, 2 otherwise), writes the round polynomial to the proof,
// absorbs it, samples the challenge and updates the phase state.
void launch_round_finish(int kind, const ef* partial, int nb, const FinArgs& a, cudaStream_t s);
int fin_kind_sums(int kind);

// --------------------------------------------------------------- constraint-program AIRs
// Zerocheck kernels for AIRs given as constraint programs (air_program.h; code, consts: the
// compiled instructions and Montgomery constants in device memory). Round 0: of the W columns
// (2^log_n Montgomery values each) the first P are in pre, the others in wit; lw the nz points' Lagrange weights (nz x 2^k, z =
// 2^k ..); eq the eq table over the rows of the subcube (2^(log_n - k)); partial[b * nz + z] over
// B = prog_zc_blocks(2^(log_n - k)) blocks. launch_prog_fold0 folds the 2W up/down columns over the
// skipped variables with the weights sel (2^k extension values) into out[c * 2^(log_n - k) + x].
// Rounds >= 1: cols holds 2W extension columns of 2^m; sums at the npts points 0, 2, 3, ..
// weighted by eq (2^(m - 1)), partial[b * npts + z] over B = prog_zc_blocks(2^(m - 1)) blocks.
int prog_zc_blocks(size_t rows);
void launch_prog_zc0(const uint32_t* wit, const uint32_t* pre, int P, int log_n, int k, const uint2* code, int n_code,
                     const uint32_t* consts, int nz, const uint32_t* lw, const ef* eq, const ef* alphas, ef* partial,
                     cudaStream_t s);
void launch_prog_fold0(const uint32_t* wit, const uint32_t* pre, int P, int log_n, int k, int W, const ef* sel, ef* out,
                       cudaStream_t s);
void launch_prog_zc_ef(const ef* cols, int m, int W, const uint2* code, int n_code, const uint32_t* consts, int npts,
                       const ef* eq, const ef* alphas, ef* partial, cudaStream_t s);
// The inner phase's batched column over W columns: out[i] = sum_c eqc[c] wit[c 2^log_n + i].
void launch_batch_cols_generic(const uint32_t* wit, int log_n, int W, const ef* eqc, ef* out, cudaStream_t s);

// --------------------------------------------------------------- batched Merkle-path checks
// One opening to check: word offsets (into the concatenated canonical proofs) of its row (128
// values), its path (ll digests, leaf level first) and its root; q is the leaf index.
struct OpeningCheck {
  uint64_t row, path, root;
  uint32_t q;
  int32_t ll;
};
// ok[i] = 1 when opening i's row hashes, through its path, to its root (p24, p16: Montgomery
// constants as in a constants blob).
void launch_check_openings(const uint32_t* words, const OpeningCheck* ops, int n, const kb::P24Consts& p24,
                           const kb::P16Consts& p16, uint8_t* ok, cudaStream_t s);

}  // namespace wl
