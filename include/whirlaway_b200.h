/* C ABI of the B200 Whirlaway prover path (Poseidon2-KoalaBear AIR).
 *
 * The reference exposes this path as a Rust library API (no FFI):
 *   AirTable::prove   crates/air/src/prove.rs:49-66   (witness by value, proof into a
 *                     caller-owned ProverState, read back via proof_data())
 *   AirTable::verify  crates/air/src/verify.rs:55-69
 *   AirSettings       crates/air/src/lib.rs:13-41 (+ WHIR_POW_BITS, lib.rs:9)
 *   sumcheck::prove   crates/sumcheck/src/prove.rs:22-35
 *   prove_poseidon2   src/examples/poseidon2.rs:85-200 (workload: constants, inputs, trace)
 * Each entry point below names the reference interface it replaces.
 *
 * Conventions
 *  - Field values cross the ABI as canonical little-endian u32 (KoalaBear, p = 2^31 - 2^24 + 1).
 *    Extension elements are 8 consecutive u32, lowest degree first.
 *  - A proof is the reference's proof_data: a sequence of field elements.
 *  - Every function returns a wl_status; nothing aborts across the boundary. The message of
 *    the last failure on a context is available from wl_last_error.
 *  - A context is single-owner: calls on one context must not overlap.
 */
#ifndef WHIRLAWAY_B200_H
#define WHIRLAWAY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  WL_OK = 0,
  WL_E_INVALID_ARG = 1,
  WL_E_CUDA = 2,
  WL_E_OOM = 3,
  WL_E_BUFFER_TOO_SMALL = 4,
  WL_E_INTERNAL = 5,
  WL_E_BUDGET = 6,
  WL_E_SCRATCH_LIMIT = 7, /* problem larger than the fixed scratch of the allocation-free entry point */
  /* verifier outcomes, mirroring AirVerifError (crates/air/src/verify.rs:26-34) */
  WL_E_INVALID_PCS_COMMITMENT = 11,
  WL_E_INVALID_PCS_OPENING = 12,
  WL_E_FS = 13,
  WL_E_SUMCHECK = 14,
  WL_E_BOUNDARY = 15,
  WL_E_SUM_MISMATCH = 16
} wl_status;

/* AirSettings (crates/air/src/lib.rs:13-41) with the folding factor
 * ConstantFromSecondRound(fold_first, fold_rest) and WHIR_POW_BITS (lib.rs:9).
 * Soundness is CapacityBound. Defaults: {128, 1, 7, 4, 4, 5, 16} (src/main.rs:13-24). */
typedef struct {
  int32_t security_bits;
  int32_t log_inv_rate;
  int32_t fold_first;
  int32_t fold_rest;
  int32_t univariate_skips;
  int32_t rs_domain_initial_reduction;
  int32_t whir_pow_bits;
} wl_air_settings;

typedef struct wl_ctx wl_ctx;
typedef struct wl_witness wl_witness;

/* Number of AIR columns (165) and of u32 in a constants blob (AIR round constants 148,
 * Poseidon16 148, Poseidon24 215; each in the order beginning/initial, partial/terminal...). */
int32_t wl_air_columns(void);
int32_t wl_constants_len(void);
void wl_default_settings(wl_air_settings* out);

/* Context on one CUDA device. hbm_budget_bytes bounds the device memory a context admits
 * for serving (0: no bound). */
wl_status wl_ctx_create(int32_t device, uint64_t hbm_budget_bytes, wl_ctx** out);
void wl_ctx_destroy(wl_ctx* ctx);
const char* wl_last_error(const wl_ctx* ctx);

/* Workload of src/examples/poseidon2.rs:104-151 on the host: one StdRng(seed 0) stream
 * gives the AIR round constants, then 16 * 2^log_n inputs (row-major), then the Poseidon16
 * and Poseidon24 constants. With input_seed >= 0 the constants come from that stream with
 * the inputs skipped and the inputs from StdRng::seed_from_u64(input_seed).
 * constants_out: wl_constants_len() u32; inputs_out: 16 << log_n u32 (may be NULL). */
wl_status wl_generate_workload(int32_t log_n, int64_t input_seed, uint32_t* constants_out, uint32_t* inputs_out);

/* Device-resident witness (165 columns of 2^log_n values, column-major).
 * wl_witness_generate replaces generate_trace_rows(...).transpose() (poseidon2.rs:122-131)
 * with a GPU trace generator; wl_witness_upload takes the reference's
 * Vec<EvaluationsList<F>> layout from host memory. */
wl_status wl_witness_upload(wl_ctx* ctx, int32_t log_n, const uint32_t* witness_colmajor, wl_witness** out);
wl_status wl_witness_generate(wl_ctx* ctx, const uint32_t* constants, int32_t log_n, const uint32_t* inputs,
                              wl_witness** out);
wl_status wl_witness_download(wl_ctx* ctx, const wl_witness* w, uint32_t* witness_colmajor);
void wl_witness_free(wl_ctx* ctx, wl_witness* w);

/* Upper bound of the proof length (u32 elements) for log_n. */
wl_status wl_proof_len_bound(const wl_air_settings* settings, int32_t log_n, size_t* out);

/* AirTable::prove (crates/air/src/prove.rs:49-66) with the WHIR parameters, domain separator
 * and challenger set up as in poseidon2.rs:155-163. The witness is a host buffer of 165
 * columns of 2^log_n values (column-major). proof_out receives proof_data; *proof_len is its
 * capacity on entry and the length on return (WL_E_BUFFER_TOO_SMALL if short).
 * timings_ms (may be NULL): commit, zerocheck, inner, whir, total. */
wl_status wl_prove(wl_ctx* ctx, const wl_air_settings* settings, const uint32_t* constants, int32_t log_n,
                   const uint32_t* witness_colmajor, uint32_t* proof_out, size_t* proof_len, double* timings_ms);
/* Same, with a device-resident witness. */
wl_status wl_prove_witness(wl_ctx* ctx, const wl_air_settings* settings, const uint32_t* constants,
                           const wl_witness* w, uint32_t* proof_out, size_t* proof_len, double* timings_ms);

/* An AIR beyond the built-in Poseidon2 one, given as a constraint program. It replaces the
 * reference's AirTable over an arbitrary p3-air Air (crates/air/src/table.rs:15-60,
 * crates/air/src/prove.rs:49-226, crates/air/src/verify.rs:55-249). There are n_columns witness
 * columns, and the constraints are evaluated on every row's up values (the row; the last row
 * repeats the one before it) and down values (the next row; the last row repeats itself), as
 * crates/air/src/utils.rs:140-160 builds them.
 * `ops` holds n_ops instructions of three int32 (op, a, b); instruction i computes value v_i:
 *   WL_AIR_UP c, WL_AIR_DOWN c    column c's up / down value (c < n_columns)
 *   WL_AIR_CONST j                consts[j] (canonical, j < n_consts)
 *   WL_AIR_ADD, _SUB, _MUL a b    v_a op v_b (a, b < i)
 *   WL_AIR_EMIT a                 the next constraint is v_a (v_i = v_a)
 * The EMITs, in order, are the n_constraints constraints, batched as sum_i alpha^i C_i.
 * constraint_degree (1..3) bounds every constraint's degree. At most 64 values may be live at
 * once (the device interpreter's register file); n_columns <= 32767. The first n_preprocessed
 * columns are preprocessed (AirTable::preprocessed_columns, crates/air/src/table.rs:19): fixed
 * by the AIR, given with the program, in the zerocheck but not committed; the verifier
 * evaluates them itself (crates/air/src/verify.rs:119-135). */
enum { WL_AIR_UP = 0, WL_AIR_DOWN = 1, WL_AIR_CONST = 2, WL_AIR_ADD = 3, WL_AIR_SUB = 4, WL_AIR_MUL = 5,
       WL_AIR_EMIT = 6 };
typedef struct {
  int32_t n_columns;
  int32_t n_constraints;
  int32_t constraint_degree;
  int32_t n_ops;
  const int32_t* ops;
  int32_t n_consts;
  const uint32_t* consts;
  int32_t n_preprocessed;       /* the first n_preprocessed columns are preprocessed (may be 0) */
  const uint32_t* preprocessed; /* their values: n_preprocessed x 2^log_n, canonical, column-major */
} wl_air_program;
/* Proves the program's AIR for a host witness (the n_columns - n_preprocessed witness columns,
 * each 2^log_n canonical values, column-major). hash_constants: Poseidon16 (148) | Poseidon24 (215) constants, as in a
 * constants blob after its AIR part. No reference counterpart beyond AirTable::prove. */
wl_status wl_prove_program(wl_ctx* ctx, const wl_air_settings* settings, const uint32_t* hash_constants,
                           const wl_air_program* program, int32_t log_n, const uint32_t* witness_colmajor,
                           uint32_t* proof_out, size_t* proof_len);
/* Verifies such a proof on the host (AirTable::verify); returns WL_OK or the verifier's error. */
wl_status wl_verify_program(const wl_air_settings* settings, const uint32_t* hash_constants,
                            const wl_air_program* program, int32_t log_n, const uint32_t* proof, size_t proof_len);
/* Upper bound of the proof length (u32 words) of wl_prove_program. */
wl_status wl_program_proof_len_bound(const wl_air_settings* settings, const wl_air_program* program, int32_t log_n,
                                     size_t* out);

/* Batch of independent proofs (each with its own witness and transcript), run back to back
 * on the context's stream; proofs are written at proof_out + i * stride. */
wl_status wl_prove_batch(wl_ctx* ctx, const wl_air_settings* settings, const uint32_t* constants, int32_t n,
                         const wl_witness* const* witnesses, uint32_t* proof_out, size_t stride, size_t* proof_lens);

/* sumcheck::prove (crates/sumcheck/src/prove.rs:22-35) for the zerocheck of
 * eq(r, x) * (a(x) * b(x) - c(x)) with a univariate skip of `skips` variables; r is sampled
 * from a fresh challenger on Poseidon16 (p16_constants: 148 u32), the three final folded
 * values are appended. a, b, c: host arrays of 2^log_n. round_ms (may be NULL) receives
 * log_n - skips + 1 per-round device times. */
wl_status wl_sumcheck_abc_prove(wl_ctx* ctx, const uint32_t* p16_constants, int32_t log_n, int32_t skips,
                                const uint32_t* a, const uint32_t* b, const uint32_t* c, uint32_t* proof_out,
                                size_t* proof_len, float* round_ms);
/* Same with device-resident inputs (canonical u32 device pointers, left unchanged). */
wl_status wl_sumcheck_abc_prove_device(wl_ctx* ctx, const uint32_t* p16_constants, int32_t log_n, int32_t skips,
                                       const uint32_t* a_dev, const uint32_t* b_dev, const uint32_t* c_dev,
                                       uint32_t* proof_out, size_t* proof_len, float* round_ms);

/* AirTable::verify (crates/air/src/verify.rs:55-249) on the host CPU: no context, no device
 * (the Merkle paths of each round's queries are checked on up to 16 host threads).
 * Checks proof_data (canonical u32 words) against the settings, the constants blob and log_n.
 * WL_OK when the proof is accepted; otherwise the AirVerifError outcome of the first failed
 * check (WL_E_INVALID_PCS_COMMITMENT, WL_E_INVALID_PCS_OPENING, WL_E_FS, WL_E_SUMCHECK,
 * WL_E_SUM_MISMATCH), or WL_E_INVALID_ARG for bad arguments or a word that is not a
 * canonical field element. */
wl_status wl_verify(const wl_air_settings* settings, const uint32_t* constants, int32_t log_n,
                    const uint32_t* proof, size_t proof_len);
/* wl_verify over n proofs on `threads` host threads (<= 0: all hardware threads); proof i has
 * log_ns[i] rows and its outcome goes to statuses[i]. Returns WL_OK when every proof was
 * checked (whatever the outcomes), else the argument error. */
wl_status wl_verify_batch(const wl_air_settings* settings, const uint32_t* constants, int32_t n,
                          const int32_t* log_ns, const uint32_t* const* proofs, const size_t* proof_lens,
                          int32_t threads, int32_t* statuses);

/* wl_verify_batch with the Merkle paths checked on the context's GPU: each proof's transcript
 * is replayed on host threads (one proof per thread, `threads` as for wl_verify_batch) with its
 * Merkle openings listed instead of hashed, then every opening of every proof (the leaf sponge
 * over the opened row and one compression per level of its path) is checked by one kernel.
 * statuses[i] equals wl_verify's outcome for proof i: a failed opening is an opening error
 * (every listed opening precedes the check that ended the replay). Same arguments as
 * wl_verify_batch plus the context; WL_OK when every proof was checked. */
wl_status wl_verify_batch_device(wl_ctx* ctx, const wl_air_settings* settings, const uint32_t* constants, int32_t n,
                                 const int32_t* log_ns, const uint32_t* const* proofs, const size_t* proof_lens,
                                 int32_t threads, int32_t* statuses);

/* Per-phase transcript dumps, for diffing against another implementation of the protocol (a
 * build of the reference with the same parameters): JSON text
 *   {"proof_len": L, "events": [{"kind", "phase", "offset", "values"}, ...]}
 * with one "phase" event where each phase (commit, batching, zerocheck, inner_sums,
 * inner_sumcheck, whir, whir_round_i, whir_final) starts in proof_data, and every "challenge"
 * (8 canonical words), "queries" batch (sorted distinct indices) and "grinding" witness, each
 * with the proof_data offset at which it is drawn. *len is the buffer capacity on entry and the
 * bytes needed (with the terminating NUL) on return; WL_E_BUFFER_TOO_SMALL when short.
 * wl_ctx_set_transcript_dump(ctx, 1) makes every later proof on ctx record its dump;
 * wl_transcript_dump returns the last one. wl_verify_transcript runs wl_verify and returns the
 * transcript as the verifier reads it (up to the first failed check) with the verify status. */
wl_status wl_ctx_set_transcript_dump(wl_ctx* ctx, int32_t on);
wl_status wl_transcript_dump(wl_ctx* ctx, char* buf, size_t* len);
wl_status wl_verify_transcript(const wl_air_settings* settings, const uint32_t* constants, int32_t log_n,
                               const uint32_t* proof, size_t proof_len, char* buf, size_t* len);

/* sumcheck::verify_with_univariate_skip (crates/sumcheck/src/verify.rs:44-69) of a proof from
 * wl_sumcheck_abc_prove: the round polynomials, the zero claim and the final values a(r),
 * b(r), c(r) against eq(r, .) * (a * b - c). Host CPU only. */
wl_status wl_sumcheck_abc_verify(const uint32_t* p16_constants, int32_t log_n, int32_t skips, const uint32_t* proof,
                                 size_t proof_len);

/* Allocation-free variant of wl_sumcheck_abc_prove_device; it has no counterpart in the
 * reference. For callers that cannot allocate device memory: processes whose device memory
 * another framework owns and has already partitioned, and latency paths that must not enter
 * an allocator (an allocation can map new memory and stall the device). It makes no device,
 * pinned or host-heap allocation. Its device scratch is a fixed 4 MiB array inside the library
 * (present on every device that loads the library, until exit), which limits log_n to 14
 * (WL_E_SCRATCH_LIMIT beyond). Inputs are canonical device arrays of 2^log_n values, left
 * unchanged; the proof (host buffer, its exact length is returned with WL_E_BUFFER_TOO_SMALL
 * when short) equals wl_sumcheck_abc_prove_device's. `stream` is a cudaStream_t (NULL: the
 * default stream). All calls share the scratch array: calls that overlap on the GPU race and
 * must be serialised. The call copies between host and device and waits for its stream
 * between rounds, so it must not be called from a stream callback or host function (where
 * CUDA calls are not permitted) and rejects a stream under graph capture (WL_E_INVALID_ARG).
 * The first call on a device looks up the array's address (a failed lookup is retried by the
 * next call). */
wl_status wl_sumcheck_abc_prove_noalloc(const uint32_t* p16_constants, int32_t log_n, int32_t skips,
                                        const uint32_t* a_dev, const uint32_t* b_dev, const uint32_t* c_dev,
                                        uint32_t* proof_out, size_t* proof_len, void* stream);

/* Serving and batching (no counterpart in the reference, which proves one instance at a time
 * in src/examples/poseidon2.rs:153-174). A server runs `workers` proofs concurrently on one
 * device, each worker on its own stream; queued jobs are admitted first-in first-out when a
 * worker is idle and the job's estimated device footprint (wl_proof_footprint_bytes) fits in
 * the remaining HBM budget. A job is the reference example's input: a constants blob, 2^log_n
 * rows of 16 inputs (copied at submission) and settings; the server generates the trace on
 * the GPU and proves it with its own transcript, so the proof equals wl_prove's for the same
 * witness. Tickets are thread-safe to submit, poll and wait on. */
typedef struct wl_server wl_server;
typedef enum { WL_JOB_QUEUED = 0, WL_JOB_RUNNING = 1, WL_JOB_DONE = 2, WL_JOB_FAILED = 3 } wl_job_state;
/* Upper bound of the device memory one proof of 2^log_n rows takes under `settings` (NULL: the
 * defaults), by phase from the prover's buffer sizes; 0 for invalid arguments. */
uint64_t wl_proof_footprint_bytes(const wl_air_settings* settings, int32_t log_n);
wl_status wl_server_create(int32_t device, int32_t workers, uint64_t hbm_budget_bytes, wl_server** out);
void wl_server_destroy(wl_server* server); /* finishes queued and running jobs first */
const char* wl_server_last_error(const wl_server* server);
wl_status wl_server_submit(wl_server* server, const wl_air_settings* settings, const uint32_t* constants,
                           int32_t log_n, const uint32_t* inputs, uint64_t* ticket);
wl_status wl_server_poll(wl_server* server, uint64_t ticket, int32_t* state);
/* Blocks until the job ends. On success copies the proof (WL_E_BUFFER_TOO_SMALL keeps the
 * result and reports the length) and releases the ticket. times_ms (may be NULL): queued,
 * running, submit-to-finish latency. */
wl_status wl_server_wait(wl_server* server, uint64_t ticket, uint32_t* proof_out, size_t* proof_len,
                         double* times_ms);
wl_status wl_server_stats(wl_server* server, uint64_t* peak_bytes_admitted, int32_t* peak_running);

// Restricts the profiling of wl_profile_enable to one kernel class (NULL or "" = all), so
// that a timed region can carry the events of its dominant kernel only. No reference
// counterpart.
wl_status wl_profile_only(wl_ctx* ctx, const char* kernel_class);

// How the prover waits for the device at each transcript round trip: 1 (the default for a
// context) busy-polls an event, keeping the calling thread on its CPU so that no OS wake-up
// delays the next round; 0 blocks in cudaStreamSynchronize (the default of server workers).
// No reference counterpart.
wl_status wl_ctx_set_spin_sync(wl_ctx* ctx, int32_t spin);

/* Autotuning of the commitment's launch plans (no reference counterpart; the reference has
 * no GPU kernels). The LDE's stage split and persistent-pass occupancy ("lde", 6 plans), the
 * leaf sponges' rows per block ("leaf", 3 plans) and the Merkle level schedule ("merkle",
 * 3 plans) each have plans that write the same result at different speeds. A context that
 * tunes (the default for wl_ctx_create; server workers do not) runs every plan the first time
 * it meets a table shape, timed with CUDA events, and keeps the fastest per device and shape
 * for every context of the process. wl_tune_force pins a family to one plan (-1: back to
 * tuning); wl_tune_report writes the kept plans and their timings as JSON (same length
 * convention as wl_transcript_dump); wl_tune_clear forgets them. */
wl_status wl_ctx_set_autotune(wl_ctx* ctx, int32_t on);
wl_status wl_tune_force(const char* family, int32_t plan);
wl_status wl_tune_report(char* buf, size_t* len);
wl_status wl_tune_clear(void);

// Number of host synchronisations of the context's stream so far (device-to-host reads
// of challenges, sums and roots). Diagnostics; no reference counterpart.
wl_status wl_ctx_host_syncs(wl_ctx* ctx, uint64_t* out);

// Total milliseconds the host has spent waiting in those synchronisations (the rest of a
// proof's wall time is host work and launches). Diagnostics; no reference counterpart.
wl_status wl_ctx_host_wait_ms(wl_ctx* ctx, double* out);

/* Instrumentation (no reference counterpart; the reference profiles with tracing spans,
 * src/examples/poseidon2.rs:91-100). With profiling on, every kernel class launched on the
 * context is bracketed by CUDA events on the context's stream; wl_profile_json writes
 * {"class": [total_ms, launches], ...} for everything since the last enable. */
wl_status wl_profile_enable(wl_ctx* ctx, int32_t on);
wl_status wl_profile_json(wl_ctx* ctx, char* buf, size_t cap);
/* The context's CUDA stream (a cudaStream_t), for callers that time work with their own
 * events, and the number of kernels the library has launched in this process. */
void* wl_ctx_stream(wl_ctx* ctx);
uint64_t wl_kernel_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* WHIRLAWAY_B200_H */
