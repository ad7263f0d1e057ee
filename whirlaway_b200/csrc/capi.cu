// C ABI (include/whirlaway_b200.h): argument checks, error mapping, witness handles.
#include <cstring>
#include <algorithm>
#include <vector>
#include <thread>
#include <atomic>
#include <exception>
#include <memory>
#include <new>

#include "../../include/whirlaway_b200.h"
#include "prover.h"
#include "server.h"
#include "verifier.h"
#include "tuner.h"

struct wl_ctx {
  std::unique_ptr<wl::Context> c;
  std::string err;
};
struct wl_server {
  std::unique_ptr<wl::Server> s;
  std::string err;
};
struct wl_witness {
  int log_n = 0;
  wl::DBuf data;  // Montgomery form, 165 columns
};

namespace {

wl_status fail(wl_ctx* ctx, wl_status st, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return st;
}

template <class F>
wl_status guarded(wl_ctx* ctx, F&& f) {
  try {
    return f();
  } catch (const wl::CudaError& e) {
    cudaGetLastError();
    wl_status st = (e.code == cudaErrorMemoryAllocation) ? WL_E_OOM : WL_E_CUDA;
    return fail(ctx, st, e.what());
  } catch (const std::invalid_argument& e) {
    return fail(ctx, WL_E_INVALID_ARG, e.what());
  } catch (const std::bad_alloc&) {
    return fail(ctx, WL_E_OOM, "host allocation failed");
  } catch (const std::exception& e) {
    return fail(ctx, WL_E_INTERNAL, e.what());
  } catch (...) {
    return fail(ctx, WL_E_INTERNAL, "unknown error");
  }
}

bool settings_ok(const wl_air_settings* s, int log_n, std::string& why) {
  if (!s) { why = "settings is NULL"; return false; }
  if (s->security_bits < 1 || s->security_bits > 256) { why = "security_bits out of range"; return false; }
  if (s->log_inv_rate < 1 || s->log_inv_rate > 4) { why = "log_inv_rate must be in [1, 4]"; return false; }
  if (s->fold_first != 7 || s->fold_rest != 4) { why = "folding factors must be (7, 4)"; return false; }
  if (s->univariate_skips < 1 || s->univariate_skips > 4) { why = "univariate_skips must be in [1, 4]"; return false; }
  if (s->univariate_skips >= log_n) { why = "univariate_skips must be < log_n"; return false; }
  if (s->rs_domain_initial_reduction < 1 || s->rs_domain_initial_reduction > s->fold_first) {
    why = "rs_domain_initial_reduction out of range";
    return false;
  }
  if (s->whir_pow_bits < 0 || s->whir_pow_bits > 30) { why = "whir_pow_bits out of range"; return false; }
  if (log_n < 2 || log_n > 22) { why = "log_n must be in [2, 22]"; return false; }
  return true;
}

wl::Settings to_settings(const wl_air_settings* s) {
  wl::Settings r;
  r.security_bits = s->security_bits;
  r.log_inv_rate = s->log_inv_rate;
  r.fold_first = s->fold_first;
  r.fold_rest = s->fold_rest;
  r.univariate_skips = s->univariate_skips;
  r.rs_reduction = s->rs_domain_initial_reduction;
  r.whir_pow_bits = s->whir_pow_bits;
  return r;
}

wl::ProofJob make_job(const wl_air_settings* s, const uint32_t* constants, int log_n) {
  wl::ProofJob job;
  job.settings = to_settings(s);
  job.log_n = log_n;
  job.air = wl::air_consts_from(constants);
  job.p16 = wl::perm_consts_from<16>(constants + wl::N_AIR_CONSTS);
  job.p24 = wl::perm_consts_from<24>(constants + wl::N_AIR_CONSTS + wl::N_P16_CONSTS);
  return job;
}

wl_status emit_proof(wl_ctx* ctx, const std::vector<uint32_t>& pr, uint32_t* out, size_t* len) {
  if (*len < pr.size() || !out) {
    size_t cap = *len;
    *len = pr.size();
    return fail(ctx, WL_E_BUFFER_TOO_SMALL,
                "proof needs " + std::to_string(pr.size()) + " elements, buffer holds " + std::to_string(cap));
  }
  memcpy(out, pr.data(), pr.size() * sizeof(uint32_t));
  *len = pr.size();
  return WL_OK;
}

void store_timings(const wl::Timings& t, double* out) {
  if (!out) return;
  out[0] = t.commit_ms;
  out[1] = t.zerocheck_ms;
  out[2] = t.inner_ms;
  out[3] = t.whir_ms;
  out[4] = t.total_ms;
}

}  // namespace

extern "C" {

int32_t wl_air_columns(void) { return wl::AIR_W; }
int32_t wl_constants_len(void) { return wl::N_CONSTS; }
void wl_default_settings(wl_air_settings* out) {
  if (out) *out = wl_air_settings{128, 1, 7, 4, 4, 5, 16};
}

wl_status wl_ctx_create(int32_t device, uint64_t budget, wl_ctx** out) {
  if (!out) return WL_E_INVALID_ARG;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return WL_E_CUDA;
  }
  if (device < 0 || device >= count) return WL_E_INVALID_ARG;
  try {
    auto* c = new wl_ctx;
    c->c = std::make_unique<wl::Context>(device, budget);
    *out = c;
    return WL_OK;
  } catch (const wl::CudaError& e) {
    cudaGetLastError();
    return e.code == cudaErrorMemoryAllocation ? WL_E_OOM : WL_E_CUDA;
  } catch (...) {
    return WL_E_INTERNAL;
  }
}

void wl_ctx_destroy(wl_ctx* ctx) { delete ctx; }

const char* wl_last_error(const wl_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

wl_status wl_generate_workload(int32_t log_n, int64_t input_seed, uint32_t* constants_out, uint32_t* inputs_out) {
  if (!constants_out || log_n < 0 || log_n > 24) return WL_E_INVALID_ARG;
  wl::StdRng rng(0);
  int ci = 0;
  for (int i = 0; i < wl::N_AIR_CONSTS; i++) constants_out[ci++] = rng.random_f();
  const size_t n = size_t(16) << log_n;
  if (input_seed < 0) {
    for (size_t i = 0; i < n; i++) {
      uint32_t v = rng.random_f();
      if (inputs_out) inputs_out[i] = v;
    }
  } else if (inputs_out) {
    wl::StdRng r2((uint64_t)input_seed);
    for (size_t i = 0; i < n; i++) inputs_out[i] = r2.random_f();
  }
  for (int i = 0; i < wl::N_P16_CONSTS + wl::N_P24_CONSTS; i++) constants_out[ci++] = rng.random_f();
  return WL_OK;
}

wl_status wl_witness_upload(wl_ctx* ctx, int32_t log_n, const uint32_t* host, wl_witness** out) {
  if (!ctx || !host || !out || log_n < 2 || log_n > 22) return fail(ctx, WL_E_INVALID_ARG, "bad witness arguments");
  return guarded(ctx, [&] {
    auto w = std::make_unique<wl_witness>();
    w->log_n = log_n;
    const size_t n = size_t(wl::AIR_W) << log_n;
    w->data = wl::DBuf(n * 4, ctx->c->stream);
    WL_CUDA(cudaMemcpyAsync(w->data.as<void>(), host, n * 4, cudaMemcpyHostToDevice, ctx->c->stream));
    wl::launch_to_mont(w->data.as<uint32_t>(), n, ctx->c->stream);
    WL_CUDA(cudaStreamSynchronize(ctx->c->stream));
    *out = w.release();
    return WL_OK;
  });
}

wl_status wl_witness_generate(wl_ctx* ctx, const uint32_t* constants, int32_t log_n, const uint32_t* inputs,
                              wl_witness** out) {
  if (!ctx || !constants || !inputs || !out || log_n < 2 || log_n > 22)
    return fail(ctx, WL_E_INVALID_ARG, "bad witness arguments");
  return guarded(ctx, [&] {
    auto w = std::make_unique<wl_witness>();
    w->log_n = log_n;
    cudaStream_t st = ctx->c->stream;
    const size_t n_in = size_t(16) << log_n;
    wl::DBuf din(n_in * 4, st);
    WL_CUDA(cudaMemcpyAsync(din.as<void>(), inputs, n_in * 4, cudaMemcpyHostToDevice, st));
    w->data = wl::DBuf((size_t(wl::AIR_W) << log_n) * 4, st);
    wl::launch_trace_gen(din.as<uint32_t>(), wl::air_consts_from(constants), w->data.as<uint32_t>(), log_n, st);
    WL_CUDA(cudaStreamSynchronize(st));
    *out = w.release();
    return WL_OK;
  });
}

wl_status wl_witness_download(wl_ctx* ctx, const wl_witness* w, uint32_t* host) {
  if (!ctx || !w || !host) return fail(ctx, WL_E_INVALID_ARG, "bad witness arguments");
  return guarded(ctx, [&] {
    const size_t n = size_t(wl::AIR_W) << w->log_n;
    WL_CUDA(cudaMemcpyAsync(host, w->data.as<void>(), n * 4, cudaMemcpyDeviceToHost, ctx->c->stream));
    WL_CUDA(cudaStreamSynchronize(ctx->c->stream));
    for (size_t i = 0; i < n; i++) host[i] = kb::from_mont(host[i]);
    return WL_OK;
  });
}

void wl_witness_free(wl_ctx* ctx, wl_witness* w) {
  if (!w) return;
  if (ctx) cudaSetDevice(ctx->c->device);
  delete w;
}

wl_status wl_proof_len_bound(const wl_air_settings* s, int32_t log_n, size_t* out) {
  std::string why;
  if (!out || !settings_ok(s, log_n, why)) return WL_E_INVALID_ARG;
  try {
    *out = wl::proof_len_bound(to_settings(s), log_n);
    return WL_OK;
  } catch (...) {
    return WL_E_INVALID_ARG;
  }
}

wl_status wl_prove_witness(wl_ctx* ctx, const wl_air_settings* s, const uint32_t* constants, const wl_witness* w,
                           uint32_t* proof_out, size_t* proof_len, double* timings_ms) {
  if (!ctx) return WL_E_INVALID_ARG;
  std::string why;
  if (!w || !constants || !proof_len) return fail(ctx, WL_E_INVALID_ARG, "NULL argument");
  if (!settings_ok(s, w->log_n, why)) return fail(ctx, WL_E_INVALID_ARG, why);
  return guarded(ctx, [&] {
    wl::ProofJob job = make_job(s, constants, w->log_n);
    wl::Timings t;
    std::vector<uint32_t> pr = wl::prove_air(*ctx->c, job, w->data.as<uint32_t>(), &t);
    store_timings(t, timings_ms);
    return emit_proof(ctx, pr, proof_out, proof_len);
  });
}

wl_status wl_prove(wl_ctx* ctx, const wl_air_settings* s, const uint32_t* constants, int32_t log_n,
                   const uint32_t* witness, uint32_t* proof_out, size_t* proof_len, double* timings_ms) {
  if (!ctx) return WL_E_INVALID_ARG;
  std::string why;
  if (!settings_ok(s, log_n, why)) return fail(ctx, WL_E_INVALID_ARG, why);
  if (!witness || !constants || !proof_len) return fail(ctx, WL_E_INVALID_ARG, "NULL argument");
  if (log_n < 2 || log_n > 22) return fail(ctx, WL_E_INVALID_ARG, "log_n out of range");
  // the witness goes up in tiles of 16 columns while the first commitment encodes
  return guarded(ctx, [&] {
    wl::ProofJob job = make_job(s, constants, log_n);
    wl::Timings t;
    std::vector<uint32_t> pr = wl::prove_air_host(*ctx->c, job, witness, &t);
    store_timings(t, timings_ms);
    return emit_proof(ctx, pr, proof_out, proof_len);
  });
}

namespace {
// A constraint program from its C description (throws std::invalid_argument when malformed).
wl::ProgramAir program_from(const wl_air_program* p, int log_n) {
  if (!p) throw std::invalid_argument("program is NULL");
  wl::ProgramAir prog = wl::ProgramAir::build(p->n_columns, p->n_constraints, p->constraint_degree, p->n_ops, p->ops,
                                              p->n_consts, p->consts);
  prog.set_preprocessed(p->n_preprocessed, p->preprocessed, log_n);
  return prog;
}
wl::ProofJob make_program_job(const wl_air_settings* s, const uint32_t* hash_constants, int log_n,
                              const wl::ProgramAir* prog) {
  wl::ProofJob job;
  job.settings = to_settings(s);
  job.log_n = log_n;
  job.p16 = wl::perm_consts_from<16>(hash_constants);
  job.p24 = wl::perm_consts_from<24>(hash_constants + wl::N_P16_CONSTS);
  job.prog = prog;
  return job;
}
}  // namespace

wl_status wl_prove_program(wl_ctx* ctx, const wl_air_settings* s, const uint32_t* hash_constants,
                           const wl_air_program* program, int32_t log_n, const uint32_t* witness,
                           uint32_t* proof_out, size_t* proof_len) {
  if (!ctx) return WL_E_INVALID_ARG;
  std::string why;
  if (!settings_ok(s, log_n, why)) return fail(ctx, WL_E_INVALID_ARG, why);
  if (!witness || !hash_constants || !program || !proof_len) return fail(ctx, WL_E_INVALID_ARG, "NULL argument");
  return guarded(ctx, [&] {
    const wl::ProgramAir prog = program_from(program, log_n);
    const wl::ProofJob job = make_program_job(s, hash_constants, log_n, &prog);
    std::vector<uint32_t> pr = wl::prove_air_host(*ctx->c, job, witness, nullptr);
    return emit_proof(ctx, pr, proof_out, proof_len);
  });
}

wl_status wl_verify_program(const wl_air_settings* s, const uint32_t* hash_constants, const wl_air_program* program,
                            int32_t log_n, const uint32_t* proof, size_t proof_len) {
  std::string why;
  if (!hash_constants || !program || (!proof && proof_len) || !settings_ok(s, log_n, why)) return WL_E_INVALID_ARG;
  for (size_t i = 0; i < proof_len; i++)
    if (proof[i] >= kb::P) return WL_E_INVALID_ARG;
  return guarded(nullptr, [&] {
    const wl::ProgramAir prog = program_from(program, log_n);
    const wl::ProofJob job = make_program_job(s, hash_constants, log_n, &prog);
    return wl_status(wl::verify_air_proof(job.settings, job.air, job.p16, job.p24, log_n, proof, proof_len, nullptr, 0,
                                          nullptr, &prog));
  });
}

wl_status wl_program_proof_len_bound(const wl_air_settings* s, const wl_air_program* program, int32_t log_n,
                                     size_t* out) {
  std::string why;
  if (!out || !program || !settings_ok(s, log_n, why)) return WL_E_INVALID_ARG;
  try {
    const wl::ProgramAir prog = program_from(program, log_n);
    *out = wl::proof_len_bound(to_settings(s), log_n, prog.W, prog.degree);
    return WL_OK;
  } catch (...) {
    return WL_E_INVALID_ARG;
  }
}

wl_status wl_prove_batch(wl_ctx* ctx, const wl_air_settings* s, const uint32_t* constants, int32_t n,
                         const wl_witness* const* ws, uint32_t* proof_out, size_t stride, size_t* proof_lens) {
  if (!ctx || !ws || !proof_out || !proof_lens || n < 0) return fail(ctx, WL_E_INVALID_ARG, "bad batch arguments");
  for (int i = 0; i < n; i++) {
    size_t len = stride;
    wl_status st = wl_prove_witness(ctx, s, constants, ws[i], proof_out + size_t(i) * stride, &len, nullptr);
    proof_lens[i] = len;
    if (st != WL_OK) return st;
  }
  return WL_OK;
}

static wl_status abc_common(wl_ctx* ctx, const uint32_t* p16c, int32_t log_n, int32_t skips, const uint32_t* a,
                            const uint32_t* b, const uint32_t* c, bool device, uint32_t* proof_out, size_t* proof_len,
                            float* round_ms) {
  if (!ctx) return WL_E_INVALID_ARG;
  if (!p16c || !a || !b || !c || !proof_len || log_n < 2 || log_n > 26 || skips < 1 || skips > 4 || skips >= log_n)
    return fail(ctx, WL_E_INVALID_ARG, "bad sumcheck arguments");
  return guarded(ctx, [&] {
    cudaStream_t st = ctx->c->stream;
    const size_t N = size_t(1) << log_n;
    wl::DBuf d(N * 12, st);
    uint32_t* da = d.as<uint32_t>();
    auto kind = device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    WL_CUDA(cudaMemcpyAsync(da, a, N * 4, kind, st));
    WL_CUDA(cudaMemcpyAsync(da + N, b, N * 4, kind, st));
    WL_CUDA(cudaMemcpyAsync(da + 2 * N, c, N * 4, kind, st));
    wl::launch_to_mont(da, 3 * N, st);
    kb::P16Consts p16 = wl::perm_consts_from<16>(p16c);
    std::vector<float> ms;
    std::vector<uint32_t> pr = wl::prove_abc(*ctx->c, p16, log_n, skips, da, da + N, da + 2 * N, &ms);
    if (round_ms) std::copy(ms.begin(), ms.end(), round_ms);
    return emit_proof(ctx, pr, proof_out, proof_len);
  });
}

wl_status wl_sumcheck_abc_prove(wl_ctx* ctx, const uint32_t* p16c, int32_t log_n, int32_t skips, const uint32_t* a,
                                const uint32_t* b, const uint32_t* c, uint32_t* proof_out, size_t* proof_len,
                                float* round_ms) {
  return abc_common(ctx, p16c, log_n, skips, a, b, c, false, proof_out, proof_len, round_ms);
}

wl_status wl_sumcheck_abc_prove_device(wl_ctx* ctx, const uint32_t* p16c, int32_t log_n, int32_t skips,
                                       const uint32_t* a, const uint32_t* b, const uint32_t* c, uint32_t* proof_out,
                                       size_t* proof_len, float* round_ms) {
  return abc_common(ctx, p16c, log_n, skips, a, b, c, true, proof_out, proof_len, round_ms);
}

// Host-only verifiers: no context, no device.
namespace {
wl_status verify_with(const wl_air_settings* s, const uint32_t* constants, int32_t log_n, const uint32_t* proof,
                      size_t proof_len, int threads) {
  std::string why;
  if (!constants || (!proof && proof_len) || !settings_ok(s, log_n, why)) return WL_E_INVALID_ARG;
  for (size_t i = 0; i < proof_len; i++)
    if (proof[i] >= kb::P) return WL_E_INVALID_ARG;  // not a canonical field element
  return guarded(nullptr, [&] {
    wl::ProofJob job = make_job(s, constants, log_n);
    return wl_status(
        wl::verify_air_proof(job.settings, job.air, job.p16, job.p24, log_n, proof, proof_len, nullptr, threads));
  });
}
}  // namespace

wl_status wl_verify(const wl_air_settings* s, const uint32_t* constants, int32_t log_n, const uint32_t* proof,
                    size_t proof_len) {
  return verify_with(s, constants, log_n, proof, proof_len, 0);
}

namespace {
wl_status emit_text(const std::string& text, char* buf, size_t* len) {
  const size_t need = text.size() + 1;
  if (!buf || *len < need) {
    *len = need;
    return WL_E_BUFFER_TOO_SMALL;
  }
  memcpy(buf, text.c_str(), need);
  *len = need;
  return WL_OK;
}
}  // namespace

wl_status wl_ctx_set_transcript_dump(wl_ctx* ctx, int32_t on) {
  if (!ctx) return WL_E_INVALID_ARG;
  ctx->c->dump_transcript = on != 0;
  if (!on) ctx->c->last_dump.clear();
  return WL_OK;
}

wl_status wl_transcript_dump(wl_ctx* ctx, char* buf, size_t* len) {
  if (!ctx || !len) return WL_E_INVALID_ARG;
  if (ctx->c->last_dump.empty()) return fail(ctx, WL_E_INVALID_ARG, "no transcript recorded (enable it, then prove)");
  return emit_text(ctx->c->last_dump, buf, len);
}

wl_status wl_verify_transcript(const wl_air_settings* s, const uint32_t* constants, int32_t log_n,
                               const uint32_t* proof, size_t proof_len, char* buf, size_t* len) {
  std::string why;
  if (!constants || !len || (!proof && proof_len) || !settings_ok(s, log_n, why)) return WL_E_INVALID_ARG;
  for (size_t i = 0; i < proof_len; i++)
    if (proof[i] >= kb::P) return WL_E_INVALID_ARG;
  return guarded(nullptr, [&] {
    wl::ProofJob job = make_job(s, constants, log_n);
    wl::TranscriptLog log;
    const int st = wl::verify_air_proof(job.settings, job.air, job.p16, job.p24, log_n, proof, proof_len, &log);
    const wl_status out = emit_text(log.json(proof_len), buf, len);
    return out != WL_OK ? out : wl_status(st);
  });
}

wl_status wl_verify_batch(const wl_air_settings* s, const uint32_t* constants, int32_t n, const int32_t* log_ns,
                          const uint32_t* const* proofs, const size_t* proof_lens, int32_t threads,
                          int32_t* statuses) {
  if (!s || !constants || n < 0 || (n && (!log_ns || !proofs || !proof_lens || !statuses)))
    return WL_E_INVALID_ARG;
  return guarded(nullptr, [&] {
    unsigned hw = std::thread::hardware_concurrency();
    int T = threads > 0 ? threads : int(hw ? hw : 1);
    T = std::max(1, std::min(T, n));
    std::atomic<int> next{0};
    auto work = [&] {
      for (int i = next++; i < n; i = next++)
        statuses[i] = verify_with(s, constants, log_ns[i], proofs[i], proof_lens[i], 1);  // one thread per proof
    };
    wl::run_on_threads(size_t(T), work);
    return WL_OK;
  });
}

wl_status wl_verify_batch_device(wl_ctx* ctx, const wl_air_settings* s, const uint32_t* constants, int32_t n,
                                 const int32_t* log_ns, const uint32_t* const* proofs, const size_t* proof_lens,
                                 int32_t threads, int32_t* statuses) {
  if (!ctx || !s || !constants || n < 0 || (n && (!log_ns || !proofs || !proof_lens || !statuses)))
    return WL_E_INVALID_ARG;
  return guarded(ctx, [&] {
    // 1) every transcript on host threads, one proof per thread, Merkle openings listed
    std::vector<std::vector<wl::MerkleOpening>> open(n);
    unsigned hw = std::thread::hardware_concurrency();
    int T = threads > 0 ? threads : int(hw ? hw : 1);
    T = std::max(1, std::min(T, std::max(n, 1)));
    std::atomic<int> next{0};
    auto work = [&] {
      for (int i = next++; i < n; i = next++) {
        std::string why;
        const uint32_t* pr = proofs[i];
        const size_t len = proof_lens[i];
        bool canonical = pr || !len;
        for (size_t k = 0; canonical && k < len; k++) canonical = pr[k] < kb::P;
        if (!canonical || !settings_ok(s, log_ns[i], why)) {
          statuses[i] = WL_E_INVALID_ARG;
          continue;
        }
        wl::ProofJob job = make_job(s, constants, log_ns[i]);
        statuses[i] = wl::verify_air_proof(job.settings, job.air, job.p16, job.p24, log_ns[i], pr, len, nullptr, 1,
                                           &open[i]);
      }
    };
    wl::run_on_threads(size_t(T), work);
    // 2) all openings in one kernel over the concatenated proofs
    std::vector<size_t> base(n + 1, 0);
    for (int i = 0; i < n; i++) base[i + 1] = base[i] + (open[i].empty() ? 0 : proof_lens[i]);
    std::vector<wl::OpeningCheck> ops;
    std::vector<int> owner;
    for (int i = 0; i < n; i++)
      for (const wl::MerkleOpening& o : open[i]) {
        ops.push_back({base[i] + o.row, base[i] + o.path, base[i] + o.root, o.q, o.ll});
        owner.push_back(i);
      }
    if (ops.empty()) return WL_OK;
    wl::Context& c = *ctx->c;
    wl::DBuf words(sizeof(uint32_t) * base[n], c.stream), dops(sizeof(wl::OpeningCheck) * ops.size(), c.stream),
        dok(ops.size(), c.stream);
    for (int i = 0; i < n; i++)
      if (!open[i].empty())
        WL_CUDA(cudaMemcpyAsync(words.as<uint32_t>() + base[i], proofs[i], sizeof(uint32_t) * proof_lens[i],
                                cudaMemcpyHostToDevice, c.stream));
    WL_CUDA(cudaMemcpyAsync(dops.as<void>(), ops.data(), sizeof(wl::OpeningCheck) * ops.size(), cudaMemcpyHostToDevice,
                            c.stream));
    const wl::ProofJob job = make_job(s, constants, log_ns[0]);
    {
      wl::ProfScope _ps(c, "check_openings");
      wl::launch_check_openings(words.as<uint32_t>(), dops.as<wl::OpeningCheck>(), int(ops.size()), job.p24, job.p16,
                                dok.as<uint8_t>(), c.stream);
    }
    std::vector<uint8_t> ok(ops.size());
    WL_CUDA(cudaMemcpyAsync(ok.data(), dok.as<void>(), ok.size(), cudaMemcpyDeviceToHost, c.stream));
    c.wait_stream();
    // 3) a failed opening comes before whatever ended the replay: an opening error
    for (size_t j = 0; j < ok.size(); j++)
      if (!ok[j]) statuses[owner[j]] = WL_E_INVALID_PCS_OPENING;
    return WL_OK;
  });
}

wl_status wl_sumcheck_abc_verify(const uint32_t* p16c, int32_t log_n, int32_t skips, const uint32_t* proof,
                                 size_t proof_len) {
  if (!p16c || (!proof && proof_len) || log_n < 2 || log_n > 26 || skips < 1 || skips > 4 || skips >= log_n)
    return WL_E_INVALID_ARG;
  for (size_t i = 0; i < proof_len; i++)
    if (proof[i] >= kb::P) return WL_E_INVALID_ARG;
  return guarded(nullptr, [&] {
    const kb::P16Consts p16 = wl::perm_consts_from<16>(p16c);
    return wl_status(wl::verify_abc_proof(p16, log_n, skips, proof, proof_len));
  });
}

wl_status wl_profile_enable(wl_ctx* ctx, int32_t on) {
  if (!ctx) return WL_E_INVALID_ARG;
  return guarded(ctx, [&] {
    ctx->c->prof_flush();
    ctx->c->prof_totals.clear();
    ctx->c->profile = on != 0;
    wl::host_clock() = wl::HostClock{};
    wl::host_clock().on = on != 0;
    ctx->c->prof_t0_ms = wl::host_now_ms();
    ctx->c->prof_wait0_ms = ctx->c->host_wait_ms;
    ctx->c->prof_syncs0 = ctx->c->host_syncs;
    return WL_OK;
  });
}

wl_status wl_profile_only(wl_ctx* ctx, const char* kernel_class) {
  if (!ctx) return WL_E_INVALID_ARG;
  return guarded(ctx, [&] {
    ctx->c->profile_only = kernel_class ? kernel_class : "";
    return WL_OK;
  });
}

wl_status wl_ctx_set_spin_sync(wl_ctx* ctx, int32_t spin) {
  if (!ctx) return WL_E_INVALID_ARG;
  ctx->c->spin_sync = spin != 0;
  return WL_OK;
}

wl_status wl_ctx_set_autotune(wl_ctx* ctx, int32_t on) {
  if (!ctx) return WL_E_INVALID_ARG;
  ctx->c->autotune = on != 0;
  return WL_OK;
}

wl_status wl_tune_force(const char* family, int32_t plan) {
  const int f = wl::tune_family_from_name(family);
  if (f < 0 || plan < -1 || plan >= wl::tune_plan_count(f)) return WL_E_INVALID_ARG;
  wl::tune_force(f, plan);
  return WL_OK;
}

wl_status wl_tune_report(char* buf, size_t* len) {
  if (!len) return WL_E_INVALID_ARG;
  return emit_text(wl::tune_json(), buf, len);
}

wl_status wl_tune_clear(void) {
  wl::tune_clear();
  return WL_OK;
}

wl_status wl_ctx_host_syncs(wl_ctx* ctx, uint64_t* out) {
  if (!ctx || !out) return WL_E_INVALID_ARG;
  *out = ctx->c->host_syncs;
  return WL_OK;
}

wl_status wl_ctx_host_wait_ms(wl_ctx* ctx, double* out) {
  if (!ctx || !out) return WL_E_INVALID_ARG;
  *out = ctx->c->host_wait_ms;
  return WL_OK;
}

wl_status wl_profile_json(wl_ctx* ctx, char* buf, size_t cap) {
  if (!ctx || !buf) return WL_E_INVALID_ARG;
  return guarded(ctx, [&] {
    ctx->c->prof_flush();
    std::string js = "{";
    bool first = true;
    for (auto& kv : ctx->c->prof_totals) {
      if (!first) js += ", ";
      first = false;
      js += "\"" + kv.first + "\": [" + std::to_string(kv.second.first) + ", " + std::to_string(kv.second.second) + "]";
    }
    const wl::HostClock& hc = wl::host_clock();
    if (hc.on) {
      const std::pair<const char*, std::pair<double, long>> host[] = {
          {"host:transcript_perm", {hc.perm_ms, hc.perms}}, {"host:alloc", {hc.alloc_ms, hc.allocs}},
          {"host:launch", {hc.launch_ms, hc.launches}}, {"host:upload", {hc.upload_ms, hc.uploads}},
          {"host:wait", {ctx->c->host_wait_ms - ctx->c->prof_wait0_ms, long(ctx->c->host_syncs - ctx->c->prof_syncs0)}},
          {"host:elapsed", {wl::host_now_ms() - ctx->c->prof_t0_ms, 1L}}};
      for (auto& h : host) {
        if (!first) js += ", ";
        first = false;
        js += "\"" + std::string(h.first) + "\": [" + std::to_string(h.second.first) + ", " + std::to_string(h.second.second) + "]";
      }
      for (auto& b : hc.busy) js += ", \"host:busy:" + b.first + "\": [" + std::to_string(b.second) + ", 1]";
    }
    js += "}";
    if (js.size() + 1 > cap) return fail(ctx, WL_E_BUFFER_TOO_SMALL, "profile buffer too small");
    memcpy(buf, js.c_str(), js.size() + 1);
    return WL_OK;
  });
}

uint64_t wl_proof_footprint_bytes(const wl_air_settings* s, int32_t log_n) {
  wl_air_settings d;
  if (!s) {
    wl_default_settings(&d);
    s = &d;
  }
  std::string why;
  if (!settings_ok(s, log_n, why)) return 0;
  return wl::proof_footprint_bytes(to_settings(s), log_n);
}

wl_status wl_server_create(int32_t device, int32_t workers, uint64_t budget, wl_server** out) {
  if (!out || workers < 1 || workers > 64) return WL_E_INVALID_ARG;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return WL_E_CUDA;
  }
  if (device < 0 || device >= count) return WL_E_INVALID_ARG;
  try {
    auto* s = new wl_server;
    s->s = std::make_unique<wl::Server>(device, workers, budget);
    *out = s;
    return WL_OK;
  } catch (const wl::CudaError& e) {
    cudaGetLastError();
    return e.code == cudaErrorMemoryAllocation ? WL_E_OOM : WL_E_CUDA;
  } catch (...) {
    return WL_E_INTERNAL;
  }
}

void wl_server_destroy(wl_server* s) { delete s; }

const char* wl_server_last_error(const wl_server* s) { return s ? s->err.c_str() : "no server"; }

static wl_status server_fail(wl_server* s, wl_status st, const std::string& m) {
  if (s) s->err = m;
  return st;
}

wl_status wl_server_submit(wl_server* s, const wl_air_settings* settings, const uint32_t* constants, int32_t log_n,
                           const uint32_t* inputs, uint64_t* ticket) {
  if (!s || !constants || !inputs || !ticket) return server_fail(s, WL_E_INVALID_ARG, "NULL argument");
  std::string why;
  if (!settings_ok(settings, log_n, why)) return server_fail(s, WL_E_INVALID_ARG, why);
  try {
    wl::ServeJob job;
    job.settings = to_settings(settings);
    job.log_n = log_n;
    job.constants.assign(constants, constants + wl::N_CONSTS);
    job.inputs.assign(inputs, inputs + (size_t(16) << log_n));
    *ticket = s->s->submit(std::move(job));
    return WL_OK;
  } catch (const std::invalid_argument& e) {
    return server_fail(s, WL_E_BUDGET, e.what());
  } catch (const std::exception& e) {
    return server_fail(s, WL_E_INTERNAL, e.what());
  }
}

wl_status wl_server_poll(wl_server* s, uint64_t ticket, int32_t* state) {
  if (!s || !state) return WL_E_INVALID_ARG;
  try {
    *state = (int32_t)s->s->poll(ticket);
    return WL_OK;
  } catch (const std::exception& e) {
    return server_fail(s, WL_E_INVALID_ARG, e.what());
  }
}

wl_status wl_server_wait(wl_server* s, uint64_t ticket, uint32_t* proof_out, size_t* proof_len, double* times_ms) {
  if (!s || !proof_len) return WL_E_INVALID_ARG;
  try {
    wl::ServeResult r = s->s->wait(ticket, false);
    if (times_ms) {
      times_ms[0] = r.start_ms - r.submit_ms;
      times_ms[1] = r.end_ms - r.start_ms;
      times_ms[2] = r.end_ms - r.submit_ms;
    }
    if (r.state == wl::JOB_FAILED) {
      s->s->release(ticket);
      return server_fail(s, WL_E_INTERNAL, r.error);
    }
    if (!proof_out || *proof_len < r.proof.size()) {
      *proof_len = r.proof.size();
      return server_fail(s, WL_E_BUFFER_TOO_SMALL, "proof buffer too small");
    }
    memcpy(proof_out, r.proof.data(), r.proof.size() * 4);
    *proof_len = r.proof.size();
    s->s->release(ticket);
    return WL_OK;
  } catch (const std::exception& e) {
    return server_fail(s, WL_E_INVALID_ARG, e.what());
  }
}

wl_status wl_server_stats(wl_server* s, uint64_t* peak_bytes, int32_t* peak_running) {
  if (!s) return WL_E_INVALID_ARG;
  if (peak_bytes) *peak_bytes = s->s->peak_in_use();
  if (peak_running) *peak_running = s->s->peak_running();
  return WL_OK;
}

void* wl_ctx_stream(wl_ctx* ctx) { return ctx ? (void*)ctx->c->stream : nullptr; }
uint64_t wl_kernel_launch_count(void) { return wl::launch_counter().load(); }

}  // extern "C"
