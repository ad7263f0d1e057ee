// Allocation-free variant of the standalone a*b - c zerocheck prover.
//
// For callers that cannot allocate device memory: a process whose device memory is owned and
// pre-partitioned by another framework (which would see any allocation of ours as memory it
// no longer has), or a latency path that must not enter an allocator (whose calls can map new
// memory and stall the device for milliseconds). Every device buffer this prover needs lives
// in one file-scope device array of fixed size, and host-side state is kept in fixed-capacity
// arrays; the call makes no cudaMalloc / cudaMallocAsync / cudaMallocHost / cudaFree call and
// no host heap allocation of its own.
//
// Limits and sharing:
//  * log_n <= 14 (and 1 <= skips <= 4, skips < log_n); larger sizes are rejected with
//    WL_E_SCRATCH_LIMIT before any device work.
//  * The scratch array (4 MiB per device that loads the library, held until the process
//    exits) is shared by all calls and keeps the last call's contents; every buffer the prover
//    reads is written earlier in the same call. Calls that overlap on the GPU (on different
//    streams or from different threads) race on it and must be serialised by the caller.
//  * The call copies to and from the host and waits for its stream between sumcheck rounds.
//    It must not be called from a stream callback or a host function (cudaLaunchHostFunc),
//    where CUDA calls are not permitted, and it cannot run on a stream that is being captured
//    into a graph: a capturing stream is rejected with WL_E_INVALID_ARG.
//  * The first call on a device looks up the array's device address (cudaGetSymbolAddress,
//    with that device current); a failed lookup is not kept, the next call retries it.
#include <cstring>
#include <mutex>

#include "../../include/whirlaway_b200.h"
#include "host.h"
#include "kernels.h"

namespace wl {
namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(4) << 20;
constexpr int NOALLOC_MAX_LOG_N = 14;
constexpr int MAX_DEVICES = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

std::mutex g_scratch_mu;
void* g_scratch_ptr[MAX_DEVICES];

// Device address of the scratch array for the current device. Looked up once per device and
// kept only on success, so that a transient failure is retried by the next call.
cudaError_t scratch_base(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= MAX_DEVICES) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return e;
    }
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return cudaSuccess;
}

// Bump allocation inside the scratch array (256-byte aligned).
struct Arena {
  unsigned char* base;
  size_t off = 0;
  template <class T>
  T* take(size_t count) {
    size_t bytes = (count * sizeof(T) + 255) & ~size_t(255);
    if (off + bytes > NOALLOC_SCRATCH_BYTES) throw std::length_error("scratch exhausted");
    T* p = reinterpret_cast<T*>(base + off);
    off += bytes;
    return p;
  }
};

// Canonical-input variants of the round-0 kernels (the inputs belong to the caller and
// stay canonical; values are converted to Montgomery form as they are read).
constexpr int NA_X = 32;

__global__ void k_abc0_eval_canon(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b,
                                  const uint32_t* __restrict__ c, int log_n, int k, int nz,
                                  const uint32_t* __restrict__ lw, const kb::ef* __restrict__ eq,
                                  kb::ef* __restrict__ partial) {
  __shared__ uint32_t w_s[32 * 16];
  const int nsk = 1 << k;
  const int tid = threadIdx.y * NA_X + threadIdx.x;
  for (int i = tid; i < nz * nsk; i += NA_X * blockDim.y) w_s[i] = lw[i];
  __syncthreads();
  const size_t N = size_t(1) << log_n, S = N >> k;
  const size_t x = size_t(blockIdx.x) * NA_X + threadIdx.x;
  const int zi = threadIdx.y;
  kb::ef res = kb::ef_zero();
  if (x < S && zi < nz) {
    const uint32_t* wz = w_s + zi * nsk;
    uint32_t va = 0, vb = 0, vc = 0;
    for (int j = 0; j < nsk; j++) {
      const size_t i = size_t(j) * S + x;
      va = kb::add(va, kb::mul(wz[j], kb::to_mont(a[i])));
      vb = kb::add(vb, kb::mul(wz[j], kb::to_mont(b[i])));
      vc = kb::add(vc, kb::mul(wz[j], kb::to_mont(c[i])));
    }
    res = kb::ef_mul_f(eq[x], kb::sub(kb::mul(va, vb), vc));
  }
  res = warp_reduce_ef(res);
  if (threadIdx.x == 0 && zi < nz) partial[size_t(blockIdx.x) * nz + zi] = res;
}

__global__ void k_abc0_fold_canon(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b,
                                  const uint32_t* __restrict__ c, int log_n, int k, const kb::ef* __restrict__ sel,
                                  kb::ef* __restrict__ out) {
  const int nsk = 1 << k;
  const size_t N = size_t(1) << log_n, S = N >> k;
  const size_t x = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (x >= S) return;
  const uint32_t* src = blockIdx.y == 0 ? a : blockIdx.y == 1 ? b : c;
  kb::ef acc = kb::ef_zero();
  for (int j = 0; j < nsk; j++) acc = kb::ef_add(acc, kb::ef_mul_f(sel[j], kb::to_mont(src[size_t(j) * S + x])));
  out[size_t(blockIdx.y) * S + x] = acc;
}

// Fixed-capacity host helpers (no heap).
constexpr int MAXC = 64;  // polynomial coefficients

// Coefficients of the polynomial through (i, ys[i]) for i < n (integer nodes).
void interpolate_fixed(const ef* ys, int n, ef* out) {
  for (int k = 0; k < n; k++) out[k] = kb::ef_zero();
  uint32_t basis[MAXC], tmp[MAXC];
  for (int i = 0; i < n; i++) {
    int deg = 0;
    basis[0] = kb::R_MOD_P;
    uint32_t denom = kb::R_MOD_P;
    for (int j = 0; j < n; j++) {
      if (j == i) continue;
      const uint32_t negj = fm(-j);
      for (int q = 0; q <= deg + 1; q++) tmp[q] = 0;
      for (int q = 0; q <= deg; q++) {
        tmp[q] = kb::add(tmp[q], kb::mul(basis[q], negj));
        tmp[q + 1] = kb::add(tmp[q + 1], basis[q]);
      }
      deg++;
      for (int q = 0; q <= deg; q++) basis[q] = tmp[q];
      denom = kb::mul(denom, fm(i - j));
    }
    const ef yi = kb::ef_mul_f(ys[i], kb::inv_m(denom));
    for (int q = 0; q < n; q++) out[q] = kb::ef_add(out[q], kb::ef_mul_f(yi, basis[q]));
  }
}
int poly_mul_fixed(const ef* a, int na, const ef* b, int nb, ef* out) {
  for (int i = 0; i < na + nb - 1; i++) out[i] = kb::ef_zero();
  for (int i = 0; i < na; i++)
    for (int j = 0; j < nb; j++) out[i + j] = kb::ef_add(out[i + j], kb::ef_mul(a[i], b[j]));
  return na + nb - 1;
}
ef poly_eval_fixed(const ef* c, int n, const ef& x) {
  ef r = kb::ef_zero();
  for (int i = n; i-- > 0;) r = kb::ef_add(kb::ef_mul(r, x), c[i]);
  return r;
}
// L_i(x) for the Lagrange basis on {0..nsk-1}, for every i.
void selectors_at(int nsk, const ef& x, ef* out) {
  for (int i = 0; i < nsk; i++) {
    ef num = kb::ef_one();
    uint32_t den = kb::R_MOD_P;
    for (int j = 0; j < nsk; j++) {
      if (j == i) continue;
      num = kb::ef_mul(num, kb::ef_sub_f(x, fm(j)));
      den = kb::mul(den, fm(i - j));
    }
    out[i] = kb::ef_mul_f(num, kb::inv_m(den));
  }
}
uint32_t selector_at_int(int nsk, int i, int z) {
  uint32_t num = kb::R_MOD_P, den = kb::R_MOD_P;
  for (int j = 0; j < nsk; j++) {
    if (j == i) continue;
    num = kb::mul(num, fm(z - j));
    den = kb::mul(den, fm(i - j));
  }
  return kb::mul(num, kb::inv_m(den));
}

// Transcript writing straight into the caller's proof buffer (canonical values).
struct FixedTranscript {
  HostChallenger ch;
  uint32_t* out;
  size_t cap, len = 0;
  void add_ext(const ef* v, int n) {
    for (int i = 0; i < n; i++)
      for (int e = 0; e < 8; e++) {
        if (len >= cap) throw std::length_error("proof buffer too small");
        out[len++] = kb::from_mont(v[i].c[e]);
        ch.observe(v[i].c[e]);
      }
  }
  ef sample_ext() {
    ef e;
    for (int i = 0; i < 8; i++) e.c[i] = ch.sample();
    return e;
  }
};

void d2h(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  WL_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
  WL_CUDA(cudaStreamSynchronize(s));
}
void h2d(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  WL_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
}

size_t abc_proof_len(int n, int k) {
  const int nsk = 1 << k;
  return size_t(8) * (size_t(3 * (nsk - 1) + 1) + size_t(4) * (n - k) + 3);
}

// The same transcript as prove_abc (prover.cu), every device buffer carved from the arena.
void prove_abc_fixed(const kb::P16Consts& p16, int n, int k, const uint32_t* a, const uint32_t* b,
                     const uint32_t* c, Arena& ar, FixedTranscript& ts, cudaStream_t st) {
  const int nsk = 1 << k;
  const size_t S = size_t(1) << (n - k);
  ts.ch.perm = &p16;
  ef r[32];
  const int nr = n + 1 - k;
  for (int i = 0; i < nr; i++) r[i] = ts.sample_ext();
  const int nz = 2 * (nsk - 1) - nsk + 1;
  ef* d_r = ar.take<ef>(nr);
  h2d(d_r, r, sizeof(ef) * nr, st);
  ef* eq = ar.take<ef>(S);
  ef* cols = ar.take<ef>(3 * S);
  ef* cols2 = ar.take<ef>(3 * S / 2 + 1);
  ef* part = ar.take<ef>((S + 31) / 32 * nz + 64);
  ef* red = ar.take<ef>(32);
  uint32_t* d_lw = ar.take<uint32_t>(size_t(nz) * nsk);
  ef* d_sel = ar.take<ef>(16);
  ef* d_ch = ar.take<ef>(1);
  // round 0
  uint32_t lw[16 * 16];
  for (int zi = 0; zi < nz; zi++)
    for (int j = 0; j < nsk; j++) lw[zi * nsk + j] = selector_at_int(nsk, j, nsk + zi);
  h2d(d_lw, lw, sizeof(uint32_t) * nz * nsk, st);
  launch_eq_table(d_r + 1, n - k, eq, st);
  const int nb0 = (int)((S + NA_X - 1) / NA_X);
  k_abc0_eval_canon<<<nb0, dim3(NA_X, nz), 0, st>>>(a, b, c, n, k, nz, d_lw, eq, part);
  WL_LAUNCH_CHECK();
  launch_reduce_partials(part, nb0, nz, red, st);
  ef sums[16];
  d2h(sums, red, sizeof(ef) * nz, st);
  ef ys[MAXC], p[MAXC], q[MAXC], pq[2 * MAXC];
  const int npts = nsk + nz;
  for (int i = 0; i < nsk; i++) ys[i] = kb::ef_zero();
  for (int i = 0; i < nz; i++) ys[nsk + i] = sums[i];
  interpolate_fixed(ys, npts, p);
  ef qv[16];
  selectors_at(nsk, r[0], qv);
  interpolate_fixed(qv, nsk, q);
  int np = poly_mul_fixed(p, npts, q, nsk, pq);
  const int deg = 3 * (nsk - 1);
  for (int i = np; i <= deg; i++) pq[i] = kb::ef_zero();
  ts.add_ext(pq, deg + 1);
  ef ch = ts.sample_ext();
  ef sum = poly_eval_fixed(pq, deg + 1, ch);
  if (sumcheck_pow_bits(128, deg) != 0) throw std::logic_error("unexpected grinding in the sumcheck");
  ef selr[16];
  selectors_at(nsk, ch, selr);
  ef mmf = kb::ef_zero();
  for (int i = 0; i < nsk; i++) mmf = kb::ef_add(mmf, kb::ef_mul(qv[i], selr[i]));
  h2d(d_sel, selr, sizeof(ef) * nsk, st);
  k_abc0_fold_canon<<<dim3((unsigned)((S + 255) / 256), 3), 256, 0, st>>>(a, b, c, n, k, d_sel, cols);
  WL_LAUNCH_CHECK();
  // rounds >= 1
  for (int round = 1; round <= n - k; round++) {
    const int m = n - k - round + 1;
    const size_t half = size_t(1) << (m - 1);
    launch_eq_table(d_r + 1 + round, m - 1, eq, st);
    if (m - 1 == 0) {
      const ef one = kb::ef_one();
      h2d(eq, &one, sizeof(ef), st);
    }
    const int nb = (int)((half + 31) / 32);
    launch_abc_eval_ef(cols, m, eq, part, st);
    launch_reduce_partials(part, nb, 2, red, st);
    ef s2[2];
    d2h(s2, red, sizeof(s2), st);
    const ef& rr = r[round];
    ef v[3];
    v[0] = kb::ef_mul(s2[0], mmf);
    v[2] = kb::ef_mul(s2[1], mmf);
    v[1] = kb::ef_mul(kb::ef_sub(sum, kb::ef_mul(v[0], kb::ef_sub(kb::ef_one(), rr))), kb::ef_inv(rr));
    ef p3[3], lin[2], p4[4];
    interpolate_fixed(v, 3, p3);
    lin[0] = kb::ef_sub(kb::ef_one(), rr);
    lin[1] = kb::ef_sub(kb::ef_add(rr, rr), kb::ef_one());
    poly_mul_fixed(p3, 3, lin, 2, p4);
    ts.add_ext(p4, 4);
    ef cc = ts.sample_ext();
    sum = poly_eval_fixed(p4, 4, cc);
    mmf = kb::ef_mul(
        kb::ef_add(kb::ef_mul(kb::ef_sub(kb::ef_one(), rr), kb::ef_sub(kb::ef_one(), cc)), kb::ef_mul(rr, cc)), mmf);
    h2d(d_ch, &cc, sizeof(ef), st);
    launch_fold_cols(cols, cols2, 3, half, d_ch, st);
    ef* t = cols;
    cols = cols2;
    cols2 = t;
  }
  ef fin[3];
  d2h(fin, cols, sizeof(fin), st);
  ts.add_ext(fin, 3);
}

}  // namespace
}  // namespace wl

extern "C" wl_status wl_sumcheck_abc_prove_noalloc(const uint32_t* p16_constants, int32_t log_n, int32_t skips,
                                                   const uint32_t* a_dev, const uint32_t* b_dev,
                                                   const uint32_t* c_dev, uint32_t* proof_out, size_t* proof_len,
                                                   void* stream) {
  if (!p16_constants || !a_dev || !b_dev || !c_dev || !proof_len || skips < 1 || skips > 4 || skips >= log_n ||
      log_n < 2)
    return WL_E_INVALID_ARG;
  if (log_n > wl::NOALLOC_MAX_LOG_N) return WL_E_SCRATCH_LIMIT;
  const size_t need = wl::abc_proof_len(log_n, skips);
  if (!proof_out || *proof_len < need) {
    *proof_len = need;
    return WL_E_BUFFER_TOO_SMALL;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) {
    cudaGetLastError();
    return WL_E_INVALID_ARG;
  }
  if (cap != cudaStreamCaptureStatusNone) return WL_E_INVALID_ARG;  // host round trips cannot be captured
  try {
    void* base = nullptr;
    if (wl::scratch_base(&base) != cudaSuccess || !base) return WL_E_CUDA;
    wl::Arena ar{static_cast<unsigned char*>(base)};
    const kb::P16Consts p16 = wl::perm_consts_from<16>(p16_constants);
    wl::FixedTranscript ts{wl::HostChallenger{}, proof_out, *proof_len};
    wl::prove_abc_fixed(p16, log_n, skips, a_dev, b_dev, c_dev, ar, ts, st);
    *proof_len = ts.len;
    return WL_OK;
  } catch (const wl::CudaError&) {
    return WL_E_CUDA;
  } catch (const std::length_error&) {
    return WL_E_SCRATCH_LIMIT;
  } catch (...) {
    return WL_E_INTERNAL;
  }
}
