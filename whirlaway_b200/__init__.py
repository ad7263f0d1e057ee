"""B200 prover path for Whirlaway's Poseidon2-KoalaBear AIR.

A thin Python face over the C ABI in include/whirlaway_b200.h, shaped like the reference's
Rust API: ``AirSettings`` (crates/air/src/lib.rs:13-41), ``AirTable.prove`` /
``AirTable.verify`` (crates/air/src/prove.rs:49-66, verify.rs:55-69) and the standalone
``sumcheck`` prover (crates/sumcheck/src/prove.rs:22-35). All compute runs in the CUDA
library built from ``csrc/``; there is no CPU fallback, and loading fails loudly when the
library is missing.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, astuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libwhirlaway_b200.so")

_u32p = ctypes.POINTER(ctypes.c_uint32)
_sizep = ctypes.POINTER(ctypes.c_size_t)

STATUS = {
    0: "OK", 1: "INVALID_ARG", 2: "CUDA", 3: "OOM", 4: "BUFFER_TOO_SMALL", 5: "INTERNAL", 6: "BUDGET",
    11: "INVALID_PCS_COMMITMENT", 12: "INVALID_PCS_OPENING", 13: "FS", 14: "SUMCHECK", 15: "BOUNDARY",
    16: "SUM_MISMATCH", 7: "SCRATCH_LIMIT",
}


class ProverError(RuntimeError):
    """A non-OK wl_status from the library."""

    def __init__(self, status: int, message: str = ""):
        self.status = status
        super().__init__(f"{STATUS.get(status, status)}: {message}")


class _AirProgram(ctypes.Structure):
    _fields_ = [("n_columns", ctypes.c_int32), ("n_constraints", ctypes.c_int32),
                ("constraint_degree", ctypes.c_int32), ("n_ops", ctypes.c_int32),
                ("ops", ctypes.POINTER(ctypes.c_int32)), ("n_consts", ctypes.c_int32),
                ("consts", ctypes.POINTER(ctypes.c_uint32)), ("n_preprocessed", ctypes.c_int32),
                ("preprocessed", ctypes.POINTER(ctypes.c_uint32))]


def _program_c(prog, preprocessed, log_n):
    """The C description of an air_program.AirProgram and its preprocessed columns (returns the
    struct and the array it points into, which the caller keeps alive)."""
    pre = np.zeros(1, np.uint32)
    if prog.n_preprocessed:
        if preprocessed is None:
            raise ValueError("the program has preprocessed columns: pass their values")
        pre = np.ascontiguousarray(preprocessed, dtype=np.uint32).reshape(-1)
        if pre.size != prog.n_preprocessed << log_n:
            raise ValueError("preprocessed must hold n_preprocessed columns of 2^log_n values")
    c = _AirProgram(prog.width, prog.n_constraints, prog.degree, prog.ops.shape[0],
                    prog.ops.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), prog.consts.size,
                    prog.consts.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), prog.n_preprocessed,
                    pre.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
    return c, pre


class _Settings(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in (
        "security_bits", "log_inv_rate", "fold_first", "fold_rest", "univariate_skips",
        "rs_domain_initial_reduction", "whir_pow_bits")]


@dataclass(frozen=True)
class AirSettings:
    """AirSettings with the reference defaults of src/main.rs:13-24."""
    security_bits: int = 128
    log_inv_rate: int = 1
    fold_first: int = 7
    fold_rest: int = 4
    univariate_skips: int = 4
    rs_domain_initial_reduction: int = 5
    whir_pow_bits: int = 16

    def _c(self) -> _Settings:
        return _Settings(*astuple(self))

    def as_array(self) -> np.ndarray:
        return np.array(astuple(self), dtype=np.int32)


_lib = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"CUDA library not built: {path} (run whirlaway_b200.build.build())")
    lib = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    sig = {
        "wl_air_columns": (ctypes.c_int32, []),
        "wl_constants_len": (ctypes.c_int32, []),
        "wl_ctx_create": (ctypes.c_int, [ctypes.c_int32, ctypes.c_uint64, ctypes.POINTER(vp)]),
        "wl_ctx_destroy": (None, [vp]),
        "wl_last_error": (ctypes.c_char_p, [vp]),
        "wl_generate_workload": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int64, _u32p, _u32p]),
        "wl_witness_upload": (ctypes.c_int, [vp, ctypes.c_int32, _u32p, ctypes.POINTER(vp)]),
        "wl_witness_generate": (ctypes.c_int, [vp, _u32p, ctypes.c_int32, _u32p, ctypes.POINTER(vp)]),
        "wl_witness_download": (ctypes.c_int, [vp, vp, _u32p]),
        "wl_witness_free": (None, [vp, vp]),
        "wl_proof_len_bound": (ctypes.c_int, [ctypes.POINTER(_Settings), ctypes.c_int32, _sizep]),
        "wl_prove": (ctypes.c_int, [vp, ctypes.POINTER(_Settings), _u32p, ctypes.c_int32, _u32p, _u32p, _sizep,
                                    ctypes.POINTER(ctypes.c_double)]),
        "wl_prove_witness": (ctypes.c_int, [vp, ctypes.POINTER(_Settings), _u32p, vp, _u32p, _sizep,
                                            ctypes.POINTER(ctypes.c_double)]),
        "wl_prove_batch": (ctypes.c_int, [vp, ctypes.POINTER(_Settings), _u32p, ctypes.c_int32,
                                          ctypes.POINTER(vp), _u32p, ctypes.c_size_t, _sizep]),
        "wl_sumcheck_abc_prove": (ctypes.c_int, [vp, _u32p, ctypes.c_int32, ctypes.c_int32, _u32p, _u32p, _u32p,
                                                 _u32p, _sizep, ctypes.POINTER(ctypes.c_float)]),
        "wl_sumcheck_abc_prove_device": (ctypes.c_int, [vp, _u32p, ctypes.c_int32, ctypes.c_int32, vp, vp, vp,
                                                        _u32p, _sizep, ctypes.POINTER(ctypes.c_float)]),
        "wl_ctx_stream": (vp, [vp]),
        "wl_kernel_launch_count": (ctypes.c_uint64, []),
        "wl_sumcheck_abc_prove_noalloc": (ctypes.c_int, [_u32p, ctypes.c_int32, ctypes.c_int32, vp, vp, vp, _u32p,
                                                         _sizep, vp]),
        "wl_proof_footprint_bytes": (ctypes.c_uint64, [ctypes.POINTER(_Settings), ctypes.c_int32]),
        "wl_verify": (ctypes.c_int, [ctypes.POINTER(_Settings), _u32p, ctypes.c_int32, _u32p, ctypes.c_size_t]),
        "wl_prove_program": (ctypes.c_int, [vp, ctypes.POINTER(_Settings), _u32p, ctypes.POINTER(_AirProgram),
                                            ctypes.c_int32, _u32p, _u32p, _sizep]),
        "wl_verify_program": (ctypes.c_int, [ctypes.POINTER(_Settings), _u32p, ctypes.POINTER(_AirProgram),
                                             ctypes.c_int32, _u32p, ctypes.c_size_t]),
        "wl_program_proof_len_bound": (ctypes.c_int, [ctypes.POINTER(_Settings), ctypes.POINTER(_AirProgram),
                                                      ctypes.c_int32, _sizep]),
        "wl_sumcheck_abc_verify": (ctypes.c_int, [_u32p, ctypes.c_int32, ctypes.c_int32, _u32p, ctypes.c_size_t]),
        "wl_verify_batch": (ctypes.c_int, [ctypes.POINTER(_Settings), _u32p, ctypes.c_int32,
                                           ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(_u32p), _sizep,
                                           ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]),
        "wl_ctx_set_transcript_dump": (ctypes.c_int, [vp, ctypes.c_int32]),
        "wl_transcript_dump": (ctypes.c_int, [vp, ctypes.c_char_p, _sizep]),
        "wl_verify_transcript": (ctypes.c_int, [ctypes.POINTER(_Settings), _u32p, ctypes.c_int32, _u32p,
                                                ctypes.c_size_t, ctypes.c_char_p, _sizep]),
        "wl_server_create": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_uint64, ctypes.POINTER(vp)]),
        "wl_server_destroy": (None, [vp]),
        "wl_server_last_error": (ctypes.c_char_p, [vp]),
        "wl_server_submit": (ctypes.c_int, [vp, ctypes.POINTER(_Settings), _u32p, ctypes.c_int32, _u32p,
                                            ctypes.POINTER(ctypes.c_uint64)]),
        "wl_server_poll": (ctypes.c_int, [vp, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int32)]),
        "wl_server_wait": (ctypes.c_int, [vp, ctypes.c_uint64, _u32p, _sizep, ctypes.POINTER(ctypes.c_double)]),
        "wl_server_stats": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_int32)]),
        "wl_profile_enable": (ctypes.c_int, [vp, ctypes.c_int32]),
        "wl_profile_json": (ctypes.c_int, [vp, ctypes.c_char_p, ctypes.c_size_t]),
        "wl_ctx_host_syncs": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_uint64)]),
        "wl_ctx_set_spin_sync": (ctypes.c_int, [vp, ctypes.c_int32]),
        "wl_ctx_set_autotune": (ctypes.c_int, [vp, ctypes.c_int32]),
        "wl_verify_batch_device": (ctypes.c_int, [vp, ctypes.POINTER(_Settings), _u32p, ctypes.c_int32,
                                                  ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(_u32p), _sizep,
                                                  ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]),
        "wl_tune_force": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int32]),
        "wl_tune_report": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_size_t)]),
        "wl_tune_clear": (ctypes.c_int, []),
        "wl_ctx_host_wait_ms": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_double)]),
        "wl_profile_only": (ctypes.c_int, [vp, ctypes.c_char_p]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _ptr(a: np.ndarray):
    assert a.dtype == np.uint32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_u32p)


def kernel_launch_count() -> int:
    """Kernels launched by the library in this process."""
    return load_library().wl_kernel_launch_count()


def air_columns() -> int:
    return load_library().wl_air_columns()


def constants_len() -> int:
    return load_library().wl_constants_len()


def generate_workload(log_n: int, input_seed: int = -1, with_inputs: bool = True):
    """Constants blob and row-major inputs of src/examples/poseidon2.rs:104-151."""
    lib = load_library()
    consts = np.zeros(constants_len(), np.uint32)
    inputs = np.zeros(16 << log_n, np.uint32) if with_inputs else None
    st = lib.wl_generate_workload(log_n, input_seed, _ptr(consts), _ptr(inputs) if with_inputs else None)
    if st:
        raise ProverError(st, "generate_workload")
    return consts, inputs


class Context:
    """One CUDA device; owns the stream, the twiddle table and pooled device memory."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0):
        self._lib = load_library()
        h = ctypes.c_void_p()
        st = self._lib.wl_ctx_create(device, hbm_budget_bytes, ctypes.byref(h))
        if st:
            raise ProverError(st, f"wl_ctx_create(device={device})")
        self.handle = h

    def check(self, st: int, what: str):
        if st:
            msg = self._lib.wl_last_error(self.handle).decode(errors="replace")
            raise ProverError(st, f"{what}: {msg}")

    @property
    def stream_ptr(self) -> int:
        """Raw cudaStream_t the library launches on (for torch.cuda.ExternalStream)."""
        return self._lib.wl_ctx_stream(self.handle) or 0

    def profile(self, on: bool = True, only: str | None = None):
        """Starts (or stops) per-kernel-class CUDA-event timing; totals restart. With `only`,
        just that kernel class is timed."""
        self.check(self._lib.wl_profile_only(self.handle, (only or "").encode()), "profile_only")
        self.check(self._lib.wl_profile_enable(self.handle, int(on)), "profile_enable")

    def profile_report(self) -> dict:
        """{kernel class: (total ms, launches)} since profiling was enabled."""
        import json
        buf = ctypes.create_string_buffer(1 << 16)
        self.check(self._lib.wl_profile_json(self.handle, buf, len(buf)), "profile_json")
        return {k: tuple(v) for k, v in json.loads(buf.value.decode()).items()}

    def set_spin_sync(self, spin: bool = True):
        """Busy-poll (True, the default) or block (False) at each host round trip."""
        self.check(self._lib.wl_ctx_set_spin_sync(self.handle, int(spin)), "set_spin_sync")

    def set_autotune(self, on: bool = True):
        """Tunes the commitment's launch plans on the first proof of each table shape."""
        self.check(self._lib.wl_ctx_set_autotune(self.handle, int(on)), "set_autotune")

    def set_transcript_dump(self, on: bool = True):
        """Records a per-phase transcript dump of every later proof on this context."""
        self.check(self._lib.wl_ctx_set_transcript_dump(self.handle, int(on)), "set_transcript_dump")

    def transcript_dump(self) -> dict:
        """The dump of the last proof (after set_transcript_dump(True))."""
        import json
        st, text = _text_call(self._lib.wl_transcript_dump, self.handle)
        self.check(st, "transcript_dump")
        return json.loads(text)

    @property
    def host_syncs(self) -> int:
        """Host synchronisations of this context's stream so far."""
        v = ctypes.c_uint64()
        self.check(self._lib.wl_ctx_host_syncs(self.handle, ctypes.byref(v)), "host_syncs")
        return v.value

    @property
    def host_wait_ms(self) -> float:
        """Milliseconds the host has spent waiting for this context's stream."""
        v = ctypes.c_double()
        self.check(self._lib.wl_ctx_host_wait_ms(self.handle, ctypes.byref(v)), "host_wait_ms")
        return v.value

    def close(self):
        if getattr(self, "handle", None):
            self._lib.wl_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Witness:
    """Device-resident witness: 165 columns of 2^log_n values."""

    def __init__(self, ctx: Context, handle: ctypes.c_void_p, log_n: int):
        self.ctx, self.handle, self.log_n = ctx, handle, log_n

    @classmethod
    def upload(cls, ctx: Context, witness_colmajor: np.ndarray, log_n: int) -> "Witness":
        w = np.ascontiguousarray(witness_colmajor, dtype=np.uint32).reshape(-1)
        if w.size != air_columns() << log_n:
            raise ValueError("witness must hold 165 columns of 2^log_n values")
        h = ctypes.c_void_p()
        ctx.check(ctx._lib.wl_witness_upload(ctx.handle, log_n, _ptr(w), ctypes.byref(h)), "witness_upload")
        return cls(ctx, h, log_n)

    @classmethod
    def generate(cls, ctx: Context, constants: np.ndarray, inputs: np.ndarray, log_n: int) -> "Witness":
        h = ctypes.c_void_p()
        ctx.check(ctx._lib.wl_witness_generate(ctx.handle, _ptr(constants), log_n, _ptr(inputs), ctypes.byref(h)),
                  "witness_generate")
        return cls(ctx, h, log_n)

    def download(self) -> np.ndarray:
        out = np.zeros(air_columns() << self.log_n, np.uint32)
        self.ctx.check(self.ctx._lib.wl_witness_download(self.ctx.handle, self.handle, _ptr(out)), "download")
        return out

    def free(self):
        if self.handle:
            self.ctx._lib.wl_witness_free(self.ctx.handle, self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def proof_len_bound(settings: AirSettings, log_n: int) -> int:
    n = ctypes.c_size_t()
    st = load_library().wl_proof_len_bound(ctypes.byref(settings._c()), log_n, ctypes.byref(n))
    if st:
        raise ProverError(st, "proof_len_bound")
    return n.value


class AirTable:
    """The Poseidon2-KoalaBear AIR table (crates/air/src/table.rs:15-99) bound to a device."""

    def __init__(self, ctx: Context, constants: np.ndarray, log_n: int, settings: AirSettings = AirSettings()):
        self.ctx, self.log_n, self.settings = ctx, log_n, settings
        self.constants = np.ascontiguousarray(constants, dtype=np.uint32)
        self.last_timings_ms = None

    def _call(self, fn, *args):
        cap = proof_len_bound(self.settings, self.log_n)
        out = np.zeros(cap, np.uint32)
        n = ctypes.c_size_t(cap)
        tm = (ctypes.c_double * 5)()
        self.ctx.check(fn(self.ctx.handle, ctypes.byref(self.settings._c()), _ptr(self.constants), *args, _ptr(out),
                          ctypes.byref(n), tm), fn.__name__)
        self.last_timings_ms = dict(zip(("commit", "zerocheck", "inner", "whir", "total"), list(tm)))
        return out[: n.value].copy()

    def prove(self, witness_colmajor: np.ndarray) -> np.ndarray:
        """AirTable::prove with a host witness; returns proof_data (canonical u32)."""
        w = np.ascontiguousarray(witness_colmajor, dtype=np.uint32).reshape(-1)
        if w.size != air_columns() << self.log_n:
            raise ValueError("witness must hold 165 columns of 2^log_n values")
        return self._call(self.ctx._lib.wl_prove, self.log_n, _ptr(w))

    def prove_witness(self, w: Witness) -> np.ndarray:
        """AirTable::prove with a device-resident witness."""
        if w.log_n != self.log_n:
            raise ValueError("witness height does not match the table")
        return self._call(self.ctx._lib.wl_prove_witness, w.handle)


def prove_program(ctx: Context, hash_constants: np.ndarray, program, log_n: int, witness_colmajor: np.ndarray,
                  settings: AirSettings = AirSettings(), preprocessed=None) -> np.ndarray:
    """AirTable::prove for an AIR given as a constraint program (air_program.AirProgram) with a
    host witness (the program's witness columns, width - n_preprocessed of them, 2^log_n
    canonical values each, column-major) and the values of its preprocessed columns, if any;
    hash_constants: the Poseidon16 | Poseidon24 constants (363 u32). Returns proof_data."""
    lib = ctx._lib
    pc, keep = _program_c(program, preprocessed, log_n)
    hc = np.ascontiguousarray(hash_constants, dtype=np.uint32)
    w = np.ascontiguousarray(witness_colmajor, dtype=np.uint32).reshape(-1)
    if w.size != (program.width - program.n_preprocessed) << log_n:
        raise ValueError("witness must hold the program's witness columns of 2^log_n values")
    cap = ctypes.c_size_t()
    ctx.check(lib.wl_program_proof_len_bound(ctypes.byref(settings._c()), ctypes.byref(pc), log_n, ctypes.byref(cap)),
              "program_proof_len_bound")
    out = np.zeros(cap.value, np.uint32)
    n = ctypes.c_size_t(cap.value)
    ctx.check(lib.wl_prove_program(ctx.handle, ctypes.byref(settings._c()), _ptr(hc), ctypes.byref(pc), log_n, _ptr(w),
                                   _ptr(out), ctypes.byref(n)), "prove_program")
    return out[: n.value].copy()


def verify_program(hash_constants: np.ndarray, program, log_n: int, proof: np.ndarray,
                   settings: AirSettings = AirSettings(), preprocessed=None) -> int:
    """AirTable::verify for a constraint-program AIR on the host: 0 when accepted, else the
    verifier status (as verify)."""
    pc, keep = _program_c(program, preprocessed, log_n)
    hc = np.ascontiguousarray(hash_constants, dtype=np.uint32)
    pr = np.ascontiguousarray(proof, dtype=np.uint32)
    return load_library().wl_verify_program(ctypes.byref(settings._c()), _ptr(hc), ctypes.byref(pc), log_n, _ptr(pr),
                                            pr.size)


def sumcheck_abc_prove(ctx: Context, p16_constants: np.ndarray, log_n: int, skips: int, a, b, c, device=False):
    """Zerocheck of eq(r, x) * (a*b - c) with a univariate skip; returns (proof, per-round ms)."""
    lib = ctx._lib
    cap = 8 * (3 * ((1 << skips) - 1) + 1 + 4 * (log_n - skips) + 3) + 64
    out = np.zeros(cap, np.uint32)
    n = ctypes.c_size_t(cap)
    ms = (ctypes.c_float * (log_n - skips + 1))()
    p16 = np.ascontiguousarray(p16_constants, dtype=np.uint32)
    if device:
        ptrs = [ctypes.c_void_p(int(t.data_ptr())) for t in (a, b, c)]
        st = lib.wl_sumcheck_abc_prove_device(ctx.handle, _ptr(p16), log_n, skips, *ptrs, _ptr(out), ctypes.byref(n),
                                              ms)
    else:
        arrs = [np.ascontiguousarray(t, dtype=np.uint32) for t in (a, b, c)]
        st = lib.wl_sumcheck_abc_prove(ctx.handle, _ptr(p16), log_n, skips, *[_ptr(t) for t in arrs], _ptr(out),
                                       ctypes.byref(n), ms)
    ctx.check(st, "sumcheck_abc_prove")
    return out[: n.value].copy(), list(ms)


def sumcheck_abc_prove_noalloc(p16_constants: np.ndarray, log_n: int, skips: int, a, b, c, stream: int = 0):
    """Allocation-free zerocheck of eq(r, x) * (a*b - c) for callers that cannot allocate
    device memory; a, b, c are CUDA tensors of canonical values (log_n <= 14)."""
    lib = load_library()
    n = ctypes.c_size_t(0)
    p16 = np.ascontiguousarray(p16_constants, dtype=np.uint32)
    ptrs = [ctypes.c_void_p(int(t.data_ptr())) for t in (a, b, c)]
    st = lib.wl_sumcheck_abc_prove_noalloc(_ptr(p16), log_n, skips, *ptrs, None, ctypes.byref(n), ctypes.c_void_p(stream))
    if st != 4:
        raise ProverError(st, "sumcheck_abc_prove_noalloc (length query)")
    out = np.zeros(n.value, np.uint32)
    st = lib.wl_sumcheck_abc_prove_noalloc(_ptr(p16), log_n, skips, *ptrs, _ptr(out), ctypes.byref(n),
                                           ctypes.c_void_p(stream))
    if st:
        raise ProverError(st, "sumcheck_abc_prove_noalloc")
    return out[: n.value].copy()


def verify(constants: np.ndarray, log_n: int, proof: np.ndarray, settings: AirSettings = AirSettings()) -> int:
    """AirTable::verify on the host CPU (no device): 0 when the proof is accepted, else the
    verifier status (11 commitment, 12 opening, 13 Fiat-Shamir, 14 sumcheck, 16 sum mismatch;
    1 for bad arguments)."""
    c = np.ascontiguousarray(constants, dtype=np.uint32)
    pr = np.ascontiguousarray(proof, dtype=np.uint32)
    return load_library().wl_verify(ctypes.byref(settings._c()), _ptr(c), log_n, _ptr(pr), pr.size)


def verify_batch(constants: np.ndarray, jobs, settings: AirSettings = AirSettings(), threads: int = 0):
    """wl_verify over [(log_n, proof), ...] on host threads; returns the list of statuses."""
    c = np.ascontiguousarray(constants, dtype=np.uint32)
    prs = [np.ascontiguousarray(p, dtype=np.uint32) for _, p in jobs]
    n = len(jobs)
    log_ns = (ctypes.c_int32 * n)(*[int(l) for l, _ in jobs])
    ptrs = (_u32p * n)(*[_ptr(p) for p in prs])
    lens = (ctypes.c_size_t * n)(*[p.size for p in prs])
    out = (ctypes.c_int32 * n)()
    st = load_library().wl_verify_batch(ctypes.byref(settings._c()), _ptr(c), n, log_ns, ptrs, lens, threads, out)
    if st:
        raise ProverError(st, "verify_batch")
    return list(out)


def _text_call(fn, *args):
    n = ctypes.c_size_t(1 << 20)
    for _ in range(2):
        buf = ctypes.create_string_buffer(n.value)
        st = fn(*args, buf, ctypes.byref(n))
        if st != 4:  # not WL_E_BUFFER_TOO_SMALL
            return st, buf.value.decode()
    raise ProverError(st, "transcript dump")


def verify_batch_device(ctx, constants: np.ndarray, jobs, settings: AirSettings = AirSettings(), threads: int = 0):
    """wl_verify_batch with the Merkle paths of all proofs checked in one GPU kernel on `ctx`'s
    device (the transcripts replay on host threads); returns the list of statuses."""
    c = np.ascontiguousarray(constants, dtype=np.uint32)
    prs = [np.ascontiguousarray(p, dtype=np.uint32) for _, p in jobs]
    n = len(jobs)
    log_ns = (ctypes.c_int32 * n)(*[int(l) for l, _ in jobs])
    ptrs = (_u32p * n)(*[_ptr(p) for p in prs])
    lens = (ctypes.c_size_t * n)(*[p.size for p in prs])
    out = (ctypes.c_int32 * n)()
    ctx.check(ctx._lib.wl_verify_batch_device(ctx.handle, ctypes.byref(settings._c()), _ptr(c), n, log_ns, ptrs, lens,
                                              threads, out), "verify_batch_device")
    return list(out)


def verify_transcript(constants: np.ndarray, log_n: int, proof: np.ndarray, settings: AirSettings = AirSettings()):
    """Runs the host verifier and returns (status, transcript dump as read by the verifier)."""
    import json
    c = np.ascontiguousarray(constants, dtype=np.uint32)
    pr = np.ascontiguousarray(proof, dtype=np.uint32)
    st, text = _text_call(load_library().wl_verify_transcript, ctypes.byref(settings._c()), _ptr(c), log_n,
                          _ptr(pr), pr.size)
    return st, json.loads(text)


def sumcheck_abc_verify(p16_constants: np.ndarray, log_n: int, skips: int, proof: np.ndarray) -> int:
    """Verifies a sumcheck_abc_prove proof on the host CPU; 0 when accepted."""
    c = np.ascontiguousarray(p16_constants, dtype=np.uint32)
    pr = np.ascontiguousarray(proof, dtype=np.uint32)
    return load_library().wl_sumcheck_abc_verify(_ptr(c), log_n, skips, _ptr(pr), pr.size)


def tune_force(family: str, plan: int):
    """Pins an autotuned family ("lde", "leaf", "merkle") to one plan (-1: tune again)."""
    st = load_library().wl_tune_force(family.encode(), plan)
    if st:
        raise ProverError(st, "tune_force")


def tune_report() -> dict:
    """The autotuner's kept plans: {family: [{device, key, plan, ms}, ...]}."""
    import json
    lib = load_library()
    n = ctypes.c_size_t(0)
    lib.wl_tune_report(None, ctypes.byref(n))
    buf = ctypes.create_string_buffer(n.value)
    st = lib.wl_tune_report(buf, ctypes.byref(n))
    if st:
        raise ProverError(st, "tune_report")
    return json.loads(buf.value.decode())


def tune_clear():
    load_library().wl_tune_clear()


def proof_footprint_bytes(log_n: int, settings: AirSettings = AirSettings()) -> int:
    """Device bytes the server reserves for one proof of 2^log_n rows under `settings`."""
    return load_library().wl_proof_footprint_bytes(ctypes.byref(settings._c()), log_n)


class Server:
    """Concurrent proving on one device: `workers` proofs in flight, FIFO admission by
    estimated HBM footprint against `hbm_budget_bytes` (0: unbounded)."""

    QUEUED, RUNNING, DONE, FAILED = 0, 1, 2, 3

    def __init__(self, device: int = 0, workers: int = 8, hbm_budget_bytes: int = 0):
        self._lib = load_library()
        h = ctypes.c_void_p()
        st = self._lib.wl_server_create(device, workers, hbm_budget_bytes, ctypes.byref(h))
        if st:
            raise ProverError(st, f"wl_server_create(device={device}, workers={workers})")
        self.handle = h

    def _check(self, st, what):
        if st:
            raise ProverError(st, f"{what}: {self._lib.wl_server_last_error(self.handle).decode(errors='replace')}")

    def submit(self, constants: np.ndarray, inputs: np.ndarray, log_n: int, settings: AirSettings = AirSettings()):
        t = ctypes.c_uint64()
        c = np.ascontiguousarray(constants, dtype=np.uint32)
        i = np.ascontiguousarray(inputs, dtype=np.uint32)
        if i.size != 16 << log_n:
            raise ValueError("inputs must hold 16 values per row")
        self._check(self._lib.wl_server_submit(self.handle, ctypes.byref(settings._c()), _ptr(c), log_n, _ptr(i),
                                               ctypes.byref(t)), "submit")
        return t.value

    def poll(self, ticket: int) -> int:
        s = ctypes.c_int32()
        self._check(self._lib.wl_server_poll(self.handle, ticket, ctypes.byref(s)), "poll")
        return s.value

    def wait(self, ticket: int, log_n: int, settings: AirSettings = AirSettings()):
        """Blocks until done; returns (proof, {queued_ms, run_ms, latency_ms})."""
        cap = proof_len_bound(settings, log_n)
        out = np.zeros(cap, np.uint32)
        n = ctypes.c_size_t(cap)
        tm = (ctypes.c_double * 3)()
        self._check(self._lib.wl_server_wait(self.handle, ticket, _ptr(out), ctypes.byref(n), tm), "wait")
        return out[: n.value].copy(), {"queued_ms": tm[0], "run_ms": tm[1], "latency_ms": tm[2]}

    def stats(self):
        b, r = ctypes.c_uint64(), ctypes.c_int32()
        self._check(self._lib.wl_server_stats(self.handle, ctypes.byref(b), ctypes.byref(r)), "stats")
        return {"peak_bytes_admitted": b.value, "peak_running": r.value}

    def close(self):
        if getattr(self, "handle", None):
            self._lib.wl_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def batch_prove(server: Server, jobs, settings: AirSettings = AirSettings()):
    """Proves independent jobs [(constants, inputs, log_n), ...] concurrently; returns the
    proofs in job order."""
    tickets = [server.submit(c, i, n, settings) for c, i, n in jobs]
    return [server.wait(t, n, settings)[0] for t, (_, _, n) in zip(tickets, jobs)]
