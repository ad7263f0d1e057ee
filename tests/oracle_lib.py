"""ctypes binding of the CPU oracle (oracle/_build/liboracle.so).

Test infrastructure only: the oracle is the checker the CUDA path is compared with.
"""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_build", "liboracle.so")
_u32p = ctypes.POINTER(ctypes.c_uint32)
_i32p = ctypes.POINTER(ctypes.c_int32)


def _p(a):
    return a.ctypes.data_as(_u32p) if a is not None else None


class Oracle:
    def __init__(self, lib):
        self.lib = lib
        lib.wlo_workload.argtypes = [ctypes.c_int, ctypes.c_int64, _u32p, _u32p]
        lib.wlo_trace.argtypes = [ctypes.c_int, _u32p, _u32p, _u32p]
        lib.wlo_prove.argtypes = [_i32p, _u32p, ctypes.c_int, _u32p, _u32p, ctypes.POINTER(ctypes.c_size_t),
                                  ctypes.POINTER(ctypes.c_double)]
        lib.wlo_verify.argtypes = [_i32p, _u32p, ctypes.c_int, _u32p, ctypes.c_size_t]
        lib.wlo_prove_abc.argtypes = [_u32p, ctypes.c_int, ctypes.c_int, _u32p, _u32p, _u32p, _u32p,
                                      ctypes.POINTER(ctypes.c_size_t)]
        lib.wlo_verify_abc.argtypes = [_u32p, ctypes.c_int, ctypes.c_int, _u32p, ctypes.c_size_t]
        prog_args = [_i32p, _u32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _i32p, ctypes.c_int, _u32p,
                     ctypes.c_int, _u32p, ctypes.c_int]
        lib.wlo_prove_program.argtypes = prog_args + [_u32p, _u32p, ctypes.POINTER(ctypes.c_size_t)]
        lib.wlo_verify_program.argtypes = prog_args + [_u32p, ctypes.c_size_t]
        lib.wlo_chacha_block.argtypes = [_u32p, ctypes.c_uint64, ctypes.c_int, _u32p]
        lib.wlo_stdrng_u32.argtypes = [ctypes.c_uint64, _u32p, ctypes.c_size_t]
        lib.wlo_poseidon2.argtypes = [ctypes.c_int, _u32p, _u32p]
        lib.wlo_ef_mul.argtypes = [_u32p, _u32p, _u32p]
        lib.wlo_ef_inv.argtypes = [_u32p, _u32p]
        lib.wlo_ntt.argtypes = [_u32p, ctypes.c_size_t, ctypes.c_int, _u32p]
        lib.wlo_whir_config.argtypes = [ctypes.c_int, _i32p, _i32p, ctypes.c_int]
        lib.wlo_set_threads.argtypes = [ctypes.c_int]
        self.ncons = lib.wlo_constants_size()
        self.cols = lib.wlo_air_cols()

    def workload(self, log_n, input_seed=-1):
        c = np.zeros(self.ncons, np.uint32)
        i = np.zeros(16 << log_n, np.uint32)
        assert self.lib.wlo_workload(log_n, input_seed, _p(c), _p(i)) == 0
        return c, i

    def trace(self, log_n, consts, inputs):
        w = np.zeros(self.cols << log_n, np.uint32)
        self.lib.wlo_trace(log_n, _p(consts), _p(inputs), _p(w))
        return w

    def prove(self, log_n, consts, witness, settings=None):
        cap = 1 << 22
        out = np.zeros(cap, np.uint32)
        n = ctypes.c_size_t(cap)
        t = (ctypes.c_double * 4)()
        s = settings.ctypes.data_as(_i32p) if settings is not None else None
        rc = self.lib.wlo_prove(s, _p(consts), log_n, _p(witness), _p(out), ctypes.byref(n), t)
        assert rc == 0, rc
        return out[: n.value].copy(), list(t)

    def verify(self, log_n, consts, proof, settings=None):
        s = settings.ctypes.data_as(_i32p) if settings is not None else None
        proof = np.ascontiguousarray(proof, dtype=np.uint32)
        return self.lib.wlo_verify(s, _p(consts), log_n, _p(proof), proof.size)

    def _program_args(self, settings, hash_consts, prog, log_n, preprocessed):
        s = settings.ctypes.data_as(_i32p) if settings is not None else None
        hc = np.ascontiguousarray(hash_consts, np.uint32)
        pre = np.ascontiguousarray(preprocessed if preprocessed is not None else np.zeros(1, np.uint32), np.uint32)
        npre = 0 if preprocessed is None else pre.size >> log_n
        return [s, _p(hc), prog.width, prog.n_constraints, prog.degree, prog.ops.shape[0],
                prog.ops.ctypes.data_as(_i32p), prog.consts.size, _p(prog.consts), npre, _p(pre), log_n], (hc, pre)

    def prove_program(self, log_n, hash_consts, prog, witness, settings=None, preprocessed=None):
        """A proof for the AIR given as a constraint program (hash_consts: P16 | P24 constants);
        preprocessed: its first columns' values (n_pre x 2^log_n), witness the other columns."""
        args, keep = self._program_args(settings, hash_consts, prog, log_n, preprocessed)
        w = np.ascontiguousarray(witness, np.uint32)
        cap = 1 << 22
        out = np.zeros(cap, np.uint32)
        n = ctypes.c_size_t(cap)
        rc = self.lib.wlo_prove_program(*args, _p(w), _p(out), ctypes.byref(n))
        assert rc == 0, rc
        return out[: n.value].copy()

    def verify_program(self, log_n, hash_consts, prog, proof, settings=None, preprocessed=None):
        args, keep = self._program_args(settings, hash_consts, prog, log_n, preprocessed)
        proof = np.ascontiguousarray(proof, dtype=np.uint32)
        return self.lib.wlo_verify_program(*args, _p(proof), proof.size)

    def prove_abc(self, p16, log_n, skips, a, b, c):
        cap = 1 << 16
        out = np.zeros(cap, np.uint32)
        n = ctypes.c_size_t(cap)
        assert self.lib.wlo_prove_abc(_p(p16), log_n, skips, _p(a), _p(b), _p(c), _p(out), ctypes.byref(n)) == 0
        return out[: n.value].copy()

    def verify_abc(self, p16, log_n, skips, proof):
        proof = np.ascontiguousarray(proof, dtype=np.uint32)
        return self.lib.wlo_verify_abc(_p(p16), log_n, skips, _p(proof), proof.size)

    def chacha_block(self, key, counter, rounds):
        out = np.zeros(16, np.uint32)
        self.lib.wlo_chacha_block(_p(np.ascontiguousarray(key, np.uint32)), counter, rounds, _p(out))
        return out

    def stdrng(self, seed, n):
        out = np.zeros(n, np.uint32)
        self.lib.wlo_stdrng_u32(seed, _p(out), n)
        return out

    def poseidon2(self, width, consts, state):
        st = np.ascontiguousarray(state, np.uint32).copy()
        self.lib.wlo_poseidon2(width, _p(np.ascontiguousarray(consts, np.uint32)), _p(st))
        return st

    def ef_mul(self, a, b):
        out = np.zeros(8, np.uint32)
        self.lib.wlo_ef_mul(_p(np.ascontiguousarray(a, np.uint32)), _p(np.ascontiguousarray(b, np.uint32)), _p(out))
        return out

    def ef_inv(self, a):
        out = np.zeros(8, np.uint32)
        self.lib.wlo_ef_inv(_p(np.ascontiguousarray(a, np.uint32)), _p(out))
        return out

    def ntt(self, coeffs, log_size):
        c = np.ascontiguousarray(coeffs, np.uint32)
        out = np.zeros(1 << log_size, np.uint32)
        self.lib.wlo_ntt(_p(c), c.size, log_size, _p(out))
        return out

    def whir_config(self, num_vars, settings=None):
        out = np.zeros(3 + 7 * 16, np.int32)
        s = settings.ctypes.data_as(_i32p) if settings is not None else None
        assert self.lib.wlo_whir_config(num_vars, s, out.ctypes.data_as(_i32p), 16) == 0
        return out


_cached = None


def build():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)


def load():
    global _cached
    if _cached is None:
        if not os.path.exists(LIB):
            build()
        _cached = Oracle(ctypes.CDLL(LIB))
    return _cached
