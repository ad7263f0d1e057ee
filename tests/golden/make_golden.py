"""Writes tests/golden/oracle_fixtures.json from the CPU oracle.

The reference holds no golden vectors for this path and cannot be run here, so these
fixtures pin the oracle itself against regressions (they are not reference outputs):
StdRng words, Poseidon2 outputs under the seed-0 constants, the workload constants, and
digests of complete proofs. Run: python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from tests import oracle_lib  # noqa: E402


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.uint32).tobytes()).hexdigest()


def build(oracle):
    consts, _ = oracle.workload(2)
    fx = {
        "stdrng_seed0_first32": [int(x) for x in oracle.stdrng(0, 32)],
        "stdrng_seed7_first8": [int(x) for x in oracle.stdrng(7, 8)],
        "constants_logn2_sha256": digest(consts),
        "constants_logn2_first8": [int(x) for x in consts[:8]],
        "poseidon16_zero": [int(x) for x in oracle.poseidon2(16, consts[148:296], np.zeros(16, np.uint32))],
        "poseidon24_zero": [int(x) for x in oracle.poseidon2(24, consts[296:], np.zeros(24, np.uint32))],
        "proofs": {},
    }
    for log_n in (5, 6):
        c, i = oracle.workload(log_n)
        w = oracle.trace(log_n, c, i)
        p, _ = oracle.prove(log_n, c, w)
        fx["proofs"][f"air_logn{log_n}"] = {"len": int(p.size), "sha256": digest(p),
                                            "first16": [int(x) for x in p[:16]]}
    rng = np.random.default_rng(2024)
    P = 0x7F000001
    a = rng.integers(0, P, 1 << 8, dtype=np.uint64)
    b = rng.integers(0, P, 1 << 8, dtype=np.uint64)
    cc = (a * b) % P
    p = oracle.prove_abc(consts[148:296], 8, 3, *(x.astype(np.uint32) for x in (a, b, cc)))
    fx["proofs"]["abc_logn8_skip3_seed2024"] = {"len": int(p.size), "sha256": digest(p)}
    return fx


if __name__ == "__main__":
    fx = build(oracle_lib.load())
    with open(os.path.join(HERE, "oracle_fixtures.json"), "w") as f:
        json.dump(fx, f, indent=1)
    print("wrote", os.path.join(HERE, "oracle_fixtures.json"))
