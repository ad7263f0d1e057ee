"""AIRs given as constraint programs (the generic-AIR path).

CPU: the oracle proves the Poseidon2 AIR written as a program to the same proof words as its
built-in Poseidon2 AIR (pinning the program semantics to the pinned AIR); oracle proofs of
other program AIRs (transitions over the down values, degrees 1 to 3, preprocessed columns)
are accepted by the oracle's and by the library's host verifiers, and proofs of broken
witnesses (or checked against other preprocessed values) are rejected.
GPU: the library's proofs equal the oracle's word for word.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from whirlaway_b200 import air_program as ap

from . import oracle_lib

P = ap.P


def settings_arr(skips=4):
    return np.array([128, 1, 7, 4, skips, 5, 16], np.int32)


def wl_settings(skips=4):
    import whirlaway_b200 as wl
    return wl.AirSettings(univariate_skips=skips)


def cubic_air(log_n, seed=1):
    """x' = x^3 + y, y' = x (degree 3, transitions only)."""
    n = 1 << log_n
    rng = np.random.default_rng(seed)
    x = np.zeros(n, np.uint64)
    y = np.zeros(n, np.uint64)
    x[0], y[0] = rng.integers(0, P, 2)
    for i in range(n - 1):
        x[i + 1] = (x[i] * x[i] % P * x[i] + y[i]) % P
        y[i + 1] = x[i]
    b = ap.AirBuilder(2)
    b.assert_zero(b.down(0) - (b.up(0) * b.up(0) * b.up(0) + b.up(1)))
    b.assert_zero(b.down(1) - b.up(0))
    return b.build(), np.concatenate([x, y]).astype(np.uint32)


def fib_air(log_n):
    """a' = b, b' = a + b (degree 1)."""
    n = 1 << log_n
    a = np.zeros(n, np.uint64)
    c = np.zeros(n, np.uint64)
    a[0], c[0] = 0, 1
    for i in range(n - 1):
        a[i + 1] = c[i]
        c[i + 1] = (a[i] + c[i]) % P
    b = ap.AirBuilder(2)
    b.assert_zero(b.down(0) - b.up(1))
    b.assert_zero(b.down(1) - b.up(0) - b.up(1))
    return b.build(), np.concatenate([a, c]).astype(np.uint32)


def mul_air(log_n, seed=2):
    """x' = x y, y' = y + 1, z = x^2 (degree 2, a local constraint beside the transitions)."""
    n = 1 << log_n
    rng = np.random.default_rng(seed)
    x = np.zeros(n, np.uint64)
    y = np.zeros(n, np.uint64)
    x[0], y[0] = rng.integers(1, P, 2)
    for i in range(n - 1):
        x[i + 1] = x[i] * y[i] % P
        y[i + 1] = (y[i] + 1) % P
    z = x * x % P
    b = ap.AirBuilder(3)
    b.assert_zero(b.down(0) - b.up(0) * b.up(1))
    b.assert_zero(b.down(1) - (b.up(1) + 1))
    b.assert_zero(b.up(2) - b.up(0) * b.up(0))
    return b.build(), np.concatenate([x, y, z]).astype(np.uint32)


AIRS = {"cubic": cubic_air, "fib": fib_air, "mul": mul_air}


def pre_air(log_n, seed=3):
    """Two preprocessed columns, f (1 on row 0) and r (fixed values), and the witness x, y with
    f x = 0 (x starts at 0), x' = x + r, y = x r + f. Returns (program, witness, preprocessed)."""
    n = 1 << log_n
    rng = np.random.default_rng(seed)
    f = np.zeros(n, np.uint64)
    f[0] = 1
    r = rng.integers(0, P, n).astype(np.uint64)
    x = np.zeros(n, np.uint64)
    for i in range(n - 1):
        x[i + 1] = (x[i] + r[i]) % P
    y = (x * r + f) % P
    b = ap.AirBuilder(4, preprocessed=2)
    F, R, X, Y = (b.up(c) for c in range(4))
    b.assert_zero(F * X)
    b.assert_zero(b.down(2) - X - R)
    b.assert_zero(Y - X * R - F)
    return b.build(), np.concatenate([x, y]).astype(np.uint32), np.concatenate([f, r]).astype(np.uint32)


@pytest.fixture(scope="module")
def oracle():
    return oracle_lib.load()


@pytest.fixture(scope="module")
def hash_consts(oracle):
    c, _ = oracle.workload(2, 0)
    return c[148:]


def test_program_compiler_on_host(tmp_path):
    """The compiled device code (registers, constants as immediates) run by a host restatement
    of the interpreter kernels equals the program evaluated instruction by instruction."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    nvcc = shutil.which("nvcc")
    if nvcc is None:
        pytest.skip("no CUDA toolkit (vector types header)")
    cuda_inc = os.path.join(os.path.dirname(os.path.dirname(os.path.realpath(nvcc))), "include")
    exe = tmp_path / "program_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(root, "whirlaway_b200", "csrc"),
                    "-I", cuda_inc, os.path.join(root, "tests", "program_host_check.cpp"),
                    "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr


def test_builder_degrees_and_checks():
    prog, w = cubic_air(8)
    assert (prog.width, prog.n_constraints, prog.degree) == (2, 2, 3)
    assert prog.evaluate_rows(w, 8).max() == 0
    b = ap.AirBuilder(2)
    with pytest.raises(IndexError):
        b.up(2)
    with pytest.raises(ValueError):
        b.build()  # no constraints
    b.assert_zero(b.up(0) * b.up(0) * b.up(1))
    with pytest.raises(ValueError):
        b.build(2)  # below the constraint's degree
    x = b.up(0)
    b.assert_zero(x * x * x * x)
    with pytest.raises(ValueError):
        b.build()  # degree 4


def test_poseidon2_program_matches_builtin_oracle(oracle):
    for log_n, skips in [(6, 4), (7, 2)]:
        c, i = oracle.workload(log_n, 5)
        w = oracle.trace(log_n, c, i)
        prog = ap.poseidon2_air_program(c[:148])
        assert prog.evaluate_rows(w, log_n).max() == 0
        s = settings_arr(skips)
        builtin, _ = oracle.prove(log_n, c, w, s)
        program = oracle.prove_program(log_n, c[148:], prog, w, s)
        assert np.array_equal(builtin, program)
        assert oracle.verify_program(log_n, c[148:], prog, program, s) == 0


@pytest.mark.parametrize("name", sorted(AIRS))
@pytest.mark.parametrize("log_n,skips", [(8, 1), (9, 3), (10, 4)])
def test_program_airs_oracle_and_host_verifier(oracle, hash_consts, name, log_n, skips):
    import whirlaway_b200 as wl
    prog, w = AIRS[name](log_n)
    assert prog.evaluate_rows(w, log_n).max() == 0
    proof = oracle.prove_program(log_n, hash_consts, prog, w, settings_arr(skips))
    assert oracle.verify_program(log_n, hash_consts, prog, proof, settings_arr(skips)) == 0
    # the library's host verifier accepts the oracle's proof and rejects a changed word
    assert wl.verify_program(hash_consts, prog, log_n, proof, wl_settings(skips)) == 0
    bad = proof.copy()
    bad[len(bad) // 3] = (int(bad[len(bad) // 3]) + 1) % P
    assert wl.verify_program(hash_consts, prog, log_n, bad, wl_settings(skips)) != 0


@pytest.mark.parametrize("name", sorted(AIRS))
def test_broken_witness_rejected(oracle, hash_consts, name):
    import whirlaway_b200 as wl
    log_n = 8
    prog, w = AIRS[name](log_n)
    bad = w.copy()
    bad[(1 << log_n) + 17] = (int(bad[(1 << log_n) + 17]) + 1) % P
    assert prog.evaluate_rows(bad, log_n).max() != 0
    proof = oracle.prove_program(log_n, hash_consts, prog, bad, settings_arr())
    assert oracle.verify_program(log_n, hash_consts, prog, proof, settings_arr()) != 0
    assert wl.verify_program(hash_consts, prog, log_n, proof, wl_settings()) != 0


@pytest.mark.parametrize("log_n,skips", [(8, 2), (10, 4)])
def test_preprocessed_columns(oracle, hash_consts, log_n, skips):
    import whirlaway_b200 as wl
    prog, w, pre = pre_air(log_n)
    assert prog.n_preprocessed == 2
    assert prog.evaluate_rows(w, log_n, pre).max() == 0
    s = settings_arr(skips)
    proof = oracle.prove_program(log_n, hash_consts, prog, w, s, preprocessed=pre)
    assert oracle.verify_program(log_n, hash_consts, prog, proof, s, preprocessed=pre) == 0
    assert wl.verify_program(hash_consts, prog, log_n, proof, wl_settings(skips), preprocessed=pre) == 0
    # other preprocessed values: the proof no longer verifies
    other = pre.copy()
    other[(1 << log_n) + 5] = (int(other[(1 << log_n) + 5]) + 1) % P
    assert oracle.verify_program(log_n, hash_consts, prog, proof, s, preprocessed=other) != 0
    assert wl.verify_program(hash_consts, prog, log_n, proof, wl_settings(skips), preprocessed=other) != 0


def test_malformed_programs_rejected(hash_consts):
    import whirlaway_b200 as wl
    prog, w = fib_air(8)
    bad = ap.AirProgram(prog.width, prog.n_constraints, prog.degree, prog.ops.copy(), prog.consts)
    bad.ops[2, 1] = 5  # an operand that is not an earlier value
    assert wl.verify_program(hash_consts, bad, 8, np.zeros(8, np.uint32), wl_settings()) == 1
    # 70 values live at once (all made before they are summed): beyond the device interpreter's
    # 64 registers, so the library rejects the program as an argument error
    wide = ap.AirBuilder(1)
    vals = [wide.up(0) + i for i in range(1, 71)]
    acc = vals[-1]
    for v in reversed(vals[:-1]):
        acc = acc + v
    wide.assert_zero(acc)
    prog_wide = wide.build()
    assert prog_wide.degree == 1
    assert wl.verify_program(hash_consts, prog_wide, 8, np.zeros(8, np.uint32), wl_settings()) == 1
    # a constant that is not a canonical field element, and no EMIT for a declared constraint
    b = ap.AirBuilder(2)
    b.assert_zero(b.up(0) - b.up(1))
    p2 = b.build()
    bad_c = ap.AirProgram(2, 1, 1, p2.ops, np.array([P], np.uint32))
    bad_c.ops = np.array([[ap.OP_CONST, 0, 0], [ap.OP_EMIT, 0, 0]], np.int32)
    assert wl.verify_program(hash_consts, bad_c, 8, np.zeros(8, np.uint32), wl_settings()) == 1
    two = ap.AirProgram(2, 2, 1, p2.ops, p2.consts)
    assert wl.verify_program(hash_consts, two, 8, np.zeros(8, np.uint32), wl_settings()) == 1
    with pytest.raises(ValueError):
        ap.AirProgram(2, 1, 1, p2.ops, p2.consts, n_preprocessed=2)
    # preprocessed values must come with a program that has preprocessed columns
    prog_pre, _, _ = pre_air(8)
    with pytest.raises(ValueError):
        wl.verify_program(hash_consts, prog_pre, 8, np.zeros(8, np.uint32), wl_settings())


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(AIRS))
@pytest.mark.parametrize("log_n,skips", [(8, 1), (10, 4), (12, 3), (18, 1)])
def test_gpu_program_matches_oracle(oracle, hash_consts, name, log_n, skips):
    """(18, 1): 2^17 rows per round-0 point, more than the interpreter grid's threads, so the
    grid-stride loops and the multi-block reductions run."""
    import whirlaway_b200 as wl
    prog, w = AIRS[name](log_n)
    want = oracle.prove_program(log_n, hash_consts, prog, w, settings_arr(skips))
    with wl.Context(0) as ctx:
        got = wl.prove_program(ctx, hash_consts, prog, log_n, w, wl_settings(skips))
    assert np.array_equal(got, want)
    assert wl.verify_program(hash_consts, prog, log_n, got, wl_settings(skips)) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("log_n,skips", [(8, 2), (12, 4)])
def test_gpu_preprocessed_matches_oracle(oracle, hash_consts, log_n, skips):
    import whirlaway_b200 as wl
    prog, w, pre = pre_air(log_n)
    want = oracle.prove_program(log_n, hash_consts, prog, w, settings_arr(skips), preprocessed=pre)
    with wl.Context(0) as ctx:
        got = wl.prove_program(ctx, hash_consts, prog, log_n, w, wl_settings(skips), preprocessed=pre)
    assert np.array_equal(got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("log_n", [8, 12])
def test_gpu_poseidon2_program_matches_builtin(oracle, log_n):
    import whirlaway_b200 as wl
    c, i = oracle.workload(log_n, 9)
    w = oracle.trace(log_n, c, i)
    prog = ap.poseidon2_air_program(c[:148])
    with wl.Context(0) as ctx:
        builtin = wl.AirTable(ctx, c, log_n).prove(w)
        program = wl.prove_program(ctx, c[148:], prog, log_n, w)
    assert np.array_equal(builtin, program)
