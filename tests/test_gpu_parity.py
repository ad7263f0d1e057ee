"""GPU parity: the CUDA prover against the CPU oracle on the same seeded inputs.

Every comparison is bit-exact (integer field arithmetic); proofs from the GPU must also be
accepted by the oracle's verifier.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def first_diff(a, b):
    n = min(a.size, b.size)
    d = np.nonzero(a[:n] != b[:n])[0]
    return int(d[0]) if d.size else (n if a.size != b.size else -1)


def test_trace_generation_matches_oracle(oracle, wl, ctx):
    log_n = 10
    consts, inputs = oracle.workload(log_n)
    w = wl.Witness.generate(ctx, consts, inputs, log_n)
    got = w.download()
    assert np.array_equal(got, oracle.trace(log_n, consts, inputs))


def test_workload_generator_matches_oracle(oracle, wl):
    for log_n, seed in [(6, -1), (6, 7), (9, -1)]:
        c1, i1 = oracle.workload(log_n, seed)
        c2, i2 = wl.generate_workload(log_n, seed)
        assert np.array_equal(c1, c2) and np.array_equal(i1, i2)


@pytest.mark.parametrize("log_n", [5, 6, 7, 8, 10, 12])
def test_prove_matches_oracle(oracle, wl, ctx, log_n):
    consts, inputs = oracle.workload(log_n)
    wit = oracle.trace(log_n, consts, inputs)
    ref, _ = oracle.prove(log_n, consts, wit)
    got = wl.AirTable(ctx, consts, log_n).prove(wit)
    assert got.size == ref.size and np.array_equal(got, ref), f"first difference at {first_diff(got, ref)}"
    assert oracle.verify(log_n, consts, got) == 0
    assert wl.verify(consts, log_n, got) == 0  # the product's host verifier


@pytest.mark.parametrize("log_n,skips", [(8, 1), (8, 2), (9, 3), (6, 3), (2, 1), (3, 2), (4, 3), (4, 1)])
def test_prove_other_skips_matches_oracle(oracle, wl, ctx, log_n, skips):
    """Univariate skips below 4: fewer round-0 points (2, 6, 14) than the 30 of the default."""
    settings = wl.AirSettings(univariate_skips=skips)
    consts, inputs = oracle.workload(log_n)
    wit = oracle.trace(log_n, consts, inputs)
    ref, _ = oracle.prove(log_n, consts, wit, settings.as_array())
    got = wl.AirTable(ctx, consts, log_n, settings).prove(wit)
    assert got.size == ref.size and np.array_equal(got, ref), f"first difference at {first_diff(got, ref)}"
    assert wl.verify(consts, log_n, got, settings) == 0


@pytest.mark.parametrize("kw", [dict(log_inv_rate=2), dict(security_bits=100), dict(rs_domain_initial_reduction=3),
                                dict(whir_pow_bits=10), dict(log_inv_rate=3, univariate_skips=3)])
@pytest.mark.parametrize("log_n", [7, 10])
def test_prove_other_settings_matches_oracle(oracle, wl, ctx, kw, log_n):
    """Non-default AirSettings: rate, security level, RS domain reduction, PoW bits."""
    settings = wl.AirSettings(**kw)
    consts, inputs = oracle.workload(log_n)
    wit = oracle.trace(log_n, consts, inputs)
    ref, _ = oracle.prove(log_n, consts, wit, settings.as_array())
    got = wl.AirTable(ctx, consts, log_n, settings).prove(wit)
    assert got.size == ref.size and np.array_equal(got, ref), f"first difference at {first_diff(got, ref)}"
    assert wl.verify(consts, log_n, got, settings) == 0


def test_transcript_dump_prover_equals_verifier(oracle, wl):
    """The GPU prover's per-phase transcript dump equals the host verifier's reading of its proof."""
    log_n = 8
    consts, inputs = oracle.workload(log_n)
    with wl.Context(0) as c:
        c.set_transcript_dump(True)
        proof = wl.AirTable(c, consts, log_n).prove(oracle.trace(log_n, consts, inputs))
        dump = c.transcript_dump()
    st, vdump = wl.verify_transcript(consts, log_n, proof)
    assert st == 0
    assert dump["proof_len"] == proof.size
    assert dump == vdump


def test_prove_device_witness_matches_host_path(oracle, wl, ctx):
    log_n = 9
    consts, inputs = oracle.workload(log_n, 3)
    table = wl.AirTable(ctx, consts, log_n)
    w = wl.Witness.generate(ctx, consts, inputs, log_n)
    p_dev = table.prove_witness(w)
    p_host = table.prove(oracle.trace(log_n, consts, inputs))
    assert np.array_equal(p_dev, p_host)
    assert oracle.verify(log_n, consts, p_dev) == 0


@pytest.mark.parametrize("log_n,skips", [(8, 3), (10, 3), (12, 2), (9, 1), (11, 4)])
def test_sumcheck_abc_matches_oracle(oracle, wl, ctx, log_n, skips):
    rng = np.random.default_rng(log_n * 10 + skips)
    p = 0x7F000001
    a = rng.integers(0, p, 1 << log_n, dtype=np.uint64)
    b = rng.integers(0, p, 1 << log_n, dtype=np.uint64)
    c = (a * b) % p
    a, b, c = (x.astype(np.uint32) for x in (a, b, c))
    consts, _ = oracle.workload(2)
    p16 = consts[148:296]
    ref = oracle.prove_abc(p16, log_n, skips, a, b, c)
    got, ms = wl.sumcheck_abc_prove(ctx, p16, log_n, skips, a, b, c)
    assert np.array_equal(got, ref), f"first difference at {first_diff(got, ref)}"
    assert oracle.verify_abc(p16, log_n, skips, got) == 0
    assert wl.sumcheck_abc_verify(p16, log_n, skips, got) == 0
    assert len(ms) == log_n - skips + 1
