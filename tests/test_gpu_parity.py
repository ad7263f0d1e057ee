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


# Production-size parity. The kernels that switch on only for large tables run here:
#  - zerocheck rounds >= 1 with at least 2^10 points per z use k_zc_full_dense and
#    k_zc_partial_dense (log_n - skips - 1 >= 10, i.e. log_n >= 15 at 4 skips);
#  - LDE passes after the first use the persistent double-buffered k_ntt_pass_async when a
#    pass has at least 4 lines per resident block (2^(n+2)-row codeword of 88 columns: 11,264
#    lines at log_n 15 and 16 against 2,368 blocks' worth);
#  - Merkle levels of at least 2^13 digests get one launch per level (5 levels at log_n 16).
# The oracle proves 2^16 rows in 10-20 s on the host threads; each proof is computed once.
_big_cache = {}


def _oracle_big(oracle, log_n, skips):
    key = (log_n, skips)
    if key not in _big_cache:
        settings = np.array([128, 1, 7, 4, skips, 5, 16], np.int32)
        consts, inputs = oracle.workload(log_n)
        wit = oracle.trace(log_n, consts, inputs)
        ref, _ = oracle.prove(log_n, consts, wit, settings)
        _big_cache[key] = (consts, inputs, wit, ref)
    return _big_cache[key]


@pytest.mark.parametrize("log_n,skips,path", [(15, 4, "device"), (16, 4, "device"), (16, 4, "host"),
                                              (16, 3, "device")])
def test_prove_production_sizes_match_oracle(oracle, wl, ctx, log_n, skips, path):
    consts, inputs, wit, ref = _oracle_big(oracle, log_n, skips)
    settings = wl.AirSettings(univariate_skips=skips)
    table = wl.AirTable(ctx, consts, log_n, settings)
    ctx.profile(True)
    if path == "device":
        w = wl.Witness.generate(ctx, consts, inputs, log_n)
        got = table.prove_witness(w)
        w.free()
    else:
        got = table.prove(wit)
    classes = ctx.profile_report()
    ctx.profile(False)
    assert "zc_eval_dense" in classes, "the dense zerocheck kernels did not run"
    assert got.size == ref.size and np.array_equal(got, ref), f"first difference at {first_diff(got, ref)}"
    assert wl.verify(consts, log_n, got, settings) == 0


@pytest.mark.parametrize("log_n,skips", [(16, 3), (18, 3), (24, 3)])
def test_sumcheck_abc_large_matches_oracle(oracle, wl, ctx, log_n, skips):
    """The a*b - c zerocheck of the sumcheck microbench at larger tables, up to its full size
    (three columns of 2^24, univariate skip 3)."""
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
    assert wl.sumcheck_abc_verify(p16, log_n, skips, got) == 0


@pytest.mark.parametrize("family,plan", [("lde", p) for p in range(6)] + [("leaf", p) for p in range(3)] +
                         [("merkle", p) for p in range(3)] + [("inner", p) for p in range(2)])
def test_every_tuned_plan_matches_oracle(oracle, wl, ctx, family, plan):
    """Every launch plan the autotuner can pick gives the same proof: with the plan forced the
    proof equals the oracle's (2^13 rows: three NTT passes, 2^15 leaves so that the Merkle
    schedules differ, 2^5-row inner-sum segments for both stagings)."""
    log_n = 13
    consts, inputs = oracle.workload(log_n)
    wit = oracle.trace(log_n, consts, inputs)
    ref, _ = oracle.prove(log_n, consts, wit)
    wl.tune_force(family, plan)
    try:
        w = wl.Witness.generate(ctx, consts, inputs, log_n)
        got = wl.AirTable(ctx, consts, log_n).prove_witness(w)
        w.free()
        got_host = wl.AirTable(ctx, consts, log_n).prove(wit)  # the tile-pipelined commitment
    finally:
        wl.tune_force(family, -1)
    assert np.array_equal(got, ref), f"first difference at {first_diff(got, ref)}"
    assert np.array_equal(got_host, ref), f"first difference at {first_diff(got_host, ref)}"


def test_autotuner_keeps_a_plan_per_shape(oracle, wl):
    """A tuning context times every plan on the first proof of a shape and keeps the fastest;
    the proof is still the oracle's, and a second proof of the shape reuses the kept plans."""
    log_n = 11
    consts, inputs = oracle.workload(log_n)
    wit = oracle.trace(log_n, consts, inputs)
    ref, _ = oracle.prove(log_n, consts, wit)
    wl.tune_clear()
    with wl.Context(0) as c:
        c.set_autotune(True)
        w = wl.Witness.generate(c, consts, inputs, log_n)
        table = wl.AirTable(c, consts, log_n)
        p1 = table.prove_witness(w)
        rep = wl.tune_report()
        p2 = table.prove_witness(w)
        w.free()
    assert np.array_equal(p1, ref) and np.array_equal(p2, ref)
    for fam, n in (("lde", 6), ("leaf", 3), ("merkle", 3), ("inner", 2)):
        assert rep[fam], fam
        for e in rep[fam]:
            assert len(e["ms"]) == n and 0 <= e["plan"] < n
            assert e["ms"][e["plan"]] == min(e["ms"])
    assert wl.tune_report() == rep  # nothing re-tuned by the second proof


def test_prove_bench_size_matches_oracle(oracle, wl, ctx):
    """The benchmark's own workload, 2^20 rows with the reference's defaults, proved on the GPU
    and by the oracle (two to three minutes of the host's threads): the proofs are identical."""
    log_n = 20
    consts, inputs = wl.generate_workload(log_n)
    w = wl.Witness.generate(ctx, consts, inputs, log_n)
    got = wl.AirTable(ctx, consts, log_n).prove_witness(w)
    wit = w.download()
    w.free()
    ref, _ = oracle.prove(log_n, consts, wit)
    assert got.size == ref.size and np.array_equal(got, ref), f"first difference at {first_diff(got, ref)}"
