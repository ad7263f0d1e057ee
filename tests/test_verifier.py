"""The product's host verifier (wl_verify, wl_sumcheck_abc_verify) on CPU, against proofs the
oracle prover makes: honest proofs are accepted, corrupted ones rejected with the
AirVerifError outcome of crates/air/src/verify.rs, and the oracle's own verifier agrees on
acceptance."""
import numpy as np
import pytest

P = 0x7F000001
OK, COMMITMENT, OPENING, FS, SUMCHECK, SUM_MISMATCH = 0, 11, 12, 13, 14, 16


def honest(oracle, log_n, settings=None):
    consts, inputs = oracle.workload(log_n)
    wit = oracle.trace(log_n, consts, inputs)
    proof, _ = oracle.prove(log_n, consts, wit, settings)
    return consts, wit, proof


@pytest.mark.parametrize("log_n", [5, 7, 9])
def test_accepts_honest_proofs(wl, oracle, log_n):
    consts, _, proof = honest(oracle, log_n)
    assert oracle.verify(log_n, consts, proof) == 0
    assert wl.verify(consts, log_n, proof) == OK


def test_settings_and_sizes_must_match(wl, oracle):
    log_n = 6
    consts, _, proof = honest(oracle, log_n)
    assert wl.verify(consts, log_n, proof) == OK
    assert wl.verify(consts, log_n + 1, proof) != OK              # other height
    assert wl.verify(consts, log_n, proof, wl.AirSettings(univariate_skips=3)) != OK
    other = consts.copy()
    other[200] = (int(other[200]) + 1) % P                        # other Poseidon16 constant
    assert wl.verify(other, log_n, proof) != OK
    other = consts.copy()
    other[5] = (int(other[5]) + 1) % P                            # other AIR round constant
    assert wl.verify(other, log_n, proof) != OK


def test_rejects_corrupted_words(wl, oracle):
    log_n = 6
    consts, _, proof = honest(oracle, log_n)
    rng = np.random.default_rng(3)
    positions = sorted(set([0, 3, 8, 20, 200, 1000, proof.size // 2, proof.size - 5, proof.size - 1]
                           + list(rng.integers(0, proof.size, 24))))
    for pos in positions:
        bad = proof.copy()
        bad[pos] = (int(bad[pos]) + 1) % P
        got = wl.verify(consts, log_n, bad)
        assert got != OK, pos
        assert (oracle.verify(log_n, consts, bad) != 0), pos
    # the root and the OOD answers belong to the commitment; the transcript changes after them
    bad = proof.copy()
    bad[0] = (int(bad[0]) + 1) % P
    assert wl.verify(consts, log_n, bad) in (SUMCHECK, SUM_MISMATCH, FS, OPENING)


def test_rejects_truncated_and_padded_proofs(wl, oracle):
    log_n = 5
    consts, _, proof = honest(oracle, log_n)
    assert wl.verify(consts, log_n, proof[:-1]) == OPENING         # the last Merkle path is short
    assert wl.verify(consts, log_n, proof[:4]) == COMMITMENT       # the root is incomplete
    assert wl.verify(consts, log_n, np.concatenate([proof, np.zeros(1, np.uint32)])) == FS
    assert wl.verify(consts, log_n, np.zeros(0, np.uint32)) == COMMITMENT


def test_rejects_non_canonical_words(wl, oracle):
    log_n = 5
    consts, _, proof = honest(oracle, log_n)
    bad = proof.copy()
    bad[10] = P + int(bad[10]) % 7  # same residue class, not canonical
    assert wl.verify(consts, log_n, bad) == 1


def test_rejects_proof_of_invalid_trace(wl, oracle):
    log_n = 6
    consts, inputs = oracle.workload(log_n)
    wit = oracle.trace(log_n, consts, inputs)
    wit[(20 << log_n) + 7] ^= 1  # break one post-round state
    proof, _ = oracle.prove(log_n, consts, wit)
    assert oracle.verify(log_n, consts, proof) != 0
    assert wl.verify(consts, log_n, proof) == SUM_MISMATCH


def test_abc_verifier(wl, oracle):
    rng = np.random.default_rng(4)
    consts, _ = oracle.workload(2)
    p16 = consts[148:296]
    for log_n, skips in ((8, 3), (10, 4), (6, 1)):
        a = rng.integers(0, P, 1 << log_n, dtype=np.uint64)
        b = rng.integers(0, P, 1 << log_n, dtype=np.uint64)
        c = (a * b) % P
        a, b, c = (x.astype(np.uint32) for x in (a, b, c))
        proof = oracle.prove_abc(p16, log_n, skips, a, b, c)
        assert wl.sumcheck_abc_verify(p16, log_n, skips, proof) == OK
        bad = proof.copy()
        bad[9] = (int(bad[9]) + 1) % P
        assert wl.sumcheck_abc_verify(p16, log_n, skips, bad) != OK
        bad = proof.copy()
        bad[-1] = (int(bad[-1]) + 1) % P  # a final value
        assert wl.sumcheck_abc_verify(p16, log_n, skips, bad) == SUM_MISMATCH
        c2 = c.copy()
        c2[5] ^= 1
        assert wl.sumcheck_abc_verify(p16, log_n, skips, oracle.prove_abc(p16, log_n, skips, a, b, c2)) != OK


def test_verifier_transcript_dump(wl, oracle):
    log_n, k = 7, 4
    consts, _, proof = honest(oracle, log_n)
    st, dump = wl.verify_transcript(consts, log_n, proof)
    assert st == OK and dump["proof_len"] == proof.size
    ev = dump["events"]
    phases = [e for e in ev if e["kind"] == "phase"]
    names = [e["phase"] for e in phases]
    assert names[:6] == ["commit", "batching", "zerocheck", "inner_sums", "inner_sumcheck", "whir"]
    assert names[-1] == "whir_final" and all(n.startswith("whir_round_") for n in names[6:-1])
    offs = [e["offset"] for e in ev]
    assert offs == sorted(offs) and offs[-1] <= proof.size
    count = lambda ph, kind: sum(1 for e in ev if e["phase"] == ph and e["kind"] == kind)
    assert count("batching", "challenge") == 1 + (log_n - k + 1)   # alpha, zerocheck challenges
    assert count("zerocheck", "challenge") == log_n - k + 1           # one per round
    assert count("inner_sums", "challenge") == 8 + 1 + k              # column batching, alpha', epsilons
    assert count("inner_sumcheck", "challenge") == log_n
    for e in ev:
        if e["kind"] == "challenge":
            assert len(e["values"]) == 8 and all(0 <= v < P for v in e["values"])
        if e["kind"] == "queries":
            assert e["values"] == sorted(set(e["values"]))
    # the commitment root is the first 8 words; the first challenge (OOD) follows it
    first = next(e for e in ev if e["kind"] == "challenge")
    assert first["phase"] == "commit" and first["offset"] == 8
    # a corrupted proof is read up to the failed check
    bad = proof.copy()
    bad[proof.size // 2] = (int(bad[proof.size // 2]) + 1) % P
    st2, dump2 = wl.verify_transcript(consts, log_n, bad)
    assert st2 != OK and len(dump2["events"]) <= len(ev)


def test_verify_batch_threads(wl, oracle):
    consts, _ = oracle.workload(5, 1)
    jobs = []
    for k, log_n in enumerate((5, 6, 7, 6, 5)):
        c, i = oracle.workload(log_n, 10 + k)  # own inputs; the constants skip the input draws
        assert np.array_equal(c, consts)
        proof, _ = oracle.prove(log_n, c, oracle.trace(log_n, c, i))
        jobs.append((log_n, proof))
    bad = jobs[2][1].copy()
    bad[100] = (int(bad[100]) + 1) % P
    jobs.append((7, bad))
    jobs.append((6, jobs[0][1]))  # wrong height for that proof
    for threads in (1, 4, 0):
        st = wl.verify_batch(consts, jobs, threads=threads)
        assert st[:5] == [OK] * 5 and st[5] != OK and st[6] != OK
        assert st == [wl.verify(consts, l, p) for l, p in jobs]


@pytest.mark.parametrize("kw", [dict(univariate_skips=2), dict(log_inv_rate=2), dict(security_bits=100),
                                dict(rs_domain_initial_reduction=3), dict(whir_pow_bits=10)])
def test_other_settings_roundtrip(wl, oracle, kw):
    """The product's WHIR schedule and verifier agree with the oracle prover on non-default
    settings (the schedule drives the transcript layout, so any mismatch rejects)."""
    log_n = 7
    s = wl.AirSettings(**kw)
    consts, _, proof = honest(oracle, log_n, s.as_array())
    assert oracle.verify(log_n, consts, proof, s.as_array()) == 0
    assert wl.verify(consts, log_n, proof, s) == OK
    assert proof.size <= wl.proof_len_bound(s, log_n)
    if kw != dict(whir_pow_bits=10):
        assert wl.verify(consts, log_n, proof) != OK  # the default settings read it differently


@pytest.mark.parametrize("log_n,skips", [(2, 1), (3, 2), (4, 3), (5, 4)])
def test_tiny_tables(wl, oracle, log_n, skips):
    """The smallest tables the settings allow (no WHIR folding round before the final one)."""
    s = wl.AirSettings(univariate_skips=skips)
    consts, _, proof = honest(oracle, log_n, s.as_array())
    assert wl.verify(consts, log_n, proof, s) == OK
    bad = proof.copy()
    bad[proof.size // 3] = (int(bad[proof.size // 3]) + 1) % P
    assert wl.verify(consts, log_n, bad, s) != OK


@pytest.mark.gpu
def test_verify_batch_device_matches_host(oracle, wl, ctx):
    """The GPU-checked batch verifier gives every proof the host verifier's outcome: honest
    proofs of several sizes are accepted; a corrupted opened row, path digest or commitment
    root is an opening error (11 for a root the commitment phase already reads), and a corrupted
    sumcheck word fails before the openings with the host's outcome."""
    consts, _ = oracle.workload(2, 1)  # with an input seed the constants do not depend on log_n
    jobs = []
    for log_n in (6, 8, 9):
        c, inputs = oracle.workload(log_n, 10 + log_n)
        assert np.array_equal(c, consts)
        jobs.append((log_n, oracle.prove(log_n, consts, oracle.trace(log_n, consts, inputs))[0]))
    dump_n, dump_p = jobs[1]
    _, tr = wl.verify_transcript(consts, dump_n, dump_p)
    phases = {e["phase"]: e["offset"] for e in tr["events"] if e["kind"] == "phase"}
    # opened rows and paths follow each "queries" event (hints, not absorbed)
    qoffs = [e["offset"] for e in tr["events"] if e["kind"] == "queries"]
    assert len(qoffs) >= 2
    bad = []
    p = dump_p.copy()
    p[qoffs[0] + 5] = (int(p[qoffs[0] + 5]) + 1) % 0x7F000001  # a word of the first opened row
    bad.append((dump_n, p))
    p = dump_p.copy()
    p[qoffs[-1] + 128 + 3] = (int(p[qoffs[-1] + 128 + 3]) + 1) % 0x7F000001  # a digest of a path
    bad.append((dump_n, p))
    p = dump_p.copy()
    p[phases["whir_round_1"] + 3] = (int(p[phases["whir_round_1"] + 3]) + 1) % 0x7F000001  # a later root
    bad.append((dump_n, p))
    p = dump_p.copy()
    p[phases["zerocheck"] + 9] = (int(p[phases["zerocheck"] + 9]) + 1) % 0x7F000001
    bad.append((dump_n, p))
    p = dump_p.copy()
    p[0] = (int(p[0]) + 1) % 0x7F000001  # the first commitment's root
    bad.append((dump_n, p))
    allj = jobs + bad
    host = wl.verify_batch(consts, allj)
    dev = wl.verify_batch_device(ctx, consts, allj)
    assert host[:3] == [0, 0, 0]
    assert all(h != 0 for h in host[3:])
    assert host[3] == OPENING and host[4] == OPENING
    assert dev == host


@pytest.mark.parametrize("kw", [{"log_inv_rate": 3}, {"univariate_skips": 2}, {"security_bits": 100},
                                {"rs_domain_initial_reduction": 3}, {"log_inv_rate": 2, "univariate_skips": 3}])
def test_merkle_batches_under_other_settings(wl, oracle, kw):
    """The Merkle checks hash a round's queries as batches of permutations (sixteen per vector,
    ragged last batch): honest proofs under other rates, skips, security levels and domain
    reductions are accepted alone and in a batch, and a changed word of the last path is an
    opening failure."""
    log_n = 10
    s = wl.AirSettings(**kw)
    consts, _, proof = honest(oracle, log_n, s.as_array())
    assert wl.verify(consts, log_n, proof, s) == OK
    bad = proof.copy()
    bad[-3] = (int(bad[-3]) + 1) % P
    assert wl.verify(consts, log_n, bad, s) == OPENING
    assert wl.verify_batch(consts, [(log_n, proof), (log_n, bad), (log_n, proof)], s, threads=2) == [OK, OPENING, OK]
