"""CPU checks of the oracle: known answers where an independent implementation exists
(ChaCha20 from the `cryptography` package), field and transform identities, and the
prover/verifier round trip with corruption detection."""
import numpy as np
import pytest

P = 0x7F000001


def test_chacha20_matches_cryptography(oracle):
    from cryptography.hazmat.primitives.ciphers import Cipher, algorithms
    for seed in range(3):
        key = np.random.default_rng(seed).integers(0, 2**32, 8, dtype=np.uint64).astype(np.uint32)
        for counter in (0, 1, 5):
            out = oracle.chacha_block(key, counter, 20)
            nonce = int(counter).to_bytes(4, "little") + b"\x00" * 12
            enc = Cipher(algorithms.ChaCha20(key.tobytes(), nonce), mode=None).encryptor()
            ks = np.frombuffer(enc.update(b"\x00" * 64), np.uint32)
            assert np.array_equal(out, ks)


def test_stdrng_stream_is_chacha12_blocks(oracle):
    # StdRng words are ChaCha12 blocks 0, 1, ... keyed by the PCG32 expansion of the seed.
    words = oracle.stdrng(0, 48)
    key = np.zeros(8, np.uint32)
    state = 0
    mul, inc = 6364136223846793005, 11634580456548416449
    for i in range(8):
        state = (state * mul + inc) % 2**64
        xs = (((state >> 18) ^ state) >> 27) & 0xFFFFFFFF
        rot = state >> 59
        key[i] = ((xs >> rot) | (xs << ((32 - rot) & 31))) & 0xFFFFFFFF
    blocks = np.concatenate([oracle.chacha_block(key, c, 12) for c in range(3)])
    assert np.array_equal(words, blocks)


def _ef_rand(rng):
    return rng.integers(0, P, 8, dtype=np.uint64).astype(np.uint32)


def test_extension_field_identities(oracle):
    rng = np.random.default_rng(1)
    one = np.array([1, 0, 0, 0, 0, 0, 0, 0], np.uint32)
    for _ in range(20):
        a, b, c = _ef_rand(rng), _ef_rand(rng), _ef_rand(rng)
        assert np.array_equal(oracle.ef_mul(oracle.ef_mul(a, b), c), oracle.ef_mul(a, oracle.ef_mul(b, c)))
        assert np.array_equal(oracle.ef_mul(a, b), oracle.ef_mul(b, a))
        assert np.array_equal(oracle.ef_mul(a, oracle.ef_inv(a)), one)
    x = np.array([0, 1, 0, 0, 0, 0, 0, 0], np.uint32)
    x8 = one
    for _ in range(8):
        x8 = oracle.ef_mul(x8, x)
    assert np.array_equal(x8, np.array([3, 0, 0, 0, 0, 0, 0, 0], np.uint32))


def test_two_adic_generator_and_frobenius_order(oracle):
    """3^127 has multiplicative order 2^24 (p - 1 = 2^24 * 127, 3 generates F_p^*), and the
    Frobenius a -> a^p of the degree-8 extension has order 8 on a generic element."""
    w = pow(3, 127, P)
    assert pow(w, 1 << 24, P) == 1 and pow(w, 1 << 23, P) != 1
    assert pow(3, (P - 1) // 2, P) != 1 and pow(3, (P - 1) // 127, P) != 1  # 3 is a generator

    def ef_pow(a, e):
        r = np.array([1, 0, 0, 0, 0, 0, 0, 0], np.uint32)
        while e:
            if e & 1:
                r = oracle.ef_mul(r, a)
            a = oracle.ef_mul(a, a)
            e >>= 1
        return r

    a = _ef_rand(np.random.default_rng(7))
    x = a
    for k in range(1, 9):
        x = ef_pow(x, P)
        assert np.array_equal(x, a) == (k == 8), k


def test_ntt_matches_naive_dft(oracle):
    rng = np.random.default_rng(2)
    for log_size in (1, 3, 6):
        n = 1 << log_size
        coeffs = rng.integers(0, P, n // 2 + 1, dtype=np.uint64)
        w = pow(3, 127 << (24 - log_size), P)
        naive = [sum(int(c) * pow(w, r * j, P) for j, c in enumerate(coeffs)) % P for r in range(n)]
        assert list(oracle.ntt(coeffs.astype(np.uint32), log_size)) == naive


def test_poseidon2_distinct_outputs(oracle):
    consts, _ = oracle.workload(2)
    p16, p24 = consts[148:296], consts[296:]
    rng = np.random.default_rng(3)
    for width, c in ((16, p16), (24, p24)):
        outs = set()
        for _ in range(50):
            s = rng.integers(0, P, width, dtype=np.uint64).astype(np.uint32)
            outs.add(tuple(oracle.poseidon2(width, c, s)))
        assert len(outs) == 50
        z = oracle.poseidon2(width, c, np.zeros(width, np.uint32))
        assert z.max() < P and z.any()


def test_whir_schedule_reference_defaults(oracle):
    cfg = oracle.whir_config(20)  # 2^12 rows x 2^8 packed columns
    num_rounds, final_vars = cfg[0], cfg[1]
    assert (num_rounds, final_vars) == (2, 5)
    rows = cfg[3:3 + 7 * (num_rounds + 1)].reshape(-1, 7)
    assert [r[0] for r in rows] == [20, 13, 9]          # variables per commitment
    assert [r[2] for r in rows] == [1, 3, 6]            # log inverse rates
    assert [r[4] for r in rows] == [112, 38, 19]        # queries
    assert [r[5] for r in rows] == [16, 14, 14]         # grinding bits


@pytest.mark.parametrize("log_n", [5, 7])
def test_oracle_prove_verify_roundtrip(oracle, log_n):
    consts, inputs = oracle.workload(log_n)
    wit = oracle.trace(log_n, consts, inputs)
    proof, _ = oracle.prove(log_n, consts, wit)
    assert oracle.verify(log_n, consts, proof) == 0
    # a corrupted transcript element is rejected
    for pos in (3, 200, proof.size // 2, proof.size - 5):
        bad = proof.copy()
        bad[pos] = (int(bad[pos]) + 1) % P
        assert oracle.verify(log_n, consts, bad) != 0
    assert oracle.verify(log_n, consts, proof[:-1]) != 0


def test_oracle_rejects_invalid_trace(oracle):
    log_n = 6
    consts, inputs = oracle.workload(log_n)
    wit = oracle.trace(log_n, consts, inputs)
    wit[(20 << log_n) + 7] ^= 1  # break one post-round state
    proof, _ = oracle.prove(log_n, consts, wit)
    assert oracle.verify(log_n, consts, proof) != 0


def test_abc_roundtrip(oracle):
    rng = np.random.default_rng(4)
    log_n, skips = 8, 3
    a = rng.integers(0, P, 1 << log_n, dtype=np.uint64)
    b = rng.integers(0, P, 1 << log_n, dtype=np.uint64)
    c = (a * b) % P
    a, b, c = (x.astype(np.uint32) for x in (a, b, c))
    consts, _ = oracle.workload(2)
    p16 = consts[148:296]
    proof = oracle.prove_abc(p16, log_n, skips, a, b, c)
    assert oracle.verify_abc(p16, log_n, skips, proof) == 0
    c2 = c.copy()
    c2[5] ^= 1
    bad = oracle.prove_abc(p16, log_n, skips, a, b, c2)
    assert oracle.verify_abc(p16, log_n, skips, bad) != 0
