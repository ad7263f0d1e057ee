"""The oracle against its committed fixtures (tests/golden/oracle_fixtures.json, written by
tests/golden/make_golden.py): StdRng words, Poseidon2 outputs, workload constants and the
digests of complete proofs stay fixed."""
import json
import os

from tests.golden.make_golden import build

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_oracle_matches_fixtures(oracle):
    with open(os.path.join(HERE, "oracle_fixtures.json")) as f:
        want = json.load(f)
    got = build(oracle)
    assert got == want
