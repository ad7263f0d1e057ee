"""Batched and served proving: every proof equals the plain single-proof GPU path bit for
bit, whether it ran alone or in a mix, and the oracle verifier accepts it."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _jobs(wl, sizes, seed0):
    jobs = []
    for k, n in enumerate(sizes):
        c, i = wl.generate_workload(n, seed0 + k)
        jobs.append((c, i, n))
    return jobs


def test_batch_matches_plain(oracle, wl, ctx):
    rng = np.random.default_rng(11)
    sizes = [int(x) for x in rng.integers(6, 12, 10)]
    jobs = _jobs(wl, sizes, 100)
    with wl.Server(0, workers=4) as srv:
        proofs = wl.batch_prove(srv, jobs)
    for (c, i, n), p in zip(jobs, proofs):
        w = wl.Witness.generate(ctx, c, i, n)
        alone = wl.AirTable(ctx, c, n).prove_witness(w)
        w.free()
        assert np.array_equal(p, alone)
    for (c, i, n), p in list(zip(jobs, proofs))[:3]:
        assert oracle.verify(n, c, p) == 0


def test_served_mix_equals_alone_and_budget_admission(wl, ctx):
    sizes = [10, 7, 12, 8, 11, 9, 10, 6]
    jobs = _jobs(wl, sizes, 500)
    # a budget that holds roughly two of the larger proofs at a time forces queueing
    budget = 2 * wl.proof_footprint_bytes(12) + wl.proof_footprint_bytes(11)
    with wl.Server(0, workers=6, hbm_budget_bytes=budget) as srv:
        tickets = [srv.submit(c, i, n) for c, i, n in jobs]
        results = [srv.wait(t, n) for t, (_, _, n) in zip(tickets, jobs)]
        stats = srv.stats()
    assert stats["peak_bytes_admitted"] <= budget
    assert stats["peak_running"] >= 2
    for (c, i, n), (p, times) in zip(jobs, results):
        w = wl.Witness.generate(ctx, c, i, n)
        alone = wl.AirTable(ctx, c, n).prove_witness(w)
        w.free()
        assert np.array_equal(p, alone)
        assert times["latency_ms"] >= times["run_ms"] > 0


def test_server_rejects_oversized_job(wl):
    c, i = wl.generate_workload(10, 1)
    with wl.Server(0, workers=1, hbm_budget_bytes=wl.proof_footprint_bytes(10) // 2) as srv:
        with pytest.raises(wl.ProverError) as e:
            srv.submit(c, i, 10)
        assert e.value.status == 6  # WL_E_BUDGET
