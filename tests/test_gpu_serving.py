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


def _pool():
    """The device's default stream-ordered pool (where the prover's buffers are carved)."""
    from cuda.bindings import driver as drv
    assert drv.cuInit(0)[0] == drv.CUresult.CUDA_SUCCESS
    err, dev = drv.cuDeviceGet(0)
    assert err == drv.CUresult.CUDA_SUCCESS
    err, pool = drv.cuDeviceGetDefaultMemPool(dev)
    assert err == drv.CUresult.CUDA_SUCCESS
    return drv, pool


def _pool_used(drv, pool, attr):
    err, v = drv.cuMemPoolGetAttribute(pool, attr)
    assert err == drv.CUresult.CUDA_SUCCESS
    return int(v)


def _pool_reset_high(drv, pool):
    err, = drv.cuMemPoolSetAttribute(pool, drv.CUmemPool_attribute.CU_MEMPOOL_ATTR_USED_MEM_HIGH,
                                      drv.cuuint64_t(0))
    assert err == drv.CUresult.CUDA_SUCCESS


@pytest.mark.parametrize("kw", [dict(), dict(log_inv_rate=3), dict(univariate_skips=2), dict(rs_domain_initial_reduction=3)])
def test_footprint_bounds_measured_device_memory(wl, kw):
    """The admission estimate (wl_proof_footprint_bytes) bounds the device memory a proof
    really takes: the pool's high-water mark over one served proof, at several sizes and
    settings (the rate scales the first commitment, the skips the zerocheck tables)."""
    import torch
    drv, pool = _pool()
    A = drv.CUmemPool_attribute
    settings = wl.AirSettings(**kw)
    with wl.Server(0, workers=1) as srv:
        for n in (10, 14, 16):
            c, i = wl.generate_workload(n, 40 + n)
            torch.cuda.synchronize()
            base = _pool_used(drv, pool, A.CU_MEMPOOL_ATTR_USED_MEM_CURRENT)
            _pool_reset_high(drv, pool)
            srv.wait(srv.submit(c, i, n, settings), n, settings)
            high = _pool_used(drv, pool, A.CU_MEMPOOL_ATTR_USED_MEM_HIGH) - base
            est = wl.proof_footprint_bytes(n, settings)
            assert high <= est, (n, kw, high, est)
            if n == 16:
                assert high >= est // 3, (n, kw, high, est)  # the bound is not vacuous


def test_served_mix_device_memory_within_admitted(wl):
    """During a served mix the pool's high-water mark stays within the bytes the server
    admitted (its peak of summed footprints of running proofs)."""
    import torch
    drv, pool = _pool()
    A = drv.CUmemPool_attribute
    sizes = [14, 12, 15, 13, 14, 11, 15, 12, 13, 14]
    jobs = _jobs(wl, sizes, 900)
    with wl.Server(0, workers=4) as srv:
        torch.cuda.synchronize()
        base = _pool_used(drv, pool, A.CU_MEMPOOL_ATTR_USED_MEM_CURRENT)
        _pool_reset_high(drv, pool)
        tickets = [srv.submit(c, i, n) for c, i, n in jobs]
        for t, (_, _, n) in zip(tickets, jobs):
            srv.wait(t, n)
        high = _pool_used(drv, pool, A.CU_MEMPOOL_ATTR_USED_MEM_HIGH) - base
        stats = srv.stats()
    assert stats["peak_running"] >= 2
    assert high <= stats["peak_bytes_admitted"], (high, stats)
